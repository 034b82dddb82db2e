"""numpy FP64 restatement of the reference's EnKF analysis -- test
infrastructure only (the checker of the GPU analysis), never part of the
product path.

DataAssimilator::update_ensemble (source/DataAssimilator.cc:95-189): for
every member k the perturbed innovation d_k = y + e_k - H_k x_k
(fill_noise_vector :630-670 gives e_k, calc_Hx :614-628 gives H x), the
Kalman gain K = P H^T (H P H^T + R)^-1 with P the sample covariance of the
augmented states about their mean divided by N - 1
(calc_sample_covariance_sparse :690-752; enkf_analysis keeps every pair,
enkf_analysis_localized applies the cutoff sphere and function), applied as x_k += K d_k (apply_kalman_gain :403-476, which solves
with GMRES; this restatement uses a dense solve). H may differ per member
(obs_index[k]); the reference requires one map for all members.
"""
from __future__ import annotations

import numpy as np

LOC_NONE, LOC_STEP, LOC_GASPARI_COHN = 0, 1, 2


def gaspari_cohn(r):
    """DataAssimilator::gaspari_cohn_function (source/DataAssimilator.cc:672-688):
    the fifth-order compactly supported correlation of Gaspari and Cohn (1999,
    eq. 4.10), support [0, 2)."""
    r = np.asarray(r, np.float64)
    out = np.zeros_like(r)
    a = r < 1.0
    ra = r[a]
    out[a] = 1.0 - 5.0 / 3.0 * ra ** 2 + 5.0 / 8.0 * ra ** 3 + 0.5 * ra ** 4 - 0.25 * ra ** 5
    b = (r >= 1.0) & (r < 2.0)
    rb = r[b]
    out[b] = (4.0 - 5.0 * rb + 5.0 / 3.0 * rb ** 2 + 5.0 / 8.0 * rb ** 3 - 0.5 * rb ** 4 + rb ** 5 / 12.0
              - 2.0 / (3.0 * rb))
    return out


def localization_weights(dist, cutoff, function):
    """Scaling of a covariance entry between two state entries at distance
    dist. The sparsity pattern (update_covariance_sparsity_pattern,
    :512-611) keeps the pairs whose support points lie within the cutoff
    sphere (distance <= cutoff); entries outside it are zero whatever the
    function. Inside, calc_sample_covariance_sparse (:729-747) scales by
    gaspari_cohn(2 dist / cutoff), by the step function (0 beyond the
    cutoff, so 1 inside), or by 1 ("none")."""
    dist = np.asarray(dist, np.float64)
    w = (dist <= cutoff).astype(np.float64)
    if function == LOC_GASPARI_COHN:
        w = w * gaspari_cohn(2.0 * dist / cutoff)
    return w


def pattern_nonzeros(points, cutoff, n_params=0):
    """n_nonzero_elements of the covariance sparsity pattern: state pairs
    within the cutoff, plus full rows and columns for the parameters."""
    p = np.asarray(points, np.float64)
    d = np.linalg.norm(p[:, None, :] - p[None, :, :], axis=-1)
    n = len(p)
    return int((d <= cutoff).sum()) + 2 * n_params * n + n_params * n_params


def localized_covariance(aug, points, n_sim, cutoff, function):
    """calc_sample_covariance_sparse (:690-752) as a dense matrix: the sample
    covariance of the augmented members (rows of aug, (N, n_sim + p)) about
    their mean, divided by N - 1, state-state entries scaled by
    localization_weights, parameter rows and columns unscaled."""
    aug = np.asarray(aug, np.float64)
    N = aug.shape[0]
    A = aug - aug.mean(axis=0)
    P = A.T @ A / (N - 1.0)
    p = np.asarray(points, np.float64)
    d = np.linalg.norm(p[:, None, :] - p[None, :, :], axis=-1)
    P[:n_sim, :n_sim] *= localization_weights(d, cutoff, function)
    return P


def enkf_analysis_localized(states, n_state, node_xyz, obs_index, obs, perturbations, cutoff, function,
                            obs_var=None, obs_cov=None, params=None, update_mask=None):
    """update_ensemble with localization: the gain K = P H^T (H P H^T + R)^-1
    of the localized P (one observation map for all members, as the
    reference requires); node_xyz (n_state, 3) are the support points of the
    state entries. P H^T and H P H^T are formed directly (the columns of the
    localized P at the observed entries), so n_state x n_obs memory."""
    X = np.asarray(states, np.float64)[:, :n_state]
    N = X.shape[0]
    idx = np.asarray(obs_index)[0]
    P_ = np.zeros((N, 0)) if params is None else np.asarray(params, np.float64)
    aug = np.concatenate([X, P_], axis=1)
    A = aug - aug.mean(axis=0)
    HA = A[:, idx]  # (N, m)
    pts = np.asarray(node_xyz, np.float64)
    opts = pts[idx]
    d_so = np.linalg.norm(pts[:, None, :] - opts[None, :, :], axis=-1)  # (n_state, m)
    d_oo = np.linalg.norm(opts[:, None, :] - opts[None, :, :], axis=-1)
    PHt = A.T @ HA / (N - 1.0)  # (n + p, m)
    PHt[:n_state] *= localization_weights(d_so, cutoff, function)
    HPHt = (HA.T @ HA / (N - 1.0)) * localization_weights(d_oo, cutoff, function)
    R = np.diag(obs_var) if obs_cov is None else np.asarray(obs_cov, np.float64)
    D = obs[None, :] + perturbations - X[:, idx]  # (N, m)
    shift = PHt @ np.linalg.solve(HPHt + R, D.T)  # (n + p, N)
    out = np.array(states, np.float64, copy=True)
    upd = shift[:n_state].T
    if update_mask is not None:
        upd = upd * (np.asarray(update_mask) != 0)
    out[:, :n_state] += upd
    out_p = None
    if params is not None:
        out_p = P_ + shift[n_state:].T
    return out, out_p


def enkf_analysis(states, n_state, obs_index, obs, perturbations, obs_var=None, obs_cov=None, params=None,
                  update_mask=None):
    """states (N, stride), params (N, p) or None, obs_index (N, m),
    obs (m,), perturbations (N, m); returns updated copies."""
    X = np.asarray(states, np.float64)[:, :n_state]
    N = X.shape[0]
    P_ = np.zeros((N, 0)) if params is None else np.asarray(params, np.float64)
    aug = np.concatenate([X, P_], axis=1)  # (N, n + p)
    mean = aug.mean(axis=0)
    A = aug - mean  # anomalies, (N, n + p)
    HX = np.stack([X[k, obs_index[k]] for k in range(N)])  # (N, m)
    HA = HX - HX.mean(axis=0)
    R = np.diag(obs_var) if obs_cov is None else np.asarray(obs_cov, np.float64)
    C = HA.T @ HA / (N - 1.0) + R
    D = obs[None, :] + perturbations - HX  # (N, m)
    Z = np.linalg.solve(C, D.T)  # (m, N)
    # P H^T Z = A^T HA Z / (N - 1)
    shift = (A.T @ (HA @ Z)) / (N - 1.0)  # (n + p, N)
    out = np.array(states, np.float64, copy=True)
    upd = shift[:n_state].T
    if update_mask is not None:
        upd = upd * (np.asarray(update_mask) != 0)
    out[:, :n_state] += upd
    out_p = None
    if params is not None:
        out_p = P_ + shift[n_state:].T
    return out, out_p


def kalman_shift_reference_case():
    """The known answer of the reference's apply_kalman_gain test
    (tests/test_data_assimilator.cc:46-168): 3 members of 4 state entries,
    2 observations of entries 1 and 3, R = diag(0.002, 0.001), fixed
    perturbations. Returns (states, obs_index, obs, perturbations, obs_var,
    expected shift (3, 4), tolerance)."""
    states = np.array([[1.0, 3.0, 6.0, 9.0], [1.5, 3.2, 6.3, 9.7], [1.1, 3.1, 6.1, 9.1]])
    obs_index = np.array([[1, 3]] * 3, np.int64)
    obs = np.array([2.5, 9.5])
    pert = np.array([[0.0008, -0.0005], [-0.001, 0.0002], [0.0002, -0.0009]])
    var = np.array([0.002, 0.001])
    expected = np.array([[0.21352564, -0.14600986, -0.02616469, 0.45321598],
                         [-0.27786325, -0.32946285, -0.31226298, -0.24346351],
                         [0.12767094, -0.20319395, -0.09290565, 0.34824753]])
    return states, obs_index, obs, pert, var, expected, 1e-4
