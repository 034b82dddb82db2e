"""numpy FP64 restatement of the reference's EnKF analysis -- test
infrastructure only (the checker of the GPU analysis), never part of the
product path.

DataAssimilator::update_ensemble (source/DataAssimilator.cc:95-189): for
every member k the perturbed innovation d_k = y + e_k - H_k x_k
(fill_noise_vector :630-670 gives e_k, calc_Hx :614-628 gives H x), the
Kalman gain K = P H^T (H P H^T + R)^-1 with P the sample covariance of the
augmented states about their mean divided by N - 1
(calc_sample_covariance_sparse :690-752, localization "none": every pair
kept), applied as x_k += K d_k (apply_kalman_gain :403-476, which solves
with GMRES; this restatement uses a dense solve). H may differ per member
(obs_index[k]); the reference requires one map for all members.
"""
from __future__ import annotations

import numpy as np


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
