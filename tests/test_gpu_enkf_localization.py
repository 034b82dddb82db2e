"""Localized EnKF analysis on the GPU (through the C ABI) against the numpy
restatement of the reference's localized covariance
(calc_sample_covariance_sparse, source/DataAssimilator.cc:690-752, whose own
known answers pin the restatement on CPU)."""
import numpy as np
import pytest
import torch

from enkf_oracle import LOC_GASPARI_COHN, LOC_NONE, LOC_STEP, enkf_analysis, enkf_analysis_localized
from pairs import rel_max

from adamantine_b200.ensemble import EnKF

pytestmark = pytest.mark.gpu

# the update is a sum of O(n_obs) FP64 products in a different order than
# numpy's: relative to the size of the update
TOL = 1e-10


def grid_problem(nodes=(21, 13, 9), pitch=24, N=12, m=60, seed=21, n_params=2):
    rng = np.random.default_rng(seed)
    origin = np.array([1e-3, -2e-3, 0.0])
    spacing = np.array([0.25e-3, 0.3e-3, 0.2e-3])
    n_state = pitch * nodes[1] * nodes[2]
    a, b, c = np.meshgrid(np.arange(pitch), np.arange(nodes[1]), np.arange(nodes[2]), indexing="ij")
    idx_all = (a + pitch * (b + nodes[1] * c)).reshape(-1)
    pts = np.zeros((n_state, 3))
    pts[idx_all] = origin + np.stack([a.reshape(-1), b.reshape(-1), c.reshape(-1)], axis=1) * spacing
    real = (np.arange(n_state) % pitch) < nodes[0]
    states = 300.0 + rng.normal(0, 20.0, (N, n_state))
    states[:, ~real] = 0.0  # row padding
    params = np.stack([np.exp(rng.normal(0, 0.1, N)), 0.35 * np.exp(rng.normal(0, 0.1, N))], axis=1)[:, :n_params]
    obs_nodes = rng.choice(np.flatnonzero(real), m, replace=False).astype(np.int64)
    idx = np.tile(obs_nodes, (N, 1))
    obs = 300.0 + rng.normal(0, 20.0, m)
    var = np.full(m, 25.0)
    pert = rng.normal(0, 5.0, (N, m))
    grid = (tuple(origin), tuple(spacing), nodes, pitch)
    return states, params, idx, obs, var, pert, n_state, pts, grid, real


def run_gpu(enkf, states, params, idx, obs, var, pert, n_state, mask=None):
    dev = torch.device("cuda")
    X = torch.tensor(states, device=dev)
    P = torch.tensor(params, device=dev) if params.shape[1] else None
    enkf.analysis(X, n_state, torch.tensor(idx, device=dev), torch.tensor(obs, device=dev),
                  torch.tensor(pert, device=dev), obs_var=torch.tensor(var, device=dev), params=P,
                  update_mask=None if mask is None else torch.tensor(mask, device=dev))
    return X.cpu().numpy(), (P.cpu().numpy() if P is not None else None)


# Cutoffs of the step function are kept away from node distances: a pair at
# exactly the cutoff is in or out of the pattern by the last bit of its
# coordinates (the GPU forms them with fused multiply-adds), and the step
# makes that visible. Gaspari-Cohn is continuous (0 at the cutoff).
@pytest.mark.parametrize("function,cutoff", [(LOC_GASPARI_COHN, 1.5e-3), (LOC_STEP, 0.9137e-3),
                                             (LOC_NONE, 0.6137e-3), (LOC_GASPARI_COHN, 20e-3)])
def test_localized_analysis_matches_restatement(function, cutoff):
    states, params, idx, obs, var, pert, n_state, pts, grid, real = grid_problem()
    enkf = EnKF()
    enkf.set_localization(function, cutoff, pts[idx[0]], grid)
    X, P = run_gpu(enkf, states, params, idx, obs, var, pert, n_state)
    ref, ref_p = enkf_analysis_localized(states, n_state, pts, idx, obs, pert, cutoff, function, obs_var=var,
                                         params=params)
    # padding entries are not support points: unchanged on the GPU
    assert (X[:, ~real] == states[:, ~real]).all()
    assert rel_max(X[:, real] - states[:, real], ref[:, real] - states[:, real]) <= TOL
    assert rel_max(P - params, ref_p - params) <= TOL
    plain, _ = enkf_analysis(states, n_state, idx, obs, pert, obs_var=var, params=params)
    assert rel_max(X[:, real] - states[:, real], plain[:, real] - states[:, real]) > 1e-3


@pytest.mark.parametrize("m", [60, 300])
def test_indefinite_step_localization_is_solved_by_lu(m):
    """A step-function Schur product is not a correlation: here H P H^T + R
    has negative eigenvalues (checked), the Cholesky stops, and the pivoted
    LU (one panel for 60 observations, five for 300) solves it."""
    states, params, idx, obs, var, pert, n_state, pts, grid, real = grid_problem(m=m, seed=4)
    cutoff = 1.2137e-3
    opts = pts[idx[0]]
    HX = states[:, idx[0]]
    HA = HX - HX.mean(0)
    from enkf_oracle import localization_weights
    rho = localization_weights(np.linalg.norm(opts[:, None] - opts[None], axis=-1), cutoff, LOC_STEP)
    C = (HA.T @ HA / (len(states) - 1.0)) * rho + np.diag(var)
    assert np.linalg.eigvalsh(C).min() < 0.0 and np.linalg.cond(C) < 1e4
    enkf = EnKF()
    enkf.set_localization("step_function", cutoff, opts, grid)
    X, P = run_gpu(enkf, states, params, idx, obs, var, pert, n_state)
    ref, ref_p = enkf_analysis_localized(states, n_state, pts, idx, obs, pert, cutoff, LOC_STEP, obs_var=var,
                                         params=params)
    assert rel_max(X[:, real] - states[:, real], ref[:, real] - states[:, real]) <= TOL
    assert rel_max(P - params, ref_p - params) <= TOL


def test_cutoff_covering_every_pair_is_the_plain_analysis():
    states, params, idx, obs, var, pert, n_state, pts, grid, real = grid_problem(seed=3)
    plain = EnKF()
    Xp, Pp = run_gpu(plain, states, params, idx, obs, var, pert, n_state)
    for fn in (LOC_STEP, LOC_NONE):
        enkf = EnKF()
        enkf.set_localization(fn, 1.0, pts[idx[0]], grid)  # 1 m: every pair
        X, P = run_gpu(enkf, states, params, idx, obs, var, pert, n_state)
        assert (X == Xp).all() and (P == Pp).all()
    # removing the localization restores the plain analysis too
    enkf = EnKF()
    enkf.set_localization("gaspari_cohn", 1e-3, pts[idx[0]], grid)
    enkf.set_localization(None, 0.0, None, None)
    X, _ = run_gpu(enkf, states, params, idx, obs, var, pert, n_state)
    assert (X == Xp).all()


def test_many_buckets_mask_and_no_params():
    """A small cutoff over a larger grid (many observation buckets, most
    nodes far from every observation) with an update mask and without
    augmented parameters."""
    states, params, idx, obs, var, pert, n_state, pts, grid, real = grid_problem(
        nodes=(70, 41, 12), pitch=72, N=20, m=400, seed=9, n_params=0)
    rng = np.random.default_rng(2)
    mask = (rng.uniform(size=states.shape) > 0.1).astype(np.uint8)
    cutoff = 0.8137e-3
    enkf = EnKF()
    enkf.set_localization("step_function", cutoff, pts[idx[0]], grid)
    X, _ = run_gpu(enkf, states, params, idx, obs, var, pert, n_state, mask=mask)
    ref, _ = enkf_analysis_localized(states, n_state, pts, idx, obs, pert, cutoff, LOC_STEP, obs_var=var,
                                     update_mask=mask)
    assert rel_max(X[:, real] - states[:, real], ref[:, real] - states[:, real]) <= TOL
    d_min = np.min(np.linalg.norm(pts[:, None, :] - pts[idx[0]][None, :, :], axis=-1), axis=1)
    far = real & (d_min > cutoff)
    assert far.any() and (X[:, far] == states[:, far]).all()


def test_localized_sharded_steps_equal_fused_analysis():
    """The localized partial update of two member blocks (as two ranks would
    form them) summed and applied gives the fused localized analysis."""
    from adamantine_b200.sharded import LibrarySteps

    states, params, idx, obs, var, pert, n_state, pts, grid, real = grid_problem(N=16, seed=31)
    dev = torch.device("cuda")
    cutoff = 1.2e-3
    fused = EnKF()
    fused.set_localization("gaspari_cohn", cutoff, pts[idx[0]], grid)
    Xf, Pf = run_gpu(fused, states, params, idx, obs, var, pert, n_state)

    enkf = EnKF()
    enkf.set_localization("gaspari_cohn", cutoff, pts[idx[0]], grid)
    steps = LibrarySteps(enkf)
    X = torch.tensor(states, device=dev)
    P = torch.tensor(params, device=dev)
    hx = steps.observe(X, n_state, torch.tensor(idx, device=dev))
    w = steps.gain(hx, torch.tensor(obs, device=dev), torch.tensor(pert, device=dev),
                   obs_var=torch.tensor(var, device=dev))
    total = steps.local_sum(X, n_state, P)
    half = 8
    u = sum(steps.partial_update(X[r * half:(r + 1) * half], n_state, P[r * half:(r + 1) * half], total,
                                 w[r * half:(r + 1) * half], first=r * half) for r in range(2))
    steps.apply(X, n_state, P, u.contiguous())
    Xs, Ps = X.cpu().numpy(), P.cpu().numpy()
    assert rel_max(Xs[:, real] - states[:, real], Xf[:, real] - states[:, real]) <= 1e-11
    assert rel_max(Ps - params, Pf - params) <= 1e-11


def test_localization_rejects_bad_arguments():
    from adamantine_b200._lib import AdmError

    states, params, idx, obs, var, pert, n_state, pts, grid, real = grid_problem()
    enkf = EnKF()
    with pytest.raises(AdmError):
        enkf.set_localization("gaspari_cohn", 0.0, pts[idx[0]], grid)
    with pytest.raises(AdmError):
        enkf.set_localization(7, 1e-3, pts[idx[0]], grid)
    origin, spacing, nodes, pitch = grid
    with pytest.raises(AdmError):
        enkf.set_localization("step_function", 1e-3, pts[idx[0]], (origin, spacing, nodes, nodes[0] - 1))
    enkf.set_localization("step_function", 1e-3, pts[idx[0]][:10], grid)
    with pytest.raises(AdmError):  # 60 observations against a localization of 10
        run_gpu(enkf, states, params, idx, obs, var, pert, n_state)


def test_gain_of_many_members_through_the_blocked_solve():
    """The gain of 100 members (more than one 64-column chunk of the blocked
    triangular solves) with a full observation covariance (the m x m
    Cholesky path; m = 150, a partial last block) against the numpy gain."""
    from adamantine_b200.sharded import LibrarySteps

    from sharded_steps import NumpySteps

    rng = np.random.default_rng(41)
    N, m = 100, 150
    hx = 300.0 + rng.normal(0.0, 20.0, (N, m))
    obs = 300.0 + rng.normal(0.0, 20.0, m)
    pert = rng.normal(0.0, 5.0, (N, m))
    a = rng.normal(size=(m, m))
    cov = a @ a.T / m + 25.0 * np.eye(m)
    dev = torch.device("cuda")
    w = LibrarySteps(EnKF()).gain(torch.tensor(hx, device=dev), torch.tensor(obs, device=dev),
                                  torch.tensor(pert, device=dev), obs_cov=torch.tensor(cov, device=dev))
    ref = NumpySteps().gain(torch.tensor(hx), torch.tensor(obs), torch.tensor(pert), obs_cov=torch.tensor(cov))
    assert rel_max(w.cpu().numpy(), ref.numpy()) <= 1e-10
