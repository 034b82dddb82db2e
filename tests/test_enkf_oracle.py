"""CPU checks of the EnKF restatement and of the ensemble workload builder."""
import numpy as np

from enkf_oracle import enkf_analysis, kalman_shift_reference_case

from adamantine_b200.workloads import ensemble_q1, surface_observations


def test_restatement_reproduces_reference_kalman_shift():
    """tests/test_data_assimilator.cc:46-168 of the reference (tolerance 1e-4
    there; the dense restatement agrees to 1e-8)."""
    states, idx, obs, pert, var, expected, tol = kalman_shift_reference_case()
    out, _ = enkf_analysis(states, 4, idx, obs, pert, obs_var=var)
    assert np.allclose(out - states, expected, rtol=1e-7, atol=1e-8)


def test_restatement_is_the_kalman_gain_formula():
    rng = np.random.default_rng(3)
    N, n, m = 6, 9, 4
    X = rng.normal(size=(N, n))
    idx = np.stack([rng.choice(n, m, replace=False) for _ in range(N)])
    obs = rng.normal(size=m)
    pert = rng.normal(size=(N, m)) * 0.1
    var = np.full(m, 0.3)
    out, _ = enkf_analysis(X, n, idx, obs, pert, obs_var=var)
    # same member map for all: the textbook P H^T (H P H^T + R)^-1 form
    idx_same = np.tile(idx[0], (N, 1))
    out2, _ = enkf_analysis(X, n, idx_same, obs, pert, obs_var=var)
    A = X - X.mean(0)
    P = A.T @ A / (N - 1)
    H = np.zeros((m, n))
    H[np.arange(m), idx[0]] = 1.0
    K = P @ H.T @ np.linalg.inv(H @ P @ H.T + np.diag(var))
    want = X + (K @ (obs[:, None] + pert.T - H @ X.T)).T
    assert np.allclose(out2, want, rtol=1e-12, atol=1e-12)
    assert not np.allclose(out, out2)


def test_ensemble_workload_is_seeded_and_ragged():
    c1, p1 = ensemble_q1()
    c2, p2 = ensemble_q1()
    assert p1 == p2 and len(p1) == 32
    layers = [p[2] for p in p1]
    assert min(layers) >= 20 and max(layers) <= 32 and len(set(layers)) > 3
    k = [p[0] for p in p1]
    assert 0.7 < min(k) and max(k) < 1.4
    for cfg, p in zip(c1, p1):
        act = cfg.geometry.active_cells().reshape(32, 64, 64)
        assert act[: p[2]].all() and not act[p[2]:].any()
        st = cfg.geometry.initial_state().reshape(32, 64, 64)
        assert (st[p[2] - 4: p[2]] == 2).all() and (st[: p[2] - 4] == 0).all()
        assert cfg.sources[0].segments[0, 4] == p[2] * 10e-3 / 32
    ij, sigma = surface_observations((65, 65), layers)
    assert ij.shape == (2000, 2) and len({tuple(r) for r in ij}) == 2000 and sigma == 5.0
