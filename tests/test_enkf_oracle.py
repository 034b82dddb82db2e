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


# ---------------------------------------------------------------- localization
def _unit_square_q1(divisions):
    """Support points of FE_Q(1) on the unit square split into
    divisions x divisions cells (the meshes of the reference's tests)."""
    t = np.linspace(0.0, 1.0, divisions + 1)
    return np.array([(x, y) for y in t for x in t])


def test_sparsity_pattern_counts_match_reference():
    """test_update_covariance_sparsity_pattern
    (tests/test_data_assimilator.cc:318-365): 2 x 2 cells, 9 support points."""
    from enkf_oracle import pattern_nonzeros
    pts = _unit_square_q1(2)
    assert pattern_nonzeros(pts, 100.0) == 81
    assert pattern_nonzeros(pts, 1.0e-6) == 9
    assert pattern_nonzeros(pts, 1.2) == 77  # opposite corners cut
    assert pattern_nonzeros(pts, 1.0e-6, n_params=2) == 49


def test_localized_covariance_matches_reference():
    """test_calc_sample_covariance_sparse
    (tests/test_data_assimilator.cc:367-572), tolerance 1e-10 there."""
    from enkf_oracle import LOC_GASPARI_COHN, LOC_STEP, localized_covariance
    pts = _unit_square_q1(1)
    v0 = np.array([2.0, 4.0, 5.0, 7.0])
    v1 = np.array([2.1, 4.3, 5.2, 7.4])
    tol = 1e-10
    assert np.allclose(localized_covariance(np.stack([v0, v0]), pts, 4, 100.0, LOC_STEP), 0.0, atol=tol)
    full = np.array([[0.005, 0.015, 0.01, 0.02], [0.015, 0.045, 0.03, 0.06], [0.01, 0.03, 0.02, 0.04],
                     [0.02, 0.06, 0.04, 0.08]])
    assert np.allclose(localized_covariance(np.stack([v0, v1]), pts, 4, 100.0, LOC_STEP), full, atol=tol)
    diag = localized_covariance(np.stack([v0, v1]), pts, 4, 1.0e-6, LOC_STEP)
    assert np.allclose(diag, np.diag(np.diag(full)), atol=tol)
    gc = localized_covariance(np.stack([v0, v1]), pts, 4, 3.0, LOC_GASPARI_COHN)
    off = ~np.eye(4, dtype=bool)
    assert np.allclose(np.diag(gc), np.diag(full), atol=tol)
    assert (gc[off] > 0.0).all() and (gc[off] < full[off]).all()
    # two augmented parameters: state-state entries localized, parameter
    # rows and columns kept
    a0 = np.concatenate([v0, [1.0, 1.5]])
    a1 = np.concatenate([v1, [1.1, 1.4]])
    P = localized_covariance(np.stack([a0, a1]), pts, 4, 1.0e-6, LOC_STEP)
    assert np.allclose(P[:4, :4], np.diag(np.diag(full)), atol=tol)
    assert np.allclose(P[4], [0.005, 0.015, 0.01, 0.02, 0.005, -0.005], atol=tol)
    assert np.allclose(P[5], [-0.005, -0.015, -0.01, -0.02, -0.005, 0.005], atol=tol)


def test_gaspari_cohn_is_the_published_function():
    """Gaspari and Cohn (1999) eq. 4.10: 1 at 0, continuous at 1, 0 from 2."""
    from enkf_oracle import gaspari_cohn
    r = np.array([0.0, 1.0 - 1e-12, 1.0, 2.0 - 1e-9, 2.0, 3.0])
    g = gaspari_cohn(r)
    assert g[0] == 1.0 and abs(g[1] - g[2]) < 1e-10 and abs(g[2] - 5.0 / 24.0) < 1e-12
    assert abs(g[3]) < 1e-8 and g[4] == 0.0 and g[5] == 0.0
    x = np.linspace(0.0, 2.0, 201)
    assert (np.diff(gaspari_cohn(x)) <= 1e-15).all()


def test_localized_analysis_with_infinite_cutoff_is_the_plain_analysis():
    from enkf_oracle import LOC_NONE, enkf_analysis_localized
    rng = np.random.default_rng(5)
    N, n, m = 5, 12, 4
    X = rng.normal(size=(N, n))
    pts = rng.uniform(size=(n, 3))
    idx = np.tile(rng.choice(n, m, replace=False), (N, 1))
    obs = rng.normal(size=m)
    pert = rng.normal(size=(N, m)) * 0.1
    var = np.full(m, 0.2)
    want, _ = enkf_analysis(X, n, idx, obs, pert, obs_var=var)
    got, _ = enkf_analysis_localized(X, n, pts, idx, obs, pert, 1e300, LOC_NONE, obs_var=var)
    assert np.allclose(got, want, rtol=1e-12, atol=1e-12)


def test_localized_analysis_is_the_gain_of_the_localized_covariance():
    """The analysis with P H^T formed directly equals K = P H^T (H P H^T +
    R)^-1 with the dense localized P of calc_sample_covariance_sparse."""
    from enkf_oracle import LOC_GASPARI_COHN, LOC_STEP, enkf_analysis_localized, localized_covariance
    rng = np.random.default_rng(8)
    N, n, m, p = 6, 30, 7, 2
    X = rng.normal(size=(N, n))
    prm = rng.normal(size=(N, p))
    pts = rng.uniform(size=(n, 3))
    idx = np.tile(rng.choice(n, m, replace=False), (N, 1))
    obs = rng.normal(size=m)
    pert = rng.normal(size=(N, m)) * 0.1
    var = np.full(m, 0.2)
    for fn, cut in ((LOC_GASPARI_COHN, 0.6), (LOC_STEP, 0.4)):
        got, got_p = enkf_analysis_localized(X, n, pts, idx, obs, pert, cut, fn, obs_var=var, params=prm)
        P = localized_covariance(np.concatenate([X, prm], axis=1), pts, n, cut, fn)
        H = np.zeros((m, n + p))
        H[np.arange(m), idx[0]] = 1.0
        K = P @ H.T @ np.linalg.inv(H @ P @ H.T + np.diag(var))
        shift = K @ (obs[:, None] + pert.T - X[:, idx[0]].T)
        assert np.allclose(got, X + shift[:n].T, rtol=1e-12, atol=1e-12)
        assert np.allclose(got_p, prm + shift[n:].T, rtol=1e-12, atol=1e-12)
