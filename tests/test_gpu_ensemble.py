"""Batched ensemble and EnKF analysis on the GPU (through the C ABI).

The batched step must equal the loop over members bit for bit (same kernel,
same per-tile arithmetic, only the launch grouping differs), every member
must match the CPU oracle run of its own configuration to 1e-9 after the
steps, and the analysis must match the numpy restatement of the
reference's EnKF update and the reference's own Kalman-shift known answer.
"""
import numpy as np
import pytest
import torch

import oracle_py
from enkf_oracle import enkf_analysis, kalman_shift_reference_case
from pairs import rel_max

from adamantine_b200.ensemble import EnKF, Ensemble
from adamantine_b200.workloads import ensemble_q1, initial_temperature

pytestmark = pytest.mark.gpu

STEP_TOL = 1e-9


def small_ensemble(n=5, method="rk_fourth_order"):
    configs, params = ensemble_q1(n_members=n, n_cells=(16, 16, 16), extent=(5e-3, 5e-3, 5e-3), min_layers=8,
                                  max_layers=16, powder_layers=3, method=method, name="test-ensemble")
    grids = [initial_temperature(c, f"test-ensemble-{k}") for k, c in enumerate(configs)]
    return configs, params, grids


def oracle_for(cfg):
    st = cfg.to_struct()
    o = oracle_py.Oracle(st, active=cfg.geometry.active_cells(), initial_state=cfg.geometry.initial_state())
    o._keep = st
    return o


def test_ragged_members_have_distinct_work():
    configs, params, grids = small_ensemble()
    e = Ensemble(configs)
    heights = {p[2] for p in params}
    assert len(heights) > 1
    assert e.n_work_items() > 0
    assert e.stride % 2 == 0


@pytest.mark.parametrize("method,cells_per_thread", [("rk_fourth_order", 1), ("rk_third_order", 1),
                                                     ("forward_euler", 1), ("rk_fourth_order", 2),
                                                     ("rk_fourth_order", 4)])
def test_batched_equals_looped_and_oracle(method, cells_per_thread):
    configs, params, grids = small_ensemble(method=method)
    e1 = Ensemble(configs)
    e2 = Ensemble(configs)
    e1.set_cells_per_thread(cells_per_thread)
    e2.set_cells_per_thread(cells_per_thread)
    assert e1.cells_per_thread() == cells_per_thread
    y1 = e1.from_grids(grids)
    y2 = y1.clone()
    dt = 1e-6
    t1 = t2 = 0.0
    for _ in range(6):
        t1 = e1.evolve_one_time_step(t1, dt, y1)
        t2 = e2.evolve_looped(t2, dt, y2)
    torch.cuda.synchronize()
    assert t1 == t2
    assert torch.equal(y1, y2)
    assert e1.device_error() == 0
    for k, cfg in enumerate(configs):
        o = oracle_for(cfg)
        yr = np.ascontiguousarray(grids[k], np.float64).reshape(-1).copy()
        tr = 0.0
        for _ in range(6):
            tr = o.evolve_one_time_step(tr, dt, yr)
        got = e1.to_grid(y1[k]).reshape(-1)
        act = o.node_active().astype(bool)
        assert rel_max(got[act], yr[act]) <= STEP_TOL, k
        # nodes of inactive cells are not degrees of freedom: unchanged
        assert np.array_equal(got[~act], np.asarray(grids[k]).reshape(-1)[~act])


def test_graph_steps_equal_single_steps():
    configs, params, grids = small_ensemble()
    e1 = Ensemble(configs)
    e2 = Ensemble(configs)
    y1 = e1.from_grids(grids)
    y2 = y1.clone()
    t1 = 0.0
    for _ in range(8):
        t1 = e1.evolve_one_time_step(t1, 1e-6, y1)
    t2 = e2.evolve_n_steps(0.0, 1e-6, 8, y2)
    torch.cuda.synchronize()
    assert t1 == t2
    assert torch.equal(y1, y2)


def test_parameter_updates_follow_the_member():
    configs, params, grids = small_ensemble(n=4)
    e = Ensemble(configs)
    # member 2: new absorptivity and conductivity scale
    from adamantine_b200.workloads import phase_change_material

    cfg2 = configs[2]
    cfg2.material = phase_change_material(k_scale=1.3)
    cfg2.sources[0].absorption_efficiency = 0.5
    e.update_material(2, cfg2)
    src = cfg2.sources[0]
    e.update_beam(2, 0, src.depth, 0.5, src.diameter, src.max_power)
    y = e.from_grids(grids)
    t = 0.0
    for _ in range(5):
        t = e.evolve_one_time_step(t, 1e-6, y)
    o = oracle_for(cfg2)
    yr = np.ascontiguousarray(grids[2], np.float64).reshape(-1).copy()
    tr = 0.0
    for _ in range(5):
        tr = o.evolve_one_time_step(tr, 1e-6, yr)
    act = o.node_active().astype(bool)
    assert rel_max(e.to_grid(y[2]).reshape(-1)[act], yr[act]) <= STEP_TOL


def test_enkf_reference_known_answer():
    states, idx, obs, pert, var, expected, tol = kalman_shift_reference_case()
    dev = torch.device("cuda")
    X = torch.tensor(states, dtype=torch.float64, device=dev)
    EnKF().analysis(X, 4, torch.tensor(idx, device=dev), torch.tensor(obs, device=dev),
                    torch.tensor(pert, device=dev), obs_var=torch.tensor(var, device=dev))
    shift = X.cpu().numpy() - states
    assert np.allclose(shift, expected, rtol=tol, atol=0.0)
    ref, _ = enkf_analysis(states, 4, idx, obs, pert, obs_var=var)
    assert rel_max(X.cpu().numpy(), ref) <= 1e-12


@pytest.mark.parametrize("dense_r", [False, True])
def test_enkf_matches_restatement(dense_r):
    rng = np.random.default_rng(7)
    N, n_state, stride, m, p = 32, 5000, 5004, 300, 2
    states = 300.0 + rng.normal(0, 20.0, (N, stride))
    params = np.stack([np.exp(rng.normal(0, 0.1, N)), 0.35 * np.exp(rng.normal(0, 0.1, N))], axis=1)
    idx = np.stack([rng.choice(n_state, m, replace=False) for _ in range(N)]).astype(np.int64)
    obs = 300.0 + rng.normal(0, 20.0, m)
    var = np.full(m, 25.0)
    cov = None
    if dense_r:
        B = rng.normal(0, 1.0, (m, m)) * 0.5
        cov = B @ B.T / m + np.diag(var)
    pert = rng.normal(0, 5.0, (N, m))
    mask = (rng.uniform(size=(N, n_state)) > 0.1).astype(np.uint8)
    ref, ref_p = enkf_analysis(states, n_state, idx, obs, pert, obs_var=None if dense_r else var, obs_cov=cov,
                               params=params, update_mask=mask)
    dev = torch.device("cuda")
    X = torch.tensor(states, device=dev)
    P = torch.tensor(params, device=dev)
    EnKF().analysis(X, n_state, torch.tensor(idx, device=dev), torch.tensor(obs, device=dev),
                    torch.tensor(pert, device=dev), obs_var=None if dense_r else torch.tensor(var, device=dev),
                    obs_cov=None if cov is None else torch.tensor(cov, device=dev), params=P,
                    update_mask=torch.tensor(mask, device=dev))
    got = X.cpu().numpy()
    # the update is small next to the state: compare the shifts
    assert rel_max(got - states, ref - states) <= 1e-9
    assert rel_max(P.cpu().numpy() - params, ref_p - params) <= 1e-9
    assert np.array_equal(got[:, n_state:], states[:, n_state:])
    assert np.array_equal(got[:, :n_state][mask == 0], states[:, :n_state][mask == 0])


def test_enkf_rejects_indefinite_covariance():
    from adamantine_b200._lib import AdmError

    states, idx, obs, pert, var, expected, tol = kalman_shift_reference_case()
    dev = torch.device("cuda")
    X = torch.tensor(states, dtype=torch.float64, device=dev)
    with pytest.raises(AdmError) as ex:
        EnKF().analysis(X, 4, torch.tensor(idx, device=dev), torch.tensor(obs, device=dev),
                        torch.tensor(pert, device=dev), obs_var=torch.tensor(-var * 1e6, device=dev))
    assert ex.value.code == 4
    bad = torch.tensor(idx, device=dev)
    bad[1, 0] = 99
    with pytest.raises(AdmError) as ex:
        EnKF().analysis(X, 4, bad, torch.tensor(obs, device=dev), torch.tensor(pert, device=dev),
                        obs_var=torch.tensor(var, device=dev))
    assert ex.value.code == 1


def test_sharded_steps_equal_fused_analysis():
    """The device building blocks of the sharded analysis, composed on one
    rank, give the fused analysis."""
    from adamantine_b200.sharded import LibrarySteps, ShardedAnalysis

    rng = np.random.default_rng(5)
    N, n_state, stride, m, p = 16, 4000, 4004, 250, 2
    states = 300.0 + rng.normal(0, 20.0, (N, stride))
    params = np.stack([np.exp(rng.normal(0, 0.1, N)), 0.35 * np.exp(rng.normal(0, 0.1, N))], axis=1)
    idx = np.stack([rng.choice(n_state, m, replace=False) for _ in range(N)]).astype(np.int64)
    obs = 300.0 + rng.normal(0, 20.0, m)
    var = np.full(m, 25.0)
    pert = rng.normal(0, 5.0, (N, m))
    dev = torch.device("cuda")
    args = dict(obs_var=torch.tensor(var, device=dev))
    X1, P1 = torch.tensor(states, device=dev), torch.tensor(params, device=dev)
    X2, P2 = X1.clone(), P1.clone()
    enkf = EnKF()
    enkf.analysis(X1, n_state, torch.tensor(idx, device=dev), torch.tensor(obs, device=dev),
                  torch.tensor(pert, device=dev), params=P1, **args)
    ShardedAnalysis(LibrarySteps(enkf))(X2, n_state, torch.tensor(idx, device=dev), torch.tensor(obs, device=dev),
                                        torch.tensor(pert, device=dev), params=P2, **args)
    assert rel_max((X2 - torch.tensor(states, device=dev)).cpu().numpy(),
                   (X1 - torch.tensor(states, device=dev)).cpu().numpy()) <= 1e-11
    assert rel_max(P2.cpu().numpy() - params, P1.cpu().numpy() - params) <= 1e-11
    ref, ref_p = enkf_analysis(states, n_state, idx, obs, pert, obs_var=var, params=params)
    assert rel_max(X2.cpu().numpy() - states, ref - states) <= 1e-9
