"""Parity of the CUDA path with the CPU oracle on the benchmark
configurations at their stated sizes (through the C ABI).

- 32x32x16 Q1 solid with a convective top: 200 forward-Euler steps of 1e-6,
  every step's vmult <= 1e-12 and the final field <= 1e-9, in all three
  launch schedules.
- 128x128x64 Q2 solid/liquid/powder (8,520,321 DoFs): one vmult <= 1e-12 and
  the per-point powder history, then 20 RK4 steps <= 1e-9, in all three
  launch schedules.
- The 32-member 64x64x32 Q1 ensemble with ragged deposited heights: 100 RK4
  steps of the batched launch, every member <= 1e-9 against its own oracle
  run.
- The 64x64x32 Q2 adjoint workload (200 RK2 steps): the oracle forward's
  misfit equals the GPU's to 1e-9 and the oracle's central difference of
  one gradient component agrees with the adjoint gradient to 1e-6.

Semantics: source/ThermalOperator.templates.hh:176-225 (vmult) and
source/ThermalPhysics.templates.hh:854-888 (evolve_one_time_step) of the
reference.
"""
import numpy as np
import pytest
import torch

import oracle_py
import oracle_runs
from pairs import rel_max

from adamantine_b200.thermal import ThermalPhysics
from adamantine_b200.workloads import (adjoint_q2, ensemble_q1, initial_temperature, interior_points,
                                       phase_change_q2, solid_q1_small)

pytestmark = pytest.mark.gpu

VMULT_TOL = 1e-12
STEP_TOL = 1e-9
FD_TOL = 1e-6
COLOURED, ATOMIC, TWO_PASS = 0, 1, 2


def oracle_for(cfg):
    st = cfg.to_struct()
    o = oracle_py.Oracle(st, active=cfg.geometry.active_cells(), initial_state=cfg.geometry.initial_state())
    o._keep = st
    return o


def flat(v):
    return np.asarray(v).reshape(-1)


@pytest.fixture(scope="module")
def solid_q1_reference():
    """The oracle's 200 forward-Euler steps of the 32x32x16 Q1 problem: the
    vmult of every step's input and the final field."""
    cfg = solid_q1_small()
    T0 = initial_temperature(cfg, "config-parity-q1", melt_pool=False)
    o = oracle_for(cfg)
    y = flat(T0).copy()
    t, dt = 0.0, 1e-6
    vm = []
    for _ in range(200):
        o.set_time(t)
        vm.append(o.vmult(y))
        t = o.evolve_one_time_step(t, dt, y)
    return cfg, T0, vm, y, t


@pytest.mark.parametrize("schedule", [COLOURED, ATOMIC, TWO_PASS])
def test_solid_q1_200_forward_euler_steps(solid_q1_reference, schedule):
    cfg, T0, vm_ref, y_ref, t_ref = solid_q1_reference
    g = ThermalPhysics(cfg)
    g.set_schedule(schedule)
    y = g.from_grid(T0)
    dst = g.initialize_dof_vector()
    t, dt = 0.0, 1e-6
    worst = 0.0
    for n in range(200):
        g.set_time(t)
        g.vmult(dst, y)
        err = rel_max(flat(g.to_grid(dst)), vm_ref[n])
        worst = max(worst, err)
        assert err <= VMULT_TOL, (n, err)
        t = g.evolve_one_time_step(t, dt, y)
    assert t == t_ref
    assert rel_max(flat(g.to_grid(y)), y_ref) <= STEP_TOL
    assert g.device_error() == 0


@pytest.fixture(scope="module")
def phase_change_reference():
    """The oracle on the 128x128x64 Q2 phase-change problem: one vmult of
    the initial field at t = 1e-4 with the per-point powder history after
    it, then (from a fresh oracle) 20 RK4 steps of 5e-7."""
    cfg = phase_change_q2()
    T0 = initial_temperature(cfg, "bench")
    o = oracle_for(cfg)
    o.set_time(1e-4)
    vm = o.vmult(flat(T0))
    powder = o.qp_powder()
    del o
    o = oracle_for(cfg)
    y = flat(T0).copy()
    t = 0.0
    for _ in range(20):
        t = o.evolve_one_time_step(t, 5e-7, y)
    return cfg, T0, vm, powder, y, t


@pytest.mark.parametrize("schedule", [COLOURED, ATOMIC, TWO_PASS])
def test_phase_change_q2_full_size(phase_change_reference, schedule):
    cfg, T0, vm_ref, powder_ref, y_ref, t_ref = phase_change_reference
    g = ThermalPhysics(cfg)
    g.set_schedule(schedule)
    g.set_time(1e-4)
    dst = g.initialize_dof_vector()
    g.vmult(dst, g.from_grid(T0))
    assert rel_max(flat(g.to_grid(dst)), vm_ref) <= VMULT_TOL
    assert np.max(np.abs(g.get_qp_powder() - powder_ref)) < 1e-12
    del g
    torch.cuda.empty_cache()
    g = ThermalPhysics(cfg)
    g.set_schedule(schedule)
    y = g.from_grid(T0)
    t = 0.0
    for _ in range(20):
        t = g.evolve_one_time_step(t, 5e-7, y)
    assert t == t_ref
    assert rel_max(flat(g.to_grid(y)), y_ref) <= STEP_TOL
    assert g.device_error() == 0


def test_ensemble_32_members_100_rk4_steps():
    from adamantine_b200.ensemble import Ensemble

    configs, params = ensemble_q1()
    assert len(configs) == 32 and len({p[2] for p in params}) > 1
    grids = [initial_temperature(c, f"ensemble-{k}") for k, c in enumerate(configs)]
    e = Ensemble(configs)
    y = e.from_grids(grids)
    t = e.evolve_n_steps(0.0, 1e-6, 100, y)
    torch.cuda.synchronize()
    assert e.device_error() == 0
    # every member's oracle run, in spawned worker processes
    workers = max(1, min(8, oracle_runs.cores() // 2))
    threads = max(1, oracle_runs.cores() // workers)
    with oracle_runs.pool(workers) as ex:
        runs = list(ex.map(oracle_runs.ensemble_member, range(32), [100] * 32, [1e-6] * 32, [threads] * 32))
    for k, (tr, yr, act) in enumerate(runs):
        assert tr == pytest.approx(t, rel=1e-15)
        got = flat(e.to_grid(y[k]))
        err = rel_max(got[act], yr[act])
        assert err <= STEP_TOL, (k, err)


def test_adjoint_workload_oracle_forward_and_gradient():
    from adamantine_b200.adjoint import AdjointProblem

    theta_true = (1.0, 1.0, 0.35, 400.0)
    theta = (1.08, 0.93, 0.35 * 1.05, 400.0 * 0.95)
    cfg = adjoint_q2()
    T0 = initial_temperature(cfg, "adjoint")
    pts = interior_points(cfg)
    obs = [50, 100, 150, 200]
    prob = AdjointProblem(cfg, T0, 0.0, 1e-6, 200, obs, pts, checkpoint_every=20)
    prob.set_targets(prob.observe(theta_true))
    J, grad = prob.gradient(theta)
    # the oracle forward at theta and at the central-difference points
    # (h = 1e-5 relative) in the conductivity scale, in spawned workers
    h = 1e-5
    tp, tm = list(theta), list(theta)
    tp[0] *= 1 + h
    tm[0] *= 1 - h
    targets = [np.asarray(x) for x in prob.targets]
    threads = max(1, oracle_runs.cores() // 3)
    with oracle_runs.pool(3) as ex:
        Jo, Jp, Jm = ex.map(oracle_runs.adjoint_misfit, [theta, tp, tm], [targets] * 3, [threads] * 3)
    assert Jo == pytest.approx(J, rel=1e-9)
    fd0 = (Jp - Jm) / (2 * h * theta[0])
    assert abs(grad[0] - fd0) <= FD_TOL * abs(fd0), (grad[0], fd0)
