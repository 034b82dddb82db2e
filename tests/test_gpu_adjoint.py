"""Hand-written adjoint of the explicit step (through the C ABI): the
transpose operator against finite differences of the GPU operator, and the
misfit gradient against central finite differences (h = 1e-5 relative) of
both the GPU forward and the CPU oracle forward.
"""
import numpy as np
import pytest
import torch

import oracle_py
from adamantine_b200.adjoint import AdjointProblem, MisfitFunction, config_at
from adamantine_b200.config import Boundary, Geometry, Source, ThermalConfig
from adamantine_b200.thermal import ThermalPhysics
from adamantine_b200.workloads import (adjoint_q2, initial_temperature, interior_points, phase_change_material,
                                       rng_for)

pytestmark = pytest.mark.gpu

FD_TOL = 1e-6
THETA_TRUE = (1.0, 1.0, 0.35, 400.0)
THETA = (1.08, 0.93, 0.35 * 1.05, 400.0 * 0.95)


def small_problem(method="rk_second_order", n_steps=40, K=10):
    cfg = adjoint_q2(n_cells=(16, 16, 8), extent=(5e-3, 5e-3, 2.5e-3), powder_layers=2, method=method)
    T0 = initial_temperature(cfg, "adjoint-test")
    pts = interior_points(cfg, n_points=60, radius=0.8e-3, depth=0.8e-3, name="adjoint-test-points")
    obs = [n_steps // 4, n_steps // 2, 3 * n_steps // 4, n_steps]
    prob = AdjointProblem(cfg, T0, 0.0, 1e-6, n_steps, obs, pts, checkpoint_every=K)
    prob.set_targets(prob.observe(THETA_TRUE))
    return cfg, T0, pts, obs, prob


def central_fd(f, theta, h=1e-5):
    g = np.zeros(4)
    for k in range(4):
        tp, tm = list(theta), list(theta)
        tp[k] *= 1 + h
        tm[k] *= 1 - h
        g[k] = (f(tp) - f(tm)) / (2 * h * theta[k])
    return g


def rel(a, b):
    return float(np.max(np.abs(np.asarray(a) - np.asarray(b)) / np.maximum(np.abs(b), 1e-300)))


def test_transpose_operator_matches_operator_derivative():
    """<(r(y + e d) - r(y - e d)) / 2e, mu> = <d, (dr/dT)^T mu>, and the
    parameter log-derivatives of mu . r, for a two-state material with a
    beam (no phase history, so r is a function of y alone)."""
    geo = Geometry(dim=3, n_cells=(16, 16, 8), extent=(5e-3, 5e-3, 2.5e-3))
    db = {"property_format": "polynomial", "n_materials": 1, "material_0.solidus": 1600.0,
          "material_0.liquidus": 1650.0, "material_0.latent_heat": 2.5e5}
    for s, k in (("solid", "20.0, 0.01, -2e-6"), ("liquid", "30.0, 0.002")):
        db[f"material_0.{s}.density"] = "7800.0, -0.1"
        db[f"material_0.{s}.specific_heat"] = "450.0, 0.2"
        for ax, f in (("x", 1.0), ("y", 0.8), ("z", 1.1)):
            db[f"material_0.{s}.thermal_conductivity_{ax}"] = ", ".join(str(float(v) * f) for v in k.split(","))
    from adamantine_b200.config import Material

    mat = Material.from_database(db, n_states=2, p_order=2)
    seg = np.array([[1e-9, 0.0, 2.5e-3, 2.5e-3, 2.5e-3], [1.0, 1.0, 4.0e-3, 2.5e-3, 2.5e-3]])
    src = Source(type="goldak", depth=300e-6, absorption_efficiency=0.4, diameter=600e-6, max_power=300.0,
                 segments=seg)
    cfg = ThermalConfig(geometry=geo, material=mat, boundary=Boundary.from_database({"type": "adiabatic"}, 3),
                        sources=[src], degree=2)
    rng = rng_for("transpose-test")
    shape = geo.node_shape(2)[::-1]
    T = 1400.0 + 400.0 * rng.uniform(0, 1, shape)
    prob = AdjointProblem(cfg, T, 0.0, 1e-6, 1, [1], np.array([[1, 1, 1]]))
    g = prob.phys
    g.set_time(2e-4)
    y = g.from_grid(T)
    d = g.from_grid(rng.uniform(-1, 1, shape))
    mu = g.from_grid(rng.uniform(-1, 1, shape))
    lam, pg = prob.vmult_transpose(y, mu)
    eps = 1e-4

    def r(v):
        out = torch.zeros_like(v)
        g.vmult(out, v)
        return out

    fd = torch.dot(r(y + eps * d) - r(y - eps * d), mu).item() / (2 * eps)
    adj = torch.dot(d, lam).item()
    # the difference quotient carries the rounding of r (~1e-16 |r| / eps,
    # about 1e-6 of the directional derivative here)
    assert abs(fd - adj) <= 1e-5 * abs(adj)

    def mu_r(theta):
        c = config_at(cfg, theta)
        g.update_material(c)
        g.update_beam(0, c.sources[0].depth, c.sources[0].absorption_efficiency, c.sources[0].diameter,
                      c.sources[0].max_power)
        return torch.dot(r(y), mu).item()

    base = (1.0, 1.0, 0.4, 300.0)
    fdp = central_fd(mu_r, base, h=1e-6) * np.asarray(base)  # log-derivatives
    assert rel(pg[0], fdp[0]) <= 1e-6
    assert rel(pg[1], fdp[1]) <= 1e-6
    assert rel(pg[2], fdp[2]) <= 1e-6
    assert rel(pg[2], fdp[3]) <= 1e-6


@pytest.mark.parametrize("method", ["rk_second_order", "forward_euler", "rk_fourth_order"])
def test_gradient_matches_gpu_finite_differences(method):
    cfg, T0, pts, obs, prob = small_problem(method=method)
    J, grad = prob.gradient(THETA)
    assert J > 0
    assert J == pytest.approx(prob.objective(THETA), rel=1e-13)
    fd = central_fd(prob.objective, THETA)
    assert rel(grad, fd) <= FD_TOL, (grad, fd)


def test_gradient_matches_oracle_finite_differences():
    cfg, T0, pts, obs, prob = small_problem()
    J, grad = prob.gradient(THETA)
    nx, ny, nz = cfg.geometry.node_shape(2)
    flat = pts[:, 0] + nx * (pts[:, 1] + ny * pts[:, 2])

    def oracle_J(theta):
        c = config_at(cfg, theta)
        st = c.to_struct()
        o = oracle_py.Oracle(st, active=c.geometry.active_cells(), initial_state=c.geometry.initial_state())
        y = np.ascontiguousarray(T0, np.float64).reshape(-1).copy()
        t, Jv = 0.0, 0.0
        for n in range(1, prob.n_steps + 1):
            t = o.evolve_one_time_step(t, prob.dt, y)
            if n in obs:
                k = obs.index(n)
                Jv += float(np.sum((y[flat] - prob.targets[k]) ** 2))
        return Jv

    assert oracle_J(THETA) == pytest.approx(J, rel=1e-9)
    fd = central_fd(oracle_J, THETA)
    assert rel(grad, fd) <= FD_TOL, (grad, fd)


def test_checkpoint_interval_does_not_change_the_gradient():
    cfg, T0, pts, obs, prob = small_problem(K=7)
    J1, g1 = prob.gradient(THETA)
    prob.checkpoint_every = 40
    J2, g2 = prob.gradient(THETA)
    assert J1 == J2
    assert rel(g1, g2) <= 1e-12
    # the automatic interval keeps the whole (small) run: no recompute
    prob.checkpoint_every = 0
    J3, g3 = prob.gradient(THETA)
    assert prob.last_checkpoint_interval() == prob.n_steps
    assert J3 == J1 and rel(g1, g3) <= 1e-12


def test_flushed_adjoint_gives_the_same_gradient():
    """Skipping tiles whose adjoint is at most 1e-30 of the stage's largest
    (the default) against skipping exact zeros only: the same gradient to
    rounding, on a mesh large enough for most tiles to be skipped."""
    cfg = adjoint_q2(n_cells=(48, 48, 16), extent=(15e-3, 15e-3, 5e-3), powder_layers=4)
    T0 = initial_temperature(cfg, "adjoint-flush")
    pts = interior_points(cfg, n_points=80, radius=0.6e-3, depth=0.6e-3, name="adjoint-flush-points")
    prob = AdjointProblem(cfg, T0, 0.0, 1e-6, 60, [30, 60], pts, checkpoint_every=20)
    prob.set_targets(prob.observe(THETA_TRUE))
    J1, g1 = prob.gradient(THETA)
    prob.set_flush(0.0)
    J0, g0 = prob.gradient(THETA)
    assert J1 == J0
    assert rel(g1, g0) <= 1e-13
    assert np.all(np.abs(g0) > 0)


def test_autograd_binding():
    cfg, T0, pts, obs, prob = small_problem(n_steps=20, K=5)
    theta = torch.tensor(THETA, dtype=torch.float64, requires_grad=True)
    J = MisfitFunction.apply(theta, prob)
    J.backward()
    J2, g = prob.gradient(THETA)
    assert J.item() == J2
    assert rel(theta.grad.numpy(), g) <= 1e-12
