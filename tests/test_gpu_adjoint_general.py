"""Adjoint of the general operator (through the C ABI): 12-point tables,
several materials, deposition-angle rotation, convective / radiative faces
and active/inactive interfaces with the powder history of the face points,
cube sources.

The transpose operator is checked against the directional derivative of the
GPU operator on every parity case (the phase state restored between the two
evaluations), and the misfit gradient against central finite differences
(h = 1e-5 relative) of the GPU forward and of the CPU oracle forward.
"""
import copy

import numpy as np
import pytest
import torch

import oracle_py
from adamantine_b200.adjoint import AdjointProblem, config_at
from adamantine_b200.config import Boundary
from adamantine_b200.workloads import adjoint_q2, initial_temperature, interior_points, rng_for
from pairs import CASES, make_case, table_material

pytestmark = pytest.mark.gpu

FD_TOL = 1e-6
THETA_TRUE = (1.0, 1.0, 0.35, 400.0)
THETA = (1.08, 0.93, 0.35 * 1.05, 400.0 * 0.95)


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


def cell_kwargs(cells):
    return {k: cells.get(k) for k in ("material_id", "deposition_cos", "deposition_sin")}


@pytest.mark.parametrize("case", CASES)
def test_transpose_operator_on_the_parity_cases(case, tmp_path):
    """<(r(y + e d) - r(y - e d)) / 2e, mu> = <d, (dr/dT)^T mu> and the
    parameter log-derivatives of mu . r, with the phase state (cells' and
    face points' powder history) restored before every evaluation."""
    cfg, cells, T = make_case(case)
    prob = AdjointProblem(cfg, T, 0.0, 1e-6, 1, [1], np.array([[1, 1, 1]]), **cell_kwargs(cells))
    g = prob.phys
    t_op = 2e-4
    rng = rng_for("transpose-" + case)
    y = g.from_grid(T)
    d = g.from_grid(rng.uniform(-1, 1, T.shape))
    mu = g.from_grid(rng.uniform(-1, 1, T.shape))
    ck = str(tmp_path / "phase.ck")
    g.save_checkpoint(ck, 0.0, y)
    scratch = torch.empty_like(y)

    def restore():
        g.load_checkpoint(ck, scratch, exact=True)
        g.set_time(t_op)

    def r(v):
        restore()
        out = torch.zeros_like(v)
        g.vmult(out, v)
        return out

    eps = 1e-4
    fd = torch.dot(r(y + eps * d) - r(y - eps * d), mu).item() / (2 * eps)
    restore()
    lam, pg = prob.vmult_transpose(y, mu)
    adj = torch.dot(d, lam).item()
    assert abs(fd - adj) <= 1e-5 * abs(adj), (fd, adj)

    def mu_r(theta):
        c = config_at(cfg, theta)
        g.update_material(c)
        for i, s in enumerate(c.sources):
            if s.type != "cube":
                g.update_beam(i, s.depth, s.absorption_efficiency, s.diameter, s.max_power)
        return torch.dot(r(y), mu).item()

    src = [s for s in cfg.sources if s.type != "cube"]
    base = (1.0, 1.0, src[0].absorption_efficiency if src else 1.0, src[0].max_power if src else 1.0)
    fdp = central_fd(mu_r, base, h=1e-6) * np.asarray(base)  # log-derivatives
    assert rel(pg[0], fdp[0]) <= 1e-6
    assert rel(pg[1], fdp[1]) <= 1e-6
    if src:
        assert rel(pg[2], fdp[2]) <= 1e-6
        assert rel(pg[2], fdp[3]) <= 1e-6
    else:
        # a cube source keeps its value: no source-strength derivative
        assert pg[2] == 0.0
        assert abs(fdp[2]) <= 1e-9 * abs(fdp[1])


def faces_config(method="rk_second_order"):
    """The adjoint workload's 16 x 16 x 8 case with a convective and
    radiative top (the powder layer) and a convective x- side; the face
    coefficients depend on temperature and state, so the face points'
    powder history enters the gradient."""
    cfg = adjoint_q2(n_cells=(16, 16, 8), extent=(5e-3, 5e-3, 2.5e-3), powder_layers=2, method=method)
    cfg = copy.deepcopy(cfg)
    mat = cfg.material
    mat.props[0, 3] = 300.0  # radiation_temperature_infty
    mat.props[0, 4] = 295.0  # convection_temperature_infty
    for st, (em, hc) in enumerate(((0.3, 2.0e4), (0.2, 1.5e4), (0.7, 0.8e4))):  # solid, liquid, powder
        mat.poly[0, 5, st, :2] = (em, 1e-4)   # emissivity
        mat.poly[0, 7, st, :2] = (hc, 3.0)    # convection coefficient
    cfg.boundary = Boundary.from_database({"type": "adiabatic", "boundary_5.type": "radiative,convective",
                                           "boundary_0.type": "convective"}, 3)
    return cfg


def top_points(cfg, n=24, radius=0.6e-3, name="adjoint-top-points"):
    """Seeded nodes of the top surface within `radius` of the scan-path start."""
    rng = rng_for(name)
    nx, ny, nz = cfg.geometry.node_shape(cfg.degree)
    h = [cfg.geometry.extent[0] / (nx - 1), cfg.geometry.extent[1] / (ny - 1)]
    seg = cfg.sources[0].segments
    i0, i1 = int((seg[0, 2] - radius) / h[0]), int((seg[0, 2] + radius) / h[0])
    j0, j1 = int((seg[0, 3] - radius) / h[1]), int((seg[0, 3] + radius) / h[1])
    cand = np.array([(i, j, nz - 1) for j in range(j0, j1 + 1) for i in range(i0, i1 + 1)])
    return cand[np.sort(rng.choice(len(cand), size=min(n, len(cand)), replace=False))]


def make_problem(cfg, cells, n_steps, K, name):
    T0 = initial_temperature(cfg, name)
    pts = np.concatenate([interior_points(cfg, n_points=40, radius=0.8e-3, depth=0.8e-3, name=name + "-in"),
                          top_points(cfg, name=name + "-top")])
    obs = [n_steps // 3, 2 * n_steps // 3, n_steps]
    prob = AdjointProblem(cfg, T0, 0.0, 1e-6, n_steps, obs, pts, checkpoint_every=K, **cell_kwargs(cells))
    prob.set_targets(prob.observe(THETA_TRUE))
    return T0, pts, obs, prob


def table_rotation_config():
    """Q1 with the two-material table material (three states), seeded
    material ids and deposition angles per cell, on the adjoint workload's
    16 x 16 x 8 box."""
    cfg = adjoint_q2(n_cells=(16, 16, 8), extent=(5e-3, 5e-3, 2.5e-3), powder_layers=2)
    cfg = copy.deepcopy(cfg)
    cfg.material = table_material()
    cfg.degree = 1
    rng = rng_for("adjoint-table-rotation-cells")
    C = cfg.geometry.n_cells_total
    ang = rng.uniform(0, np.pi, C)
    cells = {"material_id": (rng.uniform(size=C) < 0.3).astype(np.uint8), "deposition_cos": np.cos(ang),
             "deposition_sin": np.sin(ang)}
    return cfg, cells


def oracle_objective(cfg, cells, T0, pts, obs, prob):
    nx, ny, nz = cfg.geometry.node_shape(cfg.degree)
    flat = pts[:, 0] + nx * (pts[:, 1] + ny * pts[:, 2])

    def J(theta):
        c = config_at(cfg, theta)
        st = c.to_struct()
        o = oracle_py.Oracle(st, active=c.geometry.active_cells(), initial_state=c.geometry.initial_state(),
                             **cell_kwargs(cells))
        y = np.ascontiguousarray(T0, np.float64).reshape(-1).copy()
        t, Jv = 0.0, 0.0
        for n in range(1, prob.n_steps + 1):
            t = o.evolve_one_time_step(t, prob.dt, y)
            if n in obs:
                Jv += float(np.sum((y[flat] - prob.targets[obs.index(n)]) ** 2))
        return Jv

    return J


def test_faces_gradient_matches_gpu_finite_differences():
    cfg = faces_config()
    T0, pts, obs, prob = make_problem(cfg, {}, 30, 10, "adjoint-faces")
    J, grad = prob.gradient(THETA)
    assert J > 0
    assert J == pytest.approx(prob.objective(THETA), rel=1e-13)
    fd = central_fd(prob.objective, THETA)
    assert rel(grad, fd) <= FD_TOL, (grad, fd)
    # the face points' stored history through recompute: the same gradient
    # with every step kept
    prob.checkpoint_every = 30
    J2, g2 = prob.gradient(THETA)
    assert J2 == J and rel(g2, grad) <= 1e-12


def test_faces_gradient_matches_oracle_finite_differences():
    cfg = faces_config(method="rk_third_order")
    T0, pts, obs, prob = make_problem(cfg, {}, 24, 8, "adjoint-faces-oracle")
    J, grad = prob.gradient(THETA)
    oJ = oracle_objective(cfg, {}, T0, pts, obs, prob)
    assert oJ(THETA) == pytest.approx(J, rel=1e-9)
    fd = central_fd(oJ, THETA)
    assert rel(grad, fd) <= FD_TOL, (grad, fd)


def test_table_rotation_gradient_matches_gpu_and_oracle_finite_differences():
    cfg, cells = table_rotation_config()
    T0, pts, obs, prob = make_problem(cfg, cells, 30, 10, "adjoint-table-rotation")
    J, grad = prob.gradient(THETA)
    assert J > 0
    fd = central_fd(prob.objective, THETA)
    assert rel(grad, fd) <= FD_TOL, (grad, fd)
    oJ = oracle_objective(cfg, cells, T0, pts, obs, prob)
    assert oJ(THETA) == pytest.approx(J, rel=1e-9)
    fdo = central_fd(oJ, THETA)
    assert rel(grad, fdo) <= FD_TOL, (grad, fdo)
