"""Refined meshes on the GPU (through the C ABI) against the CPU
restatement (oracle/amr_oracle.py) on the same meshes: the constrained
operator and inverse mass, whole runs of the reference's amr_test.info
driver loop at FE degree 2 (refinement before step 1 and every 200 steps),
runs with coarsening after the beam (the solution and the cell states
carried through refine_and_transfer), and the uniformly refined mesh, whose
operator must be the uniform fine grid's bit for bit."""
import numpy as np
import pytest
import torch

import amr_oracle
from amr_cases import AMR_MAX, AMR_MIN, amr_test_config, run_amr

from adamantine_b200.amr import AmrThermalPhysics
from adamantine_b200.thermal import ThermalPhysics

pytestmark = pytest.mark.gpu


def both(cfg, max_level, **kw):
    g = AmrThermalPhysics(cfg, max_level, initial_state=cfg.geometry.initial_state(), **kw)
    o = amr_oracle.AmrProblem(cfg, max_level, initial_state=cfg.geometry.initial_state(), **kw)
    o.setup(300.0)
    return g, o


def field(pts, rng):
    r2 = (pts[:, 0] - 2.0) ** 2 + (pts[:, 1] - 2.5) ** 2
    return 320.0 + 1600.0 * np.exp(-r2 / 0.3) + rng.uniform(0.0, 3.0, len(pts))


@pytest.mark.parametrize("degree", [1, 2])
@pytest.mark.parametrize("boundary", ["adiabatic", "convective,radiative"])
def test_constrained_operator_and_mass_match_oracle(degree, boundary):
    cfg = amr_test_config(degree=degree, n_cells=(4, 4, 2), boundary=boundary)
    g, o = both(cfg, 2)
    g.refine_mesh(0.0, 200e-6, 200, 2)
    o.refine_mesh(0.0, 200e-6, 200, 2)
    assert g.n_dofs == o.n_dofs and len(o.hanging) > 0
    assert (g.leaves() == np.array(o.forest.sorted_leaves())).all()
    im = g.inverse_mass().cpu().numpy()
    assert np.abs(im - o.inv_mass).max() <= 1e-13 * np.abs(o.inv_mass).max()
    rng = np.random.default_rng(5)
    y = field(o.dof_points(), rng)
    dev = torch.device("cuda")
    src = torch.tensor(y, device=dev)
    dst = torch.zeros_like(src)
    for t in (20e-6, 90e-6):
        g.set_time(t)
        o.set_time(t)
        g.vmult(dst, src)
        ref = o.vmult(y)
        assert np.abs(dst.cpu().numpy() - ref).max() <= 1e-10 * np.abs(ref).max()
        for sch in ("coloured", "two_pass"):
            g.set_schedule(sch)
            dst_c = torch.zeros_like(src)
            g.vmult(dst_c, src)
            dst_r = torch.zeros_like(src)
            g.vmult(dst_r, src)
            assert torch.equal(dst_c, dst_r)  # a fixed order of additions
            assert torch.abs(dst_c - dst).max().item() <= 1e-12 * np.abs(ref).max()
        g.set_schedule("atomic")


@pytest.mark.parametrize("degree,method", [(2, "forward_euler"), (1, "forward_euler"), (2, "rk_third_order")])
def test_amr_test_run_matches_oracle(degree, method):
    """amr_test.info's loop at FE degree 1 and 2 (the GPU path's degrees;
    the reference's FE_Q(3) pin is checked on the restatement), also with
    the RK3 tableau (a stage input from two earlier stages)."""
    cfg = amr_test_config(degree=degree, method=method)
    g, o = both(cfg, 1)
    run_amr(g)
    run_amr(o)
    y = g.get_solution().cpu().numpy()
    assert g.n_dofs == o.n_dofs
    assert np.abs(y - o.y).max() <= 1e-9 * np.abs(o.y).max()
    # the reference's bounds for FE_Q(3), with its 10 % tolerance
    assert abs(y.max() - AMR_MAX) <= 0.1 * AMR_MAX and abs(y.min() - AMR_MIN) <= 0.1 * AMR_MIN


@pytest.mark.parametrize("method", ["forward_euler", "rk_fourth_order"])
def test_coarsening_after_the_beam_matches_oracle(method):
    # a 40 kW beam melts the plate within the 120 us (the cell states then
    # carry liquid fractions through every remeshing)
    cfg = amr_test_config(degree=2, n_cells=(6, 6, 2), boundary="convective,radiative", method=method,
                          max_power=40000.0)
    g, o = both(cfg, 2)
    run = lambda p: run_amr(p, dt=2e-6, duration=120e-6, every=20, n_refinements=2, coarsen=True)
    run(g)
    run(o)
    assert (g.leaves() == np.array(o.forest.sorted_leaves())).all()
    y = g.get_solution().cpu().numpy()
    assert np.abs(y - o.y).max() <= 1e-9 * np.abs(o.y).max()
    assert y.max() > 1708.0  # above the liquidus
    liquid = 0.0
    for l, lev in o.levels.items():
        lev["oracle"].set_state_to_material_properties()
        ns = g.config.material.n_states
        ref = np.asarray(lev["oracle"].cell_state()).reshape(ns, -1)
        act = np.zeros(ref.shape[1], bool)
        n = lev["n"]
        for c in lev["cells"]:
            act[c[1] + n[0] * (c[2] + n[1] * c[3])] = True
        mine = g.level_cell_state(l)
        assert np.abs(mine[:, act] - ref[:, act]).max() <= 1e-9
        liquid += ref[1, act].sum()
    assert liquid > 0.0  # cells carried their molten state through the remeshing


@pytest.mark.parametrize("degree", [1, 2])
def test_uniform_refinement_is_the_fine_grid(degree):
    cfg = amr_test_config(degree=degree, n_cells=(3, 2, 2))
    g = AmrThermalPhysics(cfg, 1)
    g.set_schedule("coloured")  # the uniform grid's default: the same additions in the same order
    g.execute({tuple(c) for c in g.leaves()}, None)
    assert (g.leaves()[:, 0] == 1).all()
    fine_cfg = amr_test_config(degree=degree, n_cells=(6, 4, 4))
    fine = ThermalPhysics(fine_cfg)
    rng = np.random.default_rng(9)
    lat = g.dof_lattice()  # the level-1 node grid: lattice / (2 / degree)
    idx = lat * degree // 2
    y = field(g.dof_points() / np.array([5e-3 / 3, 5e-3 / 2, 0.5e-3 / 2]), rng)
    grid = np.zeros((fine.nodes[2], fine.nodes[1], fine.pitch))
    grid[idx[:, 2], idx[:, 1], idx[:, 0]] = y
    dev = torch.device("cuda")
    src_f = torch.tensor(grid.reshape(-1), device=dev)
    dst_f = torch.zeros_like(src_f)
    src = torch.tensor(y, device=dev)
    dst = torch.zeros_like(src)
    for t in (10e-6, 80e-6):
        g.set_time(t)
        fine.set_time(t)
        g.vmult(dst, src)
        fine.vmult(dst_f, src_f)
        ref = dst_f.cpu().numpy().reshape(grid.shape)[idx[:, 2], idx[:, 1], idx[:, 0]]
        assert (dst.cpu().numpy() == ref).all()


@pytest.mark.parametrize("degree", [1, 2])
def test_operator_with_inactive_coarse_cells(degree):
    """Part of the upper layer carries no material: faces towards missing
    material take the convective / radiative terms on every level, faces
    between levels inside the material do not; refined along the beam
    across the edge of the material, against the restatement."""
    cfg = amr_test_config(degree=degree, n_cells=(4, 4, 2), boundary="convective,radiative")
    active = np.ones(32, np.uint8)
    active[16 + 8:] = 0  # the upper layer's back half is missing
    active[16 + 1] = 0
    g, o = both(cfg, 2, active=active)
    g.refine_mesh(0.0, 200e-6, 200, 2)
    o.refine_mesh(0.0, 200e-6, 200, 2)
    assert g.n_dofs == o.n_dofs and len(o.hanging) > 0
    im = g.inverse_mass().cpu().numpy()
    assert np.abs(im - o.inv_mass).max() <= 1e-13 * np.abs(o.inv_mass).max()
    rng = np.random.default_rng(13)
    y = field(o.dof_points(), rng)
    src = torch.tensor(y, device=torch.device("cuda"))
    dst = torch.zeros_like(src)
    for t in (30e-6, 120e-6):
        g.set_time(t)
        o.set_time(t)
        g.vmult(dst, src)
        ref = o.vmult(y)
        assert np.abs(dst.cpu().numpy() - ref).max() <= 1e-10 * np.abs(ref).max()


def test_has_melted_follows_refinement():
    """refine_and_transfer carries the has_melted flags like the cell data
    (application/adamantine.hh:339-376, 463-495): a refined leaf's children
    take its flag, a coarsened family takes its first child's."""
    cfg = amr_test_config(degree=2, n_cells=(6, 6, 2), boundary="adiabatic", max_power=40000.0)
    g = AmrThermalPhysics(cfg, 2, initial_state=cfg.geometry.initial_state())
    g.refine_mesh(0.0, 40e-6, 20, 2)
    t = 0.0
    for _ in range(20):
        t = g.evolve_one_time_step(t, 2e-6)
    g.mark_has_melted(600.0)

    def flags():
        out = {}
        lv = g.leaves()
        for l in sorted(set(lv[:, 0].tolist())):
            f = g.level_has_melted(int(l))
            n0, n1 = 6 << l, 6 << l
            for c in lv[lv[:, 0] == l]:
                out[tuple(int(v) for v in c)] = int(f[c[1] + n0 * (c[2] + n1 * c[3])])
        return out

    old = flags()
    assert any(old.values()) and not all(old.values())
    g.refine_mesh(t, t + 40e-6, 20, 2, True)
    new = flags()
    assert set(new) != set(old)
    for (l, i, j, k), f in new.items():
        src = None
        for m in range(l, -1, -1):
            s = l - m
            if (m, i >> s, j >> s, k >> s) in old:
                src = (m, i >> s, j >> s, k >> s)
                break
        if src is None:  # coarsened: the first child, down to an old leaf
            src = (l, i, j, k)
            while src not in old:
                src = (src[0] + 1, 2 * src[1], 2 * src[2], 2 * src[3])
        assert f == old[src], ((l, i, j, k), src)


def test_demo_316_short_amr_run_matches_oracle():
    """demo_316_short_amr.info's driver loop on the GPU: the same meshes as the
    restatement at every refinement, the reference's 13005 DoFs at the end,
    and the field within 1e-9 of the restatement's."""
    from amr_cases import (DEMO_AMR_DOFS, DEMO_AMR_DT, DEMO_AMR_DURATION, DEMO_AMR_EVERY,
                           demo_316_short_amr_config)

    cfg = demo_316_short_amr_config()
    g, o = both(cfg, 1)
    run = lambda p: run_amr(p, dt=DEMO_AMR_DT, duration=DEMO_AMR_DURATION, every=DEMO_AMR_EVERY, n_refinements=1,
                            coarsen=True)
    run(g)
    run(o)
    assert g.n_dofs == o.n_dofs == DEMO_AMR_DOFS
    assert (g.leaves() == np.array(o.forest.sorted_leaves())).all()
    y = g.get_solution().cpu().numpy()
    assert np.isfinite(y).all()
    assert np.abs(y - o.y).max() <= 1e-9 * np.abs(o.y).max()
