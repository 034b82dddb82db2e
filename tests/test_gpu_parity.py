"""Parity of the CUDA path (through the C ABI) with the CPU oracle.

Bars: FP64 max-norm relative error <= 1e-12 per vmult, <= 1e-9 on
temperatures after N time steps (the tolerances of the hot-path contract).
"""
import numpy as np
import pytest
import torch

from pairs import CASES, make_case, make_gpu, make_oracle, rel_max

pytestmark = pytest.mark.gpu

VMULT_TOL = 1e-12
STEP_TOL = 1e-9


def grid(v):
    return np.asarray(v).reshape(-1)


@pytest.mark.parametrize("name", CASES)
def test_vmult_parity(name):
    cfg, cells, T = make_case(name)
    o = make_oracle(cfg, cells)
    g = make_gpu(cfg, cells)
    t = 2e-4 if name != "q2_slp_partial_faces_cube" else 1e-5
    o.set_time(t)
    g.set_time(t)
    src = g.from_grid(T)
    dst = g.initialize_dof_vector(123.0)
    # three applications: the per-quadrature-point phase history changes
    for k in range(3):
        Tk = T * (1.0 + 0.05 * k)
        src = g.from_grid(Tk)
        g.vmult(dst, src)
        ref = o.vmult(grid(Tk))
        got = grid(g.to_grid(dst))
        assert rel_max(got, ref) <= VMULT_TOL, (name, k, rel_max(got, ref))
    if cfg.material.n_states == 3:
        assert np.max(np.abs(g.get_qp_powder() - o.qp_powder())) < 1e-12
    assert g.device_error() == 0


@pytest.mark.parametrize("name", CASES)
def test_vmult_add_and_inverse_mass(name):
    cfg, cells, T = make_case(name)
    o = make_oracle(cfg, cells)
    g = make_gpu(cfg, cells)
    o.set_time(1e-5)
    g.set_time(1e-5)
    base = np.random.default_rng(1).uniform(-1, 1, T.size)
    dst = g.from_grid(base)
    g.vmult_add(dst, g.from_grid(T))
    ref = base.copy()
    o.vmult_add(ref, grid(T))
    assert rel_max(grid(g.to_grid(dst)), ref) <= VMULT_TOL
    assert rel_max(grid(g.to_grid(g.get_inverse_mass_matrix())), o.inverse_mass()) <= 1e-14


@pytest.mark.parametrize("name", CASES)
def test_time_steps_parity(name):
    cfg, cells, T = make_case(name)
    o = make_oracle(cfg, cells)
    g = make_gpu(cfg, cells)
    dt = 2e-6 if cfg.degree == 2 else 5e-6
    y_ref = grid(T).copy()
    y = g.from_grid(T)
    t_ref = t = 1e-5
    for _ in range(12):
        t_ref = o.evolve_one_time_step(t_ref, dt, y_ref)
        t = g.evolve_one_time_step(t, dt, y)
    assert t == t_ref
    assert rel_max(grid(g.to_grid(y)), y_ref) <= STEP_TOL
    # the cell state after the steps (set_state_to_material_properties)
    o.set_state_to_material_properties()
    g.set_state_to_material_properties()
    assert np.max(np.abs(g.get_cell_state() - o.cell_state())) < 1e-10
    assert g.device_error() == 0


def test_graph_steps_match_single_steps():
    cfg, cells, T = make_case("q2_slp_goldak")
    g1 = make_gpu(cfg, cells)
    g2 = make_gpu(cfg, cells)
    y1 = g1.from_grid(T)
    y2 = g2.from_grid(T)
    t1 = 0.0
    for _ in range(10):
        t1 = g1.evolve_one_time_step(t1, 1e-6, y1)
    t2 = g2.evolve_n_steps(0.0, 1e-6, 10, y2)
    torch.cuda.synchronize()
    assert t1 == t2
    assert torch.equal(y1, y2)


@pytest.mark.parametrize("name", ["q2_slp_goldak", "q1_table_rotation"])
def test_material_properties_and_state(name):
    cfg, cells, T = make_case(name)
    o = make_oracle(cfg, cells)
    g = make_gpu(cfg, cells)
    pv_ref = o.evaluate_material_properties(grid(T))
    pv = g.evaluate_material_properties(g.from_grid(T)).cpu().numpy()
    assert rel_max(pv, pv_ref) < 1e-12
    assert np.max(np.abs(g.get_cell_state() - o.cell_state())) < 1e-13
    hm_ref = o.mark_has_melted(1650.0, grid(T))
    hm = g.mark_has_melted(1650.0, g.from_grid(T))
    assert np.array_equal(hm, hm_ref)


def test_activation_parity():
    cfg, cells, T = make_case("q2_slp_partial_faces_cube")
    o = make_oracle(cfg, cells)
    g = make_gpu(cfg, cells)
    y_ref = grid(T).copy()
    y = g.from_grid(T)
    dt = 2e-6
    t = 1e-5
    for _ in range(3):
        o.evolve_one_time_step(t, dt, y_ref)
        t = g.evolve_one_time_step(t, dt, y)
    # activate one layer of cells above the active region
    geo = cfg.geometry
    nx, ny, nz = geo.n_cells
    act = geo.active_cells().reshape(nz, ny, nx)
    layer = int(np.argmin(act[:, 0, 0]))
    new = np.array([x + nx * (y_ + ny * layer) for y_ in range(ny) for x in range(nx)], np.int64)
    cs = np.full(new.size, 0.5)
    sn = np.full(new.size, np.sqrt(0.75))
    o.activate_cells(new, 1700.0, y_ref, cs, sn)
    g.add_material(new, 1700.0, y, cs, sn)
    assert rel_max(grid(g.to_grid(y)), y_ref) <= STEP_TOL
    for _ in range(3):
        o.evolve_one_time_step(t, dt, y_ref)
        t = g.evolve_one_time_step(t, dt, y)
    assert rel_max(grid(g.to_grid(y)), y_ref) <= STEP_TOL
    assert g.device_error() == 0


Q1_CASES = [c for c in CASES if c.startswith("q1_")]


@pytest.mark.parametrize("cz", [2, 4])
@pytest.mark.parametrize("schedule", [0, 1, 2])
@pytest.mark.parametrize("name", Q1_CASES)
def test_q1_cells_per_thread_variants(name, schedule, cz):
    """The FE_Q(1) kernel variants with two cells (stacked in z) per thread
    and with one warp per tile (a column of four cells per thread): the same
    bars against the oracle in every launch schedule (vmult with its phase
    history over three applications, 12 time steps)."""
    cfg, cells, T = make_case(name)
    o = make_oracle(cfg, cells)
    g = make_gpu(cfg, cells)
    g.set_cells_per_thread(cz)
    g.set_schedule(schedule)
    assert g.cells_per_thread() == cz
    o.set_time(2e-4)
    g.set_time(2e-4)
    dst = g.initialize_dof_vector()
    for k in range(3):
        Tk = T * (1.0 + 0.05 * k)
        g.vmult(dst, g.from_grid(Tk))
        assert rel_max(grid(g.to_grid(dst)), o.vmult(grid(Tk))) <= VMULT_TOL, k
    if cfg.material.n_states == 3:
        assert np.max(np.abs(g.get_qp_powder() - o.qp_powder())) < 1e-12
    o2 = make_oracle(cfg, cells)
    g2 = make_gpu(cfg, cells)
    g2.set_cells_per_thread(cz)
    g2.set_schedule(schedule)
    y_ref = grid(T).copy()
    y = g2.from_grid(T)
    t_ref = t = 1e-5
    for _ in range(12):
        t_ref = o2.evolve_one_time_step(t_ref, 5e-6, y_ref)
        t = g2.evolve_one_time_step(t, 5e-6, y)
    assert rel_max(grid(g2.to_grid(y)), y_ref) <= STEP_TOL
    assert g.device_error() == 0 and g2.device_error() == 0


def test_two_cells_per_thread_is_a_q1_variant():
    cfg, cells, T = make_case("q2_slp_goldak")
    g = make_gpu(cfg, cells)
    with pytest.raises(Exception):
        g.set_cells_per_thread(2)
    with pytest.raises(Exception):
        g.set_cells_per_thread(4)
    with pytest.raises(Exception):
        g.set_cells_per_thread(3)


Q2_CASES = [c for c in CASES if c.startswith("q2_")]


@pytest.mark.parametrize("name", Q2_CASES)
def test_q2_128_cell_blocks(name):
    """The FE_Q(2) kernel variant with 128-cell blocks (z-pairs of tiles, the
    atomic schedule): the same bars against the oracle (three vmults with
    their phase history, 12 time steps), with faces and partial activation
    (pairs with one inactive tile) among the cases."""
    cfg, cells, T = make_case(name)
    o = make_oracle(cfg, cells)
    g = make_gpu(cfg, cells)
    g.set_schedule(1)
    g.set_cells_per_block(128)
    assert g.cells_per_block() == 128
    o.set_time(2e-5)
    g.set_time(2e-5)
    dst = g.initialize_dof_vector()
    for k in range(3):
        Tk = T * (1.0 + 0.05 * k)
        g.vmult(dst, g.from_grid(Tk))
        assert rel_max(grid(g.to_grid(dst)), o.vmult(grid(Tk))) <= VMULT_TOL, k
    if cfg.material.n_states == 3:
        assert np.max(np.abs(g.get_qp_powder() - o.qp_powder())) < 1e-12
    o2 = make_oracle(cfg, cells)
    g2 = make_gpu(cfg, cells)
    g2.set_schedule(1)
    g2.set_cells_per_block(128)
    y_ref = grid(T).copy()
    y = g2.from_grid(T)
    t_ref = t = 1e-5
    for _ in range(12):
        t_ref = o2.evolve_one_time_step(t_ref, 2e-6, y_ref)
        t = g2.evolve_one_time_step(t, 2e-6, y)
    assert rel_max(grid(g2.to_grid(y)), y_ref) <= STEP_TOL
    assert g.device_error() == 0 and g2.device_error() == 0


def test_cells_per_block_values():
    cfg, cells, T = make_case("q2_slp_goldak")
    g = make_gpu(cfg, cells)
    assert g.cells_per_block() == 64
    for bad in (32, 96, 256):
        with pytest.raises(Exception):
            g.set_cells_per_block(bad)
    cfg1, cells1, _ = make_case("q1_solid_convective_goldak")
    g1 = make_gpu(cfg1, cells1)
    assert g1.cells_per_block() == 128
    with pytest.raises(Exception):
        g1.set_cells_per_block(256)
    # the autotuner times the 128-cell blocks with the atomic schedule and
    # keeps whichever variant is fastest
    choice, ms = g.autotune(g.from_grid(T))
    assert g.cells_per_block() in (64, 128) and min(ms) > 0
