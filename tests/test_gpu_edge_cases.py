"""Edge cases of the operator through the C ABI against the oracle: a single
cell, a one-tile-thick strip, a mesh with no active cell (every result zero,
steps leave the field alone), activation of every cell of an empty mesh, and
both launch schedules."""
import numpy as np
import pytest
import torch

import oracle_py
from pairs import rel_max

from adamantine_b200.config import Boundary, Geometry, Source, ThermalConfig
from adamantine_b200.thermal import ThermalPhysics
from adamantine_b200.workloads import phase_change_material, rng_for

pytestmark = pytest.mark.gpu


def problem(n_cells, extent, degree, material_height=1e9, faces=False):
    geo = Geometry(dim=3, n_cells=n_cells, extent=extent, material_height=material_height, use_powder=True,
                   powder_layer=0.5 * extent[2])
    bnd = Boundary.from_database({"type": "adiabatic", "boundary_5.type": "convective"} if faces else
                                 {"type": "adiabatic"}, 3)
    mat = phase_change_material()
    mat.props[0, 4] = 300.0
    mat.poly[0, 7, :3, 0] = 20.0
    seg = np.array([[1e-9, 0.0, 0.2 * extent[0], 0.5 * extent[1], extent[2]],
                    [1.0, 1.0, 0.8 * extent[0], 0.5 * extent[1], extent[2]]])
    src = Source(type="goldak", depth=0.5 * extent[2], absorption_efficiency=0.4, diameter=0.5 * extent[0],
                 max_power=100.0, segments=seg)
    cfg = ThermalConfig(geometry=geo, material=mat, boundary=bnd, sources=[src], degree=degree,
                        time_method="rk_fourth_order")
    rng = rng_for(f"edge-{n_cells}-{degree}")
    T = 1500.0 + 300.0 * rng.uniform(0, 1, geo.node_shape(degree)[::-1])
    return cfg, T


def oracle(cfg):
    st = cfg.to_struct()
    o = oracle_py.Oracle(st, active=cfg.geometry.active_cells(), initial_state=cfg.geometry.initial_state())
    o._keep = st
    return o


@pytest.mark.parametrize("schedule", [0, 1])
@pytest.mark.parametrize("shape,degree,faces", [((1, 1, 1), 1, False), ((1, 1, 1), 2, True),
                                                ((40, 3, 1), 2, False), ((17, 1, 9), 1, True)])
def test_small_and_thin_meshes(shape, degree, faces, schedule):
    ext = tuple(1e-4 * n for n in shape)
    cfg, T = problem(shape, ext, degree, faces=faces)
    o = oracle(cfg)
    g = ThermalPhysics(cfg)
    g.set_schedule(schedule)
    o.set_time(1e-4)
    g.set_time(1e-4)
    dst = g.initialize_dof_vector()
    g.vmult(dst, g.from_grid(T))
    assert rel_max(g.to_grid(dst).reshape(-1), o.vmult(T.reshape(-1))) <= 1e-12
    y_ref = T.reshape(-1).copy()
    y = g.from_grid(T)
    t = 0.0
    for _ in range(4):
        o.evolve_one_time_step(t, 1e-7, y_ref)
        t = g.evolve_one_time_step(t, 1e-7, y)
    assert rel_max(g.to_grid(y).reshape(-1), y_ref) <= 1e-9
    assert g.device_error() == 0


@pytest.mark.parametrize("schedule", [0, 1])
def test_no_active_cell(schedule):
    cfg, T = problem((9, 7, 5), (0.9e-3, 0.7e-3, 0.5e-3), 2, material_height=-1.0)
    g = ThermalPhysics(cfg)
    g.set_schedule(schedule)
    dst = g.initialize_dof_vector(5.0)
    src = g.from_grid(T)
    g.vmult(dst, src)
    assert float(dst.abs().max().item()) == 0.0
    assert float(g.get_inverse_mass_matrix().abs().max().item()) == 0.0
    y = src.clone()
    g.evolve_one_time_step(0.0, 1e-6, y)
    assert torch.equal(y, src)
    # then every cell becomes active: the oracle with everything active
    cells = np.arange(g.n_cells, dtype=np.int64)
    g.add_material(cells, 400.0, y)
    ref = T.reshape(-1).copy()
    o2 = oracle(cfg)
    o2.activate_cells(cells, 400.0, ref)
    got = g.to_grid(y).reshape(-1)
    assert np.array_equal(got, ref)
    t = 0.0
    for _ in range(3):
        o2.evolve_one_time_step(t, 1e-7, ref)
        t = g.evolve_one_time_step(t, 1e-7, y)
    assert rel_max(g.to_grid(y).reshape(-1), ref) <= 1e-9
