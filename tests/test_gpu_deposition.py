"""Material deposition on the GPU (through the C ABI): the device activation
list against the numpy restatement of get_elements_to_activate and the
reference's activation counts, and the temperatures of a deposition run
against the CPU oracle with the same activations.
"""
import os

import numpy as np
import pytest
import torch

import oracle_py
from deposition_oracle import activate
from pairs import rel_max

from adamantine_b200.config import Boundary, Geometry, Source, ThermalConfig
from adamantine_b200.deposition import Deposition, deposition_boxes, read_material_deposition
from adamantine_b200.thermal import ThermalPhysics
from adamantine_b200.workloads import initial_temperature, phase_change_material, rng_for, serpentine_segments

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = np.load(os.path.join(HERE, "golden", "deposition_inputs.npz"))
STEP_TOL = 1e-9


def oracle_for(cfg, active):
    st = cfg.to_struct()
    o = oracle_py.Oracle(st, active=active, initial_state=cfg.geometry.initial_state())
    o._keep = st
    return o


def test_device_activation_counts_known_answers():
    """material_deposition (test_material_deposition.cc:261-368) through the
    device activation: 610 ... 720 active cells after the ten windows."""
    text = "3\n" + "\n".join(" ".join(repr(float(v)) for v in row) for row in GOLD["material_path"])
    boxes = read_material_deposition(text)
    geo = Geometry(dim=3, n_cells=(10, 10, 10), extent=(10.0, 10.0, 10.0), material_height=6.0, use_powder=True,
                   powder_layer=1.0)
    cfg = ThermalConfig(geometry=geo, material=phase_change_material(), boundary=Boundary.from_database(
        {"type": "adiabatic"}, 3), degree=1)
    g = ThermalPhysics(cfg)
    dep = Deposition(g, boxes)
    y = g.initialize_dof_vector(300.0)
    active = geo.active_cells().astype(bool)
    dt, t = 0.1, 0.1
    eps = dt / 1e12
    counts = []
    for _ in range(10):
        s = int(np.searchsorted(boxes.time, t - eps, side="left"))
        e = int(np.searchsorted(boxes.time, t + dt - eps, side="left"))
        if s < e:
            n = dep.activate_range(s, e, 300.0, y)
            cells, _ = activate(active, boxes.lo, boxes.hi, s, e, (0, 0, 0), (1.0, 1.0, 1.0), (10, 10, 10))
            assert n == cells.size
            active[cells] = True
        t += dt
        counts.append(int(active.sum()))
    assert counts == [610, 620, 630, 650, 650, 660, 670, 680, 720, 720]
    # the device's DoF set is the one of the oracle with the same cells
    o = oracle_for(cfg, active.astype(np.uint8))
    im = g.to_grid(g.get_inverse_mass_matrix()).reshape(-1)
    assert np.array_equal(im > 0, o.node_active().astype(bool))
    assert rel_max(im[im > 0], o.inverse_mass()[im > 0]) <= 1e-14


def deposition_case():
    nc, ext = (24, 24, 16), (3e-3, 3e-3, 2e-3)
    hz = ext[2] / nc[2]
    top = 10 * hz
    geo = Geometry(dim=3, n_cells=nc, extent=ext, material_height=top, use_powder=True, powder_layer=2 * hz)
    seg = serpentine_segments(rng_for("deposition-gpu"), 0.6e-3, 2.4e-3, 1.0e-3, top, 4, 250e-6, 1.2)
    src = Source(type="goldak", depth=150e-6, absorption_efficiency=0.35, diameter=300e-6, max_power=400.0,
                 segments=seg)
    cfg = ThermalConfig(geometry=geo, material=phase_change_material(), boundary=Boundary.from_database(
        {"type": "adiabatic"}, 3), sources=[src], degree=2, time_method="rk_fourth_order")
    boxes = deposition_boxes(cfg, 50e-6, 50e-6, 250e-6, 0.0)
    return cfg, boxes


def test_deposition_run_matches_oracle():
    cfg, boxes = deposition_case()
    geo = cfg.geometry
    T0 = initial_temperature(cfg, "deposition-gpu")
    g = ThermalPhysics(cfg)
    dep = Deposition(g, boxes, deposition_time=1e-5)
    y = g.from_grid(T0)
    active = geo.active_cells().astype(bool)
    o = oracle_for(cfg, active.astype(np.uint8))
    y_ref = np.ascontiguousarray(T0, np.float64).reshape(-1).copy()
    h = [geo.extent[d] / geo.n_cells[d] for d in range(3)]
    dt, t = 2e-6, 0.0
    window_end = -1.0
    n_total = 0
    for step in range(40):
        # the driver's window (application/adamantine.hh:1134-1199)
        tol = dt * 1e-6
        n_dev = dep.step(t, dt, 320.0, y)
        if t - window_end > -tol:
            s = int(np.searchsorted(boxes.time, t - tol, side="left"))
            window_end = min(t + max(1e-5, dt), np.finfo(np.float64).max)
            e = int(np.searchsorted(boxes.time, window_end, side="left"))
            if s < e:
                cells, last = activate(active, boxes.lo, boxes.hi, s, e, geo.origin, h, geo.n_cells)
                assert n_dev == cells.size
                if cells.size:
                    o.activate_cells(cells, 320.0, y_ref, boxes.cos[last], boxes.sin[last])
                    active[cells] = True
                    n_total += cells.size
            else:
                assert n_dev == 0
        else:
            assert n_dev == 0
        t_ref = o.evolve_one_time_step(t, dt, y_ref)
        t = g.evolve_one_time_step(t, dt, y)
        assert t == t_ref
    assert n_total > 0
    act = o.node_active().astype(bool)
    assert rel_max(g.to_grid(y).reshape(-1)[act], y_ref[act]) <= STEP_TOL
    assert g.device_error() == 0


def test_device_path_equals_host_path():
    """The device activation and the host rebuild give the same state."""
    cfg, boxes = deposition_case()
    geo = cfg.geometry
    T0 = initial_temperature(cfg, "deposition-gpu")
    g1, g2 = ThermalPhysics(cfg), ThermalPhysics(cfg)
    y1, y2 = g1.from_grid(T0), g2.from_grid(T0)
    dep = Deposition(g1, boxes)
    active = geo.active_cells().astype(bool)
    h = [geo.extent[d] / geo.n_cells[d] for d in range(3)]
    n = dep.activate_range(0, 60, 330.0, y1)
    cells, last = activate(active, boxes.lo, boxes.hi, 0, 60, geo.origin, h, geo.n_cells)
    assert n == cells.size > 0
    g2.add_material(cells, 330.0, y2, boxes.cos[last], boxes.sin[last])
    assert torch.equal(y1, y2)
    assert torch.equal(g1.get_inverse_mass_matrix(), g2.get_inverse_mass_matrix())
    t = 0.0
    for _ in range(5):
        t1 = g1.evolve_one_time_step(t, 2e-6, y1)
        g2.evolve_one_time_step(t, 2e-6, y2)
        t = t1
    assert torch.equal(y1, y2)
    assert np.array_equal(g1.get_cell_state(), g2.get_cell_state())
