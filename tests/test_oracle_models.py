"""Pins the oracle's heat sources and material model against the reference's
known answers (tests/test_heat_source.cc, tests/test_material_property.hh)."""
import math

import numpy as np
import pytest

import oracle_py
from adamantine_b200.config import Boundary, Geometry, Material, Source, ThermalConfig, parse_scan_path
from cases import SCAN_PATH_TXT


def rel(a, b):
    return abs(a - b) / max(abs(b), 1e-300)


def source_oracle(dim, beam_type):
    geo = Geometry(dim=dim, n_cells=(1, 1, 1)[:dim], extent=(1.0, 1.0, 1.0)[:dim])
    src = Source(type=beam_type, depth=0.1, absorption_efficiency=0.1, diameter=1.0, max_power=10.0,
                 segments=parse_scan_path(SCAN_PATH_TXT))
    mat = Material.from_database({"material_0.solid.density": 1.0, "material_0.solid.specific_heat": 1.0}, 1)
    cfg = ThermalConfig(geometry=geo, material=mat, boundary=Boundary.from_database({"type": "adiabatic"}, dim),
                        sources=[src], degree=1)
    st = cfg.to_struct()
    o = oracle_py.Oracle(st)
    o._keep = st
    return o


GOLDAK_CENTER = 2.0 * 0.1 * 10.0 / (0.5 * 0.5 * 0.1 * math.pow(math.pi / 3.0, 1.5))
GOLDAK_OFF = GOLDAK_CENTER * math.exp(-3.0 * 1.0e-4 * 1.0e-4 / 0.25 - 3.0 * 0.01 * 0.01 / 0.1 / 0.1)
EB_CENTER = -0.1 * 10.0 * 1.0 * math.log(0.1) / (math.pi * 0.5 * 0.5 * 0.1)
EB_OFF = EB_CENTER * math.exp(math.log(0.1) * 1.0e-4 * 1.0e-4 / 0.25) * (
    -3.0 * 0.01 * 0.01 / 0.1 / 0.1 + 2.0 * 0.01 / 0.1 + 1.0)


@pytest.mark.parametrize("dim", [2, 3])
@pytest.mark.parametrize("beam", ["goldak", "electron_beam"])
def test_heat_source_values(dim, beam):
    """heat_source_value_2d/3d (test_heat_source.cc:19-300) @1e-12."""
    o = source_oracle(dim, beam)
    pts = {
        2: [(0.0, 0.05), (10.0, 0.0), (8.0e-4, 0.1), (7.0e-4, 0.09)],
        3: [(0.0, 0.0, 0.05), (10.0, 0.0, 0.0), (8e-4, 0.1, 0.1), (7.0e-4, 0.1, 0.09)],
    }[dim]
    o.set_time(1.0e-7)
    assert o.source_values(0, [pts[0]])[0] == 0.0
    o.set_time(5.0e-7)
    assert o.source_values(0, [pts[1]])[0] == 0.0
    o.set_time(0.001001)
    center, off = (GOLDAK_CENTER, GOLDAK_OFF) if beam == "goldak" else (EB_CENTER, EB_OFF)
    v = o.source_values(0, [pts[2], pts[3]])
    assert rel(v[0], center) < 1e-12
    assert rel(v[1], off) < 1e-12
    o.set_time(100.0)
    assert o.source_values(0, [pts[3]])[0] == 0.0
    assert o.source_state(0)[4] == 0.0  # power off after the path


def test_heat_source_far_lanes_are_zero():
    """heat_source_vectorized_value_*: points far away evaluate to zero."""
    o = source_oracle(3, "goldak")
    o.set_time(0.001001)
    assert o.source_values(0, [(-1e10, -1e10, -1e10)])[0] == 0.0


def material_oracle(db, n_states, p_order, matid, user_index, T):
    geo = Geometry(dim=2, n_cells=(4, 5), extent=(12.0, 6.0))
    mat = Material.from_database(db, n_states=n_states, p_order=p_order)
    cfg = ThermalConfig(geometry=geo, material=mat, boundary=Boundary.from_database({"type": "adiabatic"}, 2),
                        degree=4 if False else 1)
    st = cfg.to_struct()
    o = oracle_py.Oracle(st, material_id=matid, initial_state=user_index)
    o._keep = st
    pv = o.evaluate_material_properties(np.full(o.n_nodes, T))
    return o, pv


TABLE_DB = {
    "property_format": "table",
    "n_materials": 2,
    "material_0.solid.density": "0.,1.",
    "material_0.solid.thermal_conductivity_x": "0.,10.|10.,100.",
    "material_0.solid.thermal_conductivity_z": "0.,10.|10.,100.",
    "material_1.solid.density": "0.,1.|20.,2.|30.,3.",
    "material_1.solid.thermal_conductivity_x": "0.,10.|10.,100.|20.,200.",
    "material_1.solid.thermal_conductivity_z": "0.,10.|10.,100.|20.,200.",
    "material_1.powder.density": "0.,1.|15.,2.|30.,3.",
    "material_1.powder.thermal_conductivity_x": "0.,10.|10.,100.|18.,200.",
    "material_1.powder.thermal_conductivity_z": "0.,10.|10.,100.|18.,200.",
}
POLY_DB = {
    "property_format": "polynomial",
    "n_materials": 2,
    "material_0.solid.density": "0.,1.",
    "material_0.solid.thermal_conductivity_x": "0.,1.,2.",
    "material_0.solid.thermal_conductivity_z": "0.,1.,2.",
    "material_1.solid.density": "1.,2.,3.",
    "material_1.solid.thermal_conductivity_x": "1.,100.,20.,200.",
    "material_1.solid.thermal_conductivity_z": "1.,100.,20.,200.",
    "material_1.powder.density": "15.,2.,3.",
    "material_1.powder.thermal_conductivity_x": "10.,18.,200.",
    "material_1.powder.thermal_conductivity_z": "10.,18.,200.",
}


@pytest.mark.parametrize("db,expected,p_order", [
    (TABLE_DB, [(1.0, 100.0), (1.75, 150.0), (2.0, 162.5)], 0),
    (POLY_DB, [(15.0, 465.0), (706.0, 681001.0), (720.0, 45280.0)], 4),
])
def test_material_property_table_and_polynomial(db, expected, p_order):
    """material_property_table / material_property_polynomials
    (test_material_property.hh:264-468) @1e-10 at T = 15."""
    n = np.arange(20)
    matid = np.where(n < 10, 0, 1).astype(np.uint8)
    user = np.where(n < 15, 0, 2).astype(np.uint8)
    o, pv = material_oracle(db, 3, p_order, matid, user, 15.0)
    for c in range(20):
        k = 0 if c < 10 else (1 if c < 15 else 2)
        rho, kx = expected[k]
        assert rel(pv[0, c], rho) < 1e-10
        assert rel(pv[2, c], kx) < 1e-10
        assert rel(pv[4, c], kx) < 1e-10


def test_material_ratios():
    """ratios (test_material_property.hh:92-260): powder -> liquid -> solid."""
    db = {"property_format": "polynomial", "n_materials": 1,
          "material_0.solid.density": 10.0, "material_0.solid.thermal_conductivity_x": 10.0,
          "material_0.solid.thermal_conductivity_z": 10.0, "material_0.solid.specific_heat": 10.0,
          "material_0.powder.density": 1.0, "material_0.powder.thermal_conductivity_x": 1.0,
          "material_0.powder.thermal_conductivity_z": 1.0, "material_0.powder.specific_heat": 1.0,
          "material_0.liquid.density": 1.0, "material_0.liquid.thermal_conductivity_x": 20.0,
          "material_0.liquid.thermal_conductivity_z": 20.0, "material_0.liquid.specific_heat": 20.0,
          "material_0.solidus": 50.0, "material_0.liquidus": 100.0, "material_0.latent_heat": 1000.0}
    user = np.full(20, 2, np.uint8)
    o, pv = material_oracle(db, 3, 0, None, user, 0.0)
    st = o.cell_state()
    assert np.all(st[2] == 1.0) and np.all(st[0] == 0.0) and np.all(st[1] == 0.0)
    assert np.all(pv[0] == 1.0) and np.all(pv[2] == 1.0) and np.all(pv[1] == 1.0)
    pv = o.evaluate_material_properties(np.full(o.n_nodes, 100000.0))
    st = o.cell_state()
    assert np.all(st[2] == 0.0) and np.all(st[0] == 0.0) and np.all(st[1] == 1.0)
    assert np.all(pv[0] == 1.0) and np.all(pv[2] == 20.0) and np.all(pv[1] == 20.0)
    pv = o.evaluate_material_properties(np.zeros(o.n_nodes))
    st = o.cell_state()
    assert np.all(st[2] == 0.0) and np.all(st[0] == 1.0) and np.all(st[1] == 0.0)
    assert np.all(pv[0] == 10.0) and np.all(pv[2] == 10.0) and np.all(pv[1] == 10.0)


def test_scan_path_segments():
    """ScanPath::load_segment_scan_path on tests/data/scan_path.txt: a point
    then a 2 mm line at 0.8 m/s."""
    seg = parse_scan_path(SCAN_PATH_TXT)
    assert seg.shape == (2, 5)
    assert seg[0, 0] == 1e-6 and seg[0, 1] == 0.0
    assert rel(seg[1, 0], 1e-6 + 0.002 / 0.8) < 1e-15
    assert list(seg[1, 2:]) == [0.002, 0.1, 0.1]
