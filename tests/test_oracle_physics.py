"""Pins the oracle's time stepping against tests/test_thermal_physics.hh of the
reference, including the convective-boundary gold file."""
import os

import numpy as np
import pytest

import oracle_py
from adamantine_b200.config import Boundary, Geometry, Material, Source, ThermalConfig, parse_scan_path
from cases import GOLDEN, SCAN_PATH_THERMAL_PHYSICS_TXT, unit_slp_material
from dealii_order import dof_to_node


def build(cfg, **kw):
    st = cfg.to_struct()
    o = oracle_py.Oracle(st, active=cfg.geometry.active_cells(), initial_state=cfg.geometry.initial_state(), **kw)
    o._keep = st
    return o


def uniform_eb(absorption):
    return Source(type="electron_beam", depth=1e100, absorption_efficiency=absorption, diameter=1e100,
                  max_power=1e300, segments=parse_scan_path(SCAN_PATH_THERMAL_PHYSICS_TXT))


def test_thermal_2d_explicit():
    """thermal_2d_explicit_host (test_thermal_physics.hh:77-155): l2 0.291705 @1e-3."""
    geo = Geometry(dim=2, n_cells=(4, 5), extent=(12e-3, 6e-3))
    cfg = ThermalConfig(geometry=geo, material=unit_slp_material(k=(1.0, None, 1.0), p_order=2),
                        boundary=Boundary.from_database({"type": "adiabatic"}, 2), sources=[uniform_eb(0.1)],
                        degree=2, time_method="forward_euler")
    o = build(cfg)
    y = np.zeros(o.n_nodes)
    t = 0.0
    while t < 0.1:
        t = o.evolve_one_time_step(t, 0.05, y)
    assert abs(t - 0.1) / 0.1 < 1e-3
    assert abs(np.linalg.norm(y) - 0.291705) / 0.291705 < 1e-3


def test_thermal_2d_manufactured_solution():
    """thermal_2d_manufactured_solution (test_thermal_physics.hh:157-248):
    one RK4 step of 0.1 gives 0.1 everywhere @1e-5."""
    geo = Geometry(dim=2, n_cells=(4, 5), extent=(1e3, 6e3))
    cfg = ThermalConfig(geometry=geo, material=unit_slp_material(k=(1.0, None, 1.0), p_order=1),
                        boundary=Boundary.from_database({"type": "adiabatic"}, 2),
                        sources=[uniform_eb(0.1 / 0.29317423955177113)], degree=2, time_method="rk_fourth_order")
    o = build(cfg)
    y = np.zeros(o.n_nodes)
    t = o.evolve_one_time_step(0.0, 0.1, y)
    assert t == 0.1
    assert np.max(np.abs(y - 0.1) / 0.1) < 1e-5


def test_energy_conservation():
    """energy_conservation (test_thermal_physics.hh:287-393): cube source,
    forward Euler to t=100, mean 10.5 and min == max @1e-9."""
    geo = Geometry(dim=2, n_cells=(10, 10), extent=(10.0, 10.0))
    db = {"property_format": "polynomial", "n_materials": 1}
    for s in ("solid", "powder", "liquid"):
        db[f"material_0.{s}.density"] = 0.5
        db[f"material_0.{s}.specific_heat"] = 4.0
        db[f"material_0.{s}.thermal_conductivity_x"] = 2.0
        db[f"material_0.{s}.thermal_conductivity_z"] = 2.0
    mat = Material.from_database(db, n_states=3, p_order=0)
    cube = Source(type="cube", cube_start_time=0.0, cube_end_time=5.0, cube_value=5.0,
                  cube_min=(4.0, 4.0, 0.0), cube_max=(6.0, 6.0, 0.0))
    cfg = ThermalConfig(geometry=geo, material=mat, boundary=Boundary.from_database({"type": "adiabatic"}, 2),
                        sources=[cube], degree=2, time_method="forward_euler")
    o = build(cfg)
    y = np.full(o.n_nodes, 10.0)
    t = 0.0
    while t < 100:
        t = o.evolve_one_time_step(t, 0.05, y)
    assert abs(y.mean() - 10.5) / 10.5 < 1e-9
    assert abs(y.min() - y.max()) / y.max() < 1e-9


def test_radiation_bcs():
    """radiation_bcs (test_thermal_physics.hh:395-510): 10 <= T <= 20."""
    geo = Geometry(dim=2, n_cells=(5, 5), extent=(5.0, 5.0))
    db = {"property_format": "polynomial", "n_materials": 1,
          "material_0.radiation_temperature_infty": 20.0, "material_0.convection_temperature_infty": 0.0}
    for s in ("solid", "powder", "liquid"):
        for p, v in (("density", 1.0), ("specific_heat", 1.0), ("thermal_conductivity_x", 1.0),
                     ("thermal_conductivity_z", 1.0), ("emissivity", 1.0), ("radiation_heat_transfer_coef", 1.0),
                     ("convection_heat_transfer_coef", 1.0)):
            db[f"material_0.{s}.{p}"] = v
    mat = Material.from_database(db, n_states=3, p_order=1)
    cfg = ThermalConfig(geometry=geo, material=mat, boundary=Boundary.from_database({"type": "radiative"}, 2),
                        sources=[], degree=2, time_method="forward_euler")
    o = build(cfg)
    y = np.full(o.n_nodes, 10.0)
    t = 0.0
    while t < 100:
        t = o.evolve_one_time_step(t, 0.05, y)
    assert 10.0 <= y.min() <= 20.0
    assert 10.0 < y.max() <= 20.0


def convective_case():
    geo = Geometry(dim=3, n_cells=(100, 1, 1), extent=(0.1, 0.1, 0.1))
    db = {"property_format": "polynomial", "n_materials": 1,
          "material_0.radiation_temperature_infty": 0.0, "material_0.convection_temperature_infty": 300.0}
    for s in ("solid", "powder", "liquid"):
        for p, v in (("density", 100.0), ("specific_heat", 100.0), ("thermal_conductivity_x", 1.0),
                     ("thermal_conductivity_z", 1.0), ("emissivity", 1.0),
                     ("convection_heat_transfer_coef", 50.0)):
            db[f"material_0.{s}.{p}"] = v
    mat = Material.from_database(db, n_states=3, p_order=0)
    bnd = Boundary.from_database({"type": "adiabatic", "boundary_1.type": "convective"}, 3)
    return ThermalConfig(geometry=geo, material=mat, boundary=bnd, sources=[], degree=2,
                         time_method="forward_euler")


def test_convective_bc_gold():
    """convection_bcs (test_thermal_physics.hh:512-624): 1809 nodal values of
    tests/data/convective_bc_gold.txt (deal.II DoF order) @1e-6."""
    gold = np.load(os.path.join(GOLDEN, "convective_bc_gold.npy"))
    cfg = convective_case()
    o = build(cfg)
    y = np.full(o.n_nodes, 400.0)
    t = 0.0
    while t < 1.0:
        t = o.evolve_one_time_step(t, 2.5e-4, y)
    order = dof_to_node(3, (100, 1, 1), 2)
    assert order.size == gold.size == 1809
    assert np.max(np.abs(y[order] - gold) / np.abs(gold)) < 1e-6


def test_has_melted():
    """reference_temperature (test_thermal_physics.hh:626-701)."""
    geo = Geometry(dim=2, n_cells=(1, 1), extent=(12e-3, 6e-3))
    mat = unit_slp_material(k=(1.0, None, 1.0), p_order=1)
    cfg = ThermalConfig(geometry=geo, material=mat, boundary=Boundary.from_database({"type": "adiabatic"}, 2),
                        sources=[], degree=2)
    o = build(cfg)
    y = np.full(o.n_nodes, 1000.0)
    assert not o.mark_has_melted(1500.0, y).any()
    y[:] = 1600.0
    assert o.mark_has_melted(1500.0, y).all()
    y[:] = 1100.0
    assert o.mark_has_melted(1500.0, y).all()
