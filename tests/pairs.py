"""Builds matching (CUDA library, CPU oracle) pairs for the parity tests --
test infrastructure.  Small seeded 3D problems that exercise every branch of
the operator: Q1/Q2, one to three material states, tables, several
materials, deposition angles, partial activation, Goldak / electron-beam /
cube sources and convective / radiative faces.
"""
from __future__ import annotations

import numpy as np

import oracle_py
from adamantine_b200.config import Boundary, Geometry, Material, Source, ThermalConfig
from cases import phase_change_material, seeded_rng, steel_solid_material


def rel_max(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def line_path(x0, x1, y, z, speed, t0=1e-9):
    """Point then one line along +x."""
    return np.array([[t0, 0.0, x0, y, z], [t0 + abs(x1 - x0) / speed, 1.0, x1, y, z]])


def two_state_material():
    db = {"property_format": "polynomial", "n_materials": 1, "material_0.solidus": 1600.0,
          "material_0.liquidus": 1650.0, "material_0.latent_heat": 2.5e5,
          "material_0.radiation_temperature_infty": 295.0, "material_0.convection_temperature_infty": 300.0}
    for s, k in (("solid", "20.0, 0.01"), ("liquid", "30.0, 0.0")):
        db[f"material_0.{s}.density"] = "7800.0, -0.1"
        db[f"material_0.{s}.specific_heat"] = "450.0, 0.2"
        db[f"material_0.{s}.thermal_conductivity_x"] = k
        db[f"material_0.{s}.thermal_conductivity_y"] = k
        db[f"material_0.{s}.thermal_conductivity_z"] = k
        db[f"material_0.{s}.emissivity"] = "0.4, 1e-4"
        db[f"material_0.{s}.convection_heat_transfer_coef"] = "10.0, 0.01"
    return Material.from_database(db, n_states=2, p_order=1)


def table_material():
    db = {"property_format": "table", "n_materials": 2}
    for m, scale in ((0, 1.0), (1, 1.3)):
        db[f"material_{m}.solidus"] = 1500.0
        db[f"material_{m}.liquidus"] = 1560.0
        db[f"material_{m}.latent_heat"] = 2.0e5
        for s in ("solid", "liquid", "powder"):
            f = {"solid": 1.0, "liquid": 1.2, "powder": 0.05}[s] * scale
            db[f"material_{m}.{s}.density"] = "300,7900|1000,7700|1700,7500"
            db[f"material_{m}.{s}.specific_heat"] = "300,480|900,600|1500,700|1800,760"
            db[f"material_{m}.{s}.thermal_conductivity_x"] = f"300,{15 * f}|800,{22 * f}|1600,{31 * f}"
            db[f"material_{m}.{s}.thermal_conductivity_y"] = f"300,{12 * f}|800,{18 * f}|1600,{26 * f}"
            db[f"material_{m}.{s}.thermal_conductivity_z"] = f"300,{14 * f}|800,{20 * f}|1600,{29 * f}"
    return Material.from_database(db, n_states=3)


def make_case(name):
    """Returns (ThermalConfig, cell arrays dict, initial temperature grid)."""
    rng = seeded_rng("parity-" + name)
    cells = {}
    if name == "q1_solid_convective_goldak":
        # 3D steel box, convective top, a Goldak beam resolved by the mesh
        geo = Geometry(dim=3, n_cells=(12, 10, 6), extent=(6e-3, 5e-3, 3e-3))
        bnd = Boundary.from_database({"type": "adiabatic", "boundary_5.type": "convective"}, 3)
        src = Source(type="goldak", depth=6e-4, absorption_efficiency=0.3, diameter=1.2e-3, max_power=200.0,
                     segments=line_path(1e-3, 5e-3, 2.5e-3, 3e-3, 1.0))
        cfg = ThermalConfig(geometry=geo, material=steel_solid_material(), boundary=bnd, sources=[src], degree=1,
                            time_method="forward_euler")
        T = 300.0 + rng.uniform(-1.0, 1.0, geo.node_shape(1)[::-1])
    elif name == "q2_slp_goldak":
        geo = Geometry(dim=3, n_cells=(10, 9, 8), extent=(2e-3, 1.8e-3, 1.6e-3), material_height=1.6e-3,
                       use_powder=True, powder_layer=0.6e-3)
        bnd = Boundary.from_database({"type": "adiabatic"}, 3)
        src = Source(type="goldak", depth=3e-4, absorption_efficiency=0.35, diameter=5e-4, max_power=400.0,
                     segments=line_path(0.4e-3, 1.6e-3, 0.9e-3, 1.6e-3, 1.0))
        cfg = ThermalConfig(geometry=geo, material=phase_change_material(), boundary=bnd, sources=[src], degree=2,
                            time_method="rk_fourth_order")
        T = hot_field(geo, 2, rng, peak=2100.0)
    elif name == "q2_sl_eb_faces":
        geo = Geometry(dim=3, n_cells=(9, 8, 6), extent=(1.8e-3, 1.6e-3, 1.2e-3))
        bnd = Boundary.from_database({"type": "adiabatic", "boundary_5.type": "radiative,convective",
                                      "boundary_1.type": "convective"}, 3)
        src = Source(type="electron_beam", depth=2e-4, absorption_efficiency=0.8, diameter=4e-4, max_power=500.0,
                     segments=line_path(0.3e-3, 1.5e-3, 0.8e-3, 1.2e-3, 0.8))
        cfg = ThermalConfig(geometry=geo, material=two_state_material(), boundary=bnd, sources=[src], degree=2,
                            time_method="rk_third_order")
        T = hot_field(geo, 2, rng, peak=1900.0)
    elif name == "q1_table_rotation":
        geo = Geometry(dim=3, n_cells=(14, 12, 8), extent=(2.8e-3, 2.4e-3, 1.6e-3), material_height=1.6e-3,
                       use_powder=True, powder_layer=0.4e-3)
        bnd = Boundary.from_database({"type": "adiabatic"}, 3)
        src = Source(type="goldak", depth=2e-4, absorption_efficiency=0.3, diameter=4e-4, max_power=300.0,
                     segments=line_path(0.5e-3, 2.3e-3, 1.2e-3, 1.6e-3, 1.2))
        cfg = ThermalConfig(geometry=geo, material=table_material(), boundary=bnd, sources=[src], degree=1,
                            time_method="rk_second_order")
        C = geo.n_cells_total
        ang = rng.uniform(0, np.pi, C)
        cells = {"material_id": (rng.uniform(size=C) < 0.3).astype(np.uint8),
                 "deposition_cos": np.cos(ang), "deposition_sin": np.sin(ang)}
        T = hot_field(geo, 1, rng, peak=1700.0)
    elif name == "q2_slp_partial_faces_cube":
        # part of the box is FE_Nothing: interfaces take the printed-surface type
        geo = Geometry(dim=3, n_cells=(8, 8, 10), extent=(1.6e-3, 1.6e-3, 2.0e-3), material_height=1.5e-3,
                       use_powder=True, powder_layer=0.4e-3)
        bnd = Boundary.from_database({"type": "adiabatic", "printed_surface.type": "radiative,convective"}, 3)
        mat = phase_change_material()
        mat.props[0, 3] = 300.0  # radiation_temperature_infty
        mat.props[0, 4] = 300.0  # convection_temperature_infty
        mat.poly[0, 5, :3, 0] = 0.3   # emissivity
        mat.poly[0, 7, :3, 0] = 25.0  # convection coefficient
        cube = Source(type="cube", cube_start_time=0.0, cube_end_time=1.0, cube_value=2e12,
                      cube_min=(0.4e-3, 0.4e-3, 1.0e-3), cube_max=(1.0e-3, 1.2e-3, 1.5e-3))
        cfg = ThermalConfig(geometry=geo, material=mat, boundary=bnd, sources=[cube], degree=2,
                            time_method="rk_fourth_order")
        T = hot_field(geo, 2, rng, peak=1800.0)
    else:
        raise KeyError(name)
    return cfg, cells, T


def hot_field(geo, degree, rng, peak):
    """300 K plus a seeded Gaussian hot spot near the top that crosses the
    solidus and liquidus, plus +/-1 K noise."""
    shape = geo.node_shape(degree)[::-1]  # (nz, ny, nx)
    zs = np.linspace(0, geo.extent[2], shape[0])
    ys = np.linspace(0, geo.extent[1], shape[1])
    xs = np.linspace(0, geo.extent[0], shape[2])
    Z, Y, X = np.meshgrid(zs, ys, xs, indexing="ij")
    cx, cy = geo.extent[0] * rng.uniform(0.3, 0.7), geo.extent[1] * rng.uniform(0.3, 0.7)
    top = min(geo.material_height, geo.extent[2])
    r2 = (X - cx) ** 2 + (Y - cy) ** 2 + (Z - top) ** 2
    w = 0.25 * min(geo.extent[:2])
    return 300.0 + (peak - 300.0) * np.exp(-r2 / w ** 2) + rng.uniform(-1.0, 1.0, shape)


CASES = ["q1_solid_convective_goldak", "q2_slp_goldak", "q2_sl_eb_faces", "q1_table_rotation",
         "q2_slp_partial_faces_cube"]


def make_oracle(cfg, cells):
    st = cfg.to_struct()
    geo = cfg.geometry
    o = oracle_py.Oracle(st, active=geo.active_cells(), initial_state=geo.initial_state(),
                         material_id=cells.get("material_id"), deposition_cos=cells.get("deposition_cos"),
                         deposition_sin=cells.get("deposition_sin"))
    o._keep = st
    return o


def make_gpu(cfg, cells):
    from adamantine_b200.thermal import ThermalPhysics

    return ThermalPhysics(cfg, material_id=cells.get("material_id"), deposition_cos=cells.get("deposition_cos"),
                          deposition_sin=cells.get("deposition_sin"))
