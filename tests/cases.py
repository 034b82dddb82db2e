"""Problem builders shared by the tests (test infrastructure).

Each builder restates one set-up of the reference's own tests, or one of the
synthetic workloads the benchmark uses, as a ThermalConfig.
"""
from __future__ import annotations

import os
import zlib

import numpy as np

from adamantine_b200.config import Boundary, Geometry, Material, Source, ThermalConfig, parse_scan_path

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

# tests/data/scan_path.txt of the reference, restated as segment rows
SCAN_PATH_TXT = """Number of path segments
2
Mode    x       y     z   pmod    param
1       0.000   0.1  0.1   0       1e-6
0       0.002   0.1  0.1   1       0.8
"""

# tests/data/scan_path_test_thermal_physics.txt of the reference
SCAN_PATH_THERMAL_PHYSICS_TXT = """Number of path segments
2
Mode    x       y     z   pmod    param
1       0.000   0.000  0   1.0       1e-15
0       1.0   0.000  0     1.0       1.0
"""


def unit_slp_material(k=(1.0, 1.0, 1.0), p_order=2, extra=None):
    db = {"property_format": "polynomial", "n_materials": 1}
    for s in ("solid", "powder", "liquid"):
        db[f"material_0.{s}.density"] = 1.0
        db[f"material_0.{s}.specific_heat"] = 1.0
        db[f"material_0.{s}.thermal_conductivity_x"] = k[0]
        if k[1] is not None:
            db[f"material_0.{s}.thermal_conductivity_y"] = k[1]
        db[f"material_0.{s}.thermal_conductivity_z"] = k[2]
    if extra:
        db.update(extra)
    return Material.from_database(db, n_states=3, p_order=p_order)


def zero_power_goldak(depth=0.1, diameter=1.0):
    return Source(type="goldak", depth=depth, absorption_efficiency=0.1, diameter=diameter, max_power=0.0,
                  segments=parse_scan_path(SCAN_PATH_TXT))


def operator_2d_case(material, boundary="adiabatic"):
    """test_thermal_operator.cc: 2D 12x6, 4x5 cells, FE_Q(2), QGauss(3)."""
    geo = Geometry(dim=2, n_cells=(4, 5), extent=(12.0, 6.0))
    return ThermalConfig(geometry=geo, material=material,
                         boundary=Boundary.from_database({"type": boundary}, 2),
                         sources=[zero_power_goldak()], degree=2)


# --------------------------------------------------------------------------
# Synthetic workloads (seeded); sizes named by what they are
# --------------------------------------------------------------------------
SEED = 20261203


def seeded_rng(name: str, seed: int = SEED):
    return np.random.default_rng([seed, zlib.crc32(name.encode())])


def steel_solid_material():
    """Solid only: rho 7904 kg/m^3, c_p 714 J/kg/K, k 31.4 W/m/K; h_conv 10 on top."""
    db = {
        "property_format": "polynomial",
        "n_materials": 1,
        "material_0.solid.density": 7904.0,
        "material_0.solid.specific_heat": 714.0,
        "material_0.solid.thermal_conductivity_x": 31.4,
        "material_0.solid.thermal_conductivity_y": 31.4,
        "material_0.solid.thermal_conductivity_z": 31.4,
        "material_0.solid.convection_heat_transfer_coef": 10.0,
        "material_0.convection_temperature_infty": 300.0,
    }
    return Material.from_database(db, n_states=1, p_order=0)


def phase_change_material(rng=None, k_scale=1.0, cp_scale=1.0):
    """Three states, solidus 1648 K, liquidus 1673 K, latent heat 2.9e5 J/kg.

    k_solid(T) is a seeded quadratic with k(300)=10 and k(1700)=35 (monotone),
    k_powder = 0.5% k_solid, k_liquid = 35; c_p is a seeded linear function;
    rho = 7904 for every state.
    """
    rng = rng or seeded_rng("phase_change_material")
    # quadratic through (300,10), (1700,35) with a seeded curvature that keeps
    # it monotone on [300, 1700]
    t0, t1 = 300.0, 1700.0
    c = rng.uniform(-5e-6, 5e-6)
    b = (35.0 - 10.0) / (t1 - t0) - c * (t0 + t1)
    a = 10.0 - b * t0 - c * t0 * t0
    cp0 = rng.uniform(440.0, 480.0)
    cp1 = rng.uniform(0.15, 0.25)
    ks = np.array([a, b, c]) * k_scale
    db = {"property_format": "polynomial", "n_materials": 1,
          "material_0.solidus": 1648.0, "material_0.liquidus": 1673.0, "material_0.latent_heat": 2.9e5}
    for s, kk in (("solid", ks), ("powder", 0.005 * ks), ("liquid", np.array([35.0 * k_scale, 0.0, 0.0]))):
        db[f"material_0.{s}.density"] = 7904.0
        db[f"material_0.{s}.specific_heat"] = f"{cp0 * cp_scale!r}, {cp1 * cp_scale!r}"
        for ax in ("x", "y", "z"):
            db[f"material_0.{s}.thermal_conductivity_{ax}"] = ", ".join(repr(float(v)) for v in kk)
    return Material.from_database(db, n_states=3, p_order=2)


def serpentine_segments(rng, x0, x1, y0, z, n_passes, hatch, speed, power_mod=1.0):
    """Seeded serpentine scan path rows (end_time, pmod, x, y, z)."""
    jitter = rng.uniform(-0.1, 0.1) * hatch
    rows = [[1e-9, 0.0, x0, y0 + jitter, z]]
    t = rows[0][0]
    x, y = x0, y0 + jitter
    for p in range(n_passes):
        xe = x1 if p % 2 == 0 else x0
        t += abs(xe - x) / speed
        rows.append([t, power_mod, xe, y, z])
        x = xe
        if p + 1 < n_passes:
            y2 = y + hatch
            t += hatch / speed
            rows.append([t, 0.0, x, y2, z])
            y = y2
    return np.array(rows)
