"""The reference's 3-D integration case demo_316_short_anisotropic.info
(tests/data of the reference; test_integration_3d.cc:112-115) as a
configuration of this package, and the driver loop of
application/adamantine.hh:1066-1285 for it on the CPU oracle -- test
infrastructure.

10 x 10 x 2 mm box (30 x 30 x 8 cells, Q2, Gauss), material up to 0.75 mm,
solid / powder / liquid with anisotropic conductivity (x 47.1 / 0.471 /
55.95, y and z 31.4 / 0.314 / 37.3 W/m/K), Goldak 400 W, absorption 0.3,
diameter 0.6 mm, depth 0.5 mm, along the scan path of
demo_316_short_scan_path.txt; deposition of 0.3 x 0.3 x 0.2 mm boxes with a
0.5 ms lead time; adiabatic; forward Euler, dt = 1e-5 s, duration 1 ms
(100 steps), new material at 300 K.
"""
import os

import numpy as np

from adamantine_b200.config import Boundary, Geometry, Material, Source, ThermalConfig

HERE = os.path.dirname(os.path.abspath(__file__))
DT, DURATION, NEW_T = 1e-5, 1e-3, 300.0
BOX = (0.3e-3, 0.2e-3, 0.3e-3, 0.5e-3)  # length, height, width, lead time


def demo_config():
    db = {"property_format": "polynomial", "n_materials": 1, "material_0.solidus": 1675.0,
          "material_0.liquidus": 1708.0, "material_0.latent_heat": 290000.0}
    for s, cp, k in (("solid", 714.0, (47.1, 31.4, 31.4)), ("powder", 714.0, (0.471, 0.314, 0.314)),
                     ("liquid", 847.0, (55.95, 37.3, 37.3))):
        db[f"material_0.{s}.density"] = 7904.0
        db[f"material_0.{s}.specific_heat"] = cp
        for ax, v in zip("xyz", k):
            db[f"material_0.{s}.thermal_conductivity_{ax}"] = v
    mat = Material.from_database(db, n_states=3)
    geo = Geometry(dim=3, n_cells=(30, 30, 8), extent=(10e-3, 10e-3, 2e-3), material_height=0.75e-3)
    seg = np.load(os.path.join(HERE, "golden", "integration_3d_scan_path.npy"))
    src = Source(type="goldak", depth=0.5e-3, absorption_efficiency=0.3, diameter=0.6e-3, max_power=400.0,
                 segments=seg)
    return ThermalConfig(geometry=geo, material=mat, boundary=Boundary.from_database({"type": "adiabatic"}, 3),
                         sources=[src], degree=2, time_method="forward_euler")


# demo_316_short.info (test_integration_3d.cc:117-120): the same path and
# deposition on 50 x 50 x 8 FE_Q(3) cells, isotropic conductivity (31.4 /
# 0.314 / 37.3 W/m/K), convective (h = 100 W/m^2/K) and radiative
# (emissivity 0.15) faces to 300 K, forward Euler dt = 6e-5 s to 4 ms.
SHORT_DT, SHORT_DURATION = 0.6e-4, 0.004


def demo_short_config():
    db = {"property_format": "polynomial", "n_materials": 1, "material_0.solidus": 1675.0,
          "material_0.liquidus": 1708.0, "material_0.latent_heat": 290000.0,
          "material_0.radiation_temperature_infty": 300.0, "material_0.convection_temperature_infty": 300.0}
    for s, cp, k in (("solid", 714.0, 31.4), ("powder", 714.0, 0.314), ("liquid", 847.0, 37.3)):
        db[f"material_0.{s}.density"] = 7904.0
        db[f"material_0.{s}.specific_heat"] = cp
        for ax in "xyz":
            db[f"material_0.{s}.thermal_conductivity_{ax}"] = k
        db[f"material_0.{s}.convection_heat_transfer_coef"] = 100.0
        db[f"material_0.{s}.emissivity"] = 0.15
    mat = Material.from_database(db, n_states=3)
    geo = Geometry(dim=3, n_cells=(50, 50, 8), extent=(10e-3, 10e-3, 2e-3), material_height=0.75e-3)
    seg = np.load(os.path.join(HERE, "golden", "integration_3d_scan_path.npy"))
    src = Source(type="goldak", depth=0.5e-3, absorption_efficiency=0.3, diameter=0.6e-3, max_power=400.0,
                 segments=seg)
    bnd = Boundary.from_database({"type": "convective,radiative"}, 3)
    return ThermalConfig(geometry=geo, material=mat, boundary=bnd, sources=[src], degree=3,
                         time_method="forward_euler")


def gold_text():
    return open(os.path.join(HERE, "golden", "integration_3d_gold.txt")).read().split()


def gold_short():
    return np.load(os.path.join(HERE, "golden", "integration_3d_gold_short.npz"))["values"].astype(np.float64)


def driver_dt(t, dt, duration):
    """The driver's step at time t: dt, cut so that the run ends at the
    duration (application/adamantine.hh:1110-1111)."""
    return duration - t if t + dt > duration else dt


def run_oracle(cfg, boxes, dt=DT, duration=DURATION):
    """The driver loop on the oracle (application/adamantine.hh:1063-1285):
    while t < duration, the step is cut to end at the duration
    (:1110-1111), then the deposition window, then one step. Returns (field,
    active cells, number of steps, oracle)."""
    import oracle_py
    from deposition_oracle import activate

    geo = cfg.geometry
    active = geo.active_cells().astype(bool)
    st = cfg.to_struct()
    o = oracle_py.Oracle(st, active=active.astype(np.uint8), initial_state=geo.initial_state())
    o._keep = st
    y = np.full(int(np.prod(geo.node_shape(cfg.degree))), 300.0)
    h = [geo.extent[d] / geo.n_cells[d] for d in range(3)]
    t, window_end, n = 0.0, -1.0, 0
    while t < duration:
        dt = driver_dt(t, dt, duration)
        tol = dt * 1e-6
        if t - window_end > -tol:
            s = int(np.searchsorted(boxes.time, t - tol, side="left"))
            window_end = min(t + max(0.0, dt), duration)  # geometry.deposition_time: 0
            e = int(np.searchsorted(boxes.time, window_end, side="left"))
            if s < e:
                cells, last = activate(active, boxes.lo, boxes.hi, s, e, geo.origin, h, geo.n_cells)
                if cells.size:
                    o.activate_cells(cells, NEW_T, y, boxes.cos[last], boxes.sin[last])
                    active[cells] = True
        t = o.evolve_one_time_step(t, dt, y)
        n += 1
    return y, active, n, o
