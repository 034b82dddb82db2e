"""Refined-mesh cases of the tests: the reference's amr_test.info
(test_integration_3d_amr.cc:19-58) and variants -- test infrastructure."""
import os

import numpy as np

from adamantine_b200.config import Boundary, Geometry, Material, Source, ThermalConfig

HERE = os.path.dirname(os.path.abspath(__file__))

# amr_test.info: forward Euler, 1 us steps to 250 us, refinement every 200
# steps (and before the first), one level; expected max / min of the
# temperature after the run (tolerance 10 % in the reference's test).
AMR_DT, AMR_DURATION, AMR_EVERY, AMR_MAX, AMR_MIN = 1e-6, 25e-5, 200, 329.5, 296.1


def amr_test_config(degree=3, n_cells=(4, 4, 1), boundary="adiabatic", method="forward_euler", n_states=3,
                    max_power=400.0):
    """5 x 5 x 0.5 mm plate (x length, y width, z height), solid / powder /
    liquid 316L-like properties, Goldak 400 W beam (absorption 0.3, 0.6 mm
    diameter, 0.25 mm depth) along bare_plate_L_scan_path_fast.txt."""
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
    mat = Material.from_database(db, n_states=n_states)
    geo = Geometry(dim=3, n_cells=n_cells, extent=(5e-3, 5e-3, 0.5e-3))
    seg = np.load(os.path.join(HERE, "golden", "amr_test_scan_path.npy"))
    src = Source(type="goldak", depth=0.25e-3, absorption_efficiency=0.3, diameter=0.6e-3, max_power=max_power,
                 segments=seg)
    return ThermalConfig(geometry=geo, material=mat, boundary=Boundary.from_database({"type": boundary}, 3),
                         sources=[src], degree=degree, time_method=method)


def run_amr(problem, dt=AMR_DT, duration=AMR_DURATION, every=AMR_EVERY, n_refinements=1, coarsen=False,
            on_step=None):
    """The driver loop of application/adamantine.hh:1066-1399 for a refined
    problem (oracle or GPU): refine before step 1 and every `every` steps
    over the next `every` steps, then one time step."""
    t, n = 0.0, 1
    while t < duration - 1e-12 * duration:
        if n == 1 or n % every == 0:
            problem.refine_mesh(t, t + every * dt, every, n_refinements, coarsen)
        t = problem.evolve_one_time_step(t, dt)
        if on_step is not None:
            on_step(n, t)
        n += 1
    return t


# demo_316_short_amr.info (test_integration_3d_amr.cc:60-88): forward Euler,
# 1e-4 s steps to 4 ms, refinement every 5 steps (and before the first), one
# level, coarsening after the beam; the reference expects 13005 DoFs at the
# end and a finite field.
DEMO_AMR_DT, DEMO_AMR_DURATION, DEMO_AMR_EVERY, DEMO_AMR_DOFS = 1e-4, 4e-3, 5, 13005


def demo_316_short_amr_config(degree=2):
    """demo_316_short_amr.info: 25 x 25 x 2 cells of a 5 x 5 x 0.5 mm plate
    (x length, y width, z height), FE_Q(2), convective and radiative faces,
    the amr_test material, a Goldak 400 W beam (absorption 0.3, 0.6 mm
    diameter, 0.5 mm depth) along demo_316_short_scan_path_amr.txt. Its
    material deposition adds no cell: the material height (0.75 mm) is above
    the plate, so every cell is active from the start, and the deposition
    boxes follow the scan path 0.95 mm up, above the mesh."""
    cfg = amr_test_config(degree=degree, n_cells=(25, 25, 2), boundary="convective,radiative")
    cfg.geometry = Geometry(dim=3, n_cells=(25, 25, 2), extent=(5e-3, 5e-3, 5e-4), material_height=0.75e-3)
    seg = np.load(os.path.join(HERE, "golden", "demo_316_short_amr_scan_path.npy"))
    cfg.sources = [Source(type="goldak", depth=0.5e-3, absorption_efficiency=0.3, diameter=0.6e-3,
                          max_power=400.0, segments=seg)]
    return cfg
