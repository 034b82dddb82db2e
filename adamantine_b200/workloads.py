"""Seeded synthetic workloads of the hot-path benchmark and tests.

The reference publishes no benchmark suite for this path; these builders
create problems with the shapes, sizes and value ranges of the five benchmark
configurations (mesh, FE degree, material model, source and time stepping),
with every random quantity drawn from a named, seeded numpy stream.
"""
from __future__ import annotations

import zlib

import numpy as np

from .config import Boundary, Geometry, Material, Source, ThermalConfig

SEED = 20261203


def rng_for(name: str, seed: int = SEED) -> np.random.Generator:
    return np.random.default_rng([seed, zlib.crc32(name.encode())])


# --------------------------------------------------------------- materials
def steel_solid_material() -> Material:
    """Solid only: rho 7904 kg/m^3, c_p 714 J/kg/K, k 31.4 W/m/K, h_conv 10."""
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


def phase_change_material(rng=None, k_scale: float = 1.0, cp_scale: float = 1.0) -> Material:
    """Solid / liquid / powder; solidus 1648 K, liquidus 1673 K, L = 2.9e5 J/kg.

    k_solid(T): seeded quadratic with k(300) = 10 and k(1700) = 35 W/m/K,
    monotone on [300, 1700]; k_powder = 0.5% of k_solid; k_liquid = 35.
    c_p: seeded linear function (about 500 J/kg/K at 300 K).  rho = 7904.
    k_scale and cp_scale multiply every conductivity / specific-heat
    coefficient (the perturbed parameters of the ensemble and the adjoint).
    """
    rng = rng if rng is not None else rng_for("phase_change_material")
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


# --------------------------------------------------------------- scan paths
def line_segments(x0, x1, y, z, speed, t0=1e-9):
    """A point segment then one line along x at `speed`."""
    return np.array([[t0, 0.0, x0, y, z], [t0 + abs(x1 - x0) / speed, 1.0, x1, y, z]])


def serpentine_segments(rng, x0, x1, y0, z, n_passes, hatch, speed):
    """Seeded serpentine: n_passes lines along x, hatch apart, joined by
    power-off moves (end_time, power_modifier, x, y, z rows)."""
    jitter = rng.uniform(-0.1, 0.1) * hatch
    rows = [[1e-9, 0.0, x0, y0 + jitter, z]]
    t = rows[0][0]
    x, y = x0, y0 + jitter
    for p in range(n_passes):
        xe = x1 if p % 2 == 0 else x0
        t += abs(xe - x) / speed
        rows.append([t, 1.0, xe, y, z])
        x = xe
        if p + 1 < n_passes:
            y += hatch
            t += hatch / speed
            rows.append([t, 0.0, x, y, z])
    return np.array(rows)


# --------------------------------------------------------------- configs
def solid_q1_small() -> ThermalConfig:
    """10x10x5 mm, 32x32x16 Q1, Gauss 2, solid, convective top (h = 10,
    T_inf = 300), Goldak 200 W / 0.3 / R = d = 50 um along +x at 1 m/s on the
    top mid-line; forward Euler, dt = 1e-6."""
    geo = Geometry(dim=3, n_cells=(32, 32, 16), extent=(10e-3, 10e-3, 5e-3))
    bnd = Boundary.from_database({"type": "adiabatic", "boundary_5.type": "convective"}, 3)
    src = Source(type="goldak", depth=50e-6, absorption_efficiency=0.3, diameter=100e-6, max_power=200.0,
                 segments=line_segments(0.0, 10e-3, 5e-3, 5e-3, 1.0))
    return ThermalConfig(geometry=geo, material=steel_solid_material(), boundary=bnd, sources=[src], degree=1,
                         time_method="forward_euler")


def phase_change_q2(n_cells=(128, 128, 64), extent=(20e-3, 20e-3, 10e-3), powder_layers=16,
                    method="rk_fourth_order", k_scale=1.0, cp_scale=1.0, absorptivity=0.35,
                    power=400.0) -> ThermalConfig:
    """20x20x10 mm, 128x128x64 Q2, Gauss 3, solid/liquid/powder with powder in
    the top 16 cell layers, Goldak 400 W / 0.35 (R = d = 50 um) on a seeded
    10-pass serpentine (hatch 200 um, 1 m/s); adiabatic; RK4."""
    nz = n_cells[2]
    hz = extent[2] / nz
    geo = Geometry(dim=3, n_cells=n_cells, extent=extent, material_height=extent[2] + 0.5 * hz,
                   use_powder=True, powder_layer=powder_layers * hz + 0.5 * hz)
    bnd = Boundary.from_database({"type": "adiabatic"}, 3)
    rng = rng_for("phase_change_q2-scan")
    seg = serpentine_segments(rng, 0.25 * extent[0], 0.75 * extent[0], 0.45 * extent[1], extent[2], 10,
                              200e-6, 1.0)
    src = Source(type="goldak", depth=50e-6, absorption_efficiency=absorptivity, diameter=100e-6,
                 max_power=power, segments=seg)
    mat = phase_change_material(k_scale=k_scale, cp_scale=cp_scale)
    return ThermalConfig(geometry=geo, material=mat, boundary=bnd, sources=[src], degree=2, time_method=method)


def initial_temperature(cfg: ThermalConfig, name: str, melt_pool: bool = True) -> np.ndarray:
    """300 K + U(-1, 1) noise on the (nz, ny, nx) node grid; with melt_pool a
    seeded 2000 K Gaussian spot under the scan-path start so that liquid,
    mushy and powder-to-liquid points exist."""
    geo = cfg.geometry
    rng = rng_for("initial-" + name)
    shape = geo.node_shape(cfg.degree)[::-1]
    T = 300.0 + rng.uniform(-1.0, 1.0, shape)
    if melt_pool and cfg.sources:
        seg = cfg.sources[0].segments
        cx, cy, cz = seg[0, 2], seg[0, 3], seg[0, 4]
        zs = np.linspace(geo.origin[2], geo.origin[2] + geo.extent[2], shape[0])
        ys = np.linspace(geo.origin[1], geo.origin[1] + geo.extent[1], shape[1])
        xs = np.linspace(geo.origin[0], geo.origin[0] + geo.extent[0], shape[2])
        r2 = ((xs[None, None, :] - cx) ** 2 + (ys[None, :, None] - cy) ** 2 + (zs[:, None, None] - cz) ** 2)
        T += 1700.0 * np.exp(-r2 / (0.4e-3) ** 2)
    return T


def ensemble_q1(n_members=32, n_cells=(64, 64, 32), extent=(20e-3, 20e-3, 10e-3), min_layers=20,
                max_layers=32, powder_layers=4, method="rk_fourth_order", name="ensemble_q1"):
    """Batched EnKF ensemble: n_members problems on one 64x64x32 Q1 mesh
    (20x20x10 mm, Gauss 2) with the phase-change material of phase_change_q2.

    Per member (seeded): conductivity scale and absorptivity factor drawn
    from log-normal(0, 0.1) (absorptivity = 0.35 x factor), and a deposited
    height of min_layers..max_layers cell layers (uniform), the top
    powder_layers of it powder, so the active cell counts differ. Goldak
    400 W with R = 250 um, d = 300 um (resolved by the 312.5 um cells) on the
    seeded serpentine at the member's top surface; adiabatic; RK4.

    Returns (configs, params) with params[k] = (k_scale, absorptivity,
    n_layers).
    """
    rng = rng_for(name + "-params")
    k_scale = np.exp(rng.normal(0.0, 0.1, n_members))
    absorb = 0.35 * np.exp(rng.normal(0.0, 0.1, n_members))
    layers = rng.integers(min_layers, max_layers + 1, n_members)
    seg_rng_state = rng_for(name + "-scan")
    hz = extent[2] / n_cells[2]
    base_seg = serpentine_segments(seg_rng_state, 0.25 * extent[0], 0.75 * extent[0], 0.45 * extent[1], 0.0, 10,
                                   200e-6, 1.0)
    bnd = Boundary.from_database({"type": "adiabatic"}, 3)
    configs, params = [], []
    for k in range(n_members):
        top = layers[k] * hz
        geo = Geometry(dim=3, n_cells=n_cells, extent=extent, material_height=top, use_powder=True,
                       powder_layer=powder_layers * hz)
        seg = base_seg.copy()
        seg[:, 4] = top
        src = Source(type="goldak", depth=300e-6, absorption_efficiency=float(absorb[k]), diameter=500e-6,
                     max_power=400.0, segments=seg)
        mat = phase_change_material(k_scale=float(k_scale[k]))
        configs.append(ThermalConfig(geometry=geo, material=mat, boundary=bnd, sources=[src], degree=1,
                                     time_method=method))
        params.append((float(k_scale[k]), float(absorb[k]), int(layers[k])))
    return configs, params


def surface_observations(n_nodes_xy, layers, n_obs=2000, sigma=5.0, name="ensemble_q1-obs"):
    """2000 seeded observation points on the top surface: distinct (i, j)
    node columns, and for each member the node index (i, j, layers[k]) of
    its own top surface (Q1). Returns (ij, sigma)."""
    rng = rng_for(name)
    nx, ny = n_nodes_xy
    flat = rng.choice(nx * ny, size=n_obs, replace=False)
    return np.stack([flat % nx, flat // nx], axis=1), sigma


def adjoint_q2(n_cells=(64, 64, 32), extent=(20e-3, 20e-3, 10e-3), powder_layers=8, method="rk_second_order",
               k_scale=1.0, cp_scale=1.0, absorptivity=0.35, power=400.0, name="adjoint_q2"):
    """Adjoint workload: 64x64x32 Q2 (Gauss 3) over 20x20x10 mm with the
    phase-change material (powder in the top 8 cell layers), Goldak 400 W /
    0.35 with R = 250 um, d = 300 um (resolved by the 312.5 um cells) on the
    seeded serpentine at the top surface; adiabatic; explicit RK2."""
    nz = n_cells[2]
    hz = extent[2] / nz
    geo = Geometry(dim=3, n_cells=n_cells, extent=extent, material_height=extent[2] + 0.5 * hz,
                   use_powder=True, powder_layer=powder_layers * hz + 0.5 * hz)
    bnd = Boundary.from_database({"type": "adiabatic"}, 3)
    seg = serpentine_segments(rng_for(name + "-scan"), 0.25 * extent[0], 0.75 * extent[0], 0.45 * extent[1],
                              extent[2], 10, 200e-6, 1.0)
    src = Source(type="goldak", depth=300e-6, absorption_efficiency=absorptivity, diameter=500e-6,
                 max_power=power, segments=seg)
    mat = phase_change_material(k_scale=k_scale, cp_scale=cp_scale)
    return ThermalConfig(geometry=geo, material=mat, boundary=bnd, sources=[src], degree=2, time_method=method)


def interior_points(cfg: ThermalConfig, n_points=500, radius=1.0e-3, depth=1.0e-3, name="adjoint-points"):
    """n_points distinct seeded interior nodes (i, j, k) within `radius` (in
    x and y) of the scan-path start and `depth` below the top surface, none
    on the domain boundary."""
    rng = rng_for(name)
    geo = cfg.geometry
    nx, ny, nz = geo.node_shape(cfg.degree)
    h = [geo.extent[d] / (nx - 1 if d == 0 else (ny - 1 if d == 1 else nz - 1)) for d in range(3)]
    seg = cfg.sources[0].segments
    cx, cy, top = seg[0, 2], seg[0, 3], seg[0, 4]
    i0, i1 = max(1, int((cx - radius) / h[0])), min(nx - 2, int((cx + radius) / h[0]))
    j0, j1 = max(1, int((cy - radius) / h[1])), min(ny - 2, int((cy + radius) / h[1]))
    k1 = min(nz - 2, int(round(top / h[2])) - 1)
    k0 = max(1, k1 - int(depth / h[2]))
    cand = np.array([(i, j, k) for k in range(k0, k1 + 1) for j in range(j0, j1 + 1) for i in range(i0, i1 + 1)])
    pick = rng.choice(len(cand), size=min(n_points, len(cand)), replace=False)
    return cand[np.sort(pick)]


def deposition_q2(n_cells=(256, 256, 128), extent=(40e-3, 40e-3, 20e-3), initial_layers=100, powder_layers=16,
                  n_passes=40, speed=1.2, power=400.0, name="deposition_q2"):
    """Largest single-GPU workload with deposition: 256x256x128 Q2 (Gauss 3)
    over 40x40x20 mm (67.6 M nodes), the phase-change material with powder in
    the top 16 of the initially active 100 cell layers, Goldak 400 W / 0.35
    (R = d = 50 um) on a seeded 40-pass raster (x passes from 5 to 35 mm,
    hatch 0.75 mm, 1.2 m/s) at the top surface; adiabatic; RK4. Returns the
    configuration and the deposition boxes (50 um long, 50 um high, 100 um
    wide) along the path, which activate the cell layer above the surface."""
    from .deposition import deposition_boxes

    hz = extent[2] / n_cells[2]
    top = initial_layers * hz
    geo = Geometry(dim=3, n_cells=n_cells, extent=extent, material_height=top, use_powder=True,
                   powder_layer=powder_layers * hz)
    bnd = Boundary.from_database({"type": "adiabatic"}, 3)
    seg = serpentine_segments(rng_for(name + "-scan"), 5e-3, 35e-3, 5e-3, top, n_passes, 0.75e-3, speed)
    src = Source(type="goldak", depth=50e-6, absorption_efficiency=0.35, diameter=100e-6, max_power=power,
                 segments=seg)
    cfg = ThermalConfig(geometry=geo, material=phase_change_material(), boundary=bnd, sources=[src], degree=2,
                        time_method="rk_fourth_order")
    boxes = deposition_boxes(cfg, 50e-6, 50e-6, 100e-6, 0.0)
    return cfg, boxes


def amr_q2(n_cells=(64, 64, 8), extent=(16e-3, 16e-3, 2e-3), max_level=2, speed=1.0, power=400.0,
           name="amr_q2"):
    """Refined-mesh workload: 64x64x8 coarse Q2 cells (Gauss 3) over
    16x16x2 mm (0.25 mm cells), the phase-change material (solid),
    adiabatic, Goldak 400 W / 0.3 (diameter
    0.25 mm, depth 0.2 mm) along a line across the top surface at 1 m/s; the
    beam's surroundings refined max_level = 2 times (62.5 um cells, the
    resolution of the uniform 256x256x32 grid); RK4. Returns the
    configuration and max_level."""
    geo = Geometry(dim=3, n_cells=n_cells, extent=extent)
    bnd = Boundary.from_database({"type": "adiabatic"}, 3)
    seg = line_segments(2e-3, 14e-3, 8e-3 + rng_for(name).uniform(-0.1e-3, 0.1e-3), extent[2], speed)
    src = Source(type="goldak", depth=0.2e-3, absorption_efficiency=0.3, diameter=0.25e-3, max_power=power,
                 segments=seg)
    mat = phase_change_material()
    cfg = ThermalConfig(geometry=geo, material=mat, boundary=bnd, sources=[src], degree=2,
                        time_method="rk_fourth_order")
    return cfg, max_level
