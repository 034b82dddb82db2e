"""Microstructure G/R records on the GPU (through the C ABI) against the
restatement of Microstructure::compute_G_and_R (source/Microstructure.hh:
89-207), which the reference's own gold files pin on CPU. The sums run in the
same order with the same roundings on both sides, so the records are
compared bit for bit."""
import os

import numpy as np
import pytest
import torch

from microstructure_oracle import compute_G_and_R, format_records

from adamantine_b200.config import Boundary, Geometry, ThermalConfig
from adamantine_b200.microstructure import Microstructure
from adamantine_b200.thermal import ThermalPhysics
from adamantine_b200.workloads import phase_change_material, rng_for

pytestmark = pytest.mark.gpu


def two_material_config(n_cells, extent, degree, material_height=1e9, origin=(0.0, 0.0, 0.0)):
    mat = phase_change_material()
    mat.n_materials = 2
    mat.poly[1] = mat.poly[0]
    mat.props[1] = mat.props[0]
    mat.props[1, 0] = 1500.0  # a second material with a lower liquidus
    mat.props[1, 1] = 1480.0
    geo = Geometry(dim=3, n_cells=n_cells, extent=extent, origin=origin, material_height=material_height,
                   use_powder=True, powder_layer=0.25 * extent[2])
    return ThermalConfig(geometry=geo, material=mat, boundary=Boundary.from_database({"type": "adiabatic"}, 3),
                         sources=[], degree=degree, time_method="forward_euler")


@pytest.mark.parametrize("degree", [1, 2])
def test_records_equal_restatement(degree):
    n_cells, extent, origin = (9, 6, 5), (2.7e-3, 1.8e-3, 1.5e-3), (1e-3, -2e-3, 0.5e-3)
    cfg = two_material_config(n_cells, extent, degree, material_height=origin[2] + 0.75 * extent[2] + 1e-12,
                              origin=origin)
    rng = rng_for(f"microstructure-{degree}")
    C = int(np.prod(n_cells))
    material = rng.integers(0, 2, C).astype(np.uint8)
    phys = ThermalPhysics(cfg, material_id=material)
    shape = cfg.geometry.node_shape(degree)[::-1]
    # a field around both liquidus values, so that some nodes cross each
    t_old = 1400.0 + 400.0 * rng.uniform(0, 1, shape)
    t_new = t_old - 300.0 * rng.uniform(0, 1, shape)
    ms = Microstructure(phys)
    for dt in (1e-5, 2.5e-6):  # two calls in a row on the same handle
        ms.set_old_temperature(phys.from_grid(t_old))
        got = ms.compute_G_and_R(phys.from_grid(t_new), dt)
        want = compute_G_and_R(n_cells, extent, degree, t_old, t_new, dt, cfg.material.props[:2, 0],
                               active=cfg.geometry.active_cells(), material=material, origin=origin)
        assert got.shape == want.shape and len(got) > 100
        assert np.array_equal(got, want, equal_nan=True)
        t_old, t_new = t_new, t_new - 50.0


def test_no_crossing_and_capacity():
    cfg = two_material_config((4, 4, 4), (1e-3, 1e-3, 1e-3), 2)
    phys = ThermalPhysics(cfg)
    T = phys.initialize_dof_vector(300.0)
    ms = Microstructure(phys)
    ms.set_old_temperature(T)
    assert ms.compute_G_and_R(T, 1e-6).shape == (0, 6)
    # a uniform drop through the liquidus: every support point of every
    # active cell, once per cell; G = 0, so R is inf
    ms.set_old_temperature(phys.initialize_dof_vector(2000.0))
    rec = ms.compute_G_and_R(phys.initialize_dof_vector(1000.0), 2.0)
    assert rec.shape == (64 * 27, 6)
    assert (rec[:, 3] == 0.0).all() and np.isposinf(rec[:, 5]).all()
    assert (rec[:, 4] == 2000.0 - 1000.0 / 2.0).all()


def test_file_format_and_driver_loop(tmp_path):
    """The driver loop of application/adamantine.hh:1235-1285 around real
    steps of a cooling field; the file holds the records in the reference's
    line format."""
    cfg = two_material_config((8, 8, 4), (2e-3, 2e-3, 1e-3), 2)
    phys = ThermalPhysics(cfg)
    nodes = cfg.geometry.node_shape(2)[::-1]
    z, y, x = np.meshgrid(*[np.linspace(0, e, n) for e, n in zip((1e-3, 2e-3, 2e-3), nodes)], indexing="ij")
    # a hot core at 1750 K in a 300 K block: its rim cools through the
    # liquidus within a few steps
    core = (np.abs(x - 1e-3) < 0.5e-3) & (np.abs(y - 1e-3) < 0.5e-3)
    T = phys.from_grid(np.where(core, 1750.0, 300.0))
    prefix = str(tmp_path / "G_R")
    ms = Microstructure(phys, prefix)
    t, dt, recs = 0.0, 2e-5, []
    for _ in range(20):
        ms.set_old_temperature(T)
        t_prev = T.clone()
        t = phys.evolve_one_time_step(t, dt, T)
        got = ms.compute_G_and_R(T, dt)
        want = compute_G_and_R((8, 8, 4), (2e-3, 2e-3, 1e-3), 2, phys.to_grid(t_prev), phys.to_grid(T), dt,
                               cfg.material.props[:2, 0], active=cfg.geometry.active_cells())
        assert np.array_equal(got, want, equal_nan=True)
        recs.append(got)
    ms.close()
    allr = np.concatenate(recs)
    assert len(allr) > 0
    lines = [ln for ln in open(prefix + ".txt").read().split("\n") if ln]
    assert lines == format_records(allr)
    os.remove(prefix + ".txt")
