"""The reference's own 3D known answers replayed on the CUDA path."""
import math
import os

import numpy as np
import pytest

from adamantine_b200.config import Boundary, Geometry, ThermalConfig
from cases import GOLDEN, unit_slp_material
from dealii_order import dof_to_node
from fe_assembly import BoxFE
from test_oracle_physics import convective_case

pytestmark = pytest.mark.gpu


def test_convective_bc_gold_gpu():
    """convection_bcs (test_thermal_physics.hh:512-624) on the GPU: 4001 forward
    Euler steps, 1809 values of convective_bc_gold.txt @1e-6."""
    from adamantine_b200.thermal import ThermalPhysics

    gold = np.load(os.path.join(GOLDEN, "convective_bc_gold.npy"))
    g = ThermalPhysics(convective_case())
    y = g.initialize_dof_vector(400.0)
    t = 0.0
    while t < 1.0:
        t = g.evolve_one_time_step(t, 2.5e-4, y)
    order = dof_to_node(3, (100, 1, 1), 2)
    vals = g.to_grid(y).reshape(-1)[order]
    assert np.max(np.abs(vals - gold) / np.abs(gold)) < 1e-6
    assert g.device_error() == 0


def test_spmv_anisotropic_angle_3d_gpu():
    """spmv_anisotropic_angle (test_thermal_operator.cc:415-577) on the GPU:
    vmult(e_i) == -K e_i @1e-10 with a 30 degree deposition angle."""
    from adamantine_b200.thermal import ThermalPhysics

    geo = Geometry(dim=3, n_cells=(4, 2, 2), extent=(12.0, 6.0, 6.0))
    cfg = ThermalConfig(geometry=geo, material=unit_slp_material(k=(1.0, 0.8, 0.8), p_order=1),
                        boundary=Boundary.from_database({"type": "adiabatic"}, 3), sources=[], degree=2)
    ang = math.pi / 6.0
    C = geo.n_cells_total
    g = ThermalPhysics(cfg, deposition_cos=np.full(C, math.cos(ang)), deposition_sin=np.full(C, math.sin(ang)))
    R = np.array([[math.cos(ang), -math.sin(ang)], [math.sin(ang), math.cos(ang)]])
    coef = np.zeros((3, 3))
    coef[:2, :2] = R @ np.diag([1.0, 0.8]) @ R.T
    coef[2, 2] = 0.8
    K = BoxFE(3, (4, 2, 2), (12.0, 6.0, 6.0), 2).stiffness(coef)
    n = K.shape[0]
    dst = g.initialize_dof_vector()
    for i in range(n):
        e = np.zeros(n)
        e[i] = 1.0
        g.vmult(dst, g.from_grid(e))
        got = g.to_grid(dst).reshape(-1)
        assert np.max(np.abs(got + K[:, i])) / np.max(np.abs(K[:, i])) < 1e-10
