"""Pins the CPU oracle against the reference's own operator known answers.

Restates tests/test_thermal_operator.cc of the reference: the matrix-free
operator applied to unit vectors must equal minus the assembled Laplace
matrix (isotropic, anisotropic, rotated anisotropic 3D) and the assembled
boundary terms (radiative, convective).  The assembled matrices come from the
independent dense assembly in tests/fe_assembly.py.
"""
import math

import numpy as np
import pytest

import oracle_py
from adamantine_b200.config import Boundary, Geometry, ThermalConfig
from cases import operator_2d_case, unit_slp_material
from fe_assembly import BoxFE

SIGMA = 5.670374419e-8


def maxrel(a, b):
    scale = max(np.max(np.abs(b)), 1e-300)
    return float(np.max(np.abs(a - b)) / scale)


def make_oracle(cfg):
    st = cfg.to_struct()
    o = oracle_py.Oracle(st, active=cfg.geometry.active_cells(), initial_state=cfg.geometry.initial_state())
    o._keep_struct = st
    return o


def test_m_and_vmult_of_constant():
    """thermal_operator (test_thermal_operator.cc:41-146): m()==99, vmult(1)==0."""
    cfg = operator_2d_case(unit_slp_material(k=(10.0, None, 10.0), p_order=1))
    o = make_oracle(cfg)
    assert o.n_nodes == 99
    src = np.ones(o.n_nodes)
    dst = o.vmult(src)
    assert np.abs(dst).sum() < 1e-12
    dst2 = np.ones(o.n_nodes)
    o.vmult_add(dst2, src)
    dst1 = o.vmult(src) + src
    assert abs(np.abs(dst1).sum() - np.abs(dst2).sum()) < 1e-12


def test_spmv_isotropic():
    """spmv (test_thermal_operator.cc:148-263): vmult(e_i) == -K e_i @1e-12."""
    cfg = operator_2d_case(unit_slp_material(k=(1.0, None, 1.0), p_order=2))
    o = make_oracle(cfg)
    fe = BoxFE(2, (4, 5), (12.0, 6.0), 2)
    K = fe.stiffness(np.eye(2))
    for i in range(o.n_nodes):
        e = np.zeros(o.n_nodes)
        e[i] = 1.0
        assert maxrel(o.vmult(e), -K[:, i]) < 1e-12


def test_spmv_anisotropic():
    """spmv_anisotropic (test_thermal_operator.cc:265-413): k_x=1, k_z=0."""
    cfg = operator_2d_case(unit_slp_material(k=(1.0, None, 0.0), p_order=2))
    o = make_oracle(cfg)
    fe = BoxFE(2, (4, 5), (12.0, 6.0), 2)
    K = fe.stiffness(np.diag([1.0, 0.0]))
    for i in range(o.n_nodes):
        e = np.zeros(o.n_nodes)
        e[i] = 1.0
        assert maxrel(o.vmult(e), -K[:, i]) < 1e-12


def test_spmv_anisotropic_angle_3d():
    """spmv_anisotropic_angle (test_thermal_operator.cc:415-577): 3D, 30 deg
    deposition angle, k = (1, 0.8, 0.8) @1e-10."""
    geo = Geometry(dim=3, n_cells=(4, 2, 2), extent=(12.0, 6.0, 6.0))
    mat = unit_slp_material(k=(1.0, 0.8, 0.8), p_order=1)
    cfg = ThermalConfig(geometry=geo, material=mat, boundary=Boundary.from_database({"type": "adiabatic"}, 3),
                        sources=[], degree=2)
    ang = math.pi / 6.0
    st = cfg.to_struct()
    C = geo.n_cells_total
    o = oracle_py.Oracle(st, deposition_cos=np.full(C, math.cos(ang)), deposition_sin=np.full(C, math.sin(ang)))
    R = np.array([[math.cos(ang), -math.sin(ang)], [math.sin(ang), math.cos(ang)]])
    coef2 = R @ np.diag([1.0, 0.8]) @ R.T
    coef = np.zeros((3, 3))
    coef[:2, :2] = coef2
    coef[2, 2] = 0.8
    fe = BoxFE(3, (4, 2, 2), (12.0, 6.0, 6.0), 2)
    K = fe.stiffness(coef)
    for i in range(o.n_nodes):
        e = np.zeros(o.n_nodes)
        e[i] = 1.0
        assert maxrel(o.vmult(e), -K[:, i]) < 1e-10


@pytest.mark.parametrize("kind", ["radiative", "convective"])
def test_spmv_boundary_terms(kind):
    """spmv_rad / spmv_conv (test_thermal_operator.cc:580-952): Laplace with
    coefficient -1 plus -h(T) * face mass on every outer face @1e-12."""
    emissivity = 1e5
    extra = {}
    for s in ("solid", "powder", "liquid"):
        extra[f"material_0.{s}.emissivity"] = emissivity
        extra[f"material_0.{s}.convection_heat_transfer_coef"] = 1.0
    extra["material_0.radiation_temperature_infty"] = 0.0
    extra["material_0.convection_temperature_infty"] = 0.0
    cfg = operator_2d_case(unit_slp_material(k=(1.0, None, 1.0), p_order=1, extra=extra), boundary=kind)
    o = make_oracle(cfg)
    fe = BoxFE(2, (4, 5), (12.0, 6.0), 2)
    K = fe.stiffness(np.eye(2))
    faces = list(fe.boundary_faces())
    for i in range(o.n_nodes):
        e = np.zeros(o.n_nodes)
        e[i] = 1.0
        expected = -K @ e
        for cc, ids, f in faces:
            phi, jxw = fe.face_tables(f)
            T = phi @ e[ids]
            h = emissivity * SIGMA * T * (T * T) if kind == "radiative" else np.ones_like(T)
            expected[ids] -= np.einsum("q,qi,qj,q,j->i", h, phi, phi, jxw, e[ids])
        assert maxrel(o.vmult(e), expected) < 1e-12


def test_inverse_mass_is_lumped_gauss_lobatto():
    """compute_inverse_mass_matrix (ThermalOperator.templates.hh:118-164):
    the row sums of the Gauss-Lobatto mass, inverted."""
    cfg = operator_2d_case(unit_slp_material(p_order=1))
    o = make_oracle(cfg)
    w = np.array([1.0 / 6.0, 4.0 / 6.0, 1.0 / 6.0])
    hx, hz = 3.0, 1.2
    m = np.zeros((11, 9))  # (z nodes, x nodes)
    for cz in range(5):
        for cx in range(4):
            for a in range(3):
                for b in range(3):
                    m[2 * cz + b, 2 * cx + a] += w[a] * w[b] * hx * hz
    assert maxrel(o.inverse_mass(), 1.0 / m.reshape(-1)) < 1e-14
