"""Thermoelastic displacement over include/adamantine_b200_mechanics.h.

Mirrors adamantine::MechanicalPhysics (source/MechanicalPhysics.hh) as the
driver uses it after the thermal step (application/adamantine.hh:1289-1345):
``setup_dofs`` picks the cells that carry displacement (thermally active,
solid ratio above 0.99) and forms the right-hand side from the temperature
(thermal expansion from the reference temperature, gravity); ``solve`` runs
CG on the elasticity operator (preconditioned by a geometric multigrid
V-cycle, or by the diagonal) and returns the displacement, then updates
the stress at the Gauss points from the displacement increment with the
reference's combined isotropic-kinematic J2 model (compute_stress,
source/MechanicalPhysics.cc:542-634); ``stress_state`` returns the stress,
the back stress and the plastic internal variable.
"""
from __future__ import annotations

import ctypes
from typing import Optional, Sequence

import numpy as np
import torch

from . import _lib
from .thermal import ThermalPhysics, _dev

FACES = ("x-", "x+", "y-", "y+", "z-", "z+")


class MechConfigStruct(ctypes.Structure):
    _fields_ = [
        ("lame_first", ctypes.c_double * 4),
        ("lame_second", ctypes.c_double * 4),
        ("thermal_expansion", ctypes.c_double * 4),
        ("density", ctypes.c_double * 4),
        ("reference_temperature", ctypes.c_double * 4),
        ("initial_temperature", ctypes.c_double),
        ("thermoelastic", ctypes.c_int32),
        ("gravity", ctypes.c_int32),
        ("clamped_faces", ctypes.c_int32),
        ("rel_tol", ctypes.c_double),
        ("max_iter", ctypes.c_int32),
        ("pad0", ctypes.c_int32),
        ("plastic_modulus", ctypes.c_double * 4),
        ("isotropic_hardening", ctypes.c_double * 4),
        ("elastic_limit", ctypes.c_double * 4),
    ]


def _per_material(v, n=4):
    a = np.zeros(n)
    v = np.atleast_1d(np.asarray(v, float))
    a[: len(v)] = v
    if len(v) == 1:
        a[:] = v[0]
    return a


class MechanicalPhysics:
    """Elasticity on a thermal problem's mesh (same cells, degree, nodes).

    Per material: lame_first / lame_second (the solid's Lame parameters),
    thermal_expansion, density (solid); reference_temperatures per material
    for cells that have melted, initial_temperature for the others (the
    reference's reference_temperatures list with the initial temperature
    last); clamped: box faces with zero displacement ('x-' ... 'z+', boundary
    ids 0..5). J2 plasticity per material: plastic_modulus,
    isotropic_hardening and elastic_limit (infinite, the reference's
    default, keeps the material elastic)."""

    def __init__(self, physics: ThermalPhysics, lame_first, lame_second, thermal_expansion=0.0, density=0.0,
                 reference_temperatures=None, initial_temperature: float = 300.0, thermoelastic: bool = True,
                 gravity: bool = True, clamped: Sequence[str] = ("z-",), rel_tol: float = 1e-12,
                 max_iter: int = 0, plastic_modulus=0.0, isotropic_hardening=0.0, elastic_limit=float("inf")):
        self._L = _lib.load()
        self.physics = physics
        c = MechConfigStruct()
        for name, v in (("lame_first", lame_first), ("lame_second", lame_second),
                        ("thermal_expansion", thermal_expansion), ("density", density),
                        ("reference_temperature", reference_temperatures if reference_temperatures is not None
                         else initial_temperature),
                        ("plastic_modulus", plastic_modulus), ("isotropic_hardening", isotropic_hardening),
                        ("elastic_limit", elastic_limit)):
            arr = _per_material(v)
            for k in range(4):
                getattr(c, name)[k] = arr[k]
        c.initial_temperature = float(initial_temperature)
        c.thermoelastic = int(bool(thermoelastic))
        c.gravity = int(bool(gravity))
        c.clamped_faces = sum(1 << FACES.index(f) for f in clamped)
        c.rel_tol = float(rel_tol)
        c.max_iter = int(max_iter)
        self._cfg = c
        h = ctypes.c_void_p()
        _lib.check(self._L.adm_mechanics_create(physics._h, ctypes.byref(c), ctypes.byref(h)))
        self._h = h
        self.m = physics.m()

    def close(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._L.adm_mechanics_destroy(h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def setup_dofs(self, temperature: Optional[torch.Tensor] = None):
        """MechanicalPhysics::setup_dofs + update_rhs from the thermal
        handle's cells, states and has_melted flags and the temperature."""
        _lib.check(self._L.adm_mechanics_setup(self._h, None if temperature is None else _dev(temperature)))

    def new_vector(self) -> torch.Tensor:
        return torch.zeros(3 * self.m, dtype=torch.float64, device=self.physics.device)

    def vmult(self, dst: torch.Tensor, src: torch.Tensor):
        _lib.check(self._L.adm_mechanics_vmult(self._h, _dev(dst), _dev(src)))

    def rhs(self) -> torch.Tensor:
        out = self.new_vector()
        _lib.check(self._L.adm_mechanics_rhs(self._h, _dev(out)))
        return out

    def solve(self):
        """(displacement (3 x m node vectors, consecutive), CG iterations,
        final residual norm)."""
        x = self.new_vector()
        it, res = ctypes.c_int32(), ctypes.c_double()
        _lib.check(self._L.adm_mechanics_solve(self._h, _dev(x), ctypes.byref(it), ctypes.byref(res)))
        self.iterations, self.residual = int(it.value), float(res.value)
        return x

    def set_preconditioner(self, kind: str):
        """'multigrid' (the default: V-cycle over FE_Q(1) levels of the box,
        Chebyshev smoothing, exact coarsest solve) or 'jacobi'."""
        code = {"jacobi": 0, "multigrid": 1}[kind]
        _lib.check(self._L.adm_mechanics_set_preconditioner(self._h, code))

    def multigrid_levels(self):
        """(levels, free DoFs of the coarsest level) of the hierarchy the
        last multigrid solve built (0, 0 before one)."""
        n, c = ctypes.c_int32(), ctypes.c_int64()
        _lib.check(self._L.adm_mechanics_multigrid_levels(self._h, ctypes.byref(n), ctypes.byref(c)))
        return int(n.value), int(c.value)

    @property
    def n_dofs(self) -> int:
        n, c = ctypes.c_int64(), ctypes.c_int64()
        _lib.check(self._L.adm_mechanics_n_dofs(self._h, ctypes.byref(n), ctypes.byref(c)))
        return int(n.value)

    @property
    def n_cells(self) -> int:
        n, c = ctypes.c_int64(), ctypes.c_int64()
        _lib.check(self._L.adm_mechanics_n_dofs(self._h, ctypes.byref(n), ctypes.byref(c)))
        return int(c.value)

    def node_mask(self) -> np.ndarray:
        out = np.zeros(self.m, np.uint8)
        _lib.check(self._L.adm_mechanics_node_mask(self._h, out.ctypes.data_as(ctypes.c_void_p)))
        return out

    def stress_state(self):
        """(stress [6, n_cells, nq], back stress [6, n_cells, nq], plastic
        internal variable [n_cells, nq]) at the nq = (degree + 1)^3 Gauss
        points (x fastest) of every cell of the thermal mesh; components xx,
        yy, zz, xy, xz, yz."""
        C, nq = self.physics.n_cells, self.physics.n_qp
        dev = self.physics.device
        s = torch.empty((6, C, nq), dtype=torch.float64, device=dev)
        b = torch.empty((6, C, nq), dtype=torch.float64, device=dev)
        k = torch.empty((C, nq), dtype=torch.float64, device=dev)
        _lib.check(self._L.adm_mechanics_stress_state(self._h, _dev(s), _dev(b), _dev(k)))
        return s, b, k
