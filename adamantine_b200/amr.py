"""Refined meshes of the thermal path over include/adamantine_b200_amr.h.

Mirrors the reference's adaptive driver (application/adamantine.hh):
``refine_mesh`` (:608-681) refines the cells on the beams' paths over the
next refinement window, ``compute_cells_to_refine`` (:540-606) picks them,
``refine_and_transfer`` (:312-539) moves the temperature and the cell
states to the new mesh; the operator and the time stepping are those of
ThermalPhysics with hanging-node constraints. ``AmrMesh`` is the mesh logic
alone (host, no GPU); ``AmrThermalPhysics`` the refined problem on the GPU.
"""
from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np
import torch

from . import _lib
from .config import ThermalConfig
from .thermal import _dev


def _u8(a):
    return None if a is None else np.ascontiguousarray(a, np.uint8)


def _p(a):
    return None if a is None else a.ctypes.data_as(ctypes.c_void_p)


class _Common:
    """Queries shared by the host mesh and the GPU problem."""

    _prefix = ""

    def _call(self, name, *args):
        _lib.check(getattr(self._L, self._prefix + name)(self._h, *args))

    @property
    def n_dofs(self) -> int:
        n, m = ctypes.c_int64(), ctypes.c_int64()
        self._call("n_dofs", ctypes.byref(n), ctypes.byref(m))
        return int(n.value)

    @property
    def n_nodes(self) -> int:
        """All distinct nodes of the active leaves (hanging ones included)."""
        n, m = ctypes.c_int64(), ctypes.c_int64()
        self._call("n_dofs", ctypes.byref(n), ctypes.byref(m))
        return int(m.value)

    def leaves(self) -> np.ndarray:
        """(n, 4) int32: level, i, j, k."""
        n = ctypes.c_int64()
        self._call("n_leaves", ctypes.byref(n))
        out = np.zeros((int(n.value), 4), np.int32)
        self._call("leaves", _p(out))
        return out

    def dof_lattice(self) -> np.ndarray:
        out = np.zeros((self.n_dofs, 3), np.int64)
        self._call("dof_lattice", _p(out))
        return out

    def dof_points(self) -> np.ndarray:
        """Physical coordinates of the DoFs."""
        g = self.config.geometry
        scale = np.array([g.extent[d] / g.n_cells[d] for d in range(3)]) / float(1 << (self.max_level + 1))
        return np.asarray(g.origin, float)[None, :] + self.dof_lattice() * scale[None, :]

    def _flags(self, leaf_set, leaves):
        if leaf_set is None:
            return None
        s = {tuple(int(v) for v in c) for c in leaf_set}
        return np.array([1 if tuple(int(v) for v in c) in s else 0 for c in leaves], np.uint8)


class AmrMesh(_Common):
    """Forest, balance, DoFs and hanging-node constraints (host only)."""

    _prefix = "adm_amr_mesh_"

    def __init__(self, config: ThermalConfig, max_level: int, active=None, material_id=None, initial_state=None):
        self._L = _lib.load()
        self.config = config
        self.max_level = int(max_level)
        self._struct = config.to_struct()
        h = ctypes.c_void_p()
        _lib.check(self._L.adm_amr_mesh_create(ctypes.byref(self._struct), self.max_level, ctypes.byref(h)))
        self._h = h
        a, m, i = _u8(active), _u8(material_id), _u8(initial_state)
        self._call("set_cells", _p(a), _p(m), _p(i))
        self._call("build")

    def close(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._L.adm_amr_mesh_destroy(h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def refine_mesh(self, time: float, next_refinement_time: float, time_steps_refinement: int,
                    n_refinements: int = 2, coarsen_after_beam: bool = False):
        self._call("refine_mesh", float(time), float(next_refinement_time), int(time_steps_refinement),
                   int(n_refinements), int(bool(coarsen_after_beam)))

    def execute(self, refine=None, coarsen=None):
        """refine / coarsen: collections of leaves (level, i, j, k)."""
        lv = self.leaves()
        r, c = self._flags(refine, lv), self._flags(coarsen, lv)
        self._call("execute", _p(r), _p(c))

    def constraints(self):
        """Hanging nodes: lattice coordinates (n, 3) and CSR rows (ptr, dof, w)."""
        nh, ne = ctypes.c_int64(), ctypes.c_int64()
        self._call("constraints", ctypes.byref(nh), ctypes.byref(ne), None, None, None, None)
        xyz = np.zeros((int(nh.value), 3), np.int64)
        ptr = np.zeros(int(nh.value) + 1, np.int64)
        dof = np.zeros(int(ne.value), np.int32)
        w = np.zeros(int(ne.value), np.float64)
        self._call("constraints", ctypes.byref(nh), ctypes.byref(ne), _p(xyz), _p(ptr), _p(dof), _p(w))
        return xyz, ptr, dof, w


class AmrThermalPhysics(_Common):
    """ThermalPhysics on a refined mesh (GPU): the handle owns the
    temperature vector, which follows the mesh through every refinement."""

    _prefix = "adm_amr_"

    def __init__(self, config: ThermalConfig, max_level: int, device: int = 0,
                 stream: Optional[torch.cuda.Stream] = None, active=None, material_id=None, initial_state=None,
                 initial_temperature: float = 300.0):
        if not torch.cuda.is_available():
            raise RuntimeError("adamantine_b200 needs a CUDA device (B200, sm_100a)")
        self._L = _lib.load()
        self.config = config
        self.max_level = int(max_level)
        self.device = torch.device("cuda", device)
        self.stream = stream if stream is not None else torch.cuda.current_stream(self.device)
        self._struct = config.to_struct()
        h = ctypes.c_void_p()
        _lib.check(self._L.adm_amr_create(ctypes.byref(self._struct), self.max_level, device,
                                          ctypes.c_void_p(self.stream.cuda_stream), ctypes.byref(h)))
        self._h = h
        if active is None:
            active = config.geometry.active_cells()
        if initial_state is None:
            initial_state = config.geometry.initial_state()
        a, m, i = _u8(active), _u8(material_id), _u8(initial_state)
        self._call("set_cells", _p(a), _p(m), _p(i))
        self._call("setup", float(initial_temperature))

    def close(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._L.adm_amr_destroy(h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- mesh changes
    def refine_mesh(self, time: float, next_refinement_time: float, time_steps_refinement: int,
                    n_refinements: int = 2, coarsen_after_beam: bool = False):
        """refine_mesh + refine_and_transfer (the temperature follows)."""
        self._call("refine_mesh", float(time), float(next_refinement_time), int(time_steps_refinement),
                   int(n_refinements), int(bool(coarsen_after_beam)))

    def execute(self, refine=None, coarsen=None):
        lv = self.leaves()
        r, c = self._flags(refine, lv), self._flags(coarsen, lv)
        self._call("execute", _p(r), _p(c))

    REMESH_PHASES = ("snapshot", "flag_and_execute", "nodes_and_constraints", "level_setup", "cell_state_transfer",
                     "prolongation_tables", "solution_transfer", "inverse_mass")

    def remesh_profile(self) -> dict:
        """Host wall time (ms) of the last refine_mesh / execute per phase."""
        ms = np.zeros(len(self.REMESH_PHASES))
        self._call("remesh_profile", _p(ms))
        return dict(zip(self.REMESH_PHASES, ms.tolist()))

    # ---- vectors
    def new_vector(self) -> torch.Tensor:
        return torch.zeros(self.n_dofs, dtype=torch.float64, device=self.device)

    def get_solution(self) -> torch.Tensor:
        out = torch.empty(self.n_dofs, dtype=torch.float64, device=self.device)
        self._call("get_solution", _dev(out))
        return out

    def set_solution(self, y: torch.Tensor):
        if y.numel() != self.n_dofs:
            raise ValueError("the vector does not match the mesh's DoFs")
        self._call("set_solution", _dev(y.contiguous()))

    def set_time(self, t: float):
        self._call("set_time", float(t))

    def vmult(self, dst: torch.Tensor, src: torch.Tensor):
        n = self.n_dofs
        if dst.numel() != n or src.numel() != n:
            raise ValueError("the vectors do not match the mesh's DoFs")
        self._call("vmult", _dev(dst), _dev(src))

    def inverse_mass(self) -> torch.Tensor:
        out = torch.empty(self.n_dofs, dtype=torch.float64, device=self.device)
        self._call("inverse_mass", _dev(out))
        return out

    def evolve_one_time_step(self, t: float, dt: float) -> float:
        out = ctypes.c_double()
        self._call("evolve_one_time_step", float(t), float(dt), ctypes.byref(out))
        return float(out.value)

    def level_layout(self, level: int):
        nodes = (ctypes.c_int64 * 3)()
        pitch = ctypes.c_int64()
        self._call("level_layout", int(level), nodes, ctypes.byref(pitch))
        return tuple(int(x) for x in nodes), int(pitch.value)

    def level_values(self, level: int) -> np.ndarray:
        """The temperature on a level grid, shape (z, y, x) (hanging nodes
        interpolated; nodes of no leaf of that level are 0)."""
        nodes, pitch = self.level_layout(level)
        buf = np.zeros(pitch * nodes[1] * nodes[2])
        self._call("level_values", int(level), _p(buf))
        return buf.reshape(nodes[2], nodes[1], pitch)[:, :, : nodes[0]]

    def level_cell_state(self, level: int) -> np.ndarray:
        """(n_states, cells of the level grid) state ratios of the level's
        leaves (other cells 0)."""
        n = [self.config.geometry.n_cells[d] << level for d in range(3)]
        ns = self.config.material.n_states
        out = np.zeros(ns * n[0] * n[1] * n[2])
        self._call("level_cell_state", int(level), _p(out))
        return out.reshape(ns, -1)

    def mark_has_melted(self, threshold: float):
        """Flag the leaves whose cell-average temperature exceeds threshold
        (ThermalPhysics::mark_has_melted); the flags follow refinement."""
        self._call("mark_has_melted", float(threshold))

    def level_has_melted(self, level: int) -> np.ndarray:
        n = [self.config.geometry.n_cells[d] << level for d in range(3)]
        out = np.zeros(n[0] * n[1] * n[2], np.uint8)
        self._call("level_has_melted", int(level), _p(out))
        return out

    def set_schedule(self, schedule: str):
        """'atomic' (default: one launch per level and application),
        'coloured' (eight launches) or 'two_pass' (a tile launch and a
        gather); the last two add in a fixed order."""
        self._call("set_schedule", {"coloured": 0, "atomic": 1, "two_pass": 2}[schedule])

    def synchronize(self):
        self._call("synchronize")


def _main(argv=None):
    """python -m adamantine_b200.amr [--steps N]: the refined-mesh workload
    (workloads.amr_q2: refine_mesh over a 100-step window, then N RK4
    steps); prints the mesh and the peak temperature."""
    import argparse

    from .workloads import amr_q2

    ap = argparse.ArgumentParser(description=_main.__doc__)
    ap.add_argument("--steps", type=int, default=8)
    args = ap.parse_args(argv)
    cfg, L = amr_q2()
    g = AmrThermalPhysics(cfg, L)
    dt, K = 1e-6, 100
    g.refine_mesh(0.0, K * dt, K, L)
    t = 0.0
    for _ in range(args.steps):
        t = g.evolve_one_time_step(t, dt)
    lv = g.leaves()
    print({"leaves_per_level": [int((lv[:, 0] == l).sum()) for l in range(L + 1)], "dofs": g.n_dofs,
           "t": t, "peak_temperature": float(g.get_solution().max().item())})


if __name__ == "__main__":
    _main()
