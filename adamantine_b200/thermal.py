"""Python mirror of adamantine's ThermalOperatorBase / ThermalPhysicsInterface
over the C ABI of libadamantine_b200.so.

Method names follow source/ThermalOperatorBase.hh:14-85 and
source/ThermalPhysicsInterface.hh:28-189 of the reference.  Device vectors are
torch CUDA float64 tensors of length ``m()`` in the library's padded
full-grid node layout; ``to_grid`` / ``from_grid`` convert to and from the
plain (nz, ny, nx) node grid.  torch only provides device memory and the
stream; every computation runs in the library's CUDA kernels.
"""
from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np
import torch

from . import _lib
from .config import SourceStruct, ThermalConfig


def _u8(a):
    return None if a is None else np.ascontiguousarray(a, np.uint8)


def _f64(a):
    return None if a is None else np.ascontiguousarray(a, np.float64)


def _ptr(arr, typ):
    return None if arr is None else arr.ctypes.data_as(ctypes.POINTER(typ))


def _dev(t: torch.Tensor):
    if not (t.is_cuda and t.dtype == torch.float64 and t.is_contiguous()):
        raise ValueError("expected a contiguous CUDA float64 tensor")
    return ctypes.c_void_p(t.data_ptr())


class ThermalPhysics:
    """One thermal problem (operator + explicit time stepping) on one GPU."""

    def __init__(self, config: ThermalConfig, device: int = 0, stream: Optional[torch.cuda.Stream] = None,
                 active=None, material_id=None, initial_state=None, deposition_cos=None, deposition_sin=None,
                 setup: bool = True):
        if not torch.cuda.is_available():
            raise RuntimeError("adamantine_b200 needs a CUDA device (B200, sm_100a)")
        self._L = _lib.load()
        self.config = config
        self.device = torch.device("cuda", device)
        self._struct = config.to_struct()
        # the handle's kernels run on the caller's current stream, so torch
        # copies and allocations on that stream are ordered with them
        self.stream = stream if stream is not None else torch.cuda.current_stream(self.device)
        h = ctypes.c_void_p()
        _lib.check(self._L.adm_create(ctypes.byref(self._struct), device, ctypes.c_void_p(self.stream.cuda_stream),
                                      ctypes.byref(h)))
        self._h = h
        n = ctypes.c_int64()
        _lib.check(self._L.adm_n_nodes(self._h, ctypes.byref(n)))
        self._m = int(n.value)
        _lib.check(self._L.adm_n_cells(self._h, ctypes.byref(n)))
        self.n_cells = int(n.value)
        nodes = (ctypes.c_int64 * 3)()
        pitch = ctypes.c_int64()
        _lib.check(self._L.adm_node_layout(self._h, nodes, ctypes.byref(pitch)))
        self.nodes = tuple(int(x) for x in nodes)
        self.pitch = int(pitch.value)
        self.n_states = config.material.n_states
        self.n_qp = (config.degree + 1) ** 3
        geo = config.geometry
        if active is None:
            active = geo.active_cells()
        if initial_state is None:
            initial_state = geo.initial_state()
        self.set_cells(active, material_id, initial_state, deposition_cos, deposition_sin)
        if setup:
            self.setup()

    # ------------------------------------------------------------ lifetime
    def close(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._L.adm_destroy(h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ------------------------------------------------------------ set-up
    def set_cells(self, active=None, material_id=None, initial_state=None, deposition_cos=None,
                  deposition_sin=None):
        self._cells = [_u8(active), _u8(material_id), _u8(initial_state), _f64(deposition_cos),
                       _f64(deposition_sin)]
        a, m, s, c, sn = self._cells
        _lib.check(self._L.adm_set_cells(self._h, _ptr(a, ctypes.c_uint8), _ptr(m, ctypes.c_uint8),
                                         _ptr(s, ctypes.c_uint8), _ptr(c, ctypes.c_double),
                                         _ptr(sn, ctypes.c_double)))

    def setup(self):
        _lib.check(self._L.adm_setup(self._h))

    # ------------------------------------------------------------ vectors
    def m(self) -> int:
        return self._m

    def n(self) -> int:
        return self._m

    def active_cells(self) -> np.ndarray:
        """The cells that carry material now (initial set and activations)."""
        out = np.zeros(self.n_cells, np.uint8)
        _lib.check(self._L.adm_get_active_cells(self._h, _ptr(out, ctypes.c_uint8)))
        return out

    def initialize_dof_vector(self, value: float = 0.0) -> torch.Tensor:
        return torch.full((self._m,), float(value), dtype=torch.float64, device=self.device)

    def to_grid(self, v: torch.Tensor) -> np.ndarray:
        """Device vector -> numpy (nz, ny, nx) node grid (padding dropped)."""
        nx, ny, nz = self.nodes
        a = v.detach().to("cpu").numpy().reshape(nz, ny, self.pitch)
        return np.ascontiguousarray(a[:, :, :nx])

    def from_grid(self, grid: np.ndarray) -> torch.Tensor:
        nx, ny, nz = self.nodes
        g = np.asarray(grid, np.float64).reshape(nz, ny, nx)
        full = np.zeros((nz, ny, self.pitch))
        full[:, :, :nx] = g
        return torch.from_numpy(full.reshape(-1)).to(self.device)

    # ------------------------------------------------------------ operator
    def set_time(self, t: float):
        _lib.check(self._L.adm_set_time(self._h, float(t)))

    def vmult(self, dst: torch.Tensor, src: torch.Tensor):
        _lib.check(self._L.adm_vmult(self._h, _dev(dst), _dev(src)))

    def vmult_add(self, dst: torch.Tensor, src: torch.Tensor):
        _lib.check(self._L.adm_vmult_add(self._h, _dev(dst), _dev(src)))

    def vmult_host(self, src: np.ndarray, dst: np.ndarray = None) -> np.ndarray:
        src = np.ascontiguousarray(src, np.float64)
        if dst is None:
            dst = np.empty_like(src)
        assert dst.flags.c_contiguous and dst.dtype == np.float64 and dst.size == src.size
        _lib.check(self._L.adm_vmult_host(self._h, _ptr(dst, ctypes.c_double), _ptr(src, ctypes.c_double)))
        return dst

    def compute_inverse_mass_matrix(self):
        _lib.check(self._L.adm_compute_inverse_mass_matrix(self._h))

    def get_inverse_mass_matrix(self) -> torch.Tensor:
        out = self.initialize_dof_vector()
        _lib.check(self._L.adm_get_inverse_mass_matrix(self._h, _dev(out)))
        return out

    # ------------------------------------------------------------ physics
    def evolve_one_time_step(self, t: float, dt: float, solution: torch.Tensor) -> float:
        tout = ctypes.c_double()
        _lib.check(self._L.adm_evolve_one_time_step(self._h, float(t), float(dt), _dev(solution),
                                                    ctypes.byref(tout)))
        return float(tout.value)

    def evolve_one_time_step_host(self, t: float, dt: float, solution: np.ndarray) -> float:
        assert solution.flags.c_contiguous and solution.dtype == np.float64
        tout = ctypes.c_double()
        _lib.check(self._L.adm_evolve_one_time_step_host(self._h, float(t), float(dt),
                                                         _ptr(solution, ctypes.c_double), ctypes.byref(tout)))
        return float(tout.value)

    def evolve_n_steps(self, t: float, dt: float, n_steps: int, solution: torch.Tensor) -> float:
        tout = ctypes.c_double()
        _lib.check(self._L.adm_evolve_n_steps(self._h, float(t), float(dt), int(n_steps), _dev(solution),
                                              ctypes.byref(tout)))
        return float(tout.value)

    def evaluate_material_properties(self, temperature: torch.Tensor) -> torch.Tensor:
        out = torch.zeros((8, self.n_cells), dtype=torch.float64, device=self.device)
        _lib.check(self._L.adm_evaluate_material_properties(self._h, _dev(temperature), _dev(out)))
        return out

    def set_state_to_material_properties(self):
        _lib.check(self._L.adm_set_state_to_material_properties(self._h))

    def get_state_from_material_properties(self):
        _lib.check(self._L.adm_get_state_from_material_properties(self._h))

    def get_cell_state(self) -> np.ndarray:
        out = np.zeros(self.n_states * self.n_cells)
        _lib.check(self._L.adm_get_cell_state(self._h, _ptr(out, ctypes.c_double)))
        return out.reshape(self.n_states, self.n_cells)

    def set_cell_state(self, state: np.ndarray):
        s = np.ascontiguousarray(state, np.float64).reshape(-1)
        assert s.size == self.n_states * self.n_cells
        _lib.check(self._L.adm_set_cell_state(self._h, _ptr(s, ctypes.c_double)))

    def get_qp_powder(self) -> np.ndarray:
        out = np.zeros(self.n_cells * self.n_qp)
        _lib.check(self._L.adm_get_qp_powder(self._h, _ptr(out, ctypes.c_double)))
        return out.reshape(self.n_cells, self.n_qp)

    def mark_has_melted(self, threshold: float, temperature: torch.Tensor) -> np.ndarray:
        out = np.zeros(self.n_cells, np.uint8)
        _lib.check(self._L.adm_mark_has_melted(self._h, float(threshold), _dev(temperature),
                                               _ptr(out, ctypes.c_uint8)))
        return out

    def add_material(self, cells, new_temperature: float, solution: torch.Tensor, cos=None, sin=None):
        """add_material_start + add_material_end on the fixed numbering."""
        cells = np.ascontiguousarray(cells, np.int64)
        cs, sn = _f64(cos), _f64(sin)
        _lib.check(self._L.adm_activate_cells(self._h, _ptr(cells, ctypes.c_int64), int(cells.size),
                                              float(new_temperature), _ptr(cs, ctypes.c_double),
                                              _ptr(sn, ctypes.c_double), _dev(solution)))

    def update_beam(self, i: int, depth: float, absorption_efficiency: float, diameter: float, max_power: float):
        """update_physics_parameters for beam i."""
        s = SourceStruct()
        s.depth = depth
        s.absorption_efficiency = absorption_efficiency
        s.radius_squared = (diameter / 2.0) ** 2
        s.max_power = max_power
        _lib.check(self._L.adm_update_beam(self._h, int(i), ctypes.byref(s)))

    def update_material(self, config: ThermalConfig):
        """New material tables (same shape) from config."""
        st = config.to_struct()
        _lib.check(self._L.adm_update_material(self._h, ctypes.byref(st)))

    COLOURED, ATOMIC, TWO_PASS = 0, 1, 2
    SCHEDULES = ("coloured", "atomic", "two_pass")

    def set_schedule(self, schedule: int):
        """Launch schedule: COLOURED or TWO_PASS (no atomics, bit
        reproducible) or ATOMIC."""
        _lib.check(self._L.adm_set_schedule(self._h, int(schedule)))

    def schedule(self) -> int:
        v = ctypes.c_int32()
        _lib.check(self._L.adm_get_schedule(self._h, ctypes.byref(v)))
        return int(v.value)

    def set_cells_per_thread(self, n: int):
        """FE_Q(1) operator kernel variant: 1 or 2 cells (stacked in z) per
        thread, or 4 (one warp per tile, a thread per column of 4 cells)."""
        _lib.check(self._L.adm_set_cells_per_thread(self._h, int(n)))

    def cells_per_thread(self) -> int:
        v = ctypes.c_int32()
        _lib.check(self._L.adm_get_cells_per_thread(self._h, ctypes.byref(v)))
        return int(v.value)

    def set_cells_per_block(self, n: int):
        """FE_Q(2) operator kernel variant: 64 cells per block (one tile,
        every schedule) or 128 (a z-pair of tiles, the atomic schedule)."""
        _lib.check(self._L.adm_set_cells_per_block(self._h, int(n)))

    def cells_per_block(self) -> int:
        v = ctypes.c_int32()
        _lib.check(self._L.adm_get_cells_per_block(self._h, ctypes.byref(v)))
        return int(v.value)

    def autotune(self, field: torch.Tensor):
        """Times every schedule (and, for FE degree 1, every cells-per-thread
        variant) on vmults of field, keeps the fastest; returns (schedule,
        [best ms coloured, atomic, two-pass])."""
        c = ctypes.c_int32()
        ms = np.zeros(3)
        _lib.check(self._L.adm_autotune_schedules(self._h, _dev(field), ctypes.byref(c), _ptr(ms, ctypes.c_double),
                                                  3))
        return int(c.value), ms.tolist()

    def save_checkpoint(self, path: str, time: float, solution: torch.Tensor):
        """save_checkpoint: cells, state, time and solution to one file."""
        _lib.check(self._L.adm_save_checkpoint(self._h, str(path).encode(), float(time), _dev(solution)))

    def load_checkpoint(self, path: str, solution: torch.Tensor, exact: bool = False) -> float:
        """load_checkpoint into solution; returns the saved time. exact
        restores the per-point phase history (bit-identical continuation)."""
        t = ctypes.c_double()
        _lib.check(self._L.adm_load_checkpoint(self._h, str(path).encode(), int(bool(exact)), ctypes.byref(t),
                                               _dev(solution)))
        return float(t.value)

    def device_error(self) -> int:
        code = ctypes.c_int32()
        _lib.check(self._L.adm_device_error(self._h, ctypes.byref(code)))
        return int(code.value)

    def synchronize(self):
        _lib.check(self._L.adm_synchronize(self._h))
