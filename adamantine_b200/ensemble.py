"""Batched ensemble and EnKF analysis over include/adamantine_b200_ensemble.h.

The reference advances its data-assimilation ensemble member by member
(application/adamantine.hh:2137-2142) and updates it with
DataAssimilator::update_ensemble (source/DataAssimilator.cc:95-189). Here an
``Ensemble`` holds N thermal problems on one mesh whose node vectors are the
rows of one (N, stride) CUDA float64 tensor; ``evolve_one_time_step``
advances all of them with one launch per colour and stage, and ``EnKF``
runs the FP64 analysis on the device.
"""
from __future__ import annotations

import ctypes
from typing import List, Optional, Sequence

import numpy as np
import torch

from . import _lib
from .config import ConfigStruct, SourceStruct, ThermalConfig
from .thermal import _dev, _f64, _ptr, _u8


def _dev_any(t: Optional[torch.Tensor], dtype):
    if t is None:
        return None
    if not (t.is_cuda and t.dtype == dtype and t.is_contiguous()):
        raise ValueError(f"expected a contiguous CUDA {dtype} tensor")
    return ctypes.c_void_p(t.data_ptr())


class Ensemble:
    """N thermal problems sharing one mesh, advanced together on one GPU.

    ``configs``: one ThermalConfig per member (same mesh, element, states,
    boundary types, time method and source kinds; values may differ).
    ``cells``: per member a dict with any of active, material_id,
    initial_state, deposition_cos, deposition_sin (defaults: the member's
    geometry).
    """

    def __init__(self, configs: Sequence[ThermalConfig], device: int = 0,
                 stream: Optional[torch.cuda.Stream] = None, cells: Optional[List[dict]] = None,
                 setup: bool = True):
        if not torch.cuda.is_available():
            raise RuntimeError("adamantine_b200 needs a CUDA device (B200, sm_100a)")
        self._L = _lib.load()
        self.configs = list(configs)
        self.n_members = len(self.configs)
        self.device = torch.device("cuda", device)
        self.stream = stream if stream is not None else torch.cuda.current_stream(self.device)
        self._structs = (ConfigStruct * self.n_members)()
        self._keep = []
        for i, c in enumerate(self.configs):
            st = c.to_struct()
            self._keep.append(st)
            ctypes.memmove(ctypes.byref(self._structs[i]), ctypes.byref(st), ctypes.sizeof(ConfigStruct))
        h = ctypes.c_void_p()
        _lib.check(self._L.adm_ensemble_create(self._structs, self.n_members, device,
                                               ctypes.c_void_p(self.stream.cuda_stream), ctypes.byref(h)))
        self._h = h
        n = ctypes.c_int64()
        _lib.check(self._L.adm_ensemble_stride(self._h, ctypes.byref(n)))
        self.stride = int(n.value)
        c0 = self.configs[0]
        deg = c0.degree
        self.nodes = tuple(deg * n + 1 for n in c0.geometry.n_cells[:3])
        self.pitch = self.stride // (self.nodes[1] * self.nodes[2])
        self.n_cells = c0.geometry.n_cells_total
        self.n_states = c0.material.n_states
        for i in range(self.n_members):
            kw = (cells[i] if cells is not None else None) or {}
            geo = self.configs[i].geometry
            self.set_cells(i, kw.get("active", geo.active_cells()), kw.get("material_id"),
                           kw.get("initial_state", geo.initial_state()), kw.get("deposition_cos"),
                           kw.get("deposition_sin"))
        if setup:
            self.setup()

    def close(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._L.adm_ensemble_destroy(h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ------------------------------------------------------------ set-up
    def set_cells(self, member, active=None, material_id=None, initial_state=None, deposition_cos=None,
                  deposition_sin=None):
        a, m, s, c, sn = _u8(active), _u8(material_id), _u8(initial_state), _f64(deposition_cos), \
            _f64(deposition_sin)
        _lib.check(self._L.adm_ensemble_set_cells(self._h, int(member), _ptr(a, ctypes.c_uint8),
                                                  _ptr(m, ctypes.c_uint8), _ptr(s, ctypes.c_uint8),
                                                  _ptr(c, ctypes.c_double), _ptr(sn, ctypes.c_double)))

    def setup(self):
        _lib.check(self._L.adm_ensemble_setup(self._h))

    def n_work_items(self) -> int:
        n = ctypes.c_int64()
        _lib.check(self._L.adm_ensemble_n_work_items(self._h, ctypes.byref(n)))
        return int(n.value)

    # ------------------------------------------------------------ vectors
    def solutions(self, value: float = 0.0) -> torch.Tensor:
        return torch.full((self.n_members, self.stride), float(value), dtype=torch.float64, device=self.device)

    def from_grids(self, grids: Sequence[np.ndarray]) -> torch.Tensor:
        nx, ny, nz = self.nodes
        full = np.zeros((self.n_members, nz, ny, self.pitch))
        for i, g in enumerate(grids):
            full[i, :, :, :nx] = np.asarray(g, np.float64).reshape(nz, ny, nx)
        return torch.from_numpy(full.reshape(self.n_members, -1)).to(self.device)

    def to_grid(self, v: torch.Tensor) -> np.ndarray:
        nx, ny, nz = self.nodes
        a = v.detach().to("cpu").numpy().reshape(nz, ny, self.pitch)
        return np.ascontiguousarray(a[:, :, :nx])

    def node_index(self, i, j, k):
        """Offset of node (i, j, k) inside one member's vector."""
        return np.asarray(i) + self.pitch * (np.asarray(j) + self.nodes[1] * np.asarray(k))

    def grid(self):
        """(origin, node spacing, nodes per axis, pitch) of the member vectors:
        entry a + pitch (b + nodes[1] c) is the support point origin +
        (a, b, c) spacing (FE_Q(1) and FE_Q(2) support points are uniform)."""
        geo = self.configs[0].geometry
        deg = self.configs[0].degree
        spacing = tuple(float(geo.extent[d]) / (deg * geo.n_cells[d]) for d in range(3))
        return tuple(float(o) for o in geo.origin[:3]), spacing, self.nodes, self.pitch

    def node_points(self, index) -> np.ndarray:
        """Support points (n, 3) of the entries ``index`` of a member vector."""
        origin, spacing, nodes, pitch = self.grid()
        index = np.asarray(index, np.int64)
        a = index % pitch
        b = (index // pitch) % nodes[1]
        c = index // (pitch * nodes[1])
        return np.stack([origin[0] + a * spacing[0], origin[1] + b * spacing[1], origin[2] + c * spacing[2]], axis=1)

    # ------------------------------------------------------------ stepping
    def _check(self, sol: torch.Tensor):
        if tuple(sol.shape) != (self.n_members, self.stride):
            raise ValueError(f"solutions must have shape ({self.n_members}, {self.stride})")
        return _dev(sol)

    def evolve_one_time_step(self, t: float, dt: float, solutions: torch.Tensor) -> float:
        tout = ctypes.c_double()
        _lib.check(self._L.adm_ensemble_evolve_one_time_step(self._h, float(t), float(dt), self._check(solutions),
                                                             ctypes.byref(tout)))
        return float(tout.value)

    def evolve_looped(self, t: float, dt: float, solutions: torch.Tensor) -> float:
        tout = ctypes.c_double()
        _lib.check(self._L.adm_ensemble_evolve_looped(self._h, float(t), float(dt), self._check(solutions),
                                                      ctypes.byref(tout)))
        return float(tout.value)

    def evolve_n_steps(self, t: float, dt: float, n_steps: int, solutions: torch.Tensor) -> float:
        tout = ctypes.c_double()
        _lib.check(self._L.adm_ensemble_evolve_n_steps(self._h, float(t), float(dt), int(n_steps),
                                                       self._check(solutions), ctypes.byref(tout)))
        return float(tout.value)

    # ------------------------------------------------------------ parameters and state
    def update_beam(self, member: int, i: int, depth: float, absorption_efficiency: float, diameter: float,
                    max_power: float):
        s = SourceStruct()
        s.depth = depth
        s.absorption_efficiency = absorption_efficiency
        s.radius_squared = (diameter / 2.0) ** 2
        s.max_power = max_power
        _lib.check(self._L.adm_ensemble_update_beam(self._h, int(member), int(i), ctypes.byref(s)))

    def update_material(self, member: int, config: ThermalConfig):
        st = config.to_struct()
        _lib.check(self._L.adm_ensemble_update_material(self._h, int(member), ctypes.byref(st)))

    def get_cell_state(self, member: int) -> np.ndarray:
        out = np.zeros(self.n_states * self.n_cells)
        _lib.check(self._L.adm_ensemble_get_cell_state(self._h, int(member), _ptr(out, ctypes.c_double)))
        return out.reshape(self.n_states, self.n_cells)

    def get_inverse_mass_matrix(self, member: int) -> torch.Tensor:
        out = torch.zeros(self.stride, dtype=torch.float64, device=self.device)
        _lib.check(self._L.adm_ensemble_get_inverse_mass_matrix(self._h, int(member), _dev(out)))
        return out

    def set_schedule(self, schedule: int):
        """Launch schedule of the batched stages (0 coloured, 1 atomic, 2
        two-pass)."""
        _lib.check(self._L.adm_ensemble_set_schedule(self._h, int(schedule)))

    def set_cells_per_thread(self, n: int):
        """FE_Q(1) kernel variant (1, 2 or 4 cells per thread) of the batched
        stages and the members' own launches."""
        _lib.check(self._L.adm_ensemble_set_cells_per_thread(self._h, int(n)))

    def cells_per_thread(self) -> int:
        v = ctypes.c_int32()
        _lib.check(self._L.adm_ensemble_get_cells_per_thread(self._h, ctypes.byref(v)))
        return int(v.value)

    def autotune(self, solutions: torch.Tensor, dt: float):
        """Times one batched step per schedule (and, for FE degree 1, per
        cells-per-thread variant) on a copy of solutions, keeps the fastest;
        returns (schedule, [best ms coloured, atomic, two-pass])."""
        c = ctypes.c_int32()
        ms = np.zeros(3)
        _lib.check(self._L.adm_ensemble_autotune_schedules(self._h, self._check(solutions), float(dt),
                                                           ctypes.byref(c), _ptr(ms, ctypes.c_double), 3))
        return int(c.value), ms.tolist()

    def device_error(self) -> int:
        code = ctypes.c_int32()
        _lib.check(self._L.adm_ensemble_device_error(self._h, ctypes.byref(code)))
        return int(code.value)

    def synchronize(self):
        _lib.check(self._L.adm_ensemble_synchronize(self._h))


LOC_NONE, LOC_STEP, LOC_GASPARI_COHN = 0, 1, 2
_LOC_NAMES = {"none": LOC_NONE, "step_function": LOC_STEP, "gaspari_cohn": LOC_GASPARI_COHN}


class EnKF:
    """FP64 ensemble Kalman analysis on the device (perturbed observations,
    Cholesky of H P H^T + R; localization off until set_localization)."""

    def __init__(self, device: int = 0, stream: Optional[torch.cuda.Stream] = None):
        self._L = _lib.load()
        self.device = torch.device("cuda", device)
        self.stream = stream if stream is not None else torch.cuda.current_stream(self.device)
        h = ctypes.c_void_p()
        _lib.check(self._L.adm_enkf_create(device, ctypes.c_void_p(self.stream.cuda_stream), ctypes.byref(h)))
        self._h = h

    def close(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._L.adm_enkf_destroy(h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_localization(self, function, cutoff: float, obs_points, grid):
        """Covariance localization of the following analyses
        (data_assimilation.localization_cutoff_function / _distance of the
        reference): function "none", "step_function" or "gaspari_cohn" (or
        LOC_*), obs_points (m, 3) the support points of the observed entries,
        grid = (origin, spacing, nodes, pitch) of the state vectors
        (Ensemble.grid()). obs_points=None removes the localization."""
        if obs_points is None:
            _lib.check(self._L.adm_enkf_set_localization(self._h, 0, 1.0, 0, None, None, None, None, 0))
            return
        fn = _LOC_NAMES[function.lower()] if isinstance(function, str) else int(function)
        pts = np.ascontiguousarray(obs_points, np.float64).reshape(-1, 3)
        origin, spacing, nodes, pitch = grid
        o = np.ascontiguousarray(origin, np.float64)
        sp = np.ascontiguousarray(spacing, np.float64)
        nn = np.ascontiguousarray(nodes, np.int64)
        _lib.check(self._L.adm_enkf_set_localization(
            self._h, fn, float(cutoff), len(pts), _ptr(pts, ctypes.c_double), _ptr(o, ctypes.c_double),
            _ptr(sp, ctypes.c_double), _ptr(nn, ctypes.c_int64), int(pitch)))

    def analysis(self, states: torch.Tensor, n_state: int, obs_index: torch.Tensor, obs: torch.Tensor,
                 perturbations: torch.Tensor, obs_var: Optional[torch.Tensor] = None,
                 obs_cov: Optional[torch.Tensor] = None, params: Optional[torch.Tensor] = None,
                 update_mask: Optional[torch.Tensor] = None):
        """Update states (N, stride) and params (N, n_params) in place."""
        N, stride = states.shape
        m = obs.numel()
        n_params = 0 if params is None else params.shape[1]
        _lib.check(self._L.adm_enkf_analysis(
            self._h, int(N), _dev(states), int(stride), int(n_state), _dev_any(params, torch.float64),
            int(n_params), int(m), _dev_any(obs_index, torch.int64), _dev_any(obs, torch.float64),
            _dev_any(obs_var, torch.float64), _dev_any(obs_cov, torch.float64),
            _dev_any(perturbations, torch.float64), _dev_any(update_mask, torch.uint8)))
