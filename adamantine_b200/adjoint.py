"""Adjoint gradients of an observation misfit over include/adamantine_b200_adjoint.h.

``AdjointProblem`` owns one thermal problem whose conductivity scale,
specific-heat scale, absorptivity and power are the parameters theta; its
``objective`` runs the forward steps on the GPU and ``gradient`` adds the
hand-written adjoint sweep (checkpointed every K steps).
``MisfitFunction`` is the thin torch.autograd binding used for checks: its
forward is the objective, its backward the adjoint gradient.
"""
from __future__ import annotations

import copy
import ctypes
from typing import Optional, Sequence

import numpy as np
import torch

from . import _lib
from .config import Material, ThermalConfig
from .thermal import ThermalPhysics, _dev, _ptr

# StateProperty rows (source/types.hh:40-49) scaled by the parameters
_SPECIFIC_HEAT = 1
_CONDUCTIVITY = (2, 3, 4)


def scaled_material(base: Material, k_scale: float, cp_scale: float) -> Material:
    """The material with every state's conductivities multiplied by k_scale
    and specific heats by cp_scale (polynomial coefficients and table
    values)."""
    m = copy.deepcopy(base)
    for p in _CONDUCTIVITY:
        m.poly[:, p] *= k_scale
        m.table[:, p, :, :, 1] *= k_scale
    m.poly[:, _SPECIFIC_HEAT] *= cp_scale
    m.table[:, _SPECIFIC_HEAT, :, :, 1] *= cp_scale
    return m


def config_at(base: ThermalConfig, theta: Sequence[float]) -> ThermalConfig:
    """base with theta = (k_scale, cp_scale, absorptivity, power) applied
    (absorptivity and power replace those of every beam)."""
    cfg = copy.deepcopy(base)
    cfg.material = scaled_material(base.material, float(theta[0]), float(theta[1]))
    for s in cfg.sources:
        if s.type != "cube":
            s.absorption_efficiency = float(theta[2])
            s.max_power = float(theta[3])
    return cfg


class AdjointProblem:
    """Misfit J(theta) = sum_k sum_p (T_{n_k}[node_p] - target_{k,p})^2 of an
    n_steps forward run from y0, and its gradient by the adjoint.

    base: configuration at theta = (1, 1, absorptivity, power) of its
    sources with unit scales; points: (n, 3) node coordinates (i, j, k) of
    the observed nodes; material_id / deposition_cos / deposition_sin: per
    cell, as ThermalPhysics takes them. Cube sources keep their value (the
    source parameters act on Goldak and electron beams).
    """

    def __init__(self, base: ThermalConfig, y0_grid: np.ndarray, t0: float, dt: float, n_steps: int,
                 obs_steps: Sequence[int], points: np.ndarray, targets: Optional[np.ndarray] = None,
                 device: int = 0, checkpoint_every: int = 0, material_id=None, deposition_cos=None,
                 deposition_sin=None):
        self.base = base
        self.t0, self.dt, self.n_steps = float(t0), float(dt), int(n_steps)
        self.checkpoint_every = int(checkpoint_every)
        self.obs_steps = np.ascontiguousarray(obs_steps, np.int32)
        self.phys = ThermalPhysics(base, device=device, material_id=material_id, deposition_cos=deposition_cos,
                                   deposition_sin=deposition_sin)
        pts = np.asarray(points, np.int64).reshape(-1, 3)
        self.points = pts
        self.node_index = np.ascontiguousarray(
            pts[:, 0] + self.phys.pitch * (pts[:, 1] + self.phys.nodes[1] * pts[:, 2]), np.int64)
        self._L = _lib.load()
        self.y0 = self.phys.from_grid(y0_grid)
        h = ctypes.c_void_p()
        _lib.check(self._L.adm_adjoint_create(self.phys._h, ctypes.byref(h)))
        self._h = h
        self._theta = None
        self.set_targets(np.zeros((len(self.obs_steps), len(self.node_index))) if targets is None else targets)

    def close(self):
        h = getattr(self, "_h", None)
        if h is not None and h.value:
            self._L.adm_adjoint_destroy(h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_targets(self, targets: np.ndarray):
        self.targets = np.ascontiguousarray(targets, np.float64).reshape(len(self.obs_steps), len(self.node_index))
        _lib.check(self._L.adm_adjoint_set_observations(
            self._h, len(self.obs_steps), _ptr(self.obs_steps, ctypes.c_int32), len(self.node_index),
            _ptr(self.node_index, ctypes.c_int64), _ptr(self.targets, ctypes.c_double)))

    def _apply(self, theta):
        theta = tuple(float(x) for x in theta)
        if theta == self._theta:
            return
        cfg = config_at(self.base, theta)
        self.phys.update_material(cfg)
        for i, s in enumerate(cfg.sources):
            self.phys.update_beam(i, s.depth, s.absorption_efficiency, s.diameter, s.max_power)
        self._theta = theta

    def observe(self, theta) -> np.ndarray:
        """Observed temperatures [n_obs][n_points] of forward runs at theta
        (from the initial phase state), e.g. to make targets."""
        self._apply(theta)
        none = np.zeros(1, np.int32)
        _lib.check(self._L.adm_adjoint_set_observations(self._h, 0, _ptr(none, ctypes.c_int32), 0, None, None))
        out = []
        try:
            J = ctypes.c_double()
            yk = torch.empty_like(self.y0)
            for n in self.obs_steps:
                _lib.check(self._L.adm_adjoint_objective(self._h, self.t0, self.dt, max(int(n), 1), _dev(self.y0),
                                                         ctypes.byref(J), _dev(yk)))
                v = yk if n > 0 else self.y0
                out.append(v.cpu().numpy()[self.node_index])
        finally:
            self.set_targets(self.targets)
        return np.array(out)

    def objective(self, theta) -> float:
        self._apply(theta)
        J = ctypes.c_double()
        _lib.check(self._L.adm_adjoint_objective(self._h, self.t0, self.dt, self.n_steps, _dev(self.y0),
                                                 ctypes.byref(J), None))
        return float(J.value)

    def gradient(self, theta):
        """(J, dJ/dtheta) at theta."""
        self._apply(theta)
        J = ctypes.c_double()
        g = np.zeros(4)
        _lib.check(self._L.adm_adjoint_gradient(self._h, self.t0, self.dt, self.n_steps, self.checkpoint_every,
                                                _dev(self.y0), ctypes.byref(J), _ptr(g, ctypes.c_double), None))
        return float(J.value), g / np.asarray(self._theta, np.float64)

    def last_checkpoint_interval(self) -> int:
        """The checkpoint interval the last gradient used (checkpoint_every
        0, the default: the longest segment whose stores fit in half of the
        free device memory, the whole run when it fits)."""
        k = ctypes.c_int32()
        _lib.check(self._L.adm_adjoint_checkpoint_interval(self._h, ctypes.byref(k)))
        return int(k.value)

    def set_flush(self, flush: float):
        """Adjoint values at or below flush x the stage's largest count as
        zero in the gradient (tiles of them are skipped); 0: exact zeros
        only. Default 1e-30."""
        _lib.check(self._L.adm_adjoint_set_flush(self._h, float(flush)))

    def vmult_transpose(self, y: torch.Tensor, mu: torch.Tensor):
        """((dr/dT)^T mu, log-derivatives of mu . r) at y."""
        out = torch.empty_like(y)
        g = np.zeros(3)
        _lib.check(self._L.adm_adjoint_vmult_transpose(self._h, _dev(out), _dev(y), _dev(mu),
                                                       _ptr(g, ctypes.c_double)))
        return out, g


class MisfitFunction(torch.autograd.Function):
    """J = problem.objective(theta) with the adjoint gradient as backward;
    theta is a float64 tensor (k_scale, cp_scale, absorptivity, power)."""

    @staticmethod
    def forward(ctx, theta: torch.Tensor, problem: AdjointProblem):
        J, g = problem.gradient(theta.detach().cpu().numpy())
        ctx.save_for_backward(torch.as_tensor(g, dtype=theta.dtype, device=theta.device))
        return torch.tensor(J, dtype=theta.dtype, device=theta.device)

    @staticmethod
    def backward(ctx, grad_out):
        (g,) = ctx.saved_tensors
        return grad_out * g, None
