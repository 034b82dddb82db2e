"""EnKF analysis of an ensemble whose members are split over GPUs (one
process per GPU, torch.distributed for the collectives).

The exchange follows the structure of the perturbed-observation update
(DataAssimilator::update_ensemble, source/DataAssimilator.cc:95-189, which
gathers all members on rank 0 instead): every rank observes its own members,
the ranks all-gather HX (n_obs x N doubles), every rank computes the N x N
weight matrix W redundantly, the ranks all-reduce the sums of the augmented
state, each rank forms its members' contribution to every
member's update, and a reduce-scatter delivers to each rank the sum for its
own members. Only HX, the mean and the contributions cross the
interconnect; the states stay on their GPU.

``ShardedAnalysis`` takes the device steps as an object (the library's
adm_enkf_observe / gain / local_sum / partial_update / apply), so the same
exchange runs with any implementation of the steps.
"""
from __future__ import annotations

import ctypes
from typing import Optional

import torch
import torch.distributed as dist

from . import _lib
from .thermal import _dev


def _p(t: Optional[torch.Tensor]):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


class LibrarySteps:
    """The four analysis steps on the device (include/adamantine_b200_ensemble.h)."""

    def __init__(self, enkf):
        self._L = _lib.load()
        self._enkf = enkf  # keeps the handle alive while the steps use it
        self._h = enkf._h

    def observe(self, states, n_state, obs_index):
        N, stride = states.shape
        m = obs_index.shape[1]
        hx = torch.empty((N, m), dtype=torch.float64, device=states.device)
        _lib.check(self._L.adm_enkf_observe(self._h, N, _dev(states), stride, n_state, m, _p(obs_index), _dev(hx)))
        return hx

    def gain(self, hx, obs, perturbations, obs_var=None, obs_cov=None):
        N, m = hx.shape
        w = torch.empty((N, N), dtype=torch.float64, device=hx.device)
        _lib.check(self._L.adm_enkf_gain(self._h, N, m, _dev(hx), _dev(obs), _p(obs_var), _p(obs_cov),
                                         _dev(perturbations), _dev(w)))
        return w

    def local_sum(self, states, n_state, params):
        n_local, stride = states.shape
        n_params = 0 if params is None else params.shape[1]
        out = torch.empty(n_state + n_params, dtype=torch.float64, device=states.device)
        _lib.check(self._L.adm_enkf_local_sum(self._h, n_local, _dev(states), stride, n_state, _p(params), n_params,
                                              _dev(out)))
        return out

    def partial_update(self, states, n_state, params, total, w_rows, first=0):
        """The local members' contribution to every member's update; first
        is the ensemble index of the first local member (used by the
        localized update, which reads the anomalies kept by gain)."""
        n_local, stride = states.shape
        N = w_rows.shape[1]
        n_params = 0 if params is None else params.shape[1]
        u = torch.empty((N, n_state + n_params), dtype=torch.float64, device=states.device)
        _lib.check(self._L.adm_enkf_partial_update_localized(
            self._h, n_local, int(first), N, _dev(states), stride, n_state, _p(params), n_params, _dev(total),
            _dev(w_rows.contiguous()), _dev(u)))
        return u

    def apply(self, states, n_state, params, u, update_mask=None):
        n_local, stride = states.shape
        n_params = 0 if params is None else params.shape[1]
        _lib.check(self._L.adm_enkf_apply(self._h, n_local, _dev(states), stride, n_state, _p(params), n_params,
                                          _dev(u), _p(update_mask)))


class ShardedAnalysis:
    """Analysis over the ranks of a process group; each rank holds n_local
    members (the same number on every rank), rank r members
    [r n_local, (r + 1) n_local) of the ensemble."""

    def __init__(self, steps, group=None):
        self.steps = steps
        self.group = group

    def __call__(self, states, n_state, obs_index, obs, perturbations, obs_var=None, obs_cov=None, params=None,
                 update_mask=None):
        """states (n_local, stride) and params (n_local, p) of this rank are
        updated in place; obs_index (n_local, m) are this rank's maps;
        obs (m,) and perturbations (N, m) are the same on every rank."""
        world = dist.get_world_size(self.group) if dist.is_initialized() else 1
        rank = dist.get_rank(self.group) if dist.is_initialized() else 0
        n_local = states.shape[0]
        if world > 1:
            # every rank must hold the same number of members: the gathers
            # and the reduce-scatter below are sized by it
            counts = torch.tensor([n_local, -n_local], dtype=torch.int64, device=states.device)
            dist.all_reduce(counts, op=dist.ReduceOp.MAX, group=self.group)
            if int(counts[0]) != n_local or int(-counts[1]) != n_local:
                raise ValueError(f"ShardedAnalysis needs the same member count on every rank: this rank holds "
                                 f"{n_local}, the counts range from {int(-counts[1])} to {int(counts[0])}")
        N = n_local * world
        hx_local = self.steps.observe(states, n_state, obs_index)
        if world > 1:
            hx = torch.empty((N, hx_local.shape[1]), dtype=hx_local.dtype, device=hx_local.device)
            dist.all_gather_into_tensor(hx, hx_local.contiguous(), group=self.group)
        else:
            hx = hx_local
        w = self.steps.gain(hx, obs, perturbations, obs_var=obs_var, obs_cov=obs_cov)
        # sum of the augmented state over all members (the mean is total / N)
        total = self.steps.local_sum(states, n_state, params)
        if world > 1:
            dist.all_reduce(total, group=self.group)
        u = self.steps.partial_update(states, n_state, params, total, w[rank * n_local:(rank + 1) * n_local],
                                      first=rank * n_local)
        if world > 1:
            mine = torch.empty((n_local, u.shape[1]), dtype=u.dtype, device=u.device)
            dist.reduce_scatter_tensor(mine, u.contiguous(), group=self.group)
        else:
            mine = u
        self.steps.apply(states, n_state, params, mine, update_mask)
