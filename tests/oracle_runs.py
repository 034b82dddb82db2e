"""Oracle runs of the benchmark workloads in worker processes -- test
infrastructure.

The configuration-size parity tests need many independent CPU oracle runs
(one per ensemble member, three forwards for a central difference). Each
runs in a process of a ``spawn`` pool (never ``fork``: the parent process has
a CUDA context) with a share of the host cores, and rebuilds its seeded
configuration from the workload builders, so only small arguments cross the
process boundary.
"""
from __future__ import annotations

import concurrent.futures as cf
import multiprocessing as mp
import os
import sys

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_ROOT = os.path.dirname(_HERE)
for _p in (_ROOT, os.path.join(_ROOT, "oracle"), _HERE):
    if _p not in sys.path:
        sys.path.insert(0, _p)


def _oracle(cfg, n_threads):
    import oracle_py

    cfg.n_threads = n_threads
    st = cfg.to_struct()
    o = oracle_py.Oracle(st, active=cfg.geometry.active_cells(), initial_state=cfg.geometry.initial_state())
    o._keep = st
    return o


def ensemble_member(k: int, n_steps: int, dt: float, n_threads: int):
    """Member k of the 32-member Q1 ensemble workload after n_steps RK4
    steps from its seeded initial field: (time, field, node-active mask)."""
    from adamantine_b200.workloads import ensemble_q1, initial_temperature

    configs, _ = ensemble_q1()
    cfg = configs[k]
    o = _oracle(cfg, n_threads)
    y = np.ascontiguousarray(initial_temperature(cfg, f"ensemble-{k}"), np.float64).reshape(-1).copy()
    t = 0.0
    for _ in range(n_steps):
        t = o.evolve_one_time_step(t, dt, y)
    return t, y, o.node_active().astype(bool)


def adjoint_misfit(theta, targets, n_threads: int):
    """The misfit of the 64x64x32 Q2 adjoint workload (200 RK2 steps of
    1e-6, observations at steps 50/100/150/200 of the 500 seeded interior
    nodes) from the oracle forward at parameters theta."""
    from adamantine_b200.adjoint import config_at
    from adamantine_b200.workloads import adjoint_q2, initial_temperature, interior_points

    cfg = adjoint_q2()
    T0 = initial_temperature(cfg, "adjoint")
    pts = interior_points(cfg)
    nx, ny, _ = cfg.geometry.node_shape(2)
    idx = pts[:, 0] + nx * (pts[:, 1] + ny * pts[:, 2])
    obs = [50, 100, 150, 200]
    o = _oracle(config_at(cfg, theta), n_threads)
    y = np.ascontiguousarray(T0, np.float64).reshape(-1).copy()
    t, J = 0.0, 0.0
    for n in range(1, 201):
        t = o.evolve_one_time_step(t, 1e-6, y)
        if n in obs:
            J += float(np.sum((y[idx] - targets[obs.index(n)]) ** 2))
    return J


def pool(n_workers: int):
    return cf.ProcessPoolExecutor(max_workers=n_workers, mp_context=mp.get_context("spawn"))


def cores() -> int:
    return os.cpu_count() or 1
