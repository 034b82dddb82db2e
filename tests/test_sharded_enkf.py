"""The sharded EnKF exchange (adamantine_b200.sharded) on two gloo ranks on
CPU, with numpy steps, against the single-process restatement of the
reference's update on all members."""
import os
import socket

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

from enkf_oracle import enkf_analysis

WORLD = 2


def problem():
    rng = np.random.default_rng(11)
    N, n_state, stride, m, p = 8, 300, 304, 40, 2
    states = 300.0 + rng.normal(0, 20.0, (N, stride))
    params = np.stack([np.exp(rng.normal(0, 0.1, N)), 0.35 * np.exp(rng.normal(0, 0.1, N))], axis=1)
    idx = np.stack([rng.choice(n_state, m, replace=False) for _ in range(N)]).astype(np.int64)
    obs = 300.0 + rng.normal(0, 20.0, m)
    var = np.full(m, 25.0)
    pert = rng.normal(0, 5.0, (N, m))
    mask = (rng.uniform(size=(N, n_state)) > 0.2).astype(np.uint8)
    return states, params, idx, obs, var, pert, mask, n_state


def worker(rank, port, out):
    import sys

    here = os.path.dirname(os.path.abspath(__file__))
    for pth in (here, os.path.join(os.path.dirname(here), "oracle"), os.path.dirname(here)):
        sys.path.insert(0, pth)
    from sharded_steps import NumpySteps

    from adamantine_b200.sharded import ShardedAnalysis

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=WORLD)
    states, params, idx, obs, var, pert, mask, n_state = problem()
    nl = states.shape[0] // WORLD
    sl = slice(rank * nl, (rank + 1) * nl)
    X = torch.from_numpy(states[sl].copy())
    P = torch.from_numpy(params[sl].copy())
    ShardedAnalysis(NumpySteps())(X, n_state, torch.from_numpy(idx[sl]), torch.from_numpy(obs),
                                  torch.from_numpy(pert), obs_var=torch.from_numpy(var), params=P,
                                  update_mask=torch.from_numpy(mask[sl]))
    np.save(os.path.join(out, f"x{rank}.npy"), X.numpy())
    np.save(os.path.join(out, f"p{rank}.npy"), P.numpy())
    dist.barrier()
    dist.destroy_process_group()


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_rank_exchange_equals_dense_analysis(tmp_path):
    mp.spawn(worker, args=(free_port(), str(tmp_path)), nprocs=WORLD, join=True)
    states, params, idx, obs, var, pert, mask, n_state = problem()
    ref, ref_p = enkf_analysis(states, n_state, idx, obs, pert, obs_var=var, params=params, update_mask=mask)
    X = np.concatenate([np.load(os.path.join(tmp_path, f"x{r}.npy")) for r in range(WORLD)])
    P = np.concatenate([np.load(os.path.join(tmp_path, f"p{r}.npy")) for r in range(WORLD)])
    assert np.allclose(X, ref, rtol=1e-12, atol=1e-9)
    assert np.allclose(P, ref_p, rtol=1e-12, atol=1e-12)
    assert not np.allclose(X, states)


def loc_problem():
    """A 10 x 6 x 5 node grid (pitch 10), 24 observations at nodes shared by
    every member, Gaspari-Cohn localization with a cutoff of 3 spacings."""
    rng = np.random.default_rng(12)
    N, nodes, m, p = 8, (10, 6, 5), 24, 2
    n_state = nodes[0] * nodes[1] * nodes[2]
    spacing = np.array([0.5, 0.5, 0.25])
    a, b, c = np.meshgrid(np.arange(nodes[0]), np.arange(nodes[1]), np.arange(nodes[2]), indexing="ij")
    pts = np.zeros((n_state, 3))
    idx_all = (a + nodes[0] * (b + nodes[1] * c)).reshape(-1)
    pts[idx_all] = np.stack([a.reshape(-1), b.reshape(-1), c.reshape(-1)], axis=1) * spacing
    states = 300.0 + rng.normal(0, 20.0, (N, n_state))
    params = np.stack([np.exp(rng.normal(0, 0.1, N)), 0.35 * np.exp(rng.normal(0, 0.1, N))], axis=1)
    idx = np.tile(rng.choice(n_state, m, replace=False).astype(np.int64), (N, 1))
    obs = 300.0 + rng.normal(0, 20.0, m)
    var = np.full(m, 25.0)
    pert = rng.normal(0, 5.0, (N, m))
    return states, params, idx, obs, var, pert, n_state, pts, 1.5


def worker_localized(rank, port, out):
    import sys

    here = os.path.dirname(os.path.abspath(__file__))
    for pth in (here, os.path.join(os.path.dirname(here), "oracle"), os.path.dirname(here)):
        sys.path.insert(0, pth)
    from enkf_oracle import LOC_GASPARI_COHN, localization_weights
    from sharded_steps import NumpySteps

    from adamantine_b200.sharded import ShardedAnalysis

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=WORLD)
    states, params, idx, obs, var, pert, n_state, pts, cutoff = loc_problem()
    opts = pts[idx[0]]
    d_oo = np.linalg.norm(opts[:, None] - opts[None], axis=-1)
    d_so = np.linalg.norm(pts[:, None] - opts[None], axis=-1)
    loc = (localization_weights(d_oo, cutoff, LOC_GASPARI_COHN), localization_weights(d_so, cutoff, LOC_GASPARI_COHN))
    nl = states.shape[0] // WORLD
    sl = slice(rank * nl, (rank + 1) * nl)
    X = torch.from_numpy(states[sl].copy())
    P = torch.from_numpy(params[sl].copy())
    ShardedAnalysis(NumpySteps(loc))(X, n_state, torch.from_numpy(idx[sl]), torch.from_numpy(obs),
                                     torch.from_numpy(pert), obs_var=torch.from_numpy(var), params=P)
    np.save(os.path.join(out, f"x{rank}.npy"), X.numpy())
    np.save(os.path.join(out, f"p{rank}.npy"), P.numpy())
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_localized_exchange_equals_localized_analysis(tmp_path):
    from enkf_oracle import LOC_GASPARI_COHN, enkf_analysis_localized
    mp.spawn(worker_localized, args=(free_port(), str(tmp_path)), nprocs=WORLD, join=True)
    states, params, idx, obs, var, pert, n_state, pts, cutoff = loc_problem()
    ref, ref_p = enkf_analysis_localized(states, n_state, pts, idx, obs, pert, cutoff, LOC_GASPARI_COHN,
                                         obs_var=var, params=params)
    X = np.concatenate([np.load(os.path.join(tmp_path, f"x{r}.npy")) for r in range(WORLD)])
    P = np.concatenate([np.load(os.path.join(tmp_path, f"p{r}.npy")) for r in range(WORLD)])
    assert np.allclose(X, ref, rtol=1e-12, atol=1e-9)
    assert np.allclose(P, ref_p, rtol=1e-12, atol=1e-12)
    plain, _ = enkf_analysis(states, n_state, idx, obs, pert, obs_var=var, params=params)
    assert not np.allclose(X, plain)  # the localization changes the update


def worker_lost_rank(rank, port, out):
    """Rank 1 leaves before the analysis; rank 0's collective must end with an
    error (short process-group timeout), not wait for ever."""
    import datetime
    import sys

    here = os.path.dirname(os.path.abspath(__file__))
    for pth in (here, os.path.join(os.path.dirname(here), "oracle"), os.path.dirname(here)):
        sys.path.insert(0, pth)
    from sharded_steps import NumpySteps

    from adamantine_b200.sharded import ShardedAnalysis

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=WORLD, timeout=datetime.timedelta(seconds=10))
    if rank == 1:
        return  # the rank dies between steps, with nothing in flight
    states, params, idx, obs, var, pert, mask, n_state = problem()
    nl = states.shape[0] // WORLD
    outcome = "completed"
    try:
        ShardedAnalysis(NumpySteps())(torch.from_numpy(states[:nl].copy()), n_state, torch.from_numpy(idx[:nl]),
                                      torch.from_numpy(obs), torch.from_numpy(pert), obs_var=torch.from_numpy(var))
    except Exception as e:  # noqa: BLE001 -- any collective error is the expected outcome
        outcome = "error: " + type(e).__name__
    with open(os.path.join(out, "outcome.txt"), "w") as fh:
        fh.write(outcome)


def test_lost_rank_ends_the_analysis_with_an_error(tmp_path):
    import time

    t0 = time.time()
    mp.spawn(worker_lost_rank, args=(free_port(), str(tmp_path)), nprocs=WORLD, join=True)
    outcome = open(os.path.join(tmp_path, "outcome.txt")).read()
    assert outcome.startswith("error"), outcome
    assert time.time() - t0 < 120


def worker_uneven(rank, port, out):
    import sys

    here = os.path.dirname(os.path.abspath(__file__))
    for pth in (here, os.path.join(os.path.dirname(here), "oracle"), os.path.dirname(here)):
        sys.path.insert(0, pth)
    from sharded_steps import NumpySteps

    from adamantine_b200.sharded import ShardedAnalysis

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=WORLD)
    states, params, idx, obs, var, pert, mask, n_state = problem()
    sl = slice(0, 3) if rank == 0 else slice(3, 8)  # 3 and 5 members
    outcome = "ok"
    try:
        ShardedAnalysis(NumpySteps())(torch.from_numpy(states[sl].copy()), n_state, torch.from_numpy(idx[sl]),
                                      torch.from_numpy(obs), torch.from_numpy(pert), obs_var=torch.from_numpy(var))
    except ValueError as e:
        outcome = "ValueError: " + str(e)
    with open(os.path.join(out, f"uneven{rank}.txt"), "w") as fh:
        fh.write(outcome)
    dist.barrier()
    dist.destroy_process_group()


def test_uneven_member_counts_are_rejected_on_every_rank(tmp_path):
    mp.spawn(worker_uneven, args=(free_port(), str(tmp_path)), nprocs=WORLD, join=True)
    for r in range(WORLD):
        outcome = open(os.path.join(tmp_path, f"uneven{r}.txt")).read()
        assert outcome.startswith("ValueError") and "from 3 to 5" in outcome, outcome
