"""Benchmark of the thermal hot path (one JSON line on stdout, rank 0).

Workload (default): the FP64 Q2 heat operator of the phase-change problem at
production size -- 20x20x10 mm, 128x128x64 cells, FE_Q(2) (8,520,321 DoFs),
three material states with powder in the top 16 layers, a 400 W Goldak beam
on a seeded serpentine.  One step = one ThermalOperator::vmult (operator
application with its per-quadrature-point phase update) on device-resident
vectors; value = DoFs / vmult time in GDoF/s.  Two src/dst pairs alternate so
the working set (272 MB) exceeds the 126 MB L2 between timed iterations.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

--impl reference times the reference's CPU algorithm (the oracle restatement
in oracle/, the reference itself cannot be built here) on all host cores.
Multi-GPU runs are independent replicas of the single-mesh problem (the
operator does not shard); value is the sum over ranks with max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "heat vmult GDoF/s (FP64 Q2) & %HBM peak; batched-ensemble vs looped steps/s"
SCHEDULE_NAMES = ("coloured", "atomic", "two_pass")
WORKLOAD = "phase_change_q2_128x128x64_vmult"


# FP64 work of one Q2 cell of this workload: 876 DFMA + 432 DMUL + 63 DADD
# thread instructions per cell (ncu smsp__sass_thread_inst_executed_op_d*
# counts of tile_kernel<2,3,2,1,0> on the 128x128x32 case) = 2247 FLOP.
FP64_FLOP_PER_Q2_CELL = 2247

# DRAM bytes (read + write) of one vmult of the 128x128x64 workload from ncu
# captures (dram__bytes_read.sum + dram__bytes_write.sum): the atomic
# schedule's tile-kernel launch and the two-pass schedule's tile and gather
# launches of back-to-back vmults (the autotuner's timed trials) with
# --cache-control none (L2 as the vmult loop leaves it; means over 7
# launches), and the sum over the 8 colour
# launches of the coloured schedule (L2 flushed before every launch, so
# re-reads that stay in L2 in the timed loop are counted).
DRAM_BYTES_PER_VMULT_FULL = {"atomic": 189.9e6, "two_pass": 286.1e6, "coloured": 327.0e6}
TRAFFIC_NOTE = {"atomic": "ncu --cache-control none, the tile-kernel launch of back-to-back vmults",
                "two_pass": "ncu --cache-control none, tile + gather launches of back-to-back vmults",
                "coloured": "ncu, L2 flushed before each of the 8 colour launches"}
# per schedule: the dominant kernel of one vmult, its launch pattern, and
# the number of kernel launches of one vmult of this workload (one source):
# the beam preparation (folded into the zeroing launch in the atomic
# schedule) and the operator's launches
KERNELS = {"coloured": ("adm::tile_kernel<2,3,2,0,0>", "8 colour launches", 1 + 8),
           "atomic": ("adm::tile_kernel<2,3,2,1,0>", "1 launch after adm::zero_keep_kernel", 2),
           "two_pass": ("adm::tile_kernel<2,3,2,2,0> + adm::two_pass_gather_kernel<2>",
                        "1 tile launch + 1 gather launch", 1 + 2)}


def fp64_fma_peak(device):
    """Measured FP64 FMA throughput (TFLOP/s) of the GPU, from the library's
    diagnostic microbenchmark."""
    import ctypes

    from adamantine_b200 import _lib

    L = _lib.load()
    fn = L.adm_diag_fp64_fma_rate
    fn.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_double)]
    fn.restype = ctypes.c_int
    out = ctypes.c_double(0.0)
    _lib.check(fn(device, ctypes.byref(out)))
    return out.value


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """Samples the SM clock, its maximum and the active clock-event (throttle)
    reasons during the timed region -- the fields of nvidia-smi's
    clocks.sm, clocks.max.sm and clocks_event_reasons.* -- through NVML in
    this process every 20 ms (a forked nvidia-smi could stall the launching
    thread inside a region of a few milliseconds); nvidia-smi when NVML is
    not importable."""

    QUERY = ("uuid,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, uuid):
        self.uuid = uuid
        self.samples = []  # (sm MHz, max sm MHz, set of active reason names)
        self._stop = threading.Event()
        self._thr = None
        self._nvml = None
        self._handle = None
        try:
            import pynvml

            pynvml.nvmlInit()
            self._nvml = pynvml
            want = uuid.replace("GPU-", "") if uuid else ""
            for i in range(pynvml.nvmlDeviceGetCount()):
                h = pynvml.nvmlDeviceGetHandleByIndex(i)
                u = pynvml.nvmlDeviceGetUUID(h)
                u = u.decode() if isinstance(u, bytes) else u
                if not want or want in u:
                    self._handle = h
                    break
        except Exception:
            self._nvml = None

    def _sample_nvml(self):
        n, h = self._nvml, self._handle
        sm = n.nvmlDeviceGetClockInfo(h, n.NVML_CLOCK_SM)
        smax = n.nvmlDeviceGetMaxClockInfo(h, n.NVML_CLOCK_SM)
        bits = n.nvmlDeviceGetCurrentClocksEventReasons(h)
        masks = (n.nvmlClocksEventReasonHwSlowdown, n.nvmlClocksEventReasonHwThermalSlowdown,
                 n.nvmlClocksEventReasonSwThermalSlowdown, n.nvmlClocksEventReasonSwPowerCap)
        self.samples.append((float(sm), float(smax), {nm for nm, m in zip(self.NAMES, masks) if bits & m}))

    def _sample_smi(self):
        out = subprocess.run(["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits"],
                             capture_output=True, text=True, timeout=5).stdout
        for line in out.strip().splitlines():
            f = [x.strip() for x in line.split(",")]
            if self.uuid and self.uuid not in f[0]:
                continue
            if f[1].replace(".", "").isdigit() and f[2].replace(".", "").isdigit():
                act = {nm for nm, v in zip(self.NAMES, f[5:9]) if v.strip().lower() in ("active", "1", "yes")}
                self.samples.append((float(f[1]), float(f[2]), act))

    def _run(self):
        while not self._stop.is_set():
            try:
                if self._handle is not None:
                    self._sample_nvml()
                else:
                    self._sample_smi()
            except Exception:
                pass
            self._stop.wait(0.02 if self._handle is not None else 0.2)

    def __enter__(self):
        self._thr = threading.Thread(target=self._run, daemon=True)
        self._thr.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        self._thr.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        reasons = set()
        for _, _, act in self.samples:
            reasons |= act
        return {"sm_mhz": statistics.median(s[0] for s in self.samples),
                "sm_max_mhz": max(s[1] for s in self.samples), "reasons": sorted(reasons),
                "samples": len(self.samples), "source": "NVML" if self._handle is not None else "nvidia-smi"}


SIZES = {"full": ((128, 128, 64), (20e-3, 20e-3, 10e-3), 16),
         # smaller cases of the same problem for profiler captures
         "medium": ((128, 128, 32), (20e-3, 20e-3, 5e-3), 8),
         "small": ((64, 64, 32), (10e-3, 10e-3, 5e-3), 8)}


def build_workload(size="full"):
    from adamantine_b200.workloads import initial_temperature, phase_change_q2

    n_cells, extent, powder = SIZES[size]
    cfg = phase_change_q2(n_cells=n_cells, extent=extent, powder_layers=powder)
    T = initial_temperature(cfg, "bench")
    return cfg, T


def cpu_vmult_rate(cfg, T, n_threads, budget_s=20.0, max_steps=5, keep_result=False):
    """Times the oracle's vmult (reference CPU algorithm) on the host: median
    of max_steps applications after one warm-up (fewer if budget_s runs
    out). With keep_result, also returns the first application's output."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle_py

    cfg.n_threads = n_threads
    st = cfg.to_struct()
    geo = cfg.geometry
    o = oracle_py.Oracle(st, active=geo.active_cells(), initial_state=geo.initial_state())
    o.set_time(1e-4)
    src = np.ascontiguousarray(T.reshape(-1))
    dst = np.zeros_like(src)
    o.vmult_add(dst, src)  # warm-up
    first = dst.copy() if keep_result else None
    times = []
    t_start = time.perf_counter()
    for _ in range(max_steps):
        dst[:] = 0.0
        t0 = time.perf_counter()
        o.vmult_add(dst, src)
        times.append(time.perf_counter() - t0)
        if time.perf_counter() - t_start > budget_s:
            break
    n_dofs = int(np.prod(geo.node_shape(cfg.degree)))
    med = statistics.median(times)
    if keep_result:
        return n_dofs / med / 1e9, med, len(times), first
    return n_dofs / med / 1e9, med, len(times)


def workload_config(size, world):
    """The workload description both --impl arms print (identical dicts)."""
    cfg_size = SIZES[size][0]
    n_dofs = (2 * cfg_size[0] + 1) * (2 * cfg_size[1] + 1) * (2 * cfg_size[2] + 1)
    return {"workload": WORKLOAD if size == "full" else WORKLOAD + "_" + size,
            "mesh": "x".join(map(str, cfg_size)) + " Q2", "dofs": n_dofs, "states": "solid/liquid/powder",
            "source": "Goldak 400 W", "parallelism": f"replicas x{world}"}


ENSEMBLE_WORKLOAD = "ensemble_q1_64x64x32_32members_rk4_100steps"


def run_ensemble(args, dist, local_rank):
    """Batched vs looped member-steps/s of the 32-member Q1 ensemble (ragged
    deposited heights, perturbed conductivity and absorptivity), 100 RK4
    steps of dt = 1e-6 each arm from the same start, then one EnKF analysis
    against 2000 top-surface observations (sigma = 5 K) on the augmented
    state [T; k_scale; absorptivity]."""
    import torch

    from adamantine_b200.ensemble import EnKF, Ensemble
    from adamantine_b200.workloads import ensemble_q1, initial_temperature, rng_for, surface_observations

    world = dist.get_world_size() if dist else 1
    rank = dist.get_rank() if dist else 0
    # members per GPU fixed; rank r holds its own seeded members
    configs, params = ensemble_q1(name="ensemble_q1" if rank == 0 else f"ensemble_q1-rank{rank}")
    n = len(configs)
    grids = [initial_temperature(c, f"ensemble-{k}") for k, c in enumerate(configs)]
    e = Ensemble(configs, device=local_rank)
    y0 = e.from_grids(grids)
    steps, dt = 100, 1e-6
    schedule, _ = e.autotune(y0, dt)
    stream = e.stream
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
    # warm-up (graph capture, first launches of every kernel)
    yw = y0.clone()
    e.evolve_n_steps(0.0, dt, 3, yw)
    e.evolve_looped(0.0, dt, yw)
    torch.cuda.synchronize()
    yb = y0.clone()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ev[0].record(stream)
    e.evolve_n_steps(0.0, dt, steps, yb)
    ev[1].record(stream)
    ev[1].synchronize()
    ms_b = ev[0].elapsed_time(ev[1])
    # the loop over members, each through its own single-member launches:
    # with the shipped default schedule (coloured) and with the atomic one
    looped = {}
    for name_s, sch in (("coloured", 0), ("atomic", 1)):
        e.set_schedule(sch)
        yl = y0.clone()
        e.evolve_looped(0.0, dt, yl)  # warm-up of this schedule
        yl = y0.clone()
        torch.cuda.synchronize()
        ev[2].record(stream)
        t = 0.0
        for _ in range(steps):
            t = e.evolve_looped(t, dt, yl)
        ev[3].record(stream)
        ev[3].synchronize()
        looped[name_s] = (ev[2].elapsed_time(ev[3]),
                          float(((yb - yl).abs().max() / yl.abs().max()).item()))
    e.set_schedule(schedule)
    ms_l = looped["coloured"][0]
    identical = looped["coloured"][1] == 0.0 and looped["atomic"][1] == 0.0
    max_rel_diff = max(v[1] for v in looped.values())
    assert e.device_error() == 0
    # the fair member loop: every member through its own single-member
    # handle and adm_evolve_n_steps (one CUDA graph per step), with the
    # launch schedule the single-member autotuner picks on member 0 and the
    # FE_Q(1) kernel variant that runs the loop fastest (each timed; the
    # autotuner's vmult timing need not pick the fastest for whole steps)
    from adamantine_b200.thermal import ThermalPhysics

    singles = [ThermalPhysics(c, device=local_rank, stream=stream) for c in configs]
    ys = [singles[k].from_grid(grids[k]) for k in range(n)]
    single_schedule, _ = singles[0].autotune(ys[0])
    loop_ms = {}
    for cz in (1, 2, 4):
        for k, g in enumerate(singles):  # warm-up: graph capture of every handle
            g.set_schedule(single_schedule)
            g.set_cells_per_thread(cz)
            g.evolve_n_steps(0.0, dt, 2, ys[k].clone())
        ys = [singles[k].from_grid(grids[k]) for k in range(n)]
        torch.cuda.synchronize()
        ev[2].record(stream)
        for k in range(n):
            singles[k].evolve_n_steps(0.0, dt, steps, ys[k])
        ev[3].record(stream)
        ev[3].synchronize()
        loop_ms[cz] = ev[2].elapsed_time(ev[3])
    single_cz = min(loop_ms, key=loop_ms.get)
    ms_g = loop_ms[single_cz]
    graph_loop_diff = max(float(((yb[k] - ys[k]).abs().max() / ys[k].abs().max()).item()) for k in range(n))
    assert all(g.device_error() == 0 for g in singles)
    del singles, ys
    # EnKF analysis on the forecast (member-specific top-surface node maps)
    layers = [p[2] for p in params]
    ij, sigma = surface_observations(e.nodes[:2], layers)
    idx = np.stack([e.node_index(ij[:, 0], ij[:, 1], layers[k]) for k in range(n)]).astype(np.int64)
    rng = rng_for("ensemble-analysis")
    truth = 300.0 + 50.0 * rng.uniform(0.0, 1.0, idx.shape[1])
    obs = truth + rng.normal(0.0, sigma, idx.shape[1])
    pert = rng.normal(0.0, sigma, (n * world, idx.shape[1]))  # all members, same on every rank
    dev = yb.device
    P = torch.tensor([[p[0], p[1]] for p in params], dtype=torch.float64, device=dev)
    enkf = EnKF(device=local_rank)
    var = torch.full((idx.shape[1],), sigma * sigma, dtype=torch.float64, device=dev)
    obs_d, idx_d, pert_d = (torch.tensor(obs, device=dev), torch.tensor(idx, device=dev),
                            torch.tensor(pert, device=dev))
    # the same analysis with Gaspari-Cohn localization (cutoff 1 mm, about
    # three cells), observation points at member 0's observed nodes
    enkf_loc = EnKF(device=local_rank)
    enkf_loc.set_localization("gaspari_cohn", LOC_CUTOFF, e.node_points(idx[0]), e.grid())
    # step function: H P H^T + R may be indefinite, solved by pivoted LU
    enkf_step = EnKF(device=local_rank)
    enkf_step.set_localization("step_function", LOC_CUTOFF, e.node_points(idx[0]), e.grid())
    if world > 1:
        from adamantine_b200.sharded import LibrarySteps, ShardedAnalysis

        sharded = ShardedAnalysis(LibrarySteps(enkf))
        sharded_loc = ShardedAnalysis(LibrarySteps(enkf_loc))
        sharded_step = ShardedAnalysis(LibrarySteps(enkf_step))

        def analysis(Y, Pk):
            sharded(Y, e.stride, idx_d, obs_d, pert_d, obs_var=var, params=Pk)

        def analysis_loc(Y, Pk):
            sharded_loc(Y, e.stride, idx_d, obs_d, pert_d, obs_var=var, params=Pk)

        def analysis_step(Y, Pk):
            sharded_step(Y, e.stride, idx_d, obs_d, pert_d, obs_var=var, params=Pk)
    else:

        def analysis(Y, Pk):
            enkf.analysis(Y, e.stride, idx_d, obs_d, pert_d, obs_var=var, params=Pk)

        def analysis_loc(Y, Pk):
            enkf_loc.analysis(Y, e.stride, idx_d, obs_d, pert_d, obs_var=var, params=Pk)

        def analysis_step(Y, Pk):
            enkf_step.analysis(Y, e.stride, idx_d, obs_d, pert_d, obs_var=var, params=Pk)

    def timed(fn):
        fn(yb.clone(), P.clone())  # warm-up
        ya, pa = yb.clone(), P.clone()
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        ev[0].record(stream)
        fn(ya, pa)
        ev[1].record(stream)
        ev[1].synchronize()
        return ev[0].elapsed_time(ev[1])

    ms_a = timed(analysis)
    ms_al = timed(analysis_loc)
    ms_as = timed(analysis_step)
    ms_la = looped["atomic"][0]
    if dist:
        tt = torch.tensor([ms_b, ms_l, ms_la, ms_a, ms_al, ms_as, ms_g], device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms_b, ms_l, ms_la, ms_a, ms_al, ms_as, ms_g = (float(x) for x in tt.tolist())
    return {
        "workload": ENSEMBLE_WORKLOAD, "members_per_gpu": n, "steps": steps, "dt": dt,
        "active_layers": [min(layers), max(layers)],
        "batched_member_steps_per_s": world * n * steps / (ms_b * 1e-3),
        # headline: against each member through its own graph-captured
        # single-member path with the single-member autotuner's schedule
        "looped_member_steps_per_s": world * n * steps / (ms_g * 1e-3),
        "speedup": ms_g / ms_b, "batched_ms_per_step": ms_b / steps, "looped_ms_per_step": ms_g / steps,
        "looped_path": "32 single-member handles, adm_evolve_n_steps (one CUDA graph per step), "
                       f"{SCHEDULE_NAMES[single_schedule]} schedule (single-member autotuner), "
                       f"{single_cz} cell(s) per thread (the fastest loop)",
        "looped_ms_per_step_by_cells_per_thread": {str(k): v / steps for k, v in loop_ms.items()},
        "max_rel_diff_batched_vs_graph_loop": graph_loop_diff,
        "per_step_loop": {"coloured_member_steps_per_s": world * n * steps / (ms_l * 1e-3),
                          "atomic_member_steps_per_s": world * n * steps / (ms_la * 1e-3),
                          "speedup_vs_coloured": ms_l / ms_b, "speedup_vs_atomic": ms_la / ms_b,
                          "path": "adm_ensemble_evolve_looped: each member's stages launched one by one"},
        "bit_identical_to_loops": identical, "max_rel_diff_batched_vs_looped": max_rel_diff,
        "bit_identity_note": "the atomic schedule's FP64 reductions round in launch order; the coloured and "
                             "two-pass schedules give batched = looped bit for bit (tests/test_gpu_ensemble.py, "
                             "tests/test_gpu_schedule.py)",
        "batched_schedule": SCHEDULE_NAMES[schedule],
        "batched_cells_per_thread": e.cells_per_thread(),
        "batched_path": "one CUDA graph per step (4 stages)",
        "work_items_per_sweep": e.n_work_items(),
        "enkf_analysis_ms": ms_a, "n_obs": int(idx.shape[1]), "augmented_params": 2,
        "enkf_localized_analysis_ms": ms_al, "enkf_step_localized_analysis_ms": ms_as,
        "localization": f"gaspari_cohn (Cholesky) and step_function (pivoted LU), cutoff {LOC_CUTOFF * 1e3:g} mm",
        "analysis_members": n * world,
        "analysis_path": "fused (one GPU)" if world == 1 else "sharded: all-gather HX, all-reduce sums, "
                                                            "reduce-scatter member updates (NCCL)",
    }


ADJOINT_WORKLOAD = "adjoint_q2_64x64x32_rk2_200steps"
LOC_CUTOFF = 1.0e-3


def run_adjoint(args, local_rank):
    """Adjoint gradient of the misfit at 500 interior points after steps
    50/100/150/200 (RK2, dt = 1e-6, 64x64x32 Q2) with respect to conductivity
    scale, specific-heat scale, absorptivity and power, with the checkpoint
    interval chosen from the free device memory (every stage kept when the
    stores fit): time of one gradient over the time of one forward run, the
    agreement with central differences (h = 1e-5 relative) of the forward,
    and the same with a checkpoint every 20 steps (the low-memory mode)."""
    import torch

    from adamantine_b200.adjoint import AdjointProblem
    from adamantine_b200.workloads import adjoint_q2, initial_temperature, interior_points, rng_for

    cfg = adjoint_q2()
    T0 = initial_temperature(cfg, "adjoint")
    pts = interior_points(cfg, n_points=500)
    obs = [50, 100, 150, 200]
    prob = AdjointProblem(cfg, T0, 0.0, 1e-6, 200, obs, pts, device=local_rank, checkpoint_every=0)
    schedule, _ = prob.phys.autotune(prob.y0)
    truth = (1.0, 1.0, 0.35, 400.0)
    prob.set_targets(prob.observe(truth))
    f = np.exp(rng_for("adjoint-perturbation").uniform(np.log(0.9), np.log(1.1), 4))
    theta = tuple(float(a * b) for a, b in zip(truth, f))
    def timed(fn, reps=3):
        """median wall-clock seconds of reps synchronized calls, and the last result"""
        ts, out = [], None
        for _ in range(reps):
            torch.cuda.synchronize()
            t = time.perf_counter()
            out = fn()
            torch.cuda.synchronize()
            ts.append(time.perf_counter() - t)
        return float(np.median(ts)), out

    prob.objective(theta)  # warm-up
    prob.gradient(theta)
    fwd_s, J = timed(lambda: prob.objective(theta))
    grad_s, (Jg, grad) = timed(lambda: prob.gradient(theta))
    fd = np.zeros(4)
    h = 1e-5
    for k in range(4):
        tp, tm = list(theta), list(theta)
        tp[k] *= 1 + h
        tm[k] *= 1 - h
        fd[k] = (prob.objective(tp) - prob.objective(tm)) / (2 * h * theta[k])
    rel = np.abs(grad - fd) / np.maximum(np.abs(fd), 1e-300)
    k_auto = prob.last_checkpoint_interval()
    # the same gradient with a checkpoint every 20 steps (9 of 10 segments
    # recomputed: the mode for runs whose stores do not fit)
    prob.checkpoint_every = 20
    prob.gradient(theta)  # warm-up
    fwd20_s, _ = timed(lambda: prob.objective(theta))
    grad20_s, (_, grad_20) = timed(lambda: prob.gradient(theta))
    prob.checkpoint_every = 0
    same = float(np.max(np.abs(grad_20 - grad) / np.maximum(np.abs(grad), 1e-300)))
    return {
        "workload": ADJOINT_WORKLOAD, "theta": list(theta), "J": J, "gradient": grad.tolist(),
        "fd_gradient": fd.tolist(), "fd_max_rel_err": float(rel.max()), "fd_h": h,
        "forward_ms": 1e3 * fwd_s, "gradient_ms": 1e3 * grad_s,
        "cost_ratio": grad_s / fwd_s, "checkpoint_every": k_auto,
        "checkpoint_policy": "auto: the longest segment whose stores fit in half of the free HBM "
                             "(3.5 GB of stage inputs and 11 GB of powder states for the whole run here)",
        "timing": "host wall clock, synchronized, median of 3", "forward_schedule": SCHEDULE_NAMES[schedule],
        "checkpoint_every_20": {"forward_ms": 1e3 * fwd20_s, "gradient_ms": 1e3 * grad20_s,
                                "cost_ratio": grad20_s / fwd20_s, "checkpoint_every": 20,
                                "max_rel_diff_vs_auto": same},
    }


DEPOSITION_WORKLOAD = "deposition_q2_256x256x128_rk4"


RK4_WORKLOAD = "phase_change_q2_128x128x64_rk4_step"


def run_rk4_steps(args, local_rank):
    """The time step the operator serves: RK4 steps of dt = 5e-7 on the
    128x128x64 Q2 phase-change problem through adm_evolve_n_steps (one CUDA
    graph per step: per stage the heat-source state, the tile sweep with the
    fused inverse mass and stage update). GDoF/s counts four operator
    applications per step."""
    import torch

    from adamantine_b200.thermal import ThermalPhysics

    cfg, T = build_workload(args.size)
    g = ThermalPhysics(cfg, device=local_rank)
    n = g.m()
    n_dofs = int(np.prod(cfg.geometry.node_shape(cfg.degree)))
    y = g.from_grid(T)
    schedule, sched_ms = g.autotune(y)
    dt = 5e-7
    t = g.evolve_n_steps(0.0, dt, 3, y)  # warm-up: graph capture
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(g.stream)
    t = g.evolve_n_steps(t, dt, args.rk4_steps, y)
    e1.record(g.stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / args.rk4_steps
    assert g.device_error() == 0
    # node-vector bytes a fused RK4 step must move (8 B per node per read or
    # write): stage 1 reads y (its input) and the inverse mass and writes the
    # next stage input and the running sum (32 B); stages 2-3 read their
    # input, the inverse mass and y, read and write the running sum and write
    # the next input (48 B each); stage 4 reads its input, the inverse mass,
    # y and the running sum and writes y (40 B); plus 13 B of cell data per
    # cell and stage
    alg = 168 * n + 4 * 13 * g.n_cells
    peak, kind = measured_peaks()
    return {"workload": RK4_WORKLOAD, "steps": args.rk4_steps, "dt": dt, "ms_per_step": ms,
            "gdof_per_s": 4 * n_dofs / (ms * 1e-3) / 1e9, "steps_per_s": 1e3 / ms,
            "schedule": SCHEDULE_NAMES[schedule],
            "autotune_ms_per_vmult": dict(zip(SCHEDULE_NAMES, sched_ms)),
            "algorithmic_bytes_per_step": alg, "achieved_gbs": alg / (ms * 1e-3) / 1e9,
            "hbm_frac": alg / (ms * 1e-3) / 1e9 / peak, "peak_kind": f"{kind} hbm_gbs",
            "path": "adm_evolve_n_steps (CUDA graph per step)"}


def run_deposition(args, local_rank, with_cpu):
    """RK4 steps (dt = 2e-7) of the 67.6 M-node Q2 deposition workload with
    the driver's per-step activation of the deposition boxes; throughput as
    operator applications (4 per step) x nodes / time, the fused stages'
    algorithmic HBM bytes, and (with_cpu) the oracle's time for one RK4 step
    of the same problem on the host cores (the 20-step window is 20 x that)."""
    import torch

    from adamantine_b200.deposition import Deposition
    from adamantine_b200.thermal import ThermalPhysics
    from adamantine_b200.workloads import deposition_q2, initial_temperature

    cfg, boxes = deposition_q2()
    g = ThermalPhysics(cfg, device=local_rank)
    T0 = initial_temperature(cfg, "deposition", melt_pool=False)
    y = g.from_grid(T0)
    schedule, _ = g.autotune(y)
    dep = Deposition(g, boxes)
    n_nodes = int(np.prod(cfg.geometry.node_shape(2)))
    dt = 2e-7
    t = 0.0
    activated = 0
    for _ in range(3):  # warm-up (first activation, kernel first launches)
        activated += dep.step(t, dt, 300.0, y)
        t = g.evolve_one_time_step(t, dt, y)
    torch.cuda.synchronize()
    steps = args.deposition_steps
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    n_act = 0
    ev0.record(g.stream)
    for _ in range(steps):
        n_act += dep.step(t, dt, 300.0, y)
        t = g.evolve_one_time_step(t, dt, y)
    ev1.record(g.stream)
    ev1.synchronize()
    ms = ev0.elapsed_time(ev1)
    assert g.device_error() == 0
    # microstructure records around 5 more steps (save the field, step,
    # collect the liquidus crossings): host time of the two calls
    from adamantine_b200.microstructure import Microstructure

    micro = Microstructure(g)
    ms_micro, n_records = 0.0, 0
    for _ in range(5):
        dep.step(t, dt, 300.0, y)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        micro.set_old_temperature(y)
        torch.cuda.synchronize()
        ms_micro += 1e3 * (time.perf_counter() - t0)
        t = g.evolve_one_time_step(t, dt, y)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        n_records += len(micro.compute_G_and_R(y, dt))
        ms_micro += 1e3 * (time.perf_counter() - t0)
    micro.close()
    C = g.n_cells
    # fused RK4 stages: 32 + 48 + 48 + 40 bytes per node (stage input, inverse
    # mass, y, running sum, next stage vector) and 13 bytes per cell per stage
    bytes_step = 168 * g.m() + 4 * 13 * C
    out = {
        "workload": DEPOSITION_WORKLOAD, "nodes": n_nodes, "cells": C, "steps": steps, "steps_run": steps,
        "steps_config": 2000, "dt": dt,
        "ms_per_step": ms / steps, "gdofs_per_s": 4 * n_nodes * steps / (ms * 1e-3) / 1e9,
        "hbm_gbs_algorithmic": bytes_step * steps / (ms * 1e-3) / 1e9, "cells_activated": activated + n_act,
        "boxes": boxes.n, "activation": "device append list, driver window per step",
        "schedule": SCHEDULE_NAMES[schedule],
        "microstructure_ms_per_step": ms_micro / 5, "microstructure_records_per_step": n_records / 5,
    }
    if with_cpu:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle_py

        st = cfg.to_struct()
        o = oracle_py.Oracle(st, active=cfg.geometry.active_cells(), initial_state=cfg.geometry.initial_state())
        yr = np.ascontiguousarray(T0, np.float64).reshape(-1).copy()
        k_cpu = max(1, args.deposition_cpu_steps)
        tr = 0.0
        t0 = time.perf_counter()
        for _ in range(k_cpu):
            tr = o.evolve_one_time_step(tr, dt, yr)
        cpu_s = (time.perf_counter() - t0) / k_cpu
        out["cpu_baseline"] = {"seconds_per_step": cpu_s, "steps_timed": k_cpu,
                               "seconds_20_step_window": 20 * cpu_s,
                               "window_measured": k_cpu >= 20,
                               "cores": os.cpu_count() or 1, "kind": "port",
                               "sample": f"{k_cpu} RK4 step(s) of the workload (oracle, OpenMP); the 20-step "
                                         f"window is 20 x the mean step"
                                         + ("" if k_cpu >= 20 else " (extrapolated)")}
    return out


AMR_WORKLOAD = "amr_q2_64x64x8_2levels_rk4"


def run_amr(args, local_rank):
    """RK4 steps (dt = 1 us) of the refined-mesh workload after refine_mesh
    over a 100-step window (2 levels along the beam), against the same steps
    on the uniform grid of the finest resolution (256x256x32 Q2, CUDA-graph
    steps); also one moving-window refine_mesh with coarsening after the
    beam (refine_and_transfer: host mesh rebuild, level grids, transfer)."""
    import copy

    import torch

    from adamantine_b200.amr import AmrThermalPhysics
    from adamantine_b200.thermal import ThermalPhysics
    from adamantine_b200.workloads import amr_q2

    cfg, L = amr_q2()
    dt, K = 1e-6, 100
    g = AmrThermalPhysics(cfg, L, device=local_rank)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    g.refine_mesh(0.0, K * dt, K, L)
    torch.cuda.synchronize()
    first_remesh_ms = 1e3 * (time.perf_counter() - t0)
    leaves = g.leaves()
    per_level = [int((leaves[:, 0] == l).sum()) for l in range(L + 1)]
    t = 0.0
    for _ in range(3):
        t = g.evolve_one_time_step(t, dt)
    torch.cuda.synchronize()
    steps = args.amr_steps
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(g.stream)
    for _ in range(steps):
        t = g.evolve_one_time_step(t, dt)
    ev1.record(g.stream)
    ev1.synchronize()
    ms = ev0.elapsed_time(ev1)
    y = g.get_solution().cpu().numpy()
    n_dofs, n_nodes = g.n_dofs, g.n_nodes
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    g.refine_mesh(t, t + K * dt, K, L, True)
    torch.cuda.synchronize()
    remesh_ms = 1e3 * (time.perf_counter() - t0)
    remesh_phases = g.remesh_profile()
    g.close()
    # the uniform grid of the finest cells
    fine_cfg = copy.deepcopy(cfg)
    fine_cfg.geometry.n_cells = tuple(n << L for n in cfg.geometry.n_cells)
    f = ThermalPhysics(fine_cfg, device=local_rank)
    yf = f.from_grid(np.full(tuple(reversed(fine_cfg.geometry.node_shape(2))), 300.0))
    tf = f.evolve_n_steps(0.0, dt, 3, yf)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(f.stream)
    f.evolve_n_steps(tf, dt, steps, yf)
    e1.record(f.stream)
    e1.synchronize()
    ms_fine = e0.elapsed_time(e1)
    fine_nodes = int(np.prod(fine_cfg.geometry.node_shape(2)))
    return {
        "workload": AMR_WORKLOAD, "max_level": L, "leaves_per_level": per_level, "dofs": n_dofs,
        "hanging_nodes": n_nodes - n_dofs, "steps": steps, "dt": dt, "ms_per_step": ms / steps,
        "mdofs_per_s": 4 * n_dofs * steps / (ms * 1e-3) / 1e6, "peak_temperature": float(y.max()),
        "first_refine_mesh_ms": first_remesh_ms, "refine_mesh_ms": remesh_ms, "refine_mesh_phases_ms": remesh_phases,
        "uniform_fine": {"nodes": fine_nodes, "ms_per_step": ms_fine / steps, "path": "evolve_n_steps (graphs)"},
        "speedup_vs_uniform_fine": ms_fine / ms,
    }


MECHANICS_WORKLOAD = "eshelby_inclusion_64x64x64_q1"


def run_mechanics(args, local_rank):
    """The thermoelastic solve of the reference's Eshelby case (a 1 um
    inclusion 1 K warmer, alpha = 0.01, K = 160 GPa, G = 79 GPa, in a 40 um
    cube clamped on z-) on 64^3 FE_Q(1) cells: setup (cells, right-hand side,
    diagonal), one operator application and the CG solve to 1e-12 |rhs|
    with the multigrid preconditioner, then with the diagonal one (host wall
    clock, synchronized)."""
    import torch

    from adamantine_b200.config import Boundary, Geometry, ThermalConfig
    from adamantine_b200.mechanics import MechanicalPhysics
    from adamantine_b200.thermal import ThermalPhysics
    from adamantine_b200.workloads import steel_solid_material

    n, L, a = 64, 4.0e-5, 1.0e-6
    cfg = ThermalConfig(geometry=Geometry(dim=3, n_cells=(n, n, n), extent=(L, L, L)),
                        material=steel_solid_material(), boundary=Boundary.from_database({"type": "adiabatic"}, 3),
                        sources=[], degree=1, time_method="forward_euler")
    phys = ThermalPhysics(cfg, device=local_rank)
    x = np.linspace(0.0, L, n + 1)
    Z, Y, X = np.meshgrid(x, x, x, indexing="ij")
    dist = np.sqrt((X - 2e-5) ** 2 + (Y - 2e-5) ** 2 + (Z - 2e-5) ** 2)
    T = phys.from_grid(np.where(dist < a, 3.0, 2.0))
    mech = MechanicalPhysics(phys, 160.0e9 - 2.0 / 3.0 * 79.0e9, 79.0e9, 0.01, reference_temperatures=[2.0],
                             initial_temperature=2.0, gravity=False, clamped=("z-",))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    mech.setup_dofs(T)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    src = torch.rand(3 * phys.m(), dtype=torch.float64, device=phys.device)
    dst = torch.zeros_like(src)
    mech.vmult(dst, src)  # warm-up
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(phys.stream)
    for _ in range(10):
        mech.vmult(dst, src)
    e1.record(phys.stream)
    e1.synchronize()
    apply_ms = e0.elapsed_time(e1) / 10
    # multigrid (the default): the first solve also builds the level
    # hierarchy, the second reuses it
    t2 = time.perf_counter()
    mech.solve()
    torch.cuda.synchronize()
    t3 = time.perf_counter()
    u = mech.solve()
    torch.cuda.synchronize()
    t4 = time.perf_counter()
    levels, coarse = mech.multigrid_levels()
    it_mg, res_mg = mech.iterations, mech.residual
    mech.set_preconditioner("jacobi")
    t5 = time.perf_counter()
    uj = mech.solve()
    torch.cuda.synchronize()
    t6 = time.perf_counter()
    solve_ms = 1e3 * (t4 - t3)
    return {
        "workload": MECHANICS_WORKLOAD, "dofs": mech.n_dofs, "cells": mech.n_cells,
        "setup_ms": 1e3 * (t1 - t0), "apply_ms": apply_ms, "apply_mdofs_per_s": mech.n_dofs / apply_ms / 1e3,
        "cg_iterations": it_mg, "solve_ms": solve_ms, "first_solve_ms": 1e3 * (t3 - t2),
        "ms_per_iteration": solve_ms / max(1, it_mg), "residual": res_mg,
        "multigrid_levels": levels, "coarsest_dofs": coarse,
        "max_displacement": float(u.abs().max().item()),
        "jacobi": {"cg_iterations": mech.iterations, "solve_ms": 1e3 * (t6 - t5),
                   "max_rel_difference": float((u - uj).abs().max().item() / max(uj.abs().max().item(), 1e-300))},
        "speedup_vs_jacobi": (t6 - t5) / max(t4 - t3, 1e-12),
        "solver": "CG to 1e-12 |rhs| preconditioned by a geometric multigrid V-cycle (Chebyshev(3) smoothing, "
                  "FE_Q(1) levels, dense coarsest solve); the reference: AMG-preconditioned CG",
    }


def run_reference(args, rank, world):
    """--impl reference: the oracle's vmult on all host cores (rank 0 only)."""
    if rank != 0:
        return
    cfg, T = build_workload()
    n_threads = os.cpu_count() or 1
    rates = []
    for _ in range(args.warmup):
        cpu_vmult_rate(cfg, T, n_threads, budget_s=5.0, max_steps=1)
    t_all = time.perf_counter()
    for _ in range(args.steps):
        r, med, n = cpu_vmult_rate(cfg, T, n_threads, budget_s=30.0, max_steps=1)
        rates.append(r)
    elapsed = time.perf_counter() - t_all
    value = statistics.median(rates)
    n_dofs = int(np.prod(cfg.geometry.node_shape(cfg.degree)))
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "GDoF/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * n_dofs / value / 1e9,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded; no public dataset)", "config": workload_config("full", world),
        "cpu_baseline": {"value": value, "unit": "GDoF/s", "cores": n_threads, "kind": "port",
                         "sample": f"{args.steps} full vmults of the workload (C++/OpenMP restatement of the "
                                   f"reference CPU ThermalOperator::vmult), {elapsed:.1f} s"},
        "e2e": {"value": value, "unit": "GDoF/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_ours(args, rank, world, local_rank):
    import torch

    from adamantine_b200.thermal import ThermalPhysics

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    cfg, T = build_workload(args.size)
    g = ThermalPhysics(cfg, device=local_rank)
    n_dofs = int(np.prod(cfg.geometry.node_shape(cfg.degree)))
    t_op = 1e-4
    g.set_time(t_op)
    srcs = [g.from_grid(T), g.from_grid(T * 1.0001)]
    dsts = [g.initialize_dof_vector(), g.initialize_dof_vector()]
    # the library's autotuner picks the launch schedule on this problem
    schedule, schedule_ms = g.autotune(srcs[0])
    stream = g.stream
    for i in range(args.warmup):
        g.vmult(dsts[i % 2], srcs[i % 2])
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    uuid = str(torch.cuda.get_device_properties(local_rank).uuid)
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(uuid) as clk:
        torch.cuda.synchronize()
        ev0.record(stream)
        for i in range(args.steps):
            g.vmult(dsts[i % 2], srcs[i % 2])
        ev1.record(stream)
        ev1.synchronize()
        torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    ms_max = ms
    if dist:
        tt = torch.tensor([ms], device="cuda")
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms_max = float(tt.item())
    ms_per_step = ms_max / args.steps
    value = world * n_dofs / (ms_per_step * 1e-3) / 1e9
    assert g.device_error() == 0

    # e2e: the same vmult through the host-buffer C ABI entry point
    src_h = torch.from_numpy(g.to_grid(srcs[0]).astype(np.float64)).reshape(-1)
    src_pad = torch.zeros(g.m(), dtype=torch.float64).pin_memory()
    src_pad.copy_(srcs[0].cpu())
    dst_pad = torch.zeros(g.m(), dtype=torch.float64).pin_memory()
    src_np, dst_np = src_pad.numpy(), dst_pad.numpy()
    g.vmult_host(src_np, dst_np)
    e2e_steps = max(2, min(args.steps, 10))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        g.vmult_host(src_np, dst_np)
    e2e_s = (time.perf_counter() - t0) / e2e_steps
    e2e_val = world * n_dofs / e2e_s / 1e9
    del src_h

    sched_name = SCHEDULE_NAMES[schedule]
    peak, peak_kind = measured_peaks()
    fp64_peak = fp64_fma_peak(local_rank)
    # algorithmic bytes of one vmult: read src, write dst (8 B per node each),
    # cell info (4 B per cell), per-cell powder mode (1 B) and liquid sums
    # (8 B) and the per-qp powder of cells whose powder varies inside the
    # cell (8 B read + 8 B write per qp)
    C = g.n_cells
    powder = g.get_qp_powder()
    mixed = int(np.sum(np.any(powder != powder[:, :1], axis=1)))
    alg_bytes = 16 * g.m() + 4 * C + 1 * C + 8 * C + 16 * 27 * mixed
    achieved = alg_bytes / (ms_per_step * 1e-3) / 1e9
    fp64_flop = FP64_FLOP_PER_Q2_CELL * C
    fp64_achieved = fp64_flop / (ms_per_step * 1e-3) / 1e12

    line = {
        "metric": METRIC, "value": value, "unit": "GDoF/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded; no public dataset)",
        "config": workload_config(args.size, world),
        "timing": {"l2": "two src/dst pairs alternate (272 MB working set > 126 MB L2)",
                   "events": "CUDA events on the handle's stream around the K vmults"},
        "schedule": sched_name,
        "cells_per_block": g.cells_per_block(),
        "autotune_ms_per_vmult": dict(zip(SCHEDULE_NAMES, schedule_ms)),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak,
                     "traffic": DRAM_BYTES_PER_VMULT_FULL.get(sched_name) if args.size == "full" else None,
                     "traffic_note": TRAFFIC_NOTE.get(sched_name), "peak_kind": f"{peak_kind} hbm_gbs",
                     "kernel": KERNELS[sched_name][0] + f" ({KERNELS[sched_name][1]} per vmult)",
                     "algorithmic_bytes_per_vmult": alg_bytes},
        # the operator is FP64-issue bound (per-qp physics plus sum
        # factorization), so the FP64 roofline is the binding one
        "roofline_fp64": {"bound": "fp64", "achieved": fp64_achieved, "peak": fp64_peak, "unit": "TFLOP/s",
                          "frac": fp64_achieved / fp64_peak if fp64_peak else None,
                          "flop_per_vmult": fp64_flop,
                          "peak_kind": "measured FP64 FMA rate (adm_diag_fp64_fma_rate) on this GPU"},
        "e2e": {"value": e2e_val, "unit": "GDoF/s", "h2d_bytes_per_step": 8 * g.m(),
                "d2h_bytes_per_step": 8 * g.m(), "path": "adm_vmult_host (pinned host buffers: z-slab copies overlapped with the kernel)"},
        # per vmult: the stage-prepare kernel + the schedule's launches
        "gpu_launches": args.steps * KERNELS[sched_name][2],
        "clocks": clk.summary(),
    }
    if args.rk4_steps > 0:
        line["rk4_step"] = run_rk4_steps(args, local_rank)
    if not args.no_ensemble:
        line["ensemble"] = run_ensemble(args, dist, local_rank)
    if not args.no_adjoint:
        line["adjoint"] = run_adjoint(args, local_rank)
    if args.deposition_steps > 0:
        # the host-core baselines run at N = 1 only (rank 0 would keep the
        # other ranks waiting at the closing barrier)
        line["deposition"] = run_deposition(args, local_rank, world == 1 and not args.no_cpu_baseline)
    if args.amr_steps > 0:
        line["amr"] = run_amr(args, local_rank)
    if not args.no_mechanics:
        line["mechanics"] = run_mechanics(args, local_rank)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        rate, med, n, ref_out = cpu_vmult_rate(build_workload(args.size)[0], T, os.cpu_count() or 1,
                                               keep_result=True)
        line["cpu_baseline"] = {"value": rate, "unit": "GDoF/s", "cores": os.cpu_count() or 1, "kind": "port",
                                "sample": f"{n} full vmults of the workload on the host (oracle, OpenMP), "
                                          f"median {med:.2f} s"}
        # parity of the timed path: the same vmult (autotuned schedule, a
        # fresh handle so the phase history starts as the oracle's) against
        # the oracle's first application on the same field
        gp = ThermalPhysics(cfg, device=local_rank)
        gp.set_schedule(schedule)
        gp.set_time(t_op)
        dp = gp.initialize_dof_vector()
        gp.vmult(dp, gp.from_grid(T))
        got = gp.to_grid(dp).reshape(-1)
        line["parity"] = {"max_rel": float(np.max(np.abs(got - ref_out)) / np.max(np.abs(ref_out))),
                          "tol": 1e-12, "against": "oracle vmult (C++ restatement of the reference CPU path)",
                          "schedule": sched_name}
        del gp
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-ensemble", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--rk4-steps", type=int, default=100,
                    help="graph-captured RK4 steps of the headline problem (0: skip)")
    ap.add_argument("--deposition-steps", type=int, default=2000,
                    help="RK4 steps of the deposition workload (0: skip; the configuration runs 2000)")
    ap.add_argument("--deposition-cpu-steps", type=int, default=2,
                    help="oracle RK4 steps timed for the deposition workload's CPU window (20: the full window)")
    ap.add_argument("--size", default="full", choices=sorted(SIZES))
    ap.add_argument("--no-mechanics", action="store_true")
    ap.add_argument("--amr-steps", type=int, default=50,
                    help="RK4 steps of the refined-mesh workload (0: skip it)")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
    else:
        run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
