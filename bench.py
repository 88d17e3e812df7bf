#!/usr/bin/env python
"""Benchmark of the B200 HAWASSI engine on the batched ragged 1D ensemble.

Workload (one GPU): 256 independent tank realisations advanced together --
Nx drawn from {2048, 4096, 8192, 16384} with L = 0.05 m * Nx, flat depth
U[0.5, 2] m, JONSWAP influx Hs U[0.05, 0.20] m, Tp U[1.5, 3.0] s, gamma U[1, 5]
(1024 lines, seeded phases), HS2 with kinematic breaking, RKF45 rtol 1e-6 /
atol 1e-8, per-member adaptive steps.  One bench step advances every member
through its next `--window` output samples (the reference's output interval is
the influx sampling interval, T_end / 2047 = 0.049 s), clipping steps at each
sample like the reference.  Metric: RHS grid-point evaluations per second
(RHS calls x Nx, summed over members and GPUs).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU (torchrun): each rank advances its own 256-member ensemble (seeds
offset by rank), no data-path collective: weak scaling.  With --shard fixed the
ranks split ONE 256-member ensemble instead (greedy balance of Nx log2 Nx x
expected steps, hawassi_c_b200/partition.py), gather the per-member scalars once
after the timed region, and report strong scaling.

    python bench.py --workload 2d [--steps K] [--warmup W] [--impl ours|reference]

measures the 2D twin instead: 1024 x 1024 on 300 m x 300 m, depth 5 m sloping to
0.5 m with a shoal (two reference depths), HS2 with kinematic breaking,
directional JONSWAP line source (Hs 0.5 m, Tp 6 s, s = 10, 256 x 64 seeded
components), RKF45 rtol 1e-6 / atol 1e-8; one step advances 0.5 simulated s.

    python bench.py --workload fbr005 [--steps K] [--warmup W] [--impl ours|reference]

runs the reference's own test deck 1dFBr005Bor (the deck its published "Relative
time consuming" figure comes from) with the reference's tolerances and reports
simulated seconds per wall second; one step advances 250 output samples (5 s).
"""
import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

MEMBERS = 256
WINDOW = 5
EPS_REL, EPS_ABS = 1e-6, 1e-8
T_END = 100.0
# algorithmic HBM bytes per RHS grid-point evaluation for this workload: RK vectors of
# S = 4 doubles per point streamed 35 times per 6 RHS (stage inputs, stage outputs,
# final combination and error), plus 6 per-point table fields (2 complex source
# kernels, damping, nonlinear-adjustment mask): 35/6 * 4 * 8 + 6 * 8 = 234.7 B
BYTES_PER_RHS_PT = 35.0 / 6.0 * 4 * 8 + 6 * 8
WORKLOAD = ("batched ragged 1D ensemble: 256 members/GPU, Nx in {2048,4096,8192,16384}, L=0.05*Nx, "
            "flat depth U[0.5,2] m, JONSWAP Hs U[0.05,0.20] Tp U[1.5,3.0] gamma U[1,5], HS2 + breaking, "
            "RKF45 rtol 1e-6 atol 1e-8")


# algorithmic FP64 work per RHS grid-point evaluation (the reference's c2c transforms
# at 5 N log2 N flops each, with common subexpressions shared, plus ~80 pointwise
# flops): 17 transforms for HS2 with breaking in 1D; 55 2D transforms (each 5 log2 N
# flops per point) for the 2D twin with two reference depths, breaking and walls
FFTS_PER_RHS_1D = 17
FFTS_PER_RHS_2D = 55
POINTWISE_FLOPS = 80.0


def flops_per_rhs_pt(n_points, ffts):
    return ffts * 5.0 * math.log2(n_points) + POINTWISE_FLOPS


def fp64_roofline(flops, ms, device, kernel, basis):
    """The FP64 roofline beside the HBM one: algorithmic flops of the timed launches
    over their event-timed duration, against the FP64 FMA throughput measured on this
    GPU (hw_fp64_peak_tflops).  None when that measurement fails."""
    try:
        import hawassi_c_b200 as hw
        peak = hw.fp64_peak_tflops(device)
        achieved = flops / (ms / 1e3) / 1e12
        return {"bound": "fp64", "achieved": achieved, "peak": peak, "unit": "TFLOP/s", "frac": achieved / peak,
                "kernel": kernel, "flops": basis,
                "peak_source": "measured on this GPU (DFMA microbenchmark, hw_fp64_peak_tflops)"}
    except Exception as e:   # the HBM roofline and the rest of the line stand without it
        log(f"fp64 roofline unavailable: {e}")
        return None


T_START = time.time()


def profile_traffic(workload):
    """DRAM bytes per RHS grid point of a workload's dominant kernel, from the ncu
    capture recorded in profiles/traffic.json (dram__bytes_read.sum +
    dram__bytes_write.sum of a small capture of the same kernel, divided by the RHS
    points it evaluated).  Returns (bytes per point or None, provenance text); the
    bench scales it to the launch it times, so the figure is profile-derived, not
    measured in this run."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            rec = json.load(f)[workload]
        return float(rec["dram_bytes_per_rhs_pt"]), (
            f"profile-derived: {rec['capture']} ({rec['build']}), scaled by this launch's RHS points")
    except (OSError, KeyError, ValueError, TypeError) as e:
        return None, f"no ncu capture recorded for this workload ({type(e).__name__})"


def log(msg):
    print(f"[bench +{time.time() - T_START:7.1f}s] {msg}", file=sys.stderr, flush=True)


def reduce_ranks(max_vals, sum_vals, device):
    """Whole-job figures across ranks: the max of the time-like values and the sum of
    the counts, as one MAX and one SUM all-reduce taken in the same order on every
    rank (NCCL on the GPUs, gloo in the CPU tests)."""
    import torch
    import torch.distributed as dist
    tm = torch.tensor([float(v) for v in max_vals], device=device, dtype=torch.float64)
    ts = torch.tensor([float(v) for v in sum_vals], device=device, dtype=torch.float64)
    dist.all_reduce(tm, op=dist.ReduceOp.MAX)
    dist.all_reduce(ts, op=dist.ReduceOp.SUM)
    return [float(v) for v in tm.tolist()], [float(v) for v in ts.tolist()]


def sample_members(decks, n):
    """A systematic sample of n members of the ensemble (every len/n-th seed), so a
    bounded CPU run sees the ensemble's mix of grid sizes and sea states."""
    if n >= len(decks):
        return list(decks)
    step = len(decks) / n
    return [decks[int(i * step)] for i in range(n)]


LEARNED_MEMBERS = 64   # the configuration's evaluation ensemble


def learned_vs_plain(device):
    """The third part of the metric: the learned K = 4 operator's ensemble against the
    plain 16-reference ensemble on held-out random bathymetries (the learned
    operator's configuration: Nx = 16384, L = 400 m, depth 0.05-2.0 m from 8 seeded
    bumps), with the network the project's GPU training produced
    (hawassi_c_b200/learned_k4.npy): simulated seconds per wall second of each,
    device-timed, and the eta relative L2 error of the learned members against the
    plain ones.  None when the trained network is absent."""
    from hawassi_c_b200 import decks as _decks, learned
    mlp = learned.load_mlp(device=device)
    if mlp is None:
        return None
    root = os.path.join(tempfile.gettempdir(), "hw_bench_learned")
    ev = [_decks.config4_deck(os.path.join(root, f"eval{i:04d}"), seed=100000 + i, T_end=30.0)
          for i in range(LEARNED_MEMBERS)]
    t0 = time.time()
    res = learned.compare_on_ensemble(mlp, ev, t_warm=0.5, t_end=3.0, device=device)
    mlp.close()
    res["workload"] = (f"{LEARNED_MEMBERS} held-out random bathymetries (Nx 16384, L 400 m, 8 seeded bumps, "
                       "depth 0.05-2.0 m), HS2, rtol 1e-6: learned K=4 blend vs plain 16 reference depths")
    log(f"learned vs plain: {res['speedup']:.2f}x, eta err median {res['eta_err_median']:.2e} "
        f"({time.time() - t0:.1f} s)")
    return res


def learned_vs_plain_2d(device):
    """The 2D configuration's two paths side by side: its deck (1024 x 1024 on 300 m x
    300 m, shoal bottom 0.5-5 m, harbour wall, HS2 with breaking, directional line
    source) with the plain 16-reference operator and with the learned 4-reference
    blend (the same trained network, 2D depth features): device-timed simulated
    seconds per wall second of each over 0.25-0.75 s from the same sea state over the
    whole domain, and the learned run's eta error against the plain one.  None when
    the trained network is absent."""
    from hawassi_c_b200 import decks2d, learned
    mlp = learned.load_mlp(device=device)
    if mlp is None:
        return None
    t0 = time.time()
    res = learned.compare_2d(mlp, decks2d.config5(seed=0), t_warm=0.25, t_end=0.75, device=device,
                             eps_abs=EPS_ABS, eps_rel=EPS_REL)
    mlp.close()
    res["workload"] = ("2D configuration deck (1024x1024, 300 m x 300 m, shoal 0.5-5 m, wall refl 0.5, HS2 + breaking, "
                       "rtol 1e-6): learned K=4 blend vs plain 16 reference depths, general 2D path for both")
    log(f"2D learned vs plain: {res['speedup']:.2f}x, eta err {res['eta_err']:.2e} "
        f"(uniform weights {res['eta_err_uniform_weights']:.2e}) ({time.time() - t0:.1f} s)")
    return res


def ensemble_config(args):
    """The workload description both arms print (the driver compares them)."""
    return {"workload": WORKLOAD, "members_per_gpu": args.members, "window_samples": args.window,
            "sharding": ("one fixed ensemble split over the ranks (LPT on Nx log2 Nx x expected steps)"
                         if args.shard == "fixed" else "one ensemble per rank (seeds offset by rank)"),
            "l2": "working set well above L2 (126 MB): no flush needed",
            "grid_sizes": [2048, 4096, 8192, 16384]}


def make_decks(root, rank, members, breaking=True):
    from hawassi_c_b200 import decks
    paths = []
    for m in range(members):
        seed = rank * members + m
        p = os.path.join(root, f"m{seed:05d}")
        if not os.path.exists(os.path.join(p, "input.txt")):
            decks.ensemble_member_deck(p, seed=seed, T_end=T_END, breaking=breaking)
        paths.append(p)
    return paths


# ----------------------------------------------------------------------------
# CPU side: the oracle port on the host cores (one thread per core)
# ----------------------------------------------------------------------------
def _cpu_worker(args):
    """Advance a fixed set of members through n_steps windows of output samples,
    recording (RHS grid points, wall seconds) per step; stop early past max_seconds."""
    decks, window, n_steps, max_seconds = args
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as ol
    members = []
    for d in decks:
        o = ol.Oracle(d, eps_abs=EPS_ABS, eps_rel=EPS_REL)
        tt = o.table("ttrace")
        members.append([o, tt, float(tt[0]), 1e-4, o.initial_state(), 0])
    out = []
    t_start = time.perf_counter()
    for _ in range(n_steps):
        t0 = time.perf_counter()
        pts = 0
        for mb in members:
            o, tt, t, h, y, i = mb
            c0 = o.stats()[0]
            stop = min(i + window, len(tt))
            for ti in tt[i:stop]:
                while t < ti and time.perf_counter() - t_start <= max_seconds:
                    t, h = o.evolve_apply(t, ti, h, y)
            mb[2], mb[3], mb[5] = t, h, stop
            pts += (o.stats()[0] - c0) * o.nx
        out.append((pts, time.perf_counter() - t0, sum(m[2] - float(m[1][0]) for m in members)))
        if time.perf_counter() - t_start > max_seconds:
            break
    return out


def cpu_measure(decks, workers, window, n_steps, max_seconds, timeout=None):
    """Run the oracle port on `workers` host threads (ctypes releases the GIL during
    each C call, so the threads run on separate cores); returns per-step
    (RHS grid points, max wall seconds over workers) and the simulated seconds."""
    import concurrent.futures as cf
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as ol
    ol.lib()
    shards = [decks[w::workers] for w in range(workers)]
    shards = [s for s in shards if s]
    with cf.ThreadPoolExecutor(len(shards)) as ex:
        futs = [ex.submit(_cpu_worker, (sh, window, n_steps, max_seconds)) for sh in shards]
        res = [f.result(timeout=timeout) for f in futs]
    steps = min(len(r) for r in res)
    return [(sum(r[k][0] for r in res), max(r[k][1] for r in res)) for k in range(steps)], \
        sum(r[steps - 1][2] for r in res)


def run_reference(args, rank, world):
    """--impl reference: the oracle port (the reference's algorithm, restated in C)
    on every host core, same workload, metric and window."""
    if rank != 0:
        return 0
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as ol
    ol.lib()
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    root = os.path.join(tempfile.gettempdir(), "hw_bench_decks_r0")
    decks = sample_members(make_decks(root, 0, args.members), cores)
    steps, _ = cpu_measure(decks, cores, args.window, args.warmup + args.steps, 1e9)
    timed = steps[args.warmup:]
    value = sum(p for p, _ in timed) / sum(t for _, t in timed)
    line = {
        "metric": "RHS grid-pt evals/s", "value": value, "unit": "RHS grid-point evaluations/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * sum(t for _, t in timed) / len(timed), "higher_is_better": True,
        "scaling": "strong" if args.shard == "fixed" else "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic seeded decks (JONSWAP influx, flat depths) in the "
                                                    "reference input format",
        "config": ensemble_config(args),
        "impl": "reference",
        "cpu_baseline": {"value": value, "unit": "RHS grid-point evaluations/s", "cores": cores, "kind": "port",
                         "sample": f"{len(decks)} of the ensemble's {args.members} members (every "
                                   f"{max(1, args.members // len(decks))}th seed: the same mix of grid sizes), "
                                   f"one per core, each advanced {args.window} output samples per step"},
        "e2e": {"value": value, "unit": "RHS grid-point evaluations/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ----------------------------------------------------------------------------
# GPU side
# ----------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(gpu_index), f"--query-gpu={self.FIELDS}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.f.name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


# ----------------------------------------------------------------------------
# 2D workload
# ----------------------------------------------------------------------------
STEP_2D = 0.5
# algorithmic HBM bytes per 2D RHS grid-point evaluation: the RK vectors of S = 6
# doubles per point streamed 35 times per 6 RHS, plus 15 per-point table doubles
# (two-depth weights gam_min/plus, C^2 and Om^2 of both reference depths, aal,
# damping, ChiAdj, two complex source kernels, the breaking tables bathymetry and
# pb.Char): 35/6 * 6 * 8 + 15 * 8
BYTES_PER_RHS_PT_2D = 35.0 / 6.0 * 6 * 8 + 15 * 8
WORKLOAD_2D = ("2D twin: 1024x1024 on 300 m x 300 m, depth 5 m offshore sloping to 0.5 m with a seeded shoal "
               "(two reference depths), harbour breakwater of reflection 0.5, HS2 with kinematic breaking (KBC 0.8, TC 0.2, "
               "Tchar 0.5), vertical line source of a directional JONSWAP (Hs 0.5 m, Tp 6 s, "
               "gamma 3.3, cos^2s s=10, 256x64 seeded components), 30 m damping zones, RKF45 rtol 1e-6 atol 1e-8")


def _cpu_rhs_2d(tables, threads, seconds):
    """The 2D oracle's RHS (the reference's algorithm restated in C) on `threads` host
    threads, each evaluating full-size RHS calls on its own state for ~`seconds`."""
    import concurrent.futures as cf
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as ol
    n = tables["nx"] * tables["ny"]
    # one oracle context per thread: the breaking state and work arrays are per context
    ctxs = [ol.Oracle2D(tables, EPS_ABS, EPS_REL) for _ in range(threads)]

    def work(seed):
        o = ctxs[seed]
        rng = np.random.default_rng(seed)
        y = 1e-3 * rng.standard_normal(6 * n) * np.tile(tables["aal"].ravel(), 6)
        calls, t0 = 0, time.perf_counter()
        while True:
            o.rhs(1.0 + 0.01 * calls, y)
            calls += 1
            if time.perf_counter() - t0 > seconds:
                return calls, time.perf_counter() - t0

    with cf.ThreadPoolExecutor(threads) as ex:
        res = list(ex.map(work, range(threads)))
    calls = sum(c for c, _ in res)
    wall = max(w for _, w in res)
    return calls * n / wall, calls


def run_reference_2d(args, rank, world):
    if rank != 0:
        return 0
    from hawassi_c_b200 import decks2d
    tb = decks2d.config5(seed=0)
    cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    threads = max(1, min(cores, 16))
    vals = []
    for _ in range(args.warmup + args.steps):
        v, calls = _cpu_rhs_2d(tb, threads, 8.0)
        vals.append(v)
    value = statistics.mean(vals[args.warmup:])
    line = {
        "metric": "RHS grid-pt evals/s", "value": value, "unit": "RHS grid-point evaluations/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 8000.0,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic seeded 2D deck tables", "config": {"workload": WORKLOAD_2D}, "impl": "reference",
        "cpu_baseline": {"value": value, "unit": "RHS grid-point evaluations/s", "cores": threads, "kind": "port",
                         "sample": f"full-size 1024x1024 RHS evaluations on {threads} threads, ~8 s per step"},
        "e2e": {"value": value, "unit": "RHS grid-point evaluations/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def main_2d(args, rank, world, local):
    import numpy as np
    from hawassi_c_b200 import decks2d
    tb = decks2d.config5(seed=rank)
    n = tb["nx"] * tb["ny"]
    log("2D tables ready")
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cores = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
        threads = max(1, min(cores, 16))
        v, calls = _cpu_rhs_2d(tb, threads, 12.0)
        cpu = {"value": v, "unit": "RHS grid-point evaluations/s", "cores": threads, "kind": "port",
               "sample": f"{calls} full-size 1024x1024 RHS evaluations of the 2D oracle on {threads} threads "
                         f"(~12 s)"}
        log(f"cpu baseline {v:.3e} pts/s")
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    from hawassi_c_b200.engine2d import Engine2D
    eng = Engine2D(tb, EPS_ABS, EPS_REL, device=local)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    eng.set_stream(stream.cuda_stream)
    eng.set_state(0.0, 0.02, np.zeros(6 * n))
    t_sim = 0.0
    for _ in range(args.warmup):
        t_sim += STEP_2D
        eng.run_to_time(t_sim)
    log(f"warmup to t = {t_sim}")

    def barrier():
        if world > 1:
            dist.barrier()

    s0, l0 = eng.stats(), eng.launches()
    barrier()
    torch.cuda.synchronize()
    clk = ClockSampler(local)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        t_sim += STEP_2D
        eng.run_to_time(t_sim)
    e1.record(stream)
    torch.cuda.synchronize()
    clocks = clk.stop()
    barrier()
    ms = e0.elapsed_time(e1)
    s1, l1 = eng.stats(), eng.launches()
    pts = float((s1["rhs_calls"] - s0["rhs_calls"]) * n)
    if world > 1:
        (ms,), (pts,) = reduce_ranks([ms], [pts], "cuda")
    value = pts / (ms / 1e3)
    achieved = value * BYTES_PER_RHS_PT_2D / 1e9
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except OSError:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    per_pt, traffic_source = profile_traffic("2d")
    traffic = per_pt * pts / max(1, args.steps) / (world or 1) if per_pt else None
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": traffic, "traffic_source": traffic_source,
            "kernel": "k2v_rowA..k2b_sbrow (one RHS = 9 fused FFT passes + the breaking kernels)",
            "launch": f"one step = {STEP_2D} simulated s, {pts / max(1, args.steps):.3e} RHS grid points, "
                      f"{BYTES_PER_RHS_PT_2D:.1f} algorithmic B/point",
            "peak_source": "measured (MEASURED_PEAKS.json hbm_gbs)" if "hbm_gbs" in peaks else "fallback"}
    roof_fp64 = fp64_roofline(pts / max(1, world) * flops_per_rhs_pt(n, FFTS_PER_RHS_2D), ms, local,
                              "k2v_rowA..k2b_sbrow",
                              f"{FFTS_PER_RHS_2D} 2D c2c transforms x 5 log2(Nx Ny) + {POINTWISE_FLOPS:.0f} "
                              "pointwise flops per RHS point")
    # end to end through the public API: host state in (pinned), evolve, host state out
    host = torch.empty(6 * n, dtype=torch.float64, pin_memory=True)
    hv = host.numpy()
    _, h_cur, y_cur = eng.state()
    hv[:] = y_cur
    torch.cuda.synchronize()
    r0 = eng.stats()["rhs_calls"]
    e0.record(stream)
    for _ in range(args.steps):
        eng.set_state(t_sim, h_cur, hv)
        t_sim += STEP_2D
        eng.run_to_time(t_sim)
        _, h_cur = eng.state_into(hv)
    e1.record(stream)
    torch.cuda.synchronize()
    ems = e0.elapsed_time(e1)
    e_pts = float((eng.stats()["rhs_calls"] - r0) * n)
    e2e = {"value": e_pts / (ems / 1e3), "unit": "RHS grid-point evaluations/s",
           "h2d_bytes_per_step": 6 * n * 8, "d2h_bytes_per_step": 6 * n * 8}
    if rank == 0:
        line = {
            "metric": "RHS grid-pt evals/s", "value": value, "unit": "RHS grid-point evaluations/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic seeded 2D deck tables (reference formulas, directional JONSWAP line signals)",
            "config": {"workload": WORKLOAD_2D, "nx": tb["nx"], "ny": tb["ny"], "step_sim_s": STEP_2D,
                       "l2": "working set (~0.9 GB of RK vectors and pass fields) above L2: no flush needed"},
            "rhs_points_per_step": pts / args.steps,
            "sim_s_per_wall_s": STEP_2D * args.steps / (ms / 1e3),
            "roofline": roof, "roofline_fp64": roof_fp64, "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": l1 - l0, "clocks": clocks,
            "rhs_calls": s1["rhs_calls"] - s0["rhs_calls"], "accepted": s1["accepted"] - s0["accepted"],
            "rejected": s1["rejected"] - s0["rejected"],
        }
        print(json.dumps(line), flush=True)
    eng.close()
    if world > 1:
        dist.destroy_process_group()
    return 0

# ----------------------------------------------------------------------------
# The reference's published benchmark deck (1dFBr005Bor)
# ----------------------------------------------------------------------------
FBR_DECK = os.path.join(ROOT, "tests", "golden", "fbr005")
FBR_STEP_SAMPLES = 250            # one bench step = 250 output samples = 5 simulated s
FBR_PUBLISHED_SIM_PER_WALL = 1.0 / 1.09714   # logfile.txt:35 "Relative time consuming" (hardware not recorded)
# one member of 4096 points: 8 CTAs of 512 points (the shortest phases) measured fastest
# on B200 against 1024- and 2048-point slices (9.09 / 8.33 / 7.99 sim-s per wall-s)
FBR_SLICE = 512
WORKLOAD_FBR = ("the reference's own test deck 1dFBr005Bor: 1D HS2, flat h = 1 m, kinematic breaking, IVP from "
                "initial.dat, Nx = 4096 on [-215, 215] m, output every 0.02 s to t = 120 s, the reference's "
                "tolerances (abs 1e-5, rel 1e-4) and first step 1e-4")


def _fbr_cpu(max_seconds):
    """The oracle port on one host thread through the deck's output samples from t0
    for ~max_seconds: (simulated s, wall s, RHS grid points)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as ol
    o = ol.Oracle(FBR_DECK)
    tt = o.table("ttrace")
    y = o.initial_state()
    t, h = float(tt[0]), 1e-4
    c0, w0 = o.stats()[0], time.perf_counter()
    for ti in tt[1:]:
        while t < ti:
            t, h = o.evolve_apply(t, ti, h, y)
        if time.perf_counter() - w0 > max_seconds:
            break
    wall = time.perf_counter() - w0
    pts = (o.stats()[0] - c0) * o.nx
    o.close()
    return t - float(tt[0]), wall, pts


def run_reference_fbr(args, rank, world):
    if rank != 0:
        return 0
    sim, wall, pts = _fbr_cpu(8.0 * (args.steps + args.warmup))
    value = sim / wall
    line = {
        "metric": "sim-s/wall-s", "value": value, "unit": "simulated s per wall s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * wall / max(1, args.steps + args.warmup),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": value / FBR_PUBLISHED_SIM_PER_WALL,
        "dtype": "f64", "data": "the reference's shipped deck (tests/golden/fbr005)",
        "config": {"workload": WORKLOAD_FBR}, "impl": "reference", "rhs_pts_per_s": pts / wall,
        "cpu_baseline": {"value": value, "unit": "simulated s per wall s", "cores": 1, "kind": "port",
                         "sample": f"the first {sim:.2f} simulated s from t0 on one thread"},
        "e2e": {"value": value, "unit": "simulated s per wall s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def main_fbr(args, rank, world, local):
    """The whole deck on one GPU (one member, replicas only under torchrun): each step
    advances FBR_STEP_SAMPLES output samples through hw_run, the gauge and breaking
    stages included."""
    import numpy as np
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        sim, wall, _ = _fbr_cpu(15.0)
        cpu = {"value": sim / wall, "unit": "simulated s per wall s", "cores": 1, "kind": "port",
               "sample": f"the first {sim:.2f} simulated s of the deck from t0 on one thread (~15 s)"}
        log(f"cpu baseline {cpu['value']:.3f} sim-s/wall-s")
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    import hawassi_c_b200 as hw
    slice_ = args.slice or FBR_SLICE
    eng = hw.Engine(FBR_DECK, device=local, slice=slice_)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    eng.set_stream(stream.cuda_stream)
    nt = eng.nt[0]
    need = (args.warmup + args.steps) * FBR_STEP_SAMPLES
    if need >= nt:
        raise SystemExit(f"fbr005: {args.warmup} + {args.steps} steps of {FBR_STEP_SAMPLES} samples exceed "
                         f"the deck's {nt} samples")
    i = 0
    for _ in range(args.warmup):
        i += FBR_STEP_SAMPLES
        eng.run(i, sync=False)
    torch.cuda.synchronize()

    def barrier():
        if world > 1:
            dist.barrier()

    s0 = eng.stats()
    t_start = eng.state()[0]
    barrier()
    torch.cuda.synchronize()
    clk = ClockSampler(local)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        i += FBR_STEP_SAMPLES
        eng.run(i, sync=False)
    e1.record(stream)
    torch.cuda.synchronize()
    clocks = clk.stop()
    barrier()
    ms = e0.elapsed_time(e1)
    t_end = eng.state()[0]
    s1 = eng.stats()
    sim = t_end - t_start
    pts = float((s1["rhs_calls"] - s0["rhs_calls"]) * eng.nx[0])
    if world > 1:
        (ms,), (sim, pts) = reduce_ranks([ms], [sim, pts], "cuda")
    value = sim / (ms / 1e3)
    # end to end through the public API over the same simulated window: back to t0,
    # the warm-up samples again, then the state in from pinned host memory and out
    # again every step
    eng.reset()
    i = 0
    for _ in range(args.warmup):
        i += FBR_STEP_SAMPLES
        eng.run(i, sync=False)
    host = torch.empty(4 * eng.nx[0], dtype=torch.float64, pin_memory=True)
    hv = host.numpy()
    eng.get_states(hv)
    ta = eng.state()[0]
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        eng.set_states(hv)
        i += FBR_STEP_SAMPLES
        eng.run(i, sync=False)
        eng.get_states(hv)
    e1.record(stream)
    torch.cuda.synchronize()
    ems = e0.elapsed_time(e1)
    e2e_sim = eng.state()[0] - ta
    e2e = {"value": e2e_sim / (ems / 1e3), "unit": "simulated s per wall s",
           "h2d_bytes_per_step": 4 * eng.nx[0] * 8, "d2h_bytes_per_step": 4 * eng.nx[0] * 8}
    if rank == 0:
        line = {
            "metric": "sim-s/wall-s", "value": value, "unit": "simulated s per wall s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": value / FBR_PUBLISHED_SIM_PER_WALL, "dtype": "f64",
            "data": "the reference's shipped deck (tests/golden/fbr005)",
            "config": {"workload": WORKLOAD_FBR, "step_samples": FBR_STEP_SAMPLES, "slice": slice_,
                       "l2": "single member (512 KB state) resident in L2: latency-bound, no roofline claim"},
            "rhs_pts_per_s": pts / (ms / 1e3), "rhs_calls": s1["rhs_calls"] - s0["rhs_calls"],
            "accepted": s1["accepted"] - s0["accepted"], "rejected": s1["rejected"] - s0["rejected"],
            "published_sim_s_per_wall_s": FBR_PUBLISHED_SIM_PER_WALL,
            "roofline": None, "cpu_baseline": cpu, "e2e": e2e, "clocks": clocks,
            "gpu_launches": args.steps * (2 * len(eng.class_timing()) + 1),   # per step: k_resume, k_order_class, k_evolve
        }
        print(json.dumps(line), flush=True)
    eng.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


# ----------------------------------------------------------------------------
# Config 2: one 1D run on a slope with 16 reference depths, HS3 and breaking
# ----------------------------------------------------------------------------
C2_STEP_SAMPLES = 20              # one bench step = 20 output samples (~1.95 simulated s)
C2_NREF = 16
WORKLOAD_C2 = ("1D plain FP64, varying bathymetry and breaking: L = 400 m, Nx = 16384, depth 1.0 m flat for "
               "150 m then a 1:30 slope to 0.05 m, dispersion interpolated over 16 reference depths, HS3, "
               "kinematic breaking (KBC 0.8, TC 0.2, Tchar 0.5), seeded JONSWAP influx Hs 0.15 m Tp 2.5 s "
               "gamma 3.3 (1024 lines), RKF45 rtol 1e-6 atol 1e-8, t_end 200 s")


WORKLOAD_C1 = ("1D plain FP64: periodic tank L = 200 m, Nx = 4096, flat depth 1.0 m, HS2, no breaking, seeded "
               "JONSWAP influx at x = 20 m (Hs 0.10 m, Tp 2.0 s, gamma 3.3, 1024 lines), 10 m damping zones, "
               "RKF45 rtol 1e-6 atol 1e-8, t_end 100 s")
# single runs: (deck writer, reference depths, samples per step, slice, workload text)
SINGLE = {"c1": ("config1_deck", 0, 40, 512, WORKLOAD_C1), "c2": ("config2_deck", C2_NREF, C2_STEP_SAMPLES, 0, WORKLOAD_C2)}


def _c2_deck(which="c2"):
    from hawassi_c_b200 import decks
    p = os.path.join(tempfile.gettempdir(), f"hw_bench_{which}")
    if not os.path.exists(os.path.join(p, "input.txt")):
        getattr(decks, SINGLE[which][0])(p, seed=0)
    return p


def _c2_cpu(deck, max_seconds, nref=C2_NREF):
    """The oracle port on one host thread from t0 for ~max_seconds."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_lib as ol
    o = ol.Oracle(deck, eps_abs=EPS_ABS, eps_rel=EPS_REL, nref=nref)
    tt = o.table("ttrace")
    y = o.initial_state()
    t, h = float(tt[0]), 1e-4
    c0, w0 = o.stats()[0], time.perf_counter()
    for ti in tt[1:]:
        while t < ti and time.perf_counter() - w0 <= max_seconds:
            t, h = o.evolve_apply(t, ti, h, y)
        if time.perf_counter() - w0 > max_seconds:
            break
    wall = time.perf_counter() - w0
    pts = (o.stats()[0] - c0) * o.nx
    o.close()
    return t - float(tt[0]), wall, pts


def main_c2(args, rank, world, local):
    which = args.workload
    _, nref, step_samples, slice_default, workload_text = SINGLE[which]
    deck = _c2_deck(which)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        sim, wall, pts = _c2_cpu(deck, 15.0, nref)
        cpu = {"value": pts / wall, "unit": "RHS grid-point evaluations/s", "cores": 1, "kind": "port",
               "sample": f"the first {sim:.3f} simulated s of the run from t0 on one thread (~15 s), "
                         f"{sim / wall:.4f} sim-s/wall-s"}
        log(f"cpu baseline {cpu['value']:.3e} pts/s, {sim / wall:.4f} sim-s/wall-s")
    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    import hawassi_c_b200 as hw
    slice_ = args.slice or slice_default
    eng = hw.Engine(deck, eps_abs=EPS_ABS, eps_rel=EPS_REL, nref=nref, device=local, slice=slice_)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    eng.set_stream(stream.cuda_stream)
    i = 0
    for _ in range(args.warmup):
        i += step_samples
        eng.run(i, sync=False)
    torch.cuda.synchronize()
    s0, t0 = eng.stats(), eng.state()[0]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    clk = ClockSampler(local)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        i += step_samples
        eng.run(i, sync=False)
    e1.record(stream)
    torch.cuda.synchronize()
    clocks = clk.stop()
    if world > 1:
        dist.barrier()
    ms = e0.elapsed_time(e1)
    s1, t1 = eng.stats(), eng.state()[0]
    nx = eng.nx[0]
    pts = float((s1["rhs_calls"] - s0["rhs_calls"]) * nx)
    sim = t1 - t0
    if world > 1:
        (ms,), (pts, sim) = reduce_ranks([ms], [pts, sim], "cuda")
    value = pts / (ms / 1e3)
    eng.reset()
    i = 0
    for _ in range(args.warmup):
        i += step_samples
        eng.run(i, sync=False)
    host = torch.empty(4 * nx, dtype=torch.float64, pin_memory=True)
    hv = host.numpy()
    eng.get_states(hv)
    r0 = eng.stats()["rhs_calls"]
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        eng.set_states(hv)
        i += step_samples
        eng.run(i, sync=False)
        eng.get_states(hv)
    e1.record(stream)
    torch.cuda.synchronize()
    ems = e0.elapsed_time(e1)
    e2e = {"value": float((eng.stats()["rhs_calls"] - r0) * nx) / (ems / 1e3), "unit": "RHS grid-point evaluations/s",
           "h2d_bytes_per_step": 4 * nx * 8, "d2h_bytes_per_step": 4 * nx * 8}
    if rank == 0:
        line = {
            "metric": "RHS grid-pt evals/s", "value": value, "unit": "RHS grid-point evaluations/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic seeded deck (JONSWAP influx) in the reference input format",
            "config": {"workload": workload_text, "step_samples": step_samples, "slice": slice_ or 2048,
                       "l2": "single member resident in L2: latency-bound, no roofline claim"},
            "sim_s_per_wall_s": sim / (ms / 1e3), "rhs_calls": s1["rhs_calls"] - s0["rhs_calls"],
            "accepted": s1["accepted"] - s0["accepted"], "rejected": s1["rejected"] - s0["rejected"],
            "roofline": None, "cpu_baseline": cpu, "e2e": e2e, "clocks": clocks,
            "gpu_launches": args.steps * (2 * len(eng.class_timing()) + 1),
        }
        print(json.dumps(line), flush=True)
    eng.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--members", type=int, default=MEMBERS)
    ap.add_argument("--window", type=int, default=WINDOW)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-learned", action="store_true", help="skip the learned-vs-plain ensemble comparison")
    ap.add_argument("--workload", default="ensemble", choices=["ensemble", "2d", "fbr005", "c1", "c2"])
    ap.add_argument("--slice", type=int, default=0,
                    help="fbr005: grid points per CTA of the member's cluster (0: 512)")
    ap.add_argument("--resident", type=int, default=0,
                    help="ensemble evolve grid: 0 one cluster per member, -1 persistent clusters "
                         "pulling members from a queue (the class's share), n > 0 at most n per class")
    ap.add_argument("--shard", default="replicas", choices=["replicas", "fixed"],
                    help="multi-GPU ensemble: a 256-member ensemble per rank (weak) or one split over ranks (strong)")
    ap.add_argument("--autotune", action="store_true",
                    help="pick the slice per grid size by timing candidates on the device first")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", str(args.gpus)))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if os.environ.get("WORLD_SIZE") is None:
        world = 1
    if args.workload == "2d":
        if args.impl == "reference":
            return run_reference_2d(args, rank, world)
        return main_2d(args, rank, world, local)
    if args.workload in SINGLE:
        if args.impl == "reference":
            if rank != 0:
                return 0
            sim, wall, pts = _c2_cpu(_c2_deck(args.workload), 5.0 * (args.steps + args.warmup),
                                     SINGLE[args.workload][1])
            value = pts / wall
            print(json.dumps({
                "metric": "RHS grid-pt evals/s", "value": value, "unit": "RHS grid-point evaluations/s",
                "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": 1e3 * wall / max(1, args.steps + args.warmup), "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic seeded deck",
                "config": {"workload": SINGLE[args.workload][4]}, "impl": "reference",
                "sim_s_per_wall_s": sim / wall,
                "cpu_baseline": {"value": value, "unit": "RHS grid-point evaluations/s", "cores": 1, "kind": "port",
                                 "sample": f"the first {sim:.3f} simulated s from t0 on one thread"},
                "e2e": {"value": value, "unit": "RHS grid-point evaluations/s", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}}), flush=True)
            return 0
        return main_c2(args, rank, world, local)
    if args.workload == "fbr005":
        if args.impl == "reference":
            return run_reference_fbr(args, rank, world)
        return main_fbr(args, rank, world, local)
    if args.impl == "reference":
        return run_reference(args, rank, world)

    shard = None
    if args.shard == "fixed":
        from hawassi_c_b200 import partition
        all_decks = make_decks(os.path.join(tempfile.gettempdir(), "hw_bench_decks_r0"), 0, args.members)
        costs = partition.deck_costs(all_decks, T_END)
        shard = partition.greedy_partition(costs, world)[rank]
        decks = [all_decks[i] for i in shard]
        log(f"fixed ensemble: rank {rank} runs {len(decks)} of {len(all_decks)} members")
    else:
        root = os.path.join(tempfile.gettempdir(), f"hw_bench_decks_r{rank}")
        decks = make_decks(root, rank, args.members)
    log(f"{len(decks)} decks ready")

    # CPU baseline on the host cores (spawned before any CUDA work), rank 0 at N=1 only
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cores = min(len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else os.cpu_count() or 1, 64)
        sample = sample_members(decks, cores)
        log(f"cpu baseline on {cores} threads")
        steps, sims = cpu_measure(sample, cores, args.window, 10 ** 6, 15.0, timeout=240)
        cpu = {"value": sum(p for p, _ in steps) / sum(t for _, t in steps), "unit": "RHS grid-point evaluations/s",
               "cores": cores, "kind": "port",
               "sample": f"{len(sample)} of the ensemble's members (every {max(1, len(decks) // len(sample))}th "
                         f"seed) on {cores} threads, {len(steps)} windows of {args.window} output samples from t0 "
                         f"(~15 s of CPU time, {sims:.1f} simulated s)"}
        log(f"cpu baseline {cpu['value']:.3e} pts/s")

    import torch
    import torch.distributed as dist
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    import hawassi_c_b200 as hw
    slices = None
    if args.autotune:
        from hawassi_c_b200.autotune import autotune_slices
        slices, _ = autotune_slices(decks, window=args.window, device=local, eps_abs=EPS_ABS, eps_rel=EPS_REL,
                                    log=log)
        log(f"autotuned slices {slices}")
    eng = hw.Engine(decks, eps_abs=EPS_ABS, eps_rel=EPS_REL, device=local, slices=slices, resident=args.resident)
    log("engine created")
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    eng.set_stream(stream.cuda_stream)
    nx = eng.nx

    def barrier():
        if world > 1:
            dist.barrier()

    def rhs_pts():
        return sum(eng.stats(i)["rhs_calls"] * nx[i] for i in range(eng.members))

    def rhs_flops():
        return sum(eng.stats(i)["rhs_calls"] * nx[i] * flops_per_rhs_pt(nx[i], FFTS_PER_RHS_1D)
                   for i in range(eng.members))

    def sim_time():
        return sum(eng.state(i)[0] for i in range(eng.members))

    i_stop = 0
    for _ in range(args.warmup):
        i_stop += args.window
        eng.run(i_stop, sync=True)
        log(f"warmup step to sample {i_stop}")
    torch.cuda.synchronize()
    pts0, sim0 = rhs_pts(), sim_time()
    barrier()
    torch.cuda.synchronize()
    clk = ClockSampler(local)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        i_stop += args.window
        eng.run(i_stop, sync=False)
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier()
    clocks = clk.stop()
    ms = ev0.elapsed_time(ev1)
    log(f"timed {args.steps} steps: {ms:.1f} ms")
    pts1, sim1 = rhs_pts(), sim_time()
    launches = args.steps * (2 * len(eng.class_timing()) + 1)   # per step: k_resume + per class k_order_class and k_evolve
    if world > 1:
        (ms,), (tot_pts, tot_sim) = reduce_ranks([ms], [float(pts1 - pts0), sim1 - sim0], "cuda")
    else:
        tot_pts, tot_sim = float(pts1 - pts0), sim1 - sim0
    value = tot_pts / (ms / 1e3)

    # roofline of the dominant kernel: k_evolve (99% of device time).  One step is one
    # launch of it per grid-size class, all classes running concurrently on forked
    # streams, so the launch group of one more step is timed as a unit with events
    # on the launching stream and credited with every RHS point it evaluated.
    pts_a, flops_a = rhs_pts(), rhs_flops()
    g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    g0.record(stream)
    i_stop += args.window
    eng.run(i_stop, sync=False)
    g1.record(stream)
    torch.cuda.synchronize()
    gms = g0.elapsed_time(g1)
    grp_pts = rhs_pts() - pts_a
    achieved = grp_pts * BYTES_PER_RHS_PT / (gms / 1e3) / 1e9
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except OSError:
        pass
    peak = float(peaks.get("hbm_gbs", 6650.0))
    per_pt, traffic_source = profile_traffic("ensemble")
    traffic = per_pt * grp_pts if per_pt else None   # bytes over the launch group
    classes = eng.class_timing()
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": traffic, "traffic_source": traffic_source, "kernel": "k_evolve<2048>",
            "launch": f"one step = {len(classes)} concurrent launches (one per grid-size class), "
                      f"{gms:.2f} ms, {grp_pts:.3e} RHS grid points, {BYTES_PER_RHS_PT:.1f} algorithmic B/point",
            "class_ms": [round(c[0], 3) for c in classes],
            "peak_source": "measured (MEASURED_PEAKS.json hbm_gbs)" if "hbm_gbs" in peaks else "fallback"}
    roof_fp64 = fp64_roofline(rhs_flops() - flops_a, gms, local, "k_evolve<2048>",
                              f"{FFTS_PER_RHS_1D} c2c transforms x 5 log2(Nx) + {POINTWISE_FLOPS:.0f} "
                              "pointwise flops per RHS point, per member")

    # end to end through the C ABI with host buffers: H2D of every member's state, the
    # step, D2H of every state
    tot_doubles = sum(4 * n for n in nx)
    host = torch.empty(tot_doubles, dtype=torch.float64, pin_memory=True)
    hv = host.numpy()
    eng.get_states(hv)
    barrier()
    torch.cuda.synchronize()
    pe0 = rhs_pts()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        eng.set_states(hv)
        i_stop += args.window
        eng.run(i_stop, sync=False)
        eng.get_states(hv)
    e1.record(stream)
    torch.cuda.synchronize()
    ems = e0.elapsed_time(e1)
    e_pts = float(rhs_pts() - pe0)
    if world > 1:
        (ems,), (e_pts,) = reduce_ranks([ems], [e_pts], "cuda")
    log(f"e2e {args.steps} steps: {ems:.1f} ms")
    e2e = {"value": e_pts / (ems / 1e3), "unit": "RHS grid-point evaluations/s",
           "h2d_bytes_per_step": tot_doubles * 8, "d2h_bytes_per_step": tot_doubles * 8}
    statuses = [eng.stats(i)["status"] for i in range(eng.members)]
    summary = None
    if shard is not None:
        # the one end-of-run exchange of the fixed ensemble: per-member scalars to every rank
        from hawassi_c_b200 import partition
        rows = []
        for i in range(eng.members):
            st = eng.stats(i)
            rows.append([eng.state(i)[0], st["rhs_calls"], st["accepted"], st["rejected"], st["status"],
                         eng.energy(member=i)])
        tab = partition.gather_member_scalars(shard, rows, args.members, "cuda")
        summary = {"members": int(tab.shape[0]), "sim_s": float(tab[:, 0].sum()),
                   "rhs_calls": int(tab[:, 1].sum()), "status_nonzero": int((tab[:, 4] != 0).sum())}
    learned_line = learned_line_2d = None
    if rank == 0 and world == 1 and not args.no_learned:
        eng.close()
        eng = None
        learned_line = learned_vs_plain(local)
        learned_line_2d = learned_vs_plain_2d(local)

    if rank == 0:
        line = {
            "metric": "RHS grid-pt evals/s", "value": value, "unit": "RHS grid-point evaluations/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "strong" if shard is not None else "weak", "vs_baseline": None,
            "dtype": "f64",
            "data": "synthetic seeded decks (JONSWAP influx, flat depths) in the reference input format",
            "config": ensemble_config(args),
            "slices": ({str(k): v for k, v in slices.items()} if slices else "2048 (default)"),
            "ensemble_summary": summary,
            "rhs_points_per_step": tot_pts / args.steps,
            "sim_s_per_wall_s": tot_sim / (ms / 1e3),
            "sim_s_per_wall_s_per_member": tot_sim / (ms / 1e3) / (args.members * world),
            "roofline": roof, "roofline_fp64": roof_fp64, "cpu_baseline": cpu, "e2e": e2e,
            "gpu_launches": launches,
            "clocks": clocks, "member_status_nonzero": sum(1 for s in statuses if s != 0),
            "learned_vs_plain": learned_line,
            "learned_vs_plain_2d": learned_line_2d,
        }
        print(json.dumps(line), flush=True)
    if eng:
        eng.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
