#!/usr/bin/env python
"""Throughput benchmark of the B200 BLS engine (one JSON line on rank 0).

Workload (per GPU, default): the uniform batch -- 4096 light curves x 15000
float32 points subsampled from a 2-minute cadence over one 27.4 d sector with a
1 d mid-sector gap (white noise sigma log-U[2e-4, 5e-3], 30 % with a box
transit), 5000 log-spaced periods over 0.5-13.7 d, durations [0.04, 0.06,
0.08, 0.12, 0.16, 0.20] d, Astropy-style binning (bin = min duration / 10),
likelihood objective.  Seeded synthetic data of that shape; no dataset is read.
`--workload mixed` is the uneven batch (8192 curves per GPU), `--workload
precision` the 512 x 200000-point precision stress.

  value   light curves/s with the inputs resident in HBM (device-timed with CUDA
          events over K executions of the search plan, max over ranks)
  e2e     the same through PipelinedSession.run (the batch in 8 runs of curves,
          each a BatchSession on its own stream): every step copies the curves
          from pinned host memory, searches, and copies every per-period output
          back, one run's copies overlapping another's search
  roofline  the search kernel against its binding resource, the 32-bit
          shared-memory reductions its histogram layouts issue, measured live
          with CUDA events against a live microbenchmark of that reduction
  vs_baseline  value / the plain one-call-per-curve FP64-fold GPU path (the
          reference's bls.cu built with SCALAR_T=double, launched per curve
          with its host prologue and copies) timed in the same run on a sample
          of the same curves (`plain_gpu_baseline`)
  cpu_baseline  the CPU restatement of the reference algorithm (FP64, OpenMP
          over every host core) on a bounded sample of the same curves, with
          the engine's errors against it (power, depth, best period, t0)
  top_k   the device top-5 peaks of every curve (the reference's candidate
          list) after the timed regions: time per launch, bytes against HBM,
          and the indices checked against the host rule on a sample of curves

Multi-GPU: `--gpus N` starts N ranks under torchrun (unless already launched
by torchrun); every rank searches its own share of the curves (weak scaling:
the uniform batch per rank, an LPT share of N x 8192 uneven curves), with no
data-path collective; only the timing barrier and the max over ranks use NCCL.

`--impl reference` times the reference algorithm's CPU implementation on the
host cores (the FP64 restatement; Astropy, the reference's own CPU path, is
not installed) on rank 0.
"""
from __future__ import annotations

import argparse
import gc
import json
import os
import socket
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))

METRIC = "BLS light curves/sec (batched vs plain GPU path) at ≤1e-5 power err; p50/p99"
UNIT = "light_curves/s"
DURATIONS = [0.04, 0.06, 0.08, 0.12, 0.16, 0.20]
OVERSAMPLE = 10
E2E_PARTS = 8  # runs of curves (and streams) of the end-to-end step
# 32-bit shared-memory reductions per (point, period) fold update, by the
# histogram word layout the stage kernel chose for the curve
LAYOUT_WORDS = {0: 4, 1: 3, 2: 2, 3: 2}  # split, count, tight, tight (checked)
LAYOUT_NAMES = {0: "split", 1: "count", 2: "tight", 3: "tight_checked"}
U64_BYTES_PER_FOLD = 16  # two 8-byte accumulations per update in a 64-bit design


def parse(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--workload", default="uniform", choices=["uniform", "mixed", "precision"],
                    help="uniform: the 4096 x 15000 batch (default); mixed: the uneven batch "
                         "(N log-U[1e3, 2e5], 1-13 sectors, per-curve period grids); "
                         "precision: 512 x 200000 points over ~356 d, 100000 periods "
                         "0.5-150 d (errors against the FP64 oracle on a sample)")
    ap.add_argument("--precision-sample", type=int, default=8,
                    help="precision workload: curves checked against the FP64 oracle")
    ap.add_argument("--method", default="parity", choices=["parity", "fast"])
    ap.add_argument("--curves", type=int, default=None,
                    help="curves per GPU (default 4096 uniform, 8192 mixed, 512 precision)")
    ap.add_argument("--points", type=int, default=15000)
    ap.add_argument("--periods", type=int, default=5000)
    ap.add_argument("--cpu-seconds", type=float, default=15.0,
                    help="target CPU time of the bounded cpu_baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--plain-seconds", type=float, default=8.0,
                    help="target time of the plain one-call-per-curve GPU path sample")
    ap.add_argument("--no-plain-gpu", action="store_true")
    ap.add_argument("--serving-rate", type=float, default=200.0,
                    help="Poisson arrival rate (requests/s) of the serving measurement")
    ap.add_argument("--serving-seconds", type=float, default=5.0)
    ap.add_argument("--serving-rates", default=None,
                    help="comma-separated arrival rates of a serving sweep (e.g. "
                         "50,200,1000,2000), each for --serving-seconds, compared with a "
                         "one-call-per-curve loop over the same requests")
    ap.add_argument("--serving-streams", type=int, default=4,
                    help="batches the server keeps in flight (one CUDA stream each)")
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--launch-check", action="store_true",
                    help="start the ranks, report the world size every rank sees, exit "
                         "(no GPU work)")
    args = ap.parse_args(argv)
    if args.curves is None:
        args.curves = {"uniform": 4096, "mixed": 8192, "precision": 512}[args.workload]
    return args


# ----------------------------------------------------------------- ranks ---

def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def relaunch_ranks(n: int, argv) -> int:
    """Run this script as `n` ranks under torchrun (one process per GPU) and
    return torchrun's exit code."""
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           f"--nproc-per-node={n}", "--master-addr", "127.0.0.1",
           "--master-port", str(free_port()), os.path.abspath(__file__), *argv]
    return subprocess.call(cmd)


def launch_check(args):
    """Every rank joins a process group and checks the world size with one
    all-reduce; rank 0 prints what it saw."""
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    seen = world
    if world > 1:
        dist.init_process_group("gloo", timeout=timedelta(seconds=60))
        v = torch.ones(1)
        dist.all_reduce(v)
        seen = int(v.item())
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps({"launch_check": True, "world_size": world, "ranks_seen": seen,
                          "gpus_requested": args.gpus}), flush=True)


# -------------------------------------------------------------- workload ---

def search_config(args):
    from astro_transit_gpu_b200.engine import SearchConfig
    if args.method == "fast":
        return SearchConfig("fast", n_bins=200)
    return SearchConfig("parity", objective="likelihood", oversample=OVERSAMPLE)


def method_text(args):
    return ("fixed 200 bins, fast score" if args.method == "fast" else
            "astropy-binned (oversample 10, no bin cap), likelihood objective")


def workload_config(args, n_gpus):
    common = {
        "n_curves_per_gpu": args.curves, "method": args.method,
        "objective": "fast" if args.method == "fast" else "likelihood",
        "precision": "FP64 fold, int64 fixed-point bin sums, FP32 window search, FP64 winner",
        "parallelism": f"dp{n_gpus} (curves sharded across GPUs, no data-path collective)",
        "launch": "CUDA graph replay of the plan (stage, persistent search, best peak)",
    }
    if args.workload == "precision":
        return {"workload": (f"precision stress: {args.curves} curves per GPU x 200000 float32 "
                             "points (2-min cadence, 13 sectors, ~356 d, t offset U[1300, 2700] "
                             "BTJD, sigma 5e-4, one 5e-4-deep transit), 100000 frequency-uniform "
                             "periods 0.5-150 d, 8 durations 0.02-0.30 d, " + method_text(args)),
                **common,
                "l2": "no flush: staged inputs per GPU are about 1.6 GB (L2 is 126 MB)",
                "seed": "precision_curve(default_rng(3000+rank))"}
    if args.workload == "mixed":
        return {"workload": (f"uneven batch: {args.curves} curves per GPU, N log-U[1e3, 2e5] "
                             "float32 (capped by the cadences available), 1-13 concatenated "
                             "27.4 d sectors, 2- or 30-min cadence, per-curve frequency-uniform "
                             "grids 0.5 d to baseline/2 (1000-60000 periods), 8 durations "
                             "0.02-0.30 d, " + method_text(args)),
                **common,
                "l2": "no flush: staged inputs per GPU are about 2.5 GB (L2 is 126 MB)",
                "seed": f"mixed_curve_indexed(2000, i) for i < {args.curves} x n_gpus, "
                        "LPT split over the ranks by points x periods"}
    return {"workload": (f"uniform batch: {args.curves} curves x {args.points} float32 points "
                         "(2-min cadence, 27.4 d sector, 1 d gap) per GPU, "
                         f"{args.periods} log-spaced periods 0.5-13.7 d, 6 durations "
                         "0.04-0.20 d, " + method_text(args)),
            **common, "n_points": args.points, "n_periods": args.periods,
            "n_durations": len(DURATIONS),
            "l2": ("no flush: staged inputs per GPU are %.0f MB (L2 is 126 MB)"
                   % (args.curves * args.points * 16 / 1e6)),
            "seed": "uniform_batch(seed=1000+rank)"}


def make_workload(args, rank, world):
    """Dict with t, y, dy, w (arrays [curves, n] or lists of per-curve arrays),
    periods (one grid or a list of per-curve grids) and durations."""
    import recipes as R
    from astro_transit_gpu_b200.sharding import lpt_assign

    def weights(dy):
        return (1.0 / (np.asarray(dy, np.float64) ** 2)).astype(np.float32)

    if args.workload == "precision":
        rng = np.random.default_rng(3000 + rank)
        cs = [R.precision_curve(rng) for _ in range(args.curves)]
        dy = np.stack([c[2] for c in cs])
        return {"t": np.stack([c[0] for c in cs]), "y": np.stack([c[1] for c in cs]),
                "dy": dy, "w": weights(dy), "periods": R.precision_periods(),
                "durations": list(R.PRECISION_DURATIONS)}
    if args.workload == "mixed":
        total = args.curves * world
        specs = [R.mixed_spec_indexed(2000, i) for i in range(total)]
        cost = [s[2] * s[3] for s in specs]
        mine = lpt_assign(cost, world)[rank] if world > 1 else np.arange(total)
        cs = [R.mixed_curve_indexed(2000, int(i)) for i in mine]
        return {"t": [c[0] for c in cs], "y": [c[1] for c in cs], "dy": [c[2] for c in cs],
                "w": [weights(c[2]) for c in cs], "periods": [c[3] for c in cs],
                "durations": list(R.MIXED_DURATIONS)}
    t, y, dy, _ = R.uniform_batch(n_curves=args.curves, n=args.points, seed=1000 + rank)
    return {"t": t, "y": y, "dy": dy, "w": weights(dy), "periods": R.sector_periods(args.periods),
            "durations": DURATIONS}


def curve_periods(periods, c):
    return periods[c] if isinstance(periods, list) else periods


def flat(a):
    return np.concatenate(a) if isinstance(a, list) else a


# ------------------------------------------------------------- baselines ---

def error_summary(gpu_power, gpu_depth, gpu_t0, ora, periods_of):
    """Errors of the engine against the FP64 restatement of the reference, per
    curve list: relative power error (max, median), relative depth error where
    both pick the same winning window and the FP64 runner-up trails by more
    than 1e-5 (max, median, share of periods compared), and the best peak's
    period and transit-time differences."""
    rel_p, rel_d, n_cmp, n_all, dper, dt0 = [], [], 0, 0, [], []
    for c, o in enumerate(ora):
        gp, gd, gt = gpu_power[c], gpu_depth[c], gpu_t0[c]
        rel_p.append(np.abs(gp - o["power"]) / np.maximum(o["power"], 1e-30))
        ok = (o["gap"] > 1e-5) & (np.abs(o["depth"]) > 0)
        if gd is not None:
            rel_d.append(np.abs(gd[ok] - o["depth"][ok]) / np.abs(o["depth"][ok]))
        n_cmp += int(ok.sum())
        n_all += len(ok)
        per = periods_of(c)
        bg, bo = int(np.argmax(gp)), int(np.argmax(o["power"]))
        dper.append(abs(float(per[bg]) - float(per[bo])))
        dt0.append(abs(float(gt[bg]) - float(o["t0"][bo])))
    rp = np.concatenate(rel_p)
    rd = np.concatenate(rel_d) if rel_d else np.zeros(0)
    return {"curves": len(ora), "periods": int(rp.size),
            "max_rel_power_err": float(rp.max()), "median_rel_power_err": float(np.median(rp)),
            "max_rel_depth_err": float(rd.max()) if rd.size else None,
            "median_rel_depth_err": float(np.median(rd)) if rd.size else None,
            "depth_periods_compared": n_cmp / max(n_all, 1),
            "best_period_identical": float(np.mean(np.asarray(dper) == 0.0)),
            "max_best_period_abs_diff_d": float(max(dper)),
            "max_best_t0_abs_diff_d": float(max(dt0))}


def oracle_curve(wl, c, method, nthreads):
    from oracle import oracle as O
    pc = curve_periods(wl["periods"], c)
    w64 = 1.0 / (np.asarray(wl["dy"][c], np.float64) ** 2)
    if method == "fast":
        return O.ref_fixed(wl["t"][c], wl["y"][c], w64, pc, wl["durations"], n_bins=200,
                           nthreads=nthreads)
    return O.ref_binned(wl["t"][c], wl["y"][c], w64, pc, wl["durations"], oversample=OVERSAMPLE,
                        objective="likelihood", nthreads=nthreads)


def cpu_reference(wl, method, budget_s, first=0, max_curves=None):
    """The reference algorithm restated on the CPU (FP64, all host cores) on
    curves first, first+1, ... until `budget_s` has passed: returns (curves/s,
    cores, sample description, per-curve outputs, seconds)."""
    cores = os.cpu_count() or 1
    n_tot = len(wl["t"]) if max_curves is None else min(max_curves + first, len(wl["t"]))
    outs = []
    t0 = time.perf_counter()
    c = first
    while c < n_tot:
        outs.append(oracle_curve(wl, c, method, cores))
        c += 1
        if time.perf_counter() - t0 >= budget_s:
            break
    dt = time.perf_counter() - t0
    return len(outs) / dt, cores, f"{len(outs)} curves of the workload, all periods", outs, dt


def hbm_peak_gbs():
    """(GB/s, source): the measured copy bandwidth of this pool's B200s when
    MEASURED_PEAKS.json is present, else the earlier measurement on this pool."""
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured copy bandwidth (MEASURED_PEAKS.json)"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback: earlier copy-bandwidth measurement on this pool"


def top_k_report(plan, stream, host_power, out_begin, counts, k=5, distance=10, launches=5,
                 sample=64):
    """Device top-k peaks of every curve (atb_plan_top_k: the reference's
    get_top_k_candidates(k=5, min_dist_bins=10), gpu_bls.py:146-174) after the
    timed regions: mean CUDA-event time per launch on the plan's stream, the
    algorithmic bytes (each curve's power read once, k indices written) against
    HBM, and the device indices checked against the host rule on `sample`
    curves."""
    import torch
    from astro_transit_gpu_b200.gpu_bls import top_peak_indices
    got = plan.top_k(k, distance, stream)  # warm-up, and the result checked below
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(launches):
        plan.top_k(k, distance, stream)
    e1.record(stream)
    e1.synchronize()
    ms = e0.elapsed_time(e1) / launches
    got = got.cpu().numpy()
    nc = len(counts)
    ok = all([int(i) for i in got[c] if i >= 0] ==
             top_peak_indices(host_power[int(out_begin[c]):int(out_begin[c]) + int(counts[c])],
                              k, distance)
             for c in range(min(sample, nc)))
    nbytes = 4.0 * float(np.sum(counts)) + 4.0 * k * nc
    peak, source = hbm_peak_gbs()
    achieved = nbytes / (ms * 1e-3) / 1e9
    return {"kernel": "topk_peaks_kernel", "k": k, "distance": distance, "ms": ms,
            "launches_timed": launches, "bytes_per_launch": nbytes,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_source": source},
            "equals_host_rule_on_curves": min(sample, nc) if ok else 0,
            "matches_host": bool(ok)}


def plain_gpu_baseline(wl, budget_s, device):
    """The plain one-call-per-curve FP64-fold GPU path: the reference's bls.cu
    (SCALAR_T=double, N_TILE=4, 200 fixed bins) run by the reference's host
    logic (search/gpu_bls.py:42-144, restated in oracle.ref_kernels: copies in,
    weighted-mean prologue, launch, results back) for one curve per call, on a
    random sample of the workload's curves until `budget_s` has passed.  With
    curves of unequal cost the rate is scaled by the sample's share of the
    batch's fold updates, so that it refers to the whole batch."""
    import torch
    from oracle.ref_kernels import RefKernels
    rk = RefKernels(device.index)
    nc = len(wl["t"])
    cost = np.array([len(wl["t"][c]) * len(curve_periods(wl["periods"], c)) for c in range(nc)],
                    np.float64)
    order = np.random.default_rng(7).permutation(nc)

    def call(c):
        rk.run_gpu_bls(wl["t"][c], wl["y"][c], curve_periods(wl["periods"], c), wl["durations"],
                       flux_err=wl["dy"][c], n_bins=200, dtype=np.float64)

    call(int(order[0]))  # module load, allocator
    torch.cuda.synchronize(device)
    done = []
    t0 = time.perf_counter()
    for c in order:
        call(int(c))
        done.append(int(c))
        if time.perf_counter() - t0 >= budget_s:
            break
    torch.cuda.synchronize(device)
    dt = time.perf_counter() - t0
    share = cost[done].sum() / cost.sum()
    rate = nc / (dt / share)
    return {"value": rate, "unit": UNIT,
            "path": "reference search/kernels/bls.cu compiled from source (SCALAR_T=double, "
                    "N_TILE=4), fixed 200 bins, one call per curve with the reference's host "
                    "prologue, copies and result read-back (search/gpu_bls.py:42-144)",
            "sample": f"{len(done)} of {nc} curves in {dt:.2f} s, scaled by their share "
                      f"({share:.4f}) of the batch's fold updates",
            "timing": "wall clock around the calls (each call ends with a device-to-host copy)"}


# ---------------------------------------------------------------- serving ---

SERVING_POOL = 2000  # distinct request curves; longer runs draw from them


def serving_pool(n, seed=4000):
    """`n` request curves of the uneven-batch distribution (fast method,
    4-8 durations each)."""
    import recipes as R
    rng = np.random.default_rng(seed)
    pool = []
    for _ in range(n):
        n_sec, cad, npts, n_per = R.mixed_curve_spec(rng)
        t, y, dy, per = R.mixed_curve(rng, n_sec, cad, npts, n_per)
        pool.append(dict(t=t, y=y, dy=dy, periods=per,
                         durations=R.MIXED_DURATIONS[:4 + int(rng.integers(0, 5))], method="fast"))
    return pool


def run_serving(device, rate, seconds, pool, seed=4001, n_streams=4):
    """Continuous-batching server under Poisson arrivals at `rate` requests/s
    for `seconds`: each request is a curve drawn from `pool`; returns p50/p99
    latency from submission to result and the completed rate."""
    from astro_transit_gpu_b200.serving import BLSServer
    rng = np.random.default_rng(seed)
    n_req = max(1, int(rate * seconds))
    # distinct curves while the pool lasts, then draws with replacement
    picks = (rng.permutation(len(pool))[:n_req] if n_req <= len(pool)
             else rng.integers(0, len(pool), n_req))
    gaps = rng.exponential(1.0 / rate, n_req)
    with BLSServer(device=device, memory_budget=120e9, max_batch=512,
                   n_streams=n_streams) as srv:
        # warm-up (library load, allocator pools at the sizes of large
        # batches): one request, then a burst of 64 at once; not timed
        srv.submit(**pool[0]).result(timeout=300)
        for f in [srv.submit(**r) for r in pool[:64]]:
            f.result(timeout=300)
        srv.reset_stats()
        # the objects alive now (this process's workload arrays) are not
        # scanned by the collector while the requests run, as in a server
        gc.collect()
        gc.freeze()
        # completions are counted, not kept: a client drops each result as a
        # server's client would (holding every result of a long run at 2000
        # requests/s would hold ~100 GB of host memory)
        lock, all_done = threading.Lock(), threading.Event()
        state = {"done": 0, "error": None}

        def on_done(fut):
            err = fut.exception()
            with lock:
                state["done"] += 1
                if err is not None and state["error"] is None:
                    state["error"] = err
                if state["done"] == n_req:
                    all_done.set()

        try:
            t0 = time.perf_counter()
            due = t0 + np.cumsum(gaps)
            for i, d in zip(picks, due):
                wait = d - time.perf_counter()
                if wait > 0:
                    time.sleep(wait)
                srv.submit(**pool[int(i)]).add_done_callback(on_done)
            if not all_done.wait(timeout=3600):
                raise TimeoutError("serving requests did not complete")
            wall = time.perf_counter() - t0
        finally:
            gc.unfreeze()
        if state["error"] is not None:
            raise state["error"]
        st = srv.stats()
    return {"arrivals": "Poisson", "offered_rate_per_s": rate, "requests": n_req,
            "seconds": seconds, "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"],
            "mean_ms": st["mean_ms"], "completed_curves_per_s": st["curves_per_s"],
            "wall_s": wall, "batches": st["batches"],
            "request": f"a curve drawn from {len(pool)} of the uneven-batch distribution "
                       "(N log-U[1e3, 2e5], 1-13 sectors, 1000-60000 periods), fast method, "
                       "4-8 durations 0.02-0.30 d",
            "admission": "120 GB device-memory budget, up to 512 requests per batch, "
                         f"{n_streams} batches in flight"}


def per_call_rate(device, pool, n=500):
    """Curves/s of the plain one-call-per-curve path on the same requests: one
    BoxLeastSquaresGPU.power call per curve, back to back (no arrival pacing),
    i.e. the largest rate that path sustains."""
    import torch
    from astro_transit_gpu_b200.api import BoxLeastSquaresGPU
    r0 = pool[0]
    BoxLeastSquaresGPU(r0["t"], r0["y"], r0["dy"]).power(r0["periods"], r0["durations"])
    torch.cuda.synchronize(device)
    reqs = pool[:min(n, len(pool))]
    t0 = time.perf_counter()
    for r in reqs:
        BoxLeastSquaresGPU(r["t"], r["y"], r["dy"]).power(r["periods"], r["durations"],
                                                          method="fast")
    return {"curves_per_s": len(reqs) / (time.perf_counter() - t0), "requests": len(reqs),
            "path": "one BoxLeastSquaresGPU.power call per request, back to back"}


# ------------------------------------------------------------------ arms ---

def run_reference(args):
    """--impl reference: rank 0 times the CPU implementation of the path."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    wl = make_workload(args, 0, 1)
    per_step = max(1.0, args.cpu_seconds / max(args.steps, 1))
    for _ in range(args.warmup):
        cpu_reference(wl, args.method, budget_s=0.0, max_curves=1)
    total_curves, total_s, cores = 0, 0.0, os.cpu_count() or 1
    for k in range(args.steps):
        rate, cores, _, outs, dt = cpu_reference(wl, args.method, budget_s=per_step,
                                                 first=k % 64)
        total_curves += len(outs)
        total_s += dt
    value = total_curves / total_s
    cfg = workload_config(args, args.gpus)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "gpus_used": 0, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * total_s / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": cfg,
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"{total_curves} curves over {args.steps} steps, "
                                   f"~{per_step:.1f} s of CPU work per step, all periods, "
                                   "rank 0 only"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "gpu_launches": 0,
    }
    print(json.dumps(line), flush=True)


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    args = parse(argv)
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(relaunch_ranks(args.gpus, argv))
    if args.launch_check:
        launch_check(args)
        return
    if args.impl == "reference":
        run_reference(args)
        return

    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=dev)

    from astro_transit_gpu_b200.engine import BatchSession, BLSEngine, PipelinedSession
    from astro_transit_gpu_b200.sharding import max_over_ranks as _max_over_ranks

    wl = make_workload(args, rank, world)
    t, y, w, periods, durs = wl["t"], wl["y"], wl["w"], wl["periods"], wl["durations"]
    nc = len(t)
    lens = np.array([len(tc) for tc in t], np.int64)
    engine = BLSEngine.get(dev)
    cfg = search_config(args)
    pt = np.zeros(nc + 1, np.int64)
    np.cumsum(lens, out=pt[1:])
    sess = BatchSession(engine, pt, periods, durs, cfg, y_dtype=np.float32, weighted=True)
    sess.load(flat(t), flat(y), flat(w))
    stream = torch.cuda.current_stream(dev)
    sess.run(stream)  # resident copy of the inputs + first execution
    torch.cuda.synchronize(dev)
    sess.plan.check()
    plan = sess.plan
    layout, _ = plan.curve_layout()
    sess.capture()  # the step and the search as CUDA graphs (one launch each)
    # end to end: the same batch in E2E_PARTS runs of curves on as many streams,
    # so that copies of one run overlap the search of another
    psess = PipelinedSession(engine, pt, periods, durs, cfg, parts=E2E_PARTS,
                             y_dtype=np.float32, weighted=True)
    psess.load(flat(t), flat(y), flat(w))
    psess.run(stream)
    torch.cuda.synchronize(dev)
    psess.check()
    psess.capture()

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    def max_over_ranks(x):
        return _max_over_ranks(x, device=dev)

    for _ in range(args.warmup):
        sess.search(stream)
    barrier()

    # ---- value: inputs resident in HBM
    gpus = list(range(world)) if world > 1 else [local]
    with ClockSampler(gpus if rank == 0 else []) as clocks:
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            sess.search(stream)
        e1.record(stream)
        barrier()
        ms = max_over_ranks(e0.elapsed_time(e1))

        # ---- e2e: pinned host -> device, search, every output back
        barrier()
        e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e2.record(stream)
        for _ in range(args.steps):
            psess.run(stream)
        e3.record(stream)
        barrier()
        ms_e2e = max_over_ranks(e2.elapsed_time(e3))
    sess.plan.check()
    psess.check()
    # the end-to-end outputs are the resident batch's, bit for bit
    e2e_same = all(
        np.array_equal(np.concatenate([o[k].numpy() for o in (s.host_out for s in psess.sessions)]),
                       sess.host_out[k].numpy()) for k in sess.host_out)

    # ---- roofline of the search kernel (events around each kernel)
    prof = [plan.profile(stream) for _ in range(max(3, min(args.steps, 5)))]
    ms_search = float(np.mean([p["search"] for p in prof]))
    ms_stage = float(np.mean([p["stage"] for p in prof]))
    peaks = engine.bench_peaks()
    upd = np.array([int(lens[c]) * len(curve_periods(periods, c)) for c in range(nc)], np.float64)
    u_fold = float(upd.sum())
    words = np.array([LAYOUT_WORDS[int(v)] for v in layout], np.float64)
    red_bytes = float(4.0 * (words * upd).sum())
    achieved = red_bytes / (ms_search * 1e-3) / 1e9
    peak = 4.0 * peaks["smem_red_u32_per_s"] / 1e9
    ach64 = U64_BYTES_PER_FOLD * u_fold / (ms_search * 1e-3) / 1e9
    peak64 = 8.0 * peaks["smem_red_u64_per_s"] / 1e9
    layout_share = {LAYOUT_NAMES[k]: float(upd[layout == k].sum() / u_fold)
                    for k in LAYOUT_NAMES}

    total_curves = world * nc * args.steps
    value = total_curves / (ms * 1e-3)
    e2e_value = total_curves / (ms_e2e * 1e-3)
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(args, world),
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": psess.h2d_bytes,
                "d2h_bytes_per_step": psess.d2h_bytes, "ms_per_step": ms_e2e / args.steps,
                "api": f"PipelinedSession.run ({E2E_PARTS} runs of curves on {E2E_PARTS} "
                       "streams, each a BatchSession: pinned host buffers, CUDA graph)",
                "outputs_equal_resident_run": bool(e2e_same),
                "gpu_launches": psess.kernel_count * args.steps},
        "gpu_launches": plan.kernel_count * args.steps,
        "roofline": {
            "bound": "smem",
            "kernel": "search_kernel<FIXED>" if args.method == "fast" else "search_kernel<BINNED>",
            "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic": measured_traffic(
                args.workload, args.method, nc,
                search_algorithmic_bytes(lens, [len(curve_periods(periods, c))
                                                for c in range(nc)])),
            "traffic_source": "ncu capture of a smaller launch of this workload under profiles/, "
                              "scaled to this launch (null: no capture of this workload)",
            "units": "4 B per 32-bit shared-memory reduction the fold issues: 2, 3 or 4 per "
                     "(point, period) update by the curve's histogram layout (tight, count, "
                     f"split; a checked tight period that is folded again counts 2); "
                     f"{u_fold:.3e} updates and {red_bytes / 4:.3e} reductions per launch",
            "layout_share_of_updates": layout_share,
            "peak_source": "atb_bench_smem_red_u32 (conflict-free 32-bit shared-memory "
                           "reductions, measured live on this GPU)",
            "ms_search": ms_search, "ms_stage": ms_stage,
            "fold_updates_per_s": u_fold / (ms_search * 1e-3),
            "u64_design": {"achieved": ach64, "peak": peak64, "frac": ach64 / peak64,
                           "units": "16 B per update (two 64-bit accumulations), against "
                                    "conflict-free 64-bit shared-memory reductions"},
            "dfma_peak_per_s": peaks["dfma_per_s"],
            "smem_red_u32_random_per_s": peaks["smem_red_u32_random_per_s"],
            "smem_red_u64_random_per_s": peaks["smem_red_u64_random_per_s"],
        },
        "clocks": clocks.summary() if rank == 0 else None,
    }
    if rank == 0 and world == 1 and args.workload == "precision":
        gp = sess.host_out["power"].numpy()
        gd = sess.host_out["depth"].numpy()
        gt = sess.host_out["t0"].numpy()
        ob = sess.batch.out_begin
        ns = min(args.precision_sample, nc)
        ora = [oracle_curve(wl, c, args.method, os.cpu_count() or 1) for c in range(ns)]
        sl = [slice(int(ob[c]), int(ob[c]) + len(ora[c]["power"])) for c in range(ns)]
        line["precision_vs_fp64"] = {
            **error_summary([gp[s] for s in sl], [gd[s] for s in sl], [gt[s] for s in sl], ora,
                            lambda c: curve_periods(periods, c)),
            "reference": "oracle FP64 restatement of the reference kernel (fold, sums, windows "
                         "all FP64)"}
    if rank == 0:
        try:  # an extra report: a failure here must not lose the measured line
            line["top_k"] = top_k_report(
                plan, stream, sess.host_out["power"].numpy(), np.asarray(sess.batch.out_begin),
                np.array([len(curve_periods(periods, c)) for c in range(nc)], np.int64))
        except Exception as e:  # noqa: BLE001
            line["top_k"] = {"error": repr(e)}
    gp = sess.host_out["power"].numpy().copy()  # the resident run's outputs
    gd = sess.host_out["depth"].numpy().copy()
    gt = sess.host_out["t0"].numpy().copy()
    ob = np.asarray(sess.batch.out_begin).copy()
    sess.close()
    psess.close()
    del sess, psess, plan
    gc.collect()
    torch.cuda.empty_cache()
    if rank == 0 and world == 1 and not args.no_plain_gpu:
        pg = plain_gpu_baseline(wl, args.plain_seconds, dev)
        line["plain_gpu_baseline"] = pg
        line["vs_baseline"] = value / pg["value"]
        line["vs_baseline_meaning"] = ("value / plain_gpu_baseline.value: the batched engine "
                                       "against the plain one-call-per-curve FP64-fold GPU path "
                                       "on the same curves, measured in this run")
    if world == 1 and not args.no_serving:
        # the server runs alone on the device, as in a serving process, and
        # before the CPU baseline loads every host core
        rates = ([float(r) for r in args.serving_rates.split(",")] if args.serving_rates
                 else [])
        pool = serving_pool(min(SERVING_POOL, max(64, int(max([args.serving_rate] + rates)
                                                              * args.serving_seconds))))
        line["serving"] = run_serving(dev, args.serving_rate, args.serving_seconds, pool,
                                      n_streams=args.serving_streams)
        if rates:
            line["serving_sweep"] = {
                "rates": [run_serving(dev, r, args.serving_seconds, pool,
                                      n_streams=args.serving_streams) for r in rates],
                "per_call_path": per_call_rate(dev, pool)}
    if rank == 0 and world == 1 and not args.no_cpu_baseline and args.workload != "precision":
        rate, cores, sample, outs, _ = cpu_reference(wl, args.method, args.cpu_seconds)
        sl = [slice(int(ob[c]), int(ob[c]) + len(o["power"])) for c, o in enumerate(outs)]
        line["cpu_baseline"] = {
            "value": rate, "unit": UNIT, "cores": cores, "kind": "port", "sample": sample,
            "errors_of_gpu": error_summary([gp[s] for s in sl], [gd[s] for s in sl],
                                           [gt[s] for s in sl], outs,
                                           lambda c: curve_periods(periods, c))}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


class ClockSampler:
    """nvidia-smi SM clocks and throttle reasons sampled every 200 ms."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpus):
        self.gpus = gpus
        self.rows = []
        self.proc = None

    def __enter__(self):
        if not self.gpus:
            return self
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", ",".join(str(g) for g in self.gpus)],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except (OSError, ValueError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.thread.join(timeout=2)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"]}
        sm = [float(r[1]) for r in self.rows if len(r) > 2 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 2 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows if len(r) >= 9
                          for i, v in enumerate(r[5:9]) if v.lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


def search_algorithmic_bytes(lens, counts):
    """Bytes one search launch must move: 16 B per staged point (curves start
    at multiples of 32 points), 8 B per period read and 28 B of outputs per
    period written."""
    n_pad = (np.asarray(lens, np.int64) + 31) // 32 * 32
    return float(16 * n_pad.sum() + 36 * np.asarray(counts, np.int64).sum())


def measured_traffic(workload, method, n_curves, algo_bytes):
    """DRAM bytes per search launch from the committed ncu capture of the same
    workload and method, scaled to this launch (by curves for the uniform
    batch, by algorithmic bytes for the uneven one: both captures moved their
    algorithmic bytes, so traffic grows in proportion), or None."""
    if workload == "uniform" and method == "parity":
        name = "search_kernel_uniform_batch.json"
    elif workload == "mixed" and method == "fast":
        name = "search_kernel_fixed_uneven_batch.json"
    else:
        return None
    try:
        with open(os.path.join(ROOT, "profiles", name)) as f:
            prof = json.load(f)
        if "capture_algorithmic_bytes" in prof:
            return prof["dram_bytes_per_launch"] * algo_bytes / prof["capture_algorithmic_bytes"]
        return prof["dram_bytes_per_launch"] * n_curves / prof["capture_curves"]
    except (OSError, KeyError, ValueError):
        return None


if __name__ == "__main__":
    main()
