#!/usr/bin/env python
"""Throughput benchmark of the B200 BLS engine (one JSON line on rank 0).

Workload (per GPU): the uniform batch -- 4096 light curves x 15000 float32
points subsampled from a 2-minute cadence over one 27.4 d sector with a 1 d
mid-sector gap (white noise sigma log-U[2e-4, 5e-3], 30 % with a box transit),
5000 log-spaced periods over 0.5-13.7 d, durations [0.04, 0.06, 0.08, 0.12,
0.16, 0.20] d, Astropy-style binning (bin = min duration / 10), likelihood
objective.  Seeded synthetic data of that shape; no dataset is read.

  value   light curves/s with the inputs resident in HBM (device-timed with CUDA
          events over K executions of the search plan, max over ranks)
  e2e     the same through PipelinedSession.run (the batch in 8 runs of curves,
          each a BatchSession on its own stream): every step copies the curves
          from pinned host memory, searches, and copies every per-period output
          back, one run's copies overlapping another's search
  roofline  the search kernel against its binding resource (64-bit
          shared-memory reductions), measured live with CUDA events
  cpu_baseline  the CPU restatement of the reference algorithm (FP64, OpenMP
          over every host core) on a bounded sample of the same curves

Multi-GPU (torchrun): every rank searches its own 4096 curves (weak scaling,
no data-path collective); only the timing barrier and max use NCCL.

`--impl reference` times the reference algorithm's CPU implementation on the
host cores (the FP64 restatement; Astropy, the reference's own CPU path, is
not installed) on rank 0.
"""
from __future__ import annotations

import argparse
import gc
import json
import os
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
ALG_BYTES_PER_FOLD = 16  # two 8-byte shared-memory accumulations per (point, period)
E2E_PARTS = 8  # runs of curves (and streams) of the end-to-end step


def parse():
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
    ap.add_argument("--precision-sample", type=int, default=2,
                    help="precision workload: curves checked against the FP64 oracle")
    ap.add_argument("--method", default="parity", choices=["parity", "fast"])
    ap.add_argument("--curves", type=int, default=None,
                    help="curves per GPU (default 4096 uniform, 8192 mixed)")
    ap.add_argument("--points", type=int, default=15000)
    ap.add_argument("--periods", type=int, default=5000)
    ap.add_argument("--cpu-seconds", type=float, default=15.0,
                    help="target CPU time of the bounded cpu_baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--serving-rate", type=float, default=200.0,
                    help="Poisson arrival rate (requests/s) of the serving measurement")
    ap.add_argument("--serving-seconds", type=float, default=5.0)
    ap.add_argument("--no-serving", action="store_true")
    args = ap.parse_args()
    if args.curves is None:
        args.curves = {"uniform": 4096, "mixed": 8192, "precision": 512}[args.workload]
    return args


def search_config(args):
    from astro_transit_gpu_b200.engine import SearchConfig
    if args.method == "fast":
        return SearchConfig("fast", n_bins=200)
    return SearchConfig("parity", objective="likelihood", oversample=OVERSAMPLE)


def workload_config(args, n_gpus):
    if args.workload == "precision":
        return {
            "workload": (f"precision stress: {args.curves} curves per GPU x 200000 float32 points "
                         "(2-min cadence, 13 sectors, ~356 d, t offset U[1300, 2700] BTJD, "
                         "sigma 5e-4, one 5e-4-deep transit), 100000 frequency-uniform periods "
                         "0.5-150 d, 8 durations 0.02-0.30 d, "
                         + ("fixed 200 bins, fast score" if args.method == "fast" else
                            "astropy-binned (oversample 10), likelihood objective")),
            "n_curves_per_gpu": args.curves, "method": args.method,
            "objective": "fast" if args.method == "fast" else "likelihood",
            "precision": "FP64 fold, int64 fixed-point bin sums, FP32 window search, FP64 winner",
            "l2": "no flush: staged inputs per GPU are about 1.6 GB (L2 is 126 MB)",
            "parallelism": f"dp{n_gpus} (curves sharded across GPUs, no data-path collective)",
            "seed": "precision_curve(default_rng(3000+rank))",
            "launch": "CUDA graph replay of the plan (stage, persistent search, best peak)",
        }
    if args.workload == "mixed":
        return {
            "workload": (f"uneven batch: {args.curves} curves per GPU, N log-U[1e3, 2e5] float32 "
                         "(capped by the cadences available), 1-13 concatenated 27.4 d sectors, "
                         "2- or 30-min cadence, per-curve frequency-uniform grids 0.5 d to "
                         "baseline/2 (4435-59673 periods), 8 durations 0.02-0.30 d, "
                         + ("fixed 200 bins, fast score" if args.method == "fast" else
                            "astropy-binned (oversample 10), likelihood objective")),
            "n_curves_per_gpu": args.curves, "method": args.method,
            "objective": "fast" if args.method == "fast" else "likelihood",
            "precision": "FP64 fold, int64 fixed-point bin sums, FP32 window search, FP64 winner",
            "l2": "no flush: staged inputs per GPU are about 2.5 GB (L2 is 126 MB)",
            "parallelism": f"dp{n_gpus} (curves sharded across GPUs, no data-path collective)",
            "seed": "mixed_batch(seed=2000+rank)",
            "launch": "CUDA graph replay of the plan (stage, persistent search, best peak)",
        }
    return {
        "workload": (f"uniform batch: {args.curves} curves x {args.points} float32 points "
                     "(2-min cadence, 27.4 d sector, 1 d gap) per GPU, "
                     f"{args.periods} log-spaced periods 0.5-13.7 d, 6 durations 0.04-0.20 d, "
                     + ("fixed 200 bins, fast score" if args.method == "fast" else
                        "astropy-binned (oversample 10), likelihood objective")),
        "n_curves_per_gpu": args.curves, "n_points": args.points, "n_periods": args.periods,
        "n_durations": len(DURATIONS), "method": args.method,
        "objective": "fast" if args.method == "fast" else "likelihood",
        "precision": "FP64 fold, int64 fixed-point bin sums, FP32 window search, FP64 winner",
        "l2": ("no flush: staged inputs per GPU are %.0f MB (L2 is 126 MB)"
               % (args.curves * args.points * 16 / 1e6)),
        "parallelism": f"dp{n_gpus} (curves sharded across GPUs, no data-path collective)",
        "seed": "uniform_batch(seed=1000+rank)",
        "launch": "CUDA graph replay of the plan (stage, persistent search, best peak)",
    }


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


def measured_traffic(n_curves):
    """DRAM bytes per search launch from the committed ncu capture, scaled to
    this launch's number of curves (traffic grows in proportion), or None."""
    path = os.path.join(ROOT, "profiles", "search_kernel_uniform_batch.json")
    try:
        with open(path) as f:
            prof = json.load(f)
        return prof["dram_bytes_per_launch"] * n_curves / prof["capture_curves"]
    except (OSError, KeyError, ValueError):
        return None


def make_workload(args, rank):
    """(t, y, w, periods, durations): arrays [curves, n] and one shared grid
    for the uniform batch, lists of per-curve arrays for the mixed batch."""
    import recipes as R
    if args.workload == "precision":
        rng = np.random.default_rng(3000 + rank)
        cs = [R.precision_curve(rng) for _ in range(args.curves)]
        t = np.stack([c[0] for c in cs])
        y = np.stack([c[1] for c in cs])
        w = np.stack([(1.0 / (c[2].astype(np.float64) ** 2)).astype(np.float32) for c in cs])
        return t, y, w, R.precision_periods(), list(R.C3_DURATIONS)
    if args.workload == "mixed":
        cs = R.mixed_batch(args.curves, seed=2000 + rank)
        t = [c[0] for c in cs]
        y = [c[1] for c in cs]
        w = [(1.0 / (c[2].astype(np.float64) ** 2)).astype(np.float32) for c in cs]
        return t, y, w, [c[3] for c in cs], list(R.C2_DURATIONS)
    t, y, dy, truth = R.uniform_batch(n_curves=args.curves, n=args.points, seed=1000 + rank)
    w = (1.0 / (dy.astype(np.float64) ** 2)).astype(np.float32)
    periods = R.c0_periods(args.periods)
    return t, y, w, periods, DURATIONS


def curve_periods(periods, c):
    return periods[c] if isinstance(periods, list) else periods


def cpu_reference(t, y, w, periods, durations, method, budget_s, max_curves=None):
    """The reference algorithm restated on the CPU (FP64, all host cores):
    returns (curves/s, cores, sample description, per-curve outputs)."""
    from oracle import oracle as O
    cores = os.cpu_count() or 1
    outs = []
    n_tot = len(t) if max_curves is None else min(max_curves, len(t))
    t0 = time.perf_counter()
    done = 0
    while done < n_tot:
        pc = curve_periods(periods, done)
        if method == "fast":
            outs.append(O.ref_fixed(t[done], y[done], w[done], pc, durations, n_bins=200,
                                    nthreads=cores))
        else:
            outs.append(O.ref_binned(t[done], y[done], w[done], pc, durations,
                                     oversample=OVERSAMPLE, objective="likelihood",
                                     nthreads=cores))
        done += 1
        if time.perf_counter() - t0 >= budget_s:
            break
    dt = time.perf_counter() - t0
    return done / dt, cores, f"{done} curves of the workload, all periods", outs, dt


def run_reference(args):
    """--impl reference: rank 0 times the CPU implementation of the path."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    t, y, w, periods, durs = make_workload(args, 0)
    per_step = max(1.0, args.cpu_seconds / max(args.steps, 1))
    for _ in range(args.warmup):
        cpu_reference(t, y, w, periods, durs, args.method, budget_s=0.0, max_curves=1)
    total_curves, total_s = 0, 0.0
    for k in range(args.steps):
        sl = slice(k % 64, None)
        rate, cores, _, outs, dt = cpu_reference(
            t[sl], y[sl], w[sl], periods[sl] if isinstance(periods, list) else periods, durs,
            args.method, budget_s=per_step)
        total_curves += len(outs)
        total_s += dt
    value = total_curves / total_s
    cfg = workload_config(args, args.gpus)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * total_s / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": cfg,
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"{total_curves} curves over {args.steps} steps, "
                                   f"~{per_step:.1f} s of CPU work per step, all periods"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "gpu_launches": 0,
    }
    print(json.dumps(line), flush=True)


def precision_report(args, sess, t, y, w, periods, durs):
    """Errors of the engine against the FP64 restatement of the reference on
    the first `--precision-sample` curves (every period): relative power error
    (max, median), and the best peak's period and transit-time differences."""
    from oracle import oracle as O
    gp = sess.host_out["power"].numpy()
    gt0 = sess.host_out["t0"].numpy()
    ob = sess.batch.out_begin
    rel, dper, dt0 = [], [], []
    for c in range(min(args.precision_sample, len(t))):
        if args.method == "fast":
            o = O.ref_fixed(t[c], y[c], w[c], periods, durs, n_bins=200)
        else:
            o = O.ref_binned(t[c], y[c], w[c], periods, durs, oversample=OVERSAMPLE,
                             objective="likelihood")
        n = len(o["power"])
        g = gp[ob[c]:ob[c] + n]
        rel.append(np.abs(g - o["power"]) / np.maximum(o["power"], 1e-30))
        bg, bo = int(np.argmax(g)), int(np.argmax(o["power"]))
        dper.append(abs(periods[bg] - periods[bo]))
        dt0.append(abs(gt0[ob[c] + bg] - o["t0"][bo]))
    r = np.concatenate(rel)
    return {"curves": len(rel), "periods_per_curve": len(periods),
            "max_rel_power_err": float(r.max()), "median_rel_power_err": float(np.median(r)),
            "best_period_abs_diff_d": [float(x) for x in dper],
            "best_t0_abs_diff_d": [float(x) for x in dt0],
            "reference": "oracle FP64 restatement of the reference kernel (fold, sums, windows "
                         "all FP64)"}


def run_serving(args, device):
    """Continuous-batching server under Poisson arrivals: each request is one
    curve of the uneven-batch distribution (fast method, 4-8 durations);
    returns p50/p99 latency from submission to result and the completed rate."""
    import recipes as R
    from astro_transit_gpu_b200.serving import BLSServer
    rng = np.random.default_rng(4000)
    n_req = max(1, int(args.serving_rate * args.serving_seconds))
    reqs = []
    for i in range(n_req):
        n_sec, cad, n, n_per = R.mixed_curve_spec(rng)
        t, y, dy, per = R.mixed_curve(rng, n_sec, cad, n, n_per)
        reqs.append(dict(t=t, y=y, dy=dy, periods=per,
                         durations=R.C2_DURATIONS[:4 + int(rng.integers(0, 5))], method="fast"))
    gaps = rng.exponential(1.0 / args.serving_rate, n_req)
    with BLSServer(device=device, memory_budget=120e9, max_batch=512, n_streams=2) as srv:
        # warm-up (library load, allocator pools at the sizes of large
        # batches): one request, then a burst of 64 at once; not timed
        srv.submit(**reqs[0]).result(timeout=300)
        for f in [srv.submit(**r) for r in reqs[:64]]:
            f.result(timeout=300)
        srv.reset_stats()
        # the objects alive now (this process's workload arrays) are not
        # scanned by the collector while the requests run, as in a server
        gc.collect()
        gc.freeze()
        try:
            t0 = time.perf_counter()
            due = t0 + np.cumsum(gaps)
            futs = []
            for r, d in zip(reqs, due):
                wait = d - time.perf_counter()
                if wait > 0:
                    time.sleep(wait)
                futs.append(srv.submit(**r))
            for f in futs:
                f.result(timeout=300)
        finally:
            gc.unfreeze()
        st = srv.stats()
    return {"arrivals": "Poisson", "offered_rate_per_s": args.serving_rate,
            "requests": n_req, "seconds": args.serving_seconds,
            "p50_ms": st["p50_ms"], "p99_ms": st["p99_ms"], "mean_ms": st["mean_ms"],
            "completed_curves_per_s": st["curves_per_s"], "batches": st["batches"],
            "request": "one uneven-batch curve (N log-U[1e3, 2e5], 1-13 sectors, 4435-59673 "
                       "periods), fast method, 4-8 durations 0.02-0.30 d",
            "admission": "120 GB device-memory budget, up to 512 requests per batch, "
                         "2 batches in flight"}


def main():
    args = parse()
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

    t, y, w, periods, durs = make_workload(args, rank)
    nc = len(t)
    lens = np.array([len(tc) for tc in t], np.int64)
    engine = BLSEngine.get(dev)
    cfg = search_config(args)
    pt = np.zeros(nc + 1, np.int64)
    np.cumsum(lens, out=pt[1:])
    sess = BatchSession(engine, pt, periods, durs, cfg, y_dtype=np.float32, weighted=True)
    sess.load(np.concatenate(t) if isinstance(t, list) else t,
              np.concatenate(y) if isinstance(y, list) else y,
              np.concatenate(w) if isinstance(w, list) else w)
    stream = torch.cuda.current_stream(dev)
    sess.run(stream)  # resident copy of the inputs + first execution
    torch.cuda.synchronize(dev)
    sess.plan.check()
    plan = sess.plan
    sess.capture()  # the step and the search as CUDA graphs (one launch each)
    # end to end: the same batch in E2E_PARTS runs of curves on as many streams,
    # so that copies of one run overlap the search of another
    psess = PipelinedSession(engine, pt, periods, durs, cfg, parts=E2E_PARTS,
                             y_dtype=np.float32, weighted=True)
    psess.load(np.concatenate(t) if isinstance(t, list) else t,
               np.concatenate(y) if isinstance(y, list) else y,
               np.concatenate(w) if isinstance(w, list) else w)
    psess.run(stream)
    torch.cuda.synchronize(dev)
    psess.check()
    psess.capture()

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    from astro_transit_gpu_b200.sharding import max_over_ranks as _max_over_ranks

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
    u_fold = float(sum(int(lens[c]) * len(curve_periods(periods, c)) for c in range(nc)))
    achieved = ALG_BYTES_PER_FOLD * u_fold / (ms_search * 1e-3) / 1e9
    peak = 8.0 * peaks["smem_red_u64_per_s"] / 1e9

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
            "traffic": measured_traffic(nc) if args.workload == "uniform" and args.method == "parity"
            else None,
            "units": f"{ALG_BYTES_PER_FOLD} B of 64-bit shared-memory accumulation per "
                     f"(point, period) fold update; {u_fold:.3e} updates per launch",
            "peak_source": "atb_bench_smem_red_u64 (conflict-free 64-bit shared-memory "
                           "reductions, measured live on this GPU)",
            "ms_search": ms_search, "ms_stage": ms_stage,
            "fp64_fold_rate_per_s": u_fold / (ms_search * 1e-3),
            "dfma_peak_per_s": peaks["dfma_per_s"],
            "smem_red_u64_random_per_s": peaks["smem_red_u64_random_per_s"],
        },
        "clocks": clocks.summary() if rank == 0 else None,
    }
    if rank == 0 and world == 1 and args.workload == "precision":
        line["precision_vs_fp64"] = precision_report(args, sess, t, y, w, periods, durs)
    gp = sess.host_out["power"].numpy().copy()  # the resident run's powers
    ob = np.asarray(sess.batch.out_begin).copy()
    if world == 1 and not args.no_serving:
        # the server runs alone on the device, as in a serving process, and
        # before the CPU baseline loads every host core
        sess.close()
        psess.close()
        del sess, psess, plan
        gc.collect()
        torch.cuda.empty_cache()
        line["serving"] = run_serving(args, dev)
    if rank == 0 and world == 1 and not args.no_cpu_baseline and args.workload != "precision":
        rate, cores, sample, outs, _ = cpu_reference(t, y, w, periods, durs, args.method,
                                                     args.cpu_seconds)
        rel = max(float(np.max(np.abs(gp[ob[c]:ob[c] + len(o["power"])] - o["power"])
                               / np.maximum(o["power"], 1e-30))) for c, o in enumerate(outs))
        line["cpu_baseline"] = {"value": rate, "unit": UNIT, "cores": cores, "kind": "port",
                                "sample": sample,
                                "max_rel_power_err_vs_gpu": rel}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
