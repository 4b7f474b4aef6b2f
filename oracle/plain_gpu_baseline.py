"""Timing of the plain one-call-per-curve GPU path (the denominator of the
batched-engine speed-up) beside the engine, on curves of the uniform-batch
workload (2-min cadence, 15 000 points, 5 000 log-spaced periods 0.5-13.7 d,
6 durations 0.04-0.20 d).

TEST INFRASTRUCTURE: runs the reference's own kernels (compiled from source
into oracle/_ref by oracle/Makefile) through oracle.ref_kernels, whose host
code restates the reference's CuPy wrappers, one curve per call with the host
prologue, host-to-device copies and result copies included, as the reference
does:

* fast path   search/gpu_bls.py:42-144, bls.cu with SCALAR_T=double, N_TILE=4
              (and the float build, the reference's default dtype)
* parity path search/v42_parity.py:27-107, vbls_v42_parity.cu FP64, one curve
              per launch, max_bins large enough for every period of the grid

and, for comparison, the engine on the same curves: batched (inputs resident),
and one curve per BoxLeastSquaresGPU.power call.  Prints one JSON object.

    python oracle/plain_gpu_baseline.py [--curves 4096] [--sample 32]
"""
import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))

import torch  # noqa: E402

import recipes as R  # noqa: E402
from astro_transit_gpu_b200.api import BoxLeastSquaresGPU  # noqa: E402
from astro_transit_gpu_b200.engine import BatchSession, BLSEngine, SearchConfig  # noqa: E402
from oracle.ref_kernels import RefKernels  # noqa: E402

DURATIONS = np.array([0.04, 0.06, 0.08, 0.12, 0.16, 0.20])


def per_curve_rate(fn, n):
    fn(0)  # warm-up (module load, allocator)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i in range(n):
        fn(i)
    torch.cuda.synchronize()
    return n / (time.perf_counter() - t0)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--curves", type=int, default=4096, help="batched engine batch size")
    ap.add_argument("--sample", type=int, default=32, help="curves timed one call at a time")
    ap.add_argument("--v42-sample", type=int, default=4)
    ap.add_argument("--workload", default="uniform", choices=["uniform", "mixed", "screening"],
                    help="mixed: the uneven batch (fast method only, reference bls.cu vs "
                         "the engine batched); screening: the reference's batched screening "
                         "kernel vs the engine's winner-take-all mode")
    args = ap.parse_args()
    if args.workload == "mixed":
        return mixed(args)
    if args.workload == "screening":
        return screening(args)

    nc = max(args.curves, args.sample)
    t, y, dy, _ = R.uniform_batch(n_curves=nc, n=15000, seed=1000)
    periods = R.sector_periods(5000)
    rk = RefKernels()
    out = {"workload": "uniform batch curves: 15000 points, 5000 log-spaced periods 0.5-13.7 d, "
                       "6 durations 0.04-0.20 d", "sample_curves": args.sample}

    # reference fast path (fixed 200 bins), one curve per call
    for dt, key in ((np.float64, "ref_bls_fp64_per_curve"), (np.float32, "ref_bls_fp32_per_curve")):
        out[key] = per_curve_rate(
            lambda i: rk.run_gpu_bls(t[i], y[i], periods, DURATIONS, flux_err=dy[i], n_bins=200,
                                     dtype=dt), args.sample)
    # reference parity path (astropy-binned), one curve per launch
    nb_max = int(np.ceil(periods.max() / (DURATIONS.min() / 10))) + 10
    out["ref_v42_fp64_per_curve"] = per_curve_rate(
        lambda i: rk.run_vbls_exact_parity(t[i], y[i].reshape(1, -1), periods, DURATIONS,
                                           weights_matrix=(1.0 / dy[i].astype(np.float64) ** 2)
                                           .reshape(1, -1), oversample=10, max_bins=nb_max + 2,
                                           dtype=np.float64), args.v42_sample)
    out["v42_sample_curves"] = args.v42_sample

    # the engine, one curve per public API call (host arrays in, results out)
    for method, key, kw in (("fast", "engine_fast_per_call", {"n_bins": 200}),
                            ("parity", "engine_parity_per_call",
                             {"objective": "likelihood"})):
        out[key] = per_curve_rate(
            lambda i: BoxLeastSquaresGPU(t[i], y[i], dy[i]).power(periods, DURATIONS,
                                                                  method=method, **kw),
            args.sample)

    # the engine batched, inputs resident (device time of the search)
    eng = BLSEngine.get(0)
    w = (1.0 / dy.astype(np.float64) ** 2).astype(np.float32)
    for cfg, key in ((SearchConfig("fast", n_bins=200), "engine_fast_batched"),
                     (SearchConfig("parity", objective="likelihood"), "engine_parity_batched")):
        sess = BatchSession(eng, np.arange(args.curves + 1) * 15000, periods, DURATIONS, cfg,
                            weighted=True)
        sess.load(t[:args.curves], y[:args.curves], w[:args.curves])
        sess.run()
        torch.cuda.synchronize()
        ms = min(sess.plan.profile()["search"] for _ in range(3))
        out[key] = args.curves / (ms * 1e-3)
        del sess
    out["speedup_fast_batched_vs_ref_fp64_per_curve"] = (
        out["engine_fast_batched"] / out["ref_bls_fp64_per_curve"])
    out["speedup_parity_batched_vs_ref_v42_fp64_per_curve"] = (
        out["engine_parity_batched"] / out["ref_v42_fp64_per_curve"])
    print(json.dumps(out))


def mixed(args):
    """Uneven batch, fast method (fixed 200 bins): the reference's bls.cu FP64
    one call per curve on a sample vs the engine batched; light curves/s of the
    sample are scaled by the sample's share of the batch's fold updates so
    that both rates refer to the same curve-size distribution."""
    cs = R.mixed_batch(args.curves, seed=2000)
    durs = R.MIXED_DURATIONS
    rk = RefKernels()
    rng = np.random.default_rng(0)
    idx = np.sort(rng.choice(len(cs), size=min(args.sample, len(cs)), replace=False))
    cost = np.array([len(c[0]) * len(c[3]) for c in cs], np.float64)
    rk.run_gpu_bls(cs[idx[0]][0], cs[idx[0]][1], cs[idx[0]][3], durs, flux_err=cs[idx[0]][2],
                   n_bins=200, dtype=np.float64)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i in idx:
        t, y, dy, per = cs[i]
        rk.run_gpu_bls(t, y, per, durs, flux_err=dy, n_bins=200, dtype=np.float64)
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    # seconds per unit of work on the sample, applied to the whole batch
    ref_rate = len(cs) / (dt * cost.sum() / cost[idx].sum())
    eng = BLSEngine.get(0)
    lens = np.array([len(c[0]) for c in cs], np.int64)
    pt = np.zeros(len(cs) + 1, np.int64)
    np.cumsum(lens, out=pt[1:])
    sess = BatchSession(eng, pt, [c[3] for c in cs], list(durs), SearchConfig("fast", n_bins=200),
                        weighted=True)
    sess.load(np.concatenate([c[0] for c in cs]), np.concatenate([c[1] for c in cs]),
              np.concatenate([(1.0 / c[2].astype(np.float64) ** 2).astype(np.float32)
                              for c in cs]))
    sess.run()
    torch.cuda.synchronize()
    ms = min(sess.plan.profile()["search"] for _ in range(2))
    out = {"workload": f"uneven batch of {len(cs)} curves (mixed_batch seed 2000), fast method, "
                       "fixed 200 bins, 8 durations 0.02-0.30 d",
           "ref_bls_fp64_per_curve": ref_rate, "ref_sample_curves": len(idx),
           "ref_sample_seconds": dt, "engine_fast_batched": len(cs) / (ms * 1e-3),
           "engine_ms_search": ms}
    out["speedup_fast_batched_vs_ref_fp64_per_curve"] = out["engine_fast_batched"] / ref_rate
    print(json.dumps(out))


def screening(args):
    """The reference's screening benchmark shape (scripts/final_validation.py:
    1312 points on linspace(0, 27), 100 000 periods linspace(0.5, 13), 8
    durations linspace(0.01, 0.2), 128 fixed bins): its batched screening
    kernel (float, one best record per target) against the engine's
    winner-take-all mode (FP64 fold, exact bin sums, the fast score) on the
    same targets; both device-timed with the inputs resident."""
    from astro_transit_gpu_b200.engine import CurveBatch, _i32, _i64
    nt = args.curves
    rng = np.random.default_rng(6)
    t = np.linspace(0.0, 27.0, 1312).astype(np.float32)
    sig = np.exp(rng.uniform(np.log(2e-4), np.log(5e-3), nt)).astype(np.float32)
    y = (1.0 + rng.normal(0.0, 1.0, (nt, 1312)) * sig[:, None]).astype(np.float32)
    truth = np.full(nt, np.nan)
    for c in np.flatnonzero(rng.uniform(size=nt) < 0.3):
        P = rng.uniform(0.5, 13.0)
        truth[c] = P
        y[c] = R.inject_box(t.astype(np.float64), y[c].astype(np.float64), P,
                            rng.uniform(0, P), rng.uniform(0.05, 0.2),
                            rng.uniform(3e-3, 1e-2)).astype(np.float32)
    w = np.repeat((1.0 / sig.astype(np.float64) ** 2).astype(np.float32)[:, None], 1312, 1)
    periods = np.linspace(0.5, 13.0, 100000).astype(np.float32)
    durs = np.linspace(0.01, 0.2, 8).astype(np.float32)
    dev = torch.device("cuda", 0)
    rk = RefKernels()
    fm, wm = torch.from_numpy(y).to(dev), torch.from_numpy(w).to(dev)
    # the screening kernel clips flux at 12 sigma around zero: it takes
    # normalised flux minus one, as the sector cache stores it
    # (data/sector_cache.py:57)
    fc = (fm - 1.0).contiguous()
    rk.run_vbls_massive(t, fc[:2], periods[:1000], durs, wm[:2])  # warm-up
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    ref = rk.run_vbls_massive(t, fc, periods, durs, wm, sync=False)
    e1.record()
    torch.cuda.synchronize()
    ms_ref = e0.elapsed_time(e1)
    # the engine: one shared time axis, the same float32 grids widened to float64
    eng = BLSEngine.get(0)
    from astro_transit_gpu_b200.engine import SearchConfig
    batch = CurveBatch(t=torch.from_numpy(t.astype(np.float64)).to(dev), y=fm.reshape(-1),
                       w=wm.reshape(-1), periods=torch.from_numpy(periods.astype(np.float64)).to(dev),
                       durations=torch.from_numpy(durs.astype(np.float64)).to(dev),
                       point_offset=_i64(np.arange(nt + 1) * 1312),
                       period_begin=np.zeros(nt, np.int64),
                       period_count=np.full(nt, len(periods), np.int64),
                       dur_begin=np.zeros(nt, np.int64), dur_count=_i32(np.full(nt, 8)),
                       out_begin=np.zeros(nt, np.int64), time_offset=np.zeros(nt, np.int64))
    cfg = SearchConfig("fast", n_bins=128)
    eng.screen(batch, cfg)  # warm-up
    key = torch.zeros(nt, dtype=torch.int64, device=dev)
    best = torch.empty(nt, dtype=torch.int32, device=dev)
    plan = eng.plan(batch, cfg, {"best_key": key, "best_period": best})
    plan.execute()
    torch.cuda.synchronize()
    ms_eng = min(plan.profile()["search"] for _ in range(3))
    plan.close()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    scr = eng.screen(batch, cfg)
    ms_screen = (time.perf_counter() - t0) * 1e3
    pe = scr["period"].cpu().numpy()
    pr = ref["best_period"].cpu().numpy()
    has = ~np.isnan(truth)
    out = {"workload": f"{nt} targets x 1312 points (linspace 0-27 d), 100000 periods "
                       "linspace(0.5, 13), 8 durations linspace(0.01, 0.2), 128 bins",
           "ref_v39_batched_lc_per_s": nt / (ms_ref * 1e-3), "ref_v39_ms": ms_ref,
           "engine_screen_search_lc_per_s": nt / (ms_eng * 1e-3), "engine_search_ms": ms_eng,
           "engine_screen_wall_lc_per_s": nt / (ms_screen * 1e-3),
           "speedup_search_vs_v39": ms_ref / ms_eng,
           "best_period_agreement_1pct": float(np.mean(np.abs(pe - pr) / pr < 0.01)),
           "injected_recovered_engine_1pct": float(np.mean(
               np.abs(pe[has] - truth[has]) / truth[has] < 0.01)),
           "injected_recovered_v39_1pct": float(np.mean(
               np.abs(pr[has] - truth[has]) / truth[has] < 0.01))}
    print(json.dumps(out))


if __name__ == "__main__":
    main()
