"""Write tests/golden/ref_golden.npz: outputs of the reference's own CUDA
kernels (compiled from source into oracle/_ref by oracle/Makefile) on a B200.

Run on a GPU machine from the repository root:
    python tests/golden/make_ref_golden.py
Each case stores its inputs and the kernel outputs (power, t0, duration,
depth per period) of the FP64 build (SCALAR_T=double) and, for information,
the FP32 build.  tests/test_oracle.py pins the CPU oracle against them.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, HERE)

import recipes as R  # noqa: E402
from oracle.ref_kernels import RefKernels  # noqa: E402


def sector_small(n=3000, n_periods=400, seed=7):
    t, y, dy = R.sector_curve(n=n, seed=seed)
    return t, y, dy, R.sector_periods(n_periods), R.SECTOR_DURATIONS


def fast_weighted(seed=11):
    rng = np.random.default_rng(seed)
    t = np.sort(rng.uniform(0, 12, 1500))
    y = R.inject_box(t, 1.0 + rng.normal(0, 2e-3, t.size), 2.345, 0.7, 0.12, 4e-3)
    dy = 2e-3 * (1.0 + rng.uniform(size=t.size))
    perm = rng.permutation(t.size)  # unsorted input: t_start = t[0] is not the minimum
    return t[perm], y[perm], dy[perm], np.linspace(1.0, 6.0, 700), np.array([0.05, 0.1, 0.2])


def main():
    import argparse
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.join(HERE, "ref_golden.npz"))
    args = ap.parse_args()
    rk = RefKernels()
    out = {}

    def put(name, arrays):
        for k, v in arrays.items():
            out[f"{name}__{k}"] = np.asarray(v)

    # ---- parity (V42) cases -------------------------------------------------
    v42_cases = {
        "v42_test": (R.v42_test_recipe(), 4000),
        "v42_debug": (R.v42_debug_recipe(), 2000),
        "v42_c0small": (sector_small(), 3600),
        "v42_cap": (sector_small(), 2000),  # reference default cap active for P > 7.96 d
    }
    for name, ((t, y, dy, periods, durs), max_bins) in v42_cases.items():
        w = 1.0 / dy ** 2
        r64 = rk.run_vbls_exact_parity(t, y.reshape(1, -1), periods, durs,
                                       weights_matrix=w.reshape(1, -1), oversample=10,
                                       max_bins=max_bins, dtype=np.float64)
        r32 = rk.run_vbls_exact_parity(t, y.reshape(1, -1), periods, durs,
                                       weights_matrix=w.reshape(1, -1), oversample=10,
                                       max_bins=max_bins, dtype=np.float32)
        put(name, {"t": t, "y": y, "w": w, "periods": periods, "durations": durs,
                   "max_bins": max_bins, "power": r64["power"][0], "t0": r64["t0"][0],
                   "duration": r64["duration"][0], "depth": r64["depth"][0],
                   "power_f32": r32["power"][0]})

    # multi-target on a shared time axis with per-target weights
    rng = np.random.default_rng(5)
    t = np.linspace(0.0, 20.0, 1200)
    ys, ws = [], []
    for k in range(3):
        yk = R.inject_box(t, 1.0 + rng.normal(0, 1e-3, t.size), 2.0 + k, 0.3 * k, 0.1, 3e-3)
        ys.append(yk)
        ws.append(1.0 / (1e-3 * (1.0 + rng.uniform(size=t.size))) ** 2)
    periods = np.linspace(1.5, 5.0, 300)
    durs = np.array([0.06, 0.1, 0.14])
    r64 = rk.run_vbls_exact_parity(t, np.stack(ys), periods, durs, weights_matrix=np.stack(ws),
                                   oversample=10, max_bins=2000, dtype=np.float64)
    put("v42_multi", {"t": t, "y": np.stack(ys), "w": np.stack(ws), "periods": periods,
                      "durations": durs, "max_bins": 2000, "power": r64["power"],
                      "t0": r64["t0"], "duration": r64["duration"], "depth": r64["depth"]})

    # ---- fast (bls.cu) cases ------------------------------------------------
    fast_cases = {
        "bls_astropy_test": (R.astropy_parity_recipe(), 500),
        "bls_recovery": (R.recovery_recipe(), 200),
        "bls_c0small": (sector_small(), 200),
        "bls_weighted_unsorted": (fast_weighted(), 300),
        "bls_nbins1024": (sector_small(n=2000, n_periods=200, seed=3), 1024),
    }
    for name, ((t, y, dy, periods, durs), nb) in fast_cases.items():
        r64 = rk.run_gpu_bls(t, y, periods, durs, flux_err=dy, n_bins=nb, dtype=np.float64)
        r32 = rk.run_gpu_bls(t, y, periods, durs, flux_err=dy, n_bins=nb, dtype=np.float32)
        d = {"t": t, "y": y, "periods": periods, "durations": durs, "n_bins": nb,
             "power": r64["power"], "t0": r64["t0"], "duration": r64["duration"],
             "depth": r64["depth"], "power_f32": r32["power"]}
        if dy is not None:
            d["dy"] = dy
        put(name, d)

    path = args.out
    np.savez_compressed(path, **out)
    print("wrote", path, len(out), "arrays")


if __name__ == "__main__":
    main()
