"""``run_gpu_bls`` and ``get_top_k_candidates``: the reference's fast-path host
functions (search/gpu_bls.py:42-174), backed by the B200 engine.

Arrays come back as numpy arrays (the reference returns CuPy arrays; its
callers call ``.get()`` only when the attribute exists, gpu_bls.py:150-153).
"""
from __future__ import annotations

import numpy as np


def run_gpu_bls(time, flux, periods, durations, flux_err=None, n_bins=200, dtype=np.float32):
    """Fixed-bin BLS of one light curve (gpu_bls.py:42-144)."""
    from .engine import BLSEngine, CurveBatch, SearchConfig, split_outputs

    if len(time) != len(flux):
        raise ValueError("time and flux must have the same length")
    if flux_err is not None and len(flux_err) != len(flux):
        raise ValueError("flux_err must have the same length as flux")
    if int(n_bins) < 2:
        raise ValueError(f"n_bins={n_bins} must be at least 2")
    periods_np = np.atleast_1d(np.asarray(periods, dtype=np.float64))
    durs = np.atleast_1d(np.asarray(durations, dtype=np.float64))
    y = np.asarray(flux)
    batch = CurveBatch.from_arrays([np.asarray(time, np.float64)], [y],
                                   None if flux_err is None else [flux_err],
                                   periods=periods_np, durations=durs,
                                   flux_dtype=np.float64 if y.dtype == np.float64 else np.float32)
    out = split_outputs(batch, BLSEngine.get().search(batch, SearchConfig("fast", n_bins=n_bins)))[0]
    fdt = np.float64 if np.dtype(dtype) == np.float64 else np.float32
    power = out["power"].astype(fdt, copy=False)
    b = out["best_index"]
    return {
        "best_period": float(periods_np[b]),
        "best_t0": float(out["t0"][b]),
        "best_duration": float(out["duration"][b]),
        "best_depth": float(out["depth"][b]),
        "power": power,
        "snr": float(power[b]),
        "all_t0s": out["t0"],
        "all_durs": out["duration"].astype(fdt, copy=False),
        "all_depths": out["depth"].astype(fdt, copy=False),
        "periods": periods_np,
    }


def top_peak_indices(power, k=5, distance=10):
    """Indices of the k largest peaks of `power` at least `distance` samples
    apart, largest first: the local maxima of scipy.signal.find_peaks (flat
    tops reported at their midpoint), the distance rule of find_peaks(distance)
    -- peaks taken by decreasing power, each removing the others closer than
    `distance` -- and, without any peak, the k largest values
    (gpu_bls.py:156-163).  Equal powers are taken higher index first in every
    step (a stable sort read from the end); scipy leaves that order to its
    unstable default sort, so only exact ties can differ from it."""
    from scipy.signal import find_peaks
    power = np.asarray(power)
    peaks, _ = find_peaks(power)
    if len(peaks) == 0:
        return [int(i) for i in np.argsort(power, kind="stable")[-k:][::-1]]
    order = np.argsort(power[peaks], kind="stable")
    keep = np.ones(len(peaks), bool)
    picked = []
    for j in order[::-1]:
        if not keep[j]:
            continue
        picked.append(int(peaks[j]))
        if len(picked) == k:
            break
        lo = j - 1
        while lo >= 0 and peaks[j] - peaks[lo] < distance:
            keep[lo] = False
            lo -= 1
        hi = j + 1
        while hi < len(peaks) and peaks[hi] - peaks[j] < distance:
            keep[hi] = False
            hi += 1
    return picked


def get_top_k_candidates(results, k=5, min_dist_bins=10):
    """Top-k local maxima of the power spectrum (gpu_bls.py:146-174): peaks of
    ``find_peaks(power, distance=min_dist_bins)`` ordered by power, or the k
    largest powers when there is no peak (see ``top_peak_indices``)."""

    def host(a):
        return a.get() if hasattr(a, "get") else np.asarray(a)

    power = host(results["power"])
    t0s = host(results["all_t0s"])
    durs = host(results["all_durs"])
    depths = host(results["all_depths"])
    periods = results["periods"]
    top = top_peak_indices(power, k, min_dist_bins)
    return [{"period": float(periods[i]), "t0": float(t0s[i]), "duration": float(durs[i]),
             "depth": float(depths[i]), "power": float(power[i])} for i in top]
