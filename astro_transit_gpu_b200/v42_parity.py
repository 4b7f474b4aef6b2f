"""``run_vbls_exact_parity``: the reference's multi-target parity-path host
function (search/v42_parity.py:27-107), backed by the B200 engine.

``flux_matrix`` is [n_targets, n_data] on the shared ``time_array``.
``max_bins`` defaults to the reference's 2000 (at most 1999 bins per period,
vbls_v42_parity.cu:46-47); None or 0 searches every period with its full bin
count.
"""
from __future__ import annotations

import numpy as np


def run_vbls_exact_parity(time_array, flux_matrix, periods, durations, weights_matrix=None,
                          oversample=10, max_bins=2000, dtype=None, objective="snr"):
    from .engine import BLSEngine, CurveBatch, SearchConfig

    flux = np.asarray(flux_matrix)
    if flux.ndim != 2:
        raise ValueError("flux_matrix must be [n_targets, n_data]")
    n_targets, n_data = flux.shape
    t = np.asarray(time_array, np.float64)
    if t.shape != (n_data,):
        raise ValueError("time_array must have n_data entries")
    periods = np.atleast_1d(np.asarray(periods, np.float64))
    durations = np.atleast_1d(np.asarray(durations, np.float64))
    if np.any(~(periods > 0)) or np.any(~(durations > 0)):
        raise ValueError("periods and durations must be positive")
    weights = None
    if weights_matrix is not None:
        wm = np.asarray(weights_matrix, np.float64)
        if wm.shape != flux.shape or np.any(~(wm > 0)):
            raise ValueError("weights_matrix must match flux_matrix and be positive")
        weights = [wm[i] for i in range(n_targets)]
    fdt = np.float64 if flux.dtype == np.float64 else np.float32
    batch = CurveBatch.from_arrays([t] * n_targets, [flux[i] for i in range(n_targets)],
                                   periods=periods, durations=durations, flux_dtype=fdt,
                                   weights=weights)
    cfg = SearchConfig("parity", objective=objective, oversample=int(oversample),
                       max_bins=int(max_bins) if max_bins else None)
    out = BLSEngine.get().search(batch, cfg)
    host = {k: v.cpu().numpy() for k, v in out.items()}
    odt = np.float64 if dtype is not None and np.dtype(dtype) == np.float64 else np.float32
    power = host["power"].reshape(n_targets, -1).astype(odt, copy=False)
    t0 = host["t0"].reshape(n_targets, -1)
    dur = host["duration"].reshape(n_targets, -1).astype(odt, copy=False)
    dep = host["depth"].reshape(n_targets, -1).astype(odt, copy=False)
    bi = host["best_period"].astype(np.int64)
    rows = np.arange(n_targets)
    return {
        "snr": power[rows, bi],
        "best_period": periods[bi],
        "best_t0": t0[rows, bi],
        "best_duration": dur[rows, bi],
        "best_depth": dep[rows, bi],
        "power_array": power,
        "t0_array": t0,
        "dur_array": dur,
        "depth_array": dep,
    }

