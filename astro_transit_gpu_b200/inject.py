"""Injection/recovery on the batched engine.

The reference runs one fast-path search per injected light curve
(inject/grid.py:8-62).  Here every trial of the grid becomes one curve of a
single batch: the injected curves share the original time axis, so the batch
sends one time array (time offsets 0) and one flux array per trial, and the
whole grid is searched in one persistent launch.  The injection and the
matching rule restate the reference:

* ``inject_box_transit``  inject/box.py:3-29
* ``match_candidate``     validate/match.py:1-40
* ``run_injection_recovery_experiment`` / ``calculate_recovery_map``
                          inject/grid.py:8-67 (same loop order and random
                          epochs, same default grids; n_bins 200 fast path)
"""
from __future__ import annotations

from typing import Dict, List, Optional, Sequence

import numpy as np

DEFAULT_SEARCH_PERIODS = (0.5, 20.0, 5000)          # inject/grid.py:24-25
DEFAULT_SEARCH_DURATIONS = (0.01, 0.2, 5)           # inject/grid.py:27
INJECTED_DURATION = 0.1                             # inject/grid.py:37


def inject_box_transit(time, flux, period, t0, duration, depth):
    """Multiply the in-transit flux by (1 - depth); in transit means
    |((t - t0 + P/2) mod P) - P/2| < duration/2."""
    new_flux = np.array(flux, copy=True)
    phase = (np.asarray(time) - t0 + 0.5 * period) % period - 0.5 * period
    new_flux[np.abs(phase) < 0.5 * duration] *= (1.0 - depth)
    return new_flux


_RATIOS = (("direct", 1.0), ("harmonic", 2.0), ("harmonic_3", 3.0), ("subharmonic", 0.5),
           ("subharmonic_3", 1.0 / 3.0))


def match_candidate(p_detected, t0_detected, p_true, t0_true, p_tol=0.01, t0_tol=0.1,
                    require_t0=True) -> Dict:
    """Whether a detected (period, t0) matches the true signal at a period
    ratio of 1, 2, 3, 1/2 or 1/3 (relative tolerance `p_tol`) with t0 on the
    true transit series (within `t0_tol` days)."""
    if p_true <= 0 or p_detected <= 0:
        return {"is_match": False, "match_type": "none"}
    for m_type, ratio in _RATIOS:
        p_target = p_true * ratio
        p_diff = abs(p_detected - p_target) / p_target
        if p_diff < p_tol:
            if not require_t0 or t0_true is None:
                return {"is_match": True, "match_type": m_type, "p_diff": p_diff}
            phase_diff = abs((t0_detected - t0_true) % p_true)
            phase_diff = min(phase_diff, p_true - phase_diff)
            if phase_diff < t0_tol:
                return {"is_match": True, "match_type": m_type, "p_diff": p_diff,
                        "t0_diff": phase_diff}
    return {"is_match": False, "match_type": "none", "p_diff": abs(p_detected - p_true) / p_true}


def run_injection_recovery_experiment(time, flux, periods_to_inject: Sequence[float],
                                      depths_to_inject: Sequence[float], n_trials: int = 5,
                                      search_periods=None, search_durations=None,
                                      rng: Optional[np.random.Generator] = None,
                                      device="cuda", as_dataframe: bool = True):
    """Every (period, depth, trial) injection searched in one batch.

    Epochs are drawn as the reference does -- ``time[0] + U[0,1) * P`` per
    trial in (period, depth, trial) order -- from ``rng`` or, without one,
    from ``np.random.random`` (the reference's global generator)."""
    from .engine import BLSEngine, CurveBatch, SearchConfig, _i32, _i64, split_outputs
    import torch

    if search_periods is None:
        search_periods = np.linspace(*DEFAULT_SEARCH_PERIODS)
    if search_durations is None:
        search_durations = np.linspace(*DEFAULT_SEARCH_DURATIONS)
    time = np.asarray(time, np.float64)
    flux = np.asarray(flux)
    draw = rng.random if rng is not None else np.random.random
    cells = []
    fluxes = []
    for p_inj in periods_to_inject:
        for d_inj in depths_to_inject:
            for trial in range(n_trials):
                t0_inj = time[0] + draw() * p_inj
                cells.append((float(p_inj), float(d_inj), trial, float(t0_inj)))
                fluxes.append(inject_box_transit(time, flux, p_inj, t0_inj, INJECTED_DURATION,
                                                 d_inj))
    nc = len(cells)
    if nc == 0:
        return [] if not as_dataframe else __import__("pandas").DataFrame([])
    n = len(time)
    per = np.atleast_1d(np.asarray(search_periods, np.float64))
    dur = np.atleast_1d(np.asarray(search_durations, np.float64))
    fdt = np.float64 if flux.dtype == np.float64 else np.float32

    def dev(a):
        return torch.from_numpy(np.ascontiguousarray(a)).to(device)

    batch = CurveBatch(
        t=dev(time), y=dev(np.concatenate(fluxes).astype(fdt)), w=None, periods=dev(per),
        durations=dev(dur), point_offset=_i64(np.arange(nc + 1) * n),
        period_begin=np.zeros(nc, np.int64), period_count=np.full(nc, len(per), np.int64),
        dur_begin=np.zeros(nc, np.int64), dur_count=_i32(np.full(nc, len(dur))),
        out_begin=_i64(np.arange(nc) * len(per)), time_offset=np.zeros(nc, np.int64))
    outs = split_outputs(batch, BLSEngine.get(device).search(batch, SearchConfig("fast", n_bins=200)))
    rows: List[Dict] = []
    for (p_inj, d_inj, trial, t0_inj), o in zip(cells, outs):
        b = o["best_index"]
        best_p, best_t0 = float(per[b]), float(o["t0"][b])
        m = match_candidate(best_p, best_t0, p_inj, t0_inj)
        rows.append({"injected_period": p_inj, "injected_depth": d_inj, "trial": trial,
                     "injected_t0": t0_inj, "is_recovered": m["is_match"],
                     "match_type": m["match_type"], "detected_period": best_p,
                     "detected_t0": best_t0, "snr": float(o["power"][b])})
    if not as_dataframe:
        return rows
    import pandas as pd
    return pd.DataFrame(rows)


def calculate_recovery_map(df):
    """Recovered fraction per (injected period, injected depth) cell."""
    return df.groupby(["injected_period", "injected_depth"])["is_recovered"].mean().unstack()
