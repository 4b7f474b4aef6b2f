"""Drop-in public API: ``BoxLeastSquaresGPU(t, y, dy).power(...)``.

Mirrors ``search/api.py:27-140`` of the reference (same class, same
``BLSResult``/``Candidate`` fields, same validation errors) and adds per-period
``depth``, ``depth_err``, ``transit_time``, ``duration`` and ``window`` arrays,
an ``objective=`` keyword for the parity method and a batched entry point
:func:`power_batch`.

Behavioural differences from the reference, all deliberate:

* the fold runs in FP64 and bin sums in exact 64-bit fixed point whatever
  ``dtype`` says (``dtype`` only sets the dtype of the returned arrays);
* ``method="parity"`` caps the bin count at ``max_bins - 1`` with the
  reference's default ``max_bins=2000`` (vbls_v42_parity.cu:46-47), so a
  reference caller gets the reference's results; above 7.96 d with 0.004 d
  bins that cap distorts the spectrum, and ``max_bins=None`` (or 0) searches
  every period with its full bin count instead;
* exact ties between windows go to the lowest start bin, then the lowest
  duration index.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Any, Dict, List, Optional, Sequence

import numpy as np

from .engine import BLSEngine, CurveBatch, SearchConfig, is_shared_grid, split_outputs
from .gpu_bls import get_top_k_candidates


@dataclass
class Candidate:
    period: float
    t0: float
    duration: float
    depth: float
    power: float


@dataclass
class BLSResult:
    best_period: float
    best_t0: float
    best_duration: float
    best_depth: float
    best_power: float
    periods: np.ndarray
    power: np.ndarray
    top_candidates: List[Candidate]
    metadata: Dict[str, Any]
    # additions: per-period statistics of the best window
    depth: Optional[np.ndarray] = None
    depth_err: Optional[np.ndarray] = None
    transit_time: Optional[np.ndarray] = None
    duration: Optional[np.ndarray] = None
    window: Optional[np.ndarray] = field(default=None, repr=False)


def _validate(t, y, dy, periods, durations):
    """search/api.py:51-70 plus the length checks of gpu_bls.py:50-54."""
    periods = np.atleast_1d(np.asarray(periods, dtype=np.float64))
    durations = np.atleast_1d(np.asarray(durations, dtype=np.float64))
    if periods.size == 0 or durations.size == 0:
        raise ValueError("periods and durations must not be empty.")
    if np.any(~(periods > 0)):
        raise ValueError("All periods must be positive.")
    if np.any(~(durations > 0)):
        raise ValueError("All durations must be positive.")
    t = np.asarray(t)
    y = np.asarray(y)
    if t.shape != y.shape or t.ndim != 1:
        raise ValueError("time and flux must be 1-D arrays of the same length")
    if np.any(np.isnan(t)) or np.any(np.isnan(y)):
        raise ValueError("Input time or flux contains NaNs.")
    if not (np.all(np.isfinite(t)) and np.all(np.isfinite(y))):
        raise ValueError("Input time or flux contains infinite values.")
    if not np.all(np.isfinite(periods)) or not np.all(np.isfinite(durations)):
        raise ValueError("periods and durations must be finite.")
    if dy is not None:
        dy = np.asarray(dy)
        if np.any(~(dy > 0)):
            raise ValueError("flux_err must be strictly positive for weighted BLS.")
        if len(dy) != len(y):
            raise ValueError("flux_err and flux must have the same length.")
        if not np.all(np.isfinite(dy)):
            raise ValueError("flux_err must be finite.")
    return periods, durations


def _config(method: str, n_bins: int, kwargs: Dict[str, Any]) -> SearchConfig:
    if method == "parity":
        max_bins = kwargs.get("max_bins", 2000)  # the reference's default, api.py:75
        return SearchConfig(method="parity", objective=kwargs.get("objective", "snr"),
                            oversample=int(kwargs.get("oversample", 10)),
                            max_bins=int(max_bins) if max_bins else None)
    if method == "fast":
        if kwargs.get("objective", "fast") != "fast":
            raise ValueError("method='fast' has a single objective; use method='parity'")
        return SearchConfig(method="fast", n_bins=int(n_bins))
    raise ValueError(f"unknown method {method!r} (expected 'fast' or 'parity')")


def _result(periods, out, cfg: SearchConfig, dtype, n_data: int, orig_periods,
            top_idx=None) -> BLSResult:
    """`top_idx`: the device top-5 peak indices (-1 padded); without them the
    host find_peaks path of gpu_bls.get_top_k_candidates is used."""
    fdt = np.dtype(dtype)
    fdt = np.float64 if fdt == np.float64 else np.float32
    power = out["power"].astype(fdt, copy=False)
    bi = int(out["best_index"]) if out.get("best_index", -1) >= 0 else int(np.argmax(power))
    if top_idx is not None:
        top = [Candidate(float(periods[i]), float(out["t0"][i]), float(out["duration"][i]),
                         float(out["depth"][i]), float(power[i])) for i in top_idx if i >= 0]
    else:
        raw = {"power": power, "all_t0s": out["t0"], "all_durs": out["duration"],
               "all_depths": out["depth"], "periods": periods}
        top = [Candidate(float(c["period"]), float(c["t0"]), float(c["duration"]),
                         float(c["depth"]), float(c["power"]))
               for c in get_top_k_candidates(raw, k=5)]
    # the reference reports max_bins as n_bins for the parity method (api.py:103)
    meta = {"n_bins": cfg.n_bins if cfg.method == "fast" else cfg.max_bins,
            "max_bins": cfg.max_bins if cfg.method == "parity" else None,
            "dtype": str(dtype), "n_data": n_data, "method": cfg.method,
            "objective": cfg.objective or ("fast" if cfg.method == "fast" else "snr"),
            "oversample": cfg.oversample if cfg.method == "parity" else None,
            "engine": "astro_transit_gpu_b200"}
    return BLSResult(best_period=float(periods[bi]), best_t0=float(out["t0"][bi]),
                     best_duration=float(out["duration"][bi]), best_depth=float(out["depth"][bi]),
                     best_power=float(power[bi]), periods=orig_periods, power=power,
                     top_candidates=top, metadata=meta,
                     depth=out["depth"].astype(fdt, copy=False),
                     depth_err=out["depth_err"].astype(fdt, copy=False),
                     transit_time=out["t0"], duration=out["duration"].astype(fdt, copy=False),
                     window=out["window"])


class BoxLeastSquaresGPU:
    """Astropy-compatible Box Least Squares on the B200 engine."""

    def __init__(self, t: np.ndarray, y: np.ndarray, dy: Optional[np.ndarray] = None):
        self.t = t
        self.y = y
        self.dy = dy

    def power(self, periods: np.ndarray, durations: np.ndarray, n_bins: int = 200,
              dtype: Any = np.float32, method: str = "fast", **kwargs) -> BLSResult:
        """BLS power spectrum over ``periods`` (see search/api.py:36-49).

        method="fast"   fixed ``n_bins`` phase bins, two-sided score (bls.cu)
        method="parity" Astropy-style bins of min(durations)/oversample; kwargs
                        ``oversample`` (10), ``max_bins`` (2000 as the
                        reference: at most 1999 bins; None or 0 = no cap),
                        ``objective`` ("snr" as the reference, or "likelihood")
        """
        orig = periods
        p, d = _validate(self.t, self.y, self.dy, periods, durations)
        cfg = _config(method, n_bins, kwargs)
        y = np.asarray(self.y)
        fdt = np.float64 if y.dtype == np.float64 else np.float32
        batch = CurveBatch.from_arrays([np.asarray(self.t, np.float64)], [y],
                                       None if self.dy is None else [self.dy],
                                       periods=p, durations=d, flux_dtype=fdt)
        out = split_outputs(batch, BLSEngine.get().search(batch, cfg))[0]
        return _result(p, out, cfg, dtype, len(y), orig if orig is not None else p)


def power_batch(times: Sequence[np.ndarray], fluxes: Sequence[np.ndarray],
                flux_errs: Optional[Sequence[Optional[np.ndarray]]] = None, periods=None,
                durations=None, n_bins: int = 200, dtype: Any = np.float32,
                method: str = "parity", **kwargs) -> List[BLSResult]:
    """Many light curves in one persistent launch.

    ``periods``/``durations`` are one shared grid or one grid per curve."""
    if flux_errs is None:
        flux_errs = [None] * len(times)
    per_curve_p = not is_shared_grid(periods)
    grids_p = periods if per_curve_p else [periods] * len(times)
    per_curve_d = not is_shared_grid(durations)
    grids_d = durations if per_curve_d else [durations] * len(times)
    checked_p, checked_d = [], []
    for t, y, e, pg, dg in zip(times, fluxes, flux_errs, grids_p, grids_d):
        p, d = _validate(t, y, e, pg, dg)
        checked_p.append(p)
        checked_d.append(d)
    cfg = _config(method, n_bins, kwargs)
    fdt = np.float64 if all(np.asarray(y).dtype == np.float64 for y in fluxes) else np.float32
    batch = CurveBatch.from_arrays([np.asarray(t, np.float64) for t in times], fluxes, flux_errs,
                                   periods=checked_p if per_curve_p else checked_p[0],
                                   durations=checked_d if per_curve_d else checked_d[0],
                                   flux_dtype=fdt)
    plan = BLSEngine.get().plan(batch, cfg)
    try:
        plan.execute()
        plan.check()
        top = plan.top_k(5, 10).cpu().numpy()  # peaks found on the device
        outs = split_outputs(batch, plan.outputs)
    finally:
        plan.close()
    return [_result(p, o, cfg, dtype, len(y), p, top_idx=tk)
            for p, o, y, tk in zip(checked_p, outs, fluxes, top)]
