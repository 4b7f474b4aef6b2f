"""Batched BLS engine over device tensors.

A :class:`CurveBatch` holds a ragged batch of light curves (each with its own
length, period grid and duration grid) in device memory; :class:`BLSEngine`
binds it to output tensors in a :class:`SearchPlan`, whose ``execute`` only
enqueues the engine's kernels on a CUDA stream (no allocation, no host
synchronisation, so it can be captured in a CUDA graph).

PyTorch is used for device memory and streams only; all compute runs in the
sm_100a kernels of ``libastrotransit_b200.so``.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field, replace
from typing import Dict, List, Optional, Sequence

import numpy as np
import torch

from . import _native as N


@dataclass
class SearchConfig:
    """What to compute.

    method     "fast"   -- fixed ``n_bins`` phase bins, two-sided score (bls.cu)
               "parity" -- bin = min(duration)/oversample, dip-only (V42 kernel)
    objective  "fast" for method="fast"; "snr" (reference) or "likelihood"
               for method="parity"
    max_bins   None = no cap; an int reproduces the reference's cap
               n_bins = min(n_bins, max_bins-1) (vbls_v42_parity.cu:46-47)
    tile_periods  periods per work-queue tile (1..64); 0 = chosen from the
               batch size, or the value BLSEngine.autotune found for this
               kind of batch.  Results never depend on it.
    merge_run  fold strategy: expected time-ordered points per bin from
               which a thread adds the points it holds once when they share a
               slot (0 = the default 8, or the value the autotuner found;
               < 0 = never).  Results never depend on it.
    cta_threads  threads per search CTA: 512 (two CTAs per SM) or 256 (four
               per SM); 0 = the geometry's default, or the autotuner's value.
               Results never depend on it.
    """
    method: str = "parity"
    objective: Optional[str] = None
    n_bins: int = 200
    oversample: int = 10
    max_bins: Optional[int] = None
    tile_periods: int = 0
    merge_run: int = 0
    cta_threads: int = 0

    def params(self) -> N.Params:
        if self.method == "fast":
            obj = self.objective or "fast"
            if obj != "fast":
                raise ValueError("method='fast' uses the reference's fast score")
            return N.Params(N.GEOM_FIXED, N.OBJ_FAST, int(self.n_bins), int(self.oversample), 0,
                            int(self.tile_periods), int(self.merge_run),
                            int(self.cta_threads))
        if self.method == "parity":
            obj = self.objective or "snr"
            if obj not in ("snr", "likelihood"):
                raise ValueError("method='parity' supports objective 'snr' or 'likelihood'")
            mb = 0 if self.max_bins is None else int(self.max_bins)
            return N.Params(N.GEOM_BINNED, N.OBJECTIVES[obj], int(self.n_bins),
                            int(self.oversample), mb, int(self.tile_periods),
                            int(self.merge_run), int(self.cta_threads))
        raise ValueError(f"unknown method {self.method!r} (expected 'fast' or 'parity')")


def is_shared_grid(g) -> bool:
    """True when ``g`` is one 1-D grid (rather than one grid per curve)."""
    if isinstance(g, np.ndarray):
        return g.ndim <= 1
    try:
        return np.asarray(g, dtype=np.float64).ndim <= 1
    except (ValueError, TypeError):
        return False


def _i64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.int64))


def _i32(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32))


@dataclass
class CurveBatch:
    """Ragged batch in device memory plus its host-side index arrays."""
    t: torch.Tensor                 # float64 [sum n]  (or the shared axis, see time_offset)
    y: torch.Tensor                 # float32 or float64 [sum n]
    w: Optional[torch.Tensor]       # float32 [sum n] or None (unit weights)
    periods: torch.Tensor           # float64
    durations: torch.Tensor         # float64
    point_offset: np.ndarray        # int64 [n_curves+1]
    period_begin: np.ndarray        # int64 [n_curves]
    period_count: np.ndarray        # int64 [n_curves]
    dur_begin: np.ndarray           # int64 [n_curves]
    dur_count: np.ndarray           # int32 [n_curves]
    out_begin: np.ndarray           # int64 [n_curves]
    time_offset: Optional[np.ndarray] = None
    _keep: list = field(default_factory=list, repr=False)

    @property
    def n_curves(self) -> int:
        return len(self.period_count)

    @property
    def n_out(self) -> int:
        return int(np.max(self.out_begin + self.period_count)) if self.n_curves else 0

    @property
    def device(self) -> torch.device:
        return self.t.device

    @classmethod
    def from_arrays(cls, times: Sequence[np.ndarray], fluxes: Sequence[np.ndarray],
                    flux_errs: Optional[Sequence[Optional[np.ndarray]]] = None,
                    periods=None, durations=None, device="cuda",
                    flux_dtype=np.float32, weights=None) -> "CurveBatch":
        """Pack host arrays into a device batch.

        ``periods``/``durations`` are either one array shared by every curve or a
        sequence with one array per curve.  Weights are 1/dy^2 rounded to float32
        (None = unit weights, as gpu_bls.py:63-64); ``weights`` passes per-curve
        weight arrays directly instead of ``flux_errs``."""
        nc = len(times)
        if len(fluxes) != nc:
            raise ValueError("times and fluxes must have the same number of curves")
        lens = np.array([len(t) for t in times], dtype=np.int64)
        for t, y in zip(times, fluxes):
            if len(t) != len(y):
                raise ValueError("time and flux must have the same length")
        pt = np.zeros(nc + 1, np.int64)
        np.cumsum(lens, out=pt[1:])
        t_all = np.concatenate([np.asarray(t, np.float64) for t in times]) if nc else np.zeros(0)
        y_all = np.concatenate([np.asarray(y, flux_dtype) for y in fluxes])
        w_all = None
        if weights is not None:
            ws = [np.asarray(wc, np.float32) for wc in weights]
            if any(len(wc) != n for wc, n in zip(ws, lens)):
                raise ValueError("weights and flux must have the same length")
            w_all = np.concatenate(ws)
        elif flux_errs is not None and any(e is not None for e in flux_errs):
            ws = []
            for e, n in zip(flux_errs, lens):
                if e is None:
                    ws.append(np.ones(n, np.float32))
                else:
                    e = np.asarray(e, np.float64)
                    if len(e) != n:
                        raise ValueError("flux_err and flux must have the same length")
                    ws.append((1.0 / (e * e)).astype(np.float32))
            w_all = np.concatenate(ws)

        def grids(g, name):
            if g is None:
                raise ValueError(f"{name} must be given")
            if is_shared_grid(g):
                arr = np.atleast_1d(np.asarray(g, np.float64))
                return arr, np.zeros(nc, np.int64), np.full(nc, len(arr), np.int64)
            if len(g) != nc:
                raise ValueError(f"{name}: one grid per curve expected")
            arrs = [np.atleast_1d(np.asarray(a, np.float64)) for a in g]
            cnt = np.array([len(a) for a in arrs], np.int64)
            beg = np.zeros(nc, np.int64)
            np.cumsum(cnt[:-1], out=beg[1:])
            return np.concatenate(arrs), beg, cnt

        per, pbeg, pcnt = grids(periods, "periods")
        dur, dbeg, dcnt = grids(durations, "durations")
        # the kernels flag these too (ATB_EDATA); rejecting them here runs nothing
        for name, arr in (("periods", per), ("durations", dur)):
            if not np.all(np.isfinite(arr) & (arr > 0)):
                raise ValueError(f"{name} must be positive and finite")
        if np.any(dcnt < 1) or np.any(dcnt > 32):
            raise ValueError("each curve needs 1 to 32 durations")
        obeg = np.zeros(nc, np.int64)
        np.cumsum(pcnt[:-1], out=obeg[1:])

        def dev(a):
            return torch.from_numpy(a).pin_memory().to(device, non_blocking=True)

        return cls(t=dev(t_all), y=dev(y_all), w=None if w_all is None else dev(w_all),
                   periods=dev(per), durations=dev(dur), point_offset=pt, period_begin=pbeg,
                   period_count=pcnt, dur_begin=dbeg, dur_count=_i32(dcnt), out_begin=obeg)


OUTPUT_FIELDS = ("power", "depth", "depth_err", "t0", "duration", "window")
_OUT_DTYPES = {"power": torch.float32, "depth": torch.float32, "depth_err": torch.float32,
               "t0": torch.float64, "duration": torch.float32, "window": torch.int32}


def _ptr(x: Optional[torch.Tensor]):
    return None if x is None else ctypes.c_void_p(x.data_ptr())


class SearchPlan:
    """A batch bound to output tensors; ``execute`` enqueues the search."""

    def __init__(self, engine: "BLSEngine", batch: CurveBatch, config: SearchConfig,
                 outputs: Dict[str, torch.Tensor], stream: Optional[torch.cuda.Stream] = None):
        """With `stream`, the plan is set up and released in that stream's
        order (atb_plan_create_async) and must be executed on it."""
        self.engine = engine
        self.stream = stream
        self.batch = batch
        self.config = config
        self.outputs = outputs
        lib = engine.handle.lib
        self._lib = lib
        # host index arrays must stay alive for the duration of the call only
        idx = {k: getattr(batch, k) for k in ("point_offset", "period_begin", "period_count",
                                              "dur_begin", "out_begin")}
        idx = {k: _i64(v) for k, v in idx.items()}
        dcnt = _i32(batch.dur_count)
        toff = None if batch.time_offset is None else _i64(batch.time_offset)
        b = N.Batch()
        b.n_curves = batch.n_curves
        b.y_is_f64 = 1 if batch.y.dtype == torch.float64 else 0
        b.point_offset = idx["point_offset"].ctypes.data_as(N._i64p)
        b.time_offset = toff.ctypes.data_as(N._i64p) if toff is not None else None
        b.period_begin = idx["period_begin"].ctypes.data_as(N._i64p)
        b.period_count = idx["period_count"].ctypes.data_as(N._i64p)
        b.dur_begin = idx["dur_begin"].ctypes.data_as(N._i64p)
        b.dur_count = dcnt.ctypes.data_as(N._i32p)
        b.out_begin = idx["out_begin"].ctypes.data_as(N._i64p)
        b.t, b.y, b.w = _ptr(batch.t), _ptr(batch.y), _ptr(batch.w)
        b.periods, b.durations = _ptr(batch.periods), _ptr(batch.durations)
        o = N.Outputs()
        for k in OUTPUT_FIELDS:
            setattr(o, k, _ptr(outputs.get(k)))
        o.best_period = _ptr(outputs.get("best_period"))
        o.best_key = _ptr(outputs.get("best_key"))
        self._params = config.params()
        ptr = ctypes.c_void_p()
        with torch.cuda.device(batch.device):
            if stream is None:
                rc = lib.atb_plan_create(engine.handle.ptr, ctypes.byref(self._params),
                                         ctypes.byref(b), ctypes.byref(o), ctypes.byref(ptr))
            else:
                rc = lib.atb_plan_create_async(engine.handle.ptr, ctypes.byref(self._params),
                                               ctypes.byref(b), ctypes.byref(o),
                                               ctypes.c_void_p(stream.cuda_stream),
                                               ctypes.byref(ptr))
        N.raise_for(rc, engine.handle.ptr, "plan creation")
        self.ptr = ptr

    @property
    def kernel_count(self) -> int:
        return int(self._lib.atb_plan_kernel_count(self.ptr))

    @property
    def scratch_bytes(self) -> int:
        return int(self._lib.atb_plan_scratch_bytes(self.ptr))

    def execute(self, stream: Optional[torch.cuda.Stream] = None) -> None:
        s = stream if stream is not None else (
            self.stream or torch.cuda.current_stream(self.batch.device))
        rc = self._lib.atb_plan_execute(self.ptr, ctypes.c_void_p(s.cuda_stream))
        N.raise_for(rc, self.engine.handle.ptr, "plan execution")

    def profile(self, stream: Optional[torch.cuda.Stream] = None) -> Dict[str, float]:
        """Execute once with CUDA events between the kernels (synchronises);
        returns milliseconds of the staging, search and best-peak kernels."""
        s = stream if stream is not None else torch.cuda.current_stream(self.batch.device)
        ms = [ctypes.c_float(0.0) for _ in range(3)]
        rc = self._lib.atb_plan_profile(self.ptr, ctypes.c_void_p(s.cuda_stream),
                                        *(ctypes.byref(m) for m in ms))
        N.raise_for(rc, self.engine.handle.ptr, "plan profile")
        return {"stage": ms[0].value, "search": ms[1].value, "best": ms[2].value}

    def top_k(self, k: int = 5, distance: int = 10,
              stream: Optional[torch.cuda.Stream] = None) -> torch.Tensor:
        """Device top-k peaks of every curve's power after an execution:
        int32 [n_curves, k] period indices (largest peak first, -1 padding),
        as the reference's find_peaks(power, distance) + sort."""
        s = stream if stream is not None else (
            self.stream or torch.cuda.current_stream(self.batch.device))
        out = torch.empty((self.batch.n_curves, k), dtype=torch.int32, device=self.batch.device)
        rc = self._lib.atb_plan_top_k(self.ptr, int(k), int(distance), _ptr(out),
                                      ctypes.c_void_p(s.cuda_stream))
        N.raise_for(rc, self.engine.handle.ptr, "top-k peaks")
        return out

    def curve_layout(self):
        """After an execution: (layout, occupancy_bits) per curve, numpy int32.
        layout is ATB_LAYOUT_SPLIT / COUNT / TIGHT / TIGHT_CHECKED (0 / 1 / 2 /
        3), the histogram word layout the search used; occupancy_bits is the bit length of the
        curve's bound on points per bin (64: no bound).  Synchronous."""
        nc = self.batch.n_curves
        lay = np.zeros(nc, np.int32)
        bits = np.zeros(nc, np.int32)
        rc = self._lib.atb_plan_curve_layout(
            self.ptr, lay.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
            bits.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)))
        N.raise_for(rc, self.engine.handle.ptr, "curve layout")
        return lay, bits

    def check(self) -> None:
        """Synchronise and raise ValueError if the last execution saw invalid data."""
        rc = self._lib.atb_plan_check(self.ptr)
        N.raise_for(rc, self.engine.handle.ptr, "input data")

    def close(self) -> None:
        if getattr(self, "ptr", None):
            self._lib.atb_plan_destroy(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class BLSEngine:
    """Engine bound to one CUDA device."""

    _instances: Dict[int, "BLSEngine"] = {}

    def __init__(self, device=None):
        if not torch.cuda.is_available():
            raise RuntimeError("BLSEngine needs a CUDA device (no CPU fallback)")
        dev = torch.device("cuda", torch.cuda.current_device() if device is None else
                           torch.device(device).index or 0)
        self.device = dev
        self.handle = N.Handle(dev.index)
        from .tuning import TuningTable, table_path
        name = torch.cuda.get_device_name(dev)
        # settings BLSEngine.autotune found for kinds of batch on this kind of
        # device, persisted across processes
        self.tuning = TuningTable(table_path(name, torch.cuda.get_device_capability(dev)), name,
                                  self.handle.lib.atb_version().decode()).load()
        self.last_tune: Dict[str, float] = {}

    @classmethod
    def get(cls, device=None) -> "BLSEngine":
        idx = torch.cuda.current_device() if device is None else (torch.device(device).index or 0)
        eng = cls._instances.get(idx)
        if eng is None:
            eng = cls(torch.device("cuda", idx))
            cls._instances[idx] = eng
        return eng

    def bench_peaks(self) -> Dict[str, float]:
        """Measured denominators of the search kernel's roofline on this device:
        32- and 64-bit shared-memory reductions/s (conflict-free and random
        bins) and FP64 fused multiply-adds/s."""
        out = {}
        v = ctypes.c_double(0.0)
        lib = self.handle.lib
        for name, fn, pat in (("smem_red_u32_per_s", lib.atb_bench_smem_red_u32, 0),
                              ("smem_red_u32_random_per_s", lib.atb_bench_smem_red_u32, 1),
                              ("smem_red_u64_per_s", lib.atb_bench_smem_red_u64, 0),
                              ("smem_red_u64_random_per_s", lib.atb_bench_smem_red_u64, 1)):
            rc = fn(self.handle.ptr, pat, ctypes.byref(v))
            N.raise_for(rc, self.handle.ptr, "smem benchmark")
            out[name] = v.value
        rc = self.handle.lib.atb_bench_dfma(self.handle.ptr, ctypes.byref(v))
        N.raise_for(rc, self.handle.ptr, "dfma benchmark")
        out["dfma_per_s"] = v.value
        return out

    @staticmethod
    def allocate_outputs(batch: CurveBatch, fields: Sequence[str] = OUTPUT_FIELDS,
                         best: bool = True) -> Dict[str, torch.Tensor]:
        n = batch.n_out
        out = {k: torch.empty(n, dtype=_OUT_DTYPES[k], device=batch.device) for k in fields}
        if best:
            out["best_period"] = torch.empty(batch.n_curves, dtype=torch.int32,
                                             device=batch.device)
        return out

    @staticmethod
    def tune_key(batch: CurveBatch, config: SearchConfig):
        """The kind of batch a tuned setting applies to: method, and the
        powers of two of the curve count, mean points and mean periods."""
        nc = max(batch.n_curves, 1)
        pts = float(batch.point_offset[-1]) / nc
        per = float(np.sum(batch.period_count)) / nc
        b = lambda v: int(np.log2(max(v, 1.0)))  # noqa: E731
        return (config.method, b(nc), b(pts), b(per))

    # fold strategies the autotuner tries (merge_run)
    FOLD_CANDIDATES = (0, -1, 4, 16)
    # CTA sizes the autotuner tries (cta_threads)
    SHAPE_CANDIDATES = (512, 256)

    def _time_search(self, batch: CurveBatch, cfg: SearchConfig, repeats: int) -> float:
        plan = SearchPlan(self, batch, cfg, self.allocate_outputs(batch))
        try:
            plan.execute()
            torch.cuda.synchronize(batch.device)
            return min(plan.profile()["search"] for _ in range(max(1, repeats)))
        finally:
            plan.close()

    def autotune(self, batch: CurveBatch, config: SearchConfig,
                 candidates: Sequence[int] = (8, 16, 32, 64),
                 fold_candidates: Sequence[int] = FOLD_CANDIDATES,
                 shape_candidates: Sequence[int] = SHAPE_CANDIDATES, repeats: int = 2,
                 persist: bool = True) -> Dict[str, int]:
        """Time the search kernel on `batch` over the knobs that never change
        a result -- first the CTA sizes in `shape_candidates` (cta_threads),
        then, at the fastest of those, the tile sizes in `candidates`
        (periods per work-queue tile), then the fold strategies in
        `fold_candidates` (merge_run values) -- keep the
        fastest setting for this kind of batch (``tune_key``) in the engine's
        tuning table, written to its file unless `persist` is false, and
        return it.  Later plans whose config leaves a knob at 0 use the tuned
        value, in this process and in later ones."""
        times: Dict[str, float] = {}
        best_nt, best_ms = int(config.cta_threads), None
        for nt in shape_candidates:
            ms = self._time_search(batch, replace(config, cta_threads=int(nt)), repeats)
            times[f"cta={int(nt)}"] = ms
            if best_ms is None or ms < best_ms:
                best_nt, best_ms = int(nt), ms
        best_tp, best_ms = None, None
        for tp in candidates:
            cfg = replace(config, cta_threads=best_nt, tile_periods=int(tp))
            ms = self._time_search(batch, cfg, repeats)
            times[f"cta={best_nt},tile={int(tp)}"] = ms
            if best_ms is None or ms < best_ms:
                best_tp, best_ms = int(tp), ms
        best_fold = int(config.merge_run)
        for mr in fold_candidates:
            cfg = replace(config, cta_threads=best_nt, tile_periods=best_tp, merge_run=int(mr))
            ms = self._time_search(batch, cfg, repeats)
            times[f"cta={best_nt},tile={best_tp},merge_run={mr}"] = ms
            if ms < best_ms:
                best_fold, best_ms = int(mr), ms
        settings = {"tile_periods": best_tp, "merge_run": best_fold}
        if best_nt:
            settings["cta_threads"] = best_nt
        self.tuning.put(self.tune_key(batch, config),
                        {**settings, "search_ms": times, "best_ms": best_ms})
        if persist:
            self.tuning.save()
        self.last_tune = times
        return settings

    def tuned_config(self, batch: CurveBatch, config: SearchConfig) -> SearchConfig:
        """`config` with every knob it leaves at 0 set from the tuning table
        (when this kind of batch has been tuned)."""
        tuned = self.tuning.get(self.tune_key(batch, config))
        if not tuned:
            return config
        upd = {k: int(tuned[k]) for k in ("tile_periods", "merge_run", "cta_threads")
               if k in tuned and getattr(config, k) == 0}
        return replace(config, **upd) if upd else config

    def plan(self, batch: CurveBatch, config: SearchConfig,
             outputs: Optional[Dict[str, torch.Tensor]] = None,
             stream: Optional[torch.cuda.Stream] = None) -> SearchPlan:
        if outputs is None:
            outputs = self.allocate_outputs(batch)
        return SearchPlan(self, batch, self.tuned_config(batch, config), outputs, stream)

    def screen(self, batch: CurveBatch, config: SearchConfig,
               stream: Optional[torch.cuda.Stream] = None) -> Dict[str, torch.Tensor]:
        """Winner-take-all search (the reference's screening mode keeps only a
        best record per target): no per-period array is written -- each
        period raises its curve's packed (power, ~index) record with an
        atomicMax -- then every curve's winning period is searched once more
        to report its window.  Returns per-curve tensors best_index (int32, -1
        when no period has a valid window), period, power, depth, depth_err,
        t0, duration, window: what the full search reports at its best period
        (synchronises)."""
        s = stream if stream is not None else torch.cuda.current_stream(batch.device)
        nc = batch.n_curves
        with torch.cuda.stream(s):
            key = torch.zeros(nc, dtype=torch.int64, device=batch.device)
            best = torch.empty(nc, dtype=torch.int32, device=batch.device)
        plan = self.plan(batch, config, {"best_key": key, "best_period": best})
        try:
            plan.execute(s)
            plan.check()
        finally:
            plan.close()
        # the winning period of every curve, gathered on the device
        with torch.cuda.stream(s):
            pbeg = torch.from_numpy(_i64(batch.period_begin)).to(batch.device)
            idx = torch.clamp(best.to(torch.int64), min=0) + pbeg
            win_p = batch.periods[idx].contiguous()
        one = CurveBatch(t=batch.t, y=batch.y, w=batch.w, periods=win_p,
                         durations=batch.durations, point_offset=batch.point_offset,
                         period_begin=np.arange(nc, dtype=np.int64),
                         period_count=np.ones(nc, np.int64), dur_begin=batch.dur_begin,
                         dur_count=batch.dur_count, out_begin=np.arange(nc, dtype=np.int64),
                         time_offset=batch.time_offset)
        out = {k: v for k, v in self.search(one, config, s).items() if k != "best_period"}
        out["best_index"] = best
        out["period"] = win_p
        return out

    def search(self, batch: CurveBatch, config: SearchConfig,
               stream: Optional[torch.cuda.Stream] = None) -> Dict[str, torch.Tensor]:
        """Plan, execute, check (synchronises) and return the output tensors.
        The plan is made, run and released in `stream`'s order (default: the
        current stream), so its scratch comes from the engine's stream-ordered
        pool and no device-wide allocation or release runs per call."""
        s = stream if stream is not None else torch.cuda.current_stream(batch.device)
        plan = self.plan(batch, config, stream=s)
        try:
            plan.execute(s)
            plan.check()
            return plan.outputs
        finally:
            plan.close()

    def debug_fold(self, t: torch.Tensor, y: torch.Tensor, w: Optional[torch.Tensor],
                   periods: torch.Tensor, durations: torch.Tensor,
                   config: SearchConfig) -> torch.Tensor:
        """Per-point histogram slots [n_periods, n] of one curve (verification)."""
        n, npd = t.numel(), periods.numel()
        out = torch.empty((npd, n), dtype=torch.int32, device=t.device)
        prm = config.params()
        s = torch.cuda.current_stream(t.device)
        rc = self.handle.lib.atb_debug_fold(self.handle.ptr, ctypes.byref(prm), _ptr(t), _ptr(y),
                                            _ptr(w), n, _ptr(periods), npd, _ptr(durations),
                                            durations.numel(), _ptr(out),
                                            ctypes.c_void_p(s.cuda_stream))
        N.raise_for(rc, self.handle.ptr, "debug fold")
        return out


def split_outputs(batch: CurveBatch, outputs: Dict[str, torch.Tensor]) -> List[Dict[str, np.ndarray]]:
    """Host copies of the outputs, one dict per curve."""
    return split_host_outputs(batch, {k: v.cpu().numpy() for k, v in outputs.items()})


def split_host_outputs(batch: CurveBatch, host: Dict[str, np.ndarray]) -> List[Dict[str, np.ndarray]]:
    """One dict per curve of views into host output arrays (every output field
    and, when present, the per-curve best index)."""
    res = []
    for c in range(batch.n_curves):
        b, n = int(batch.out_begin[c]), int(batch.period_count[c])
        d = {k: host[k][b:b + n] for k in OUTPUT_FIELDS if k in host}
        if "best_period" in host:
            d["best_index"] = int(host["best_period"][c])
        res.append(d)
    return res


class BatchSession:
    """A fixed-shape batch kept resident on the device and fed from pinned host
    memory: the end-to-end path of a batch user.

    The period and duration grids are uploaded once; every :meth:`run` copies
    the light curves (t float64, y, w float32) from pinned host buffers to the
    device, executes the plan and copies every per-period output plus the
    per-curve best index back to pinned host buffers, all on one stream.
    """

    def __init__(self, engine: BLSEngine, point_offset: np.ndarray, periods, durations,
                 config: SearchConfig, y_dtype=np.float32, weighted: bool = True,
                 fields: Sequence[str] = OUTPUT_FIELDS):
        dev = engine.device
        pt = _i64(point_offset)
        n_pts = int(pt[-1])
        nc = len(pt) - 1
        tdt = torch.float64 if np.dtype(y_dtype) == np.float64 else torch.float32
        self.host = {
            "t": torch.empty(n_pts, dtype=torch.float64).pin_memory(),
            "y": torch.empty(n_pts, dtype=tdt).pin_memory(),
        }
        if weighted:
            self.host["w"] = torch.empty(n_pts, dtype=torch.float32).pin_memory()
        self.dev_in = {k: torch.empty_like(v, device=dev) for k, v in self.host.items()}
        per, pbeg, pcnt = _grid_arrays(periods, nc)
        dur, dbeg, dcnt = _grid_arrays(durations, nc)
        obeg = np.zeros(nc, np.int64)
        np.cumsum(pcnt[:-1], out=obeg[1:])
        self.batch = CurveBatch(
            t=self.dev_in["t"], y=self.dev_in["y"], w=self.dev_in.get("w"),
            periods=torch.from_numpy(per).to(dev), durations=torch.from_numpy(dur).to(dev),
            point_offset=pt, period_begin=pbeg, period_count=pcnt, dur_begin=dbeg,
            dur_count=_i32(dcnt), out_begin=obeg)
        self.outputs = BLSEngine.allocate_outputs(self.batch, fields)
        self.host_out = {k: torch.empty(v.shape, dtype=v.dtype).pin_memory()
                         for k, v in self.outputs.items()}
        self.plan = engine.plan(self.batch, config, self.outputs)
        self.step_graph = None    # H2D copies + search + D2H copies
        self.search_graph = None  # the search alone (inputs resident)
        # recorded after each step: load() waits for it before it overwrites
        # the pinned inputs the step's copies read
        self._step_done: Optional[torch.cuda.Event] = None

    @property
    def h2d_bytes(self) -> int:
        return sum(v.numel() * v.element_size() for v in self.host.values())

    @property
    def d2h_bytes(self) -> int:
        return sum(v.numel() * v.element_size() for v in self.host_out.values())

    def load(self, t: np.ndarray, y: np.ndarray, w: Optional[np.ndarray] = None) -> None:
        """Fill the pinned host input buffers (flattened, curve after curve).
        Waits first for the last step enqueued by :meth:`run`, whose
        host-to-device copies read these buffers."""
        if self._step_done is not None:
            self._step_done.synchronize()
        self.host["t"].numpy()[:] = np.ravel(t)
        self.host["y"].numpy()[:] = np.ravel(y)
        if "w" in self.host:
            self.host["w"].numpy()[:] = np.ravel(w)

    def _enqueue_step(self, s: torch.cuda.Stream) -> None:
        for k, v in self.host.items():
            self.dev_in[k].copy_(v, non_blocking=True)
        self.plan.execute(s)
        for k, v in self.outputs.items():
            self.host_out[k].copy_(v, non_blocking=True)

    def capture(self) -> None:
        """Record the session's step (input copies, the search's kernels, output
        copies) and the search alone into two CUDA graphs; afterwards
        :meth:`run` and :meth:`search` replay them with one launch each.  The
        graphs read the pinned host buffers, so :meth:`load` between replays
        feeds new light curves of the same shape."""
        dev = self.batch.device
        torch.cuda.synchronize(dev)
        side = torch.cuda.Stream(dev)
        g_step, g_search = torch.cuda.CUDAGraph(), torch.cuda.CUDAGraph()
        with torch.cuda.graph(g_step, stream=side):
            self._enqueue_step(side)
        with torch.cuda.graph(g_search, stream=side):
            self.plan.execute(side)
        torch.cuda.synchronize(dev)
        self.step_graph, self.search_graph = g_step, g_search

    def run(self, stream: Optional[torch.cuda.Stream] = None) -> Dict[str, torch.Tensor]:
        """Enqueue H2D inputs, the search and D2H outputs on `stream` (one graph
        launch after :meth:`capture`); the pinned host outputs are valid once
        the stream has synchronised."""
        s = stream if stream is not None else torch.cuda.current_stream(self.batch.device)
        with torch.cuda.stream(s):
            if self.step_graph is not None:
                self.step_graph.replay()
            else:
                self._enqueue_step(s)
        if self._step_done is None:
            self._step_done = torch.cuda.Event()
        self._step_done.record(s)
        return self.host_out

    def search(self, stream: Optional[torch.cuda.Stream] = None) -> None:
        """Enqueue the search on the resident inputs (graph replay after
        :meth:`capture`)."""
        s = stream if stream is not None else torch.cuda.current_stream(self.batch.device)
        if self.search_graph is not None:
            with torch.cuda.stream(s):
                self.search_graph.replay()
        else:
            self.plan.execute(s)

    def close(self) -> None:
        """Release the graphs, the plan and the device and pinned buffers
        (after the work enqueued so far has finished)."""
        torch.cuda.synchronize(self.batch.device)
        self.step_graph = self.search_graph = None
        self.plan.close()
        self.dev_in, self.outputs, self.host, self.host_out = {}, {}, {}, {}


class PipelinedSession:
    """A fixed-shape batch split into ``parts`` runs of consecutive curves,
    each a :class:`BatchSession` with its own stream.  A step forks from the
    caller's stream, runs every part (inputs in, search, outputs back) on its
    own stream and joins again, so one part's copies cross PCIe while another
    part searches, and one search's last tiles overlap the next one's first.
    Each curve's result depends only on that curve, so the results are those
    of one session over the whole batch."""

    def __init__(self, engine: BLSEngine, point_offset: np.ndarray, periods, durations,
                 config: SearchConfig, parts: int = 4, y_dtype=np.float32,
                 weighted: bool = True, fields: Sequence[str] = OUTPUT_FIELDS):
        pt = _i64(point_offset)
        nc = len(pt) - 1
        if nc < 1:
            raise ValueError("a pipelined session needs at least one curve")
        self.bounds = self.run_bounds(nc, parts)
        self.point_offset = pt
        self.device = engine.device
        self.sessions: List[BatchSession] = []
        self.streams = [torch.cuda.Stream(engine.device) for _ in self.bounds[1:]]
        for a, b in zip(self.bounds[:-1], self.bounds[1:]):
            per = periods if is_shared_grid(periods) else list(periods[a:b])
            dur = durations if is_shared_grid(durations) else list(durations[a:b])
            self.sessions.append(BatchSession(engine, pt[a:b + 1] - pt[a], per, dur, config,
                                              y_dtype, weighted, fields))

    @staticmethod
    def run_bounds(n_curves: int, parts: int) -> List[int]:
        """Curve boundaries of min(parts, n_curves) runs of nearly equal
        size: run i holds curves bounds[i] .. bounds[i+1]-1, none is empty."""
        if n_curves < 1:
            raise ValueError("a pipelined session needs at least one curve")
        parts = max(1, min(int(parts), n_curves))
        return [i * n_curves // parts for i in range(parts + 1)]

    @property
    def h2d_bytes(self) -> int:
        return sum(s.h2d_bytes for s in self.sessions)

    @property
    def d2h_bytes(self) -> int:
        return sum(s.d2h_bytes for s in self.sessions)

    @property
    def kernel_count(self) -> int:
        return sum(s.plan.kernel_count for s in self.sessions)

    def load(self, t: np.ndarray, y: np.ndarray, w: Optional[np.ndarray] = None) -> None:
        """Fill every part's pinned host input buffers (flattened curves)."""
        t, y = np.ravel(t), np.ravel(y)
        w = None if w is None else np.ravel(w)
        for s, a, b in zip(self.sessions, self.bounds[:-1], self.bounds[1:]):
            lo, hi = int(self.point_offset[a]), int(self.point_offset[b])
            s.load(t[lo:hi], y[lo:hi], None if w is None else w[lo:hi])

    def capture(self) -> None:
        for s in self.sessions:
            s.capture()

    def _each(self, stream: Optional[torch.cuda.Stream], fn) -> None:
        main = stream if stream is not None else torch.cuda.current_stream(self.device)
        fork = torch.cuda.Event()
        fork.record(main)
        for s, st in zip(self.sessions, self.streams):
            st.wait_event(fork)
            fn(s, st)
            done = torch.cuda.Event()
            done.record(st)
            main.wait_event(done)

    def run(self, stream: Optional[torch.cuda.Stream] = None) -> List[Dict[str, torch.Tensor]]:
        """Enqueue one step; `stream` (default: the current stream) waits for
        every part, after which each part's pinned host outputs are valid."""
        self._each(stream, lambda s, st: s.run(st))
        return [s.host_out for s in self.sessions]

    def search(self, stream: Optional[torch.cuda.Stream] = None) -> None:
        """The searches alone on the resident inputs, joined on `stream`."""
        self._each(stream, lambda s, st: s.search(st))

    def check(self) -> None:
        for s in self.sessions:
            s.plan.check()

    def close(self) -> None:
        for s in self.sessions:
            s.close()


def _grid_arrays(g, nc):
    if is_shared_grid(g):
        arr = np.atleast_1d(np.asarray(g, np.float64))
        return arr, np.zeros(nc, np.int64), np.full(nc, len(arr), np.int64)
    arrs = [np.atleast_1d(np.asarray(a, np.float64)) for a in g]
    cnt = np.array([len(a) for a in arrs], np.int64)
    beg = np.zeros(nc, np.int64)
    np.cumsum(cnt[:-1], out=beg[1:])
    return np.concatenate(arrs), beg, cnt
