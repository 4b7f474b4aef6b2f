"""atb_search_curve_static: the entry point that allocates nothing.

Some callers cannot allocate GPU memory while they run -- a host application
that has already reserved nearly all of the device's memory for its own pool,
or a latency-critical loop where cudaMalloc/cudaFree (which may synchronise
the whole device) are not allowed.  For them the library offers a single-curve
search whose working memory is an array built into the library.  These tests
call it through the C ABI and check that two calls in a row give exactly what
the regular (allocating) plan API gives for the same curves.

This file is named so that pytest collects it after every other test.
"""
import ctypes

import numpy as np
import pytest
import torch

import recipes as R
from astro_transit_gpu_b200 import _native as N
from astro_transit_gpu_b200.engine import BLSEngine, CurveBatch, SearchConfig, split_outputs

pytestmark = pytest.mark.gpu

FIELDS = ("power", "depth", "depth_err", "t0", "duration", "window")
DTYPES = {"power": torch.float32, "depth": torch.float32, "depth_err": torch.float32,
          "t0": torch.float64, "duration": torch.float32, "window": torch.int32}


def _ptr(x):
    return None if x is None else ctypes.c_void_p(x.data_ptr())


def call_static(t, y, w, periods, durations, cfg, with_best=True):
    """One call of atb_search_curve_static on cuda:0; returns host outputs
    (best_index is -7 when the call is made without a best-index output)."""
    dev = torch.device("cuda", 0)
    tt = torch.tensor(np.asarray(t, np.float64), device=dev)
    yy = torch.tensor(np.asarray(y), device=dev)
    ww = None if w is None else torch.tensor(np.asarray(w, np.float32), device=dev)
    pp = torch.tensor(np.asarray(periods, np.float64), device=dev)
    dd = torch.tensor(np.asarray(durations, np.float64), device=dev)
    out = {k: torch.full((pp.numel(),), -7, dtype=v, device=dev) for k, v in DTYPES.items()}
    best = torch.full((1,), -7, dtype=torch.int32, device=dev)
    err = ctypes.create_string_buffer(256)
    prm = cfg.params()
    rc = N.load().atb_search_curve_static(
        ctypes.byref(prm), _ptr(tt), _ptr(yy), 1 if yy.dtype == torch.float64 else 0, _ptr(ww),
        tt.numel(), _ptr(pp), pp.numel(), _ptr(dd), dd.numel(),
        *(_ptr(out[k]) for k in FIELDS), _ptr(best) if with_best else None,
        ctypes.c_void_p(torch.cuda.current_stream(dev).cuda_stream), err, len(err))
    host = {k: v.cpu().numpy() for k, v in out.items()}
    host["best_index"] = int(best.item())
    return rc, err.value.decode(), host


def call_plan(t, y, w, periods, durations, cfg):
    """The same search through the regular plan API."""
    b = CurveBatch.from_arrays([t], [np.asarray(y)], periods=periods, durations=durations,
                               flux_dtype=np.asarray(y).dtype, weights=None if w is None else [w])
    return split_outputs(b, BLSEngine.get(0).search(b, cfg))[0]


def assert_same(a, b, name):
    for k in FIELDS:
        assert a[k].dtype == b[k].dtype, (name, k)
        bad = np.flatnonzero(a[k] != b[k])
        assert bad.size == 0, (name, k, bad[:5], a[k][bad[:5]], b[k][bad[:5]])
    assert a["best_index"] == b["best_index"], name


def test_static_entry_matches_plan_api_on_two_calls_in_a_row():
    # call 1: astropy-binned geometry, likelihood objective, float32 flux with weights
    t, y, dy = R.sector_curve(n=15000, seed=11)
    y32 = y.astype(np.float32)
    w = (1.0 / dy ** 2).astype(np.float32)
    periods = R.sector_periods(1200)
    cfg = SearchConfig("parity", objective="likelihood")
    rc, msg, got = call_static(t, y32, w, periods, R.SECTOR_DURATIONS, cfg)
    assert rc == N.ATB_OK, msg
    assert_same(got, call_plan(t, y32, w, periods, R.SECTOR_DURATIONS, cfg), "call 1")

    # call 2, straight after: fixed bins, float64 flux, unit weights, unsorted times,
    # a shorter curve -- the array still holds call 1's larger staging
    rng = np.random.default_rng(3)
    t2 = rng.permutation(np.sort(rng.uniform(200.0, 230.0, 3001)))
    y2 = R.inject_box(t2, 1.0 + rng.normal(0, 1e-3, t2.size), 2.7, 201.0, 0.1, 3e-3)
    periods2 = np.linspace(1.0, 8.0, 777)
    cfg2 = SearchConfig("fast", n_bins=400)
    rc, msg, got2 = call_static(t2, y2, None, periods2, [0.05, 0.1, 0.2], cfg2)
    assert rc == N.ATB_OK, msg
    assert_same(got2, call_plan(t2, y2, None, periods2, [0.05, 0.1, 0.2], cfg2), "call 2")
    assert abs(periods2[got2["best_index"]] - 2.7) < 0.02


def test_static_entry_rejects_what_exceeds_its_scratch():
    cfg = SearchConfig("parity")
    n = N.STATIC_MAX_POINTS + 1
    t = np.linspace(0.0, 30.0, n)
    rc, msg, _ = call_static(t, np.ones(n, np.float32), None, [1.0, 2.0], [0.1], cfg)
    assert rc == N.ATB_EINVAL and "static scratch" in msg
    # periods needing more bins than one shared-memory histogram holds, where
    # the search would need a global histogram: bins finer than the bin-range
    # passes take (oversample > 16), windows too long for a pass, fixed bins
    t = np.linspace(0.0, 30.0, 1000)
    y = np.ones(1000, np.float32)
    rc, msg, _ = call_static(t, y, None, [25.0], [0.01], SearchConfig("parity", oversample=20))
    assert rc == N.ATB_EINVAL and "bins" in msg
    rc, msg, _ = call_static(t, y, None, [25.0], [0.002, 1.5], cfg)
    assert rc == N.ATB_EINVAL and "bins" in msg
    rc, msg, _ = call_static(t, y, None, [25.0], [0.1], SearchConfig("fast", n_bins=100000))
    assert rc == N.ATB_EINVAL and "n_bins" in msg


def test_static_entry_searches_long_periods_in_bin_range_passes():
    """Astropy-binned periods whose bins do not fit one shared-memory
    histogram (here up to 125 000 bins of 0.0002 d) are searched in bin-range
    passes through shared memory, which need no allocated memory: the
    outputs equal the plan API's, bit for bit."""
    rng = np.random.default_rng(21)
    t = np.sort(rng.uniform(1000.0, 1030.0, 6000))
    y = R.inject_box(t, 1.0 + rng.normal(0, 1e-3, t.size), 11.3, 1003.0, 0.12, 5e-3)
    y32 = y.astype(np.float32)
    w = (1.0 / (1e-3 * (1.0 + rng.uniform(size=t.size))) ** 2).astype(np.float32)
    periods = np.concatenate([np.linspace(0.9, 3.0, 40), np.geomspace(10.0, 25.0, 24)])
    durs = [0.002, 0.01, 0.05, 0.12]
    for cfg in (SearchConfig("parity", objective="likelihood"),
                SearchConfig("parity", objective="snr", max_bins=0)):
        rc, msg, got = call_static(t, y32, w, periods, durs, cfg)
        assert rc == N.ATB_OK, msg
        assert_same(got, call_plan(t, y32, w, periods, durs, cfg), cfg.objective)


def test_static_entry_recovers_from_invalid_data_and_runs_without_best_index():
    """A call that meets a NaN flux reports ATB_EDATA; the shared array still
    serves the next call, which matches the plan API bit for bit.  That call
    passes no best-index output, and its grid has more work-queue tiles than
    the launch has CTAs (every CTA takes several tiles)."""
    cfg = SearchConfig("parity", objective="snr")
    t, y, dy = R.sector_curve(n=4000, seed=12)
    y32 = y.astype(np.float32)
    w = (1.0 / dy ** 2).astype(np.float32)
    bad = y32.copy()
    bad[1234] = np.nan
    rc, msg, _ = call_static(t, bad, w, R.sector_periods(300), R.SECTOR_DURATIONS, cfg)
    assert rc == N.ATB_EDATA and "non-finite" in msg
    # 40 000 periods: 625 tiles of 64 against at most 2 CTAs per SM
    periods = np.geomspace(0.5, 13.7, 40000)
    rc, msg, got = call_static(t, y32, w, periods, R.SECTOR_DURATIONS, cfg, with_best=False)
    assert rc == N.ATB_OK, msg
    assert got["best_index"] == -7  # nothing was written there
    ref = call_plan(t, y32, w, periods, R.SECTOR_DURATIONS, cfg)
    got["best_index"] = ref["best_index"]
    assert_same(got, ref, "after invalid data")
    # and a fixed-bin call after it, with the best index, still agrees
    cfg2 = SearchConfig("fast", n_bins=200)
    rc, msg, got2 = call_static(t, y32, w, R.sector_periods(500), R.SECTOR_DURATIONS, cfg2)
    assert rc == N.ATB_OK, msg
    assert_same(got2, call_plan(t, y32, w, R.sector_periods(500), R.SECTOR_DURATIONS, cfg2), "fixed")
