"""GPU tests of the histogram word layouts.

Uniform-weight curves whose bin occupancy is provably below 2^12 points use
the two-word layout (ATB_LAYOUT_TIGHT); the others use the three- or four-word
layouts.  The layout must never change a result: every case is bit-exact
against the oracle's mirror of the engine arithmetic, and for every TIGHT curve
the largest bin occupancy actually reached (counted from the per-point slots
of the same fold) stays below the curve's bound.
"""
import numpy as np
import pytest

import recipes as R
from oracle import oracle as O

pytestmark = pytest.mark.gpu

SPLIT, COUNT, TIGHT, CHECKED = 0, 1, 2, 3
FIELDS = ("power", "depth", "depth_err", "t0", "duration", "window")


def _cfg(kind, **kw):
    from astro_transit_gpu_b200.engine import SearchConfig
    if kind == "fixed":
        return SearchConfig("fast", n_bins=kw.get("n_bins") or 200)
    return SearchConfig("parity", objective="snr", max_bins=kw.get("max_bins"), oversample=10)


def run_with_layout(engine, t, y, w, periods, durations, cfg):
    from astro_transit_gpu_b200.engine import CurveBatch, split_outputs
    b = CurveBatch.from_arrays([t], [np.asarray(y, np.float32)], periods=periods,
                               durations=durations, weights=None if w is None else [w])
    plan = engine.plan(b, cfg)
    try:
        plan.execute()
        plan.check()
        lay, bits = plan.curve_layout()
        out = split_outputs(b, plan.outputs)[0]
    finally:
        plan.close()
    return out, int(lay[0]), int(bits[0])


def oracle_for(t, y, w, periods, durs, cfg):
    y = np.asarray(y, np.float32)
    if cfg.method == "fast":
        return O.eng_fixed(t, y, w, periods, durs, n_bins=cfg.n_bins)
    return O.eng_binned(t, y, w, periods, durs, max_bins=cfg.max_bins or 0)


def max_occupancy(engine, t, y, w, periods, durs, cfg):
    import torch
    dev = engine.device
    slots = engine.debug_fold(
        torch.tensor(t, device=dev), torch.tensor(np.asarray(y, np.float32), device=dev),
        None if w is None else torch.tensor(w, device=dev), torch.tensor(periods, device=dev),
        torch.tensor(durs, device=dev), cfg).cpu().numpy()
    worst = 0
    for row in slots:
        cnt = np.bincount(row)
        if cfg.method == "fast":
            cnt = cnt[:-1] if cnt.size > 1 else cnt  # the out-of-range slot is never read
        worst = max(worst, int(cnt.max()))
    return worst


def expected_bits(t, periods, durs, cfg):
    """The kernel's occupancy bound restated: M = (floor(T/P_min) + 3) * K,
    K = most points within one (slightly widened) bin width; 64 = no bound."""
    t = np.asarray(t, np.float64)
    if np.any(np.diff(t) < 0):
        return 64
    if cfg.method == "fast":
        width = periods.max() / cfg.n_bins
    else:
        width = durs.min() / cfg.oversample
        # a bin cap that the largest period reaches piles points into its last bin
        if cfg.max_bins and np.ceil(periods.max() * (1 / width)) + cfg.oversample >= cfg.max_bins:
            return 64
    width = width * (1 + 1e-6) + 1e-12
    k = int((np.searchsorted(t, t + width, side="right") - np.arange(t.size)).max())
    m = (np.floor((t[-1] - t[0]) * (1 / periods).max() * (1 + 1e-9)) + 3) * k
    return 64 if m >= 4096 else int(m).bit_length()


def clustered(n_clusters=40, per_cluster=60, span=27.0, seed=3):
    """Uniform weights, tight bursts of simultaneous samples."""
    rng = np.random.default_rng(seed)
    centres = np.sort(rng.uniform(0, span, n_clusters))
    t = np.sort(np.concatenate([c + rng.uniform(0, 1e-4, per_cluster) for c in centres]))
    y = R.inject_box(t, 1.0 + rng.normal(0, 1e-3, t.size), 3.3, 0.4, 0.12, 3e-3)
    return t + 2000.0, y


CASES = {
    # name: (t, y, w, periods, durations, kind, n_bins, expected layout)
    "sector_uniform": lambda: (*R.sector_curve(n=15000, seed=2)[:2], None, R.sector_periods(600),
                           R.SECTOR_DURATIONS, "binned", None, TIGHT),
    # fixed 200 bins: bound 3819 points, 12 bits (the largest tight layout)
    "sector_uniform_fixed": lambda: (*R.sector_curve(n=15000, seed=2)[:2], None, R.sector_periods(600),
                                 R.SECTOR_DURATIONS, "fixed", 200, TIGHT),
    # bursts of 60 simultaneous samples: bound 3300 points, bins reach 60+
    "clustered": lambda: (*clustered(seed=3), None, np.geomspace(0.5, 13.7, 500),
                          np.array([0.04, 0.1]), "binned", None, TIGHT),
    "clustered_fixed": lambda: (*clustered(seed=5), None, np.geomspace(0.5, 13.7, 500),
                                np.array([0.04, 0.1]), "fixed", 2000, TIGHT),
    # the reference's default cap (max_bins=2000) where no period reaches it:
    # 0.004 d bins up to 7.9 d need at most 1985 bins
    "sector_uniform_cap_not_reached": lambda: (*R.sector_curve(n=15000, seed=2)[:2], None,
                                           R.sector_periods(600, pmax=7.9), R.SECTOR_DURATIONS,
                                           "binned", 2000, TIGHT),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_tight_layout_bound_holds_and_results_bit_exact(engine, name):
    t, y, w, periods, durs, kind, n_bins, expect = CASES[name]()
    cfg = _cfg(kind, n_bins=n_bins, max_bins=n_bins if kind == "binned" else None)
    g, lay, bits = run_with_layout(engine, t, y, w, periods, durs, cfg)
    assert lay == expect, (lay, bits)
    assert bits == expected_bits(t, periods, durs, cfg) <= 12
    assert max_occupancy(engine, t, y, w, periods, durs, cfg) < (1 << bits)
    o = oracle_for(t, y, w, periods, durs, cfg)
    for k in FIELDS:
        assert np.array_equal(np.asarray(g[k]), np.asarray(o[k])), (name, k)


def test_layout_falls_back_when_no_bound(engine):
    """Without a proven occupancy bound, sparse-on-average uniform curves use
    the checked tight layout; a cap that the grid reaches, or non-uniform
    weights, use the count and split layouts."""
    rng = np.random.default_rng(8)
    periods, durs = np.geomspace(0.5, 5.0, 200), np.array([0.05, 0.1])
    # dense: 20000 samples within 0.05 d -> a bound of ~6000 points per bin
    t = np.sort(rng.uniform(0, 0.05, 20000)) + 10.0
    y = 1.0 + rng.normal(0, 1e-3, t.size)
    cases = [
        (t, y, None, "binned", None, CHECKED),
        # unsorted times: no bound is computed
        (rng.permutation(R.sector_curve(n=4000, seed=4)[0]), rng.normal(1, 1e-3, 4000), None,
         "binned", None, CHECKED),
        (t, y, None, "fixed", None, CHECKED),
        # a bin cap that the grid reaches folds many points into the last bin
        (*R.sector_curve(n=4000, seed=4)[:2], None, "binned", 500, COUNT),
        # non-uniform weights
        (*R.sector_curve(n=4000, seed=4)[:2], rng.uniform(1e5, 2e5, 4000).astype(np.float32),
         "binned", None, SPLIT),
    ]
    for t_, y_, w_, kind, mb, expect in cases:
        cfg = _cfg(kind, max_bins=mb)
        g, lay, bits = run_with_layout(engine, t_, y_, w_, periods, durs, cfg)
        assert lay == expect, (expect, lay, bits)
        if w_ is None and expect != CHECKED:
            assert bits == expected_bits(t_, periods, durs, cfg) == 64
        o = oracle_for(t_, y_, w_, periods, durs, cfg)
        for k in FIELDS:
            assert np.array_equal(np.asarray(g[k]), np.asarray(o[k])), (expect, k)


@pytest.mark.parametrize("kind", ["binned", "fixed"])
def test_checked_tight_layout_refolds_overflowing_periods(engine, kind):
    """12 000 samples within 0.002 d among 8 000 spread over 27 d: at every
    period more than 2^12 points share one bin, so every period's count check
    fails and the period is folded again in the count layout; a batch mixing
    that curve with ordinary ones, and the curve alone, match the oracle bit
    for bit."""
    from astro_transit_gpu_b200.engine import CurveBatch, split_outputs
    rng = np.random.default_rng(12)
    t = np.sort(np.concatenate([rng.uniform(0, 0.002, 12000),
                                rng.uniform(0.5, 27.0, 8000)])) + 3000.0
    y = R.inject_box(t, 1.0 + rng.normal(0, 1e-3, t.size), 2.2, 3000.7, 0.1, 3e-3)
    y = y.astype(np.float32)
    periods, durs = np.geomspace(0.5, 10.0, 300), np.array([0.04, 0.08, 0.16])
    cfg = _cfg(kind, n_bins=200)
    g, lay, _ = run_with_layout(engine, t, y, None, periods, durs, cfg)
    assert lay == CHECKED
    o = oracle_for(t, y, None, periods, durs, cfg)
    for k in FIELDS:
        assert np.array_equal(np.asarray(g[k]), np.asarray(o[k])), k
    assert max_occupancy(engine, t, y, None, periods, durs, cfg) >= 4096
    # in a batch with curves that pass the check
    t2, y2 = R.sector_curve(n=9000, seed=13)[:2]
    b = CurveBatch.from_arrays([t2, t, t2], [y2.astype(np.float32), y, y2.astype(np.float32)],
                               periods=periods, durations=durs)
    outs = split_outputs(b, engine.search(b, cfg))
    o2 = oracle_for(t2, y2, None, periods, durs, cfg)
    for k in FIELDS:
        assert np.array_equal(np.asarray(outs[1][k]), np.asarray(o[k])), k
        assert np.array_equal(np.asarray(outs[0][k]), np.asarray(o2[k])), k
        assert np.array_equal(np.asarray(outs[2][k]), np.asarray(o2[k])), k
