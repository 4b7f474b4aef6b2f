"""GPU parity tests: the sm_100a engine against the CPU oracle.

* bit-exact: per-point histogram slots, and every per-period output against the
  oracle's mirror of the engine arithmetic (oracle.eng_*);
* tolerance: per-period power within 1e-5 relative of the FP64 restatement of
  the reference (oracle.ref_*), the same best period, the same winning window
  wherever the FP64 runner-up trails by more than 1e-5;
* batching: a ragged batch gives bit-identically what single-curve runs give;
* edge cases the reference's inputs can reach.
"""
import numpy as np
import pytest
import torch

import recipes as R
from oracle import oracle as O

pytestmark = pytest.mark.gpu

POWER_RTOL = 1e-5  # relative power error bound against the FP64 oracle
FIELDS = ("power", "depth", "depth_err", "t0", "duration", "window")


def run(engine, t, y, w, periods, durations, cfg):
    from astro_transit_gpu_b200.engine import CurveBatch, split_outputs
    y = np.asarray(y)
    b = CurveBatch.from_arrays([t], [y], periods=periods, durations=durations,
                               flux_dtype=np.float64 if y.dtype == np.float64 else np.float32,
                               weights=None if w is None else [w])
    return split_outputs(b, engine.search(b, cfg))[0]


def cfg_binned(objective="snr", max_bins=None, oversample=10):
    from astro_transit_gpu_b200.engine import SearchConfig
    return SearchConfig("parity", objective=objective, max_bins=max_bins, oversample=oversample)


def cfg_fixed(n_bins):
    from astro_transit_gpu_b200.engine import SearchConfig
    return SearchConfig("fast", n_bins=n_bins)


def assert_bit_exact(gpu, ora, name=""):
    for k in FIELDS:
        a, b = np.asarray(gpu[k]), np.asarray(ora[k])
        assert a.dtype == b.dtype, (name, k)
        bad = np.flatnonzero(a != b)
        assert bad.size == 0, (name, k, bad[:5], a[bad[:5]], b[bad[:5]])


def weighted_unsorted(n=3000, seed=9):
    rng = np.random.default_rng(seed)
    t = np.sort(rng.uniform(100.0, 140.0, n))
    y = R.inject_box(t, 1.0 + rng.normal(0, 1e-3, n), 4.2, 101.0, 0.15, 2e-3)
    dy = 1e-3 * np.exp(rng.normal(0, 0.5, n))
    perm = rng.permutation(n)
    return t[perm], y[perm].astype(np.float32), (1 / dy[perm] ** 2).astype(np.float32)


# ------------------------------------------------------------ bit-exact ---

def test_fold_slots_bit_exact(engine):
    """Per-point bin indices (V42 slots and fixed-bin slots) equal the FP64 fold."""
    t, y, dy = R.sector_curve(n=5000, seed=1)
    w = (1 / dy ** 2).astype(np.float32)
    periods = np.concatenate([R.sector_periods(300), [3.71, 0.5, 13.7, 1.0, 2.0, 4.0]])
    dev = engine.device
    tt = torch.tensor(t, device=dev)
    yy = torch.tensor(y.astype(np.float32), device=dev)
    ww = torch.tensor(w, device=dev)
    pp = torch.tensor(periods, device=dev)
    dd = torch.tensor(R.SECTOR_DURATIONS, device=dev)
    slots = engine.debug_fold(tt, yy, ww, pp, dd, cfg_binned()).cpu().numpy()
    ora = O.eng_binned(t, y.astype(np.float32), w, periods, R.SECTOR_DURATIONS, point_bins=True)
    assert np.array_equal(slots, ora["point_bins"])
    # counts per bin follow from the indices
    for p in (0, 150, 305):
        nb = int(ora["point_bins"][p].max()) + 1
        assert np.array_equal(np.bincount(slots[p], minlength=nb),
                              np.bincount(ora["point_bins"][p], minlength=nb))
    slots = engine.debug_fold(tt, yy, ww, pp, dd, cfg_fixed(200)).cpu().numpy()
    ora = O.eng_fixed(t, y.astype(np.float32), w, periods, R.SECTOR_DURATIONS, n_bins=200,
                      point_bins=True)
    ora_slots = np.where(ora["point_bins"] < 0, 201, ora["point_bins"])
    assert np.array_equal(slots, ora_slots)


def test_fold_slots_bit_exact_precision_sample(engine):
    """1e7 per-point bin indices of a precision-stress curve (200 000 points
    over 13 sectors, t offset > 1300 d) at 50 periods spread over its
    0.5-150 d grid, including the bin-range-pass periods, against the FP64
    fold; then every output of those periods bit-exact."""
    rng = np.random.default_rng(77)
    t, y, dy, _ = R.precision_curve(rng)
    w = (1 / dy.astype(np.float64) ** 2).astype(np.float32)
    periods = R.precision_periods()[::2000]
    durs = R.PRECISION_DURATIONS
    dev = engine.device
    slots = engine.debug_fold(torch.tensor(t, device=dev), torch.tensor(y, device=dev),
                              torch.tensor(w, device=dev), torch.tensor(periods, device=dev),
                              torch.tensor(durs, device=dev), cfg_binned()).cpu().numpy()
    assert slots.size == 50 * 200_000
    ora = O.eng_binned(t, y, w, periods, durs, objective="likelihood", point_bins=True)
    assert np.array_equal(slots, ora["point_bins"])
    g = run(engine, t, y, w, periods, durs, cfg_binned("likelihood"))
    assert_bit_exact(g, ora, "precision sample")


def test_binned_negative_phase_points_join_slot_1(engine):
    """Points whose rounded d*(1/P) reaches an integer that the exact d/P stays
    below get a phase just under 0, and int(ph/bin_dur) = 0 puts them in V42
    slot 1: the fold counts them in a guard entry that joins slot 1."""
    from fractions import Fraction
    n = 3000
    t = np.arange(n) * 0.1
    rng = np.random.default_rng(4)
    y = R.inject_box(t, 1.0 + rng.normal(0, 1e-3, n), 1.1, 0.35, 0.2, 3e-3).astype(np.float32)
    periods = np.array([0.3, 1.1, 0.1 * 7, 1.3, 0.9, 2.3])
    durs = np.array([0.05, 0.1, 0.2])
    d = t - t[0]
    neg = sum(1 for P in periods for k, di in zip(np.floor(d * (1.0 / P)), d)
              if Fraction(float(di)) < Fraction(float(P)) * Fraction(float(k)))
    assert neg > 100  # the case is present
    dev = engine.device
    slots = engine.debug_fold(torch.tensor(t, device=dev), torch.tensor(y, device=dev), None,
                              torch.tensor(periods, device=dev), torch.tensor(durs, device=dev),
                              cfg_binned()).cpu().numpy()
    assert np.array_equal(slots, O.eng_binned(t, y, None, periods, durs, point_bins=True)["point_bins"])
    for objective in ("snr", "likelihood"):
        g = run(engine, t, y, None, periods, durs, cfg_binned(objective))
        assert_bit_exact(g, O.eng_binned(t, y, None, periods, durs, objective=objective), objective)


def test_fold_outside_the_fast_form_range(engine):
    """Time spans so long that |d/P| * P/bin_dur reaches 2^40 (astropy bins)
    or |d/P| reaches 1e15 (fixed bins): the fold takes floor() and the full
    clamp per point, still bit-exact against the oracle."""
    rng = np.random.default_rng(12)
    n = 2000
    dev = engine.device
    for t_span, periods, cfg, ora in (
            (2e10, np.array([0.9, 1.3, 2.0]), cfg_binned(), O.eng_binned),
            (3e15, np.array([1.1, 1.7, 2.9]), cfg_fixed(64), O.eng_fixed)):
        t = np.sort(rng.uniform(0.0, t_span, n))
        y = (1.0 + rng.normal(0, 1e-3, n)).astype(np.float32)
        durs = np.array([0.1, 0.2])
        slots = engine.debug_fold(torch.tensor(t, device=dev), torch.tensor(y, device=dev), None,
                                  torch.tensor(periods, device=dev), torch.tensor(durs, device=dev),
                                  cfg).cpu().numpy()
        kw = {} if ora is O.eng_binned else {"n_bins": 64}
        want = ora(t, y, None, periods, durs, point_bins=True, **kw)["point_bins"]
        if ora is O.eng_fixed:
            want = np.where(want < 0, 65, want)
        assert np.array_equal(slots, want)
        g = run(engine, t, y, None, periods, durs, cfg)
        assert_bit_exact(g, ora(t, y, None, periods, durs, **kw))


@pytest.mark.parametrize("objective", ["snr", "likelihood"])
def test_binned_bit_exact_reference_recipe(engine, objective):
    t, y, dy, periods, durs = R.v42_test_recipe()
    w = (1 / dy ** 2).astype(np.float32)
    g = run(engine, t, y, w, periods, durs, cfg_binned(objective))
    o = O.eng_binned(t, y, w, periods, durs, objective=objective)
    assert_bit_exact(g, o, objective)


def test_binned_bit_exact_sector_float32(engine):
    t, y, dy = R.sector_curve(n=15000, seed=0)
    y32 = y.astype(np.float32)
    w = (1 / dy ** 2).astype(np.float32)
    periods = R.sector_periods(1000)
    g = run(engine, t, y32, w, periods, R.SECTOR_DURATIONS, cfg_binned("likelihood"))
    o = O.eng_binned(t, y32, w, periods, R.SECTOR_DURATIONS, objective="likelihood")
    assert_bit_exact(g, o, "sector")


@pytest.mark.parametrize("n", [1, 7, 9, 4095, 5003])
def test_binned_bit_exact_odd_lengths(engine, n):
    """Curves whose length is not a multiple of the per-thread chunk (padding)."""
    rng = np.random.default_rng(n)
    t = np.sort(rng.uniform(0, 27.4, n)) + 1300.0
    y = (1.0 + rng.normal(0, 1e-3, n)).astype(np.float32)
    periods, durs = np.geomspace(0.5, 13.7, 300), np.array([0.04, 0.08, 0.16])
    for w in (None, np.full(n, 4e5, np.float32), rng.uniform(1e5, 1e6, n).astype(np.float32)):
        g = run(engine, t, y, w, periods, durs, cfg_binned())
        o = O.eng_binned(t, y, w, periods, durs)
        assert_bit_exact(g, o, f"n={n}")
        g = run(engine, t, y, w, periods, durs, cfg_fixed(200))
        o = O.eng_fixed(t, y, w, periods, durs, n_bins=200)
        assert_bit_exact(g, o, f"fixed n={n}")


def test_binned_bit_exact_weighted_unsorted(engine):
    t, y, w = weighted_unsorted()
    periods, durs = np.geomspace(0.7, 15.0, 700), np.array([0.05, 0.1, 0.2, 0.3])
    g = run(engine, t, y, w, periods, durs, cfg_binned())
    o = O.eng_binned(t, y, w, periods, durs)
    assert_bit_exact(g, o, "weighted")


def test_binned_bit_exact_reference_cap(engine):
    t, y, dy = R.sector_curve(n=3000, seed=7)
    w = (1 / dy ** 2).astype(np.float32)
    periods = R.sector_periods(400)
    g = run(engine, t, y, w, periods, R.SECTOR_DURATIONS, cfg_binned(max_bins=2000))
    o = O.eng_binned(t, y, w, periods, R.SECTOR_DURATIONS, max_bins=2000)
    assert_bit_exact(g, o, "cap")


def test_binned_global_histogram_fallback(engine):
    """Periods whose bin count exceeds shared memory are searched in bin-range
    passes through shared memory; results stay bit-exact (here up to ~60k
    bins)."""
    rng = np.random.default_rng(4)
    t = np.sort(rng.uniform(0, 60.0, 4000))
    y = R.inject_box(t, 1.0 + rng.normal(0, 1e-3, t.size), 11.0, 3.0, 0.05, 3e-3)
    w = np.full(t.size, 1e6, np.float32)
    periods = np.array([2.0, 5.0, 11.0, 12.0])
    durs = np.array([0.002, 0.02, 0.05])
    g = run(engine, t, y, w, periods, durs, cfg_binned())
    o = O.eng_binned(t, y, w, periods, durs)
    assert_bit_exact(g, o, "fallback")


@pytest.mark.parametrize("weighted", [False, True])
def test_binned_bin_range_passes_long_windows(engine, weighted):
    """Bin-range passes with long windows (up to 800 bins), a transit near the
    end of the period (the V42 padding bins), a grid mixing periods that fit
    shared memory with ones that do not, and a bin cap that does not bind:
    bit-exact against the oracle."""
    rng = np.random.default_rng(14 + weighted)
    t = np.sort(rng.uniform(0, 356.0, 20000)) + 1500.0
    y = R.inject_box(t, 1.0 + rng.normal(0, 1e-3, t.size), 97.3, 1590.0, 0.3, 2e-3)
    w = (rng.uniform(2e5, 1e6, t.size) if weighted else np.full(t.size, 4e5)).astype(np.float32)
    periods = np.concatenate([np.geomspace(0.7, 13.0, 40), np.geomspace(14.0, 170.0, 30)])
    durs = np.array([0.01, 0.05, 0.2, 0.4, 0.8])  # bin 0.001 d: windows of 10..800 bins
    for mb in (None, 10 ** 6):
        g = run(engine, t, y, w, periods, durs, cfg_binned("likelihood", max_bins=mb))
        o = O.eng_binned(t, y, w, periods, durs, objective="likelihood", max_bins=mb or 0)
        assert_bit_exact(g, o, f"passes w={weighted} mb={mb}")


def test_fixed_global_histogram_fallback(engine):
    """Fixed bins beyond one CTA's shared memory use per-CTA global
    histograms; bit-exact."""
    t, f, _, periods, durs = R.astropy_parity_recipe()
    g = run(engine, t, f, None, periods[::10], durs, cfg_fixed(20000))
    o = O.eng_fixed(t, f, None, periods[::10], durs, n_bins=20000)
    assert_bit_exact(g, o, "fixed-glob")


@pytest.mark.parametrize("n_bins", [200, 500, 1024, 3000])
def test_fixed_bit_exact(engine, n_bins):
    t, f, _, periods, durs = R.astropy_parity_recipe()
    g = run(engine, t, f, None, periods, durs, cfg_fixed(n_bins))
    o = O.eng_fixed(t, f, None, periods, durs, n_bins=n_bins)
    assert_bit_exact(g, o, f"fixed{n_bins}")


def test_fixed_bit_exact_weighted_unsorted(engine):
    t, y, w = weighted_unsorted(n=2000, seed=3)
    periods, durs = np.linspace(1.0, 6.0, 500), np.array([0.05, 0.1, 0.2])
    g = run(engine, t, y, w, periods, durs, cfg_fixed(300))
    o = O.eng_fixed(t, y, w, periods, durs, n_bins=300)
    assert_bit_exact(g, o, "fixed-weighted")


# ------------------------------------------------ tolerance vs FP64 ref ---

def test_power_within_tolerance_of_fp64_reference(engine):
    t, y, dy = R.sector_curve(n=15000, seed=0)
    periods = R.sector_periods(2000)
    w64 = 1 / dy ** 2
    for objective in ("snr", "likelihood"):
        g = run(engine, t, y, w64.astype(np.float32), periods, R.SECTOR_DURATIONS,
                cfg_binned(objective))
        a = O.ref_binned(t, y, w64, periods, R.SECTOR_DURATIONS, objective=objective)
        rel = np.abs(g["power"] - a["power"]) / a["power"]
        assert rel.max() <= POWER_RTOL, rel.max()
        assert np.argmax(g["power"]) == np.argmax(a["power"])
        ok = a["gap"] > 1e-5
        assert np.array_equal(g["window"][ok], a["window"][ok])
        assert np.max(np.abs(g["t0"][ok] - a["t0"][ok])) < 1e-9
        assert np.max(np.abs(g["depth"][ok] - a["depth"][ok]) / np.abs(a["depth"][ok])) < 1e-5
    # the injected transit is the best peak
    assert abs(periods[np.argmax(g["power"])] - 3.71) < 0.01


def test_fast_power_within_tolerance_of_fp64_reference(engine):
    t, f, _, periods, durs = R.astropy_parity_recipe()
    g = run(engine, t, f, None, periods, durs, cfg_fixed(500))
    a = O.ref_fixed(t, f, None, periods, durs, n_bins=500)
    rel = np.abs(g["power"] - a["power"]) / a["power"]
    assert rel.max() <= POWER_RTOL
    assert np.argmax(g["power"]) == np.argmax(a["power"])


# ------------------------------------------------------------- batching ---

def test_ragged_batch_equals_single_curve_runs(engine):
    from astro_transit_gpu_b200.engine import CurveBatch, split_outputs
    rng = np.random.default_rng(21)
    ts, ys, ws, ps, ds = [], [], [], [], []
    for k, n in enumerate([37, 1000, 5003, 12000, 1]):
        t = np.sort(rng.uniform(0, 27.4, n)) + 1300.0 + k
        y = (1.0 + rng.normal(0, 1e-3, n)).astype(np.float32)
        ts.append(t); ys.append(y)
        ws.append(np.full(n, 1e6 * (k + 1), np.float32))
        ps.append(np.geomspace(0.5, 13.7, 100 + 97 * k))
        ds.append(np.array([0.04, 0.08, 0.16])[: 1 + k % 3])
    b = CurveBatch.from_arrays(ts, ys, periods=ps, durations=ds, weights=ws)
    outs = split_outputs(b, engine.search(b, cfg_binned()))
    for k in range(len(ts)):
        single = run(engine, ts[k], ys[k], ws[k], ps[k], ds[k], cfg_binned())
        assert_bit_exact(outs[k], single, f"curve{k}")
        o = O.eng_binned(ts[k], ys[k], ws[k], ps[k], ds[k])
        assert_bit_exact(outs[k], o, f"oracle{k}")
        assert outs[k]["best_index"] == int(np.argmax(single["power"]))


def test_results_are_bit_deterministic(engine):
    t, y, dy = R.sector_curve(n=8000, seed=4)
    w = (1 / dy ** 2).astype(np.float32)
    periods = R.sector_periods(1500)
    a = run(engine, t, y, w, periods, R.SECTOR_DURATIONS, cfg_binned())
    b = run(engine, t, y, w, periods, R.SECTOR_DURATIONS, cfg_binned())
    assert_bit_exact(a, b, "rerun")


# -------------------------------------------------------------- edge cases ---

def test_edge_cases(engine):
    # one point: no window has points both in and out of transit
    g = run(engine, np.array([1.0]), np.array([1.0], np.float32), None, [1.0, 2.0], [0.1],
            cfg_binned())
    assert np.all(g["power"] == 0) and np.all(g["window"] == -1)
    # constant flux: zero depth everywhere, identical to the oracle
    t = np.linspace(0, 10, 500)
    y = np.ones(500, np.float32)
    g = run(engine, t, y, None, np.linspace(1, 3, 50), [0.1, 0.2], cfg_binned())
    o = O.eng_binned(t, y, None, np.linspace(1, 3, 50), [0.1, 0.2])
    assert_bit_exact(g, o, "flat")
    assert np.all(g["power"] == 0)
    # durations longer than some periods, single period, float64 flux
    t, f, _, _, _ = R.recovery_recipe()
    g = run(engine, t, f, None, [0.3], [0.05, 0.25, 0.5], cfg_binned())
    o = O.eng_binned(t, f, None, [0.3], [0.05, 0.25, 0.5])
    assert_bit_exact(g, o, "long-durations")
    # a CTA size the library has no kernel for is an argument error
    from astro_transit_gpu_b200.engine import SearchConfig
    with pytest.raises(ValueError, match="cta_threads"):
        run(engine, t, f, None, [0.3], [0.05], SearchConfig("parity", cta_threads=384))


# -------------------------------------------------------- drop-in API ---

def test_api_synthetic_recovery():
    """tests/test_synthetic_recovery.py: best period within 0.01 of the truth."""
    from astro_transit_gpu_b200 import run_gpu_bls
    t, f, _, periods, durs = R.recovery_recipe()
    res = run_gpu_bls(t, f, periods, durs)
    assert abs(res["best_period"] - 7.432) < 0.01


def test_api_v42_parity_recipe():
    """tests/test_v42_parity.py's assertions, against the FP64 restatement
    (Astropy itself is not available): corr > 0.99999, max |diff| < 1e-4."""
    from astro_transit_gpu_b200 import BoxLeastSquaresGPU
    t, y, dy, periods, durs = R.v42_test_recipe()
    res = BoxLeastSquaresGPU(t, y, dy).power(periods, durs, method="parity", dtype=np.float64,
                                             max_bins=4000)
    a = O.ref_binned(t, y, 1 / dy ** 2, periods, durs, max_bins=4000)
    assert np.corrcoef(a["power"], res.power)[0, 1] > 0.99999
    assert np.max(np.abs(a["power"] - res.power)) < 1e-4
    assert res.power.dtype == np.float64
    assert abs(res.best_period - 3.521) < 0.01
    assert len(res.top_candidates) == 5
    assert res.depth is not None and res.transit_time is not None


def test_api_fast_astropy_recipe():
    """tests/test_astropy_parity.py's best-period and top-1 checks."""
    from astro_transit_gpu_b200 import BoxLeastSquaresGPU
    t, f, _, periods, durs = R.astropy_parity_recipe()
    res = BoxLeastSquaresGPU(t, f).power(periods, durs, n_bins=500, dtype=np.float32)
    assert abs(res.best_period - 3.456) < 0.01
    assert abs(res.top_candidates[0].period - 3.456) < 0.01
    a = O.ref_fixed(t, f, None, periods, durs, n_bins=500)
    assert np.corrcoef(a["power"], res.power)[0, 1] > 0.9999


def test_api_grid_consistency():
    """tests/test_cpu_gpu_grid_consistency.py: best period and depth of the box."""
    from astro_transit_gpu_b200 import run_gpu_bls
    t = np.linspace(0, 10, 5000)
    f = R.inject_box(t, np.ones_like(t), 3.456, 1.2, 0.1, 0.01)
    f += np.random.default_rng(0).normal(0, 1e-4, len(t))
    res = run_gpu_bls(t, f, np.linspace(2.0, 5.0, 500), np.linspace(0.05, 0.15, 3))
    assert abs(res["best_period"] - 3.456) < 0.01
    assert abs(res["best_depth"] - 0.01) < 0.005


def test_api_multi_target_parity():
    from astro_transit_gpu_b200 import run_vbls_exact_parity
    rng = np.random.default_rng(5)
    t = np.linspace(0.0, 20.0, 1200)
    ys = np.stack([R.inject_box(t, 1.0 + rng.normal(0, 1e-3, t.size), 2.0 + k, 0.3 * k, 0.1, 3e-3)
                   for k in range(3)])
    ws = (1.0 / (1e-3 * (1.0 + rng.uniform(size=ys.shape))) ** 2)
    periods, durs = np.linspace(1.5, 5.0, 300), np.array([0.06, 0.1, 0.14])
    r = run_vbls_exact_parity(t, ys, periods, durs, weights_matrix=ws, max_bins=2000)
    for k in range(3):
        o = O.eng_binned(t, ys[k], ws[k].astype(np.float32), periods, durs, max_bins=2000)
        assert np.array_equal(r["power_array"][k], o["power"])
        assert abs(r["best_period"][k] - (2.0 + k)) < 0.02


# --------------------------------------------------------------- graphs ---

def test_batch_session_graph_replay_matches_eager(engine):
    """The captured step (copies + search + copies) gives bit-identical
    outputs to the eager step, and picks up new host data on replay."""
    from astro_transit_gpu_b200.engine import BatchSession, SearchConfig
    t, y, dy, _ = R.uniform_batch(n_curves=6, n=3000, seed=5)
    w = (1 / dy.astype(np.float64) ** 2).astype(np.float32)
    periods, durs = R.sector_periods(400), R.SECTOR_DURATIONS
    pt = np.arange(7, dtype=np.int64) * 3000
    cfg = SearchConfig("parity", objective="likelihood")
    eager = BatchSession(engine, pt, periods, durs, cfg, weighted=True)
    eager.load(t, y, w)
    eager.run()
    torch.cuda.synchronize()
    ref = {k: v.clone() for k, v in eager.host_out.items()}
    graphed = BatchSession(engine, pt, periods, durs, cfg, weighted=True)
    graphed.load(t[::-1], y[::-1], w[::-1])  # different data during capture
    graphed.capture()
    graphed.load(t, y, w)
    graphed.run()
    torch.cuda.synchronize()
    graphed.plan.check()
    for k in ref:
        assert torch.equal(graphed.host_out[k], ref[k]), k
    # new inputs through the same graph
    graphed.load(t[::-1], y[::-1], w[::-1])
    graphed.run()
    torch.cuda.synchronize()
    eager.load(t[::-1], y[::-1], w[::-1])
    eager.run()
    torch.cuda.synchronize()
    for k in ref:
        assert torch.equal(graphed.host_out[k], eager.host_out[k]), k
    # load() straight after run(), with no synchronisation, waits for the
    # step's copies: the step still searches the inputs it was started with
    graphed.load(t, y, w)
    graphed.run()
    graphed.load(t[::-1], y[::-1], w[::-1])
    torch.cuda.synchronize()
    for k in ref:
        assert torch.equal(graphed.host_out[k], ref[k]), k


@pytest.mark.parametrize("graphs", [False, True])
def test_pipelined_session_equals_one_session(engine, graphs):
    """A ragged batch (own period grid per curve) split into runs of curves on
    their own streams gives, bit for bit, one session's outputs."""
    from astro_transit_gpu_b200.engine import BatchSession, PipelinedSession, SearchConfig
    cs = R.mixed_batch(n_curves=7, seed=31, max_points=4000)
    t, y, dy, per = zip(*cs)
    w = [(1 / d.astype(np.float64) ** 2).astype(np.float32) for d in dy]
    pt = np.zeros(8, np.int64)
    np.cumsum([len(a) for a in t], out=pt[1:])
    per = [p[:: max(1, len(p) // 700)] for p in per]
    durs = list(R.MIXED_DURATIONS)
    cfg = SearchConfig("parity", objective="likelihood")
    one = BatchSession(engine, pt, per, durs, cfg)
    one.load(np.concatenate(t), np.concatenate(y), np.concatenate(w))
    one.run()
    torch.cuda.synchronize()
    one.plan.check()
    ps = PipelinedSession(engine, pt, per, durs, cfg, parts=3)
    ps.load(np.concatenate(t), np.concatenate(y), np.concatenate(w))
    if graphs:
        ps.capture()
    outs = ps.run()
    torch.cuda.synchronize()
    ps.check()
    assert ps.bounds == [0, 2, 4, 7]
    for k, v in one.host_out.items():
        assert torch.equal(torch.cat([o[k] for o in outs]), v), k
    ps.close()
    one.close()


# ------------------------------------------------------ winner-take-all ---

@pytest.mark.parametrize("method", ["fast", "parity"])
def test_screen_equals_full_search_at_its_best_period(engine, method):
    """The winner-take-all mode (no per-period output, packed atomicMax per
    curve, then the winner searched again) reports exactly what the full
    search reports at its best period."""
    from astro_transit_gpu_b200.engine import CurveBatch, SearchConfig
    rng = np.random.default_rng(31)
    ts, ys, es, ps = [], [], [], []
    for i in range(7):
        n_sec, cad, n, n_per = R.mixed_curve_spec(rng)
        t, y, dy, per = R.mixed_curve(rng, n_sec, cad, min(n, 8000), min(n_per, 3000))
        ts.append(t); ys.append(1.0 + y); es.append(dy); ps.append(per)
    cfg = (SearchConfig("fast", n_bins=128) if method == "fast" else
           SearchConfig("parity", objective="likelihood"))
    b = CurveBatch.from_arrays(ts, ys, es, periods=ps, durations=R.MIXED_DURATIONS[:6],
                               device=engine.device)
    full = {k: v.cpu().numpy() for k, v in engine.search(b, cfg).items()}
    scr = {k: v.cpu().numpy() for k, v in engine.screen(b, cfg).items()}
    for c in range(b.n_curves):
        bi = int(full["best_period"][c])
        assert int(scr["best_index"][c]) == bi
        g = int(b.out_begin[c]) + bi
        assert scr["period"][c] == ps[c][bi]
        for k in FIELDS:
            assert scr[k][c] == full[k][g], (c, k)


# ------------------------------------------------------------ autotuning ---

def test_tile_size_never_changes_results_and_autotune_picks_one(engine, tmp_path):
    """Every tile size (periods per work-queue tile) gives bit-identical
    outputs; the autotuner times the candidates and later plans of the same
    kind of batch use the winner."""
    from astro_transit_gpu_b200.engine import CurveBatch, SearchConfig
    t, y, dy, _ = R.uniform_batch(n_curves=3, n=3000, seed=17)
    per = [np.geomspace(0.5, 13.7, n) for n in (700, 1500, 333)]
    b = CurveBatch.from_arrays(list(t), list(y), list(dy), periods=per,
                               durations=R.SECTOR_DURATIONS, device=engine.device)
    ref = None
    for tp, nt in ((0, 0), (1, 256), (7, 512), (8, 256), (64, 0)):
        cfg = SearchConfig("parity", objective="likelihood", tile_periods=tp, cta_threads=nt)
        out = {k: v.cpu().numpy() for k, v in engine.search(b, cfg).items()}
        if ref is None:
            ref = out
        for k in ref:
            assert np.array_equal(out[k], ref[k]), (tp, k)
    cfg = SearchConfig("parity", objective="likelihood")
    from astro_transit_gpu_b200.tuning import TuningTable
    saved = engine.tuning
    engine.tuning = TuningTable(str(tmp_path / "tuning.json"), saved.device_name,
                                saved.library)
    try:
        best = engine.autotune(b, cfg, candidates=(8, 64), fold_candidates=(0, 1, -1),
                               shape_candidates=(512, 256))
        assert best["tile_periods"] in (8, 64)
        assert best["merge_run"] in (0, 1, -1)
        assert best["cta_threads"] in (512, 256)
        assert len(engine.last_tune) == 7
        key = engine.tune_key(b, cfg)
        assert engine.tuning.get(key)["tile_periods"] == best["tile_periods"]
        # persisted: a table read back from the file holds the same setting
        again = TuningTable(engine.tuning.path, saved.device_name, saved.library).load()
        assert {k: again.get(key)[k] for k in best} == best
        assert engine.tuned_config(b, cfg).tile_periods == best["tile_periods"]
        # the tuned plan gives what the default plan gave
        out = {k: v.cpu().numpy() for k, v in engine.search(b, cfg).items()}
        for k in ref:
            assert np.array_equal(out[k], ref[k]), k
    finally:
        engine.tuning = saved
