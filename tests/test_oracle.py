"""CPU tests of the FP64 oracle: pinned against the reference's own code and
golden vectors, known-answer tests, and the engine-mirror arithmetic."""
import math
import os

import numpy as np
import pytest

import recipes as R
from oracle import oracle as O

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def _rel(a, b, floor=1e-300):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b) / np.maximum(np.abs(b), floor)


# ---------------------------------------------------------------- pinning ---

def test_fixed_oracle_matches_reference_cpu_emulator():
    """Oracle (fixed-bin geometry) vs the reference's own CPU restatement
    tests/debug_emu.py:4-64, recorded in emu_golden.npz by make_emu_golden.py.
    debug_emu folds raw time with n_bins = ceil(oversample*P/min_dur) and
    returns sqrt(max s^2/(W_in(1-r))) = sqrt(max fast score / W_total)."""
    g = np.load(os.path.join(GOLDEN, "emu_golden.npz"))
    durations = g["durations"]
    for case in ("unit", "weighted"):
        t, y, dy, ref = g[case + "_t"], g[case + "_y"], g[case + "_dy"], g[case + "_power"]
        w = 1.0 / dy ** 2
        assert t[0] == 0.0  # debug_emu folds t itself; the oracle folds t - t[0]
        for p, r in zip(g["periods"], ref):
            nb = int(math.ceil(int(g["oversample"]) * p / durations.min()))
            o = O.ref_fixed(t, y, w, [p], durations, n_bins=nb)
            mine = math.sqrt(o["power"][0] ** 2 / w.sum())
            assert abs(mine - r) <= 1e-12 * r, (case, p, mine, r)


def _ref_golden():
    path = os.path.join(GOLDEN, "ref_golden.npz")
    if not os.path.exists(path):
        pytest.skip("ref_golden.npz not generated yet (tests/golden/make_ref_golden.py)")
    return np.load(path)


def _cases(g, prefix):
    return sorted({k.split("__")[0] for k in g.files if k.startswith(prefix)})


def _near_tie_mask(gap, tol):
    return np.asarray(gap) > tol


def test_binned_oracle_matches_reference_kernel_fp64():
    """Oracle vs vbls_v42_parity_kernel (SCALAR_T=double) run on a B200."""
    g = _ref_golden()
    cases = _cases(g, "v42_")
    assert cases
    for name in cases:
        f = lambda k: g[f"{name}__{k}"]
        y = f("y")
        w = f("w")
        ys = y if y.ndim == 2 else y[None]
        ws = w if w.ndim == 2 else w[None]
        for row in range(ys.shape[0]):
            o = O.ref_binned(f("t"), ys[row], ws[row], f("periods"), f("durations"),
                             oversample=10, max_bins=int(f("max_bins")), objective="snr")
            ref = {k: (f(k) if f(k).ndim == 1 else f(k)[row]) for k in
                   ("power", "t0", "duration", "depth")}
            ok = _near_tie_mask(o["gap"], 1e-9)
            rp = _rel(o["power"], ref["power"], 1e-12)
            assert rp.max() <= 1e-9, (name, row, rp.max())
            # the winning window (duration, transit time, depth) where it is not a near-tie
            assert np.array_equal(o["duration"][ok], ref["duration"][ok]), name
            assert np.max(np.abs(o["t0"][ok] - ref["t0"][ok])) <= 1e-9, name
            assert np.max(_rel(o["depth"][ok], ref["depth"][ok], 1e-12)) <= 1e-9, name


def test_fixed_oracle_matches_reference_kernel_fp64():
    """Oracle vs bls_kernel (SCALAR_T=double, N_TILE per the reference's smem
    halving) run on a B200, with the host prologue of gpu_bls.py."""
    g = _ref_golden()
    for name in _cases(g, "bls_"):
        f = lambda k: g[f"{name}__{k}"]
        dy = g[f"{name}__dy"] if f"{name}__dy" in g.files else None
        w = None if dy is None else 1.0 / (dy * dy)
        o = O.ref_fixed(f("t"), f("y"), w, f("periods"), f("durations"), n_bins=int(f("n_bins")))
        ok = _near_tie_mask(o["gap"], 1e-9)
        rp = _rel(o["power"], f("power"), 1e-12)
        assert rp.max() <= 1e-9, (name, rp.max())
        assert np.array_equal(o["duration"][ok], f("duration")[ok]), name
        assert np.max(np.abs(o["t0"][ok] - f("t0")[ok])) <= 1e-9, name
        assert np.max(_rel(o["depth"][ok], f("depth")[ok], 1e-12)) <= 1e-8, name


# ------------------------------------------------------- known answers ---

def _exact_box_curve(n_cycles=10, depth=0.01):
    """Binary-exact samples: t = k * 2^-7, P = 2 (256 samples per cycle), a
    16-sample transit starting at phase sample 32."""
    k = np.arange(256 * n_cycles)
    t = k * 2.0 ** -7
    y = np.ones_like(t)
    j = k % 256
    y[(j >= 32) & (j < 48)] = 1.0 - depth
    return t, y


def test_known_answer_noiseless_box_binned():
    t, y = _exact_box_curve()
    dur = 16 * 2.0 ** -7
    o = O.ref_binned(t, y, None, [2.0], [dur, 2 * dur], oversample=16, objective="snr")
    w_in, w = 16 * 10, t.size
    w_out = w - w_in
    depth = 0.01
    assert o["depth"][0] == pytest.approx(depth, rel=1e-12)
    assert o["duration"][0] == dur
    assert o["t0"][0] == pytest.approx(40 * 2.0 ** -7, abs=1e-12)
    snr = depth / math.sqrt(1.0 / w_in + 1.0 / w_out)
    assert o["power"][0] == pytest.approx(snr, rel=1e-12)
    ll = O.ref_binned(t, y, None, [2.0], [dur, 2 * dur], oversample=16, objective="likelihood")
    assert ll["power"][0] == pytest.approx(0.5 * depth ** 2 * w_in * w_out / w, rel=1e-12)
    e = O.eng_binned(t, y, None, [2.0], [dur, 2 * dur], oversample=16, objective="snr")
    assert e["window"][0] == o["window"][0]
    assert e["power"][0] == pytest.approx(snr, rel=1e-7)
    assert e["depth"][0] == pytest.approx(depth, rel=1e-7)


def test_known_answer_noiseless_box_fixed():
    t, y = _exact_box_curve()
    # 256 bins per period: each sample its own bin; a 16-bin window is the transit
    dur = 16 * 2.0 ** -7
    o = O.ref_fixed(t, y, None, [2.0], [dur], n_bins=256)
    w_in, w = 160, t.size
    depth = 0.01
    assert o["depth"][0] == pytest.approx(depth, rel=1e-12)
    # fast score = W * snr^2
    assert o["power"][0] == pytest.approx(math.sqrt(depth ** 2 * w_in * (w - w_in)), rel=1e-12)
    assert o["t0"][0] == pytest.approx(32 * 2.0 ** -7, abs=1e-12)  # box start (bls.cu:134)
    e = O.eng_fixed(t, y, None, [2.0], [dur], n_bins=256)
    assert e["window"][0] == o["window"][0]
    assert e["power"][0] == pytest.approx(o["power"][0], rel=1e-7)


def test_likelihood_is_half_snr_squared():
    t, y, dy, periods, durs = R.v42_test_recipe()
    w = 1 / dy ** 2
    s = O.ref_binned(t, y, w, periods, durs, objective="snr")
    ll = O.ref_binned(t, y, w, periods, durs, objective="likelihood")
    ok = s["gap"] > 1e-9
    assert np.allclose(ll["power"][ok], 0.5 * s["power"][ok] ** 2, rtol=1e-10)


def test_injection_recovered_by_oracle():
    t, f, _, periods, durs = R.recovery_recipe()
    o = O.ref_fixed(t, f, None, periods, durs, n_bins=200)
    assert abs(periods[np.argmax(o["power"])] - 7.432) < 0.01


# --------------------------------------------------- engine arithmetic ---

@pytest.mark.parametrize("recipe", ["v42_test", "sector", "weighted"])
@pytest.mark.parametrize("objective", ["snr", "likelihood"])
def test_engine_mirror_close_to_fp64_binned(recipe, objective):
    """The engine's arithmetic (fixed-point sums, FP32 search, FP64 winner) stays
    within 1e-6 relative power of the FP64 restatement and picks the same window
    wherever the FP64 runner-up is more than 1e-5 behind."""
    if recipe == "v42_test":
        t, y, dy, periods, durs = R.v42_test_recipe()
    elif recipe == "sector":
        t, y, dy = R.sector_curve(n=4000, seed=3)
        periods, durs = R.sector_periods(600), R.SECTOR_DURATIONS
    else:
        rng = np.random.default_rng(9)
        t = np.sort(rng.uniform(100.0, 140.0, 3000))
        y = R.inject_box(t, 1.0 + rng.normal(0, 1e-3, t.size), 4.2, 101.0, 0.15, 2e-3)
        dy = 1e-3 * np.exp(rng.normal(0, 0.5, t.size))
        periods, durs = np.geomspace(0.7, 15.0, 500), np.array([0.05, 0.1, 0.2, 0.3])
    w = (1.0 / dy ** 2).astype(np.float32)
    a = O.ref_binned(t, y, w.astype(np.float64), periods, durs, objective=objective)
    b = O.eng_binned(t, y, w, periods, durs, objective=objective)
    assert _rel(b["power"], a["power"], 1e-12).max() <= 1e-6
    ok = a["gap"] > 1e-5
    assert np.array_equal(a["window"][ok], b["window"][ok])
    assert np.max(np.abs(a["t0"][ok] - b["t0"][ok])) <= 1e-9


def test_engine_mirror_close_to_fp64_fixed():
    t, f, _, periods, durs = R.astropy_parity_recipe()
    a = O.ref_fixed(t, f, None, periods, durs, n_bins=500)
    b = O.eng_fixed(t, f, None, periods, durs, n_bins=500)
    assert _rel(b["power"], a["power"], 1e-12).max() <= 1e-6
    ok = a["gap"] > 1e-5
    assert np.array_equal(a["window"][ok], b["window"][ok])


def test_engine_stage_is_order_independent():
    """The fixed-point staging (shift, scales, totals) does not depend on point order."""
    t, y, dy = R.sector_curve(n=2000, seed=5)
    w = (1 / dy ** 2).astype(np.float32)
    perm = np.random.default_rng(0).permutation(t.size)
    _, qw, qy, st = O.eng_stage(t, y, w)
    _, qw2, qy2, st2 = O.eng_stage(t[perm], y[perm], w[perm])
    s1, s2 = st.as_dict(), st2.as_dict()
    s1.pop("t_start"); s2.pop("t_start")
    assert s1 == s2
    assert np.array_equal(np.sort(qy), np.sort(qy2))
    assert np.abs(qw).max() <= 2 ** 27 and np.abs(qy).max() <= 2 ** 27


def test_cap_reproduces_reference_pileup():
    """max_bins caps n_bins at max_bins-1 and clamps indices (vbls_v42_parity.cu:46-47,70)."""
    t, y, dy = R.sector_curve(n=1500, seed=2)
    periods = np.array([5.0, 9.0, 12.0])
    o = O.eng_binned(t, y, (1 / dy ** 2).astype(np.float32), periods, R.SECTOR_DURATIONS,
                     max_bins=2000, point_bins=True)
    pb = o["point_bins"]
    assert pb[0].max() <= 1260  # ceil(5/0.004) = 1250 real bins, uncapped
    assert pb[1].max() == 1999 and pb[2].max() == 1999
    assert (pb[2] == 1999).sum() > (pb[1] == 1999).sum()  # more pile-up at longer period


def test_binned_slots_match_exact_restatement_at_cycle_edges():
    """The oracle's per-point V42 slot, min(int(ph * inv_bin) + 1, n_bins)
    with ph = fma(-P, floor(d * (1/P)), d) (vbls_v42_parity.cu:65-70), against
    an independent restatement: the fma rounded once from its exact rational
    value.  Times on a 0.1 d grid put many points where d*(1/P) rounds onto
    an integer the exact d/P stays below, so ph is just under 0 and int()
    gives 0 (slot 1)."""
    from fractions import Fraction
    n = 1500
    t = np.arange(n) * 0.1
    y = np.ones(n, np.float32)
    periods = np.array([0.3, 1.1, 0.1 * 7, 0.9])
    durs = np.array([0.05, 0.1])
    pb = O.eng_binned(t, y, None, periods, durs, point_bins=True)["point_bins"]
    d = t - t[0]
    ibd = 1.0 / (0.05 / 10)
    negative = 0
    for p, P in enumerate(periods):
        nb = math.ceil(P * ibd) + 10
        ks = np.floor(d * (1.0 / P))
        for i in range(n):
            exact = Fraction(float(d[i])) - Fraction(float(P)) * Fraction(float(ks[i]))
            ph = float(exact)  # round to nearest, as one fma does
            negative += ph < 0.0
            slot = min(int(ph * ibd) + 1, nb)
            assert pb[p, i] == slot, (P, i, ph)
    assert negative > 50


def test_oracle_rejects_bad_arguments():
    t = np.linspace(0, 1, 10)
    with pytest.raises(ValueError):
        O.ref_binned(t, t, None, [1.0], [0.1], oversample=0)
    with pytest.raises(ValueError):
        O.ref_binned(t, t, None, [1.0], [0.1], max_bins=5, oversample=10)
    with pytest.raises(ValueError):
        O.ref_fixed(t, t, None, [1.0], [0.1], n_bins=1)
    with pytest.raises(ValueError):
        O.eng_stage(t, t, np.zeros(10, np.float32))


@pytest.mark.parametrize("geometry", ["binned", "fixed"])
def test_engine_mirror_windows_longer_than_any_period_are_skipped(geometry):
    """A duration whose window is longer than every period's bin count (here
    1e12 d, far beyond 2^31 bins, where the engine clamps window lengths to
    2^28 bins) never wins: the outputs equal the search without it, with the
    same window keys since it is the last duration."""
    t, y, dy = R.sector_curve(n=3000, seed=5)
    w = (1.0 / dy ** 2).astype(np.float32)
    periods = R.sector_periods(200)
    durs = [0.05, 0.1]
    run = (lambda d: O.eng_binned(t, y.astype(np.float32), w, periods, d, objective="snr")) \
        if geometry == "binned" else \
        (lambda d: O.eng_fixed(t, y.astype(np.float32), w, periods, d, n_bins=200))
    a, b = run(durs), run(durs + [1e12])
    for k in ("power", "depth", "depth_err", "t0", "duration"):
        assert np.array_equal(a[k], b[k]), k
    # window keys are start * n_durations + duration index
    ok = a["window"] >= 0
    assert np.array_equal(a["window"][ok] // 2 * 3 + a["window"][ok] % 2, b["window"][ok])
