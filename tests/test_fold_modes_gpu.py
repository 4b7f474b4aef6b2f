"""The fold strategies (point by point, or a thread's points added once when
they provably share a slot) are chosen per period from the expected points
per bin; they only change how many shared-memory reductions are issued, and
the CTA size (512 or 256 threads) only how the work is split.  Every
strategy in both CTA sizes, forced
on curves where it does and does not pay (dense and sparse, time-ordered and
not, with gaps longer than the period, ragged lengths that leave warps
partly empty, uniform and non-uniform weights), must give bit-identical
outputs to the oracle's mirror of the engine arithmetic."""
import numpy as np
import pytest

import recipes as R
from oracle import oracle as O

pytestmark = pytest.mark.gpu

FIELDS = ("power", "depth", "depth_err", "t0", "duration", "window")
# merge_run: the default; point by point only; merged wherever possible
MODES = [0, -1, 1]
# (merge_run, cta_threads): each fold mode in both CTA sizes
SETTINGS = [(0, 0), (-1, 0), (1, 0), (0, 256), (1, 256), (-1, 512)]


def _search(engine, t, y, w, periods, durs, cfg):
    from astro_transit_gpu_b200.engine import CurveBatch, split_outputs
    b = CurveBatch.from_arrays([t], [np.asarray(y, np.float32)], periods=periods,
                               durations=durs, weights=None if w is None else [w])
    return split_outputs(b, engine.search(b, cfg))[0]


def dense_curve(n=30001, seed=5):
    """2-minute cadence over 3 sectors: ~1000 points per fixed bin at 5 d."""
    rng = np.random.default_rng(seed)
    t, y, dy, per = R.mixed_curve(rng, 3, R.CADENCE_2MIN, n, 300)
    return t, y, None


def gapped_curve(seed=6):
    """Dense runs separated by gaps longer than the periods searched, so that
    one warp's 128 consecutive points can span several cycles."""
    rng = np.random.default_rng(seed)
    t = np.concatenate([k * 7.3 + np.sort(rng.uniform(0, 0.4, 700)) for k in range(9)]) + 1500.0
    y = R.inject_box(t, 1.0 + rng.normal(0, 1e-3, t.size), 1.9, 1500.2, 0.1, 4e-3)
    return t, y.astype(np.float32), None


def unsorted_weighted(seed=7):
    rng = np.random.default_rng(seed)
    t = np.sort(rng.uniform(0, 40, 12003)) + 2000.0
    y = R.inject_box(t, 1.0 + rng.normal(0, 1e-3, t.size), 3.3, 2000.5, 0.12, 3e-3)
    w = (1.0 / (1e-3 * np.exp(rng.normal(0, 0.3, t.size))) ** 2).astype(np.float32)
    perm = rng.permutation(t.size)
    perm[:6000] = np.arange(6000)  # half the curve keeps its time order
    return t[perm], y[perm].astype(np.float32), w[perm]


CURVES = {"dense": dense_curve, "gapped": gapped_curve, "unsorted_weighted": unsorted_weighted}


@pytest.mark.parametrize("name", sorted(CURVES))
@pytest.mark.parametrize("method", ["fast", "parity"])
def test_every_fold_mode_is_bit_exact(engine, name, method):
    from astro_transit_gpu_b200.engine import SearchConfig
    t, y, w = CURVES[name]()
    span = t.max() - t.min()
    periods = np.geomspace(0.5, min(40.0, 0.45 * span), 240)
    durs = np.array([0.03, 0.06, 0.12, 0.2])
    if method == "fast":
        ora = O.eng_fixed(t, y, w, periods, durs, n_bins=200)
    else:
        ora = O.eng_binned(t, y, w, periods, durs, objective="likelihood")
    for mr, nt in SETTINGS:
        if method == "fast":
            cfg = SearchConfig("fast", n_bins=200, merge_run=mr, cta_threads=nt)
        else:
            cfg = SearchConfig("parity", objective="likelihood", merge_run=mr, cta_threads=nt)
        g = _search(engine, t, y, w, periods, durs, cfg)
        for k in FIELDS:
            bad = np.flatnonzero(g[k] != ora[k])
            assert bad.size == 0, (name, method, mr, nt, k, bad[:5])


def test_fold_modes_in_a_ragged_batch(engine):
    """A batch of dense and sparse curves of ragged lengths: every mode gives
    the default mode's outputs, bit for bit."""
    from astro_transit_gpu_b200.engine import CurveBatch, SearchConfig
    rng = np.random.default_rng(8)
    ts, ys, ps = [], [], []
    for k, (n_sec, cad, n) in enumerate([(2, R.CADENCE_2MIN, 20000), (5, 30 / 1440, 5000),
                                         (1, R.CADENCE_2MIN, 333), (4, R.CADENCE_2MIN, 65537),
                                         (13, 30 / 1440, 1201)]):
        t, y, dy, per = R.mixed_curve(rng, n_sec, cad, n, 150 + 37 * k)
        ts.append(t)
        ys.append(y)
        ps.append(per)
    b = CurveBatch.from_arrays(ts, ys, periods=ps, durations=R.MIXED_DURATIONS[:6])
    ref = None
    for mr, nt in SETTINGS:
        cfg = SearchConfig("fast", n_bins=200, merge_run=mr, cta_threads=nt)
        out = {k: v.cpu().numpy() for k, v in engine.search(b, cfg).items()}
        ref = ref or out
        for k in ref:
            assert np.array_equal(out[k], ref[k]), (mr, nt, k)
