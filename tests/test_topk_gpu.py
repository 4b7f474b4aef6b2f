"""Device top-k peaks against the host find_peaks(power, distance) + sort of
the reference (gpu_bls.get_top_k_candidates), on search outputs and on
synthetic spectra with plateaus and edge cases; power_batch (device peaks)
against one BoxLeastSquaresGPU.power call per curve (host peaks)."""
import numpy as np
import pytest
import torch

import recipes as R

pytestmark = pytest.mark.gpu


def host_topk(power, k, distance):
    from astro_transit_gpu_b200.gpu_bls import top_peak_indices
    return top_peak_indices(power, k, distance)


def _plan(engine, n_curves, n_periods):
    from astro_transit_gpu_b200.engine import CurveBatch, SearchConfig
    t, y, dy, _ = R.uniform_batch(n_curves=n_curves, n=2000, seed=8)
    per = [np.geomspace(0.5, 10.0, n) for n in n_periods]
    b = CurveBatch.from_arrays(list(t), list(y), list(dy), periods=per,
                               durations=R.SECTOR_DURATIONS, device=engine.device)
    plan = engine.plan(b, SearchConfig("fast", n_bins=200))
    plan.execute()
    torch.cuda.synchronize()
    return plan


def test_topk_matches_find_peaks_on_search_outputs(engine):
    plan = _plan(engine, 6, [3000, 1200, 2500, 800, 3000, 50])
    try:
        for k, dist in ((5, 10), (8, 3), (1, 1)):
            got = plan.top_k(k, dist).cpu().numpy()
            pw = plan.outputs["power"].cpu().numpy()
            for c in range(plan.batch.n_curves):
                b, n = int(plan.batch.out_begin[c]), int(plan.batch.period_count[c])
                ref = host_topk(pw[b:b + n], k, dist)
                assert [int(i) for i in got[c] if i >= 0] == ref, (c, k, dist)
    finally:
        plan.close()


def test_topk_synthetic_spectra_plateaus_and_fallback(engine):
    rng = np.random.default_rng(3)
    lens = [1000, 500, 2, 40, 300, 700]
    plan = _plan(engine, len(lens), lens)
    try:
        spectra = []
        for c, n in enumerate(lens):
            x = rng.permutation(n).astype(np.float32)  # distinct values
            if c == 1:  # flat-topped peaks of several widths
                for a, w in ((50, 2), (120, 5), (300, 4), (400, 3)):
                    x[a:a + w] = n + a
            if c == 3:  # monotone: no peak, the fallback returns the largest values
                x = np.arange(n, dtype=np.float32)
            if c == 4:  # a plateau that touches the end is not a peak
                x[-6:] = n + 10
            spectra.append(x)
        pw = plan.outputs["power"]
        for c, x in enumerate(spectra):
            b = int(plan.batch.out_begin[c])
            pw[b:b + len(x)] = torch.from_numpy(x).to(pw.device)
        got = plan.top_k(5, 10).cpu().numpy()
        for c, x in enumerate(spectra):
            assert [int(i) for i in got[c] if i >= 0] == host_topk(x, 5, 10), c
    finally:
        plan.close()


def test_power_batch_equals_single_calls_with_device_peaks(engine):
    from astro_transit_gpu_b200.api import BoxLeastSquaresGPU, power_batch
    rng = np.random.default_rng(21)
    curves = []
    for i in range(4):
        n_sec, cad, n, n_per = R.mixed_curve_spec(rng)
        t, y, dy, per = R.mixed_curve(rng, n_sec, cad, min(n, 5000), min(n_per, 2000))
        curves.append((t, 1.0 + y, dy, per))
    durs = R.MIXED_DURATIONS[:5]
    for method in ("fast", "parity"):
        batch = power_batch([c[0] for c in curves], [c[1] for c in curves],
                            [c[2] for c in curves], periods=[c[3] for c in curves],
                            durations=durs, method=method)
        for (t, y, dy, per), rb in zip(curves, batch):
            r1 = BoxLeastSquaresGPU(t, y, dy).power(per, durs, method=method)
            assert np.array_equal(rb.power, r1.power)
            assert rb.best_period == r1.best_period and rb.best_t0 == r1.best_t0
            assert rb.top_candidates == r1.top_candidates
