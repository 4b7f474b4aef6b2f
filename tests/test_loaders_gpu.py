"""GPU tests: a sector-cache batch (shared time axis, padding dropped) and the
batched injection/recovery grid give the same results as one search per
curve, and those results are the oracle's (its mirror of the engine
arithmetic), bit for bit."""
import numpy as np
import pytest

import recipes as R
from oracle import oracle as O

pytestmark = pytest.mark.gpu

FIELDS = ("power", "depth", "depth_err", "t0", "duration", "window")


def test_sector_cache_batch_equals_per_target_searches(engine, tmp_path):
    from astro_transit_gpu_b200.engine import CurveBatch, SearchConfig, split_outputs
    from astro_transit_gpu_b200.sector_cache import load_sector_cache
    rng = np.random.default_rng(2)
    L = 1312
    t = (1325.0 + np.arange(L) * (30.0 / 1440)).astype(np.float32)
    lens = [1312, 1200, 900, 1311]
    flux = np.zeros((4, L), np.float32)
    err = np.ones((4, L), np.float32)
    for i, n in enumerate(lens):
        f = rng.normal(0, 1e-3, n)
        if i == 1:
            f = R.inject_box(t[:n].astype(np.float64), 1.0 + f, 3.3, 1326.0, 0.15, 4e-3) - 1.0
        flux[i, :n] = f
        err[i, :n] = 1e-3 * (1 + i)
    np.savez(tmp_path / "data.npz", time=t, flux=flux, flux_err=err,
             tic_ids=np.arange(4) + 5, is_vectorized=True)
    sc = load_sector_cache(str(tmp_path))
    assert sc.shared_time is not None
    periods, durs = np.geomspace(0.5, 13.0, 700), np.array([0.05, 0.1, 0.2])
    for cfg in (SearchConfig("fast", n_bins=200), SearchConfig("parity", objective="snr")):
        b = sc.batch(periods, durs, device=engine.device)
        got = split_outputs(b, engine.search(b, cfg))
        for i in range(4):
            ref_b = CurveBatch.from_arrays([sc.times[i]], [sc.fluxes[i]], [sc.flux_errs[i]],
                                           periods=periods, durations=durs, device=engine.device)
            ref = split_outputs(ref_b, engine.search(ref_b, cfg))[0]
            w = (1.0 / (np.asarray(sc.flux_errs[i], np.float64) ** 2)).astype(np.float32)
            y = np.asarray(sc.fluxes[i], np.float32)
            ora = (O.eng_fixed(sc.times[i], y, w, periods, durs, n_bins=200)
                   if cfg.method == "fast" else
                   O.eng_binned(sc.times[i], y, w, periods, durs, objective="snr"))
            for k in FIELDS:
                assert np.array_equal(got[i][k], ref[k]), (cfg.method, i, k)
                assert np.array_equal(got[i][k], ora[k]), (cfg.method, i, k, "oracle")
    # the injected transit is found
    b = sc.batch(periods, durs, device=engine.device)
    o = split_outputs(b, engine.search(b, SearchConfig("fast", n_bins=200)))[1]
    assert abs(periods[o["best_index"]] - 3.3) < 0.05


def test_injection_recovery_batch_equals_one_search_per_trial(engine):
    from astro_transit_gpu_b200.gpu_bls import run_gpu_bls
    from astro_transit_gpu_b200.inject import (calculate_recovery_map, inject_box_transit,
                                               match_candidate,
                                               run_injection_recovery_experiment)
    rng0 = np.random.default_rng(12)
    t = R.sector_times(rng0, 4000)
    y = (1.0 + rng0.normal(0.0, 1e-3, t.size)).astype(np.float32)  # normalised flux near 1
    periods = np.linspace(0.5, 12.0, 1500)
    df = run_injection_recovery_experiment(t, y, [2.5, 6.1], [3e-3, 1e-2], n_trials=3,
                                           search_periods=periods,
                                           rng=np.random.default_rng(5))
    assert len(df) == 12
    rng = np.random.default_rng(5)
    durs = np.linspace(0.01, 0.2, 5)
    for p in (2.5, 6.1):
        for d in (3e-3, 1e-2):
            for trial in range(3):
                t0 = t[0] + rng.random() * p
                yi = inject_box_transit(t, y, p, t0, 0.1, d)
                res = run_gpu_bls(t, yi, periods, durs)
                if trial == 0:
                    ora = O.eng_fixed(t, np.asarray(yi), None, periods, durs, n_bins=200)
                    assert np.array_equal(res["power"], ora["power"]), (p, d)
                    assert np.array_equal(res["all_t0s"], ora["t0"]), (p, d)
                row = df[(df.injected_period == p) & (df.injected_depth == d)
                         & (df.trial == trial)].iloc[0]
                assert row.detected_period == res["best_period"]
                assert row.detected_t0 == res["best_t0"]
                assert row.is_recovered == match_candidate(res["best_period"], res["best_t0"],
                                                           p, t0)["is_match"]
    rec = calculate_recovery_map(df)
    assert rec.loc[2.5, 1e-2] == 1.0  # deep short-period transits are always recovered
