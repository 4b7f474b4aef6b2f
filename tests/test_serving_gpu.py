"""GPU tests of the continuous-batching server: every request's result is
bit-identical alone and in a mix (different sizes, grids and methods arriving
together), and latency statistics are reported."""
import numpy as np
import pytest

import recipes as R

pytestmark = pytest.mark.gpu

FIELDS = ("power", "depth", "depth_err", "t0", "duration", "window")


def _requests(n=12, seed=4):
    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(n):
        n_sec, cad, npts, nper = R.mixed_curve_spec(rng)
        t, y, dy, per = R.mixed_curve(rng, n_sec, cad, min(npts, 6000), min(nper, 1500))
        method = "fast" if i % 3 == 0 else "parity"
        durs = R.MIXED_DURATIONS[: 4 + i % 5]
        reqs.append(dict(t=t, y=y, dy=dy, periods=per, durations=durs, method=method,
                         objective=None if method == "fast" else "likelihood"))
    return reqs


def _alone(engine, r):
    from astro_transit_gpu_b200.engine import CurveBatch, SearchConfig, split_outputs
    cfg = (SearchConfig("fast", n_bins=200) if r["method"] == "fast" else
           SearchConfig("parity", objective=r["objective"]))
    b = CurveBatch.from_arrays([r["t"]], [r["y"]], [r["dy"]], periods=r["periods"],
                               durations=r["durations"])
    return split_outputs(b, engine.search(b, cfg))[0]


def test_results_identical_alone_and_in_the_mix(engine):
    from astro_transit_gpu_b200.serving import BLSServer
    reqs = _requests()
    with BLSServer(max_batch=64, n_streams=2) as srv:
        futs = [srv.submit(**r) for r in reqs]
        got = [f.result(timeout=300) for f in futs]
        st = srv.stats()
    for r, g in zip(reqs, got):
        ref = _alone(engine, r)
        for k in FIELDS:
            assert np.array_equal(g[k], ref[k]), k
        assert g["best_index"] == ref["best_index"]
    assert st["completed"] == len(reqs)
    assert 0 < st["p50_ms"] <= st["p99_ms"]
    assert st["batches"] >= 2  # two configurations never share a batch


def test_budget_forces_small_batches_and_results_still_match(engine):
    from astro_transit_gpu_b200.serving import BLSServer, request_bytes
    reqs = _requests(n=6, seed=9)
    biggest = max(request_bytes(len(r["t"]), len(r["periods"]), len(r["durations"]))
                  for r in reqs)
    with BLSServer(memory_budget=biggest, max_batch=64, n_streams=3) as srv:
        got = [f.result(timeout=300) for f in [srv.submit(**r) for r in reqs]]
    st = srv.stats()
    assert st["max_held_bytes"] <= biggest and st["completed"] == len(reqs)
    assert st["batches"] >= 3  # the budget split the six requests
    for r, g in zip(reqs, got):
        ref = _alone(engine, r)
        for k in FIELDS:
            assert np.array_equal(g[k], ref[k]), k


def test_timeout_and_cancellation_before_admission(engine):
    """One stream and one request per batch: while a large request runs, a
    request with a tiny timeout expires in the queue (TimeoutError) and a
    cancelled one never runs; a later request without a timeout completes
    with the same result as alone."""
    import concurrent.futures as cf
    from astro_transit_gpu_b200.serving import BLSServer
    rng = np.random.default_rng(17)
    big_t, big_y, big_dy, big_p = R.mixed_curve(rng, 13, R.CADENCE_2MIN, 150000, 40000)
    small = _requests(n=2, seed=23)
    with BLSServer(max_batch=1, n_streams=1) as srv:
        f_big = srv.submit(big_t, big_y, big_dy, periods=big_p, durations=R.MIXED_DURATIONS)
        f_exp = srv.submit(**small[0], timeout=1e-6)
        f_can = srv.submit(**small[0])
        cancelled = f_can.cancel()
        f_ok = srv.submit(**small[1])
        f_big.result(timeout=300)
        with pytest.raises(cf.TimeoutError):
            f_exp.result(timeout=300)
        got = f_ok.result(timeout=300)
        st = srv.stats()
    assert cancelled and f_can.cancelled()
    assert st["expired"] == 1 and st["cancelled"] == 1 and st["completed"] == 2
    ref = _alone(engine, small[1])
    for k in FIELDS:
        assert np.array_equal(got[k], ref[k]), k
