"""Host logic of the continuous-batching server: batch formation (arrival
order, configuration grouping, memory budget, batch size)."""
from collections import namedtuple

from astro_transit_gpu_b200.serving import admit, request_bytes

R = namedtuple("R", "name cfg nbytes")


def key(r):
    return r.cfg


def names(rs):
    return [r.name for r in rs]


def test_admit_groups_by_configuration_in_arrival_order():
    pend = [R("a", 1, 10), R("b", 2, 10), R("c", 1, 10), R("d", 1, 10)]
    take, rest, held = admit(pend, key, 0, 1000, 8)
    assert names(take) == ["a", "c", "d"] and names(rest) == ["b"] and held == 30


def test_admit_respects_budget_without_overtaking():
    pend = [R("a", 1, 40), R("b", 1, 50), R("c", 1, 5), R("d", 2, 5)]
    take, rest, held = admit(pend, key, 20, 100, 8)
    # b does not fit (20 + 40 + 50 > 100); c must not overtake it
    assert names(take) == ["a"] and names(rest) == ["b", "c", "d"] and held == 60


def test_admit_respects_batch_size_and_empty_queue():
    pend = [R(str(i), 0, 1) for i in range(5)]
    take, rest, held = admit(pend, key, 0, 100, 2)
    assert names(take) == ["0", "1"] and names(rest) == ["2", "3", "4"] and held == 2
    take, rest, held = admit([], key, 7, 100, 2)
    assert take == [] and len(rest) == 0 and held == 7


def test_admit_waits_when_the_head_does_not_fit():
    take, rest, held = admit([R("big", 0, 90)], key, 20, 100, 8)
    assert take == [] and names(rest) == ["big"] and held == 20


def test_request_bytes_grows_with_the_request():
    assert request_bytes(1000, 100, 4) < request_bytes(2000, 100, 4) < request_bytes(2000, 200, 4)


def test_prune_drops_expired_and_cancelled_requests_in_order():
    from concurrent.futures import Future
    from astro_transit_gpu_b200.serving import prune
    P = namedtuple("P", "name future deadline")
    a, b, c, d = (P("a", Future(), None), P("b", Future(), 5.0), P("c", Future(), 20.0),
                  P("d", Future(), None))
    assert c.future.cancel()
    keep, expired, cancelled = prune([a, b, c, d], now=10.0)
    assert names(keep) == ["a", "d"] and names(expired) == ["b"] and names(cancelled) == ["c"]
    keep, expired, cancelled = prune([a, b, d], now=1.0)
    assert names(keep) == ["a", "b", "d"] and not expired and not cancelled


def test_requests_that_would_fail_a_batch_are_rejected_at_submission():
    """A request with invalid data would make the whole batch it joins fail
    (the engine flags the batch), so submit() rejects it on its own."""
    import numpy as np
    import pytest
    from astro_transit_gpu_b200.serving import check_request
    t = np.linspace(0.0, 27.0, 500)
    y = np.ones(500, np.float32)
    dy = np.full(500, 1e-3)
    per, dur = np.array([1.0, 2.0]), np.array([0.05, 0.1])
    check_request(t, y, dy, per, dur)  # valid
    check_request(t, y, None, per, dur)
    bad_y = y.copy()
    bad_y[7] = np.nan
    bad_dy = dy.copy()
    bad_dy[3] = 0.0
    cases = [
        ((t[:0], y[:0], None, per, dur), "at least one point"),
        ((t, bad_y, dy, per, dur), "NaNs"),
        ((t, y, bad_dy, per, dur), "flux_err"),
        ((t, y, np.full(500, 1e-25), per, dur), "overflows"),
        ((t, y, dy, np.array([1.0, -1.0]), dur), "periods"),
        ((t, y, dy, np.array([]), dur), "periods"),
        ((t, y, dy, per, np.array([0.05, np.inf])), "durations"),
        ((t, y, dy, per, np.linspace(0.01, 0.3, 33)), "durations"),
    ]
    for args, msg in cases:
        with pytest.raises(ValueError, match=msg):
            check_request(*args)
