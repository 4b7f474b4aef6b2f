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
