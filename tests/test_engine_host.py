"""Host-side logic of the engine module that needs no GPU."""
import pytest

from astro_transit_gpu_b200.engine import PipelinedSession


@pytest.mark.parametrize("n_curves,parts", [(1, 8), (7, 3), (8, 8), (9, 8), (4096, 8), (5, 1)])
def test_pipelined_run_bounds_cover_every_curve_once(n_curves, parts):
    b = PipelinedSession.run_bounds(n_curves, parts)
    assert b[0] == 0 and b[-1] == n_curves
    assert len(b) == min(parts, n_curves) + 1
    sizes = [hi - lo for lo, hi in zip(b[:-1], b[1:])]
    assert min(sizes) >= 1 and max(sizes) - min(sizes) <= 1


def test_pipelined_run_bounds_reject_an_empty_batch():
    with pytest.raises(ValueError):
        PipelinedSession.run_bounds(0, 4)
