"""Host-side behaviour of the drop-in API that needs no GPU: input validation
mirrors search/api.py:51-70, top-k selection mirrors gpu_bls.py:146-174, and
the compute path refuses to run without CUDA (no CPU fallback)."""
import numpy as np
import pytest
import torch

from astro_transit_gpu_b200 import BoxLeastSquaresGPU, get_top_k_candidates
from astro_transit_gpu_b200.engine import CurveBatch, SearchConfig, is_shared_grid


def _curve(n=100):
    t = np.linspace(0, 10, n)
    return t, np.ones(n), np.full(n, 1e-3)


@pytest.mark.parametrize("periods,durations,msg", [
    ([-1.0, 2.0], [0.1], "periods must be positive"),
    ([0.0], [0.1], "periods must be positive"),
    ([1.0], [-0.1], "durations must be positive"),
])
def test_grid_validation(periods, durations, msg):
    t, y, dy = _curve()
    with pytest.raises(ValueError, match=msg):
        BoxLeastSquaresGPU(t, y, dy).power(periods, durations)


def test_nan_and_dy_validation():
    t, y, dy = _curve()
    y2 = y.copy(); y2[3] = np.nan
    with pytest.raises(ValueError, match="NaN"):
        BoxLeastSquaresGPU(t, y2, dy).power([1.0], [0.1])
    dy2 = dy.copy(); dy2[0] = 0.0
    with pytest.raises(ValueError, match="strictly positive"):
        BoxLeastSquaresGPU(t, y, dy2).power([1.0], [0.1])
    with pytest.raises(ValueError, match="same length"):
        BoxLeastSquaresGPU(t, y, dy[:-1]).power([1.0], [0.1])
    with pytest.raises(ValueError, match="method"):
        BoxLeastSquaresGPU(t, y, dy).power([1.0], [0.1], method="nope")


def test_search_config_params():
    p = SearchConfig("parity").params()
    assert (p.geometry, p.objective, p.oversample, p.max_bins) == (1, 1, 10, 0)
    p = SearchConfig("parity", objective="likelihood", max_bins=2000).params()
    assert (p.objective, p.max_bins) == (2, 2000)
    p = SearchConfig("fast", n_bins=500).params()
    assert (p.geometry, p.objective, p.n_bins) == (0, 0, 500)
    with pytest.raises(ValueError):
        SearchConfig("fast", objective="snr").params()


def test_shared_grid_detection():
    assert is_shared_grid(np.linspace(1, 2, 5))
    assert is_shared_grid([1.0, 2.0])
    assert not is_shared_grid([np.linspace(1, 2, 5), np.linspace(1, 3, 7)])
    assert not is_shared_grid(np.ones((2, 3)))


def test_top_k_candidates_follow_find_peaks():
    from scipy.signal import find_peaks
    rng = np.random.default_rng(0)
    power = rng.random(400)
    res = {"power": power, "all_t0s": np.arange(400.0), "all_durs": np.ones(400),
           "all_depths": np.zeros(400), "periods": np.linspace(1, 5, 400)}
    top = get_top_k_candidates(res, k=5)
    peaks, _ = find_peaks(power, distance=10)
    want = peaks[np.argsort(power[peaks])[::-1][:5]]
    assert [c["t0"] for c in top] == [float(i) for i in want]
    flat = dict(res, power=np.arange(10.0))  # monotone: no interior peak
    assert [c["t0"] for c in get_top_k_candidates(flat, k=3)] == [9.0, 8.0, 7.0]


@pytest.mark.skipif(torch.cuda.is_available(), reason="checks the no-GPU behaviour")
def test_no_cpu_fallback_without_cuda():
    t, y, dy = _curve()
    with pytest.raises((RuntimeError, AssertionError)):
        BoxLeastSquaresGPU(t, y, dy).power([1.0, 2.0], [0.1], method="parity")
    with pytest.raises((RuntimeError, AssertionError)):
        CurveBatch.from_arrays([t], [y], periods=[1.0], durations=[0.1])


def test_top_peak_indices_matches_find_peaks_without_ties():
    """On spectra without exact ties the host top-k equals scipy's
    find_peaks(distance) followed by the reference's sort."""
    from scipy.signal import find_peaks
    from astro_transit_gpu_b200.gpu_bls import top_peak_indices
    rng = np.random.default_rng(5)
    for n, k, dist in ((500, 5, 10), (2000, 8, 3), (50, 5, 1), (3, 5, 10)):
        x = rng.permutation(n).astype(np.float64) + rng.uniform(0, 0.5, n)
        x = np.convolve(x, np.ones(3) / 3, mode="same")
        peaks, _ = find_peaks(x, distance=dist)
        if len(peaks) == 0:
            ref = list(np.argsort(x)[-k:][::-1])
        else:
            ref = list(peaks[np.argsort(x[peaks])[::-1][:k]])
        assert top_peak_indices(x, k, dist) == [int(i) for i in ref]
    # equal powers: the higher index first
    assert top_peak_indices(np.array([0, 2, 0, 2, 0.0]), 2, 1) == [3, 1]


@pytest.mark.parametrize("periods, durations, msg", [
    ([1.0, float("nan")], [0.1], "periods must be positive and finite"),
    ([1.0, -2.0], [0.1], "periods must be positive and finite"),
    ([1.0], [0.1, 0.0], "durations must be positive and finite"),
    ([1.0], [float("inf")], "durations must be positive and finite"),
    ([1.0], [], "durations must be positive|1 to 32 durations"),
    ([1.0], list(np.linspace(0.01, 0.3, 33)), "1 to 32 durations"),
])
def test_curve_batch_rejects_invalid_grids_before_device_work(periods, durations, msg):
    """Invalid grids are rejected on the host, before any copy or launch (the
    kernels also flag them, as ATB_EDATA)."""
    t, y, dy = _curve()
    with pytest.raises(ValueError, match=msg):
        CurveBatch.from_arrays([t], [y], periods=periods, durations=durations)
