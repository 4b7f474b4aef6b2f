"""Host tests of the sector-cache reader and the injection/matching helpers
(no GPU): formats, padding removal, the shared time axis, the reference's
injection and matching rules."""
import numpy as np
import pytest

from astro_transit_gpu_b200.inject import inject_box_transit, match_candidate
from astro_transit_gpu_b200.sector_cache import FLUX_ERR_PAD_SENTINEL, load_sector_cache


def _write_vectorized(path, lens, L=64, seed=0, interior_flag=False):
    rng = np.random.default_rng(seed)
    t = (1325.0 + np.arange(L) * (2.0 / 1440)).astype(np.float32)
    flux = np.zeros((len(lens), L), np.float32)
    err = np.full((len(lens), L), FLUX_ERR_PAD_SENTINEL, np.float32)
    for i, n in enumerate(lens):
        flux[i, :n] = rng.normal(0, 1e-3, n)
        err[i, :n] = 1e-3
    if interior_flag:
        err[0, 3] = 0.95  # a real point above the threshold: masked, not a prefix
    np.savez(path, time=t, flux=flux, flux_err=err, tic_ids=np.arange(len(lens)) + 100,
             is_vectorized=True)
    return t, flux, err


def test_vectorized_cache_drops_padding_and_shares_time(tmp_path):
    lens = [64, 50, 17]
    t, flux, err = _write_vectorized(tmp_path / "data.npz", lens)
    sc = load_sector_cache(str(tmp_path))
    assert list(sc.tic_ids) == [100, 101, 102]
    assert [len(x) for x in sc.times] == lens
    assert sc.shared_time is not None and np.array_equal(sc.shared_time, t.astype(np.float64))
    for i, n in enumerate(lens):
        assert np.array_equal(sc.fluxes[i], flux[i, :n])
        assert np.array_equal(sc.times[i], t[:n].astype(np.float64))
    tgt = sc.target(101)
    assert len(tgt["time"]) == 50 and sc.target(999) is None


def test_vectorized_cache_with_interior_mask_has_no_shared_axis(tmp_path):
    _write_vectorized(tmp_path / "c.npz", [40, 30], interior_flag=True)
    sc = load_sector_cache(str(tmp_path / "c.npz"))
    assert sc.shared_time is None
    assert len(sc.times[0]) == 39


def test_flat_cache(tmp_path):
    rng = np.random.default_rng(1)
    lens = [5, 9, 3]
    t = np.concatenate([np.sort(rng.uniform(0, 10, n)) for n in lens])
    f = rng.normal(0, 1, t.size)
    e = np.full(t.size, 0.01)
    offs = np.concatenate([[0], np.cumsum(lens)])
    np.savez(tmp_path / "f.npz", time=t, flux=f, flux_err=e, tic_ids=np.array([7, 8, 9]),
             offsets=offs, is_vectorized=False)
    sc = load_sector_cache(str(tmp_path / "f.npz"))
    assert [len(x) for x in sc.times] == lens
    assert np.array_equal(sc.times[1], t[5:14])
    # offsets without the final end, as the reference also accepts
    np.savez(tmp_path / "g.npz", time=t, flux=f, flux_err=e, tic_ids=np.array([7, 8, 9]),
             offsets=offs[:-1], is_vectorized=False)
    sc2 = load_sector_cache(str(tmp_path / "g.npz"))
    assert [len(x) for x in sc2.times] == lens


def test_inject_box_transit_matches_the_rule():
    t = np.linspace(0, 10, 1001)
    f = np.ones_like(t)
    g = inject_box_transit(t, f, 2.0, 0.5, 0.2, 0.01)
    phase = (t - 0.5 + 1.0) % 2.0 - 1.0
    inside = np.abs(phase) < 0.1
    assert np.allclose(g[inside], 0.99) and np.all(g[~inside] == 1.0)
    assert np.all(f == 1.0)  # input untouched


@pytest.mark.parametrize("p_det,t0_det,expect", [
    (3.0, 1.0, "direct"), (6.0, 4.0, "harmonic"), (1.5, 1.0, "subharmonic"),
    (9.0, 7.0, "harmonic_3"), (1.0, 1.0, "subharmonic_3"), (3.2, 1.0, "none"),
    (3.0, 1.5, "none")])
def test_match_candidate(p_det, t0_det, expect):
    m = match_candidate(p_det, t0_det, 3.0, 1.0)
    assert m["match_type"] == expect and m["is_match"] == (expect != "none")
    assert match_candidate(3.0, 1.5, 3.0, 1.0, require_t0=False)["is_match"]
    assert not match_candidate(0.0, 1.0, 3.0, 1.0)["is_match"]
