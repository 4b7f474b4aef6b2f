"""The two single-call C entry points a maintainer binds into the reference,
called through ctypes exactly as the reference-side ctypes stubs bind them
(the stubs take CuPy arrays; torch tensors stand in here, the pointers are
the same kind):

* atb_run_gpu_bls            run_gpu_bls + bls_kernel (search/gpu_bls.py:42-144)
* atb_run_vbls_exact_parity  run_vbls_exact_parity + vbls_v42_parity_kernel
                             (search/v42_parity.py:27-107), several targets on
                             one time axis, with and without the reference's
                             default bin cap max_bins=2000

Outputs are compared bit for bit with the oracle's mirror of the engine
arithmetic (oracle.eng_*) and within 1e-5 relative power with the FP64
restatement of the reference (oracle.ref_*).
"""
import ctypes

import numpy as np
import pytest
import torch

import recipes as R
from astro_transit_gpu_b200 import _native as N
from oracle import oracle as O

pytestmark = pytest.mark.gpu

POWER_RTOL = 1e-5  # relative power error bound against the FP64 oracle


def stub_library():
    """The library bound the way the reference-side ctypes stubs bind it."""
    c = ctypes
    lib = c.CDLL(N.lib_path())
    lib.atb_create.argtypes = [c.c_int, c.POINTER(c.c_void_p)]
    lib.atb_run_gpu_bls.argtypes = [c.c_void_p] * 4 + [c.c_int64, c.c_void_p, c.c_int64,
                                                       c.c_void_p, c.c_int32, c.c_int32] + \
        [c.c_void_p] * 4 + [c.POINTER(c.c_int32), c.c_void_p]
    lib.atb_run_vbls_exact_parity.argtypes = [c.c_void_p] * 4 + [c.c_int64, c.c_int64,
                                                                 c.c_void_p, c.c_int64,
                                                                 c.c_void_p] + \
        [c.c_int32] * 4 + [c.c_void_p] * 6
    lib.atb_last_error.argtypes = [c.c_void_p, c.c_char_p, c.c_size_t]
    h = c.c_void_p()
    assert lib.atb_create(0, c.byref(h)) == N.ATB_OK
    return lib, h


@pytest.fixture(scope="module")
def stub():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return stub_library()


def _p(x):
    return 0 if x is None else x.data_ptr()


def _err(lib, h):
    buf = ctypes.create_string_buffer(512)
    lib.atb_last_error(h, buf, len(buf))
    return buf.value.decode()


def call_run_gpu_bls(stub, t, y, dy, periods, durations, n_bins):
    lib, h = stub
    dev = torch.device("cuda", 0)
    tt = torch.tensor(np.asarray(t, np.float64), device=dev)
    yy = torch.tensor(np.asarray(y, np.float32), device=dev)
    ww = None if dy is None else torch.tensor(
        (1.0 / np.asarray(dy, np.float64) ** 2).astype(np.float32), device=dev)
    pp = torch.tensor(np.asarray(periods, np.float64), device=dev)
    dd = torch.tensor(np.asarray(durations, np.float64), device=dev)
    power, dur, depth = (torch.full((pp.numel(),), -7.0, dtype=torch.float32, device=dev)
                         for _ in range(3))
    t0 = torch.full((pp.numel(),), -7.0, dtype=torch.float64, device=dev)
    best = ctypes.c_int32(-7)
    rc = lib.atb_run_gpu_bls(h, _p(tt), _p(yy), _p(ww), tt.numel(), _p(pp), pp.numel(), _p(dd),
                             dd.numel(), n_bins, _p(power), _p(t0), _p(dur), _p(depth),
                             ctypes.byref(best), torch.cuda.current_stream(dev).cuda_stream)
    assert rc == N.ATB_OK, _err(lib, h)
    return {"power": power.cpu().numpy(), "t0": t0.cpu().numpy(),
            "duration": dur.cpu().numpy(), "depth": depth.cpu().numpy()}, best.value


def call_run_vbls(stub, t, ys, ws, periods, durations, oversample, max_bins, objective):
    lib, h = stub
    dev = torch.device("cuda", 0)
    nt, nd = ys.shape
    tt = torch.tensor(np.asarray(t, np.float64), device=dev)
    yy = torch.tensor(np.asarray(ys, np.float32), device=dev)
    ww = None if ws is None else torch.tensor(np.asarray(ws, np.float32), device=dev)
    pp = torch.tensor(np.asarray(periods, np.float64), device=dev)
    dd = torch.tensor(np.asarray(durations, np.float64), device=dev)
    np_ = pp.numel()
    power, dur, depth = (torch.full((nt, np_), -7.0, dtype=torch.float32, device=dev)
                         for _ in range(3))
    t0 = torch.full((nt, np_), -7.0, dtype=torch.float64, device=dev)
    best = torch.full((nt,), -7, dtype=torch.int32, device=dev)
    rc = lib.atb_run_vbls_exact_parity(
        h, _p(tt), _p(yy), _p(ww), nt, nd, _p(pp), np_, _p(dd), dd.numel(), oversample, max_bins,
        N.OBJECTIVES[objective], _p(power), _p(t0), _p(dur), _p(depth), _p(best),
        torch.cuda.current_stream(dev).cuda_stream)
    assert rc == N.ATB_OK, _err(lib, h)
    return ({"power": power.cpu().numpy(), "t0": t0.cpu().numpy(),
             "duration": dur.cpu().numpy(), "depth": depth.cpu().numpy()},
            best.cpu().numpy())


def assert_fields_equal(got, ora, fields, name):
    for k in fields:
        a, b = got[k], ora[k]
        assert a.dtype == b.dtype, (name, k)
        bad = np.flatnonzero(a != b)
        assert bad.size == 0, (name, k, bad[:5], a[bad[:5]], b[bad[:5]])


def test_run_gpu_bls_entry_point_weighted(stub):
    t, y, dy = R.sector_curve(n=6000, seed=31)
    y = y.astype(np.float32)
    periods = R.sector_periods(800)
    got, best = call_run_gpu_bls(stub, t, y, dy, periods, R.SECTOR_DURATIONS, 200)
    w = (1.0 / dy.astype(np.float64) ** 2).astype(np.float32)
    o = O.eng_fixed(t, y, w, periods, R.SECTOR_DURATIONS, n_bins=200)
    assert_fields_equal(got, o, ("power", "t0", "duration", "depth"), "run_gpu_bls")
    a = O.ref_fixed(t, y, 1.0 / dy.astype(np.float64) ** 2, periods, R.SECTOR_DURATIONS, n_bins=200)
    rel = np.abs(got["power"] - a["power"]) / a["power"]
    assert rel.max() <= POWER_RTOL, rel.max()
    # the best index is the first maximum (gpu_bls.py:131, cupy.argmax)
    assert best == int(np.argmax(got["power"]))
    assert best == int(np.argmax(a["power"]))
    assert abs(periods[best] - 3.71) < 0.02


def test_run_gpu_bls_entry_point_unit_weights(stub):
    t, f, _, periods, durs = R.astropy_parity_recipe()
    got, best = call_run_gpu_bls(stub, t, f.astype(np.float32), None, periods, durs, 500)
    o = O.eng_fixed(t, f.astype(np.float32), None, periods, durs, n_bins=500)
    assert_fields_equal(got, o, ("power", "t0", "duration", "depth"), "run_gpu_bls unit")
    assert best == int(np.argmax(got["power"]))
    assert abs(periods[best] - 3.456) < 0.01


@pytest.mark.parametrize("objective", ["snr", "likelihood"])
@pytest.mark.parametrize("max_bins", [2000, 0])
def test_run_vbls_exact_parity_entry_point_multi_target(stub, max_bins, objective):
    """Four targets on one time axis; the grid reaches 13.7 d, where 0.004 d
    bins exceed the reference's default cap of 1999 bins (max_bins=2000)."""
    rng = np.random.default_rng(41)
    t = R.sector_times(rng, 4000)
    truth = [2.3, 3.71, 5.2, 9.1]
    ys = np.stack([R.inject_box(t, 1.0 + rng.normal(0, 1e-3, t.size), P, t[0] + 0.3 * k,
                                0.12, 2.5e-3) for k, P in enumerate(truth)]).astype(np.float32)
    ws = (1.0 / (1e-3 * (1.0 + 0.5 * rng.uniform(size=ys.shape))) ** 2).astype(np.float32)
    periods = R.sector_periods(700)
    got, best = call_run_vbls(stub, t, ys, ws, periods, R.SECTOR_DURATIONS, 10, max_bins, objective)
    for k in range(len(truth)):
        gk = {f: v[k] for f, v in got.items()}
        o = O.eng_binned(t, ys[k], ws[k], periods, R.SECTOR_DURATIONS, max_bins=max_bins,
                         objective=objective)
        assert_fields_equal(gk, o, ("power", "t0", "duration", "depth"), f"target {k}")
        a = O.ref_binned(t, ys[k], ws[k].astype(np.float64), periods, R.SECTOR_DURATIONS,
                         max_bins=max_bins, objective=objective)
        ok = a["power"] > 0
        rel = np.abs(gk["power"][ok] - a["power"][ok]) / a["power"][ok]
        assert rel.max() <= POWER_RTOL, (k, rel.max())
        assert np.all(gk["power"][~ok] == 0)
        assert best[k] == int(np.argmax(gk["power"]))
        if max_bins == 0 or truth[k] < 7.9:  # the cap distorts periods above 7.96 d
            assert abs(periods[best[k]] - truth[k]) < 0.02 * truth[k], (k, periods[best[k]])


def test_entry_points_map_invalid_input_to_status_codes(stub):
    lib, h = stub
    dev = torch.device("cuda", 0)
    t = torch.linspace(0, 10, 100, dtype=torch.float64, device=dev)
    y = torch.ones(100, dtype=torch.float32, device=dev)
    p = torch.tensor([1.0, 2.0], dtype=torch.float64, device=dev)
    d = torch.tensor([0.1], dtype=torch.float64, device=dev)
    out = torch.empty(2, dtype=torch.float32, device=dev)
    s = torch.cuda.current_stream(dev).cuda_stream
    # n_bins < 2 (gpu_bls.py:101-102 rejects out-of-range bin counts with ValueError)
    rc = lib.atb_run_gpu_bls(h, _p(t), _p(y), 0, 100, _p(p), 2, _p(d), 1, 1, _p(out), 0, 0, 0,
                             None, s)
    assert rc == N.ATB_EINVAL
    # a NaN flux value is found by the staging kernel: invalid data, not a crash
    y[5] = float("nan")
    rc = lib.atb_run_gpu_bls(h, _p(t), _p(y), 0, 100, _p(p), 2, _p(d), 1, 200, _p(out), 0, 0, 0,
                             None, s)
    assert rc == N.ATB_EDATA and "non-finite" in _err(lib, h)
    # the handle stays usable
    y[5] = 1.0
    rc = lib.atb_run_gpu_bls(h, _p(t), _p(y), 0, 100, _p(p), 2, _p(d), 1, 200, _p(out), 0, 0, 0,
                             None, s)
    assert rc == N.ATB_OK
