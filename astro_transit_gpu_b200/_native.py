"""ctypes binding of ``libastrotransit_b200.so`` (C ABI in include/astrotransit_b200.h).

The library is the only compute path: if it is missing or cannot be loaded,
every entry point raises.  There is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os
import threading

from . import build as _build

ATB_OK = 0
ATB_EINVAL = 1
ATB_ENOMEM = 2
ATB_ECUDA = 3
ATB_EINTERNAL = 4
ATB_EDATA = 5

GEOM_FIXED = 0
GEOM_BINNED = 1

OBJ_FAST = 0
OBJ_SNR = 1
OBJ_LIKELIHOOD = 2
OBJECTIVES = {"fast": OBJ_FAST, "snr": OBJ_SNR, "likelihood": OBJ_LIKELIHOOD}

# every symbol the header declares
EXPORTS = (
    "atb_create", "atb_destroy", "atb_last_error", "atb_version",
    "atb_plan_create", "atb_plan_execute", "atb_plan_check", "atb_plan_kernel_count",
    "atb_plan_scratch_bytes", "atb_plan_destroy", "atb_search", "atb_run_gpu_bls",
    "atb_run_vbls_exact_parity", "atb_debug_fold", "atb_plan_profile",
    "atb_bench_smem_red_u64", "atb_bench_smem_red_u32", "atb_bench_dfma", "atb_search_curve_static",
    "atb_plan_curve_layout", "atb_plan_create_async", "atb_plan_top_k",
)

# limit of atb_search_curve_static (ATB_STATIC_MAX_POINTS in the header)
STATIC_MAX_POINTS = 65536

_vp = ctypes.c_void_p
_i32 = ctypes.c_int32
_i64 = ctypes.c_int64
_i64p = ctypes.POINTER(ctypes.c_int64)
_i32p = ctypes.POINTER(ctypes.c_int32)


class Params(ctypes.Structure):
    _fields_ = [("geometry", _i32), ("objective", _i32), ("n_bins", _i32),
                ("oversample", _i32), ("max_bins", _i32), ("tile_periods", _i32),
                ("merge_run", _i32), ("cta_threads", _i32)]


class Batch(ctypes.Structure):
    _fields_ = [("n_curves", _i32), ("y_is_f64", _i32),
                ("point_offset", _i64p), ("time_offset", _i64p),
                ("period_begin", _i64p), ("period_count", _i64p),
                ("dur_begin", _i64p), ("dur_count", _i32p), ("out_begin", _i64p),
                ("t", _vp), ("y", _vp), ("w", _vp), ("periods", _vp), ("durations", _vp)]


class Outputs(ctypes.Structure):
    _fields_ = [("power", _vp), ("depth", _vp), ("depth_err", _vp), ("t0", _vp),
                ("duration", _vp), ("window", _vp), ("best_period", _vp), ("best_key", _vp)]


class NativeError(RuntimeError):
    """A CUDA or internal failure reported by the engine library."""


_lib = None
_lock = threading.Lock()


def lib_path() -> str:
    return _build.LIB


def load(build_if_missing: bool = True):
    """Load (building if needed) the engine library; raises if unavailable."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        path = _build.LIB
        if build_if_missing and _build.needs_build():
            _build.build()
        if not os.path.exists(path):
            raise ImportError(f"engine library not built: {path}")
        L = ctypes.CDLL(path)
        L.atb_create.argtypes = [ctypes.c_int, ctypes.POINTER(_vp)]
        L.atb_destroy.argtypes = [_vp]
        L.atb_destroy.restype = None
        L.atb_last_error.argtypes = [_vp, ctypes.c_char_p, ctypes.c_size_t]
        L.atb_version.restype = ctypes.c_char_p
        L.atb_plan_create.argtypes = [_vp, ctypes.POINTER(Params), ctypes.POINTER(Batch),
                                      ctypes.POINTER(Outputs), ctypes.POINTER(_vp)]
        L.atb_plan_create_async.argtypes = [_vp, ctypes.POINTER(Params), ctypes.POINTER(Batch),
                                            ctypes.POINTER(Outputs), _vp, ctypes.POINTER(_vp)]
        L.atb_plan_execute.argtypes = [_vp, _vp]
        L.atb_plan_top_k.argtypes = [_vp, _i32, _i32, _vp, _vp]
        L.atb_plan_check.argtypes = [_vp]
        L.atb_plan_kernel_count.argtypes = [_vp]
        L.atb_plan_scratch_bytes.argtypes = [_vp]
        L.atb_plan_scratch_bytes.restype = _i64
        L.atb_plan_curve_layout.argtypes = [_vp, _i32p, _i32p]
        L.atb_plan_destroy.argtypes = [_vp]
        L.atb_plan_destroy.restype = None
        L.atb_search.argtypes = [_vp, ctypes.POINTER(Params), ctypes.POINTER(Batch),
                                 ctypes.POINTER(Outputs), _vp]
        L.atb_run_gpu_bls.argtypes = [_vp, _vp, _vp, _vp, _i64, _vp, _i64, _vp, _i32, _i32,
                                      _vp, _vp, _vp, _vp, _i32p, _vp]
        L.atb_run_vbls_exact_parity.argtypes = [_vp, _vp, _vp, _vp, _i64, _i64, _vp, _i64, _vp,
                                                _i32, _i32, _i32, _i32, _vp, _vp, _vp, _vp, _vp,
                                                _vp]
        L.atb_debug_fold.argtypes = [_vp, ctypes.POINTER(Params), _vp, _vp, _vp, _i64, _vp, _i64,
                                     _vp, _i32, _vp, _vp]
        _fp = ctypes.POINTER(ctypes.c_float)
        _dp = ctypes.POINTER(ctypes.c_double)
        L.atb_plan_profile.argtypes = [_vp, _vp, _fp, _fp, _fp]
        L.atb_bench_smem_red_u64.argtypes = [_vp, ctypes.c_int, _dp]
        L.atb_bench_smem_red_u32.argtypes = [_vp, ctypes.c_int, _dp]
        L.atb_bench_dfma.argtypes = [_vp, _dp]
        L.atb_search_curve_static.argtypes = [ctypes.POINTER(Params), _vp, _vp, _i32, _vp, _i64,
                                              _vp, _i64, _vp, _i32, _vp, _vp, _vp, _vp, _vp, _vp,
                                              _vp, _vp, ctypes.c_char_p, ctypes.c_size_t]
        for fn in ("atb_search_curve_static", "atb_plan_profile", "atb_bench_smem_red_u64",
                   "atb_bench_smem_red_u32", "atb_bench_dfma",
                   "atb_create", "atb_last_error", "atb_plan_create", "atb_plan_create_async",
                   "atb_plan_execute", "atb_plan_top_k",
                   "atb_plan_check", "atb_plan_kernel_count", "atb_search", "atb_run_gpu_bls",
                   "atb_run_vbls_exact_parity", "atb_debug_fold"):
            getattr(L, fn).restype = ctypes.c_int
        _lib = L
        return L


def last_error(handle) -> str:
    buf = ctypes.create_string_buffer(1024)
    load().atb_last_error(handle, buf, len(buf))
    return buf.value.decode(errors="replace")


def raise_for(rc: int, handle, what: str) -> None:
    """Map a status code to the reference's exception types (api.py:54-70,
    gpu_bls.py:101-114): invalid input -> ValueError, allocation -> MemoryError."""
    if rc == ATB_OK:
        return
    msg = f"{what}: {last_error(handle) if handle else ''}".rstrip(": ")
    if rc in (ATB_EINVAL, ATB_EDATA):
        raise ValueError(msg)
    if rc == ATB_ENOMEM:
        raise MemoryError(msg)
    raise NativeError(f"{msg} (status {rc})")


class Handle:
    """One engine handle on one CUDA device."""

    def __init__(self, device: int = 0):
        self.lib = load()
        h = _vp()
        rc = self.lib.atb_create(int(device), ctypes.byref(h))
        if rc != ATB_OK:
            raise NativeError(f"atb_create(device={device}) failed with status {rc}")
        self.ptr = h
        self.device = device

    def close(self):
        if self.ptr:
            self.lib.atb_destroy(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
