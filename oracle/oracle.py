"""ctypes wrapper of the FP64 CPU oracle (``bls_oracle.c``).

TEST INFRASTRUCTURE ONLY: the oracle the CUDA engine is tested against.  Imported by the
test-suite, by ``__graft_entry__.smoke()`` and by the CPU-baseline leg of
``bench.py``; never by the product package.

Two families (see the header of ``bls_oracle.c``):

* ``ref_binned`` / ``ref_fixed`` -- FP64 restatement of the reference kernels
  (``search/kernels/vbls_v42_parity.cu`` and ``search/kernels/bls.cu`` with
  SCALAR_T=double, host prologues ``search/v42_parity.py:42-67`` and
  ``search/gpu_bls.py:57-78``).
* ``eng_stage`` / ``eng_binned`` / ``eng_fixed`` -- the engine's exact
  arithmetic, which the CUDA engine must reproduce bit for bit.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libbls_oracle.so")
_lib = None
_lock = threading.Lock()

OBJECTIVES = {"fast": 0, "snr": 1, "likelihood": 2}

_dp = ctypes.POINTER(ctypes.c_double)
_fp = ctypes.POINTER(ctypes.c_float)
_ip = ctypes.POINTER(ctypes.c_int32)
_i64 = ctypes.c_int64
_i32 = ctypes.c_int32


class StageStats(ctypes.Structure):
    _fields_ = [
        ("t_start", ctypes.c_double),
        ("shift", ctypes.c_double),
        ("qw_tot", ctypes.c_int64),
        ("qy_tot", ctypes.c_int64),
        ("qy_abs", ctypes.c_int64),
        ("s_w", ctypes.c_int32),
        ("s_y", ctypes.c_int32),
    ]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


def build() -> str:
    """Compile the oracle (and, when the reference checkout exists, its kernels)."""
    subprocess.run(["make", "-s", "-C", _HERE, "all"], check=True)
    return _LIB_PATH


def lib():
    global _lib
    with _lock:
        if _lib is None:
            if not os.path.exists(_LIB_PATH):
                build()
            L = ctypes.CDLL(_LIB_PATH)
            L.orc_ref_binned.argtypes = [_i64, _dp, _dp, _dp, _i64, _dp, _i32, _dp, _i32, _i32,
                                         _i32, _i32, _dp, _dp, _dp, _dp, _dp, _ip, _dp]
            L.orc_ref_fixed.argtypes = [_i64, _dp, _dp, _dp, _i64, _dp, _i32, _dp, _i32, _i32,
                                        _dp, _dp, _dp, _dp, _dp, _ip, _dp]
            L.orc_eng_stage.argtypes = [_i64, _dp, _dp, _fp, _dp, _ip, _ip,
                                        ctypes.POINTER(StageStats)]
            L.orc_eng_binned.argtypes = [_i64, _dp, _ip, _ip, ctypes.POINTER(StageStats), _i64,
                                         _dp, _i32, _dp, _i32, _i32, _i32, _i32, _fp, _fp, _fp,
                                         _dp, _fp, _ip, _ip]
            L.orc_eng_fixed.argtypes = [_i64, _dp, _ip, _ip, ctypes.POINTER(StageStats), _i64,
                                        _dp, _i32, _dp, _i32, _i32, _fp, _fp, _fp, _dp, _fp, _ip,
                                        _ip]
            for fn in ("orc_ref_binned", "orc_ref_fixed", "orc_eng_stage", "orc_eng_binned",
                       "orc_eng_fixed"):
                getattr(L, fn).restype = ctypes.c_int
            _lib = L
    return _lib


def _d(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _ptr(a, typ):
    if a is None:
        return None
    return a.ctypes.data_as(typ)


def _check(rc, what):
    if rc != 0:
        raise ValueError(f"oracle {what} failed with status {rc}")


def _outputs(np_, fdt):
    return {
        "power": np.zeros(np_, fdt), "depth": np.zeros(np_, fdt),
        "depth_err": np.zeros(np_, fdt), "t0": np.zeros(np_, np.float64),
        "duration": np.zeros(np_, fdt), "window": np.zeros(np_, np.int32),
    }


def ref_binned(t, y, w, periods, durations, oversample=10, max_bins=0, objective="snr",
               nthreads=0):
    """FP64 astropy-binned BLS as the V42 kernel computes it (SCALAR_T=double)."""
    t, y, periods, durations = _d(t), _d(y), _d(periods), _d(durations)
    w = None if w is None else _d(w)
    out = _outputs(len(periods), np.float64)
    out["gap"] = np.zeros(len(periods), np.float64)
    rc = lib().orc_ref_binned(len(t), _ptr(t, _dp), _ptr(y, _dp), _ptr(w, _dp), len(periods),
                              _ptr(periods, _dp), len(durations), _ptr(durations, _dp),
                              int(oversample), int(max_bins or 0), OBJECTIVES[objective], int(nthreads),
                              *(_ptr(out[k], _dp) for k in ("power", "depth", "depth_err", "t0",
                                                             "duration")),
                              _ptr(out["window"], _ip), _ptr(out["gap"], _dp))
    _check(rc, "ref_binned")
    return out


def ref_fixed(t, y, w, periods, durations, n_bins=200, nthreads=0):
    """FP64 fixed-bin BLS as bls.cu computes it (SCALAR_T=double), incl. host prologue."""
    t, y, periods, durations = _d(t), _d(y), _d(periods), _d(durations)
    w = None if w is None else _d(w)
    out = _outputs(len(periods), np.float64)
    out["gap"] = np.zeros(len(periods), np.float64)
    rc = lib().orc_ref_fixed(len(t), _ptr(t, _dp), _ptr(y, _dp), _ptr(w, _dp), len(periods),
                             _ptr(periods, _dp), len(durations), _ptr(durations, _dp),
                             int(n_bins), int(nthreads),
                             *(_ptr(out[k], _dp) for k in ("power", "depth", "depth_err", "t0",
                                                            "duration")),
                             _ptr(out["window"], _ip), _ptr(out["gap"], _dp))
    _check(rc, "ref_fixed")
    return out


def eng_stage(t, y, w=None):
    """The engine's deterministic fixed-point staging of one curve.

    ``w`` is the FP32 weight array (None = unit weights); ``y`` is promoted to
    FP64 exactly as the engine promotes it."""
    t, y = _d(t), _d(y)
    w = None if w is None else np.ascontiguousarray(w, dtype=np.float32)
    n = len(t)
    dt = np.zeros(n, np.float64)
    qw = np.zeros(n, np.int32)
    qy = np.zeros(n, np.int32)
    st = StageStats()
    rc = lib().orc_eng_stage(n, _ptr(t, _dp), _ptr(y, _dp), _ptr(w, _fp), _ptr(dt, _dp),
                             _ptr(qw, _ip), _ptr(qy, _ip), ctypes.byref(st))
    _check(rc, "eng_stage")
    return dt, qw, qy, st


def eng_binned(t, y, w, periods, durations, oversample=10, max_bins=0, objective="snr",
               nthreads=0, point_bins=False):
    """The engine's arithmetic for the astropy-binned geometry (bit-exact target)."""
    dt, qw, qy, st = eng_stage(t, y, w)
    periods, durations = _d(periods), _d(durations)
    out = _outputs(len(periods), np.float32)
    pb = np.zeros(len(periods) * len(dt), np.int32) if point_bins else None
    rc = lib().orc_eng_binned(len(dt), _ptr(dt, _dp), _ptr(qw, _ip), _ptr(qy, _ip),
                              ctypes.byref(st), len(periods), _ptr(periods, _dp), len(durations),
                              _ptr(durations, _dp), int(oversample), int(max_bins or 0),
                              OBJECTIVES[objective], int(nthreads),
                              _ptr(out["power"], _fp), _ptr(out["depth"], _fp),
                              _ptr(out["depth_err"], _fp), _ptr(out["t0"], _dp),
                              _ptr(out["duration"], _fp), _ptr(out["window"], _ip),
                              _ptr(pb, _ip))
    _check(rc, "eng_binned")
    out["stats"] = st.as_dict()
    if pb is not None:
        out["point_bins"] = pb.reshape(len(periods), len(dt))
    return out


def eng_fixed(t, y, w, periods, durations, n_bins=200, nthreads=0, point_bins=False):
    """The engine's arithmetic for the fixed-bin geometry (bit-exact target)."""
    dt, qw, qy, st = eng_stage(t, y, w)
    periods, durations = _d(periods), _d(durations)
    out = _outputs(len(periods), np.float32)
    pb = np.zeros(len(periods) * len(dt), np.int32) if point_bins else None
    rc = lib().orc_eng_fixed(len(dt), _ptr(dt, _dp), _ptr(qw, _ip), _ptr(qy, _ip),
                             ctypes.byref(st), len(periods), _ptr(periods, _dp), len(durations),
                             _ptr(durations, _dp), int(n_bins), int(nthreads),
                             _ptr(out["power"], _fp), _ptr(out["depth"], _fp),
                             _ptr(out["depth_err"], _fp), _ptr(out["t0"], _dp),
                             _ptr(out["duration"], _fp), _ptr(out["window"], _ip), _ptr(pb, _ip))
    _check(rc, "eng_fixed")
    out["stats"] = st.as_dict()
    if pb is not None:
        out["point_bins"] = pb.reshape(len(periods), len(dt))
    return out
