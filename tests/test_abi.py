"""The C-ABI library builds, loads without a GPU and exports every symbol the
header declares (no compute calls here)."""
import ctypes
import os
import re

from astro_transit_gpu_b200 import _native as N
from astro_transit_gpu_b200 import build as B

HEADER = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include",
                      "astrotransit_b200.h")


def declared_symbols():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"\b(atb_[a-z_0-9]+)\s*\(", text)))


def test_header_and_binding_agree():
    assert declared_symbols() == sorted(N.EXPORTS)


def test_library_loads_and_exports_every_symbol():
    L = N.load()
    for name in declared_symbols():
        assert hasattr(L, name), name
    assert b"sm_100a" in L.atb_version()


def test_library_is_sm100a_only():
    assert "arch=compute_100a,code=sm_100a" in " ".join(B.NVCC_FLAGS)
    assert "-fmad=false" in B.NVCC_FLAGS


def test_null_handles_are_rejected_without_a_device():
    L = N.load()
    assert L.atb_last_error(None, None, 0) == 0
    assert L.atb_plan_create(None, None, None, None, None) == N.ATB_EINVAL
    assert L.atb_plan_execute(None, None) == N.ATB_EINVAL
    assert L.atb_plan_kernel_count(None) == 0


def test_structs_match_header_layout():
    # int32 x8 params; batch: 2 ints + 7 host pointers + 5 device pointers
    assert ctypes.sizeof(N.Params) == 32
    assert ctypes.sizeof(N.Batch) == 8 + 12 * 8
    assert ctypes.sizeof(N.Outputs) == 8 * 8


def test_params_field_offsets():
    # the eight int32 fields of atb_params in header order
    names = ["geometry", "objective", "n_bins", "oversample", "max_bins", "tile_periods",
             "merge_run", "cta_threads"]
    assert [f[0] for f in N.Params._fields_] == names
    assert [getattr(N.Params, f).offset for f in names] == [4 * i for i in range(8)]


def test_static_entry_validates_before_touching_the_device():
    """Argument errors of the no-allocation entry point are found on the host
    (no CUDA call is made): an unsupported CTA size and a bad point count.
    The array arguments are host addresses that are never dereferenced."""
    L = N.load()
    dummy = (ctypes.c_double * 8)()
    p = ctypes.cast(dummy, ctypes.c_void_p)
    err = ctypes.create_string_buffer(256)

    def call(prm, n=8):
        return L.atb_search_curve_static(ctypes.byref(prm), p, p, 0, None, n, p, 2, p, 1, p,
                                         None, None, None, None, None, None, None, err,
                                         len(err))

    prm = N.Params(N.GEOM_FIXED, N.OBJ_FAST, 200, 10, 0, 0, 0, 256)
    assert call(prm) == N.ATB_EINVAL and b"cta_threads" in err.value
    prm = N.Params(N.GEOM_FIXED, N.OBJ_FAST, 200, 10, 0, 0, 0, 0)
    assert call(prm, n=N.STATIC_MAX_POINTS + 1) == N.ATB_EINVAL and b"points" in err.value
