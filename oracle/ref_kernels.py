"""Launcher for the reference's own CUDA kernels, compiled from source into
``oracle/_ref/*.cubin`` by ``oracle/Makefile``.

TEST INFRASTRUCTURE ONLY: used to write golden vectors (tests/golden/
make_ref_golden.py) and to time the reference's plain one-call-per-curve GPU
path.  The host logic below restates the reference's CuPy host wrappers
(launch geometry, shared-memory sizing, prologue arithmetic) so that the
kernels see exactly the arguments the reference passes:

* ``run_gpu_bls``            search/gpu_bls.py:42-144
* ``run_vbls_exact_parity``  search/v42_parity.py:27-107

Device memory is managed with PyTorch, kernels are loaded and launched with
the CUDA driver API (cuda-python).  The elementwise prologue and the totals
run as PyTorch ops instead of CuPy ops (same IEEE operations; reduction order
may differ in the last bit).
"""
from __future__ import annotations

import ctypes
import os

import numpy as np
import torch
from cuda.bindings import driver as cu

_HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(_HERE, "_ref")


def _check(res):
    err = res[0] if isinstance(res, tuple) else res
    if err != cu.CUresult.CUDA_SUCCESS:
        raise RuntimeError(f"CUDA driver error {err}")
    return res[1] if isinstance(res, tuple) and len(res) == 2 else res


class RefKernels:
    """The reference kernels bls_kernel (N_TILE 1/2/4, float/double) and
    vbls_v42_parity_kernel (float/double), loaded into the current context."""

    def __init__(self, device=None):
        torch.cuda.init()
        self.device = torch.device("cuda", torch.cuda.current_device() if device is None else device)
        torch.zeros(1, device=self.device)  # make the primary context current
        self.mods = {}
        self.funcs = {}
        for name, fn in [(f"bls_f{b}_t{t}", "bls_kernel") for b in (32, 64) for t in (1, 2, 4)] + \
                        [("v42_f32", "vbls_v42_parity_kernel"), ("v42_f64", "vbls_v42_parity_kernel")]:
            path = os.path.join(REF_DIR, name + ".cubin")
            if not os.path.exists(path):
                raise FileNotFoundError(f"{path} missing: run `make -C oracle ref` where the "
                                        "reference checkout exists")
            with open(path, "rb") as f:
                data = f.read()
            mod = _check(cu.cuModuleLoadData(data))
            self.mods[name] = mod
            self.funcs[name] = _check(cu.cuModuleGetFunction(mod, fn.encode()))
        dev = _check(cu.cuCtxGetDevice())
        self.max_shm = _check(cu.cuDeviceGetAttribute(
            cu.CUdevice_attribute.CU_DEVICE_ATTRIBUTE_MAX_SHARED_MEMORY_PER_BLOCK, dev))

    def _launch(self, name, grid, block, smem, args):
        holders = []
        for kind, v in args:
            if kind == "p":
                holders.append(ctypes.c_void_p(int(v)))
            elif kind == "i":
                holders.append(ctypes.c_int(int(v)))
            elif kind == "f":
                holders.append(ctypes.c_float(float(v)))
            elif kind == "d":
                holders.append(ctypes.c_double(float(v)))
            else:
                raise ValueError(kind)
        arr = (ctypes.c_void_p * len(holders))(*[ctypes.addressof(h) for h in holders])
        f = self.funcs[name]
        if smem > 48 * 1024:
            _check(cu.cuFuncSetAttribute(
                f, cu.CUfunction_attribute.CU_FUNC_ATTRIBUTE_MAX_DYNAMIC_SHARED_SIZE_BYTES,
                int(smem)))
        stream = torch.cuda.current_stream(self.device).cuda_stream
        _check(cu.cuLaunchKernel(f, grid[0], grid[1], 1, block, 1, 1, int(smem),
                                 cu.CUstream(stream), ctypes.addressof(arr), 0))

    def run_gpu_bls(self, time, flux, periods, durations, flux_err=None, n_bins=200,
                    dtype=np.float64):
        """search/gpu_bls.py:42-144 (fast path), returning numpy arrays."""
        tdt = torch.float64 if np.dtype(dtype) == np.float64 else torch.float32
        bits = 64 if tdt == torch.float64 else 32
        dev = self.device
        time_g = torch.as_tensor(np.asarray(time), device=dev).to(tdt)
        flux_g = torch.as_tensor(np.asarray(flux), device=dev).to(tdt).clone()
        if flux_err is not None:
            err = torch.as_tensor(np.asarray(flux_err), device=dev).to(tdt)
            w = 1.0 / (err * err)
        else:
            w = torch.ones_like(flux_g)
        w_sum = torch.sum(w)
        w_mean = torch.sum(flux_g * w) / w_sum
        flux_g -= w_mean
        periods_np = np.asarray(periods)
        inv_p = torch.as_tensor(1.0 / periods_np, device=dev).to(tdt)
        durs = torch.as_tensor(np.asarray(durations), device=dev).to(tdt)
        n_data, n_periods, n_dur = len(time_g), len(inv_p), len(durs)
        out = [torch.zeros(n_periods, dtype=tdt, device=dev) for _ in range(4)]
        n_tile = 4
        tpb = 1
        while tpb < n_bins or tpb < 128:
            tpb *= 2
        if tpb > 1024:
            raise ValueError(f"n_bins={n_bins} is too large (max 1024)")
        item = 8 if bits == 64 else 4
        smem = (n_tile * n_bins * 2 + tpb * 4) * item
        while n_tile > 1 and smem > self.max_shm:
            n_tile //= 2
            smem = (n_tile * n_bins * 2 + tpb * 4) * item
        if smem > self.max_shm:
            raise MemoryError("shared memory limit exceeded")
        blocks = (n_periods + n_tile - 1) // n_tile
        t_start = float(time_g[0]) if n_data > 0 else 0.0
        sc = "d" if bits == 64 else "f"
        self._launch(f"bls_f{bits}_t{n_tile}", (blocks, 1), tpb, smem, [
            ("p", time_g.data_ptr()), ("p", flux_g.data_ptr()), ("p", w.data_ptr()),
            ("i", n_data), ("p", inv_p.data_ptr()), ("i", n_periods), ("p", durs.data_ptr()),
            ("i", n_dur), ("i", n_bins), (sc, t_start)] + [("p", o.data_ptr()) for o in out])
        power, t0, dur, depth = (o.cpu().numpy() for o in out)
        b = int(np.argmax(power))
        return {"power": power, "t0": t0, "duration": dur, "depth": depth, "best_index": b,
                "best_period": float(periods_np[b])}

    def run_vbls_exact_parity(self, time_array, flux_matrix, periods, durations,
                              weights_matrix=None, oversample=10, max_bins=2000,
                              dtype=np.float64):
        """search/v42_parity.py:27-107 (parity path), returning numpy arrays."""
        tdt = torch.float64 if np.dtype(dtype) == np.float64 else torch.float32
        bits = 64 if tdt == torch.float64 else 32
        npdt = np.float64 if bits == 64 else np.float32
        dev = self.device
        flux_matrix = np.asarray(flux_matrix)
        n_targets, n_data = flux_matrix.shape
        n_periods, n_dur = len(periods), len(durations)
        t_start = npdt(np.asarray(time_array)[0])
        fm = torch.as_tensor(flux_matrix, device=dev).to(tdt).contiguous()
        tg = torch.as_tensor(np.asarray(time_array), device=dev).to(tdt)
        dt = (tg - float(t_start)).to(tdt)
        if weights_matrix is None:
            wm = torch.ones((n_targets, n_data), dtype=tdt, device=dev)
        else:
            wm = torch.as_tensor(np.asarray(weights_matrix), device=dev).to(tdt).contiguous()
        pg = torch.as_tensor(np.asarray(periods), device=dev).to(tdt)
        dg = torch.as_tensor(np.asarray(durations), device=dev).to(tdt)
        outs = [torch.zeros(n_targets * n_periods, dtype=tdt, device=dev) for _ in range(4)]
        sum_y = torch.sum(fm * wm, dim=1).to(tdt).contiguous()
        sum_w = torch.sum(wm, dim=1).to(tdt).contiguous()
        item = 8 if bits == 64 else 4
        smem = (max_bins + 150) * item * 2
        sc = "d" if bits == 64 else "f"
        self._launch(f"v42_f{bits}", (n_periods, n_targets), 256, smem, [
            ("p", fm.data_ptr()), ("p", dt.data_ptr()), ("p", pg.data_ptr()), ("p", dg.data_ptr()),
            ("p", wm.data_ptr())] + [("p", o.data_ptr()) for o in outs] + [
            ("i", n_data), ("i", n_dur), ("i", oversample), ("i", max_bins),
            (sc, float(t_start)), ("p", sum_y.data_ptr()), ("p", sum_w.data_ptr()),
            ("i", n_targets)])
        power, t0, dur, dep = (o.reshape(n_targets, n_periods).cpu().numpy() for o in outs)
        return {"power": power, "t0": t0, "duration": dur, "depth": dep,
                "best_index": np.argmax(power, axis=1)}
