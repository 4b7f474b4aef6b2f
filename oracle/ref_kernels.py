"""Launcher for the reference's own CUDA kernels, compiled from source into
``oracle/_ref/*.cubin`` by ``oracle/Makefile``.

TEST INFRASTRUCTURE ONLY: used to write golden vectors (tests/golden/
make_ref_golden.py) and to time the reference's plain one-call-per-curve GPU
path.  The host logic below restates the reference's CuPy host wrappers
(launch geometry, shared-memory sizing, prologue arithmetic) so that the
kernels see exactly the arguments the reference passes:

* ``run_gpu_bls``            search/gpu_bls.py:42-144
* ``run_vbls_exact_parity``  search/v42_parity.py:27-107
* ``run_vbls_massive``       search/vbls.py:62-188 (the batched screening
                             kernel, built for 1312 points, 128 bins, 8
                             durations, float)

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
        v39 = os.path.join(REF_DIR, "v39_f32_n1312_b128_d8.cubin")
        if os.path.exists(v39):
            with open(v39, "rb") as f:
                mod = _check(cu.cuModuleLoadData(f.read()))
            self.mods["v39"] = mod
            self.funcs["v39"] = _check(cu.cuModuleGetFunction(mod, b"vbls_v39_weighted_kernel"))
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

    def run_vbls_massive(self, time_array, flux_matrix, periods, durations, weights_matrix=None,
                         target_batch_size=4000, period_batch_size=20000, sync=True):
        """search/vbls.py:62-188 with the Blackwell kernel (float, 128 bins,
        1312 points, 8 durations): per-target best power (SNR), t0, duration,
        depth and period, as torch tensors on the device."""
        if "v39" not in self.funcs:
            raise FileNotFoundError("oracle/_ref/v39_f32_n1312_b128_d8.cubin missing")
        dev = self.device

        def on_dev(x):
            x = x if isinstance(x, torch.Tensor) else torch.as_tensor(np.asarray(x))
            return x.to(dev).to(torch.float32).contiguous()

        fm = on_dev(flux_matrix)
        n_t, n_data = fm.shape
        if n_data != 1312 or len(durations) != 8:
            raise ValueError("the compiled screening kernel takes 1312 points and 8 durations")
        tg = torch.as_tensor(np.asarray(time_array), device=dev).to(torch.float32)
        t_start = float(tg[0].item())
        dt = (tg - t_start).to(torch.float32).contiguous()
        wm = torch.ones_like(fm) if weights_matrix is None else on_dev(weights_matrix)
        durs = np.asarray(durations, np.float32)
        res = cu.cuModuleGetGlobal(self.mods["v39"], b"c_durations")
        _check(res[0])
        _check(cu.cuMemcpyHtoD(res[1], durs.ctypes.data, durs.nbytes))
        outs = [torch.zeros(n_t, dtype=torch.float32, device=dev) for _ in range(5)]
        per = np.asarray(periods, np.float32)
        smem = 3 * n_data * 4 + 2 * 16 * (128 + 1) * 4
        for p0 in range(0, len(per), period_batch_size):
            pb = per[p0:p0 + period_batch_size]
            pairs = torch.as_tensor(np.stack([pb, (1.0 / pb).astype(np.float32)], 1),
                                    device=dev).contiguous()
            for t0 in range(0, n_t, target_batch_size):
                t1 = min(t0 + target_batch_size, n_t)
                self._launch("v39", ((len(pb) + 15) // 16, t1 - t0), 512, smem, [
                    ("p", fm[t0].data_ptr()), ("p", dt.data_ptr()), ("p", pairs.data_ptr()),
                    ("p", wm[t0].data_ptr())] +
                    [("p", o[t0].data_ptr()) for o in (outs[0], outs[1], outs[2], outs[3],
                                                       outs[4])] +
                    [("i", len(pb)), ("f", t_start)])
        if sync:
            torch.cuda.synchronize(dev)
        return {"snr": outs[0], "best_t0": outs[1], "best_duration": outs[2],
                "best_depth": outs[3], "best_period": outs[4]}
