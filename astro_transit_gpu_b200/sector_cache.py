"""Reader of the reference's consolidated sector cache (``data.npz``), feeding
the engine a ragged batch without the cache's padding.

The cache (data/sector_cache.py:96-210 in the reference) comes in two forms:

* vectorized (``is_vectorized``): one common float32 time axis [L], flux and
  flux_err matrices [targets, L] padded at the end with flux 0 and flux_err
  1.0 (the sentinel, constants.py:13-14); a target's points are those with
  flux_err below 0.9 (FLUX_ERR_PAD_THRESHOLD, sector_cache.py:189-196);
* flat: concatenated time/flux/flux_err with ``offsets`` [targets(+1)]
  (sector_cache.py:198-208).

``SectorCurves.batch`` packs the kept points of every target into one
``CurveBatch``.  For the vectorized form, when each target's kept points are a
prefix of the common axis (the builder pads at the end), every curve reads the
one shared time axis on the device (time offsets 0), so the 1312-point padding
and the time copies are never sent.
"""
from __future__ import annotations

import os
from dataclasses import dataclass
from typing import List, Optional

import numpy as np

FLUX_ERR_PAD_SENTINEL = 1.0   # constants.py:13
FLUX_ERR_PAD_THRESHOLD = 0.9  # constants.py:14


@dataclass
class SectorCurves:
    tic_ids: np.ndarray            # int64 [targets]
    times: List[np.ndarray]        # per target, float64 (kept points only)
    fluxes: List[np.ndarray]       # float32
    flux_errs: List[np.ndarray]    # float32
    shared_time: Optional[np.ndarray] = None  # the common axis when every target is a prefix

    def __len__(self) -> int:
        return len(self.tic_ids)

    def target(self, tic_id: int):
        """(time, flux, flux_err) of one target, or None (get_target_data)."""
        idx = np.flatnonzero(self.tic_ids == int(tic_id))
        if idx.size == 0:
            return None
        i = int(idx[0])
        return {"time": self.times[i], "flux": self.fluxes[i], "flux_err": self.flux_errs[i]}

    def batch(self, periods, durations, device="cuda", use_errors: bool = True):
        """A CurveBatch of every target (weights 1/flux_err^2 rounded to
        float32, or unit weights), sharing the time axis when possible."""
        import torch
        from .engine import CurveBatch, _i32, _i64, is_shared_grid
        nc = len(self)
        lens = np.array([len(t) for t in self.times], np.int64)
        pt = np.zeros(nc + 1, np.int64)
        np.cumsum(lens, out=pt[1:])
        y_all = np.concatenate(self.fluxes).astype(np.float32) if nc else np.zeros(0, np.float32)
        w_all = None
        if use_errors:
            e = np.concatenate(self.flux_errs).astype(np.float64)
            w_all = (1.0 / (e * e)).astype(np.float32)

        def grids(g):
            if is_shared_grid(g):
                arr = np.atleast_1d(np.asarray(g, np.float64))
                return arr, np.zeros(nc, np.int64), np.full(nc, len(arr), np.int64)
            arrs = [np.atleast_1d(np.asarray(a, np.float64)) for a in g]
            cnt = np.array([len(a) for a in arrs], np.int64)
            beg = np.zeros(nc, np.int64)
            np.cumsum(cnt[:-1], out=beg[1:])
            return np.concatenate(arrs), beg, cnt

        per, pbeg, pcnt = grids(periods)
        dur, dbeg, dcnt = grids(durations)
        obeg = np.zeros(nc, np.int64)
        np.cumsum(pcnt[:-1], out=obeg[1:])

        def dev(a):
            return torch.from_numpy(np.ascontiguousarray(a)).to(device)

        if self.shared_time is not None:
            t_dev = dev(np.asarray(self.shared_time, np.float64))
            t_off = np.zeros(nc, np.int64)
        else:
            t_dev = dev(np.concatenate(self.times).astype(np.float64))
            t_off = None
        return CurveBatch(t=t_dev, y=dev(y_all), w=None if w_all is None else dev(w_all),
                          periods=dev(per), durations=dev(dur), point_offset=_i64(pt),
                          period_begin=pbeg, period_count=pcnt, dur_begin=dbeg,
                          dur_count=_i32(dcnt), out_begin=obeg,
                          time_offset=None if t_off is None else _i64(t_off))


def load_sector_cache(path: str) -> SectorCurves:
    """Read a cache directory (``data.npz`` inside) or an ``.npz`` file."""
    if os.path.isdir(path):
        path = os.path.join(path, "data.npz")
    with np.load(path, allow_pickle=False) as data:
        keys = set(data.files)
        tic = np.asarray(data["tic_ids"], np.int64)
        vec = bool(data["is_vectorized"]) if "is_vectorized" in keys else False
        time = np.asarray(data["time"])
        flux = np.asarray(data["flux"])
        ferr = np.asarray(data["flux_err"])
        offsets = np.asarray(data["offsets"], np.int64) if "offsets" in keys else None
    if vec:
        if flux.ndim != 2 or flux.shape != ferr.shape or flux.shape[1] != time.shape[0]:
            raise ValueError("vectorized cache: flux/flux_err must be [targets, len(time)]")
        keep = ferr < FLUX_ERR_PAD_THRESHOLD
        t64 = time.astype(np.float64)
        times, fluxes, errs = [], [], []
        prefix = True
        for i in range(flux.shape[0]):
            m = keep[i]
            n = int(m.sum())
            prefix = prefix and bool(m[:n].all())
            times.append(t64[m])
            fluxes.append(flux[i][m].astype(np.float32))
            errs.append(ferr[i][m].astype(np.float32))
        return SectorCurves(tic, times, fluxes, errs, shared_time=t64 if prefix else None)
    if offsets is None:
        raise ValueError("flat cache without offsets")
    ends = list(offsets[1:]) + [len(flux)] if len(offsets) == len(tic) else list(offsets[1:])
    starts = list(offsets[:len(tic)])
    times = [time[a:b].astype(np.float64) for a, b in zip(starts, ends)]
    fluxes = [flux[a:b].astype(np.float32) for a, b in zip(starts, ends)]
    errs = [ferr[a:b].astype(np.float32) for a, b in zip(starts, ends)]
    return SectorCurves(tic, times, fluxes, errs)
