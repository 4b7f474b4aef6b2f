"""Continuous-batching search server on one GPU.

Requests (one light curve and its own period/duration grid each) are
submitted from any thread and return a ``concurrent.futures.Future``.  A
worker thread forms batches from the waiting requests -- first come, first
served, among requests with the same search configuration -- as long as the
device-memory budget and the batch size allow, and launches each batch as one
plan (stage, persistent search, best peak) on one of several CUDA streams.
Batches already on the GPU keep running while the next ones are formed and
launched, so requests that arrive meanwhile are admitted as soon as memory
and a stream are free, and their work overlaps on the device.  A finished
batch is split into per-request results (the same arrays
``split_outputs`` gives) and its memory returns to the budget.

Every curve's result depends only on that curve (staging, folding and window
search are per curve and the arithmetic is exact up to the final FP32/FP64
formulas), so a request gets the same result alone and in any mix.

Latency is measured per request from ``submit`` to the moment its result is
ready; :meth:`BLSServer.stats` reports p50/p99 and the completed rate.

A request can carry a timeout: if it is still waiting for admission when the
timeout has passed, it is dropped and its future raises ``TimeoutError``.  A
client can also ``cancel()`` its future while the request waits; an admitted
request runs to completion (its batch is already on the GPU).
"""
from __future__ import annotations

import threading
import time
from collections import deque
from concurrent.futures import Future, InvalidStateError
from dataclasses import dataclass, field
from typing import Dict, List, Optional

import numpy as np
import torch

from .engine import BLSEngine, CurveBatch, SearchConfig, split_host_outputs


@dataclass(eq=False)
class _Request:
    t: np.ndarray
    y: np.ndarray
    w: Optional[np.ndarray]
    periods: np.ndarray
    durations: np.ndarray
    config: SearchConfig
    flux_dtype: type
    nbytes: int
    arrival: float
    future: Future = field(default_factory=Future)
    done: float = 0.0
    deadline: Optional[float] = None  # admission deadline (perf_counter seconds)


@dataclass(eq=False)
class _Batch:
    requests: List[_Request]
    batch: CurveBatch
    plan: object
    stream: torch.cuda.Stream
    event: torch.cuda.Event
    nbytes: int
    host_out: Dict[str, torch.Tensor]  # pinned copies of the outputs, valid after `event`


def admit(pending, key, held: int, budget: int, max_batch: int):
    """Form the next batch: the oldest request and the following ones with the
    same configuration, in arrival order, while the batch has fewer than
    `max_batch` requests and the bytes held stay within `budget`; the first
    same-configuration request that does not fit ends the batch (no later one
    overtakes it).  Returns (batch, remaining requests in order, bytes held)."""
    pending = deque(pending)
    if not pending:
        return [], pending, held
    k0 = key(pending[0])
    take, rest, used, closed = [], deque(), held, False
    for r in pending:
        if (not closed and key(r) == k0 and len(take) < max_batch
                and used + r.nbytes <= budget):
            take.append(r)
            used += r.nbytes
        else:
            if key(r) == k0:
                closed = True
            rest.append(r)
    return take, rest, used


def prune(pending, now: float):
    """Split the waiting requests into those that keep waiting (in arrival
    order), those whose admission deadline has passed, and those whose client
    cancelled them."""
    keep, expired, cancelled = deque(), [], []
    for r in pending:
        if r.future.cancelled():
            cancelled.append(r)
        elif r.deadline is not None and now > r.deadline:
            expired.append(r)
        else:
            keep.append(r)
    return keep, expired, cancelled


def check_request(t: np.ndarray, y: np.ndarray, dy, periods: np.ndarray,
                  durations: np.ndarray) -> None:
    """Reject, at submission, what would fail a whole batch later: one
    request's invalid data makes the engine report ATB_EDATA for the batch it
    joins, so every other request in that batch would fail with it.  The rules
    are the reference's (search/api.py:53-70) plus the engine's grid limits."""
    if len(t) < 1:
        raise ValueError("a request needs at least one point")
    if not (np.all(np.isfinite(t)) and np.all(np.isfinite(y))):
        raise ValueError("Input time or flux contains NaNs or infinite values.")
    if dy is not None and not np.all(np.isfinite(dy) & (dy > 0)):
        raise ValueError("flux_err must be finite and strictly positive.")
    if dy is not None:
        with np.errstate(over="ignore"):
            w = (1.0 / (dy * dy)).astype(np.float32)
        if not np.all(np.isfinite(w)):
            raise ValueError("flux_err too small: its float32 weight 1/flux_err^2 overflows")
    if len(periods) < 1 or not np.all(np.isfinite(periods) & (periods > 0)):
        raise ValueError("periods must be positive and finite")
    if not 1 <= len(durations) <= 32 or not np.all(np.isfinite(durations) & (durations > 0)):
        raise ValueError("durations: 1 to 32, positive and finite")


def request_bytes(n_points: int, n_periods: int, n_durations: int) -> int:
    """Device bytes a request holds while its batch runs: inputs (t f64, y, w
    f32), staged points (16 B), the grids and the per-period outputs (28 B),
    rounded up for the plan's descriptors."""
    return int(n_points * (16 + 16) + n_periods * (8 + 28) + n_durations * 8 + 4096)


class BLSServer:
    """Continuous-batching BLS server (one GPU, one worker thread).

    memory_budget  device bytes the in-flight batches may hold (admission)
    max_batch      most requests in one batch
    n_streams      batches in flight at once
    """

    def __init__(self, device=0, memory_budget: float = 120e9, max_batch: int = 512,
                 n_streams: int = 4):
        self.engine = BLSEngine.get(device)
        self.device = self.engine.device
        self.memory_budget = int(memory_budget)
        self.max_batch = int(max_batch)
        self.streams = [torch.cuda.Stream(self.device) for _ in range(max(1, n_streams))]
        self._pending: deque = deque()
        self._inflight: List[_Batch] = []
        self._held = 0
        self._cv = threading.Condition()
        self._stop = False
        self._latencies: List[float] = []
        self._t_first: Optional[float] = None
        self._t_last: Optional[float] = None
        self._batches = 0
        self._max_held = 0
        self._expired = 0
        self._cancelled = 0
        # the queue is pruned only when a client cancelled a request or the
        # earliest admission deadline has passed (not on every poll)
        self._cancel_seen = False
        self._next_deadline = float("inf")
        self._worker = threading.Thread(target=self._run, name="bls-server", daemon=True)
        self._worker.start()

    # ---------------------------------------------------------------- client
    def submit(self, t, y, dy=None, periods=None, durations=None, method: str = "fast",
               n_bins: int = 200, objective: Optional[str] = None, oversample: int = 10,
               max_bins: Optional[int] = None, timeout: Optional[float] = None) -> Future:
        """Queue one search; the future resolves to the curve's per-period
        outputs (power, depth, depth_err, t0, duration, window) and best_index.
        `timeout` (seconds): if the request is still waiting for admission
        that long after submission, it is dropped and the future raises
        TimeoutError.  Cancelling the future while the request waits drops it
        too."""
        if periods is None or durations is None:
            raise ValueError("periods and durations must be given")
        t = np.ascontiguousarray(t, np.float64)
        y = np.asarray(y)
        fdt = np.float64 if y.dtype == np.float64 else np.float32
        y = np.ascontiguousarray(y, fdt)
        if len(t) != len(y):
            raise ValueError("time and flux must have the same length")
        w = None
        if dy is not None:
            dy = np.asarray(dy, np.float64)
            if len(dy) != len(y):
                raise ValueError("flux_err and flux must have the same length")
            with np.errstate(over="ignore", divide="ignore"):  # rejected below
                w = (1.0 / (dy * dy)).astype(np.float32)
        cfg = (SearchConfig("fast", n_bins=int(n_bins)) if method == "fast" else
               SearchConfig("parity", objective=objective or "snr", oversample=int(oversample),
                            max_bins=max_bins))
        cfg.params()  # validates the combination
        per = np.atleast_1d(np.asarray(periods, np.float64))
        dur = np.atleast_1d(np.asarray(durations, np.float64))
        check_request(t, y, dy, per, dur)
        now = time.perf_counter()
        req = _Request(t, y, w, per, dur, cfg, fdt,
                       request_bytes(len(t), len(per), len(dur)), now,
                       deadline=None if timeout is None else now + float(timeout))
        if req.nbytes > self.memory_budget:
            raise MemoryError(f"request needs {req.nbytes} bytes, budget {self.memory_budget}")
        req.future.add_done_callback(self._on_done)
        with self._cv:
            if self._stop:
                raise RuntimeError("server is closed")
            self._pending.append(req)
            if req.deadline is not None:
                self._next_deadline = min(self._next_deadline, req.deadline)
            self._cv.notify()
        return req.future

    def _on_done(self, fut: Future) -> None:
        if fut.cancelled():
            with self._cv:
                self._cancel_seen = True

    def stats(self) -> Dict[str, float]:
        with self._cv:
            lat = np.array(self._latencies)
            span = (self._t_last - self._t_first) if self._t_first is not None else 0.0
            return {
                "completed": int(lat.size), "batches": self._batches,
                "p50_ms": float(np.percentile(lat, 50) * 1e3) if lat.size else float("nan"),
                "p99_ms": float(np.percentile(lat, 99) * 1e3) if lat.size else float("nan"),
                "mean_ms": float(lat.mean() * 1e3) if lat.size else float("nan"),
                "curves_per_s": float(lat.size / span) if span > 0 else float("nan"),
                "max_held_bytes": self._max_held,
                "expired": self._expired, "cancelled": self._cancelled,
            }

    def reset_stats(self) -> None:
        """Forget the latencies and batch count gathered so far (after a
        warm-up, say)."""
        with self._cv:
            self._latencies.clear()
            self._t_first = self._t_last = None
            self._batches = 0
            self._expired = self._cancelled = 0

    def close(self) -> None:
        """Finish every submitted request, then stop the worker."""
        with self._cv:
            self._stop = True
            self._cv.notify()
        self._worker.join()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---------------------------------------------------------------- worker
    @staticmethod
    def _key(r: _Request):
        c = r.config
        return (c.method, c.objective, c.n_bins, c.oversample, c.max_bins, r.flux_dtype,
                r.w is not None)

    def _admit(self) -> List[_Request]:
        take, self._pending, self._held = admit(self._pending, self._key, self._held,
                                                self.memory_budget, self.max_batch)
        # from here on a request runs; one cancelled a moment ago is dropped
        run = []
        for r in take:
            if r.future.set_running_or_notify_cancel():
                run.append(r)
            else:
                self._held -= r.nbytes
                self._cancelled += 1
        self._max_held = max(self._max_held, self._held)
        return run

    def _launch(self, reqs: List[_Request], stream: torch.cuda.Stream) -> _Batch:
        with torch.cuda.stream(stream):
            batch = CurveBatch.from_arrays(
                [r.t for r in reqs], [r.y for r in reqs],
                periods=[r.periods for r in reqs], durations=[r.durations for r in reqs],
                device=self.device, flux_dtype=reqs[0].flux_dtype,
                weights=[r.w for r in reqs] if reqs[0].w is not None else None)
            plan = self.engine.plan(batch, reqs[0].config, stream=stream)
            plan.execute(stream)
            # outputs back to pinned host memory in the batch's stream order, so
            # the worker only slices them once the batch's event has fired
            host_out = {k: torch.empty(v.shape, dtype=v.dtype, pin_memory=True)
                        for k, v in plan.outputs.items()}
            for k, v in plan.outputs.items():
                host_out[k].copy_(v, non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(stream)
        return _Batch(reqs, batch, plan, stream, ev, sum(r.nbytes for r in reqs), host_out)

    def _finish(self, b: _Batch) -> None:
        try:
            b.plan.check()
            # each request gets its own copy: the batch's pinned buffers go back
            # to the host allocator's cache now, however long clients keep results
            outs = [{k: v.copy() if isinstance(v, np.ndarray) else v for k, v in d.items()}
                    for d in split_host_outputs(b.batch,
                                                {k: v.numpy() for k, v in b.host_out.items()})]
            b.host_out = {}
            err = None
        except Exception as e:  # invalid data: every request of the batch fails
            outs, err = None, e
        finally:
            b.plan.close()
        now = time.perf_counter()
        with self._cv:
            self._held -= b.nbytes
            self._batches += 1
            for r in b.requests:
                r.done = now
                self._latencies.append(r.done - r.arrival)
                self._t_first = r.arrival if self._t_first is None else min(self._t_first,
                                                                            r.arrival)
                self._t_last = now
        for i, r in enumerate(b.requests):
            if err is None:
                r.future.set_result(outs[i])
            else:
                r.future.set_exception(err)

    def _run(self) -> None:
        try:
            self._loop()
        except BaseException as e:  # never leave a client waiting on a dead worker
            with self._cv:
                self._stop = True
                waiting = list(self._pending) + [r for b in self._inflight for r in b.requests]
                self._pending.clear()
            for r in waiting:
                if not r.future.done():
                    r.future.set_exception(RuntimeError(f"server worker failed: {e!r}"))
            raise

    def _loop(self) -> None:
        torch.cuda.set_device(self.device)
        while True:
            # retire finished batches
            for b in [b for b in self._inflight if b.event.query()]:
                self._inflight.remove(b)
                self._finish(b)
            expired = []
            with self._cv:
                now = time.perf_counter()
                if self._cancel_seen or now > self._next_deadline:
                    self._cancel_seen = False
                    self._pending, expired, cancelled = prune(self._pending, now)
                    self._expired += len(expired)
                    self._cancelled += len(cancelled)
                    self._next_deadline = min((r.deadline for r in self._pending
                                               if r.deadline is not None), default=float("inf"))
            for r in expired:
                try:
                    r.future.set_exception(TimeoutError(
                        "request not admitted within its timeout"))
                except InvalidStateError:  # cancelled by its client meanwhile
                    pass
            with self._cv:
                busy = {id(b.stream) for b in self._inflight}
                free = [s for s in self.streams if id(s) not in busy]
                reqs = self._admit() if free else []
                if not reqs:
                    if self._stop and not self._pending and not self._inflight:
                        return
                    if not self._inflight:
                        self._cv.wait(timeout=0.05)
                        continue
            if reqs:
                try:
                    self._inflight.append(self._launch(reqs, free[0]))
                except Exception as e:
                    with self._cv:
                        self._held -= sum(r.nbytes for r in reqs)
                    for r in reqs:
                        r.future.set_exception(e)
                continue
            time.sleep(20e-6)  # batches on the GPU: poll their events
