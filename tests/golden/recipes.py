"""Seeded synthetic light-curve recipes shared by the golden-vector scripts,
the tests and the benchmark.

The recipes follow the reference test-suite's inputs (``tests/test_v42_parity.py:12-24``,
``tests/test_astropy_parity.py:15-23``, ``tests/test_synthetic_recovery.py:10-20``)
and the benchmark workload shapes (single 27.4 d sector with a mid-sector gap,
box transits injected multiplicatively as ``inject/box.py:21-27`` does).
"""
from __future__ import annotations

import numpy as np


def inject_box(t, f, period, t0, duration, depth):
    """Multiplicative box transit, as inject/box.py:3-29 defines it:
    in transit where |((t - t0 + P/2) mod P) - P/2| < duration/2."""
    f = np.array(f, dtype=np.float64, copy=True)
    ph = (t - t0 + 0.5 * period) % period - 0.5 * period
    f[np.abs(ph) < 0.5 * duration] *= 1.0 - depth
    return f


def v42_test_recipe():
    """tests/test_v42_parity.py:12-24 (seed 42, 2000 points, dip 0.01 at P=3.521)."""
    np.random.seed(42)
    time = np.linspace(0, 27, 2000).astype(np.float64)
    flux = np.random.normal(0, 0.003, size=2000).astype(np.float64)
    ph = (time % 3.521) / 3.521
    flux[ph < (0.1 / 3.521)] -= 0.01
    flux -= np.mean(flux)
    dy = np.ones_like(flux) * 0.003
    periods = np.linspace(3.0, 4.0, 1000).astype(np.float64)
    durations = np.array([0.05, 0.1, 0.15])
    return time, flux - np.median(flux), dy, periods, durations


def v42_debug_recipe():
    """tests/debug_v42.py:11-24 (200 points)."""
    np.random.seed(42)
    time = np.linspace(0, 27, 200).astype(np.float64)
    flux = np.random.normal(0, 0.003, size=200).astype(np.float64)
    ph = (time % 3.521) / 3.521
    flux[ph < (0.1 / 3.521)] -= 0.01
    flux -= np.median(flux)
    dy = np.ones_like(flux) * 0.003
    return time, flux - np.median(flux), dy, np.linspace(3.0, 4.0, 1000), np.array([0.05, 0.1, 0.15])


def astropy_parity_recipe():
    """tests/test_astropy_parity.py:15-23 (5000 points, P=3.456, fast path n_bins=500)."""
    np.random.seed(42)
    t = np.linspace(0, 10, 5000)
    f = inject_box(t, np.ones_like(t), 3.456, 0.5, 0.1, 0.01)
    f += np.random.normal(0, 0.001, len(t))
    return t, f, None, np.linspace(1.0, 5.0, 1000), np.array([0.05, 0.1, 0.15])


def recovery_recipe():
    """tests/test_synthetic_recovery.py:10-20 (P=7.432, t0=1.5, dur 0.15, depth 0.01)."""
    t = np.linspace(0, 20, 5000)
    f = inject_box(t, np.ones_like(t), 7.432, 1.5, 0.15, 0.01)
    np.random.seed(42)
    f += np.random.normal(0, 0.001, len(t))
    return t, f, None, np.linspace(5.0, 10.0, 1000), np.linspace(0.05, 0.25, 5)


SECTOR_DAYS = 27.4
SECTOR_DURATIONS = np.array([0.04, 0.06, 0.08, 0.12, 0.16, 0.20])


def sector_periods(n=5000, pmin=0.5, pmax=13.7):
    """Log-spaced period grid of the single-curve workload."""
    return np.geomspace(pmin, pmax, n)


def sector_times(rng, n, t_offset=1325.0, gap=1.0):
    """n sorted times over one 27.4 d sector with a `gap`-day hole at mid-sector."""
    out = np.empty(0)
    lo, hi = 0.5 * (SECTOR_DAYS - gap), 0.5 * (SECTOR_DAYS + gap)
    while out.size < n:
        u = SECTOR_DAYS * rng.uniform(size=2 * n)
        u = u[(u < lo) | (u >= hi)]
        out = np.concatenate([out, u])
    return t_offset + np.sort(out[:n])


def sector_curve(n=15000, seed=0):
    """Single-curve workload: N points over a sector with a 1 d mid-sector gap,
    y = 1 + N(0, 1e-3) with a box transit P=3.71, t0=1326.2, dur=0.10,
    depth=1.5e-3, dy = 1e-3."""
    rng = np.random.default_rng(seed)
    t = sector_times(rng, n)
    y = 1.0 + rng.normal(0.0, 1e-3, n)
    y = inject_box(t, y, 3.71, 1326.2, 0.10, 1.5e-3)
    dy = np.full(n, 1e-3)
    return t, y, dy


CADENCE_2MIN = 2.0 / 1440.0


def cadence_grid(t_offset=1325.0, gap=1.0):
    """2-minute cadence over one sector minus a mid-sector gap."""
    t = np.arange(0.0, SECTOR_DAYS, CADENCE_2MIN)
    lo, hi = 0.5 * (SECTOR_DAYS - gap), 0.5 * (SECTOR_DAYS + gap)
    return t_offset + t[(t < lo) | (t >= hi)]


def uniform_batch(n_curves=4096, n=15000, seed=1, transit_fraction=0.3):
    """Uniform batch: every curve has n float32 points subsampled from the
    2-minute cadence grid of one sector with a gap, white noise sigma drawn
    log-uniform in [2e-4, 5e-3], and `transit_fraction` of the curves carry a
    box transit (P U[0.5,13], dur U[0.03,0.25], depth U[3e-4,1e-2]).

    Returns (t [n_curves, n] float64, y [n_curves, n] float32,
    dy [n_curves, n] float32, truth list)."""
    rng = np.random.default_rng(seed)
    grid = cadence_grid()
    t = np.empty((n_curves, n), np.float64)
    y = np.empty((n_curves, n), np.float32)
    dy = np.empty((n_curves, n), np.float32)
    truth = []
    for c in range(n_curves):
        idx = np.sort(rng.choice(grid.size, size=n, replace=False))
        tc = grid[idx]
        sig = float(np.exp(rng.uniform(np.log(2e-4), np.log(5e-3))))
        yc = 1.0 + rng.normal(0.0, sig, n)
        tr = None
        if rng.uniform() < transit_fraction:
            P = rng.uniform(0.5, 13.0)
            dur = rng.uniform(0.03, 0.25)
            dep = rng.uniform(3e-4, 1e-2)
            t0 = tc[0] + rng.uniform(0.0, P)
            yc = inject_box(tc, yc, P, t0, dur, dep)
            tr = (P, t0, dur, dep)
        t[c] = tc
        y[c] = yc.astype(np.float32)
        dy[c] = sig
        truth.append(tr)
    return t, y, dy, truth


MIXED_DURATIONS = np.geomspace(0.02, 0.3, 8)


def mixed_curve_spec(rng):
    """One curve of the uneven-batch distribution: N log-uniform in
    [1e3, 2e5], 1-13 concatenated sectors, 2- or 30-minute cadence (N capped
    by the cadences available), a frequency-uniform period grid from 0.5 d to
    baseline/2 with step 1/(84 baseline) in frequency (clipped to 1 000-60 000
    periods)."""
    n_sec = int(rng.integers(1, 14))
    cad = CADENCE_2MIN if rng.uniform() < 0.5 else 30.0 / 1440.0
    avail = int(n_sec * (SECTOR_DAYS - 1.0) / cad)
    n = min(int(np.exp(rng.uniform(np.log(1e3), np.log(2e5)))), avail)
    base = n_sec * SECTOR_DAYS
    fmin, fmax = 2.0 / base, 2.0
    n_per = int(np.clip((fmax - fmin) * 84.0 * base, 1000, 60000))
    return n_sec, cad, n, n_per


def mixed_curve(rng, n_sec, cad, n, n_per, t_offset=None, transit_fraction=0.3):
    """Times (sorted, gaps at each mid-sector), float32 flux with white noise
    and an optional box transit, float32 dy, and the curve's period grid."""
    t_offset = rng.uniform(1300.0, 2700.0) if t_offset is None else t_offset
    grid = []
    for s in range(n_sec):
        g = np.arange(0.0, SECTOR_DAYS, cad)
        lo, hi = 0.5 * (SECTOR_DAYS - 1.0), 0.5 * (SECTOR_DAYS + 1.0)
        grid.append(t_offset + s * SECTOR_DAYS + g[(g < lo) | (g >= hi)])
    grid = np.concatenate(grid)
    t = grid[np.sort(rng.choice(grid.size, size=n, replace=False))]
    sig = float(np.exp(rng.uniform(np.log(2e-4), np.log(5e-3))))
    y = 1.0 + rng.normal(0.0, sig, n)
    if rng.uniform() < transit_fraction:
        P = rng.uniform(0.5, min(40.0, 0.5 * n_sec * SECTOR_DAYS))
        y = inject_box(t, y, P, t[0] + rng.uniform(0.0, P), rng.uniform(0.03, 0.25),
                       rng.uniform(3e-4, 1e-2))
    base = n_sec * SECTOR_DAYS
    periods = 1.0 / np.linspace(2.0, 2.0 / base, n_per)
    return t, y.astype(np.float32), np.full(n, sig, np.float32), periods


def mixed_batch(n_curves=8192, seed=2, max_points=None):
    """Uneven batch: lists of per-curve (t, y, dy, periods); `max_points`
    optionally caps N (smaller test batches of the same shape family)."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n_curves):
        n_sec, cad, n, n_per = mixed_curve_spec(rng)
        if max_points is not None:
            n = min(n, max_points)
        out.append(mixed_curve(rng, n_sec, cad, n, n_per))
    return out


def precision_curve(rng, n=200_000, n_sec=13, sigma=5e-4):
    """Precision-stress curve: t offset U[1300, 2700] BTJD, 13 concatenated
    sectors (~356 d) at 2-min cadence with mid-sector gaps, n points, white
    noise sigma and one box transit (P U[0.5, 40] d, duration U[0.05, 0.3] d,
    depth 5e-4).  Returns (t, y float32, dy float32, (P, t0, duration))."""
    t_offset = rng.uniform(1300.0, 2700.0)
    grid = []
    for s in range(n_sec):
        g = np.arange(0.0, SECTOR_DAYS, CADENCE_2MIN)
        lo, hi = 0.5 * (SECTOR_DAYS - 1.0), 0.5 * (SECTOR_DAYS + 1.0)
        grid.append(t_offset + s * SECTOR_DAYS + g[(g < lo) | (g >= hi)])
    grid = np.concatenate(grid)
    t = grid[np.sort(rng.choice(grid.size, size=min(n, grid.size), replace=False))]
    P, dur = rng.uniform(0.5, 40.0), rng.uniform(0.05, 0.3)
    t0 = t[0] + rng.uniform(0.0, P)
    y = inject_box(t, 1.0 + rng.normal(0.0, sigma, t.size), P, t0, dur, 5e-4)
    return t, y.astype(np.float32), np.full(t.size, sigma, np.float32), (P, t0, dur)


def precision_periods(n=100_000, pmin=0.5, pmax=150.0):
    """Frequency-uniform grid over [pmin, pmax] (largest period first)."""
    return 1.0 / np.linspace(1.0 / pmin, 1.0 / pmax, n)[::-1]


PRECISION_DURATIONS = np.geomspace(0.02, 0.3, 8)


def mixed_spec_indexed(seed, i):
    """(n_sectors, cadence, n, n_periods) of curve i of the indexed uneven
    batch: every curve draws from its own generator, seeded by (seed, i), so a
    rank can make exactly its share of a large batch."""
    return mixed_curve_spec(np.random.default_rng([int(seed), int(i)]))


def mixed_curve_indexed(seed, i):
    """Curve i of the indexed uneven batch: (t, y, dy, periods)."""
    rng = np.random.default_rng([int(seed), int(i)])
    return mixed_curve(rng, *mixed_curve_spec(rng))
