"""Generate tests/golden/emu_golden.npz from the reference's own CPU code.

The reference ships a pure-Python restatement of the Astropy-style binned BLS
(``tests/debug_emu.py:4-64``, ``emulate_astropy``).  This script imports that
file from a reference checkout (``--ref``, default /root/reference) and records
its output for the input recipe of ``tests/debug_emu.py:66-83`` /
``tests/debug_v42.py:11-24`` over a grid of periods, plus a weighted variant.
It runs only where the reference checkout exists; the .npz it writes is
committed and is what the tests read.
"""
import argparse
import importlib.util
import os

import numpy as np


def load_emu(ref_root):
    path = os.path.join(ref_root, "tests", "debug_emu.py")
    spec = importlib.util.spec_from_file_location("ref_debug_emu", path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.emulate_astropy


def recipe(seed=42, n=200, weighted=False):
    # tests/debug_emu.py:67-77
    rs = np.random.RandomState(seed)
    time = np.linspace(0, 27, n).astype(np.float64)
    flux = rs.normal(0, 0.003, size=n).astype(np.float64)
    ph = (time % 3.521) / 3.521
    flux[ph < (0.1 / 3.521)] -= 0.01
    flux -= np.median(flux)
    dy = np.ones_like(flux) * 0.003
    if weighted:
        dy = dy * (1.0 + 0.5 * rs.uniform(size=n))
    return time, flux, dy


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default="/root/reference")
    ap.add_argument("--out", default=os.path.join(os.path.dirname(__file__), "emu_golden.npz"))
    args = ap.parse_args()
    emulate = load_emu(args.ref)
    durations = np.array([0.05, 0.1, 0.15])
    periods = np.concatenate([np.linspace(3.0, 4.0, 21), [3.521, 1.37, 6.9, 11.3]])
    cases = {}
    for name, weighted in (("unit", False), ("weighted", True)):
        t, y, dy = recipe(weighted=weighted)
        pw = np.array([emulate(t, y, dy, p, durations, 10) for p in periods])
        cases[name] = (t, y, dy, pw)
    np.savez_compressed(
        args.out, periods=periods, durations=durations, oversample=10,
        **{f"{k}_{f}": v for k, (t, y, dy, pw) in cases.items()
           for f, v in (("t", t), ("y", y), ("dy", dy), ("power", pw))})
    print("wrote", args.out)


if __name__ == "__main__":
    main()
