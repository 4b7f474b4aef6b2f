"""bench.py --gpus N starts N ranks under torchrun when it is not already
running under one (one process per GPU); this checks that launcher on CPU with
two gloo ranks, through the same code path, and the bench's argument
defaults."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)


def test_bench_launches_two_ranks_that_see_each_other():
    env = {k: v for k, v in os.environ.items()
           if k not in ("WORLD_SIZE", "RANK", "LOCAL_RANK", "MASTER_ADDR", "MASTER_PORT")}
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--gpus", "2",
                        "--launch-check"], capture_output=True, text=True, timeout=240, env=env,
                       cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
    assert len(lines) == 1, r.stdout  # rank 0 alone prints
    assert lines[0]["world_size"] == 2 and lines[0]["ranks_seen"] == 2


def test_bench_defaults():
    import bench
    a = bench.parse([])
    assert (a.gpus, a.workload, a.curves, a.method) == (1, "uniform", 4096, "parity")
    assert a.warmup >= 3
    assert bench.parse(["--workload", "mixed"]).curves == 8192
    assert bench.parse(["--workload", "precision"]).curves == 512
    assert bench.LAYOUT_WORDS == {0: 4, 1: 3, 2: 2, 3: 2}


def test_indexed_uneven_batch_is_split_by_lpt_without_overlap():
    import numpy as np
    import recipes as R
    from astro_transit_gpu_b200.sharding import lpt_assign
    specs = [R.mixed_spec_indexed(2000, i) for i in range(64)]
    cost = [s[2] * s[3] for s in specs]
    parts = lpt_assign(cost, 4)
    assert sorted(np.concatenate(parts).tolist()) == list(range(64))
    loads = [sum(cost[i] for i in p) for p in parts]
    assert max(loads) <= 4 / 3 * max(sum(cost) / 4, max(cost))
    # a curve is the same whichever rank makes it
    a = R.mixed_curve_indexed(2000, 5)
    b = R.mixed_curve_indexed(2000, 5)
    assert all(np.array_equal(x, y) for x, y in zip(a, b))
    assert len(a[0]) == specs[5][2] and len(a[3]) == specs[5][3]


def test_traffic_is_scaled_from_the_committed_captures():
    """roofline.traffic: the committed ncu captures give their own launches'
    DRAM bytes back, and scale with curves (uniform) or algorithmic bytes
    (uneven)."""
    import json
    import os
    import bench
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    uni = json.load(open(os.path.join(root, "profiles", "search_kernel_uniform_batch.json")))
    fix = json.load(open(os.path.join(root, "profiles", "search_kernel_fixed_uneven_batch.json")))
    assert bench.measured_traffic("uniform", "parity", uni["capture_curves"], 1.0) == \
        uni["dram_bytes_per_launch"]
    assert bench.measured_traffic("uniform", "parity", 4096, 1.0) == \
        4 * uni["dram_bytes_per_launch"]
    a = fix["capture_algorithmic_bytes"]
    assert bench.measured_traffic("mixed", "fast", 512, a) == fix["dram_bytes_per_launch"]
    assert bench.measured_traffic("mixed", "fast", 8192, 16 * a) == \
        16 * fix["dram_bytes_per_launch"]
    assert bench.measured_traffic("mixed", "parity", 8192, a) is None
    # the capture's algorithmic bytes are those of its 512 curves
    import recipes as R
    cs = [R.mixed_curve_indexed(2000, i) for i in range(512)]
    assert bench.search_algorithmic_bytes([len(c[0]) for c in cs], [len(c[3]) for c in cs]) == a
