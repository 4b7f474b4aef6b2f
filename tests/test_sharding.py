"""Multi-GPU host logic on CPU: the LPT split of a ragged batch and the
collectives bench.py uses, run as two gloo ranks (world_size 2)."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from astro_transit_gpu_b200.sharding import gather_best, lpt_assign, max_over_ranks, shard_of


def test_lpt_assign_is_a_balanced_partition():
    rng = np.random.default_rng(3)
    # ragged costs: points x periods, both log-uniform
    costs = np.exp(rng.uniform(np.log(1e3), np.log(2e5), 500)) * \
        np.exp(rng.uniform(np.log(1e3), np.log(6e4), 500))
    for world in (1, 2, 3, 8):
        parts = lpt_assign(costs, world)
        allc = np.concatenate(parts)
        assert np.array_equal(np.sort(allc), np.arange(costs.size))  # disjoint and complete
        loads = np.array([costs[p].sum() for p in parts])
        # LPT bound: max load <= mean load + largest single cost
        assert loads.max() <= costs.sum() / world + costs.max() + 1e-6
        assert all(np.array_equal(shard_of(costs, r, world), parts[r]) for r in range(world))


def test_lpt_assign_edge_cases():
    assert [p.tolist() for p in lpt_assign([], 2)] == [[], []]
    assert [p.tolist() for p in lpt_assign([5.0], 3)] == [[0], [], []]
    with pytest.raises(ValueError):
        lpt_assign([1.0], 0)
    with pytest.raises(ValueError):
        shard_of([1.0], 2, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, costs, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        mine = shard_of(costs, rank, world)
        # each rank "times" its shard: the job time is the slowest rank's
        local_ms = float(costs[mine].sum()) * 1e-6
        job_ms = max_over_ranks(local_ms)
        # best-peak records of this rank's curves: (curve, best period index, power)
        rec = np.stack([mine.astype(np.float64), mine * 7.0 % 13, np.sqrt(mine + 1.0)], axis=1)
        allrec = gather_best(rec)
        q.put((rank, mine.tolist(), local_ms, job_ms, allrec))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_time_and_gather():
    rng = np.random.default_rng(11)
    costs = rng.uniform(1.0, 100.0, 37)
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, costs, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort(key=lambda r: r[0])
    shards = [np.array(r[1]) for r in res]
    assert np.array_equal(np.sort(np.concatenate(shards)), np.arange(costs.size))
    assert res[0][3] == res[1][3] == pytest.approx(max(r[2] for r in res))
    # every rank receives every curve's record, in rank order
    expect = np.concatenate([np.stack([s.astype(np.float64), s * 7.0 % 13, np.sqrt(s + 1.0)], 1)
                             for s in shards])
    for r in res:
        assert np.array_equal(r[4], expect)
