"""Sharding of independent pairs across ranks (iqm_b200.parallel): LPT partition properties on one
process, and the score gather over two gloo ranks on the CPU."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from iqm_b200 import fsim_plane_size, parallel


def test_shard_lpt_partition_and_balance():
    rng = np.random.Generator(np.random.PCG64(7))
    sizes = [(int(rng.integers(256, 2049)), int(rng.integers(256, 2049))) for _ in range(256)]
    costs = [parallel.pair_cost("fsim", w, h) for w, h in sizes]
    for world in (1, 2, 3, 8):
        shards = parallel.shard_lpt(costs, world)
        flat = sorted(i for s in shards for i in s)
        assert flat == list(range(len(costs)))          # every pair exactly once
        loads = [sum(costs[i] for i in s) for s in shards]
        # LPT bound: max load <= mean load + largest item
        assert max(loads) <= sum(costs) / world + max(costs) + 1e-6
        assert shards == parallel.shard_lpt(costs, world)  # deterministic on every rank


def test_shard_lpt_edge_cases():
    assert parallel.shard_lpt([], 3) == [[], [], []]
    assert parallel.shard_lpt([5.0], 2) == [[0], []]
    # equal costs: round-robin by rank order
    assert parallel.shard_lpt([1.0] * 4, 2) == [[0, 2], [1, 3]]
    with pytest.raises(ValueError):
        parallel.shard_lpt([1.0], 0)


def test_pair_cost_uses_fsim_plane():
    assert fsim_plane_size(1920, 1080) == (480, 270)
    assert fsim_plane_size(3840, 2160) == (480, 270)
    assert fsim_plane_size(300, 200) == (300, 200)
    assert parallel.pair_cost("ssim", 100, 50) == 8.0 * 100 * 50
    assert parallel.pair_cost("fsim", 1920, 1080) > parallel.pair_cost("ssim", 1920, 1080)


def _fake_eval(items):
    # stands in for a metric: two scores per pair from the pair's pixels
    return [(float(a.mean()), float(b.sum())) for a, b in items]


def _worker(rank, world, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rng = np.random.Generator(np.random.PCG64(3))
        pairs = [(rng.random((h, h + 3)), rng.random((h, h + 3))) for h in range(5, 16)]
        costs = [parallel.pair_cost("fsim", a.shape[1], a.shape[0]) for a, _ in pairs]
        out = parallel.evaluate_sharded(_fake_eval, pairs, costs, rank, world)
        q.put((rank, out))
    finally:
        dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_evaluate_sharded_gloo_two_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    rng = np.random.Generator(np.random.PCG64(3))
    pairs = [(rng.random((h, h + 3)), rng.random((h, h + 3))) for h in range(5, 16)]
    want = np.array(_fake_eval(pairs))
    for r in (0, 1):
        assert res[r].shape == want.shape
        np.testing.assert_array_equal(res[r], want)
