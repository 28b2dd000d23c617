"""Multi-rank certificate logic on CPU with gloo, world size 2: the pair
partition covers every pair exactly once, balances the cost, and the gather
reassembles per-pair results in the original order (no GPU needed)."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from fastlinkingnumbers_b200 import sharding, workloads


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, off, pairs, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    costs = sharding.pair_costs(off, pairs)
    mine = sharding.shard_pairs(costs, world, rank)
    # Stand-in for the per-pair linking numbers this rank would compute.
    values = pairs[mine, 0] * 1000.0 + pairs[mine, 1] + 0.25
    full = sharding.gather_pair_results(mine, values, len(pairs))
    np.save(os.path.join(out_dir, f"r{rank}.npy"), full)
    np.save(os.path.join(out_dir, f"m{rank}.npy"), mine)
    dist.barrier()
    dist.destroy_process_group()


def test_shard_and_gather_two_ranks(tmp_path):
    off, _ = workloads.mixed_batch(seed=1, n_loops=40, hi=4096)
    rng = np.random.default_rng(0)
    pairs = np.array(sorted({tuple(sorted(rng.choice(40, 2, replace=False))) for _ in range(300)}),
                     dtype=np.int32)
    mp.spawn(_worker, args=(2, _free_port(), off, pairs, str(tmp_path)), nprocs=2, join=True)
    r0, r1 = np.load(tmp_path / "r0.npy"), np.load(tmp_path / "r1.npy")
    expect = pairs[:, 0] * 1000.0 + pairs[:, 1] + 0.25
    assert np.array_equal(r0, expect) and np.array_equal(r1, expect)
    m0, m1 = np.load(tmp_path / "m0.npy"), np.load(tmp_path / "m1.npy")
    assert len(np.intersect1d(m0, m1)) == 0 and len(m0) + len(m1) == len(pairs)
    c = sharding.pair_costs(off, pairs)
    assert abs(c[m0].sum() - c[m1].sum()) <= c.max()  # LPT bound


def test_shard_pairs_is_deterministic_partition():
    c = np.random.default_rng(3).random(1000)
    parts = [sharding.shard_pairs(c, 4, r) for r in range(4)]
    assert np.array_equal(np.sort(np.concatenate(parts)), np.arange(1000))
    loads = [c[p].sum() for p in parts]
    assert max(loads) - min(loads) <= c.max()
    with pytest.raises(ValueError):
        sharding.shard_pairs(c, 2, 2)
