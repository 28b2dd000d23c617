"""Multi-GPU certificates: loop pairs are independent, so a certificate over
N ranks partitions the pairs by estimated cost (no data-path collective) and
gathers the per-pair results once at the end (about 20 bytes per pair).

Used with one process per GPU (torchrun); the host logic here is tested with
gloo ranks on CPU.
"""
from __future__ import annotations

import heapq

import numpy as np


def pair_costs(loop_offsets, pairs, method: str = "barneshut") -> np.ndarray:
    """Work estimate per pair: n_i n_j for the direct sum, (n_i + n_j) log2 for BH."""
    n = np.diff(np.asarray(loop_offsets, dtype=np.int64)).astype(np.float64)
    pairs = np.asarray(pairs).reshape(-1, 2)
    a, b = n[pairs[:, 0]], n[pairs[:, 1]]
    if method == "directsum":
        return a * b
    return (a + b) * np.log2(a + b + 2.0)


def shard_pairs(costs, world: int, rank: int) -> np.ndarray:
    """Indices of the pairs rank `rank` evaluates: longest-processing-time
    first onto the least-loaded rank (ties -> lower rank), deterministic on
    every rank."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad world/rank")
    costs = np.asarray(costs, dtype=np.float64)
    order = np.argsort(-costs, kind="stable")
    heap = [(0.0, r) for r in range(world)]
    owner = np.empty(len(costs), dtype=np.int64)
    for p in order:
        load, r = heapq.heappop(heap)
        owner[p] = r
        heapq.heappush(heap, (load + costs[p], r))
    return np.nonzero(owner == rank)[0]


def gather_pair_results(local_idx, local_values, npairs: int, group=None) -> np.ndarray:
    """All-gathers (index, value) shards into one array in pair order."""
    import torch
    import torch.distributed as dist
    idx = torch.as_tensor(np.asarray(local_idx, dtype=np.int64))
    val = torch.as_tensor(np.asarray(local_values, dtype=np.float64))
    world = dist.get_world_size(group)
    sizes = [torch.zeros(1, dtype=torch.int64) for _ in range(world)]
    dist.all_gather(sizes, torch.tensor([len(idx)], dtype=torch.int64), group=group)
    m = int(max(s.item() for s in sizes))
    pad_i = torch.full((m,), -1, dtype=torch.int64)
    pad_v = torch.zeros(m, dtype=torch.float64)
    pad_i[:len(idx)] = idx
    pad_v[:len(val)] = val
    all_i = [torch.empty(m, dtype=torch.int64) for _ in range(world)]
    all_v = [torch.empty(m, dtype=torch.float64) for _ in range(world)]
    dist.all_gather(all_i, pad_i, group=group)
    dist.all_gather(all_v, pad_v, group=group)
    out = np.full(npairs, np.nan)
    for i, v in zip(all_i, all_v):
        keep = i >= 0
        out[i[keep].numpy()] = v[keep].numpy()
    return out
