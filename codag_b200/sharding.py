"""Spreading one chunked file over several GPUs (one process per GPU).

Chunks are independent, so a file shards without any exchange: each rank decodes its own
chunks into its own memory.  The shard plan balances algorithmic bytes (compressed bytes
read + decoded bytes written) with longest-processing-time-first assignment: chunks sorted
by cost, each given to the least-loaded rank.  Every rank computes the same plan from the
same metadata, so no plan is sent around.  A consumer that needs the whole decoded file on
one GPU gathers the ranks' chunks once (`gather_to`); nothing else crosses devices.
"""
from __future__ import annotations

import heapq

import numpy as np


def lpt_shards(cost: np.ndarray, n_ranks: int) -> list[np.ndarray]:
    """Chunk indices per rank (each ascending), balancing the sum of `cost`."""
    cost = np.asarray(cost, dtype=np.int64)
    if n_ranks < 1:
        raise ValueError("n_ranks must be positive")
    order = np.argsort(-cost, kind="stable")
    heap = [(0, r) for r in range(n_ranks)]
    owner = np.empty(cost.size, dtype=np.int64)
    for i in order:
        load, r = heapq.heappop(heap)
        owner[i] = r
        heapq.heappush(heap, (load + int(cost[i]), r))
    return [np.nonzero(owner == r)[0] for r in range(n_ranks)]


def chunk_costs(comp_len: np.ndarray, chunk_bytes: int) -> np.ndarray:
    """Algorithmic bytes of each chunk: its stream plus its decoded chunk."""
    return np.asarray(comp_len, dtype=np.int64) + int(chunk_bytes)


def imbalance(cost: np.ndarray, shards: list[np.ndarray]) -> float:
    """max rank load / mean rank load (1.0 = perfect)."""
    loads = np.array([int(np.asarray(cost)[s].sum()) for s in shards], dtype=np.float64)
    return float(loads.max() / max(loads.mean(), 1e-9))


def gather_to(local_out, local_idx: np.ndarray, n_chunks: int, chunk_bytes: int, dst: int = 0, group=None):
    """Collects every rank's decoded chunks on rank `dst` (one gather of padded buffers).

    local_out holds this rank's chunks back to back in `local_idx` order.  Returns the whole
    decoded file (n_chunks * chunk_bytes bytes, chunk i at i * chunk_bytes) on `dst` and
    None elsewhere."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    rank = dist.get_rank(group)
    counts = torch.zeros(world, dtype=torch.int64, device=local_out.device)
    counts[rank] = local_idx.size
    dist.all_reduce(counts, group=group)
    cmax = int(counts.max().item())
    buf = torch.zeros(cmax * chunk_bytes, dtype=torch.uint8, device=local_out.device)
    buf[:local_out.numel()] = local_out
    idx = torch.full((cmax,), -1, dtype=torch.int64, device=local_out.device)
    idx[:local_idx.size] = torch.from_numpy(np.asarray(local_idx, dtype=np.int64)).to(local_out.device)
    bufs = [torch.empty_like(buf) for _ in range(world)] if rank == dst else None
    idxs = [torch.empty_like(idx) for _ in range(world)] if rank == dst else None
    dist.gather(buf, bufs, dst=dst, group=group)
    dist.gather(idx, idxs, dst=dst, group=group)
    if rank != dst:
        return None
    out = torch.empty(n_chunks * chunk_bytes, dtype=torch.uint8, device=local_out.device)
    for b, ix in zip(bufs, idxs):
        for k, c in enumerate(ix.tolist()):
            if c >= 0:
                out[c * chunk_bytes:(c + 1) * chunk_bytes] = b[k * chunk_bytes:(k + 1) * chunk_bytes]
    return out
