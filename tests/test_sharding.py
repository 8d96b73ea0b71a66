"""Sharding a chunked file over ranks: the plan on the CPU, and the multi-rank path (plan on
every rank, local decode, one gather to rank 0) as two gloo processes on the CPU, with the
oracle standing in for each rank's GPU decode."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from codag_b200 import sharding


def test_lpt_covers_every_chunk_once_and_balances():
    rng = np.random.default_rng(1)
    cost = rng.integers(1000, 200_000, 5000)
    for n in (1, 2, 3, 8):
        shards = sharding.lpt_shards(cost, n)
        allidx = np.sort(np.concatenate(shards))
        assert np.array_equal(allidx, np.arange(cost.size))
        assert all(np.all(np.diff(s) > 0) for s in shards)
        assert sharding.imbalance(cost, shards) < 1.01


def test_lpt_is_deterministic_and_handles_more_ranks_than_chunks():
    cost = np.array([5, 5, 5])
    a = sharding.lpt_shards(cost, 5)
    b = sharding.lpt_shards(cost, 5)
    assert all(np.array_equal(x, y) for x, y in zip(a, b))
    assert sum(s.size for s in a) == 3 and sum(s.size == 0 for s in a) == 2


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    from codag_b200 import native
    from oracle import oracle_py
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        ch = 131072
        col = native.gen_rlev2_column(40 * ch // 8, 77, 8)  # the same file on every rank
        comp, off, ln = native.encode_rlev2(col, ch, 8)
        n = ln.size
        shards = sharding.lpt_shards(sharding.chunk_costs(ln, ch), world)
        mine = shards[rank]
        out = np.zeros(mine.size * ch, np.uint8)
        st = oracle_py.decode_batch(comp, off[mine], ln[mine], out, np.arange(mine.size, dtype=np.uint64) * ch,
                                    [ch] * mine.size, [ch] * mine.size, [1] * mine.size, [8] * mine.size,
                                    [0] * mine.size)
        assert not st.any()
        full = sharding.gather_to(torch.from_numpy(out), mine, n, ch, dst=0)
        if rank == 0:
            ok = np.array_equal(full.numpy()[:col.size], col.view(np.uint8))
            q.put((ok, [s.size for s in shards]))
    finally:
        dist.destroy_process_group()


def test_two_rank_shard_decode_and_gather(oracle, native):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    ok, sizes = q.get(timeout=10)
    assert ok and sum(sizes) == 64 and min(sizes) > 0
