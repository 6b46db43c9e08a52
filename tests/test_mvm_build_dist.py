"""Host logic of the multi-GPU control-matrix build, on the CPU.

Two gloo ranks each fill their shard of a known matrix (column c holds the
value c + 1000 * row) and gather it; every rank must end up with the whole
matrix, and the shards must tile the columns exactly once in whole blocks.
"""
import os

import numpy as np
import pytest


def test_shards_tile_columns():
    from maos_b200.mvm_build import column_shard
    for ngrad in (1, 255, 256, 257, 2656, 33840):
        for world in (1, 2, 3, 8):
            cols = np.concatenate([column_shard(ngrad, r, world) for r in range(world)])
            assert np.array_equal(cols, np.arange(ngrad))
            for r in range(world):
                c = column_shard(ngrad, r, world)
                assert len(c) == 0 or (c[0] % 256 == 0)


def _worker(rank, world, port, q):
    import torch.distributed as dist
    from maos_b200.mvm_build import column_shard, gather_columns
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        ngrad, nact = 1000, 7
        cols = column_shard(ngrad, rank, world, block=128)
        local = (cols[None, :] + 1000.0 * np.arange(nact)[:, None]).astype(np.float32)
        M = gather_columns(local, ngrad, block=128)
        want = (np.arange(ngrad)[None, :] + 1000.0 * np.arange(nact)[:, None]).astype(np.float32)
        q.put((rank, bool(np.array_equal(M, want))))
    finally:
        dist.destroy_process_group()


def test_gather_two_ranks_gloo():
    import multiprocessing as mp
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = dict(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res == {0: True, 1: True}
