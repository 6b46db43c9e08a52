"""Host logic of the control-matrix MVM split over GPUs by gradient columns
(the reference's cuda/mvmfull_iwfs.cu), on the CPU: column blocks that follow
WFS boundaries, and two gloo ranks whose partial products (a NumPy stand-in
for each rank's GPU product) are summed by the all-reduce into M g on every
rank."""
import os

import numpy as np


def test_wfs_blocks_tile_the_columns():
    from maos_b200.mvm_dist import even_column_blocks, wfs_column_blocks
    offs = [0, 5640, 11280, 16920, 22560, 28200]  # six WFS of 5,640 gradients (30 m MCAO)
    for world in (1, 2, 3, 4, 6, 8):
        b = wfs_column_blocks(offs, 33840, world)
        assert len(b) == world and b[0][0] == 0 and b[-1][1] == 33840
        assert all(b[r][1] == b[r + 1][0] for r in range(world - 1))
        # every boundary is a WFS boundary (or the end)
        assert all(c0 in offs + [33840] for c0, _ in b)
    assert wfs_column_blocks(offs, 33840, 2) == [(0, 16920), (16920, 33840)]
    assert wfs_column_blocks(offs, 33840, 3) == [(0, 11280), (11280, 22560), (22560, 33840)]
    e = even_column_blocks(1001, 4)
    assert e[0][0] == 0 and e[-1][1] == 1001 and all(e[r][1] == e[r + 1][0] for r in range(3))


def _worker(rank, world, port, q):
    import torch.distributed as dist
    from maos_b200.mvm_dist import DistributedMVM
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        rng = np.random.default_rng(5)
        nact, ngrad, nb = 37, 300, 3
        M = rng.standard_normal((nact, ngrad)).astype(np.float32)
        g = rng.standard_normal((nb, ngrad)).astype(np.float32)
        offs = [0, 100, 180, 300 - 60]
        holder = {}

        def local(gl):  # this rank's columns only
            c0, c1 = holder["d"].c0, holder["d"].c1
            assert gl.shape == (nb, c1 - c0)
            return gl.astype(np.float64) @ M[:, c0:c1].T.astype(np.float64)

        d = DistributedMVM(None, ngrad, nact, nbatch=nb, wfs_offsets=offs, local_apply=local)
        holder["d"] = d
        a = d.apply(g)
        want = g.astype(np.float64) @ M.T.astype(np.float64)
        q.put((rank, float(np.abs(a - want).max() / np.abs(want).max()), d.blocks))
    finally:
        dist.destroy_process_group()


def test_partial_products_reduce_to_the_whole_product_gloo():
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
    res = {}
    for _ in ps:
        r, err, blocks = q.get(timeout=120)
        res[r] = (err, blocks)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert res[0][1] == res[1][1] == [(0, 180), (180, 300)]
    assert res[0][0] < 1e-6 and res[1][0] < 1e-6
