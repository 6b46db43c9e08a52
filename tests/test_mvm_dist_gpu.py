"""The GPU path of the column-split MVM (maos_b200.mvm_dist) on one rank of
an NCCL process group: the rank's mb_mvm product followed by the all-reduce
equals the FP64 product of the BF16-rounded matrix to 1e-5.  (The split and
the reduction over two ranks are tested on the CPU, test_mvm_dist.py: this
pool gives one GPU per call, and ranks that wait on one another are not run
on one GPU.)"""
import os
import socket

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_column_split_mvm_one_rank_nccl():
    import torch.distributed as dist
    from maos_b200.mvm_dist import DistributedMVM
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("nccl", rank=0, world_size=1, device_id=torch.device("cuda", 0))
    try:
        rng = np.random.default_rng(12)
        nact, ngrad, nb = 401, 3000, 8
        M = rng.standard_normal((nact, ngrad))
        g = rng.standard_normal((nb, ngrad)).astype(np.float32)
        d = DistributedMVM(M, ngrad, nact, nbatch=nb, dtype=1, wfs_offsets=[0, 1000, 2000])
        a = d.apply(torch.tensor(g, device="cuda")).cpu().numpy().astype(np.float64)
        d.close()
        Mr = torch.from_numpy(M).to(torch.bfloat16).to(torch.float64).numpy()
        want = g.astype(np.float64) @ Mr.T
        assert np.linalg.norm(a - want) / np.linalg.norm(want) < 1e-5
        assert d.blocks == [(0, ngrad)]
    finally:
        dist.destroy_process_group()
