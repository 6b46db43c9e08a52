"""The control-matrix MVM split over GPUs by gradient columns.

The reference's multi-GPU MVM (cuda/mvmfull_iwfs.cu:29-31) gives each GPU
the columns of the control matrix that belong to its WFS: every GPU
multiplies its own gradients by its own columns, and one reduction of the
nact-long partial command vectors (per instance) gives the commands.  Here
one process per GPU holds an ``mb_mvm`` of its column block (FP32, BF16 or
FP8 storage, any batch), and the partial commands are summed by one
``torch.distributed`` all-reduce (NCCL between GPUs) of nbatch x nact FP32
values per step; the gradients never leave the GPU that measured them.

The column blocks follow WFS boundaries when the WFS offsets are given (the
reference's split), otherwise equal shares.  The host logic (partition,
reduction, result on every rank) is tested with two gloo ranks on the CPU
and a NumPy stand-in for the local product.
"""
from __future__ import annotations

from typing import Callable, Optional, Sequence

import numpy as np


def wfs_column_blocks(wfs_offsets: Sequence[int], ngrad: int, world: int):
    """[c0, c1) column range of every rank: consecutive WFS per rank, the
    ranks' gradient counts as even as WFS boundaries allow (greedy, in WFS
    order).  wfs_offsets: first gradient of each WFS (ascending, from 0)."""
    off = list(wfs_offsets) + [ngrad]
    nw = len(off) - 1
    if world >= nw:
        blocks = [(off[w], off[w + 1]) for w in range(nw)]
        return blocks + [(ngrad, ngrad)] * (world - nw)
    blocks, w = [], 0
    for r in range(world):
        target = off[w] + (ngrad - off[w]) / (world - r)
        w1 = w + 1
        while w1 < nw - (world - r - 1) and abs(off[w1 + 1] - target) <= abs(off[w1] - target):
            w1 += 1
        if r == world - 1:
            w1 = nw
        blocks.append((off[w], off[w1]))
        w = w1
    return blocks


def even_column_blocks(ngrad: int, world: int):
    """Equal shares of the columns, in order."""
    b = np.linspace(0, ngrad, world + 1).round().astype(int)
    return [(int(b[r]), int(b[r + 1])) for r in range(world)]


class DistributedMVM:
    """a = M g for nbatch instances with M's columns split over the ranks of a
    process group.  M: the full control matrix [nact, ngrad] (each rank keeps
    only its columns) or None with ``local_apply`` given; blocks: the ranks'
    column ranges (default: WFS blocks when wfs_offsets is given, else equal
    shares).  local_apply(g_local) -> partial [nbatch, nact] replaces the
    GPU product (host tests)."""

    def __init__(self, M: Optional[np.ndarray], ngrad: int, nact: int, nbatch: int = 1, dtype: int = 1,
                 wfs_offsets: Optional[Sequence[int]] = None, blocks=None, group=None,
                 local_apply: Optional[Callable] = None, device: Optional[int] = None):
        import torch.distributed as dist
        self.group = group
        self.rank, self.world = dist.get_rank(group), dist.get_world_size(group)
        self.ngrad, self.nact, self.nbatch = int(ngrad), int(nact), int(nbatch)
        if blocks is None:
            blocks = (wfs_column_blocks(wfs_offsets, self.ngrad, self.world) if wfs_offsets is not None
                      else even_column_blocks(self.ngrad, self.world))
        assert len(blocks) == self.world and blocks[0][0] == 0 and blocks[-1][1] == self.ngrad
        assert all(blocks[r][1] == blocks[r + 1][0] for r in range(self.world - 1))
        self.blocks = blocks
        self.c0, self.c1 = blocks[self.rank]
        self._local = local_apply
        if local_apply is None:
            import ctypes as C

            import torch

            from . import native
            self._lib = native.load()
            self._dev = torch.device("cuda", torch.cuda.current_device() if device is None else device)
            Mloc = np.asfortranarray(np.asarray(M, dtype=np.float64)[:, self.c0:self.c1])
            self._h = C.c_void_p()
            if self.c1 > self.c0:
                native.check(self._lib.mb_mvm_create(Mloc.ctypes.data_as(C.POINTER(C.c_double)), self.nact,
                                                     self.c1 - self.c0, int(dtype), self.nbatch, C.byref(self._h)),
                             "mb_mvm_create")
            self._out = torch.zeros(self.nbatch, self.nact, dtype=torch.float32, device=self._dev)

    def apply(self, g):
        """g: this rank's gradients, either the whole [nbatch, ngrad] (the
        rank's columns are taken) or just its block [nbatch, c1 - c0].
        Returns the commands [nbatch, nact] on every rank (a CUDA tensor on
        the GPU path, a NumPy array on the host path)."""
        import torch.distributed as dist
        if self._local is not None:
            import torch
            gl = np.asarray(g)
            if gl.shape[-1] == self.ngrad:
                gl = gl[..., self.c0:self.c1]
            part = torch.from_numpy(np.ascontiguousarray(self._local(gl), dtype=np.float32))
            dist.all_reduce(part, group=self.group)
            return part.numpy()
        import ctypes as C

        import torch

        from .native import check
        if g.shape[-1] == self.ngrad:
            g = g[..., self.c0:self.c1]
        g = g.contiguous()
        s = torch.cuda.current_stream(self._dev)
        if self.c1 > self.c0:
            check(self._lib.mb_mvm_apply_device(self._h, C.c_void_p(g.data_ptr()), C.c_void_p(self._out.data_ptr()),
                                                C.c_void_p(s.cuda_stream)), "mb_mvm_apply_device")
        else:
            self._out.zero_()
        dist.all_reduce(self._out, group=self.group)  # one reduction of nbatch x nact per step
        return self._out

    def close(self):
        h = getattr(self, "_h", None)
        if h:
            self._lib.mb_mvm_free(h)
            self._h = None
