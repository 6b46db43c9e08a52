"""Control-matrix build on the GPU: many right-hand sides through the same
tomography + fit operators at once.

The reference assembles its MVM control matrix by solving the tomography and
fit normal equations for every gradient (``maos/setup_recon_mvm.c:115-229``;
on the GPU ``cuda/mvm_trans.cu:46-360``), with the iteration counts raised well
above the per-step ones so that the result approximates the converged linear
operator ``M = FitL^-1 FitR TomoL^-1 TomoR``.  Here column ``c`` of ``M`` is the
DM command vector that a cold-started reconstruction step returns for the
unit gradient ``e_c``; ``rhs_batch`` columns run as the instances of one
batched reconstructor (shared operator tables, one CUDA graph per batch).
FP32 arithmetic with FP64 CG scalars, like every solve in this package.
"""
from __future__ import annotations

import dataclasses
import time
from typing import Optional

import numpy as np

from .native import check


def build_control_matrix(sysm, fit, rhs_batch: int = 256, tomo_maxit: Optional[int] = None,
                         fit_maxit: Optional[int] = None, columns=None, device: int = 0,
                         scale: float = 1e-6):
    """M (nact x ngrad, FP32) and a report dict.

    ``columns``: gradient indices to build (default: all, giving the whole
    matrix); the returned array then has one column per requested index.
    ``scale``: size of the unit gradient actually applied (the result is
    divided by it), keeping the solves in the usual FP32 range."""
    import torch
    from .recon import Reconstructor
    tomo_maxit = int(tomo_maxit or 10 * sysm.cfg.tomo_maxit)
    fs = dataclasses.replace(fit, maxit=int(fit_maxit or 10 * fit.maxit))
    ngrad, nact = int(sysm.ngrad), int(fs.nact)
    cols = np.arange(ngrad) if columns is None else np.asarray(columns, dtype=np.int64)
    B = int(min(rhs_batch, len(cols)))
    R = Reconstructor(sysm, nbatch=B, maxit=tomo_maxit, fit=fs, device=device)
    out = np.empty((nact, len(cols)), dtype=np.float32)
    stream = torch.cuda.Stream(device=device)
    g = torch.zeros((B, ngrad), dtype=torch.float32, device=f"cuda:{device}")
    a = torch.empty((B, nact), dtype=torch.float32, device=f"cuda:{device}")
    worst = 0.0
    t0 = time.perf_counter()
    try:
        for c0 in range(0, len(cols), B):
            n = min(B, len(cols) - c0)
            with torch.cuda.stream(stream):
                g.zero_()
                rows = torch.arange(n, device=g.device)
                g[rows, torch.as_tensor(cols[c0:c0 + n], device=g.device)] = scale
            stream.synchronize()
            check(R.lib.mb_recon_reset(R.h), "mb_recon_reset")
            R.step_device(g.data_ptr(), stream.cuda_stream)
            stream.synchronize()
            a.copy_(torch.as_tensor(_DeviceArray(R.fit_solution_ptr(), (B, nact)), device=g.device))
            torch.cuda.synchronize(device)
            out[:, c0:c0 + n] = (a[:n].cpu().numpy().T / scale)
            worst = max(worst, float(np.max(R.residual()[:n])))
    finally:
        R.close()
    report = {"columns": int(len(cols)), "rhs_batch": B, "tomo_maxit": tomo_maxit, "fit_maxit": fs.maxit,
              "max_tomo_residual": worst, "seconds": time.perf_counter() - t0}
    return out, report


class _DeviceArray:
    """A library-owned FP32 device array, seen through the CUDA array interface."""

    def __init__(self, ptr: int, shape):
        self.__cuda_array_interface__ = {"shape": tuple(shape), "typestr": "<f4", "data": (int(ptr), False),
                                         "version": 3}


def column_shard(ngrad: int, rank: int, world: int, block: int = 256):
    """Gradient indices this rank builds: whole RHS blocks, dealt out in
    contiguous runs (rank r gets blocks [r*nblk/world, (r+1)*nblk/world))."""
    nblk = (ngrad + block - 1) // block
    b0, b1 = rank * nblk // world, (rank + 1) * nblk // world
    return np.arange(b0 * block, min(b1 * block, ngrad), dtype=np.int64)


def gather_columns(local: np.ndarray, ngrad: int, group=None, block: int = 256) -> np.ndarray:
    """Assemble the full matrix on every rank from each rank's column shard
    (one all_gather of equal-size padded slabs; NCCL over NVLink between GPUs,
    gloo on the host)."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group)
    nact = local.shape[0]
    width = max(len(column_shard(ngrad, r, world, block)) for r in range(world))
    backend = dist.get_backend(group)
    dev = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    slab = torch.zeros((nact, width), dtype=torch.float32, device=dev)
    slab[:, :local.shape[1]] = torch.as_tensor(local, device=dev)
    parts = [torch.empty_like(slab) for _ in range(world)]
    dist.all_gather(parts, slab, group=group)
    out = np.empty((nact, ngrad), dtype=np.float32)
    for r in range(world):
        cols = column_shard(ngrad, r, world, block)
        out[:, cols] = parts[r][:, :len(cols)].cpu().numpy()
    return out


def build_control_matrix_distributed(sysm, fit, rhs_batch: int = 256, group=None, **kw):
    """The control matrix built by all ranks of the process group, each on its
    own GPU with its own share of the unit gradients (no data exchange until
    the final gather).  Returns (M on every rank, this rank's report)."""
    import torch.distributed as dist
    rank, world = dist.get_rank(group), dist.get_world_size(group)
    cols = column_shard(int(sysm.ngrad), rank, world, rhs_batch)
    local, rep = build_control_matrix(sysm, fit, rhs_batch=rhs_batch, columns=cols, **kw)
    return gather_columns(local, int(sysm.ngrad), group, rhs_batch), rep


def main():
    """python -m maos_b200.mvm_build [--system elt_39m] [--rhs-batch 256]
    Builds the whole control matrix of a preset on GPU 0 and prints the
    report (columns, seconds, columns per second, worst tomography residual)
    as one JSON line."""
    import argparse
    import json
    from . import config, fit_assemble, geometry
    ap = argparse.ArgumentParser()
    ap.add_argument("--system", default="elt_39m", choices=sorted(config.PRESETS))
    ap.add_argument("--rhs-batch", type=int, default=256)
    a = ap.parse_args()
    sysm = geometry.build_tomo(config.PRESETS[a.system]())
    fit = fit_assemble.build_fit_assembled(sysm)
    M, rep = build_control_matrix(sysm, fit, rhs_batch=a.rhs_batch)
    rep.update({"system": a.system, "shape": list(M.shape), "ngrad": int(sysm.ngrad),
                "columns_per_s": rep["columns"] / rep["seconds"],
                "finite": bool(np.isfinite(M).all())})
    print(json.dumps(rep))


if __name__ == "__main__":
    main()
