"""One batched reconstruction step of a preset, for profilers.

    python -m maos_b200.profile_step [--system mcao_30m] [--batch 32] [--steps 1]

Builds the system, sets up a reconstructor with the DM fit for `batch`
instances and runs `steps` graph steps on random gradients; prints "ok".
Under ncu, each step's kernels appear in order: k_gp, k_pupil_rows (right-hand
side), k_hxt_rows, then per FDPCG iteration k_pupil_rows, k_hxt_rows,
k_fd_fwd, k_fd_mul, k_fd_inv, k_cg_update_p, then the fit.
"""
from __future__ import annotations

import argparse


def main():
    import torch
    from . import config, fit_setup, geometry
    from .recon import Reconstructor
    ap = argparse.ArgumentParser()
    ap.add_argument("--system", default="mcao_30m", choices=sorted(config.PRESETS))
    ap.add_argument("--batch", type=int, default=32)
    ap.add_argument("--steps", type=int, default=1)
    a = ap.parse_args()
    s = geometry.build_tomo(config.PRESETS[a.system]())
    fs = fit_setup.build_fit(s)
    R = Reconstructor(s, nbatch=a.batch, fit=fs)
    g = torch.randn(a.batch * s.ngrad, device="cuda") * 1e-6
    st = torch.cuda.Stream()
    for _ in range(a.steps):
        R.step_device(g.data_ptr(), st.cuda_stream)
    torch.cuda.synchronize()
    R.close()
    print("ok")


if __name__ == "__main__":
    main()
