"""One batched reconstruction step of a preset, for profilers.

    python -m maos_b200.profile_step [--system mcao_30m] [--batch 32] [--steps 1]
    python -m maos_b200.profile_step --mvm bf16 [--batch 32] [--steps 1]
    python -m maos_b200.profile_step --wfs [--system mcao_30m] [--batch 8] [--steps 1]
    python -m maos_b200.profile_step --stages [--system mcao_30m] [--batch 1]

Builds the system, sets up a reconstructor with the DM fit for `batch`
instances and runs `steps` graph steps on random gradients; prints "ok".
Under ncu, each step's kernels appear in order: k_gp, k_pupil_rows (right-hand
side), k_hxt_rows, then per FDPCG iteration k_pupil_rows, k_hxt_rows,
k_fd_fwd, k_fd_mul, k_fd_inv, k_cg_update_p, then the fit.

With --wfs, the system's geometric WFS (every WFS, its atmosphere and DMs,
noise on) runs `steps` times for `batch` instances instead (k_wfs_geom).

The DM fit is the assembled one (the reference default) unless --fit grid.
With --stages, the step is timed with CUDA events over 50 graph launches
and every kernel of a CG iteration is timed alone (mb_time_stages); the
times are printed.

With --mvm, a random control matrix of the system's shape (nact x ngrad) is
installed in that storage type and `steps` batched MVMs are applied instead
(k_gsplit, k_mvm_tc, k_mvm_reduce for BF16/FP8 at 4 or more instances).
"""
from __future__ import annotations

import argparse


def main():
    import torch
    from . import config, fit_assemble, fit_setup, geometry
    from .recon import Reconstructor
    ap = argparse.ArgumentParser()
    ap.add_argument("--system", default="mcao_30m", choices=sorted(config.PRESETS))
    ap.add_argument("--batch", type=int, default=32)
    ap.add_argument("--steps", type=int, default=1)
    ap.add_argument("--mvm", choices=["fp32", "bf16", "fp8"], default=None)
    ap.add_argument("--wfs", action="store_true")
    ap.add_argument("--fit", choices=["assembled", "grid"], default="assembled")
    ap.add_argument("--stages", action="store_true")
    ap.add_argument("--fdpcg-mode", type=int, default=1, choices=[0, 1, 2],
                    help="form of the FDPCG preconditioner (mb_fdpcg_mode) for the plain steps")
    a = ap.parse_args()
    s = geometry.build_tomo(config.PRESETS[a.system]())
    fs = fit_setup.build_fit(s) if (a.fit == "grid" or a.wfs) else fit_assemble.build_fit_assembled(s)
    if a.wfs:
        from .turbulence import FrozenFlowAtmosphere
        from .wfs import GeomWfs
        W = GeomWfs.for_system(s, FrozenFlowAtmosphere(s.cfg, 1), fit=fs, nbatch=a.batch)
        dm = torch.randn(a.batch, W.nact, device="cuda") * 1e-7
        for k in range(a.steps):
            W.grad(k, dm=dm, seed=1)
        torch.cuda.synchronize()
        W.close()
        print("ok")
        return
    if a.mvm:
        import ctypes as C
        import numpy as np
        from . import native
        lib = native.load()
        M = np.asfortranarray(np.random.default_rng(0).standard_normal((int(fs.nact), int(s.ngrad))))
        h = C.c_void_p()
        native.check(lib.mb_mvm_create(M.ctypes.data_as(C.POINTER(C.c_double)), M.shape[0], M.shape[1],
                                       ["fp32", "bf16", "fp8"].index(a.mvm), a.batch, C.byref(h)), "mb_mvm_create")
        del M
        g = torch.randn(a.batch * s.ngrad, device="cuda")
        out = torch.empty(a.batch * int(fs.nact), device="cuda")
        st = torch.cuda.Stream()
        for _ in range(a.steps):
            native.check(lib.mb_mvm_apply_device(h, C.c_void_p(g.data_ptr()), C.c_void_p(out.data_ptr()),
                                                 C.c_void_p(st.cuda_stream)), "mb_mvm_apply_device")
        torch.cuda.synchronize()
        lib.mb_mvm_free(h)
        print("ok")
        return
    R = Reconstructor(s, nbatch=a.batch, fit=fs)
    g = torch.randn(a.batch * s.ngrad, device="cuda") * 1e-6
    st = torch.cuda.Stream()
    if a.stages:
        import ctypes as C
        from . import native
        rows, _ = R.autotune(reps=20)
        for _ in range(5):
            R.step_device(g.data_ptr(), st.cuda_stream)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(st):
            e0.record(st)
            for _ in range(50):
                R.step_device(g.data_ptr(), st.cuda_stream)
            e1.record(st)
        torch.cuda.synchronize()
        lib = R.lib
        lib.mb_kernel_launches(1)
        R.step_device(g.data_ptr(), st.cuda_stream)
        torch.cuda.synchronize()
        nk = lib.mb_kernel_launches(1)
        print(f"{a.system} batch {a.batch} fit {a.fit}: step {e0.elapsed_time(e1) / 50:.4f} ms, {nk} kernels, "
              f"pupil rows {rows}, fdpcg form {lib.mb_fdpcg_mode(R.h, -1) if s.fdpcg is not None else 0}")
        if s.fdpcg is not None:
            for mode in (1, 2):
                got = R.fdpcg_mode(mode)
                for _ in range(3):
                    R.step_device(g.data_ptr(), st.cuda_stream)
                with torch.cuda.stream(st):
                    e0.record(st)
                    for _ in range(50):
                        R.step_device(g.data_ptr(), st.cuda_stream)
                    e1.record(st)
                torch.cuda.synchronize()
                print(f"  fdpcg form {got}: step {e0.elapsed_time(e1) / 50:.4f} ms")
        ns = lib.mb_num_stages()
        ms, by, lp = (C.c_float * ns)(), (C.c_double * ns)(), (C.c_int * ns)()
        native.check(lib.mb_time_stages(R.h, 50, ms, by, lp), "mb_time_stages")
        for i in range(ns):
            print(f"  {lib.mb_stage_name(i).decode():14s} {ms[i] * 1000:8.2f} us x {lp[i]:3d} = "
                  f"{ms[i] * lp[i]:.4f} ms")
        R.close()
        return
    if s.fdpcg is not None:
        R.fdpcg_mode(a.fdpcg_mode)
    for _ in range(a.steps):
        R.step_device(g.data_ptr(), st.cuda_stream)
    torch.cuda.synchronize()
    R.close()
    print("ok")


if __name__ == "__main__":
    main()
