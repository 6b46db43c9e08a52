"""The gpu_* glue (maos_b200/glue/maos_gpu_glue.c) builds against the
reference's headers and exports every reconstruction entry point of
cuda/gpu.h that maos calls; and the reference's own top-level CPU tomofit
(maos/recon.c:55), on the RECON_T the glue reads, equals the oracle's
tomography + assembled fit (CPU only)."""
import ctypes
import os
import subprocess

import numpy as np
import pytest

from oracle import refbridge

pytestmark = [pytest.mark.ref,
              pytest.mark.skipif(not (refbridge.available() and os.path.exists(refbridge.GLUE_LIB)),
                                 reason="reference library or glue not built")]

ENTRY_POINTS = ["gpu_init", "gpu_cleanup", "gpu_setup_recon", "gpu_setup_recon_mvm", "gpu_update_recon",
                "gpu_update_recon_cn2", "gpu_recon_reset", "gpu_recon_free", "gpu_tomo", "gpu_fit",
                "gpu_recon_mvm"]


def test_glue_exports_the_recon_entry_points():
    out = subprocess.run(["nm", "-D", "--defined-only", refbridge.GLUE_LIB], capture_output=True, text=True,
                         check=True).stdout
    names = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    missing = [n for n in ENTRY_POINTS if n not in names]
    assert not missing, missing


def test_reference_tomofit_equals_the_oracle():
    from conftest import get_fit_assembled, get_system
    from maos_b200 import turbulence
    from oracle.recon_oracle import SparseFitOracle, TomoOracle, fit_solve, tomo_solve
    s = get_system("ltao_8m")
    fs = get_fit_assembled("ltao_8m")
    frames = turbulence.gradient_frames(s, seed=3, nframe=2)
    with refbridge.RefProcess(nthread=4) as R:
        R.call("setup", refbridge.system_desc(s, split=1))
        R.call("fit_assemble", refbridge.fit_assembled_desc(fs, s.cfg))
        R.call("glue_prepare", 1, s.cfg.tomo_maxit, fs.maxit)
        to, fo = TomoOracle(s), SparseFitOracle(s, fs)
        x = a = None
        for k in range(2):
            got, _ = R.call("glue_cpu_step", frames[k])
            x, _ = tomo_solve(to, frames[k], x0=x)
            a, _ = fit_solve(fo, x, a0=a)
            assert np.linalg.norm(got - a) <= 1e-9 * np.linalg.norm(a)
