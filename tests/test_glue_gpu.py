"""The gpu_* entry points maos links against, driven by those names.

maos_b200/glue/maos_gpu_glue.c implements gpu_init, gpu_setup_recon,
gpu_tomo, gpu_fit, gpu_recon_reset, gpu_setup_recon_mvm and gpu_recon_mvm
(cuda/gpu.h:27-57) on the maos_b200 C ABI.  It is compiled against the
reference's own headers and loaded, with the reference's own library, in the
reference worker process (oracle/refbridge.py), where the reference's setup
path (oracle/ref/ref_driver.c) has built PARMS_T / RECON_T / POWFS_T / SIM_T.

The DM commands of gpu_tomo + gpu_fit over three warm-started steps are
compared with the reference's own CPU tomofit (maos/recon.c:55: muv_solve on
RL/RR with the FDPCG or no preconditioner, then muv_solve on FL/FR) on the
same gradient cells, with the same iteration counts: relative L2 <= 1e-4
(the FP32 tolerance of the DM-command gate).  gpu_recon_mvm is compared with
the FP64 product of the same control matrix: 1e-5.
"""
import numpy as np
import pytest

from oracle import refbridge

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not (refbridge.available() and __import__("os").path.exists(refbridge.GLUE_LIB)),
                                 reason="reference library or glue not built")]

SOLVE_TOL = 1e-4
MVM_TOL = 1e-5


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(b))


@pytest.mark.parametrize("name,gpu_fit", [("ltao_8m", 1), ("mcao_30m", 1), ("ltao_8m", 2)])
def test_gpu_entry_points_match_reference_tomofit(name, gpu_fit):
    from conftest import get_fit, get_fit_assembled, get_system
    from maos_b200 import turbulence
    s = get_system(name)
    with refbridge.RefProcess(nthread=8) as R:
        R.call("setup", refbridge.system_desc(s, split=1))
        if s.cfg.tomo_precond == 1:
            R.call("fdpcg_set", s.fdpcg.Mbinv, s.fdpcg.perm, s.fdpcg.scale)
        if gpu_fit == 1:  # the assembled fit, maos's default
            fs = get_fit_assembled(name)
            R.call("fit_assemble", refbridge.fit_assembled_desc(fs, s.cfg))
        else:             # the grid fit with its slaving term
            fs = get_fit(name)
            R.call("fit_setup", refbridge.fit_desc(fs))
            R.call("fit_setup_slave", s.cfg.fit_actthres)
        R.call("glue_prepare", gpu_fit, s.cfg.tomo_maxit, fs.maxit)
        R.call("glue_setup")
        frames = turbulence.gradient_frames(s, seed=3, nframe=3)
        for k in range(3):
            a_gpu = R.call("glue_step", frames[k])
            a_cpu, _ = R.call("glue_cpu_step", frames[k])
            assert a_gpu.shape == a_cpu.shape
            assert rel(a_gpu, a_cpu) < SOLVE_TOL, (k, rel(a_gpu, a_cpu))
        # gpu_recon_reset restarts cold: the first step again
        R.call("glue_reset")
        a0 = R.call("glue_step", frames[0])
        rng = np.random.default_rng(9)
        M = rng.standard_normal((len(a0), s.ngrad)) * 1e-3
        g = frames[1]
        got = R.call("glue_mvm", M, g)
        assert rel(got, M @ g) < MVM_TOL
        R.call("glue_cleanup")
