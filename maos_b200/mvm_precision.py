"""Storage precision of the control-matrix MVM against the reconstruction error.

For a control matrix ``M`` (from :mod:`maos_b200.mvm_build`) and a frozen-flow
gradient sequence, the DM commands ``a = M g`` applied in FP64 on the host are
the reference; the same products from the GPU MVM with FP32, BF16 and
FP8-E4M3 (per-row scale) storage give ``a_dt``.  Errors are measured as
wavefront error on the fit grid in the science direction (fit direction 0),
with the pupil weighting ``W = W0 - W1 W1^T`` of ``lib/mkw.c``:

  residual WFE  = sqrt(<e^T W e>),  e = phi - HA a        (phi: true OPD)
  command error = sqrt(<d^T W d>),  d = HA (a_dt - a)

averaged over the steps.  The reconstruction is open loop (each step's
commands from that step's gradients), so the residual is the tomography +
fitting + noise error of the MVM reconstructor itself.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import native
from .native import check
from .turbulence import DeviceAtmosphere, FrozenFlowAtmosphere

DTYPES = (("fp32", native.MB_MVM_F32), ("bf16", native.MB_MVM_BF16), ("fp8_e4m3", native.MB_MVM_FP8))


def frozen_flow(sysm, fit, nsteps: int, seed: int = 11, dt: float = None, device: str = "cuda"):
    """Gradients [nsteps][ngrad] with noise and the true science OPD on the
    fit grid [nsteps][nfloc] of consecutive frozen-flow steps (sampled on
    `device`, FP64)."""
    import torch
    dt = sysm.cfg.sim_dt if dt is None else dt
    atm = DeviceAtmosphere(FrozenFlowAtmosphere(sysm.cfg, seed), device=device)
    rng = np.random.default_rng(seed + 104729)
    px, py = fit_points(fit)
    fx = torch.as_tensor(px, device=device)
    fy = torch.as_tensor(py, device=device)
    g = np.empty((nsteps, sysm.ngrad))
    phi = np.empty((nsteps, fx.numel()))
    for k in range(nsteps):
        g[k] = atm.gradients(sysm, k * dt, rng, noise=True)
        phi[k] = atm.opd(fx, fy, float(fit.thetax[0]), float(fit.thetay[0]), float(fit.hs[0]),
                         k * dt).cpu().numpy()
    return g, phi


def fit_points(fit):
    """Coordinates of the fit grid's points (a full grid, or the metapupil
    points of the assembled fit)."""
    fl = fit.floc
    if hasattr(fl, "points"):
        return fl.points()
    return ((fl.ox + np.arange(fl.nx) * fl.dx)[None, :].repeat(fl.ny, 0).ravel(),
            (fl.oy + np.arange(fl.ny) * fl.dy)[:, None].repeat(fl.nx, 1).ravel())


def science_HA(fit):
    """The DM-to-fit-grid ray tracing of fit direction 0 (DMs side by side);
    for the assembled fit it includes the extrapolation to weakly coupled
    actuators that maos applies to the commands."""
    import scipy.sparse as sps
    if getattr(fit, "HA0", None) is not None:
        return fit.HA0
    return sps.hstack([fit.HA[0][d] for d in range(len(fit.dms))]).tocsr()


def _wfe(fit, v: np.ndarray) -> np.ndarray:
    """Piston-removed, pupil-weighted RMS of each row of v (same units as v)."""
    q = np.einsum("ij,ij->i", v, (fit.W0 @ v.T).T) - (v @ fit.W1) ** 2
    return np.sqrt(np.maximum(q, 0.0))


def mvm_apply(M: np.ndarray, g: np.ndarray, dtype: int, batch: int = 64) -> np.ndarray:
    """a = M g on the GPU with the given storage type, host FP64 in and out."""
    lib = native.load()
    nact, ngrad = M.shape
    Mc = np.asfortranarray(M, dtype=np.float64)
    h = C.c_void_p()
    check(lib.mb_mvm_create(Mc.ctypes.data_as(C.POINTER(C.c_double)), nact, ngrad, dtype, batch, C.byref(h)),
          "mb_mvm_create")
    out = np.empty((g.shape[0], nact))
    try:
        gb = np.zeros((batch, ngrad))
        ob = np.empty((batch, nact))
        for k0 in range(0, g.shape[0], batch):
            n = min(batch, g.shape[0] - k0)
            gb[:n] = g[k0:k0 + n]
            gb[n:] = 0.0
            check(lib.mb_recon_mvm(h, gb.ctypes.data_as(C.POINTER(C.c_double)),
                                   ob.ctypes.data_as(C.POINTER(C.c_double))), "mb_recon_mvm")
            out[k0:k0 + n] = ob[:n]
    finally:
        lib.mb_mvm_free(h)
    return out


def study(sysm, fit, M: np.ndarray, nsteps: int = 400, seed: int = 11, gate: float = 0.01,
          device: str = "cuda") -> dict:
    """The precision report: residual WFE, each storage type's command error
    (nm RMS and as a fraction of the residual) and whether it is within
    ``gate`` of the residual."""
    g, phi = frozen_flow(sysm, fit, nsteps, seed, device=device)
    HA0 = science_HA(fit)
    a64 = g @ np.asarray(M, dtype=np.float64).T
    res = _wfe(fit, phi - (HA0 @ a64.T).T)
    out = {"steps": int(nsteps), "dt_s": float(sysm.cfg.sim_dt), "shape": [int(M.shape[0]), int(M.shape[1])],
           "residual_wfe_nm": float(np.sqrt(np.mean(res ** 2)) * 1e9), "gate_fraction": gate, "dtypes": {}}
    for name, dt in DTYPES:
        a = mvm_apply(M, g, dt)
        err = _wfe(fit, (HA0 @ (a - a64).T).T)
        e = float(np.sqrt(np.mean(err ** 2)))
        frac = e / math.sqrt(np.mean(res ** 2))
        rel = float(np.linalg.norm(a - a64) / np.linalg.norm(a64))
        out["dtypes"][name] = {"command_error_wfe_nm": e * 1e9, "fraction_of_residual": frac,
                               "relative_command_error": rel, "within_gate": bool(frac <= gate)}
    return out
