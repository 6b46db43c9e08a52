"""Host-side mirror of the reference's GPU reconstruction interface.

``Reconstructor`` wraps one ``mb_recon`` handle.  Its methods follow the
entry points of ``cuda/gpu.h`` that ``maos/recon.c`` and ``maos/sim.c`` call:

=====================  ==========================================
reference (cuda/gpu.h)  here
=====================  ==========================================
gpu_setup_recon        ``Reconstructor(system, nbatch=...)``
gpu_update_recon       ``update_nea(iwfs, neai, ptt)``
gpu_update_recon_cn2   ``update_cn2(l2c, fdpcg)``
gpu_recon_reset        ``reset()``
gpu_tomo               ``tomo(grad)`` -> (opdr, cgres)
gpu_fit                ``fit()`` -> (dmfit, cgres)
gpu_recon_free         ``close()``
=====================  ==========================================

Argument meaning and units are the reference's (gradients in radians, x then
y per WFS; OPD in metres).  Errors raise :class:`maos_b200.native.MbError`.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import native
from .native import (MbCsc, MbFdpcgDesc, MbFdpcgGeom, MbFitDesc, MbFitSparseDesc, MbGrid, MbReconDesc,
                     MbWfsDesc, check)


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _grid(g) -> MbGrid:
    return MbGrid(int(g.nx), int(g.ny), float(g.dx), float(g.dy), float(g.ox), float(g.oy),
                  float(getattr(g, "ht", 0.0)))


def fdpcg_desc(fd, keep: list) -> MbFdpcgDesc:
    perm = np.ascontiguousarray(fd.perm, dtype=np.int64)
    # column-major complex blocks, interleaved re/im
    mb = np.ascontiguousarray(fd.Mbinv.transpose(0, 2, 1)).ravel()
    mbi = np.empty(mb.size * 2)
    mbi[0::2] = mb.real
    mbi[1::2] = mb.imag
    keep += [perm, mbi]
    md = mg = C.POINTER(C.c_double)()
    if getattr(fd, "mhat_data", None) is not None and getattr(fd, "mhat_diag", None) is not None:
        d = np.ascontiguousarray(fd.mhat_data.transpose(0, 2, 1)).ravel()
        mdi = np.empty(d.size * 2)
        mdi[0::2] = d.real
        mdi[1::2] = d.imag
        mgd = np.ascontiguousarray(fd.mhat_diag, dtype=np.float64).ravel()
        keep += [mdi, mgd]
        md, mg = _dptr(mdi), _dptr(mgd)
    gp = C.POINTER(MbFdpcgGeom)()
    g = getattr(fd, "geom", None)
    if g is not None and mg:
        def cplx(a):
            a = np.ascontiguousarray(a, dtype=np.complex128).ravel()
            o = np.empty(2 * a.size)
            o[0::2] = a.real
            o[1::2] = a.imag
            keep.append(o)
            return _dptr(o)
        sel = sorted(g["sel"].items())
        sdx = np.ascontiguousarray([k[0] for k, _ in sel], dtype=np.int32)
        sdy = np.ascontiguousarray([k[1] for k, _ in sel], dtype=np.int32)
        neam = np.ascontiguousarray(g["neam"], dtype=np.float64)
        keep += [sdx, sdy, neam]
        geo = MbFdpcgGeom(int(g["nxp"]), int(g["nyp"]), float(g["dxp"]), int(g["pos"]), int(g["adimx"]),
                          int(g["adimy"]), cplx(g["gx"]), cplx(g["gy"]), len(sel),
                          sdx.ctypes.data_as(C.POINTER(C.c_int)), sdy.ctypes.data_as(C.POINTER(C.c_int)),
                          cplx([v for _, v in sel]), int(g["needscale"]), _dptr(neam))
        keep.append(geo)
        gp = C.pointer(geo)
    return MbFdpcgDesc(int(fd.nb), int(fd.bs), int(fd.scale),
                       perm.ctypes.data_as(C.POINTER(C.c_long)), _dptr(mbi), md, mg, gp)


def csc_desc(A, keep: list) -> MbCsc:
    """A scipy sparse matrix as an ``mb_csc`` (compressed sparse column)."""
    if A is None:
        return MbCsc()
    A = A.tocsc()
    A.sort_indices()
    p = np.ascontiguousarray(A.indptr, dtype=np.int32)
    i = np.ascontiguousarray(A.indices, dtype=np.int32)
    x = np.ascontiguousarray(A.data, dtype=np.float64)
    keep += [p, i, x]
    return MbCsc(int(A.shape[0]), int(A.shape[1]), p.ctypes.data_as(C.POINTER(C.c_int)),
                 i.ctypes.data_as(C.POINTER(C.c_int)), _dptr(x))


def fit_sparse_desc(sf, keep: list) -> MbFitSparseDesc:
    """Flatten a :class:`maos_b200.fit_assemble.SparseFit` (FR, FL) into an
    ``mb_fit_sparse_desc``."""
    cols = []
    for a in (sf.FRU, sf.FRV, sf.FLU, sf.FLV):
        c = np.ascontiguousarray(np.asarray(a, dtype=np.float64).ravel(order="F"))
        keep.append(c)
        cols.append(c)
    return MbFitSparseDesc(csc_desc(sf.FRM, keep), int(sf.FRU.shape[1]), _dptr(cols[0]), _dptr(cols[1]),
                           csc_desc(sf.FLM, keep), int(sf.FLU.shape[1]), _dptr(cols[2]), _dptr(cols[3]),
                           int(sf.maxit))


def fit_desc(fs, keep: list) -> MbFitDesc:
    """Flatten a :class:`maos_b200.fit_setup.FitSystem` into an ``mb_fit_desc``."""
    W0 = fs.W0.tocsc()
    W0.sort_indices()
    arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in
            (fs.thetax, fs.thetay, fs.wt, fs.hs, W0.data, fs.W1)]
    w0p = np.ascontiguousarray(W0.indptr, dtype=np.int32)
    w0i = np.ascontiguousarray(W0.indices, dtype=np.int32)
    am = (MbGrid * len(fs.dms))(*[_grid(d.amap) for d in fs.dms])
    nw = np.ascontiguousarray(fs.NW.ravel(order="F"), dtype=np.float64)
    keep += arrs + [w0p, w0i, am, nw]
    return MbFitDesc(_grid(fs.floc), len(fs.thetax), _dptr(arrs[0]), _dptr(arrs[1]), _dptr(arrs[2]),
                     _dptr(arrs[3]), w0p.ctypes.data_as(C.POINTER(C.c_int)),
                     w0i.ctypes.data_as(C.POINTER(C.c_int)), _dptr(arrs[4]), _dptr(arrs[5]),
                     len(fs.dms), am, int(fs.NW.shape[1]), _dptr(nw), int(fs.maxit),
                     csc_desc(getattr(fs, "actslave", None), keep))


def tomo_desc(sysm, nbatch: int = 1, split: int = 1, maxit: Optional[int] = None, fit=None):
    """Flatten a :class:`maos_b200.geometry.TomoSystem` (and optionally a
    :class:`maos_b200.fit_setup.FitSystem`) into an ``mb_recon_desc``.

    Returns (desc, keep) -- ``keep`` holds the numpy arrays the descriptor
    points into and must outlive the setup call."""
    keep = []
    cfg = sysm.cfg
    xm = (MbGrid * len(sysm.xmaps))(*[_grid(g) for g in sysm.xmaps])
    l2c = np.ascontiguousarray(sysm.l2c, dtype=np.float64)
    keep += [xm, l2c]
    ws = (MbWfsDesc * len(sysm.wfs))()
    gp_cache = {}
    for i, w in enumerate(sysm.wfs):
        key = id(w.GP)
        if key not in gp_cache:
            G = w.GP.tocsc()
            G.sort_indices()
            arrs = (np.ascontiguousarray(w.salocx, dtype=np.float64),
                    np.ascontiguousarray(w.salocy, dtype=np.float64),
                    np.ascontiguousarray(G.indptr, dtype=np.int32),
                    np.ascontiguousarray(G.indices, dtype=np.int32),
                    np.ascontiguousarray(G.data, dtype=np.float64))
            gp_cache[key] = arrs
            keep += list(arrs)
        sx, sy, gpp, gpi, gpx = gp_cache[key]
        neai = np.zeros((w.nsa, 3))
        neai[:, 0] = w.saneai[:w.nsa]
        neai[:, 1] = w.saneai[w.nsa:]
        neai = np.ascontiguousarray(neai.ravel())
        keep.append(neai)
        ptt = None
        if w.PTT is not None:
            ptt = np.ascontiguousarray(w.PTT.ravel(order="F"))
            keep.append(ptt)
        ws[i] = MbWfsDesc(float(w.thetax), float(w.thetay), float(w.hs), int(w.nsa), float(w.dsa),
                          _dptr(sx), _dptr(sy), gpp.ctypes.data_as(C.POINTER(C.c_int)),
                          gpi.ctypes.data_as(C.POINTER(C.c_int)), _dptr(gpx), _dptr(neai),
                          _dptr(ptt) if ptt is not None else C.POINTER(C.c_double)())
    keep.append(ws)
    fdp = C.POINTER(MbFdpcgDesc)()
    if cfg.tomo_precond == 1:
        fd = fdpcg_desc(sysm.fdpcg, keep)
        keep.append(fd)
        fdp = C.pointer(fd)
    fitp = C.POINTER(MbFitDesc)()
    fsp = C.POINTER(MbFitSparseDesc)()
    if fit is not None and hasattr(fit, "FLM"):   # the assembled fit (maos_b200.fit_assemble)
        fd = fit_sparse_desc(fit, keep)
        keep.append(fd)
        fsp = C.pointer(fd)
    elif fit is not None:                         # the grid-form fit (maos_b200.fit_setup)
        fd = fit_desc(fit, keep)
        keep.append(fd)
        fitp = C.pointer(fd)
    d = MbReconDesc(_grid(sysm.pmap), len(sysm.xmaps), xm, _dptr(l2c), len(sysm.wfs), ws,
                    int(cfg.tomo_maxit if maxit is None else maxit), int(cfg.tomo_precond),
                    int(split), fdp, int(nbatch), fitp, fsp)
    return d, keep


class Reconstructor:
    """One tomography reconstructor (``curecon_t``) on the current GPU."""

    def __init__(self, sysm, nbatch: int = 1, split: int = 1, maxit: Optional[int] = None,
                 device: int = 0, fit=None):
        self.lib = native.load()
        check(self.lib.mb_init(device), "mb_init")
        self.sys = sysm
        self.fit_sys = fit
        self.nbatch = nbatch
        self.device = int(device)
        d, keep = tomo_desc(sysm, nbatch=nbatch, split=split, maxit=maxit, fit=fit)
        h = C.c_void_p()
        check(self.lib.mb_setup_recon(C.byref(d), C.byref(h)), "mb_setup_recon")
        self.h = h
        self.ngrad = int(self.lib.mb_ngrad(h))
        self.nxtot = int(self.lib.mb_nxtot(h))
        self.nact = int(self.lib.mb_nact(h))

    def close(self):
        if getattr(self, "h", None):
            self.lib.mb_recon_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _vec(self, a, n):
        a = np.ascontiguousarray(a, dtype=np.float64).reshape(self.nbatch, n)
        return a

    def autotune(self, reps: int = 20):
        """Pick the fastest pupil-row blocking for this batch (mb_autotune);
        returns (rows kept, {rows: ms per operator})."""
        rows = C.c_int()
        ms = (C.c_float * 3)()
        check(self.lib.mb_autotune(self.h, int(reps), C.byref(rows), ms), "mb_autotune")
        return rows.value, {r: ms[i] for i, r in enumerate((4, 8, 16)) if ms[i] >= 0}

    def fdpcg_mode(self, mode: int) -> int:
        """Form of the FDPCG preconditioner in the CG step (mb_fdpcg_mode):
        1 three kernels, 2 one fused cluster kernel, 0 the fused one when it
        fits; returns the form in use."""
        rc = self.lib.mb_fdpcg_mode(self.h, int(mode))
        if rc < 0:
            check(rc, "mb_fdpcg_mode")
        return rc

    def fdpcg_shape(self, ni: int = -1) -> int:
        """Instances per block-solve CTA of the three-kernel FDPCG form
        (mb_fdpcg_shape): 2, 4, 8 or 16, -1 to query; returns the shape in use."""
        rc = self.lib.mb_fdpcg_shape(self.h, int(ni))
        if rc < 0:
            check(rc, "mb_fdpcg_shape")
        return rc

    def reset(self):
        check(self.lib.mb_recon_reset(self.h), "mb_recon_reset")

    def tomo(self, grad):
        g = self._vec(grad, self.ngrad)
        x = np.empty((self.nbatch, self.nxtot))
        res = np.empty(self.nbatch, dtype=np.float32)
        check(self.lib.mb_tomo(self.h, _dptr(g), _dptr(x), res.ctypes.data_as(C.POINTER(C.c_float))),
              "mb_tomo")
        return x, res

    def tomo_only(self, grad):
        """gpu_tomo without copying the layer OPD back (the fit reads it on the device)."""
        g = self._vec(grad, self.ngrad)
        check(self.lib.mb_tomo(self.h, _dptr(g), C.POINTER(C.c_double)(), C.POINTER(C.c_float)()),
              "mb_tomo")

    def fit(self):
        """gpu_fit: DM fit of the current tomography solution -> (dmfit, cgres)."""
        a = np.empty((self.nbatch, self.nact))
        res = np.empty(self.nbatch, dtype=np.float32)
        check(self.lib.mb_fit(self.h, _dptr(a), res.ctypes.data_as(C.POINTER(C.c_float))), "mb_fit")
        return a, res

    def step_device(self, d_grad_ptr: int, stream_ptr: int = 0):
        """Tomography + fit of one step on the device (one graph launch)."""
        check(self.lib.mb_recon_step_device(self.h, C.c_void_p(d_grad_ptr), C.c_void_p(stream_ptr)),
              "mb_recon_step_device")

    def fit_solution_ptr(self) -> int:
        return int(self.lib.mb_fit_solution(self.h))

    def fit_solution(self):
        """The fit's DM commands of every instance as a torch CUDA float32
        view [nbatch, nact] of the reconstructor's own buffer (no copy; valid
        until the next step overwrites it or the reconstructor is closed)."""
        import torch
        ptr = self.fit_solution_ptr()
        if not ptr:
            raise RuntimeError("reconstructor has no DM fit")

        class _View:
            __cuda_array_interface__ = {"shape": (self.nbatch, self.nact), "typestr": "<f4",
                                        "data": (ptr, False), "version": 2, "strides": None}
        return torch.as_tensor(_View(), device=f"cuda:{self.device}")

    # serving: instances as slots (no counterpart in the reference)
    def reset_slot(self, slot: int, stream_ptr: int = 0):
        check(self.lib.mb_recon_reset_slot(self.h, int(slot), C.c_void_p(stream_ptr)), "mb_recon_reset_slot")

    def slot_upload(self, slot: int, grad_ptr: int, stream_ptr: int = 0):
        """Enqueue the copy of one slot's FP32 gradients (host or device pointer)."""
        check(self.lib.mb_slot_upload(self.h, int(slot), C.c_void_p(grad_ptr), C.c_void_p(stream_ptr)),
              "mb_slot_upload")

    def slot_download(self, slot: int, out_ptr: int, stream_ptr: int = 0):
        """Enqueue the copy of one slot's FP32 DM commands (or layer OPD without a fit)."""
        check(self.lib.mb_slot_download(self.h, int(slot), C.c_void_p(out_ptr), C.c_void_p(stream_ptr)),
              "mb_slot_download")

    def serve_step(self, active, grad_ptr: int, out_ptr: int, stream_ptr: int = 0):
        """Upload the active slots' gradients, step them, download their results."""
        m = np.ascontiguousarray(active, dtype=np.int32)
        if m.shape != (self.nbatch,):
            raise ValueError(f"active must have {self.nbatch} entries")
        check(self.lib.mb_recon_serve_step(self.h, m.ctypes.data_as(C.POINTER(C.c_int)), C.c_void_p(grad_ptr),
                                           C.c_void_p(out_ptr), C.c_void_p(stream_ptr)), "mb_recon_serve_step")

    def step_slots(self, active, stream_ptr: int = 0):
        """One step of the slots whose flag in `active` [nbatch] is non-zero."""
        m = np.ascontiguousarray(active, dtype=np.int32)
        if m.shape != (self.nbatch,):
            raise ValueError(f"active must have {self.nbatch} entries")
        check(self.lib.mb_recon_step_slots(self.h, m.ctypes.data_as(C.POINTER(C.c_int)),
                                           C.c_void_p(stream_ptr)), "mb_recon_step_slots")

    def apply_fit_R(self, x):
        xi = self._vec(x, self.nxtot)
        out = np.empty((self.nbatch, self.nact))
        check(self.lib.mb_apply_fit_R(self.h, _dptr(xi), _dptr(out)), "mb_apply_fit_R")
        return out

    def apply_fit_L(self, a):
        ai = self._vec(a, self.nact)
        out = np.empty((self.nbatch, self.nact))
        check(self.lib.mb_apply_fit_L(self.h, _dptr(ai), _dptr(out)), "mb_apply_fit_L")
        return out

    def tomo_device(self, d_grad_ptr: int, stream_ptr: int = 0):
        check(self.lib.mb_tomo_device(self.h, C.c_void_p(d_grad_ptr), C.c_void_p(stream_ptr)),
              "mb_tomo_device")

    def solution_ptr(self) -> int:
        return int(self.lib.mb_tomo_solution(self.h))

    def residual(self):
        res = np.empty(self.nbatch, dtype=np.float32)
        check(self.lib.mb_tomo_residual(self.h, res.ctypes.data_as(C.POINTER(C.c_float))),
              "mb_tomo_residual")
        return res

    def update_nea(self, iwfs: int, neai: np.ndarray, ptt: Optional[np.ndarray]):
        """gpu_update_recon for one WFS: inverse NEA [nsa][3] (cx, cy, cxy) and
        the tip/tilt projector, 2 x 2nsa (passed column-major, as the ABI
        takes it) or None."""
        ne = np.ascontiguousarray(neai, dtype=np.float64).ravel()
        pt = None
        if ptt is not None:
            pt = np.asarray(ptt, dtype=np.float64)
            pt = np.ascontiguousarray(pt.ravel(order="F") if pt.ndim == 2 else pt)
        check(self.lib.mb_update_recon_nea(self.h, iwfs, _dptr(ne),
                                           _dptr(pt) if pt is not None else C.POINTER(C.c_double)()),
              "mb_update_recon_nea")

    def update_neam(self, neam):
        """The FDPCG part of gpu_update_recon: new mean NEA per WFS, the data
        term and blocks rebuilt on the device (mb_update_recon_neam)."""
        v = np.ascontiguousarray(neam, dtype=np.float64)
        check(self.lib.mb_update_recon_neam(self.h, _dptr(v)), "mb_update_recon_neam")

    def fdpcg_data(self):
        """The device's FDPCG data term as complex [nb, bs, bs] (row, column)."""
        fd = self.sys.fdpcg
        out = np.empty(fd.nb * fd.bs * fd.bs * 2)
        check(self.lib.mb_fdpcg_data(self.h, _dptr(out)), "mb_fdpcg_data")
        c = (out[0::2] + 1j * out[1::2]).reshape(fd.nb, fd.bs, fd.bs)  # [b][col][row]
        return c.transpose(0, 2, 1)

    def update_cn2(self, l2c, fd=None):
        keep = []
        l2 = np.ascontiguousarray(l2c, dtype=np.float64)
        fdp = C.POINTER(MbFdpcgDesc)()
        if fd is not None:
            d = fdpcg_desc(fd, keep)
            keep.append(d)
            fdp = C.pointer(d)
        check(self.lib.mb_update_recon_cn2(self.h, _dptr(l2), fdp), "mb_update_recon_cn2")

    # operator applications (parity tests)
    def apply_R(self, grad):
        g = self._vec(grad, self.ngrad)
        out = np.empty((self.nbatch, self.nxtot))
        check(self.lib.mb_apply_tomo_R(self.h, _dptr(g), _dptr(out)), "mb_apply_tomo_R")
        return out

    def apply_L(self, x):
        xi = self._vec(x, self.nxtot)
        out = np.empty((self.nbatch, self.nxtot))
        check(self.lib.mb_apply_tomo_L(self.h, _dptr(xi), _dptr(out)), "mb_apply_tomo_L")
        return out

    def apply_fdpcg(self, x):
        xi = self._vec(x, self.nxtot)
        out = np.empty((self.nbatch, self.nxtot))
        check(self.lib.mb_apply_fdpcg(self.h, _dptr(xi), _dptr(out)), "mb_apply_fdpcg")
        return out

    def apply_hx(self, x):
        xi = self._vec(x, self.nxtot)
        np_ = self.sys.pmap.n
        out = np.empty((self.nbatch, len(self.sys.wfs), np_))
        check(self.lib.mb_apply_hx(self.h, _dptr(xi), _dptr(out)), "mb_apply_hx")
        return out


class ReconGroup:
    """Reconstructors of different geometries stepped together
    (mb_group_*): one graph per step, the tomography operators launched once
    for all members' instances, each member's CG updates, preconditioner and
    fit in between.  Members stay owned by the caller and must outlive the
    group; each member's result equals its own step's."""

    def __init__(self, members):
        self.members = list(members)
        self.lib = self.members[0].lib
        hs = (C.c_void_p * len(self.members))(*[r.h for r in self.members])
        h = C.c_void_p()
        check(self.lib.mb_group_create(hs, len(self.members), C.byref(h)), "mb_group_create")
        self.h = h

    @property
    def graph_kernels(self) -> int:
        """Kernel launches of one group step."""
        return int(self.lib.mb_group_graph_kernels(self.h))

    def step_device(self, d_grad_ptrs, stream_ptr: int = 0):
        """One step of every member: d_grad_ptrs[i] points to member i's FP32
        gradients [nbatch_i, ngrad_i] on the device; the commands stay in each
        member's fit_solution()."""
        ptrs = (C.c_void_p * len(self.members))(*[C.c_void_p(int(p)) for p in d_grad_ptrs])
        check(self.lib.mb_group_step_device(self.h, ptrs, C.c_void_p(stream_ptr)), "mb_group_step_device")

    def close(self):
        if getattr(self, "h", None):
            self.lib.mb_group_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
