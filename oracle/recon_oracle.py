"""CPU oracle for the reconstruction hot path -- TEST INFRASTRUCTURE ONLY.

This module restates, in FP64 numpy, the reference CPU reconstruction that
MAOS runs when the GPU is off.  It is the checker: only ``tests/``,
``__graft_entry__.smoke()`` and the ``cpu_baseline`` leg of ``bench.py`` may
import it.  The product path (``maos_b200``) never calls it.

Restated functions (reference file:line):

* ``prop_matrix``   -- ``lib/prop_grid.c`` ``prop_grid_stat`` via
                       ``lib/accphi.c:414-420`` (bilinear ray tracing from a
                       square layer grid to the square pupil grid, cone scale
                       ``1-ht/hs``, displacement ``theta*ht``).
* ``tomo_R``        -- ``maos/recon_utils.c:397`` ``TomoR``:
                       ``x = Hx^T GP^T NEA^-1 (I - TT PTT) g``.
* ``tomo_L``        -- ``maos/recon_utils.c:447`` ``TomoL``:
                       ``Hx^T GP^T NEA^-1 (I - TT PTT) GP Hx x + L2^T L2 x``.
* ``fdpcg_precond`` -- ``maos/fdpcg.c:661``: per-layer FFT, permutation,
                       block multiply, inverse permutation, inverse FFT.
* ``pcg``           -- ``lib/pcg.c:28``: (preconditioned) conjugate gradient
                       with warm restart, restart every 100 iterations,
                       returns ``sqrt(r.r / b.b)`` after the last iteration.
* ``mvm``           -- ``maos/recon.c:300``: ``a = M g``.

Parity of this restatement is pinned against the reference's own compiled
CPU code (``oracle/ref``) by ``tests/test_oracle_pin.py``.
"""
from __future__ import annotations

import math
from typing import Callable, List, Optional

import numpy as np
import scipy.sparse as sps

EPS_PROP = 1e-12  # lib/accphi.c:26


def prop_matrix(src, dst, dispx: float, dispy: float, scale: float) -> sps.csr_matrix:
    """Bilinear ray-tracing matrix from grid ``src`` (a layer) onto grid ``dst``.

    Point (ix, iy) of ``dst`` at (x, y) samples ``src`` at
    ``u = (x*scale + dispx - src.ox)/src.dx`` (same for y).  A point is used
    when ``0 <= u <= nx-1`` and ``0 <= v <= ny-1`` (``prop_grid_stat``'s
    no-wrap rule); the weights are the usual bilinear ones."""
    xs = dst.ox + np.arange(dst.nx) * dst.dx
    ys = dst.oy + np.arange(dst.ny) * dst.dy
    u = (xs * scale + dispx - src.ox) / src.dx
    v = (ys * scale + dispy - src.oy) / src.dy
    iu = np.floor(u).astype(np.int64)
    fu = u - iu
    iv = np.floor(v).astype(np.int64)
    fv = v - iv
    # a point exactly on the last column/row uses that point alone
    edge_u = (iu == src.nx - 1) & (fu < EPS_PROP)
    edge_v = (iv == src.ny - 1) & (fv < EPS_PROP)
    iu = np.where(edge_u, src.nx - 2, iu); fu = np.where(edge_u, 1.0, fu)
    iv = np.where(edge_v, src.ny - 2, iv); fv = np.where(edge_v, 1.0, fv)
    okx = (u >= 0) & (iu >= 0) & (iu <= src.nx - 2)
    oky = (v >= 0) & (iv >= 0) & (iv <= src.ny - 2)
    rows, cols, vals = [], [], []
    IY, IX = np.meshgrid(np.arange(dst.ny), np.arange(dst.nx), indexing="ij")
    ok = oky[IY] & okx[IX]
    r = (IX + IY * dst.nx)[ok]
    ix, iy = iu[IX[ok]], iv[IY[ok]]
    fx, fy = fu[IX[ok]], fv[IY[ok]]
    for dxo, dyo, w in ((0, 0, (1 - fx) * (1 - fy)), (1, 0, fx * (1 - fy)),
                        (0, 1, (1 - fx) * fy), (1, 1, fx * fy)):
        rows.append(r)
        cols.append((ix + dxo) + (iy + dyo) * src.nx)
        vals.append(w)
    H = sps.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                       shape=(dst.n, src.n))
    H.sum_duplicates()
    return H


def laplacian_map_matrix(nx: int, ny: int, cf: float) -> sps.csr_matrix:
    """``lib/laplacian.c:70`` ``mklaplacian_map``: cf*(-I + (4 periodic neighbours)/4)."""
    idx = np.arange(nx * ny)
    ix, iy = idx % nx, idx // nx
    rows = np.repeat(idx, 5)
    cols = np.stack([((iy - 1) % ny) * nx + ix, iy * nx + (ix - 1) % nx, idx,
                     iy * nx + (ix + 1) % nx, ((iy + 1) % ny) * nx + ix], axis=1).ravel()
    vals = np.tile([0.25 * cf, 0.25 * cf, -cf, 0.25 * cf, 0.25 * cf], nx * ny)
    return sps.csr_matrix((vals, (rows, cols)), shape=(nx * ny, nx * ny))


class TomoOracle:
    """FP64 tomography operators on one :class:`maos_b200.geometry.TomoSystem`."""

    def __init__(self, sysm, split: int = 1):
        """``split`` mirrors ``recon.split``: when non-zero the left-hand
        operator skips the tip/tilt projection (recon_utils.c:459-464) while
        the right-hand side always applies it."""
        from maos_b200.geometry import laplacian_coef
        self.split = split
        from maos_b200.config import TOMOSCALE
        self.sys = sysm
        cfg = sysm.cfg
        self.H = []  # H[w][l]: pmap x xmap_l
        for w in sysm.wfs:
            row = []
            for l, g in enumerate(sysm.xmaps):
                ht = sysm.ht[l]
                scale = 1.0 - ht / w.hs
                row.append(prop_matrix(g, sysm.pmap, w.thetax * ht, w.thetay * ht, scale))
            self.H.append(row)
        self.L2 = [laplacian_map_matrix(g.nx, g.nx, laplacian_coef(cfg.r0, sysm.wt[l], g.dx)
                                        * math.sqrt(cfg.tomo_cxxscale * TOMOSCALE))
                   for l, g in enumerate(sysm.xmaps)]
        self.xoff = sysm.x_offsets()
        self.goff = sysm.g_offsets()

    # -- helpers ---------------------------------------------------------
    def split_x(self, x):
        return [x[self.xoff[l]:self.xoff[l + 1]] for l in range(len(self.sys.xmaps))]

    def split_g(self, g):
        return [g[self.goff[w]:self.goff[w + 1]] for w in range(len(self.sys.wfs))]

    def _ttfr(self, gw, w):
        tab = self.sys.wfs[w]
        if tab.PTT is None:
            return gw
        return gw - tab.TT @ (tab.PTT @ gw)

    def _nea_gpt(self, gw, w, alpha):
        tab = self.sys.wfs[w]
        return alpha * (tab.GP.T @ (tab.saneai * gw))

    def _iprop(self, opd_w: List[np.ndarray]) -> List[np.ndarray]:
        out = []
        for l in range(len(self.sys.xmaps)):
            acc = np.zeros(self.sys.xmaps[l].n)
            for w in range(len(self.sys.wfs)):
                acc += self.H[w][l].T @ opd_w[w]
            out.append(acc)
        return out

    # -- operators -------------------------------------------------------
    def hx(self, x):
        """Hx: layers -> pupil OPD per WFS (Tomo_prop_do, recon_utils.c:220)."""
        xs = self.split_x(x)
        return [sum(self.H[w][l] @ xs[l] for l in range(len(xs))) for w in range(len(self.sys.wfs))]

    def tomo_R(self, g, alpha=1.0):
        gs = self.split_g(np.asarray(g, dtype=np.float64))
        opd = [self._nea_gpt(self._ttfr(gs[w], w), w, alpha) for w in range(len(gs))]
        return np.concatenate(self._iprop(opd))

    def tomo_L(self, x, alpha=1.0):
        x = np.asarray(x, dtype=np.float64)
        opd = self.hx(x)
        gg = [self.sys.wfs[w].GP @ opd[w] for w in range(len(opd))]
        if not self.split:
            gg = [self._ttfr(gg[w], w) for w in range(len(gg))]
        opd2 = [self._nea_gpt(gg[w], w, alpha) for w in range(len(gg))]
        out = self._iprop(opd2)
        xs = self.split_x(x)
        for l in range(len(xs)):
            out[l] += alpha * (self.L2[l].T @ (self.L2[l] @ xs[l]))
        return np.concatenate(out)

    def fdpcg_precond(self, r):
        fd = self.sys.fdpcg
        xs = self.split_x(np.asarray(r, dtype=np.float64))
        specs = []
        for l, g in enumerate(self.sys.xmaps):
            f = np.fft.fft2(xs[l].reshape(g.ny, g.nx))
            if fd.scale:
                f /= math.sqrt(g.nx * g.ny)
            specs.append(f.ravel())
        xhat = np.concatenate(specs)
        xhat2 = xhat[fd.perm].reshape(fd.nb, fd.bs)
        y = np.einsum("bij,bj->bi", fd.Mbinv, xhat2).ravel()
        out_hat = np.empty_like(xhat)
        out_hat[fd.perm] = y
        out = []
        for l, g in enumerate(self.sys.xmaps):
            f = out_hat[self.xoff[l]:self.xoff[l + 1]].reshape(g.ny, g.nx)
            z = np.fft.ifft2(f) * (g.nx * g.ny)  # unnormalised inverse, like cfft2(+1)
            if fd.scale:
                z /= math.sqrt(g.nx * g.ny)
            out.append(z.real.ravel())
        return np.concatenate(out)


def pcg(x0: Optional[np.ndarray], Amul: Callable, Mmul: Optional[Callable], b: np.ndarray,
        warm: bool, maxiter: int):
    """``lib/pcg.c:28``.  ``Amul(x)`` returns A*x; ``Mmul(r)`` returns M^-1 r.

    Returns (x, residual) with residual = sqrt(r.r/b.b) after the last step."""
    b = np.asarray(b, dtype=np.float64)
    x = np.zeros_like(b) if (x0 is None or not warm) else np.array(x0, dtype=np.float64)
    r0z0 = float(b @ b)
    r = z = p = None
    r0z1 = 0.0
    res = float("nan")
    for k in range(maxiter):
        if k % 100 == 0:
            r = b - Amul(x)
            z = Mmul(r) if Mmul else r
            p = z.copy()
            r0z1 = float(r @ z)
        Ap = Amul(p)
        ak = r0z1 / float(p @ Ap)
        if not math.isfinite(ak):
            ak = 0.0
            break
        x = x + ak * p
        r = r - ak * Ap
        if k + 1 == maxiter:
            res = math.sqrt(float(r @ r) / r0z0)
            break
        z = Mmul(r) if Mmul else r
        r0z2 = float(r @ z)
        bk = r0z2 / r0z1
        p = bk * p + z
        r0z1 = r0z2
    return x, res


def tomo_solve(orc: TomoOracle, grad, x0=None, maxit=None):
    """One tomography step: RHS then (FD)PCG, warm-started from x0 (recon.c:55-83)."""
    sysm = orc.sys
    maxit = sysm.cfg.tomo_maxit if maxit is None else maxit
    rhs = orc.tomo_R(grad)
    M = orc.fdpcg_precond if sysm.fdpcg is not None else None
    return pcg(x0, orc.tomo_L, M, rhs, x0 is not None, maxit)


def mvm(M: np.ndarray, g: np.ndarray) -> np.ndarray:
    """``maos/recon.c:300``: DM commands from the control matrix."""
    return np.asarray(M, dtype=np.float64) @ np.asarray(g, dtype=np.float64)


class FitOracle:
    """FP64 DM-fit operators (grid form) on a :class:`maos_b200.fit_setup.FitSystem`.

    ``fit_R``: ``maos/recon_utils.c:483`` FitR with HXF (bilinear ray tracing
    from the layers onto the fit grid along each fit direction);
    ``fit_L``: ``maos/recon_utils.c:536`` FitL, with the slaving term when
    the fit system carries one."""

    def __init__(self, tomo_sys, fit_sys):
        self.t = tomo_sys
        self.f = fit_sys
        self.HXF = [[prop_matrix(g, fit_sys.floc, tx * g.ht, ty * g.ht, 1.0) for g in tomo_sys.xmaps]
                    for tx, ty in zip(fit_sys.thetax, fit_sys.thetay)]
        self.xoff = tomo_sys.x_offsets()
        self.aoff = fit_sys.act_offsets()

    def _applyW(self, v, f):
        wt = self.f.wt[f]
        return wt * (self.f.W0 @ v) - wt * self.f.W1 * (self.f.W1 @ v)

    def _hat(self, xp):
        out = []
        for d in range(len(self.f.dms)):
            acc = np.zeros(len(self.f.dms[d].act))
            for f in range(len(xp)):
                acc += self.f.HA[f][d].T @ xp[f]
            out.append(acc)
        return np.concatenate(out)

    def fit_R(self, x, alpha=1.0):
        x = np.asarray(x, dtype=np.float64)
        xs = [x[self.xoff[l]:self.xoff[l + 1]] for l in range(len(self.t.xmaps))]
        xp = []
        for f in range(len(self.f.thetax)):
            v = sum(self.HXF[f][l] @ xs[l] for l in range(len(xs)))
            xp.append(self._applyW(v, f))
        return alpha * self._hat(xp)

    def fit_L(self, a, alpha=1.0):
        a = np.asarray(a, dtype=np.float64)
        As = [a[self.aoff[d]:self.aoff[d + 1]] for d in range(len(self.f.dms))]
        xp = []
        for f in range(len(self.f.thetax)):
            v = sum(self.f.HA[f][d] @ As[d] for d in range(len(As)))
            xp.append(self._applyW(v, f))
        out = self._hat(xp)
        if self.f.NW.shape[1]:
            out = out + self.f.NW @ (self.f.NW.T @ a)
        if getattr(self.f, "actslave", None) is not None:  # recon_utils.c:555-557
            out = out + self.f.actslave @ a
        return alpha * out


class SparseFitOracle:
    """FP64 assembled DM fit (``lib/muv.c:37`` muv on ``fit->FR`` / ``fit->FL``,
    the operators ``maos/recon.c:93`` muv_solve applies):
    ``fit_R x = FR.M x - FR.U (FR.V' x)``, ``fit_L a = FL.M a - FL.U (FL.V' a)``
    on a :class:`maos_b200.fit_assemble.SparseFit`."""

    def __init__(self, tomo_sys, sf):
        self.t = tomo_sys
        self.f = sf

    def fit_R(self, x, alpha=1.0):
        x = np.asarray(x, dtype=np.float64)
        return alpha * (self.f.FRM @ x - self.f.FRU @ (self.f.FRV.T @ x))

    def fit_L(self, a, alpha=1.0):
        a = np.asarray(a, dtype=np.float64)
        return alpha * (self.f.FLM @ a - self.f.FLU @ (self.f.FLV.T @ a))


def fit_solve(fo, x_layers, a0=None, maxit=None):
    """DM fit of one step: FitR then CG on FitL, warm-started from a0 (recon.c:89-93)."""
    maxit = fo.f.maxit if maxit is None else maxit
    rhs = fo.fit_R(x_layers)
    return pcg(a0, fo.fit_L, None, rhs, a0 is not None, maxit)
