"""DM-fit tables: fit grid, W0/W1 weighting, DM actuator grids, low-rank terms.

Host-side counterpart of ``maos/setup_recon_fit.c`` and
``maos/setup_recon_prep.c`` (floc / aloc) for the grid-form fit the
reference's GPU path uses (``cuda/fit.cu`` ``cufit_grid``):

    FitR x = sum_f wt_f HA_f^T (W0 - W1 W1^T) Hxp_f x
    FitL a = sum_f wt_f HA_f^T (W0 - W1 W1^T) HA_f a + NW (NW^T a)

* ``floc``    the fit grid; ``fit.pos`` inherits ``tomo.pos`` so it is the
              tomography pupil grid itself (setup_recon_prep.c:112).
* ``W0, W1``  restated from ``lib/mkw.c:41`` (``mkw_amp``): 9-point bilinear
              weighting from the annular amplitude sampled on ``floc``.
* DMs         an ``order x order`` square of actuators at pitch ``dm.dx``,
              offset by ``dm.offset`` pitches, every point an actuator: the
              reference's grid-form GPU fit requires ``fit.square=1``
              (maos/setup_parms.c:3001-3003).  The square grows by one ring
              while a fit-direction ray from ``floc`` would leave it, so the
              bilinear influence (``lib/mkh.c`` ``mkh``) is plain bilinear
              interpolation on the square.
* ``NW``      piston per DM and tip/tilt on the upper DMs
              (setup_recon_fit.c:110-165, ``fit.lrt_piston``/``lrt_tt``),
              restricted to actuators with coupling > 0.1 (``genactcpl``,
              lib/slaving.c:25).
* ``actslave`` the slaving term ``cufit_grid::L`` adds (cuda/fit.cu:232-234),
              built by ``lib/slaving.c:63`` slaving from the coupling of each
              grid actuator (``fit.actslave``, on by default).

The assembled fit with actuators inside the metapupil, the reference's
default, is ``maos_b200.fit_assemble``.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import List, Optional

import numpy as np
import scipy.sparse as sps

from .geometry import Grid, annulus_fraction

EPS = 1e-15  # sys/common.h:88


@dataclass
class DmTables:
    ht: float
    amap: Grid            # square actuator grid
    act: np.ndarray       # indices of the actuators in amap (compact aloc order; all of them)
    locx: np.ndarray      # aloc coordinates
    locy: np.ndarray


@dataclass
class FitSystem:
    floc: Grid
    thetax: np.ndarray
    thetay: np.ndarray
    wt: np.ndarray
    hs: np.ndarray
    W0: sps.csr_matrix
    W1: np.ndarray
    dms: List[DmTables]
    NW: np.ndarray        # [nact_total, nnw] in compact aloc order (DMs concatenated)
    maxit: int
    HA: list              # HA[f][d]: csr (nfloc x nact_d), for the oracle and setup
    actslave: Optional[sps.csr_matrix] = None  # nact_total x nact_total, block diagonal

    @property
    def nact(self) -> int:
        return sum(len(d.act) for d in self.dms)

    def act_offsets(self):
        return np.concatenate([[0], np.cumsum([len(d.act) for d in self.dms])]).astype(np.int64)


def mkw_amp(g: Grid, amp: np.ndarray):
    """``lib/mkw.c:41`` mkw_amp on a full square grid; ``amp`` must sum to 1."""
    nx, ny = g.nx, g.ny
    n = nx * ny
    if abs(amp.sum() - 1) > 1e-6:
        raise ValueError("amp must be normalised to sum to 1")
    A = amp.reshape(ny, nx)

    def ok(ix, iy):
        return 0 <= ix < nx and 0 <= iy < ny

    def a(ix, iy):
        return A[iy, ix]

    rows, cols, vals = [], [], []
    W1 = np.zeros(n)
    for iy in range(ny):
        for ix in range(nx):
            il = ix + iy * nx
            camp = a(ix, iy)
            wt2 = 0.0
            for jy in range(iy - 1, iy + 2):
                for jx in range(ix - 1, ix + 2):
                    if not ok(jx, jy):
                        continue
                    bamp = a(jx, jy)
                    wt = 0.0
                    if abs(ix - jx) == 1 and abs(iy - jy) == 1:
                        if ok(ix, jy) and ok(jx, iy):
                            wt += (camp + bamp + a(ix, jy) + a(jx, iy)) / 144.0
                    elif abs(iy - jy) == 1:
                        for ioff in (-1, 1):
                            if ok(ix + ioff, jy) and ok(jx + ioff, iy):
                                wt += (camp + bamp) / 48.0 + (a(ix + ioff, jy) + a(jx + ioff, iy)) / 144.0
                    elif abs(ix - jx) == 1:
                        for joff in (-1, 1):
                            if ok(ix, jy + joff) and ok(jx, iy + joff):
                                wt += (camp + bamp) / 48.0 + (a(ix, jy + joff) + a(jx, iy + joff)) / 144.0
                    else:
                        for joff in (-1, 1):
                            for ioff in (-1, 1):
                                if ok(ix, iy + joff) and ok(ix + ioff, iy) and ok(ix + ioff, iy + joff):
                                    wt += (camp / 16.0 + (a(ix, iy + joff) + a(ix + ioff, iy)) / 48.0
                                           + a(ix + ioff, iy + joff) / 144.0)
                                    wt2 += (camp / 9.0 + (a(ix, iy + joff) + a(ix + ioff, iy)) / 18.0
                                            + a(ix + ioff, iy + joff) / 36.0)
                    if wt > 0:
                        rows.append(jx + jy * nx)
                        cols.append(il)
                        vals.append(wt)
            W1[il] = wt2
    W0 = sps.csc_matrix((vals, (rows, cols)), shape=(n, n))
    s = W1.sum()
    if abs(s - 1) > 1e-12:
        W1 = W1 / s
        W0 = W0 / s
    return sps.csr_matrix(W0), W1


SNAP = 1e-9


def snap(u: np.ndarray) -> np.ndarray:
    """Round coordinates within 1e-9 of a grid point onto it (exact-edge rays)."""
    r = np.round(u)
    return np.where(np.abs(u - r) < SNAP, r, u)


def mkh_grid(src: Grid, act: np.ndarray, dst: Grid, dispx: float, dispy: float,
             scale: float) -> sps.csr_matrix:
    """``lib/mkh.c:47`` mkh: bilinear influence of the active points of ``src``
    (compact order ``act``) at every point of ``dst``.  Corners that are not
    active actuators are dropped; weights are not renormalised."""
    pos = -np.ones(src.n, dtype=np.int64)
    pos[act] = np.arange(len(act))
    xs = dst.ox + np.arange(dst.nx) * dst.dx
    ys = dst.oy + np.arange(dst.ny) * dst.dy
    X, Y = np.meshgrid(xs, ys)
    u = snap((X.ravel() * scale + dispx - src.ox) / src.dx)
    v = snap((Y.ravel() * scale + dispy - src.oy) / src.dy)
    iu = np.floor(u).astype(np.int64)
    iv = np.floor(v).astype(np.int64)
    fu = u - iu
    fv = v - iv
    rows, cols, vals = [], [], []
    r = np.arange(dst.n)
    for dx_, dy_, w in ((0, 0, (1 - fu) * (1 - fv)), (1, 0, fu * (1 - fv)),
                        (0, 1, (1 - fu) * fv), (1, 1, fu * fv)):
        jx, jy = iu + dx_, iv + dy_
        inb = (jx >= 0) & (jx < src.nx) & (jy >= 0) & (jy < src.ny) & (w > EPS)
        idx = np.where(inb, jx + jy * src.nx, 0)
        c = np.where(inb, pos[idx], -1)
        ok = c >= 0
        rows.append(r[ok]); cols.append(c[ok]); vals.append(w[ok])
    H = sps.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                       shape=(dst.n, len(act)))
    H.sum_duplicates()
    return H


def _covers(g: Grid, floc: Grid, thetax, thetay) -> bool:
    """Every fit-direction ray from ``floc`` lands inside ``g`` (within 1e-9)."""
    for tx, ty in zip(thetax, thetay):
        for xs, th, o, d, n in ((floc.xs(), tx, g.ox, g.dx, g.nx), (floc.ys(), ty, g.oy, g.dy, g.ny)):
            u = (xs + th * g.ht - o) / d
            if u.min() < -SNAP or u.max() > n - 1 + SNAP:
                return False
    return True


def build_fit(sysm) -> FitSystem:
    cfg = sysm.cfg
    floc = sysm.pmap
    nfit = len(cfg.fit_thetax)
    thetax = np.asarray(cfg.fit_thetax, dtype=np.float64)
    thetay = np.asarray(cfg.fit_thetay, dtype=np.float64)
    wt = np.asarray(cfg.fit_wt, dtype=np.float64)
    hs = np.full(nfit, math.inf)
    # amplitude on floc: annulus coverage of each cell, normalised to sum 1
    X, Y = np.meshgrid(floc.xs() - floc.dx / 2, floc.ys() - floc.dy / 2)
    amp = annulus_fraction(X.ravel(), Y.ravel(), floc.dx, cfg.din / 2, cfg.D / 2, nsub=8)
    amp = amp / amp.sum()
    W0, W1 = mkw_amp(floc, amp)
    dms = []
    for d in cfg.dms:
        n = d.order
        ox = (d.offset - (n // 2)) * d.dx if n % 2 == 0 else (d.offset - (n - 1) / 2) * d.dx
        g = Grid(n, n, d.dx, d.dx, ox, ox, d.ht)
        while not _covers(g, floc, thetax, thetay):
            g = Grid(g.nx + 2, g.ny + 2, g.dx, g.dy, g.ox - g.dx, g.oy - g.dy, g.ht)
        XX, YY = np.meshgrid(g.xs(), g.ys())
        act = np.arange(g.n)
        dms.append(DmTables(d.ht, g, act, XX.ravel(), YY.ravel()))
    HA = [[mkh_grid(dm.amap, dm.act, floc, tx * dm.ht, ty * dm.ht, 1.0) for dm in dms]
          for tx, ty in zip(thetax, thetay)]
    # low-rank terms (setup_recon_fit.c:110-165)
    fitscl = 1.0 / floc.n
    ndm = len(dms)
    nnw = (ndm if cfg.fit_lrt_piston else 0) + (2 * (ndm - 1) if cfg.fit_lrt_tt else 0)
    off = np.concatenate([[0], np.cumsum([len(dm.act) for dm in dms])])
    NW = np.zeros((int(off[-1]), nnw))
    # actuator coupling (lib/slaving.c:25 genactcpl)
    from .fit_assemble import genactcpl, loc_create_map, slaving, square_loc
    cpl = genactcpl(HA, W1)
    actslave = None
    if cfg.fit_actslave:
        sl = [slaving(loc_create_map(square_loc(dm.amap), 0), cpl[k], cfg.fit_actthres, 1.0 / floc.n)
              for k, dm in enumerate(dms)]
        if any(m is not None for m in sl):
            actslave = sps.block_diag([m if m is not None else sps.csr_matrix((len(dms[k].act),) * 2)
                                       for k, m in enumerate(sl)], format="csr")
    if nnw:
        inw = 0
        if cfg.fit_lrt_piston:
            for k in range(ndm):
                NW[off[k]:off[k + 1], inw + k] = np.where(cpl[k] > 0.1, fitscl, 0.0)
            inw += ndm
        if cfg.fit_lrt_tt:
            diam0 = 2 * math.sqrt(np.max(dms[0].locx ** 2 + dms[0].locy ** 2))
            factor = fitscl * 2.0 / diam0
            for k in range(1, ndm):
                m = cpl[k] > 0.1
                NW[off[k]:off[k + 1], inw + 2 * (k - 1)] = np.where(m, dms[k].locx * factor, 0.0)
                NW[off[k]:off[k + 1], inw + 2 * (k - 1) + 1] = np.where(m, dms[k].locy * factor, 0.0)
    return FitSystem(floc, thetax, thetay, wt, hs, W0, W1, dms, NW, cfg.fit_maxit, HA, actslave)
