"""Host-side construction of the tomography operator tables.

This module plays the part of the reference's CPU setup
(``maos/setup_recon_prep.c``, ``maos/setup_recon.c``, ``lib/mkg.c``,
``lib/laplacian.c``, ``math/loc.c:create_metapupil``): it turns an
:class:`~maos_b200.config.AOConfig` into the arrays the reconstruction hot path
consumes -- the same tables ``gpu_setup_recon`` (``cuda/recon.cu:477``) reads
out of ``RECON_T``:

* ``pmap``   square pupil grid of ``ploc`` (``tomo.square=1``), one per system;
* ``xmap``   one square grid per reconstructed layer, cone-scaled sampling;
* per WFS    ``saloc`` (subaperture lower-left corners), ``GP`` (sparse
             average-gradient operator from ``ploc``), ``saneai`` (inverse NEA,
             scaled by TOMOSCALE), ``TT``/``PTT`` (tip/tilt removal);
* per layer  the biharmonic regularisation weight ``l2c``.

Grid conventions follow ``map_t``: point ``(ix, iy)`` sits at
``(ox + ix*dx, oy + iy*dy)`` and is stored at ``ix + iy*nx``.
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import List, Optional

import numpy as np
import scipy.sparse as sps

from .config import AOConfig, AS2RAD, TOMOSCALE


@dataclass
class Grid:
    nx: int
    ny: int
    dx: float
    dy: float
    ox: float
    oy: float
    ht: float = 0.0

    @property
    def n(self) -> int:
        return self.nx * self.ny

    def xs(self) -> np.ndarray:
        return self.ox + np.arange(self.nx) * self.dx

    def ys(self) -> np.ndarray:
        return self.oy + np.arange(self.ny) * self.dy


def nextfftsize(n: int) -> int:
    """Smallest even size >= n built from at most two of the radices 2,3,5,7.

    Restates ``math/mathmisc.c:327`` (``nextfftsize``)."""
    if n == 0:
        n = 1
    radixs = (2, 3, 5, 7)
    while True:
        n2, n3 = n, 1
        selected = [0, 0, 0, 0]
        irad = 0
        while irad < 4:
            r = radixs[irad]
            if n2 % r == 0:
                selected[irad] = 1
                n2 //= r
                n3 *= r
            else:
                irad += 1
        if sum(selected) > 2:
            n2 = n
        n += 1
        if not (n2 > 1 or (n3 & 1) == 1):
            return n3


def create_metapupil(dirs: np.ndarray, D: float, ht: float, dx: float, guard: float,
                     nin: int = 0, square: bool = True, offset: float = 0.0) -> Grid:
    """Square grid covering every direction's beam footprint at height ``ht``.

    ``dirs`` is 3 x ndir (thetax, thetay, hs).  Restates
    ``math/loc.c:1471`` (``create_metapupil``) for ``square=1``."""
    R = D / 2
    minx = miny = math.inf
    maxx = maxy = -math.inf
    for k in range(dirs.shape[1]):
        tx, ty, hs = dirs[0, k], dirs[1, k], dirs[2, k]
        RR = (1.0 - ht / hs) * R + guard
        for v in (tx * ht - RR, tx * ht + RR):
            minx, maxx = min(minx, v), max(maxx, v)
        for v in (ty * ht - RR, ty * ht + RR):
            miny, maxy = min(miny, v), max(maxy, v)
    if square:
        maxx = max(abs(minx), abs(maxx)); minx = -maxx
        maxy = max(abs(miny), abs(maxy)); miny = -maxy
    offset = offset - math.floor(offset)
    mind = minx / dx
    adjust = mind - math.floor(mind) - offset
    if adjust < 0:
        adjust += 1
    minx -= adjust * dx
    mind = miny / dx
    adjust = mind - math.floor(mind) - offset
    if adjust < 0:
        adjust += 1
    miny -= adjust * dx
    ox, oy = minx, miny
    nx = int(math.ceil((maxx - ox) / dx)) + 1
    ny = int(math.ceil((maxy - oy) / dx)) + 1
    if square:
        nx = ny = max(nx, ny)
    if nin > 1:
        nin = int(nin)
        ox = ox - ((nin - nx) // 2) * dx
        oy = oy - ((nin - ny) // 2) * dx
        nx = ny = nin
    return Grid(int(nx), int(ny), float(dx), float(dx), float(ox), float(oy), float(ht))


def laplacian_coef(r0: float, weight: float, dx: float) -> float:
    """``lib/laplacian.c:26`` (``laplacian_coef``)."""
    return ((2.0 * math.pi / 0.5e-6) * math.sqrt((r0 / dx) ** (5.0 / 3.0) / 3.44 / weight)
            * (2.0 - 2 ** (-1.0 / 3.0) - 2 ** (-1.0 / 6.0)) ** -0.5)


def annulus_fraction(xc: np.ndarray, yc: np.ndarray, w: float, rin: float, rout: float,
                     nsub: int = 16) -> np.ndarray:
    """Fraction of each w x w cell (lower-left corners xc, yc) inside the annulus."""
    s = (np.arange(nsub) + 0.5) / nsub * w
    sx = xc[:, None, None] + s[None, None, :]
    sy = yc[:, None, None] + s[None, :, None]
    r2 = sx * sx + sy * sy
    inside = (r2 <= rout * rout) & (r2 >= rin * rin)
    return inside.mean(axis=(1, 2))


# ---------------------------------------------------------------------------
# Average-gradient operator (lib/mkg.c, same-plane case)
# ---------------------------------------------------------------------------
_TOL = 5e-16


def _ceil_t(a: float) -> int:
    return int(round(a)) if abs(a - round(a)) < _TOL else int(math.ceil(a))


def _floor_t(a: float) -> int:
    return int(round(a)) if abs(a - round(a)) < _TOL else int(math.floor(a))


def mkg_same_plane(pgrid: Grid, amp: np.ndarray, salocx: np.ndarray, salocy: np.ndarray,
                   dsa: float) -> sps.csr_matrix:
    """Average-gradient operator from the square pupil grid to subapertures.

    Restates ``lib/mkg.c:mkgt`` (lines 109-452) for the case the reference
    takes when the OPD grid is the pupil grid itself (``same=1``: ``scale=1``,
    no displacement) with ``do_partial=1``: each pupil point's bilinear
    influence is integrated over the four quadrants inside the subaperture,
    weighted by the 3x3 amplitude neighbourhood, and the row is normalised by
    the illuminated area (subapertures under 1 % area are zeroed).  Returns
    the (2*nsa) x (nx*ny) matrix with x gradients first, then y."""
    nx, ny = pgrid.nx, pgrid.ny
    dp = pgrid.dx
    dp1 = 1.0 / dp
    nsa = len(salocx)
    dsa2 = dsa / 2.0 * dp1
    amp_thres = dsa2 * dsa2 * 4 * 0.01
    pofx = (0.0 - pgrid.ox) * dp1 + dsa2
    pofy = (0.0 - pgrid.oy) * dp1 + dsa2
    ampm = amp.reshape(ny, nx)

    def ampat(ix: int, iy: int) -> float:
        if 0 <= ix < nx and 0 <= iy < ny:
            return float(ampm[iy, ix])
        return 0.0

    rows: List[int] = []
    cols: List[int] = []
    vals: List[float] = []
    for isa in range(nsa):
        scx = salocx[isa] * dp1 + pofx
        scy = salocy[isa] * dp1 + pofy
        limx1, limx2 = scx - dsa2, scx + dsa2
        limy1, limy2 = scy - dsa2, scy + dsa2
        ampsum = 0.0
        ent = []  # (ipix, wx, wy)
        for limy in range(_ceil_t(limy1) - 1, _floor_t(limy2) + 2):
            for limx in range(_ceil_t(limx1) - 1, _floor_t(limx2) + 2):
                if not (0 <= limx < nx and 0 <= limy < ny):
                    continue
                ipix = limx + limy * nx
                amp2 = [[ampat(limx + i - 1, limy + j - 1) for i in range(3)] for j in range(3)]
                weight = [0.0, 0.0]
                for (a1, a2, indx, signx) in ((limx - limx2, limx - limx1, (0, 1), 1.0),
                                              (limx1 - limx, limx2 - limx, (2, 1), -1.0)):
                    for (b1, b2, indy, signy) in ((limy - limy2, limy - limy1, (0, 1), 1.0),
                                                  (limy1 - limy, limy2 - limy, (2, 1), -1.0)):
                        al1 = max(a1, 0.0); al2 = min(a2, 1.0)
                        be1 = max(b1, 0.0); be2 = min(b2, 1.0)
                        valid = not (al1 > 1 - _TOL or al2 < -_TOL or be1 > 1 - _TOL or be2 < -_TOL)
                        wa = [(al2 ** 2 - al1 ** 2) * 0.5 - (al2 ** 3 - al1 ** 3) / 3,
                              ((1 - al1) ** 3 - (1 - al2) ** 3) / 3,
                              (al2 ** 2 - al1 ** 2) * 0.5,
                              (al2 - al1) - (al2 ** 2 - al1 ** 2) * 0.5]
                        wb = [(be2 ** 2 - be1 ** 2) * 0.5 - (be2 ** 3 - be1 ** 3) / 3,
                              ((1 - be1) ** 3 - (1 - be2) ** 3) / 3,
                              (be2 ** 2 - be1 ** 2) * 0.5,
                              (be2 - be1) - (be2 ** 2 - be1 ** 2) * 0.5]
                        a00 = amp2[indy[0]][indx[0]]; a01 = amp2[indy[0]][indx[1]]
                        a10 = amp2[indy[1]][indx[0]]; a11 = amp2[indy[1]][indx[1]]
                        if valid and abs(a00) > _TOL and abs(a01) > _TOL and abs(a10) > _TOL and abs(a11) > _TOL:
                            weight[0] += ((wb[0] * a00 + wb[1] * a10) * wa[2]
                                          + (wb[0] * a01 + wb[1] * a11) * wa[3]) * dp1 * signx
                            weight[1] += ((wb[2] * a00 + wb[3] * a10) * wa[0]
                                          + (wb[2] * a01 + wb[3] * a11) * wa[1]) * dp1 * signy
                            ampsum += wa[3] * wb[3] * amp2[1][1]
                ent.append((ipix, weight[0], weight[1]))
        norm = 1.0 / ampsum if ampsum > amp_thres else 0.0
        for ipix, wx, wy in ent:
            if abs(wx) > _TOL:
                rows.append(isa); cols.append(ipix); vals.append(wx * norm)
            if abs(wy) > _TOL:
                rows.append(isa + nsa); cols.append(ipix); vals.append(wy * norm)
    G = sps.csr_matrix((vals, (rows, cols)), shape=(2 * nsa, nx * ny))
    G.sum_duplicates()
    G.data[np.abs(G.data) <= 1e-14] = 0.0  # dspdroptol(GS0, 1e-14)
    G.eliminate_zeros()
    return G


# ---------------------------------------------------------------------------
# The tomography system
# ---------------------------------------------------------------------------
@dataclass
class WfsTables:
    thetax: float
    thetay: float
    hs: float
    nsa: int
    dsa: float
    salocx: np.ndarray
    salocy: np.ndarray
    saa: np.ndarray
    GP: sps.csr_matrix          # 2nsa x nploc
    saneai: np.ndarray          # 2nsa diagonal of the inverse NEA (x TOMOSCALE)
    sanea: np.ndarray           # 2nsa diagonal NEA^2 (rad^2), unscaled
    trs: bool
    PTT: Optional[np.ndarray]   # 2 x 2nsa (None if no tip/tilt removal)
    TT: Optional[np.ndarray]    # 2nsa x 2
    neam: float                 # mean NEA (rad / sqrt(TOMOSCALE)) for FDPCG


@dataclass
class TomoSystem:
    cfg: AOConfig
    pmap: Grid
    xmaps: List[Grid]
    ht: np.ndarray
    wt: np.ndarray
    os: np.ndarray
    wfs: List[WfsTables]
    l2c: np.ndarray                 # per-layer biharmonic coefficient (x cxxscale x TOMOSCALE)
    amp: np.ndarray                 # pupil amplitude on pmap
    fdpcg: Optional[object] = None  # FdpcgTables

    @property
    def nx_total(self) -> int:
        return sum(g.n for g in self.xmaps)

    @property
    def ngrad(self) -> int:
        return sum(2 * w.nsa for w in self.wfs)

    def x_offsets(self) -> np.ndarray:
        return np.concatenate([[0], np.cumsum([g.n for g in self.xmaps])]).astype(np.int64)

    def g_offsets(self) -> np.ndarray:
        return np.concatenate([[0], np.cumsum([2 * w.nsa for w in self.wfs])]).astype(np.int64)


def all_dirs(cfg: AOConfig) -> np.ndarray:
    """3 x ndir (thetax, thetay, hs) of every WFS and fit direction."""
    cols = [(w.thetax, w.thetay, cfg.powfs[w.powfs].hs) for w in cfg.wfs]
    cols += [(tx, ty, math.inf) for tx, ty in zip(cfg.fit_thetax, cfg.fit_thetay)]
    return np.array(cols, dtype=np.float64).T


def make_saloc(p, D: float, din: float):
    """Subaperture lower-left corners, area fractions, and the kept subset."""
    order, dsa = p.order, p.dsa
    c = (np.arange(order) - order / 2.0) * dsa
    X, Y = np.meshgrid(c, c)
    sx, sy = X.ravel(), Y.ravel()
    saa = annulus_fraction(sx, sy, dsa, din / 2, D / 2, nsub=16)
    keep = saa >= p.saat
    saa = saa / saa.max()
    return sx[keep].copy(), sy[keep].copy(), saa[keep].copy()


def _pad_until_interior(g: Grid, pmap: Grid, cfg: AOConfig, dirs: np.ndarray) -> Grid:
    """Grow a layer grid by one ring until every ray from the pupil grid lands
    at least half a point inside it.

    ``create_metapupil`` can put the pupil footprint exactly on a layer's last
    row (ground layer, on-axis beam); there the reference's include/skip test
    depends on the last bit of an FP64 sum.  One extra ring removes that
    ambiguity without changing any interior value."""
    while True:
        worst = math.inf
        for k in range(dirs.shape[1]):
            tx, ty, hs = dirs[:, k]
            scale = 1.0 - g.ht / hs
            for xs0, th, o, d, n in ((pmap.xs(), tx, g.ox, g.dx, g.nx),
                                     (pmap.ys(), ty, g.oy, g.dy, g.ny)):
                u = (xs0 * scale + th * g.ht - o) / d
                worst = min(worst, u.min(), (n - 1) - u.max())
        if worst >= 0.5:
            return g
        g = Grid(g.nx + 2, g.ny + 2, g.dx, g.dy, g.ox - g.dx, g.oy - g.dy, g.ht)


def build_tomo(cfg: AOConfig) -> TomoSystem:
    dirs = all_dirs(cfg)
    # ploc / pmap: setup_recon_prep.c:37 (create_metapupil at ht=0, square)
    dxp = cfg.atmr_dx / cfg.tomo_pos
    pmap = create_metapupil(dirs, cfg.D, 0.0, dxp, cfg.tomo_guard * dxp, square=True)
    pxs = pmap.xs() - dxp / 2
    pys = pmap.ys() - dxp / 2
    PX, PY = np.meshgrid(pxs, pys)
    amp = annulus_fraction(PX.ravel(), PY.ravel(), dxp, cfg.din / 2, cfg.D / 2, nsub=8)

    # layers: setup_recon_prep.c:1117-1133 and setup_recon_xloc (169-238)
    hs_r = cfg.powfs[0].hs if math.isfinite(cfg.powfs[0].hs) else math.inf
    ht = np.array(cfg.atmr_ht, dtype=np.float64)
    os_ = np.array(cfg.atmr_os, dtype=np.int64)
    wt = np.clip(np.array(cfg.atmr_wt, dtype=np.float64), 0.01, 1)
    wt = wt / np.abs(wt).sum()
    dxl = np.array([(cfg.atmr_dx / o) * (1.0 - h / hs_r) for h, o in zip(ht, os_)])
    nin0 = 0
    if cfg.tomo_precond == 1:
        nxs = []
        for h, o, d in zip(ht, os_, dxl):
            g = create_metapupil(dirs, cfg.D, h, d, cfg.tomo_guard * d, square=True)
            nxs.append(g.nx // o)
        nxmax, nxmin = max(nxs), min(nxs)
        nin0 = nextfftsize(int(max(nxmax, nxmin * 1.5)))
        while nin0 & 1:
            nin0 = nextfftsize(nin0 + 1)
    xmaps = [create_metapupil(dirs, cfg.D, h, d, cfg.tomo_guard * d, nin=nin0 * o, square=True)
             for h, o, d in zip(ht, os_, dxl)]
    for l in range(len(xmaps)):
        xmaps[l] = _pad_until_interior(xmaps[l], pmap, cfg, dirs)

    # biharmonic weight per layer (tomo.cu:159-163 / laplacian.c:26)
    l2c = np.array([(laplacian_coef(cfg.r0, w, g.dx) * 0.25) ** 2 * cfg.tomo_cxxscale * TOMOSCALE
                    for w, g in zip(wt, xmaps)])

    # WFS tables
    rng = np.random.default_rng(cfg.seed + 1000)
    gp_cache = {}
    wfs_tabs = []
    for iw, w in enumerate(cfg.wfs):
        p = cfg.powfs[w.powfs]
        if w.powfs not in gp_cache:
            sx, sy, saa = make_saloc(p, cfg.D, cfg.din)
            G = mkg_same_plane(pmap, amp, sx, sy, p.dsa)
            gp_cache[w.powfs] = (sx, sy, saa, G)
        sx, sy, saa, G = gp_cache[w.powfs]
        nsa = len(sx)
        # NEA (setup_recon.c:52-170): geometric WFS, seeing-limited area scaling
        if p.nea_range_as is not None:
            nea_as = rng.uniform(p.nea_range_as[0], p.nea_range_as[1], size=nsa)
            neasq = (nea_as * AS2RAD) ** 2 / p.dtrat
        else:
            neasq = np.full(nsa, (p.nearecon_mas / 206265000.0) ** 2 / p.dtrat)
        neasq = neasq / saa
        sanea = np.concatenate([neasq, neasq])
        saneai = TOMOSCALE / sanea
        # mean NEA for FDPCG (setup_recon.c:175-232)
        sel = saa > 0.9
        neam = math.sqrt((sanea[:nsa][sel].sum() + sanea[nsa:][sel].sum()) / sel.sum() / 2)
        neam /= math.sqrt(TOMOSCALE)
        TT = PTT = None
        if p.trs:
            TT = np.zeros((2 * nsa, 2))
            TT[:nsa, 0] = 1
            TT[nsa:, 1] = 1
            # dcellpinv(TT, saneai): (TT' W TT)^-1 TT' W   (setup_recon.c:255)
            WT = TT * saneai[:, None]
            PTT = np.linalg.solve(TT.T @ WT, WT.T)
        wfs_tabs.append(WfsTables(w.thetax, w.thetay, p.hs, nsa, p.dsa, sx, sy, saa, G, saneai,
                                  sanea, p.trs, PTT, TT, neam))
    sysm = TomoSystem(cfg, pmap, xmaps, ht, wt, os_, wfs_tabs, l2c, amp)
    if cfg.tomo_precond == 1:
        from .fdpcg_setup import fdpcg_prepare
        sysm.fdpcg = fdpcg_prepare(sysm)
    return sysm
