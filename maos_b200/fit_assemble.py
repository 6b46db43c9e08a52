"""Assembled DM fit: the reference's default fit, with in-pupil actuators.

Host-side counterpart of the reference's fit setup for ``fit.square=0``,
``fit.assemble=1``, ``gpu.fit=1`` (its defaults, ``config/maos/recon.conf``,
``config/maos/sim.conf:79``): the tables that ``cuda/solve.cu``
``cusolve_sparse`` hands to the GPU as ``recon->fit->FR`` and ``FL``::

    rhs   = FR.M x - FR.U (FR.V' x)          (lib/muv.c:37 muv)
    FL a  = FL.M a - FL.U (FL.V' a)

Steps, each following the reference routine cited beside it:

* ``floc``   ``create_metapupil(dirs, D, 0, atmr.dx/fit.pos, guard)``, the
             circular metapupil (``maos/setup_recon_prep.c:111-128``,
             ``math/loc.c:1471``, ``math/matmath.c:556`` circle_symbolic);
* ``W0, W1`` ``mkw_circular(floc, 0, 0, D/2)`` (``lib/mkw.c:363``; the
             default ``mkw_annular`` with ``rin = 0``, ``setup_recon_prep.c:152``);
* ``aloc``   per DM ``create_metapupil(dirs, D, ht, dx, offset, dm.guard*dx)``
             (``setup_recon_prep.c:298-320``); every loc gets its map by
             ``loc_create_map_npad(loc, 1)`` with the ghost points of
             ``math/loc.c:259-331``, which ``mkh`` reads (``labs``);
* ``HXF, HA`` ``mkh`` (``lib/mkh.c:47-140``);
* ``actcpl`` ``genactcpl`` (``lib/slaving.c:25``), ``actinterp``
             ``act_extrap`` (``lib/slaving.c:536-636``), ``HA <- HA actinterp``
             (``maos/setup_recon_fit.c:86-98``);
* ``NW``     piston and upper-DM tip/tilt (``setup_recon_fit.c:106-165``);
* ``actslave`` ``slaving`` (``lib/slaving.c:63-225``) with ``sclsq = 1/nfloc``;
* ``FR, FL`` ``setup_fit_matrix`` (``setup_recon_fit.c:186-293``): the
             Tikhonov term ``tikcr*4/nact`` on the diagonal, the slaving term,
             ``FL.U = [FR.U, NW]``, ``FL.V = [FR.U, -NW]``.

The result is pinned to the reference's own ``setup_fit`` on the same inputs
(``tests/test_fit_assemble_pin.py``).
"""
from __future__ import annotations

import math
from dataclasses import dataclass
from typing import List, Optional

import numpy as np
import scipy.sparse as sps

from .geometry import Grid, all_dirs

EPS = 1e-15  # sys/common.h:88


# ---------------------------------------------------------------------------
# loc_t with its map
# ---------------------------------------------------------------------------
@dataclass
class Loc:
    """Points (x fastest, as map2loc leaves them) and their index map."""
    locx: np.ndarray
    locy: np.ndarray
    dx: float
    ht: float = 0.0
    mox: float = 0.0
    moy: float = 0.0
    map: Optional[np.ndarray] = None  # [ny][nx] 1-based index; negative: ghost of that point

    @property
    def nloc(self) -> int:
        return len(self.locx)

    @property
    def n(self) -> int:
        return len(self.locx)

    def points(self):
        return self.locx, self.locy


def _round_half_away(v):
    return np.where(v >= 0, np.floor(v + 0.5), -np.floor(-v + 0.5))


def loc_create_map(loc: Loc, npad: int) -> Loc:
    """``math/loc.c:208`` loc_create_map_npad with the ghost extension of
    ``LOC_MAP_EXTEND`` (on by default): an empty map point with an existing
    neighbour takes the negative index of the neighbour of lowest level, the
    nearest one (edge before corner), and among equals the one nearest the
    centre; ``npad`` levels."""
    dx = abs(loc.dx)
    xmin, xmax = float(loc.locx.min()), float(loc.locx.max())
    ymin, ymax = float(loc.locy.min()), float(loc.locy.max())
    if npad > 0:
        xmin -= npad * dx
        ymin -= npad * dx
        xmax += npad * dx
        ymax += npad * dx
    nx = int(_round_half_away((xmax - xmin) * (1.0 / dx))) + 1
    ny = int(_round_half_away((ymax - ymin) * (1.0 / dx))) + 1
    m = np.zeros((ny, nx), dtype=np.int64)
    ix = _round_half_away((loc.locx - xmin) * (1.0 / dx)).astype(np.int64)
    iy = _round_half_away((loc.locy - ymin) * (1.0 / dx)).astype(np.int64)
    m[iy, ix] = np.arange(1, loc.nloc + 1)
    if loc.nloc < nx * ny:
        level = np.zeros((ny, nx), dtype=np.int64)
        lx, ly = loc.locx, loc.locy
        for cur in range(npad + 1):
            while True:
                found = 0
                for y in range(ny):
                    for x in range(nx):
                        if m[y, x]:
                            continue
                        count = 0
                        min_level, min_sep, min_rad = 1 << 62, 1 << 30, math.inf
                        mjx = mjy = 0
                        for jy in range(max(0, y - 1), min(ny, y + 2)):
                            for jx in range(max(0, x - 1), min(nx, x + 2)):
                                sep = abs(y - jy) + abs(x - jx)
                                iphi = abs(int(m[jy, jx]))
                                if (sep == 1 or sep == 2) and iphi:
                                    iphi -= 1
                                    rad = lx[iphi] * lx[iphi] + ly[iphi] * ly[iphi]
                                    if level[jy, jx] < min_level:
                                        min_level, min_rad, min_sep = int(level[jy, jx]), rad, sep
                                        mjy, mjx = jy, jx
                                        count = 1
                                    elif level[jy, jx] == min_level:
                                        count += 1
                                        if sep < min_sep:
                                            min_sep, mjy, mjx = sep, jy, jx
                                        elif sep == min_sep and rad < min_rad:
                                            min_rad, mjy, mjx = rad, jy, jx
                        if (min_level == cur and count == 3) or min_level < cur:
                            m[y, x] = -abs(int(m[mjy, mjx]))
                            level[y, x] = min_level + 1
                            found += 1
                if not found:
                    break
    return Loc(loc.locx, loc.locy, loc.dx, loc.ht, xmin, ymin, m)


def map_get(L: Loc, ix, iy):
    """``math/loc.h:32`` loc_map_get: 0 outside the map."""
    ny, nx = L.map.shape
    ix = np.asarray(ix)
    iy = np.asarray(iy)
    ok = (ix >= 0) & (ix < nx) & (iy >= 0) & (iy < ny)
    return np.where(ok, L.map[np.clip(iy, 0, ny - 1), np.clip(ix, 0, nx - 1)], 0)


def circle_symbolic(A: np.ndarray, cx: float, cy: float, dx: float, dy: float, r: float):
    """``math/matmath.c:556``: mark a point when it, or one of its eight
    neighbours, lies within r (the thresholds mix map and metre units exactly
    as the reference does)."""
    ny, nx = A.shape
    r2 = r * r
    r2l = (r - 1.5) * (r - 1.5)
    r2u = (r + 2.5) * (r + 2.5)
    iy = np.arange(ny)[:, None].astype(np.float64)
    ix = np.arange(nx)[None, :].astype(np.float64)
    r2r = (ix * dx - cx) * (ix * dx - cx) + (iy * dy - cy) * (iy * dy - cy)
    hit = r2r < r2l
    mid = (~hit) & (r2r < r2u)
    near = np.zeros_like(hit)
    for jy in (-1.0, 0.0, 1.0):
        iiy = iy + jy
        rr2y = (iiy * dy - cy) * (iiy * dy - cy)
        for jx in (-1.0, 0.0, 1.0):
            iix = ix + jx
            near |= ((iix * dx - cx) * (iix * dx - cx) + rr2y) <= r2
    A[hit | (mid & near)] = 1


def metapupil_loc(dirs: np.ndarray, D: float, ht: float, dx: float, offset: float, guard: float) -> Loc:
    """``math/loc.c:1471`` create_metapupil with ``square=0``, then
    ``map2loc`` (``math/loc.c:404``)."""
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
    offset = offset - math.floor(offset)
    for axis in (0, 1):
        mn = minx if axis == 0 else miny
        mind = mn / dx
        adjust = mind - math.floor(mind) - offset
        if adjust < 0:
            adjust += 1
        mn -= adjust * dx
        if axis == 0:
            minx = mn
        else:
            miny = mn
    ox, oy = minx, miny
    nx = int(math.ceil((maxx - ox) / dx)) + 1
    ny = int(math.ceil((maxy - oy) / dx)) + 1
    A = np.zeros((ny, nx))
    for k in range(dirs.shape[1]):
        tx, ty, hs = dirs[0, k], dirs[1, k], dirs[2, k]
        sx = -ox + tx * ht
        sy = -oy + ty * ht
        RR = R * (1.0 - ht / hs) + guard
        circle_symbolic(A, sx, sy, dx, dx, RR)
    iy, ix = np.nonzero(A > 1e-15)
    order = np.lexsort((ix, iy))  # y outer, x inner
    ix, iy = ix[order], iy[order]
    return Loc(ix * dx + ox, iy * dx + oy, dx, ht)


def square_loc(g: Grid) -> Loc:
    """map2loc of a full grid (every point kept)."""
    X, Y = np.meshgrid(np.arange(g.nx) * g.dx + g.ox, np.arange(g.ny) * g.dy + g.oy)
    return Loc(X.ravel(), Y.ravel(), g.dx, g.ht)


# ---------------------------------------------------------------------------
# W0 / W1 (lib/mkw.c)
# ---------------------------------------------------------------------------
NRES = 50  # lib/mkw.c:21


def _inside(px, py, icx, icy, icr2):
    return (px - icx) ** 2 + (py - icy) ** 2 < icr2


def _outside(px, py, icx, icy, icr2):
    return (px - icx) ** 2 + (py - icy) ** 2 > icr2


_D = (np.arange(NRES) + 0.5) / NRES  # sub-sample offsets in (0, 1)


def _wt_corner(ix, iy, jx, jy, icx, icy, icr):
    icr2 = icr * icr
    cs = ((ix, iy), (ix, jy), (jx, iy), (jx, jy))
    if all(_inside(a, b, icx, icy, icr2) for a, b in cs):
        return 1.0 / 36.0
    if all(_outside(a, b, icx, icy, icr2) for a, b in cs):
        return 0.0
    ddx = (jx - ix) / NRES
    ddy = (jy - iy) / NRES
    dy = ((np.arange(NRES) + 0.5) * ddy)[:, None]
    dx = ((np.arange(NRES) + 0.5) * ddx)[None, :]
    m = (ix + dx - icx) ** 2 + (iy + dy - icy) ** 2 < icr2
    w = (1.0 - np.abs(dx)) * (1.0 - np.abs(dy)) * np.abs(dx * dy)
    return float(_ordered_sum(np.where(m, w, 0.0))) / NRES / NRES


def _ordered_sum(a):
    """Row-major sequential sum (the reference's loop order)."""
    s = 0.0
    for v in np.asarray(a).ravel():
        s += v
    return s


def _wt_lr(ix, iy, jx, jy, icx, icy, icr):
    icr2 = icr * icr
    cs = ((ix, iy + 1), (ix, iy - 1), (jx, iy + 1), (jx, iy - 1))
    if all(_inside(a, b, icx, icy, icr2) for a, b in cs):
        return 1.0 / 9.0
    if all(_outside(a, b, icx, icy, icr2) for a, b in cs):
        return 0.0
    ddx = (jx - ix) / NRES
    ddy = 1.0 / NRES
    dy = ((np.arange(NRES) + 0.5) * ddy)[:, None]
    dx = ((np.arange(NRES) + 0.5) * ddx)[None, :]
    w = (1.0 - np.abs(dx)) * (1.0 - np.abs(dy)) ** 2 * np.abs(dx)
    up = (ix + dx - icx) ** 2 + (iy + dy - icy) ** 2 < icr2
    lo = (ix + dx - icx) ** 2 + (iy - dy - icy) ** 2 < icr2
    t = np.stack([np.where(up, w, 0.0), np.where(lo, w, 0.0)], axis=-1)
    return float(_ordered_sum(t)) / NRES / NRES


def _wt_ud(ix, iy, jx, jy, icx, icy, icr):
    icr2 = icr * icr
    cs = ((ix - 1, iy), (ix - 1, jy), (ix + 1, iy), (ix + 1, jy))
    if all(_inside(a, b, icx, icy, icr2) for a, b in cs):
        return 1.0 / 9.0
    if all(_outside(a, b, icx, icy, icr2) for a, b in cs):
        return 0.0
    ddy = (jy - iy) / NRES
    ddx = 1.0 / NRES
    dy = ((np.arange(NRES) + 0.5) * ddy)[:, None]
    dx = ((np.arange(NRES) + 0.5) * ddx)[None, :]
    w = (1.0 - np.abs(dx)) ** 2 * (1.0 - np.abs(dy)) * np.abs(dy)
    up = (ix + dx - icx) ** 2 + (iy + dy - icy) ** 2 < icr2
    lo = (ix - dx - icx) ** 2 + (iy + dy - icy) ** 2 < icr2
    t = np.stack([np.where(up, w, 0.0), np.where(lo, w, 0.0)], axis=-1)
    return float(_ordered_sum(t)) / NRES / NRES


def _wt_center(ix, iy, icx, icy, icr):
    icr2 = icr * icr
    cs = ((ix + 1, iy + 1), (ix + 1, iy - 1), (ix - 1, iy + 1), (ix - 1, iy - 1))
    if all(_inside(a, b, icx, icy, icr2) for a, b in cs):
        return 4.0 / 9.0
    if all(_outside(a, b, icx, icy, icr2) for a, b in cs):
        return 0.0
    d = ((np.arange(NRES) + 0.5) * (1.0 / NRES))
    dy = d[:, None]
    dx = d[None, :]
    w = ((1.0 - np.abs(dx)) * (1.0 - np.abs(dy))) ** 2
    terms = []
    for sx, sy in ((-1, -1), (1, -1), (-1, 1), (1, 1)):  # lower left, lower right, upper left, upper right
        terms.append(np.where((ix + sx * dx - icx) ** 2 + (iy + sy * dy - icy) ** 2 < icr2, w, 0.0))
    return float(_ordered_sum(np.stack(terms, axis=-1))) / NRES / NRES


def mkw_circular(L: Loc, cx: float, cy: float, cr: float):
    """``lib/mkw.c:363`` mkw_circular on loc ``L`` (its map must exist).
    Returns (W0 csc, W1)."""
    nloc = L.nloc
    idx = 1.0 / L.dx
    icx = (cx - L.mox) * idx
    icy = (cy - L.moy) * idx
    icr = cr * idx
    sc = 1.0 / (math.pi * icr ** 2)
    cache = {}
    rows, cols, vals = [], [], []
    W1 = np.zeros(nloc)
    for il in range(nloc):
        ix = int(_round_half_away((L.locx[il] - L.mox) * idx))
        iy = int(_round_half_away((L.locy[il] - L.moy) * idx))
        wt2 = 0.0
        for jy in range(iy - 1, iy + 2):
            for jx in range(ix - 1, ix + 2):
                a1 = int(map_get(L, jx, jy))
                if a1 <= 0:
                    continue
                a1 -= 1
                key = (ix, iy, jx, jy)
                if key not in cache:
                    if abs(ix - jx) == 1 and abs(iy - jy) == 1:
                        cache[key] = _wt_corner(ix, iy, jx, jy, icx, icy, icr)
                    elif abs(iy - jy) == 1:
                        cache[key] = _wt_ud(ix, iy, jx, jy, icx, icy, icr)
                    elif abs(ix - jx) == 1:
                        cache[key] = _wt_lr(ix, iy, jx, jy, icx, icy, icr)
                    else:
                        cache[key] = _wt_center(ix, iy, icx, icy, icr)
                wt = cache[key]
                if wt > 0:
                    rows.append(a1)
                    cols.append(il)
                    vals.append(wt * sc)
                wt2 += wt
        W1[il] = wt2 * sc
    W0 = sps.csc_matrix((vals, (rows, cols)), shape=(nloc, nloc))
    s1 = _ordered_sum(W1)
    if abs(s1 - 1) > 1e-12:
        W1 = W1 * (1.0 / s1)
        W0 = W0 * (1.0 / s1)
    return sps.csc_matrix(W0), W1


# ---------------------------------------------------------------------------
# ray tracing (lib/mkh.c)
# ---------------------------------------------------------------------------
def mkh(src: Loc, dstx: np.ndarray, dsty: np.ndarray, dispx: float, dispy: float, scale: float) -> sps.csr_matrix:
    """``lib/mkh.c:47`` mkh: bilinear influence of the points of ``src`` (its
    map, ghosts included through ``labs``) at the points (dstx, dsty);
    returns ndst x nsrc.  Weights at or below EPS are dropped and duplicates
    (two corners on one ghosted point) summed; no renormalisation."""
    dx_in1 = 1.0 / src.dx
    dx_in2 = scale * dx_in1
    disx = (dispx - src.mox) * dx_in1
    disy = (dispy - src.moy) * dx_in1
    fx1 = dstx * dx_in2 + disx
    fy1 = dsty * dx_in2 + disy
    nxp = np.floor(fx1).astype(np.int64)
    nyp = np.floor(fy1).astype(np.int64)
    fx1 = fx1 - nxp
    fy1 = fy1 - nyp
    fx = (1.0 - fx1, fx1)
    fy = (1.0 - fy1, fy1)
    rows, cols, vals = [], [], []
    r = np.arange(len(dstx))
    for iy in (0, 1):
        for ix in (0, 1):
            w = fx[ix] * fy[iy]
            iphi = np.abs(map_get(src, nxp + ix, nyp + iy))
            ok = (w > EPS) & (iphi > 0)
            rows.append(r[ok])
            cols.append(iphi[ok] - 1)
            vals.append(w[ok])
    H = sps.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))),
                       shape=(len(dstx), src.nloc))
    H.sum_duplicates()
    H.data[np.abs(H.data) < EPS] = 0.0
    H.eliminate_zeros()
    return H


# ---------------------------------------------------------------------------
# actuator coupling, extrapolation, slaving (lib/slaving.c)
# ---------------------------------------------------------------------------
def genactcpl(HA, W1: np.ndarray) -> List[np.ndarray]:
    """``lib/slaving.c:25`` genactcpl: HA[f][d]^T W1 summed over directions,
    then 1 where above max/nfit, else scaled by nfit/max."""
    nfit = len(HA)
    out = []
    for d in range(len(HA[0])):
        c = np.zeros(HA[0][d].shape[1])
        for f in range(nfit):
            c = c + HA[f][d].T @ W1
        thres = c.max() / nfit
        scale = 1.0 / thres if thres != 0 else 0.0
        c = np.where((c > thres) | (thres == 0), 1.0, c * scale)
        out.append(c)
    return out


_NEIGH4 = [(ix, iy) for iy in (-1, 0, 1) for ix in (-1, 0, 1) if abs(ix + iy) == 1]


def act_extrap(L: Loc, cpl: np.ndarray, thres: float) -> sps.csr_matrix:
    """``lib/slaving.c:536`` act_extrap_do: an actuator coupled below thres
    takes the coupling-weighted average of itself and its 4 neighbours above
    max(0.1, its coupling) (all 4 neighbours when none is); applied
    ceil(sqrt(nact/pi) - sqrt(sum(cpl)/pi)) + 1 times in all."""
    nact = L.nloc
    rows, cols, vals = [], [], []
    mx = _round_half_away((L.locx - L.mox) / L.dx).astype(np.int64)
    my = _round_half_away((L.locy - L.moy) / L.dx).astype(np.int64)
    for ia in range(nact):
        if cpl[ia] < thres:
            thres2 = max(0.1, cpl[ia])
            near_active = 0
            for iy in (-1, 0, 1):
                for ix in (-1, 0, 1):
                    if abs(ix) + abs(iy) == 2:
                        continue
                    k1 = int(map_get(L, mx[ia] + ix, my[ia] + iy))
                    if k1 > 0 and cpl[k1 - 1] >= thres2:
                        near_active += 1
            ent = []
            s = 0.0
            for iy in (-1, 0, 1):
                for ix in (-1, 0, 1):
                    if abs(ix) + abs(iy) == 2:
                        continue
                    k1 = int(map_get(L, mx[ia] + ix, my[ia] + iy))
                    if k1 > 0:
                        if not near_active:
                            ent.append((k1 - 1, 1.0))
                            s += 1.0
                        elif cpl[k1 - 1] >= thres2 or (ix == 0 and iy == 0):
                            ent.append((k1 - 1, cpl[k1 - 1]))
                            s += cpl[k1 - 1]
            if ent:
                scl = 1.0 / s
                for k, v in ent:
                    rows.append(ia); cols.append(k); vals.append(v * scl)
        else:
            rows.append(ia); cols.append(ia); vals.append(1.0)
    out = sps.csr_matrix((vals, (rows, cols)), shape=(nact, nact))
    nring = int(math.ceil(math.sqrt(nact / math.pi) - math.sqrt(_ordered_sum(cpl) / math.pi)))
    for _ in range(nring):
        out = (out @ out).tocsr()
    return out


def slaving(L: Loc, cpl: np.ndarray, thres: float, sclsq: float) -> Optional[sps.csr_matrix]:
    """``lib/slaving.c:63`` slaving for one DM without stuck or floating
    actuators: for each actuator coupled below thres a column of S that ties it
    to its 4 neighbours (to the better coupled ones, weighted by their
    coupling, else to all with -0.1 scl/count), self = minus the sum;
    returns S S^T, or None when no actuator is slaved."""
    scl = math.sqrt(sclsq)
    nact = L.nloc
    if not np.any(cpl < thres):
        return None
    mx = _round_half_away((L.locx - L.mox) / L.dx).astype(np.int64)
    my = _round_half_away((L.locy - L.moy) / L.dx).astype(np.int64)
    rows, cols, vals = [], [], []
    for ia in range(nact):
        if cpl[ia] >= thres:
            continue
        thres2 = max(0.1, cpl[ia])
        near_active = near_exist = 0
        for ix, iy in _NEIGH4:
            k1 = int(map_get(L, mx[ia] + ix, my[ia] + iy))
            if k1 > 0:
                near_exist += 1
                if cpl[k1 - 1] > thres2:
                    near_active += 1
        if not near_exist:
            raise ValueError("isolated actuator")
        value = -scl * 0.1 / near_exist if not near_active else 0.0
        valsum = 0.0
        for ix, iy in _NEIGH4:
            k1 = int(map_get(L, mx[ia] + ix, my[ia] + iy))
            if k1 > 0:
                if not near_active:
                    v = value
                elif cpl[k1 - 1] > cpl[ia]:
                    v = -scl * max(0.1, cpl[k1 - 1])
                else:
                    continue
                valsum += v
                rows.append(k1 - 1); cols.append(ia); vals.append(v)
        rows.append(ia); cols.append(ia); vals.append(-valsum)
    S = sps.csc_matrix((vals, (rows, cols)), shape=(nact, nact))
    return (S @ S.T).tocsr()


# ---------------------------------------------------------------------------
# the assembled fit
# ---------------------------------------------------------------------------
@dataclass
class SparseFit:
    """FR / FL of the assembled fit (DMs concatenated, layers concatenated)."""
    floc: Loc
    alocs: List[Loc]
    dm_ht: np.ndarray
    W0: sps.csc_matrix
    W1: np.ndarray
    thetax: np.ndarray
    thetay: np.ndarray
    wt: np.ndarray
    hs: np.ndarray
    actcpl: List[np.ndarray]
    actinterp: sps.csr_matrix      # nact x nact, block diagonal
    actslave: Optional[sps.csr_matrix]
    NW: np.ndarray                 # nact x nnw
    FRM: sps.csr_matrix            # nact x nxtot
    FRU: np.ndarray                # nact x nfit
    FRV: np.ndarray                # nxtot x nfit
    FLM: sps.csr_matrix            # nact x nact
    FLU: np.ndarray                # nact x (nfit + nnw)
    FLV: np.ndarray
    maxit: int
    tikcr: float
    HA0: Optional[sps.csr_matrix] = None  # nfloc x nact: HA (with actinterp) of fit direction 0

    @property
    def nact(self) -> int:
        return sum(a.nloc for a in self.alocs)

    def act_offsets(self):
        return np.concatenate([[0], np.cumsum([a.nloc for a in self.alocs])]).astype(np.int64)


def build_fit_assembled(sysm, actslave: Optional[bool] = None, actinterp: bool = True,
                        actthres: Optional[float] = None, tikcr: Optional[float] = None,
                        fit_pos: Optional[int] = None, dm_guard: int = 1) -> SparseFit:
    """The assembled fit of ``sysm`` with the reference's defaults
    (``fit.actslave = fit.actinterp = 1``, ``fit.actthres = 0.1``,
    ``fit.tikcr`` from the configuration, ``dm.guard = 1``, ``tomo.guard`` for
    floc)."""
    cfg = sysm.cfg
    tikcr = cfg.fit_tikcr if tikcr is None else tikcr
    actslave = cfg.fit_actslave if actslave is None else actslave
    actthres = cfg.fit_actthres if actthres is None else actthres
    pos = cfg.tomo_pos if fit_pos is None else fit_pos
    dirs = all_dirs(cfg)
    dxr = cfg.atmr_dx / pos
    floc = metapupil_loc(dirs, cfg.D, 0.0, dxr, 0.0, cfg.tomo_guard * dxr)
    floc = loc_create_map(floc, 1)
    W0, W1 = mkw_circular(floc, 0.0, 0.0, cfg.D / 2)
    alocs = []
    for d in cfg.dms:
        offset = d.offset + (int(round(d.order)) % 2) * 0.5
        a = metapupil_loc(dirs, cfg.D, d.ht, d.dx, offset, dm_guard * d.dx)
        alocs.append(loc_create_map(a, 1))
    nfit = len(cfg.fit_thetax)
    thetax = np.asarray(cfg.fit_thetax, dtype=np.float64)
    thetay = np.asarray(cfg.fit_thetay, dtype=np.float64)
    wt = np.asarray(cfg.fit_wt, dtype=np.float64)
    hs = np.full(nfit, math.inf)
    xlocs = [loc_create_map(square_loc(g), 0) for g in sysm.xmaps]
    # HXF (setup_recon_fit.c:26-43) and HA (:48-98)
    HXF = [[mkh(xl, floc.locx, floc.locy, thetax[f] * (xl.ht - floc.ht), thetay[f] * (xl.ht - floc.ht),
                1.0 - (xl.ht - floc.ht) / hs[f]) for xl in xlocs] for f in range(nfit)]
    HA = [[mkh(al, floc.locx, floc.locy, thetax[f] * (al.ht - floc.ht), thetay[f] * (al.ht - floc.ht),
               1.0 - (al.ht - floc.ht) / hs[f]) for al in alocs] for f in range(nfit)]
    cpl = genactcpl(HA, W1)
    ndm = len(alocs)
    interp = [act_extrap(alocs[d], cpl[d], actthres) if actinterp else None for d in range(ndm)]
    if actinterp:
        HA = [[(HA[f][d] @ interp[d]).tocsr() for d in range(ndm)] for f in range(nfit)]
    # low-rank terms (setup_recon_fit.c:106-165)
    fitscl = 1.0 / floc.nloc
    nnw = (ndm if cfg.fit_lrt_piston else 0) + (2 * (ndm - 1) if cfg.fit_lrt_tt else 0)
    off = np.concatenate([[0], np.cumsum([a.nloc for a in alocs])]).astype(np.int64)
    nact = int(off[-1])
    NW = np.zeros((nact, nnw))
    inw = 0
    if cfg.fit_lrt_piston:
        for d in range(ndm):
            NW[off[d]:off[d + 1], inw + d] = np.where(cpl[d] > 0.1, fitscl, 0.0)
        inw += ndm
    if cfg.fit_lrt_tt:
        r2 = alocs[0].locx ** 2 + alocs[0].locy ** 2
        factor = fitscl * 2.0 / (math.sqrt(r2.max()) * 2)
        for d in range(1, ndm):
            m = cpl[d] > 0.1
            NW[off[d]:off[d + 1], inw + 2 * (d - 1)] = np.where(m, alocs[d].locx * factor, 0.0)
            NW[off[d]:off[d + 1], inw + 2 * (d - 1) + 1] = np.where(m, alocs[d].locy * factor, 0.0)
    slaves = [slaving(alocs[d], cpl[d], actthres, 1.0 / floc.nloc) if actslave else None for d in range(ndm)]
    # FR (setup_recon_fit.c:204-254)
    nxl = [xl.nloc for xl in xlocs]
    FRM = sps.csr_matrix((nact, int(sum(nxl))))
    blocks = [[None] * len(xlocs) for _ in range(ndm)]
    for l in range(len(xlocs)):
        for f in range(nfit):
            if abs(wt[f]) < 1e-12:
                continue
            tmp = (W0 @ HXF[f][l]).tocsc()
            for d in range(ndm):
                t = wt[f] * (HA[f][d].T @ tmp)
                blocks[d][l] = t if blocks[d][l] is None else blocks[d][l] + t
    FRM = sps.bmat(blocks, format="csr")
    FRV = np.zeros((int(sum(nxl)), nfit))
    FRU = np.zeros((nact, nfit))
    xo = np.concatenate([[0], np.cumsum(nxl)]).astype(np.int64)
    for f in range(nfit):
        if abs(wt[f]) < 1e-12:
            continue
        s = math.sqrt(wt[f])
        for l in range(len(xlocs)):
            FRV[xo[l]:xo[l + 1], f] = (HXF[f][l].T @ W1) * s
        for d in range(ndm):
            FRU[off[d]:off[d + 1], f] = (HA[f][d].T @ W1) * s
    # FL (setup_recon_fit.c:257-293)
    fl = [[None] * ndm for _ in range(ndm)]
    for d in range(ndm):
        for f in range(nfit):
            if abs(wt[f]) < 1e-12:
                continue
            tmp = (W0 @ HA[f][d]).tocsc()
            for e in range(ndm):
                t = wt[f] * (HA[f][e].T @ tmp)
                fl[e][d] = t if fl[e][d] is None else fl[e][d] + t
    if abs(tikcr) > 1e-15:
        maxeig = 4.0 / nact
        for d in range(ndm):
            fl[d][d] = fl[d][d] + tikcr * maxeig * sps.identity(fl[d][d].shape[0])
    for d in range(ndm):
        if slaves[d] is not None:
            fl[d][d] = fl[d][d] + slaves[d]
    FLM = sps.bmat(fl, format="csr")
    FLU = np.concatenate([FRU, NW], axis=1)
    FLV = np.concatenate([FRU, -NW], axis=1)
    interp_full = sps.block_diag([interp[d] if interp[d] is not None else sps.identity(alocs[d].nloc)
                                  for d in range(ndm)], format="csr")
    slave_full = None
    if any(s is not None for s in slaves):
        slave_full = sps.block_diag([s if s is not None else sps.csr_matrix((alocs[d].nloc, alocs[d].nloc))
                                     for d, s in enumerate(slaves)], format="csr")
    HA0 = sps.hstack([HA[0][d] for d in range(ndm)]).tocsr()
    return SparseFit(floc, alocs, np.array([d.ht for d in cfg.dms]), W0, W1, thetax, thetay, wt, hs, cpl,
                     interp_full, slave_full, NW, FRM.tocsr(), FRU, FRV, FLM.tocsr(), FLU, FLV,
                     cfg.fit_maxit, tikcr, HA0)
