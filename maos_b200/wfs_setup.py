"""Tables of the geometric Shack-Hartmann WFS on the simulation side.

The reference builds, per WFS type (``maos/setup_powfs.c``):

* ``pts`` / ``loc`` (lines 256-335): ``nx = 2*round(dsa/(2*powfs.dx))``
  OPD points across each subaperture, spacing ``dx = dsa/nx``, at
  ``saloc + dx/2 + i*dx`` (cell centres), concatenated per subaperture;
* ``amp`` (line 337, ``maos/utils.c:446`` ``mkamp`` without an amplitude map):
  ``locannular`` (``math/loc.c:815-862``), the fraction of each point's cell
  inside the annulus, by 10 x 10 supersampling of cells near the edge;
* ``GS0`` (line 565): ``mkg(loc, loc, amp, saloc, 1, 0, 0, 1)``, the average
  gradient of each subaperture (``lib/mkg.c:109-452``).

Here the points of all subapertures are laid on one square fine grid with two
empty rings around them (amplitude zero off the subapertures' points, which
is how ``mkg`` sees a point that is not in ``loc``), and ``GS0`` is stored as
one dense stencil per subaperture over the ``(nx+2)^2`` grid points it
touches: its own ``nx^2`` points and the adjacent ring, whose half cells lie
inside the subaperture.  Subapertures with the same amplitude neighbourhood
have bit-identical stencils; those are stored once (a 30 m pupil of 2,900
subapertures needs a few hundred).
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import List

import numpy as np
import scipy.sparse as sps

from .geometry import Grid

_TOL = 5e-16     # lib/mkg.c:52
_EPS = 1e-15     # sys/common.h EPS (locannular's inner-radius test)


def loccircle(phi: np.ndarray, x: np.ndarray, y: np.ndarray, dx: float, cx: float, cy: float, r: float,
              val: float) -> None:
    """phi += val x (fraction of each point's dx-cell inside the circle).

    Restates ``math/loc.c:815`` (``loccircle``): points well inside get the
    full value; points within 1.5 cells of the edge are supersampled 10 x 10."""
    nres = 10
    cres = (nres - 1.0) / 2.0
    res = 1.0 / nres
    dxres = res * dx
    res2 = res * res
    r2 = r * r
    r2l = (r - dx * 1.5) * (r - dx * 1.5)
    r2u = (r + dx * 1.5) * (r + dx * 1.5)
    r2r = (x - cx) ** 2 + (y - cy) ** 2
    inner = r2r < r2l
    phi[inner] += val
    edge = np.nonzero(~inner & (r2r < r2u))[0]
    if edge.size:
        xe = x[edge][:, None, None]
        ye = y[edge][:, None, None]
        k = np.arange(nres, dtype=np.float64)
        iiy = ye + (k[None, :, None] - cres) * dxres
        rr2y = (iiy - cy) * (iiy - cy)
        iix = xe + (k[None, None, :] - cres) * dxres
        rr2r = (iix - cx) * (iix - cx) + rr2y
        tot = np.count_nonzero(rr2r <= r2, axis=(1, 2))
        phi[edge] += tot.astype(np.float64) * res2 * val


def locannular(x: np.ndarray, y: np.ndarray, dx: float, r: float, rin: float) -> np.ndarray:
    """``math/loc.c:857`` ``locannular`` centred on the origin with value 1."""
    phi = np.zeros(x.shape, dtype=np.float64)
    loccircle(phi, x, y, dx, 0.0, 0.0, r, 1.0)
    if rin > _EPS:
        loccircle(phi, x, y, dx, 0.0, 0.0, rin, -1.0)
    return phi


def _ceil_t(a: np.ndarray) -> np.ndarray:
    r = np.round(a)
    return np.where(np.abs(a - r) < _TOL, r, np.ceil(a)).astype(np.int64)


def _floor_t(a: np.ndarray) -> np.ndarray:
    r = np.round(a)
    return np.where(np.abs(a - r) < _TOL, r, np.floor(a)).astype(np.int64)


def _quad_weights(a1: np.ndarray, a2: np.ndarray):
    """BOUND0/BOUND1 and the four integral weights of ``lib/mkg.c`` DO_CALC."""
    a1 = np.maximum(a1, 0.0)
    a2 = np.minimum(a2, 1.0)
    ok = ~((a1 > 1.0 - _TOL) | (a2 < -_TOL))
    w0 = (a2 * a2 - a1 * a1) * 0.5 - (a2 ** 3 - a1 ** 3) / 3
    w1 = ((1 - a1) ** 3 - (1 - a2) ** 3) / 3
    w2 = (a2 * a2 - a1 * a1) * 0.5
    w3 = (a2 - a1) - (a2 * a2 - a1 * a1) * 0.5
    return ok, (w0, w1, w2, w3)


def gs0_stencils(amp: np.ndarray, ix0: np.ndarray, iy0: np.ndarray, salocx: np.ndarray, salocy: np.ndarray,
                 dsa: float, dx: float, nxsa: int):
    """Average-gradient stencils of every subaperture: ``[nsa, 2, W*W]`` with
    ``W = nxsa + 2`` (x weights, then y), window row-major from grid point
    ``(ix0-1, iy0-1)``.

    Restates ``lib/mkg.c:mkgt`` for ``xloc == ploc`` (``same``), ``scale=1``,
    no displacement, ``do_partial=1``, vectorised over subapertures: for every
    point of the window and each of its four quadrants inside the subaperture,
    the bilinear influence integrated over the quadrant, weighted by the 3x3
    amplitude neighbourhood (quadrants with a zero corner skipped), summed in
    the reference's quadrant order; rows normalised by the illuminated area
    (zero under 1 % of a full subaperture).  ``amp`` is the fine grid's
    amplitude ``[ny, nx]``; ``ix0, iy0`` the grid index of each subaperture's
    first point.  The loc map origin the reference uses is the lowest point,
    ``min(saloc) + dx/2``."""
    nsa = len(salocx)
    W = nxsa + 2
    dp1 = 1.0 / dx
    dsa2 = dsa / 2.0 * dp1
    amp_thres = dsa2 * dsa2 * 4 * 0.01
    xmin = float(np.min(salocx)) + dx * 0.5
    ymin = float(np.min(salocy)) + dx * 0.5
    pox = (0.0 - xmin) * dp1 + dsa2
    poy = (0.0 - ymin) * dp1 + dsa2
    scx = salocx * dp1 + pox
    scy = salocy * dp1 + poy
    limx1, limx2 = scx - dsa2, scx + dsa2
    limy1, limy2 = scy - dsa2, scy + dsa2
    mx0 = _ceil_t(limx1) - 1
    my0 = _ceil_t(limy1) - 1
    if np.any(_floor_t(limx2) + 1 - mx0 + 1 != W) or np.any(_floor_t(limy2) + 1 - my0 + 1 != W):
        raise ValueError("subaperture window is not (nxsa+2) points wide")
    # map index m of the reference's loc map is grid index m + (ix0 of the lowest subaperture)
    gx = ix0 - (int(np.min(ix0)) + 0)
    if np.any(mx0 + 1 != gx) or np.any(my0 + 1 != iy0 - int(np.min(iy0))):
        raise ValueError("fine grid is not aligned with the subapertures")
    a = np.arange(W)
    limx = (mx0[:, None] + a[None, :]).astype(np.float64)   # [nsa, W]
    limy = (my0[:, None] + a[None, :]).astype(np.float64)
    # 3x3 amplitude neighbourhoods: A[n, j, i] = amp at grid (iy0-2+j, ix0-2+i)
    jj = (iy0[:, None] - 2 + np.arange(W + 2)[None, :])
    ii = (ix0[:, None] - 2 + np.arange(W + 2)[None, :])
    A = amp[jj[:, :, None], ii[:, None, :]]                 # [nsa, W+2, W+2]
    xq = [(limx - limx2[:, None], limx - limx1[:, None], 0, 1.0),
          (limx1[:, None] - limx, limx2[:, None] - limx, 2, -1.0)]
    yq = [(limy - limy2[:, None], limy - limy1[:, None], 0, 1.0),
          (limy1[:, None] - limy, limy2[:, None] - limy, 2, -1.0)]
    yw = [(_quad_weights(b1, b2), i0, sg) for b1, b2, i0, sg in yq]
    xw = [(_quad_weights(a1, a2), i0, sg) for a1, a2, i0, sg in xq]
    wx = np.zeros((nsa, W, W))
    wy = np.zeros((nsa, W, W))
    ampsum_pt = np.zeros((nsa, W, W))
    A11 = A[:, 1:1 + W, 1:1 + W]
    for (okx, wa), ix_, signx in xw:
        for (oky, wb), iy_, signy in yw:
            A00 = A[:, iy_:iy_ + W, ix_:ix_ + W]
            A01 = A[:, iy_:iy_ + W, 1:1 + W]
            A10 = A[:, 1:1 + W, ix_:ix_ + W]
            m = (okx[:, None, :] & oky[:, :, None]
                 & (np.abs(A00) > _TOL) & (np.abs(A01) > _TOL) & (np.abs(A10) > _TOL) & (np.abs(A11) > _TOL))
            wa_ = [w[:, None, :] for w in wa]
            wb_ = [w[:, :, None] for w in wb]
            cx = ((wb_[0] * A00 + wb_[1] * A10) * wa_[2] + (wb_[0] * A01 + wb_[1] * A11) * wa_[3]) * dp1 * signx
            cy = ((wb_[2] * A00 + wb_[3] * A10) * wa_[0] + (wb_[2] * A01 + wb_[3] * A11) * wa_[1]) * dp1 * signy
            wx = np.where(m, wx + cx, wx)
            wy = np.where(m, wy + cy, wy)
            ampsum_pt = np.where(m, ampsum_pt + wa_[3] * wb_[3] * A11, ampsum_pt)
    ampsum = ampsum_pt.reshape(nsa, -1).sum(axis=1)
    norm = np.where(ampsum > amp_thres, 1.0 / np.where(ampsum > 0, ampsum, 1.0), 0.0)
    wx = np.where(np.abs(wx) > _TOL, wx, 0.0) * norm[:, None, None]
    wy = np.where(np.abs(wy) > _TOL, wy, 0.0) * norm[:, None, None]
    st = np.stack([wx.reshape(nsa, -1), wy.reshape(nsa, -1)], axis=1)
    st[np.abs(st) < 1e-14] = 0.0   # dspdroptol(GS0, 1e-14)
    return st


@dataclass
class GeomPowfs:
    """One WFS type's fine grid, amplitude and gradient stencils."""
    nxsa: int                 # OPD points across a subaperture
    dx: float                 # their spacing
    dsa: float
    grid: Grid                # fine grid (two empty rings around the points)
    amp: np.ndarray           # [ny, nx] amplitude on the grid, zero off the points
    ix0: np.ndarray           # int32 [nsa]: grid index of each subaperture's first point
    iy0: np.ndarray
    stencil_id: np.ndarray    # int32 [nsa]
    stencils: np.ndarray      # [nst, 2, (nxsa+2)^2] unique stencils

    @property
    def W(self) -> int:
        return self.nxsa + 2

    def gs0(self) -> sps.csr_matrix:
        """The (2 nsa) x (grid points) average-gradient operator, x rows first."""
        nsa = len(self.ix0)
        W = self.W
        r, c = np.divmod(np.arange(W * W), W)
        cols = ((self.iy0[:, None] - 1 + r[None, :]) * self.grid.nx + (self.ix0[:, None] - 1 + c[None, :]))
        st = self.stencils[self.stencil_id]          # [nsa, 2, W*W]
        rows = np.concatenate([np.repeat(np.arange(nsa), W * W), np.repeat(np.arange(nsa) + nsa, W * W)])
        G = sps.csr_matrix((np.concatenate([st[:, 0].ravel(), st[:, 1].ravel()]),
                            (rows, np.concatenate([cols.ravel(), cols.ravel()]))), shape=(2 * nsa, self.grid.n))
        G.eliminate_zeros()
        return G


def build_geom_powfs(salocx: np.ndarray, salocy: np.ndarray, dsa: float, sim_dx: float, D: float,
                     din: float) -> GeomPowfs:
    """Fine grid, amplitude and stencils of one WFS type (subaperture lower-left
    corners ``salocx, salocy``, size ``dsa``, requested OPD spacing ``sim_dx``)."""
    nxsa = 2 * int(round(0.5 * dsa / sim_dx))
    dx = dsa / nxsa
    pad = 2
    x0 = float(np.min(salocx)) + 0.5 * dx
    y0 = float(np.min(salocy)) + 0.5 * dx
    kx = np.rint((salocx - np.min(salocx)) / dx).astype(np.int64)
    ky = np.rint((salocy - np.min(salocy)) / dx).astype(np.int64)
    nx = int(kx.max()) + nxsa + 2 * pad
    ny = int(ky.max()) + nxsa + 2 * pad
    grid = Grid(nx, ny, dx, dx, x0 - pad * dx, y0 - pad * dx)
    ix0 = (kx + pad).astype(np.int32)
    iy0 = (ky + pad).astype(np.int32)
    # the subapertures' points, at the coordinates the reference computes
    # (pts origin saloc + dx/2, then + i*dx)
    nsa = len(salocx)
    k = np.arange(nxsa)
    px = (salocx + dx * 0.5)[:, None, None] + (k * dx)[None, None, :] + 0 * k[None, :, None]
    py = (salocy + dx * 0.5)[:, None, None] + (k * dx)[None, :, None] + 0 * k[None, None, :]
    a = locannular(px.ravel(), py.ravel(), dx, D * 0.5, din * 0.5).reshape(nsa, nxsa, nxsa)
    amp = np.zeros((ny, nx))
    gi = (iy0[:, None, None] + k[None, :, None]) * nx + (ix0[:, None, None] + k[None, None, :])
    amp.ravel()[gi.ravel()] = a.ravel()
    st = gs0_stencils(amp, ix0.astype(np.int64), iy0.astype(np.int64), np.asarray(salocx, dtype=np.float64),
                      np.asarray(salocy, dtype=np.float64), dsa, dx, nxsa)
    flat = np.ascontiguousarray(st.reshape(nsa, -1))
    uniq, inv = np.unique(flat.view(np.dtype((np.void, flat.dtype.itemsize * flat.shape[1]))).ravel(),
                          return_inverse=True)
    first = np.zeros(len(uniq), dtype=np.int64)
    first[inv[::-1]] = np.arange(nsa)[::-1]
    stencils = st[first]
    return GeomPowfs(nxsa, dx, dsa, grid, amp, ix0, iy0, inv.astype(np.int32).ravel(), stencils)


@dataclass
class GeomWfsSystem:
    """Every WFS of a system: its type's tables, direction and noise."""
    powfs: List[GeomPowfs]
    wfs_powfs: List[int]
    thetax: np.ndarray
    thetay: np.ndarray
    hs: np.ndarray
    nea: List[np.ndarray]     # per WFS [3, nsa]: sqrt-NEA xx, yy, xy (rad)

    @property
    def nwfs(self) -> int:
        return len(self.wfs_powfs)

    def nsa(self, iwfs: int) -> int:
        return len(self.powfs[self.wfs_powfs[iwfs]].ix0)

    @property
    def ngrad(self) -> int:
        return sum(2 * self.nsa(i) for i in range(self.nwfs))

    def g_offsets(self) -> np.ndarray:
        return np.concatenate([[0], np.cumsum([2 * self.nsa(i) for i in range(self.nwfs)])]).astype(np.int64)


def build_geom_wfs(sysm, sim_dx: float = 1.0 / 64) -> GeomWfsSystem:
    """Geometric WFS tables for every WFS of a tomography system.  The
    subapertures are the reconstructor's own (``sysm.wfs``); the OPD spacing
    is ``powfs.dx`` (1/64 m in the reference's Shack-Hartmann configurations,
    ``config/maos/shwfs_lgs.conf:6``)."""
    cfg = sysm.cfg
    key = {}
    powfs: List[GeomPowfs] = []
    wp: List[int] = []
    for iw, w in enumerate(sysm.wfs):
        ip = cfg.wfs[iw].powfs
        if ip not in key:
            key[ip] = len(powfs)
            powfs.append(build_geom_powfs(w.salocx, w.salocy, w.dsa, sim_dx, cfg.D, cfg.din))
        wp.append(key[ip])
    nea = []
    for w in sysm.wfs:
        s = np.sqrt(np.asarray(w.sanea, dtype=np.float64))
        nea.append(np.stack([s[:w.nsa], s[w.nsa:], np.zeros(w.nsa)]))
    return GeomWfsSystem(powfs, wp, np.array([w.thetax for w in sysm.wfs]), np.array([w.thetay for w in sysm.wfs]),
                         np.array([w.hs for w in sysm.wfs]), nea)
