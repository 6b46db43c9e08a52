"""FP64 oracle of the geometric WFS -- TEST INFRASTRUCTURE ONLY.

Restates, for the checks of the device WFS (``maos_b200/csrc/wfs.cu``):

* ``lib/accphi.c:426`` ``prop_grid``: bilinear interpolation of a square map
  at points ``(x*scale + displace - o)/d``, with wrap-around (atmosphere) or
  skipping points off the map (DMs), the ``+1`` neighbour taken as 0 at the
  last column or row;
* ``cuda/wfsgrad.cu`` geometric branch (``gpu_wfsgrad_iwfs``): OPD = the
  atmosphere along the WFS's cone (``cuda/accphi.cu:508`` ``gpu_atm2loc``:
  displacement ``ht*theta - v*dt*isim``, scale ``1 - ht/hs``) minus the DMs
  (``gpu_dm2loc``, displacement ``ht*theta``), then ``GS0 * OPD``;
* ``cuda/wfsgrad.cu:47`` ``add_geom_noise_do``: ``gx += n1*nea_xx``,
  ``gy += n2*nea_yy + n1*nea_xy`` with two standard normals per
  subaperture.  The normals come from the counter-based generator the device
  path uses (Philox4x32-10, Salmon et al., SC 2011, with a Box-Muller pair),
  restated here so the two are comparable draw by draw.

Only tests, ``smoke()`` and the CPU-baseline leg of ``bench.py`` use this.
"""
from __future__ import annotations

import math
from typing import List, Optional, Sequence

import numpy as np

_M0 = np.uint64(0xD2511F53)
_M1 = np.uint64(0xCD9E8D57)
_W0 = np.uint32(0x9E3779B9)
_W1 = np.uint32(0xBB67AE85)
_MASK = np.uint64(0xFFFFFFFF)


def philox4x32_10(ctr: np.ndarray, key: np.ndarray) -> np.ndarray:
    """Philox4x32 with 10 rounds: ``ctr`` [..., 4] uint32, ``key`` [..., 2]
    uint32 -> [..., 4] uint32 (the published round function: two 32x32->64
    multiplies, the high halves xor-ed with the other counter words and the
    key, the key bumped by the Weyl constants between rounds)."""
    c = [np.asarray(ctr[..., i], dtype=np.uint64) for i in range(4)]
    k0 = np.asarray(key[..., 0], dtype=np.uint32).copy()
    k1 = np.asarray(key[..., 1], dtype=np.uint32).copy()
    for r in range(10):
        p0 = _M0 * c[0]
        p1 = _M1 * c[2]
        hi0, lo0 = p0 >> np.uint64(32), p0 & _MASK
        hi1, lo1 = p1 >> np.uint64(32), p1 & _MASK
        c = [(hi1 ^ c[1] ^ k0.astype(np.uint64)) & _MASK, lo1, (hi0 ^ c[3] ^ k1.astype(np.uint64)) & _MASK, lo0]
        if r < 9:
            k0 = (k0 + _W0).astype(np.uint32)
            k1 = (k1 + _W1).astype(np.uint32)
    return np.stack([x.astype(np.uint32) for x in c], axis=-1)


def geom_normals(seed: int, isim: int, iwfs: int, inst: int, nsa: int):
    """The two standard normals per subaperture the device draws: counter
    (isa, iwfs, isim, inst), key (seed low, seed high), Box-Muller on the
    first two words mapped to (0, 1]."""
    isa = np.arange(nsa, dtype=np.uint64)
    ctr = np.zeros((nsa, 4), dtype=np.uint32)
    ctr[:, 0] = isa.astype(np.uint32)
    ctr[:, 1] = np.uint32(iwfs)
    ctr[:, 2] = np.uint32(isim & 0xFFFFFFFF)
    ctr[:, 3] = np.uint32(inst)
    key = np.array([seed & 0xFFFFFFFF, (seed >> 32) & 0xFFFFFFFF], dtype=np.uint32)
    out = philox4x32_10(ctr, np.broadcast_to(key, (nsa, 2)))
    u1 = (out[:, 0].astype(np.float64) + 1.0) * 2.0 ** -32
    u2 = out[:, 1].astype(np.float64) * 2.0 ** -32
    r = np.sqrt(-2.0 * np.log(u1))
    return r * np.cos(2 * math.pi * u2), r * np.sin(2 * math.pi * u2)


def prop_grid(screen: np.ndarray, ox: float, oy: float, dx: float, x: np.ndarray, y: np.ndarray, alpha: float,
              dispx: float, dispy: float, scale: float, wrap: bool) -> np.ndarray:
    """``alpha * bilinear(screen)`` at points (x, y) as ``lib/accphi.c:426``
    computes it; ``screen`` is [ny, nx] (x fastest)."""
    ny, nx = screen.shape
    dx1 = 1.0 / dx
    dx2 = scale * dx1
    bx = (dispx - ox) * dx1
    by = (dispy - oy) * dx1
    u = x * dx2 + bx
    v = y * dx2 + by
    iu = np.floor(u).astype(np.int64)
    iv = np.floor(v).astype(np.int64)
    fu = u - iu
    fv = v - iv
    out = np.zeros(x.shape, dtype=np.float64)
    if wrap:
        iu = np.mod(iu, nx)
        iv = np.mod(iv, ny)
        ok = np.ones(x.shape, dtype=bool)
    else:
        ok = (iu >= 0) & (iu <= nx - 1) & (iv >= 0) & (iv <= ny - 1)
    iu, iv, fu, fv = iu[ok], iv[ok], fu[ok], fv[ok]
    iu1 = np.where(iu == nx - 1, 0, iu + 1)
    iv1 = np.where(iv == ny - 1, 0, iv + 1)
    m00 = screen[iv, iu]
    m10 = screen[iv, iu1]
    m01 = screen[iv1, iu]
    m11 = screen[iv1, iu1]
    out[ok] = alpha * ((m00 + (m10 - m00) * fu) * (1.0 - fv) + (m01 + (m11 - m01) * fu) * fv)
    return out


class Screen:
    """A square map with its origin, spacing and height (and wind, for an
    atmosphere layer)."""

    def __init__(self, data: np.ndarray, ox: float, oy: float, dx: float, ht: float, vx: float = 0.0,
                 vy: float = 0.0):
        self.data = np.asarray(data, dtype=np.float64)
        self.ox, self.oy, self.dx, self.ht, self.vx, self.vy = ox, oy, dx, ht, vx, vy


def wfs_opd(geom, iwfs: int, atm: Sequence[Screen], dms: Sequence[Screen], isim: int, dt: float) -> np.ndarray:
    """OPD of WFS ``iwfs`` on its fine grid ([ny, nx]), atmosphere minus DMs."""
    P = geom.powfs[geom.wfs_powfs[iwfs]]
    g = P.grid
    X, Y = np.meshgrid(g.ox + np.arange(g.nx) * g.dx, g.oy + np.arange(g.ny) * g.dy)
    x, y = X.ravel(), Y.ravel()
    tx, ty, hs = float(geom.thetax[iwfs]), float(geom.thetay[iwfs]), float(geom.hs[iwfs])
    opd = np.zeros(x.size)
    for s in atm:
        scale = 1.0 - s.ht / hs if math.isfinite(hs) else 1.0
        opd += prop_grid(s.data, s.ox, s.oy, s.dx, x, y, 1.0, s.ht * tx - s.vx * dt * isim,
                         s.ht * ty - s.vy * dt * isim, scale, True)
    for s in dms:
        scale = 1.0 - s.ht / hs if math.isfinite(hs) else 1.0
        opd += prop_grid(s.data, s.ox, s.oy, s.dx, x, y, -1.0, s.ht * tx, s.ht * ty, scale, False)
    return opd.reshape(g.ny, g.nx)


def geom_noise(geom, seed: int, isim: int, inst: int = 0) -> np.ndarray:
    """The noise the device adds to every WFS's gradients (x then y)."""
    out = []
    for iw in range(geom.nwfs):
        nsa = geom.nsa(iw)
        n1, n2 = geom_normals(seed, isim, iw, inst, nsa)
        nea = geom.nea[iw]
        out.append(np.concatenate([n1 * nea[0], n2 * nea[1] + n1 * nea[2]]))
    return np.concatenate(out)


def geom_grads(geom, atm: Sequence[Screen], dms: Sequence[Screen], isim: int, dt: float, seed: int = 0,
               inst: int = 0, gs0: Optional[List] = None) -> np.ndarray:
    """Gradients of every WFS, x then y per WFS: GS0 * OPD, plus the noise
    when ``seed`` is non-zero."""
    out = []
    for iw in range(geom.nwfs):
        G = gs0[geom.wfs_powfs[iw]] if gs0 is not None else geom.powfs[geom.wfs_powfs[iw]].gs0()
        out.append(G @ wfs_opd(geom, iw, atm, dms, isim, dt).ravel())
    g = np.concatenate(out)
    return g + geom_noise(geom, seed, isim, inst) if seed else g
