"""Fourier-domain preconditioner (FDPCG) tables.

Restates ``maos/fdpcg.c:331-580`` (``fdpcg_prepare``).  Instead of assembling
the full sparse Fourier-domain matrix and permuting it, each bs x bs block is
built directly: a block gathers the layer frequencies that alias to one
subaperture-grid frequency, and the only couplings between them come from the
pupil frequencies that alias to the same members.  The block order and the
member order inside a block are the reference's permutation
(``fdpcg_perm``, ``maos/fdpcg.c:119``), so ``Mbinv[b]`` here equals the
reference's ``fdpcg->Mbinv->p[b]`` and ``perm`` its ``fdpcg->perm``.

Per block (complex, ``^H`` = conjugate transpose):

    M = diag(invpsd) + sum_wfs P_w^H Mmid P_w / neam_w^2,
    Mmid(f1, f2) = (conj(gx_f1) gx_f2 + conj(gy_f1) gy_f2) R(f2 - f1)
    (R: autocorrelation of the kept selection spectrum, fdpcg_saselect; with
    only its centre c kept, Mmid = c^2 (|gx|^2+|gy|^2) on the diagonal)
    (scaled by nx*ny when every layer has the same oversampling)
    Mbinv = pinv(Hermitian part of M), singular values below 1e-7 * max dropped
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np


@dataclass
class FdpcgTables:
    bs: int                 # block size = sum(os^2)
    nb: int                 # number of blocks = adim^2
    adimx: int
    adimy: int
    scale: int              # 1: FFTs are normalised by 1/sqrt(nx*ny) (cfft2s)
    perm: np.ndarray        # int64 [nb*bs]: index into the natural-order concatenated FFT of x
    Mbinv: np.ndarray       # complex128 [nb, bs, bs]
    nxtot: int
    # M before inversion, split so that a device can rebuild Mbinv after a
    # Cn2 update: the WFS (data) term, and the diagonal invpsd term at the
    # layer weights of this setup (it scales with each layer's l2c); both
    # already multiplied by nx*ny when the oversampling is uniform.
    mhat_data: np.ndarray = None   # complex128 [nb, bs, bs]
    mhat_diag: np.ndarray = None   # float64 [nb, bs]
    # The geometry a device needs to form mhat_data itself when the noise
    # changes: the pupil frequency grid, the average-gradient transfer
    # functions, the selection autocorrelation and each WFS's mean NEA.
    geom: dict = None


def _saselect(nxp, nyp, dxp, salocx, salocy, saa):
    """fdpcg_saselect (fdpcg.c:71): the clipped selection spectrum, as the
    autocorrelation of its kept coefficients.

    The selection spectrum (FFT of the full-subaperture corners on the pupil
    grid) keeps every coefficient whose magnitude reaches the zero-frequency
    one; spconvolvop (math/sp.c:926) makes it a cyclic convolution, so the
    data term's sel^H sel couples pupil frequencies i and i + d with
    R(d) = sum_s conj(v_{s+d}) v_s over the kept coefficients v.  Returns
    {(dx, dy): R} (with only the centre kept: {(0, 0): c^2})."""
    xsel = np.zeros((nyp, nxp), dtype=np.complex128)
    offx, offy = nxp // 2, nyp // 2
    for x, y, a in zip(salocx, salocy, saa):
        if a > 0.9:
            ix = int(x / dxp + offx)  # C truncation toward zero
            iy = int(y / dxp + offy)
            xsel[iy, ix] = 1.0 / (nxp * nyp)
    f = np.fft.fftshift(np.fft.fft2(np.fft.fftshift(xsel)))
    c = f[nyp // 2, nxp // 2].real
    ky, kx = np.nonzero(np.abs(f) >= c)
    R = {}
    for y1, x1 in zip(ky, kx):
        for y2, x2 in zip(ky, kx):
            d = ((x1 - x2) % nxp, (y1 - y2) % nyp)
            R[d] = R.get(d, 0) + np.conj(f[y1, x1]) * f[y2, x2]
    return R


def _fdpcg_g(nx, ny, dx, dsa):
    """Average-gradient transfer functions gx, gy on the shifted pupil grid (fdpcg.c:199)."""
    os_ = int(round(dsa / dx))
    if abs(dsa - dx * os_) > 1e-10:
        raise ValueError("dsa must be a multiple of dx")
    wt = np.full(os_ + 1, 1.0 / os_ / dsa)
    wt[0] = wt[os_] = 0.5 / os_ / dsa
    st = np.arange(os_ + 1) * dx
    fy = (np.arange(ny) - ny // 2) / (ny * dx)
    fx = (np.arange(nx) - nx // 2) / (nx * dx)
    FY, FX = np.meshgrid(fy, fx, indexing="ij")  # [iy, ix]
    cf = 2j * math.pi
    tx = np.zeros((ny, nx), np.complex128)
    ty = np.zeros((ny, nx), np.complex128)
    for k in range(os_ + 1):
        tx += wt[k] * (np.exp(cf * (FX * dsa + FY * st[k])) - np.exp(cf * (FY * st[k])))
        ty += wt[k] * (np.exp(cf * (FY * dsa + FX * st[k])) - np.exp(cf * (FX * st[k])))
    return tx, ty


def _invpsd_layer(nx, ny, dx, r0, wt, cxxscale, tomoscale):
    """Spectrum of L2^T L2 for one periodic layer (fdpcg.c:375-403), shifted order."""
    from .geometry import laplacian_coef
    cf = laplacian_coef(r0, wt, dx) * math.sqrt(cxxscale * tomoscale)
    k = np.zeros((ny, nx))
    # column 0 of L2^T L2 with L2 = cf*(-I + 0.25*(4 neighbours)), periodic
    for (ox, oy, v) in ((0, 0, 1.25), (1, 0, -0.5), (-1, 0, -0.5), (0, 1, -0.5), (0, -1, -0.5),
                        (1, 1, 0.125), (1, -1, 0.125), (-1, 1, 0.125), (-1, -1, 0.125),
                        (2, 0, 0.0625), (-2, 0, 0.0625), (0, 2, 0.0625), (0, -2, 0.0625)):
        k[oy % ny, ox % nx] += v * cf * cf
    psd = np.fft.fftshift(np.fft.fft2(k))
    mx = np.abs(psd.real).max()
    return psd.real + mx * math.sqrt(2.220446049250313e-16)


def block_members(nx, ny, os_, adimx, adimy, shift):
    """fdpcg_perm (fdpcg.c:119) with half=0: member index lists in block order."""
    nps = len(nx)
    noff = np.concatenate([[0], np.cumsum([a * b for a, b in zip(nx, ny)])])
    out = []
    blocks = []
    adimx2 = adimx // 2
    for ixh in range(2):
        ix0, ix1 = (-adimx2, 1) if ixh == 0 else (1, adimx2)
        for iy in range(-(adimy // 2), adimy // 2):
            for ix in range(ix0, ix1):
                blocks.append((ix, iy))
                for ips in range(nps):
                    for jos in range(os_[ips]):
                        jy = iy + adimy * jos
                        if shift:
                            if jy < 0:
                                jy += ny[ips]
                        else:
                            jy = jy + ny[ips] // 2
                            if jy >= ny[ips]:
                                jy -= ny[ips]
                        for ios in range(os_[ips]):
                            jx = ix + adimx * ios
                            if shift:
                                if jx < 0:
                                    jx += nx[ips]
                            else:
                                jx = jx + nx[ips] // 2
                                if jx >= nx[ips]:
                                    jx -= nx[ips]
                            out.append(noff[ips] + jx + jy * nx[ips])
    return np.array(out, dtype=np.int64), blocks


def fdpcg_prepare(sysm) -> FdpcgTables:
    from .config import TOMOSCALE
    cfg = sysm.cfg
    w0 = sysm.wfs[0]
    nps = len(sysm.xmaps)
    pos = cfg.tomo_pos
    os_ = [int(o) for o in sysm.os]
    nx = [g.nx for g in sysm.xmaps]
    ny = [g.ny for g in sysm.xmaps]
    nxp = nx[0] // os_[0] * pos
    nyp = ny[0] // os_[0] * pos
    dxp = sysm.pmap.dx
    needscale = int(any(o != os_[0] for o in os_))
    bs = sum(o * o for o in os_)
    adimx, adimy = nx[0] // os_[0], ny[0] // os_[0]
    nb = adimx * adimy
    nxtot = sum(a * b for a, b in zip(nx, ny))

    Rsel = _saselect(nxp, nyp, dxp, w0.salocx, w0.salocy, w0.saa)
    gx, gy = _fdpcg_g(nxp, nyp, dxp, w0.dsa)  # [iy, ix] shifted pupil grid
    invpsd = [_invpsd_layer(nx[i], ny[i], sysm.xmaps[i].dx, cfg.r0, sysm.wt[i],
                            cfg.tomo_cxxscale, TOMOSCALE) for i in range(nps)]
    ht = np.array(cfg.atmr_ht, dtype=np.float64)
    dkx = 1.0 / (nxp * dxp)
    dky = 1.0 / (nyp * dxp)

    perm0, blocks = block_members(nx, ny, os_, adimx, adimy, shift=0)
    perm1, _ = block_members(nx, ny, os_, adimx, adimy, shift=1)
    Mb = np.zeros((nb, bs, bs), dtype=np.complex128)
    Md = np.zeros((nb, bs, bs), dtype=np.complex128)
    Mg = np.zeros((nb, bs), dtype=np.float64)
    # member descriptors (layer, shifted jx, shifted jy) in block order
    mem_l = np.concatenate([[ips] * (os_[ips] ** 2) for ips in range(nps)])
    nxp2, nyp2 = nxp // 2, nyp // 2
    for b, (ix, iy) in enumerate(blocks):
        memb = perm0[b * bs:(b + 1) * bs]
        # decode shifted layer coordinates
        lj = []
        for m, l in zip(memb, mem_l):
            off = sum(nx[k] * ny[k] for k in range(l))
            r = m - off
            lj.append((l, r % nx[l], r // nx[l]))
        diag = np.array([invpsd[l][jy, jx] for (l, jx, jy) in lj], dtype=np.float64)
        M = np.zeros((bs, bs), dtype=np.complex128)
        # pupil frequencies aliasing to this block (centred kx = ix + adimx*m)
        # and each WFS's propagation vector from them to the block's members
        pf, pv = [], []
        for mxp in range(pos):
            for myp in range(pos):
                kx = ix + adimx * mxp
                ky = iy + adimy * myp
                kx = (kx + nxp2) % nxp - nxp2
                ky = (ky + nyp2) % nyp - nyp2
                pxi, pyi = kx + nxp2, ky + nyp2
                fxg, fyg = kx * dkx, ky * dky
                vw = []
                for w in sysm.wfs:
                    v = np.zeros(bs, np.complex128)
                    for a, (l, jx, jy) in enumerate(lj):
                        # layer frequency that pupil frequency (kx,ky) maps to
                        ljx = (kx + nx[l] // 2 + nx[l]) % nx[l]
                        ljy = (ky + ny[l] // 2 + ny[l]) % ny[l]
                        if ljx != jx or ljy != jy:
                            continue
                        fx = (jx - nx[l] // 2) * dkx
                        fy = (jy - ny[l] // 2) * dky
                        dispx = ht[l] * w.thetax
                        dispy = ht[l] * w.thetay
                        shiftv = np.exp(2j * math.pi * (fx * dispx + fy * dispy))
                        ratio = nxp // nx[l]
                        if ratio in (0, 1):
                            val = shiftv
                        elif ratio == 2:
                            val = shiftv * (1 + math.cos(2 * math.pi * fxg * dxp)) \
                                * (1 + math.cos(2 * math.pi * fyg * dxp)) * 0.5
                        else:
                            raise ValueError("unsupported layer/pupil sampling ratio")
                        v[a] = val / w.neam
                    vw.append(v)
                pf.append((pxi, pyi))
                pv.append(vw)
        # M += P^H Mmid P with Mmid(f1, f2) = sum_g conj(g_f1) g_f2 R(f2 - f1)
        for i1, (x1, y1) in enumerate(pf):
            for i2, (x2, y2) in enumerate(pf):
                r = Rsel.get(((x2 - x1) % nxp, (y2 - y1) % nyp))
                if r is None:
                    continue
                mm = (np.conj(gx[y1, x1]) * gx[y2, x2] + np.conj(gy[y1, x1]) * gy[y2, x2]) * r
                if mm == 0:
                    continue
                for k in range(len(sysm.wfs)):
                    M += np.outer(np.conj(pv[i1][k]), pv[i2][k]) * mm
        if not needscale:
            M *= nx[0] * ny[0]
            diag = diag * (nx[0] * ny[0])
        Md[b] = M
        Mg[b] = diag
        M = M + np.diag(diag)
        M = 0.5 * (M + M.conj().T)
        M[np.abs(M) < 1e-15] = 0  # cspdroptol(Mhat, EPS), EPS = 1e-15 (sys/common.h:88)
        U, s, Vh = np.linalg.svd(M)
        thr = 1e-7 * s[0]
        si = np.where(s > thr, 1.0 / np.where(s > thr, s, 1.0), 0.0)
        # reference drops all singular values from the first one under threshold
        first = np.argmax(s <= thr) if np.any(s <= thr) else len(s)
        si[first:] = 0.0
        Mb[b] = (Vh.conj().T * si) @ U.conj().T
    geom = {"nxp": nxp, "nyp": nyp, "dxp": dxp, "pos": pos, "adimx": adimx, "adimy": adimy,
            "gx": gx, "gy": gy, "sel": Rsel, "needscale": needscale,
            "neam": np.array([w.neam for w in sysm.wfs], dtype=np.float64)}
    return FdpcgTables(bs=bs, nb=nb, adimx=adimx, adimy=adimy, scale=needscale,
                       perm=perm1, Mbinv=Mb, nxtot=nxtot, mhat_data=Md, mhat_diag=Mg, geom=geom)
