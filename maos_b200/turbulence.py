"""Seeded synthetic WFS gradients for benchmarks and tests.

No public dataset is involved: the reference simulates its own atmosphere.
This module stands in for ``lib/turbulence.c`` + the geometric WFS of
``maos/wfsgrad.c`` with the same physics at reduced fidelity:

* von Karman phase screens by the FFT method, one per atmosphere layer, with
  r0 scaled by the layer's Cn^2 weight (r0_l = r0 * wt_l^(-3/5)), OPD in metres
  at 500 nm;
* frozen flow: layer l moves by ``ws_l * dt`` per step in a seeded random
  direction;
* geometric gradients: the exact subaperture-average slope
  (1/dsa^2) * integral of the OPD difference across opposite edges, with the
  edges sampled at 8 points (trapezoid rule) through bilinear interpolation of
  every layer along the guide-star cone;
* additive Gaussian noise with the per-subaperture NEA of the system.
"""
from __future__ import annotations

import math
from typing import List

import numpy as np

from .config import AOConfig


def vonkarman_screen(n: int, dx: float, r0: float, L0: float, rng: np.random.Generator) -> np.ndarray:
    """n x n OPD screen (m) with a von Karman spectrum, r0 at 500 nm."""
    fx = np.fft.fftfreq(n, d=dx)
    FX, FY = np.meshgrid(fx, fx)
    f2 = FX * FX + FY * FY + 1.0 / (L0 * L0)
    psd = 0.0229 * r0 ** (-5.0 / 3.0) * f2 ** (-11.0 / 6.0)  # rad^2 m^2
    psd[0, 0] = 0.0
    df = 1.0 / (n * dx)
    c = (rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))) * np.sqrt(psd) * df
    phase = np.real(np.fft.ifft2(c)) * n * n
    return phase * 0.5e-6 / (2 * math.pi)


class FrozenFlowAtmosphere:
    def __init__(self, cfg: AOConfig, seed: int, size_m: float = 0.0):
        rng = np.random.default_rng(seed)
        self.cfg = cfg
        self.dx = cfg.atm_dx
        fov = max([math.hypot(w.thetax, w.thetay) for w in cfg.wfs] + [0.0])
        need = cfg.D + 2 * fov * max(cfg.atm_ht) + 8.0
        size = max(size_m, need * 2)
        n = 1 << int(math.ceil(math.log2(size / self.dx)))
        self.n = n
        wt = np.asarray(cfg.atm_wt, dtype=np.float64)
        wt = wt / wt.sum()
        self.screens = [vonkarman_screen(n, self.dx, cfg.r0 * w ** (-3.0 / 5.0), cfg.L0, rng) for w in wt]
        ws = cfg.atm_ws if cfg.atm_ws else [10.0] * len(wt)
        ang = rng.uniform(0, 2 * math.pi, size=len(wt))
        self.vx = np.array(ws) * np.cos(ang)
        self.vy = np.array(ws) * np.sin(ang)

    def opd(self, x: np.ndarray, y: np.ndarray, thetax: float, thetay: float, hs: float,
            t: float) -> np.ndarray:
        """OPD (m) seen along the cone toward (thetax, thetay, hs) at pupil points (x, y)."""
        out = np.zeros_like(x, dtype=np.float64)
        n = self.n
        for l, h in enumerate(self.cfg.atm_ht):
            scale = 1.0 - h / hs if math.isfinite(hs) else 1.0
            u = (x * scale + thetax * h - self.vx[l] * t) / self.dx + n / 2
            v = (y * scale + thetay * h - self.vy[l] * t) / self.dx + n / 2
            iu = np.floor(u).astype(np.int64)
            iv = np.floor(v).astype(np.int64)
            fu = u - iu
            fv = v - iv
            iu %= n
            iv %= n
            iu1 = (iu + 1) % n
            iv1 = (iv + 1) % n
            S = self.screens[l]
            out += ((1 - fu) * (1 - fv) * S[iv, iu] + fu * (1 - fv) * S[iv, iu1]
                    + (1 - fu) * fv * S[iv1, iu] + fu * fv * S[iv1, iu1])
        return out


def geometric_gradients(sysm, atm: FrozenFlowAtmosphere, t: float, rng: np.random.Generator,
                        noise: bool = True, nedge: int = 8) -> np.ndarray:
    """Average-slope gradients (rad) of every WFS of ``sysm``, x then y, plus noise."""
    out: List[np.ndarray] = []
    s = (np.arange(nedge + 1) / nedge)
    wq = np.full(nedge + 1, 1.0 / nedge)
    wq[0] = wq[-1] = 0.5 / nedge
    for w in sysm.wfs:
        dsa = w.dsa
        x0 = w.salocx[:, None]
        y0 = w.salocy[:, None]
        e = s[None, :] * dsa
        # x slope: right edge minus left edge, integrated along y
        right = atm.opd(np.broadcast_to(x0 + dsa, (w.nsa, nedge + 1)), y0 + e, w.thetax, w.thetay, w.hs, t)
        left = atm.opd(np.broadcast_to(x0, (w.nsa, nedge + 1)), y0 + e, w.thetax, w.thetay, w.hs, t)
        gx = ((right - left) * wq).sum(axis=1) / dsa
        top = atm.opd(x0 + e, np.broadcast_to(y0 + dsa, (w.nsa, nedge + 1)), w.thetax, w.thetay, w.hs, t)
        bot = atm.opd(x0 + e, np.broadcast_to(y0, (w.nsa, nedge + 1)), w.thetax, w.thetay, w.hs, t)
        gy = ((top - bot) * wq).sum(axis=1) / dsa
        g = np.concatenate([gx, gy])
        if noise:
            g = g + rng.standard_normal(g.size) * np.sqrt(w.sanea)
        out.append(g)
    return np.concatenate(out)


def gradient_frames(sysm, seed: int, nframe: int, dt: float = None, noise: bool = True) -> np.ndarray:
    """[nframe][ngrad] gradients of consecutive frozen-flow steps for one seed."""
    dt = sysm.cfg.sim_dt if dt is None else dt
    atm = FrozenFlowAtmosphere(sysm.cfg, seed)
    rng = np.random.default_rng(seed + 7919)
    return np.stack([geometric_gradients(sysm, atm, k * dt, rng, noise) for k in range(nframe)])


class DeviceAtmosphere:
    """The same frozen-flow atmosphere sampled with torch on a device (FP64):
    ``opd`` and ``gradients`` restate ``FrozenFlowAtmosphere.opd`` and
    ``geometric_gradients`` so that long gradient sequences of large systems
    take seconds instead of minutes."""

    def __init__(self, atm: FrozenFlowAtmosphere, device: str = "cuda"):
        import torch
        self.atm = atm
        self.dev = device
        self.screens = [torch.as_tensor(s, dtype=torch.float64, device=device) for s in atm.screens]

    def opd(self, x, y, thetax: float, thetay: float, hs: float, t: float):
        import torch
        a = self.atm
        out = torch.zeros_like(x, dtype=torch.float64)
        n = a.n
        for l, h in enumerate(a.cfg.atm_ht):
            scale = 1.0 - h / hs if math.isfinite(hs) else 1.0
            u = (x * scale + thetax * h - float(a.vx[l]) * t) / a.dx + n / 2
            v = (y * scale + thetay * h - float(a.vy[l]) * t) / a.dx + n / 2
            iu = torch.floor(u)
            iv = torch.floor(v)
            fu = u - iu
            fv = v - iv
            iu = iu.long() % n
            iv = iv.long() % n
            iu1 = (iu + 1) % n
            iv1 = (iv + 1) % n
            S = self.screens[l]
            out += ((1 - fu) * (1 - fv) * S[iv, iu] + fu * (1 - fv) * S[iv, iu1]
                    + (1 - fu) * fv * S[iv1, iu] + fu * fv * S[iv1, iu1])
        return out

    def gradients(self, sysm, t: float, rng: np.random.Generator, noise: bool = True, nedge: int = 8):
        """Average-slope gradients (rad) of every WFS, x then y, plus noise (host array)."""
        import torch
        s = torch.arange(nedge + 1, dtype=torch.float64, device=self.dev) / nedge
        wq = torch.full((nedge + 1,), 1.0 / nedge, dtype=torch.float64, device=self.dev)
        wq[0] = wq[-1] = 0.5 / nedge
        out = []
        for w in sysm.wfs:
            dsa = w.dsa
            x0 = torch.as_tensor(w.salocx, dtype=torch.float64, device=self.dev)[:, None]
            y0 = torch.as_tensor(w.salocy, dtype=torch.float64, device=self.dev)[:, None]
            e = s[None, :] * dsa
            shp = (w.nsa, nedge + 1)
            right = self.opd((x0 + dsa).expand(shp), y0 + e, w.thetax, w.thetay, w.hs, t)
            left = self.opd(x0.expand(shp), y0 + e, w.thetax, w.thetay, w.hs, t)
            gx = ((right - left) * wq).sum(dim=1) / dsa
            top = self.opd(x0 + e, (y0 + dsa).expand(shp), w.thetax, w.thetay, w.hs, t)
            bot = self.opd(x0 + e, y0.expand(shp), w.thetax, w.thetay, w.hs, t)
            gy = ((top - bot) * wq).sum(dim=1) / dsa
            g = torch.cat([gx, gy]).cpu().numpy()
            if noise:
                g = g + rng.standard_normal(g.size) * np.sqrt(w.sanea)
            out.append(g)
        return np.concatenate(out)
