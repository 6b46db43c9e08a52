"""AO system descriptions for the reconstruction hot path.

A configuration names the telescope, the wavefront sensors (WFS), the
reconstructed atmosphere layers, the DM-fit directions and the DMs, in the
units the MAOS reference uses (metres, radians, seconds).  The presets are the
three system types the benchmarks use:

* ``ltao_8m``   -- 8 m LTAO, 4 sodium LGS on a 10" ring, 20x20 subapertures,
                   2 layers on a 0.2 m grid, plain CG (30 iterations).
* ``mcao_30m``  -- 30 m NFIRAOS-like MCAO, 6 LGS (35" pentagon + centre),
                   60x60 subapertures, 6 layers on 0.5 m / 1.0 m grids,
                   FDPCG (30 iterations), 2 DMs, 9 fit directions.
* ``scao_8m``   -- 8 m SCAO, one on-axis NGS, 20x20 subapertures.

Parameter names follow the reference's configuration keys
(``config/maos/recon.conf``, ``shwfs_lgs.conf``, ``dm_dual.conf``,
``fit_sq34.conf``, ``atm_mk13n50p.conf``) so a value can be traced back.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Optional, Tuple

import math

AS2RAD = math.pi / 180.0 / 3600.0
TOMOSCALE = 1e-12  # maos/maos.c:30 -- scales saneai and L2^2 for FP32 range


@dataclass
class PowfsSpec:
    """One WFS type (reference ``powfs.*`` keys)."""

    order: int                 # subapertures across the pupil
    dsa: float                 # subaperture size (m)
    hs: float                  # guide star range (m); inf for NGS
    nearecon_mas: float = 20.0 # NEA used in reconstruction, milli-arcsec
    nea_range_as: Optional[Tuple[float, float]] = None  # per-subaperture uniform NEA (arcsec)
    trs: bool = True           # tip/tilt removal (LGS)
    saat: float = 0.3          # relative-area threshold to keep a subaperture
    dtrat: int = 1


@dataclass
class WfsSpec:
    powfs: int
    thetax: float  # rad
    thetay: float  # rad


@dataclass
class DmSpec:
    ht: float      # conjugation height (m)
    dx: float      # actuator pitch (m)
    order: int     # actuators across
    offset: float = 0.0  # fractional grid offset (dm.offset)


@dataclass
class AOConfig:
    name: str
    D: float
    din: float
    powfs: List[PowfsSpec]
    wfs: List[WfsSpec]
    # reconstructed layers (atmr.*)
    atmr_dx: float
    atmr_ht: List[float]
    atmr_wt: List[float]
    atmr_os: List[int]
    r0: float
    L0: float
    # simulated atmosphere (atm.*) used by the synthetic gradient generator
    atm_ht: List[float]
    atm_wt: List[float]
    atm_ws: List[float] = field(default_factory=list)
    atm_dx: float = 1.0 / 16
    # tomography (tomo.*)
    tomo_pos: int = 2
    tomo_guard: int = 1
    tomo_maxit: int = 30
    tomo_precond: int = 1      # 0: CG, 1: FDPCG
    tomo_cxxscale: float = 1.0
    # DM fit (fit.*)
    fit_thetax: List[float] = field(default_factory=lambda: [0.0])
    fit_thetay: List[float] = field(default_factory=lambda: [0.0])
    fit_wt: List[float] = field(default_factory=lambda: [1.0])
    fit_maxit: int = 4
    fit_tikcr: float = 1e-7
    fit_lrt_piston: bool = True
    fit_lrt_tt: bool = True
    fit_actslave: bool = True     # slave weakly coupled actuators (fit.actslave)
    fit_actthres: float = 0.1     # coupling below which an actuator is slaved (fit.actthres)
    dms: List[DmSpec] = field(default_factory=list)
    sim_dt: float = 1.0 / 800
    seed: int = 1
    grad_noise: bool = True

    @property
    def npsr(self) -> int:
        return len(self.atmr_ht)

    @property
    def nwfs(self) -> int:
        return len(self.wfs)


def ltao_8m(seed: int = 1) -> AOConfig:
    """8 m LTAO: 4 LGS at 90 km on a 10" ring, 20x20 x 0.4 m, 2 layers, 1 DM 21x21."""
    lgs = PowfsSpec(order=20, dsa=0.4, hs=90e3, nearecon_mas=50.0, trs=True)
    wfs = [WfsSpec(0, 10 * AS2RAD * math.cos(a), 10 * AS2RAD * math.sin(a))
           for a in (0.0, 0.5 * math.pi, math.pi, 1.5 * math.pi)]
    return AOConfig(
        name="ltao_8m", D=8.0, din=0.1, powfs=[lgs], wfs=wfs,
        atmr_dx=0.4, atmr_ht=[0.0, 10e3], atmr_wt=[0.7, 0.3], atmr_os=[2, 2],
        r0=0.15, L0=30.0, atm_ht=[0.0, 10e3], atm_wt=[0.7, 0.3], atm_ws=[10.0, 20.0],
        atm_dx=0.2, tomo_pos=2, tomo_maxit=30, tomo_precond=0,
        fit_thetax=[0.0], fit_thetay=[0.0], fit_wt=[1.0], fit_maxit=4,
        fit_lrt_tt=False,
        dms=[DmSpec(ht=0.0, dx=0.4, order=21)], seed=seed)


def mcao_30m(seed: int = 1) -> AOConfig:
    """30 m NFIRAOS-like MCAO with FDPCG (sizes quoted in the module docstring)."""
    lgs = PowfsSpec(order=60, dsa=0.5, hs=90e3, nea_range_as=(0.02, 0.1), trs=True)
    wfs = [WfsSpec(0, 0.0, 0.0)]
    for k in range(5):
        a = 0.5 * math.pi + 2 * math.pi * k / 5
        wfs.append(WfsSpec(0, 35 * AS2RAD * math.cos(a), 35 * AS2RAD * math.sin(a)))
    fx = [0, 0.5, 0, -0.5, 0, 0.5, -0.5, -0.5, 0.5]
    fy = [0, 0, 0.5, 0, -0.5, 0.5, 0.5, -0.5, -0.5]
    fw = [4 / 9, 1 / 9, 1 / 9, 1 / 9, 1 / 9, 1 / 36, 1 / 36, 1 / 36, 1 / 36]
    atm_ht = [0.0, 500.0, 1000.0, 2000.0, 4000.0, 8000.0, 16000.0]
    atm_wt = [0.4557, 0.1295, 0.0442, 0.0506, 0.1167, 0.0926, 0.1107]
    # 6 reconstructed layers: the 4 km layer is split between its neighbours.
    atmr_ht = [0.0, 500.0, 1000.0, 2000.0, 8000.0, 16000.0]
    atmr_wt = [0.4557, 0.1295, 0.0442, 0.0506 + 0.1167 / 2, 0.0926 + 0.1167 / 2, 0.1107]
    return AOConfig(
        name="mcao_30m", D=30.0, din=3.6, powfs=[lgs], wfs=wfs,
        atmr_dx=1.0, atmr_ht=atmr_ht, atmr_wt=atmr_wt, atmr_os=[2, 2, 1, 1, 1, 1],
        r0=0.186, L0=30.0, atm_ht=atm_ht, atm_wt=atm_wt,
        atm_ws=[5.6, 5.77, 6.25, 7.57, 13.31, 19.06, 12.14], atm_dx=0.25,
        tomo_pos=2, tomo_maxit=30, tomo_precond=1,
        fit_thetax=[v * 34 * AS2RAD for v in fx], fit_thetay=[v * 34 * AS2RAD for v in fy],
        fit_wt=fw, fit_maxit=4,
        dms=[DmSpec(ht=0.0, dx=0.5, order=63), DmSpec(ht=11.2e3, dx=0.5, order=76, offset=0.5)],
        seed=seed)


def scao_8m(seed: int = 1) -> AOConfig:
    """8 m SCAO with one on-axis NGS (no tip/tilt removal), 20x20 x 0.4 m."""
    ngs = PowfsSpec(order=20, dsa=0.4, hs=math.inf, nearecon_mas=20.0, trs=False)
    return AOConfig(
        name="scao_8m", D=8.0, din=0.1, powfs=[ngs], wfs=[WfsSpec(0, 0.0, 0.0)],
        atmr_dx=0.4, atmr_ht=[0.0], atmr_wt=[1.0], atmr_os=[2],
        r0=0.15, L0=30.0, atm_ht=[0.0, 10e3], atm_wt=[0.7, 0.3], atm_ws=[10.0, 20.0],
        atm_dx=0.2, tomo_pos=2, tomo_maxit=30, tomo_precond=0,
        fit_lrt_tt=False, dms=[DmSpec(ht=0.0, dx=0.4, order=21)], seed=seed)


def elt_39m(seed: int = 1) -> AOConfig:
    """39 m ELT-like MCAO for the large control-matrix build: 6 LGS at 90 km on a
    45" hexagon, 80x80 x 0.4875 m, 9 reconstructed layers at 0-20 km
    (0.4875 m grids at 0 and 0.5 km, 0.975 m above), 3 DMs at 0, 4 and 12.7 km."""
    lgs = PowfsSpec(order=80, dsa=39.0 / 80, hs=90e3, nea_range_as=(0.02, 0.1), trs=True)
    wfs = [WfsSpec(0, 45 * AS2RAD * math.cos(math.pi * k / 3), 45 * AS2RAD * math.sin(math.pi * k / 3))
           for k in range(6)]
    fx = [0, 0.5, 0, -0.5, 0, 0.5, -0.5, -0.5, 0.5]
    fy = [0, 0, 0.5, 0, -0.5, 0.5, 0.5, -0.5, -0.5]
    fw = [4 / 9, 1 / 9, 1 / 9, 1 / 9, 1 / 9, 1 / 36, 1 / 36, 1 / 36, 1 / 36]
    ht = [0.0, 500.0, 1000.0, 2000.0, 4000.0, 8000.0, 12000.0, 16000.0, 20000.0]
    wt = [0.45, 0.13, 0.05, 0.05, 0.09, 0.09, 0.06, 0.05, 0.03]
    return AOConfig(
        name="elt_39m", D=39.0, din=4.0, powfs=[lgs], wfs=wfs,
        atmr_dx=0.975, atmr_ht=ht, atmr_wt=wt, atmr_os=[2, 2, 1, 1, 1, 1, 1, 1, 1],
        r0=0.186, L0=30.0, atm_ht=ht, atm_wt=wt,
        atm_ws=[5.6, 5.8, 6.3, 7.6, 13.3, 19.1, 15.0, 12.1, 10.0], atm_dx=0.25,
        tomo_pos=2, tomo_maxit=30, tomo_precond=1,
        fit_thetax=[v * 40 * AS2RAD for v in fx], fit_thetay=[v * 40 * AS2RAD for v in fy],
        fit_wt=fw, fit_maxit=4,
        dms=[DmSpec(ht=0.0, dx=39.0 / 80, order=81), DmSpec(ht=4e3, dx=39.0 / 80, order=85, offset=0.5),
             DmSpec(ht=12.7e3, dx=0.975, order=49)],
        seed=seed)


PRESETS = {"ltao_8m": ltao_8m, "mcao_30m": mcao_30m, "scao_8m": scao_8m, "elt_39m": elt_39m}
