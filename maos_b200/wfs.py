"""Geometric Shack-Hartmann WFS on the device (``mb_geom_wfs_*``).

The simulation side upstream of the reconstruction: the gradients each WFS
measures of the atmosphere seen through the DMs (the reference's
``gpu_wfsgrad_queue`` geometric branch), so a closed loop runs on the GPU
without a host round trip::

    W = GeomWfs.for_system(sysm, atm, fit=fit, nbatch=32)
    g = W.grad(isim, dm=cmds, seed=1)     # torch float32 [nbatch, ngrad]

``atm`` is a ``turbulence.FrozenFlowAtmosphere`` (or one per instance); its
layers move by ``v dt`` per step.  ``dm`` (device float32 [nbatch, nact], in
the fit's actuator order) is subtracted.  The tables come from
``wfs_setup.build_geom_wfs``.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional, Sequence

import numpy as np

from . import native
from .native import check
from .wfs_setup import GeomWfsSystem, build_geom_wfs


def _arr(a, dt):
    return np.ascontiguousarray(np.asarray(a, dtype=dt))


class GeomWfs:
    def __init__(self, geom: GeomWfsSystem, layers: Sequence[tuple], dms: Sequence[tuple], dt: float,
                 nbatch: int = 1):
        """``layers``: (nx, ny, dx, ox, oy, ht, vx, vy) per atmosphere layer;
        ``dms``: (nx, ny, dx, ox, oy, ht) per DM."""
        import torch
        self.lib = native.load()
        self.geom = geom
        self.nbatch = int(nbatch)
        nw = geom.nwfs
        P = [geom.powfs[geom.wfs_powfs[i]] for i in range(nw)]
        # unique stencils of every WFS type, concatenated
        st_base, st_off, st_data = [], [], []
        off = 0
        for p in geom.powfs:
            st_base.append(len(st_off))
            for k in range(len(p.stencils)):
                st_off.append(off)
                st_data.append(p.stencils[k].ravel())
                off += p.stencils[k].size
        k = self._keep = {}

        def put(name, a, dt_):
            k[name] = _arr(a, dt_)
            return k[name].ctypes.data_as(C.POINTER(C.c_int if dt_ == np.int32 else
                                                   (C.c_long if dt_ == np.int64 else C.c_double)))

        d = native.MbGeomWfsDesc()
        d.nwfs = nw
        d.nsa = put("nsa", [len(p.ix0) for p in P], np.int32)
        d.nxsa = put("nxsa", [p.nxsa for p in P], np.int32)
        d.dx = put("dx", [p.dx for p in P], np.float64)
        d.gox = put("gox", [p.grid.ox for p in P], np.float64)
        d.goy = put("goy", [p.grid.oy for p in P], np.float64)
        d.thetax = put("thetax", geom.thetax, np.float64)
        d.thetay = put("thetay", geom.thetay, np.float64)
        d.hs = put("hs", geom.hs, np.float64)
        d.sa_ix = put("sa_ix", np.concatenate([p.ix0 for p in P]), np.int32)
        d.sa_iy = put("sa_iy", np.concatenate([p.iy0 for p in P]), np.int32)
        d.sa_stencil = put("sa_st", np.concatenate([p.stencil_id + st_base[geom.wfs_powfs[i]]
                                                    for i, p in enumerate(P)]), np.int32)
        d.nstencil = len(st_off)
        d.stencil_off = put("st_off", st_off, np.int64)
        d.stencils = put("stencils", np.concatenate(st_data), np.float64)
        d.stencil_len = int(off)
        d.nea = put("nea", np.concatenate([geom.nea[i].ravel() for i in range(nw)]), np.float64)
        L = list(layers)
        d.natm = len(L)
        if L:
            cols = list(zip(*L))
            d.atm_nx = put("anx", cols[0], np.int32)
            d.atm_ny = put("any", cols[1], np.int32)
            for name, j in (("atm_dx", 2), ("atm_ox", 3), ("atm_oy", 4), ("atm_ht", 5), ("atm_vx", 6), ("atm_vy", 7)):
                setattr(d, name, put(name, cols[j], np.float64))
        M = list(dms)
        d.ndm = len(M)
        if M:
            cols = list(zip(*M))
            d.dm_nx = put("dnx", cols[0], np.int32)
            d.dm_ny = put("dny", cols[1], np.int32)
            for name, j in (("dm_dx", 2), ("dm_ox", 3), ("dm_oy", 4), ("dm_ht", 5)):
                setattr(d, name, put(name, cols[j], np.float64))
        d.dt = float(dt)
        d.nbatch = self.nbatch
        h = C.c_void_p()
        check(self.lib.mb_geom_wfs_create(C.byref(d), C.byref(h)), "mb_geom_wfs_create")
        self.h = h
        self.layers = L
        self.ngrad = int(self.lib.mb_geom_wfs_ngrad(h))
        self.nact = int(self.lib.mb_geom_wfs_nact(h))
        self.out = torch.empty(self.nbatch, self.ngrad, dtype=torch.float32, device="cuda")

    @classmethod
    def for_system(cls, sysm, atm, fit=None, nbatch: int = 1, sim_dx: float = 1.0 / 64,
                   geom: Optional[GeomWfsSystem] = None) -> "GeomWfs":
        """WFS of ``sysm`` looking through the ``fit``'s DMs (none when
        ``fit`` is None) at ``atm`` (a FrozenFlowAtmosphere, or a list of
        ``nbatch`` of them with the same layer geometry)."""
        atms = list(atm) if isinstance(atm, (list, tuple)) else [atm] * nbatch
        a0 = atms[0]
        n, dx = a0.n, a0.dx
        o = -n / 2 * dx
        layers = [(n, n, dx, o, o, float(h), float(a0.vx[l]), float(a0.vy[l])) for l, h in enumerate(a0.cfg.atm_ht)]
        dms = [] if fit is None else [(dm.amap.nx, dm.amap.ny, dm.amap.dx, dm.amap.ox, dm.amap.oy, dm.ht)
                                      for dm in fit.dms]
        W = cls(geom if geom is not None else build_geom_wfs(sysm, sim_dx), layers, dms, sysm.cfg.sim_dt, nbatch)
        for i in range(nbatch):
            W.set_atmosphere(i, atms[i])
        return W

    def set_atm(self, inst: int, layer: int, screen: np.ndarray) -> None:
        s = _arr(screen, np.float64)
        check(self.lib.mb_geom_wfs_set_atm(self.h, int(inst), int(layer), s.ctypes.data_as(C.POINTER(C.c_double))),
              "mb_geom_wfs_set_atm")

    def set_wind(self, inst: int, layer: int, vx: float, vy: float) -> None:
        check(self.lib.mb_geom_wfs_set_wind(self.h, int(inst), int(layer), float(vx), float(vy)),
              "mb_geom_wfs_set_wind")

    def set_atmosphere(self, inst: int, atm) -> None:
        """Screens and winds of a FrozenFlowAtmosphere for one instance."""
        for l, s in enumerate(atm.screens):
            self.set_atm(inst, l, s)
            self.set_wind(inst, l, atm.vx[l], atm.vy[l])

    def grad(self, isim: int, dm=None, seed: int = 0, out=None, stream=None):
        """Gradients of step ``isim`` for every instance (device float32
        [nbatch, ngrad], x then y per WFS); ``dm``: device float32
        [nbatch, nact] commands or None."""
        import torch
        o = self.out if out is None else out
        st = stream if stream is not None else torch.cuda.current_stream()
        dp = C.c_void_p(dm.data_ptr()) if dm is not None else None
        check(self.lib.mb_geom_wfs_grad(self.h, int(isim), dp, C.c_void_p(o.data_ptr()), C.c_ulonglong(seed),
                                        C.c_void_p(st.cuda_stream)), "mb_geom_wfs_grad")
        return o

    def close(self) -> None:
        if getattr(self, "h", None):
            self.lib.mb_geom_wfs_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
