"""Bridge to the compiled reference CPU path -- TEST INFRASTRUCTURE ONLY.

``oracle/_ref/libmaosref.so`` is the MAOS reference's own CPU reconstruction
(sys/, math/, lib/, maos/ compiled from its sources by ``oracle/ref/Makefile``)
plus a flat driver (``oracle/ref/ref_driver.c``).  It is loaded in a separate
process started with ``spawn``: the reference installs signal handlers and its
own OpenMP runtime at load time, and it reads ``$HOME``; the worker runs in
``oracle/_ref/home`` with ``HOME=.`` so nothing is written outside the
repository.

Only tests, ``smoke()`` and the CPU-baseline leg of ``bench.py`` use this.
"""
from __future__ import annotations

import ctypes
import multiprocessing as mp
import os
from typing import Any

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_ref", "libmaosref.so")
GLUE_LIB = os.path.join(HERE, "_ref", "libmaosgpuglue.so")


def available() -> bool:
    return os.path.exists(LIB)


# --------------------------------------------------------------------------
# worker side
# --------------------------------------------------------------------------
_D = ctypes.POINTER(ctypes.c_double)
_I = ctypes.POINTER(ctypes.c_int)
_L = ctypes.POINTER(ctypes.c_long)


def _dp(a):
    return np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(_D)


class _Worker:
    def __init__(self, nthread: int):
        self.lib = ctypes.CDLL(LIB)
        L = self.lib
        L.ref_new.restype = ctypes.c_void_p
        L.ref_new.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int]
        for name in ("ref_set_system", "ref_set_pmap", "ref_set_layer", "ref_set_wfs", "ref_set_neam",
                     "ref_finalize", "ref_get_ptt", "ref_tomoR", "ref_tomoL", "ref_hx",
                     "ref_fdpcg_prepare", "ref_fdpcg_get", "ref_fdpcg_set", "ref_fdpcg_precond",
                     "ref_tomo_pcg"):
            getattr(L, name).restype = ctypes.c_int
        L.ref_tomo_pcg.restype = ctypes.c_double
        L.ref_mkg.restype = ctypes.c_long
        self.nthread = nthread
        self.h = None
        self.keep = []

    def setup(self, d):
        L = self.lib
        h = L.ref_new(d["nwfs"], d["nps"], self.nthread)
        self.h = ctypes.c_void_p(h)
        L.ref_set_system(self.h, ctypes.c_double(d["r0"]), ctypes.c_double(d["cxxscale"]),
                         ctypes.c_double(d["dt"]), d["pos"], d["split"], d["precond"], d["maxit"])
        p = d["pmap"]
        L.ref_set_pmap(self.h, p[0], p[1], ctypes.c_double(p[2]), ctypes.c_double(p[3]),
                       ctypes.c_double(p[4]))
        for i, lay in enumerate(d["layers"]):
            nx, ny, dx, ox, oy, ht, wt, os_ = lay
            L.ref_set_layer(self.h, i, nx, ny, ctypes.c_double(dx), ctypes.c_double(ox),
                            ctypes.c_double(oy), ctypes.c_double(ht), ctypes.c_double(wt), os_)
        for i, w in enumerate(d["wfs"]):
            arrs = [np.ascontiguousarray(w[k], dtype=np.float64) for k in
                    ("salocx", "salocy", "saa", "gp_x", "saneai", "sanea")]
            gp_p = np.ascontiguousarray(w["gp_p"], dtype=np.int32)
            gp_i = np.ascontiguousarray(w["gp_i"], dtype=np.int32)
            self.keep += arrs + [gp_p, gp_i]
            L.ref_set_wfs(self.h, i, ctypes.c_double(w["thetax"]), ctypes.c_double(w["thetay"]),
                          ctypes.c_double(w["hs"]), w["nsa"], ctypes.c_double(w["dsa"]),
                          arrs[0].ctypes.data_as(_D), arrs[1].ctypes.data_as(_D),
                          arrs[2].ctypes.data_as(_D), gp_p.ctypes.data_as(_I),
                          gp_i.ctypes.data_as(_I), arrs[3].ctypes.data_as(_D),
                          arrs[4].ctypes.data_as(_D), arrs[5].ctypes.data_as(_D), int(w["trs"]))
            L.ref_set_neam(self.h, i, ctypes.c_double(w["neam"]))
        L.ref_finalize(self.h)
        self.nx = d["nxtot"]
        self.ng = d["ngrad"]
        self.np = d["pmap"][0] * d["pmap"][1]
        self.nsa = [w["nsa"] for w in d["wfs"]]
        return True

    def ptt(self, iwfs):
        out = np.zeros(4 * self.nsa[iwfs])
        n = self.lib.ref_get_ptt(self.h, iwfs, out.ctypes.data_as(_D))
        return None if n < 0 else out.reshape(2, 2 * self.nsa[iwfs], order="F").copy()

    def tomoR(self, g, alpha=1.0):
        out = np.zeros(self.nx)
        self.lib.ref_tomoR(self.h, _dp(g), ctypes.c_double(alpha), out.ctypes.data_as(_D))
        return out

    def tomoL(self, x, alpha=1.0):
        out = np.zeros(self.nx)
        self.lib.ref_tomoL(self.h, _dp(x), ctypes.c_double(alpha), out.ctypes.data_as(_D))
        return out

    def hx(self, iwfs, x):
        out = np.zeros(self.np)
        self.lib.ref_hx(self.h, iwfs, _dp(x), out.ctypes.data_as(_D))
        return out

    def fdpcg_prepare(self):
        nb = ctypes.c_long(0)
        bs = ctypes.c_long(0)
        scale = self.lib.ref_fdpcg_prepare(self.h, ctypes.byref(nb), ctypes.byref(bs))
        nb, bs = nb.value, bs.value
        mb = np.zeros(nb * bs * bs * 2)
        perm = np.zeros(nb * bs, dtype=np.int64)
        self.lib.ref_fdpcg_get(self.h, mb.ctypes.data_as(_D), perm.ctypes.data_as(_L))
        mbc = (mb[0::2] + 1j * mb[1::2]).reshape(nb, bs, bs).transpose(0, 2, 1)  # col-major blocks
        return {"scale": scale, "Mbinv": mbc, "perm": perm}

    def fdpcg_set(self, Mbinv, perm, scale):
        nb, bs, _ = Mbinv.shape
        cm = np.ascontiguousarray(Mbinv.transpose(0, 2, 1)).ravel()
        mb = np.empty(cm.size * 2)
        mb[0::2] = cm.real
        mb[1::2] = cm.imag
        pm = np.ascontiguousarray(perm, dtype=np.int64)
        self.keep += [mb, pm]
        self.lib.ref_fdpcg_set(self.h, ctypes.c_long(nb), ctypes.c_long(bs), mb.ctypes.data_as(_D),
                               pm.ctypes.data_as(_L), int(scale))
        return True

    def fdpcg_precond(self, r):
        out = np.zeros(self.nx)
        self.lib.ref_fdpcg_precond(self.h, _dp(r), out.ctypes.data_as(_D))
        return out

    def pcg(self, b, x0, warm, maxit, precond):
        x = np.array(x0, dtype=np.float64) if x0 is not None else np.zeros(self.nx)
        res = self.lib.ref_tomo_pcg(self.h, _dp(b), x.ctypes.data_as(_D), int(warm), int(maxit),
                                    int(precond))
        return x, res

    def mkg(self, grid, amp, salocx, salocy, dsa):
        L = self.lib
        nnz = L.ref_mkg(grid[0], grid[1], ctypes.c_double(grid[2]), ctypes.c_double(grid[3]),
                        ctypes.c_double(grid[4]), _dp(amp), len(salocx), ctypes.c_double(dsa),
                        _dp(salocx), _dp(salocy))
        ncol = grid[0] * grid[1]
        p = np.zeros(ncol + 1, dtype=np.int32)
        i = np.zeros(nnz, dtype=np.int32)
        x = np.zeros(nnz)
        nr = ctypes.c_long(0)
        nc = ctypes.c_long(0)
        L.ref_mkg_get(p.ctypes.data_as(_I), i.ctypes.data_as(_I), x.ctypes.data_as(_D),
                      ctypes.byref(nr), ctypes.byref(nc))
        return p, i, x, nr.value, nc.value

    def wfs_gs0(self, salocx, salocy, dsa, nx, D, din):
        """The reference's WFS pts loc, amplitude and GS0 (CSC) for one powfs."""
        L = self.lib
        L.ref_wfs_gs0.restype = ctypes.c_long
        nsa = len(salocx)
        nnz = L.ref_wfs_gs0(nsa, ctypes.c_double(dsa), int(nx), _dp(salocx), _dp(salocy), ctypes.c_double(D),
                            ctypes.c_double(din))
        nloc = nsa * nx * nx
        lx = np.zeros(nloc)
        ly = np.zeros(nloc)
        amp = np.zeros(nloc)
        p = np.zeros(nloc + 1, dtype=np.int32)
        i = np.zeros(nnz, dtype=np.int32)
        x = np.zeros(nnz)
        nr = ctypes.c_long(0)
        nc = ctypes.c_long(0)
        L.ref_wfs_gs0_get(lx.ctypes.data_as(_D), ly.ctypes.data_as(_D), amp.ctypes.data_as(_D),
                          p.ctypes.data_as(_I), i.ctypes.data_as(_I), x.ctypes.data_as(_D),
                          ctypes.byref(nr), ctypes.byref(nc))
        self._wfs_ng = int(nr.value)
        return lx, ly, amp, p, i, x, nr.value, nc.value

    def prop_grid(self, grid, screen, locx, locy, alpha, dispx, dispy, scale, wrap, out=None):
        """out + prop_grid(screen on grid (nx, ny, dx, ox, oy), points) of the reference."""
        out = np.zeros(len(locx)) if out is None else np.array(out, dtype=np.float64)
        self.lib.ref_prop_grid(int(grid[0]), int(grid[1]), ctypes.c_double(grid[2]), ctypes.c_double(grid[3]),
                               ctypes.c_double(grid[4]), _dp(np.asarray(screen).ravel()), ctypes.c_long(len(locx)),
                               _dp(locx), _dp(locy), ctypes.c_double(alpha), ctypes.c_double(dispx),
                               ctypes.c_double(dispy), ctypes.c_double(scale), int(wrap), out.ctypes.data_as(_D))
        return out

    def wfs_geom_grads(self, thetax, thetay, hs, maps, dt, isim, nthread=None):
        """Geometric gradients [nwfs, 2 nsa] of the powfs last built by
        wfs_gs0: maps = [(data [ny, nx], dx, ox, oy, ht, vx, vy, alpha, wrap)]."""
        L = self.lib
        nw = len(thetax)
        i32 = lambda a: np.ascontiguousarray(a, dtype=np.int32)
        f64 = lambda a: np.ascontiguousarray(a, dtype=np.float64)
        nx = i32([m[0].shape[1] for m in maps])
        ny = i32([m[0].shape[0] for m in maps])
        cols = [f64([m[k] for m in maps]) for k in range(1, 8)]
        wrap = i32([m[8] for m in maps])
        scr = f64(np.concatenate([np.ascontiguousarray(m[0], dtype=np.float64).ravel() for m in maps]))
        th = [f64(thetax), f64(thetay), f64(hs)]
        out = np.zeros(nw * self._wfs_ng)
        L.ref_wfs_geom_grads(nw, th[0].ctypes.data_as(_D), th[1].ctypes.data_as(_D), th[2].ctypes.data_as(_D),
                             len(maps), nx.ctypes.data_as(_I), ny.ctypes.data_as(_I),
                             *[c.ctypes.data_as(_D) for c in cols], wrap.ctypes.data_as(_I),
                             scr.ctypes.data_as(_D), ctypes.c_double(dt), ctypes.c_long(isim),
                             int(nthread or self.nthread), out.ctypes.data_as(_D))
        return out.reshape(nw, self._wfs_ng)

    def fit_setup(self, fd):
        L = self.lib
        keep = []

        def d(a):
            a = np.ascontiguousarray(a, dtype=np.float64)
            keep.append(a)
            return a.ctypes.data_as(_D)

        def i32(a):
            a = np.ascontiguousarray(a, dtype=np.int32)
            keep.append(a)
            return a.ctypes.data_as(_I)

        L.ref_fit_setup(self.h, fd["nfit"], d(fd["thetax"]), d(fd["thetay"]), d(fd["wt"]),
                        d(fd["hs"]), fd["nf"], i32(fd["w0_p"]), i32(fd["w0_i"]), d(fd["w0_x"]),
                        d(fd["w1"]), fd["ndm"], d(fd["dmht"]), d(fd["dmdx"]), i32(fd["nact"]),
                        d(fd["alocx"]), d(fd["alocy"]), fd["nnw"], d(fd["nw"]))
        self.keep += keep
        self.na = int(np.sum(fd["nact"]))
        self.nfit = fd["nfit"]
        return True

    def fit_setup_slave(self, thres=0.1):
        """Add the reference's own slaving term (genactcpl + slaving) to the grid fit."""
        self.lib.ref_fit_setup_slave.argtypes = [ctypes.c_double]
        return bool(self.lib.ref_fit_setup_slave(ctypes.c_double(thres)))

    def fitR(self, x, alpha=1.0):
        out = np.zeros(self.na)
        self.lib.ref_fitR(self.h, _dp(x), ctypes.c_double(alpha), out.ctypes.data_as(_D))
        return out

    def fitL(self, a, alpha=1.0):
        out = np.zeros(self.na)
        self.lib.ref_fitL(self.h, _dp(a), ctypes.c_double(alpha), out.ctypes.data_as(_D))
        return out

    def fit_pcg(self, b, a0, warm, maxit):
        a = np.array(a0, dtype=np.float64) if a0 is not None else np.zeros(self.na)
        self.lib.ref_fit_pcg.restype = ctypes.c_double
        res = self.lib.ref_fit_pcg(self.h, _dp(b), a.ctypes.data_as(_D), int(warm), int(maxit))
        return a, res

    def fit_ha(self, f, d, nrow, ncol):
        L = self.lib
        L.ref_fit_ha.restype = ctypes.c_long
        nnz = L.ref_fit_ha(f, d, None, None, None)
        p = np.zeros(ncol + 1, dtype=np.int32)
        i = np.zeros(nnz, dtype=np.int32)
        x = np.zeros(nnz)
        L.ref_fit_ha(f, d, p.ctypes.data_as(_I), i.ctypes.data_as(_I), x.ctypes.data_as(_D))
        return p, i, x

    # assembled fit (fit.square=0): metapupil locs, loc maps, mkw_circular, setup_fit
    def metapupil(self, dirs, D, ht, dx, offset, guard, square=0):
        L = self.lib
        L.ref_metapupil.restype = ctypes.c_long
        dd = np.asfortranarray(dirs, dtype=np.float64)
        n = L.ref_metapupil(dd.shape[1], dd.ctypes.data_as(_D), ctypes.c_double(D), ctypes.c_double(ht),
                            ctypes.c_double(dx), ctypes.c_double(offset), ctypes.c_double(guard), int(square))
        x = np.zeros(n)
        y = np.zeros(n)
        L.ref_metapupil_get(x.ctypes.data_as(_D), y.ctypes.data_as(_D))
        return x, y

    def loc_map(self, x, y, dx, npad):
        L = self.lib
        nx, ny = ctypes.c_long(), ctypes.c_long()
        ox, oy = ctypes.c_double(), ctypes.c_double()
        L.ref_loc_map(ctypes.c_long(len(x)), _dp(x), _dp(y), ctypes.c_double(dx), int(npad), ctypes.byref(nx),
                      ctypes.byref(ny), ctypes.byref(ox), ctypes.byref(oy))
        m = np.zeros(nx.value * ny.value, dtype=np.int64)
        L.ref_loc_map_get(m.ctypes.data_as(_L))
        return m.reshape(ny.value, nx.value), ox.value, oy.value

    def mkw_circular(self, x, y, dx, npad, cx, cy, cr):
        L = self.lib
        L.ref_mkw_circular.restype = ctypes.c_long
        nnz = L.ref_mkw_circular(ctypes.c_long(len(x)), _dp(x), _dp(y), ctypes.c_double(dx), int(npad),
                                 ctypes.c_double(cx), ctypes.c_double(cy), ctypes.c_double(cr))
        n = len(x)
        p = np.zeros(n + 1, dtype=np.int32)
        i = np.zeros(nnz, dtype=np.int32)
        xv = np.zeros(nnz)
        w1 = np.zeros(n)
        L.ref_mkw_amp_get(p.ctypes.data_as(_I), i.ctypes.data_as(_I), xv.ctypes.data_as(_D),
                          w1.ctypes.data_as(_D))
        return p, i, xv, w1

    def fit_assemble(self, fd):
        """The reference's setup_fit on the given floc, W0/W1 and aloc."""
        L = self.lib
        keep = []

        def d(a):
            a = np.ascontiguousarray(a, dtype=np.float64)
            keep.append(a)
            return a.ctypes.data_as(_D)

        def i32(a):
            a = np.ascontiguousarray(a, dtype=np.int32)
            keep.append(a)
            return a.ctypes.data_as(_I)

        L.ref_fit_assemble(self.h, fd["nfit"], d(fd["thetax"]), d(fd["thetay"]), d(fd["wt"]), d(fd["hs"]),
                           ctypes.c_long(fd["nf"]), d(fd["flocx"]), d(fd["flocy"]), ctypes.c_double(fd["fdx"]),
                           i32(fd["w0_p"]), i32(fd["w0_i"]), d(fd["w0_x"]), d(fd["w1"]), fd["ndm"],
                           d(fd["dmht"]), d(fd["dmdx"]), i32(fd["nact"]), d(fd["alocx"]), d(fd["alocy"]),
                           int(fd["actslave"]), int(fd["actinterp"]), ctypes.c_double(fd["actthres"]),
                           ctypes.c_double(fd["tikcr"]), int(fd["lrt_piston"]), int(fd["lrt_tt"]))
        self.keep += keep
        self.na = int(np.sum(fd["nact"]))
        return True

    def fitas_sparse(self, which):
        """0 FR.M, 1 FL.M, 2 actinterp, 3 actslave as (p, i, x, nrow, ncol) CSC, or None."""
        L = self.lib
        L.ref_fitas_sp.restype = ctypes.c_long
        nr, nc = ctypes.c_long(), ctypes.c_long()
        nnz = L.ref_fitas_sp(int(which), None, None, None, ctypes.byref(nr), ctypes.byref(nc))
        if nnz < 0:
            return None
        p = np.zeros(nc.value + 1, dtype=np.int32)
        i = np.zeros(nnz, dtype=np.int32)
        x = np.zeros(nnz)
        L.ref_fitas_sp(int(which), p.ctypes.data_as(_I), i.ctypes.data_as(_I), x.ctypes.data_as(_D),
                       ctypes.byref(nr), ctypes.byref(nc))
        return p, i, x, nr.value, nc.value

    def fitas_dense(self, which):
        """0 FR.U, 1 FR.V, 2 FL.U, 3 FL.V, 4 actcpl, 5 NW (column-major), or None."""
        L = self.lib
        L.ref_fitas_dense.restype = ctypes.c_long
        nr, nc = ctypes.c_long(), ctypes.c_long()
        n = L.ref_fitas_dense(int(which), None, ctypes.byref(nr), ctypes.byref(nc))
        if n < 0:
            return None
        out = np.zeros(n)
        L.ref_fitas_dense(int(which), out.ctypes.data_as(_D), ctypes.byref(nr), ctypes.byref(nc))
        return out.reshape((nr.value, nc.value), order="F")

    def fitas_rhs(self, x):
        out = np.zeros(self.na)
        self.lib.ref_fitas_rhs(self.h, _dp(x), out.ctypes.data_as(_D))
        return out

    def fitas_L(self, a):
        out = np.zeros(self.na)
        self.lib.ref_fitas_L(_dp(a), out.ctypes.data_as(_D))
        return out

    def fitas_pcg(self, b, a0, warm, maxit):
        a = np.array(a0, dtype=np.float64) if a0 is not None else np.zeros(self.na)
        self.lib.ref_fitas_pcg.restype = ctypes.c_double
        res = self.lib.ref_fitas_pcg(_dp(b), a.ctypes.data_as(_D), int(warm), int(maxit))
        return a, res

    def mkw_amp(self, grid, amp):
        L = self.lib
        L.ref_mkw_amp.restype = ctypes.c_long
        nnz = L.ref_mkw_amp(grid[0], grid[1], ctypes.c_double(grid[2]), ctypes.c_double(grid[3]),
                            ctypes.c_double(grid[4]), _dp(amp))
        n = grid[0] * grid[1]
        p = np.zeros(n + 1, dtype=np.int32)
        i = np.zeros(nnz, dtype=np.int32)
        x = np.zeros(nnz)
        w1 = np.zeros(n)
        L.ref_mkw_amp_get(p.ctypes.data_as(_I), i.ctypes.data_as(_I), x.ctypes.data_as(_D),
                          w1.ctypes.data_as(_D))
        return p, i, x, w1

    def loc_coords(self, grid):
        n = grid[0] * grid[1]
        x = np.zeros(n)
        y = np.zeros(n)
        self.lib.ref_loc_coords(grid[0], grid[1], ctypes.c_double(grid[2]), ctypes.c_double(grid[3]),
                                ctypes.c_double(grid[4]), x.ctypes.data_as(_D), y.ctypes.data_as(_D))
        return x, y


    # the gpu_* glue (maos_b200/glue/maos_gpu_glue.c) on RECON_T built by the reference
    def glue_prepare(self, gpu_fit, tomo_maxit, fit_maxit):
        """PARMS_T / RECON_T / SIM_T as maos holds them after setup (no GPU needed)."""
        L = self.lib
        V = ctypes.c_void_p
        L.ref_glue_prepare.restype = ctypes.c_int
        nd = L.ref_glue_prepare(self.h, int(gpu_fit), int(tomo_maxit), int(fit_maxit))
        if nd < 0:
            raise RuntimeError("no fit set up in the reference driver")
        L.ref_glue_grad_cell.restype = V
        L.ref_glue_grad_cell.argtypes = [V, _D]
        L.ref_glue_cell_get.restype = ctypes.c_long
        L.ref_glue_cell_get.argtypes = [V, _D]
        L.ref_glue_cell_free.argtypes = [V]
        L.ref_glue_cpu_step.restype = ctypes.c_double
        L.ref_glue_cpu_step.argtypes = [V, _D]
        L.ref_glue_dm_cell.restype = V
        L.ref_glue_dm_cell.argtypes = [V, ctypes.c_int]
        hs = (V * 4)()
        L.ref_glue_handles(self.h, hs)
        self.gh = [V(v) for v in hs]  # parms, powfs, recon, simu
        self.glue_grid = int(gpu_fit) == 2
        return nd

    def glue_setup(self):
        """Load the glue and run gpu_init + gpu_setup_recon (needs a GPU)."""
        V = ctypes.c_void_p
        G = ctypes.CDLL(GLUE_LIB)
        G.gpu_init.restype = ctypes.c_int
        G.gpu_init.argtypes = [V, ctypes.POINTER(ctypes.c_int), ctypes.c_int]
        G.gpu_setup_recon.argtypes = [V, V, V]
        G.gpu_tomo.argtypes = [V, V]
        G.gpu_fit.argtypes = [ctypes.POINTER(V), V]
        G.gpu_recon_reset.argtypes = [V]
        G.gpu_setup_recon_mvm.argtypes = [V, V, V]
        G.gpu_recon_mvm.argtypes = [ctypes.POINTER(V), V]
        self.glue = G
        if not G.gpu_init(self.gh[0], None, 0):
            raise RuntimeError("gpu_init found no GPU")
        G.gpu_setup_recon(self.gh[0], self.gh[1], self.gh[2])
        self.dm_cell = V(0)
        return True

    def _cell_out(self, c):
        L = self.lib
        n = L.ref_glue_cell_get(c, None)
        out = np.zeros(n)
        L.ref_glue_cell_get(c, out.ctypes.data_as(_D))
        return out

    def glue_step(self, g):
        """gpu_tomo then gpu_fit of one step; the DM commands."""
        L, G = self.lib, self.glue
        c = ctypes.c_void_p(L.ref_glue_grad_cell(self.h, _dp(g)))
        G.gpu_tomo(self.gh[3], c)
        G.gpu_fit(ctypes.byref(self.dm_cell), self.gh[3])
        L.ref_glue_cell_free(c)
        return self._cell_out(self.dm_cell)

    def glue_cpu_step(self, g):
        """The reference's own CPU tomofit of one step on its own SIM_T."""
        L = self.lib
        c = ctypes.c_void_p(L.ref_glue_grad_cell(self.h, _dp(g)))
        out = np.zeros(self.na)
        res = L.ref_glue_cpu_step(c, out.ctypes.data_as(_D))
        L.ref_glue_cell_free(c)
        return out, res

    def glue_reset(self):
        self.glue.gpu_recon_reset(self.gh[0])

    def glue_mvm(self, M, g):
        """gpu_setup_recon_mvm with recon->MVM = M, then gpu_recon_mvm(g)."""
        L, G = self.lib, self.glue
        Mf = np.asfortranarray(M, dtype=np.float64)
        L.ref_glue_set_mvm(self.h, Mf.ctypes.data_as(_D), ctypes.c_long(Mf.shape[0]), ctypes.c_long(Mf.shape[1]))
        G.gpu_setup_recon_mvm(self.gh[0], self.gh[2], self.gh[1])
        dm = ctypes.c_void_p(L.ref_glue_dm_cell(self.h, int(self.glue_grid)))
        c = ctypes.c_void_p(L.ref_glue_grad_cell(self.h, _dp(g)))
        G.gpu_recon_mvm(ctypes.byref(dm), c)
        out = self._cell_out(dm)
        L.ref_glue_cell_free(c)
        L.ref_glue_cell_free(dm)
        return out

    def glue_cleanup(self):
        self.glue.gpu_cleanup()
        return True

    # .bin files through the reference's writebin / read_by_id (maos_b200.binio checks)
    def bin_write_dmat(self, fn, a, header=""):
        a = np.asfortranarray(a, dtype=np.float64)
        L = self.lib
        L.ref_bin_write_dmat.argtypes = [ctypes.c_char_p, _D, ctypes.c_long, ctypes.c_long, ctypes.c_char_p]
        return L.ref_bin_write_dmat(fn.encode(), a.ctypes.data_as(_D), a.shape[0], a.shape[1], header.encode())

    def bin_write_dcell3(self, fn, a, b):
        a = np.asfortranarray(a, dtype=np.float64)
        b = np.asfortranarray(b, dtype=np.float64)
        L = self.lib
        L.ref_bin_write_dcell3.argtypes = [ctypes.c_char_p, _D, ctypes.c_long, ctypes.c_long, _D, ctypes.c_long,
                                           ctypes.c_long]
        return L.ref_bin_write_dcell3(fn.encode(), a.ctypes.data_as(_D), a.shape[0], a.shape[1],
                                      b.ctypes.data_as(_D), b.shape[0], b.shape[1])

    def bin_read_dmat(self, fn, cap=1 << 20):
        L = self.lib
        L.ref_bin_read_dmat.restype = ctypes.c_long
        buf = np.empty(cap)
        nx, ny = ctypes.c_long(), ctypes.c_long()
        hdr = ctypes.create_string_buffer(4096)
        n = L.ref_bin_read_dmat(fn.encode(), buf.ctypes.data_as(_D), ctypes.c_long(cap), ctypes.byref(nx),
                                ctypes.byref(ny), hdr, ctypes.c_long(4096))
        if n < 0:
            raise ValueError("array larger than the buffer")
        return buf[:n].reshape((nx.value, ny.value), order="F").copy(), hdr.value.decode()

    def bin_read_dcell(self, fn, cap=1 << 20, kcap=64):
        L = self.lib
        L.ref_bin_read_dcell.restype = ctypes.c_long
        buf = np.empty(cap)
        nx = (ctypes.c_long * kcap)()
        ny = (ctypes.c_long * kcap)()
        nc = ctypes.c_long()
        n = L.ref_bin_read_dcell(fn.encode(), buf.ctypes.data_as(_D), ctypes.c_long(cap), ctypes.byref(nc), nx, ny,
                                 ctypes.c_long(kcap))
        if n < 0:
            raise ValueError("cell larger than the buffer")
        out, off = [], 0
        for k in range(nc.value):
            m = nx[k] * ny[k]
            out.append(buf[off:off + m].reshape((nx[k], ny[k]), order="F").copy() if m else None)
            off += m
        return out


    # servo_new / servo_filter (lib/servo.c): commands after each of the given errors
    def servo_run(self, merrs, ap, al, dt, ep):
        L = self.lib
        L.ref_servo_new.restype = ctypes.c_void_p
        L.ref_servo_new.argtypes = [ctypes.c_long, _D, ctypes.c_int, ctypes.c_int, ctypes.c_double, _D, ctypes.c_int,
                                    ctypes.c_int]
        L.ref_servo_filter.argtypes = [ctypes.c_void_p, _D, ctypes.c_long, _D]
        L.ref_servo_free.argtypes = [ctypes.c_void_p]
        merrs = np.ascontiguousarray(merrs, dtype=np.float64)
        nstep, n = merrs.shape
        apv = np.ascontiguousarray(ap if ap is not None else np.zeros(1), dtype=np.float64)
        epm = np.asfortranarray(ep, dtype=np.float64)
        h = L.ref_servo_new(n, apv.ctypes.data_as(_D), 0 if ap is None else len(apv), al, dt, epm.ctypes.data_as(_D),
                            epm.shape[0], epm.shape[1])
        out = np.empty((nstep, n))
        for k in range(nstep):
            row = np.ascontiguousarray(merrs[k])
            L.ref_servo_filter(ctypes.c_void_p(h), row.ctypes.data_as(_D), n, out[k].ctypes.data_as(_D))
        L.ref_servo_free(ctypes.c_void_p(h))
        return out


def _serve(conn, nthread, home):
    # The reference formats $HOME/.aos/... into a 64-byte buffer
    # (math/fft.c fnwisdom); run from inside the home folder with HOME="."
    # so the path stays short wherever the repository lives.
    os.chdir(home)
    os.environ["HOME"] = "."
    os.environ["USER"] = "maosref"
    os.environ["OMP_NUM_THREADS"] = str(nthread)
    w = _Worker(nthread)
    while True:
        msg = conn.recv()
        if msg is None:
            break
        name, args, kw = msg
        try:
            conn.send(("ok", getattr(w, name)(*args, **kw)))
        except Exception as e:  # pragma: no cover - surfaced to the caller
            conn.send(("err", repr(e)))


class RefProcess:
    """Handle on a worker process holding the reference library."""

    def __init__(self, nthread: int = 1):
        if not available():
            raise FileNotFoundError(f"{LIB} not built (make -C oracle/ref)")
        ctx = mp.get_context("spawn")
        self.conn, child = ctx.Pipe()
        home = os.path.join(HERE, "_ref", "home")
        os.makedirs(os.path.join(home, ".aos", "cache"), exist_ok=True)
        self.proc = ctx.Process(target=_serve, args=(child, nthread, home), daemon=True)
        self.proc.start()

    def call(self, name: str, *args, **kw) -> Any:
        self.conn.send((name, args, kw))
        st, val = self.conn.recv()
        if st != "ok":
            raise RuntimeError(f"reference call {name} failed: {val}")
        return val

    def close(self):
        try:
            self.conn.send(None)
        except Exception:
            pass
        self.proc.join(timeout=10)
        if self.proc.is_alive():
            self.proc.kill()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def fit_desc(fs) -> dict:
    """Flatten a FitSystem for ``ref_fit_setup``."""
    W0 = fs.W0.tocsc()
    W0.sort_indices()
    return {"nfit": len(fs.thetax), "thetax": fs.thetax, "thetay": fs.thetay, "wt": fs.wt,
            "hs": np.where(np.isfinite(fs.hs), fs.hs, np.inf), "nf": fs.floc.n,
            "w0_p": W0.indptr, "w0_i": W0.indices, "w0_x": W0.data, "w1": fs.W1,
            "ndm": len(fs.dms), "dmht": [d.ht for d in fs.dms], "dmdx": [d.amap.dx for d in fs.dms],
            "nact": [len(d.act) for d in fs.dms],
            "alocx": np.concatenate([d.locx for d in fs.dms]),
            "alocy": np.concatenate([d.locy for d in fs.dms]),
            "nnw": fs.NW.shape[1], "nw": np.asfortranarray(fs.NW).ravel(order="F")}


def fit_assembled_desc(sf, cfg) -> dict:
    """Flatten a maos_b200.fit_assemble.SparseFit's inputs for ``ref_fit_assemble``."""
    W0 = sf.W0.tocsc()
    W0.sort_indices()
    return {"nfit": len(sf.thetax), "thetax": sf.thetax, "thetay": sf.thetay, "wt": sf.wt, "hs": sf.hs,
            "nf": sf.floc.nloc, "flocx": sf.floc.locx, "flocy": sf.floc.locy, "fdx": sf.floc.dx,
            "w0_p": W0.indptr, "w0_i": W0.indices, "w0_x": W0.data, "w1": sf.W1,
            "ndm": len(sf.alocs), "dmht": [a.ht for a in sf.alocs], "dmdx": [a.dx for a in sf.alocs],
            "nact": [a.nloc for a in sf.alocs], "alocx": np.concatenate([a.locx for a in sf.alocs]),
            "alocy": np.concatenate([a.locy for a in sf.alocs]),
            "actslave": int(sf.actslave is not None), "actinterp": 1, "actthres": 0.1, "tikcr": sf.tikcr,
            "lrt_piston": int(cfg.fit_lrt_piston), "lrt_tt": int(cfg.fit_lrt_tt)}


def system_desc(sysm, split: int = 1) -> dict:
    """Flatten a TomoSystem into the driver's setup arguments."""
    cfg = sysm.cfg
    d = {"nwfs": len(sysm.wfs), "nps": len(sysm.xmaps), "r0": cfg.r0,
         "cxxscale": cfg.tomo_cxxscale, "dt": cfg.sim_dt, "pos": cfg.tomo_pos, "split": split,
         "precond": cfg.tomo_precond, "maxit": cfg.tomo_maxit, "nxtot": sysm.nx_total,
         "ngrad": sysm.ngrad}
    p = sysm.pmap
    d["pmap"] = (p.nx, p.ny, p.dx, p.ox, p.oy)
    d["layers"] = [(g.nx, g.ny, g.dx, g.ox, g.oy, float(sysm.ht[l]), float(sysm.wt[l]),
                    int(sysm.os[l])) for l, g in enumerate(sysm.xmaps)]
    ws = []
    for w in sysm.wfs:
        G = w.GP.tocsc()
        G.sort_indices()
        ws.append({"thetax": w.thetax, "thetay": w.thetay, "hs": w.hs, "nsa": w.nsa, "dsa": w.dsa,
                   "salocx": w.salocx, "salocy": w.salocy, "saa": w.saa, "gp_p": G.indptr,
                   "gp_i": G.indices, "gp_x": G.data, "saneai": w.saneai, "sanea": w.sanea,
                   "trs": w.trs, "neam": w.neam})
    d["wfs"] = ws
    return d
