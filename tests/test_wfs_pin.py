"""Pin the geometric-WFS tables and the OPD ray tracing to the reference.

``maos_b200.wfs_setup`` (fine grid, ``locannular`` amplitude, ``mkg`` GS0
stencils) is compared with the reference's own ``ptsnew``/``pts2loc``/
``locannular``/``mkg`` on the same subapertures, and the oracle's
``prop_grid`` with the reference's ``prop_grid`` (``lib/accphi.c:426``), both
run from ``oracle/_ref/libmaosref.so``.
"""
import numpy as np
import pytest
import scipy.sparse as sps

from oracle import refbridge
from oracle import wfs_oracle

pytestmark = [pytest.mark.ref,
              pytest.mark.skipif(not refbridge.available(), reason="reference library not built")]


@pytest.fixture(scope="module")
def ref_proc():
    with refbridge.RefProcess(nthread=4) as R:
        yield R


@pytest.mark.parametrize("name", ["ltao_8m", "mcao_30m"])
def test_gs0_and_amp_match_reference(name, ref_proc):
    from conftest import get_system
    from maos_b200 import wfs_setup
    s = get_system(name)
    w = s.wfs[0]
    P = wfs_setup.build_geom_powfs(w.salocx, w.salocy, w.dsa, 1.0 / 64, s.cfg.D, s.cfg.din)
    lx, ly, amp, p, i, x, nr, nc = ref_proc.call("wfs_gs0", w.salocx, w.salocy, w.dsa, P.nxsa, s.cfg.D, s.cfg.din)
    gx = np.rint((lx - P.grid.ox) / P.grid.dx).astype(np.int64)
    gy = np.rint((ly - P.grid.oy) / P.grid.dy).astype(np.int64)
    # the reference's points sit on the fine grid
    assert np.abs(P.grid.ox + gx * P.grid.dx - lx).max() < 1e-12
    assert np.abs(P.grid.oy + gy * P.grid.dy - ly).max() < 1e-12
    col = gy * P.grid.nx + gx
    # amplitude: bit-exact on the points, zero elsewhere
    assert np.array_equal(P.amp.ravel()[col], amp)
    assert P.amp.sum() == pytest.approx(amp.sum(), rel=1e-15)
    Gref = sps.csc_matrix((x, i, p), shape=(nr, nc))
    G = P.gs0()
    assert G.nnz == Gref.nnz                       # nothing off the reference's points
    d = (G[:, col] - Gref).tocoo()
    assert (np.abs(d.data).max() if d.nnz else 0.0) <= 1e-14 * np.abs(Gref.data).max()


def test_prop_grid_matches_reference(ref_proc):
    rng = np.random.default_rng(5)
    nx, ny, dx, ox, oy = 37, 29, 0.25, -4.6, -3.4
    scr = rng.standard_normal((ny, nx))
    x = rng.uniform(-7.0, 7.0, 4000)
    y = rng.uniform(-6.0, 6.0, 4000)
    x[:5] = ox + (nx - 1) * dx + np.array([0.0, 0.1, 0.2, 0.24, 0.249])   # the last column
    for wrap in (1, 0):
        for alpha, dxp, dyp, scale in ((1.0, 0.3, -1.7, 1.0), (-0.7, -2.2, 0.9, 0.85)):
            ref = ref_proc.call("prop_grid", (nx, ny, dx, ox, oy), scr, x, y, alpha, dxp, dyp, scale, wrap)
            ours = wfs_oracle.prop_grid(scr, ox, oy, dx, x, y, alpha, dxp, dyp, scale, bool(wrap))
            assert np.abs(ours - ref).max() <= 1e-13 * np.abs(ref).max()


def test_geom_gradients_match_reference(ref_proc):
    """The whole geometric WFS (atmosphere with wind and wrap-around, a DM,
    GS0) of the oracle against the reference's prop_grid + GS0 product."""
    from conftest import get_fit, get_system
    from maos_b200 import wfs_setup
    from maos_b200.turbulence import FrozenFlowAtmosphere
    s = get_system("ltao_8m")
    fit = get_fit("ltao_8m")
    geom = wfs_setup.build_geom_wfs(s)
    P = geom.powfs[0]
    w = s.wfs[0]
    ref_proc.call("wfs_gs0", w.salocx, w.salocy, w.dsa, P.nxsa, s.cfg.D, s.cfg.din)
    atm = FrozenFlowAtmosphere(s.cfg, 4)
    n, dx = atm.n, atm.dx
    o = -n / 2 * dx
    layers = [wfs_oracle.Screen(sc, o, o, dx, float(h), float(atm.vx[l]), float(atm.vy[l]))
              for l, (sc, h) in enumerate(zip(atm.screens, s.cfg.atm_ht))]
    a = np.random.default_rng(8).standard_normal(fit.nact) * 1e-7
    dms = []
    off = fit.act_offsets()
    for k, dm in enumerate(fit.dms):
        dms.append(wfs_oracle.Screen(a[off[k]:off[k + 1]].reshape(dm.amap.ny, dm.amap.nx), dm.amap.ox, dm.amap.oy,
                                     dm.amap.dx, dm.ht))
    maps = [(L.data, L.dx, L.ox, L.oy, L.ht, L.vx, L.vy, 1.0, 1) for L in layers]
    maps += [(D.data, D.dx, D.ox, D.oy, D.ht, 0.0, 0.0, -1.0, 0) for D in dms]
    isim = 17
    ref = ref_proc.call("wfs_geom_grads", geom.thetax, geom.thetay, geom.hs, maps, s.cfg.sim_dt, isim).ravel()
    ours = wfs_oracle.geom_grads(geom, layers, dms, isim, s.cfg.sim_dt)
    assert np.linalg.norm(ours - ref) <= 1e-12 * np.linalg.norm(ref)
