"""Pin the FP64 oracle against the reference's own compiled CPU path.

The reference (sys/, math/, lib/, maos/ of MAOS) is built by
``oracle/ref/Makefile`` into ``oracle/_ref/libmaosref.so``; these tests run its
``TomoR``/``TomoL``/``fdpcg_prepare``/``fdpcg_precond``/``pcg``/``mkg``/
``dcellpinv`` on the same tables as the oracle and require agreement to FP64
round-off.
"""
import numpy as np
import pytest

from oracle import refbridge
from oracle.recon_oracle import TomoOracle, pcg

pytestmark = [pytest.mark.ref,
              pytest.mark.skipif(not refbridge.available(), reason="reference library not built")]


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300))


@pytest.fixture(scope="module")
def ref_proc():
    with refbridge.RefProcess(nthread=4) as R:
        yield R


@pytest.mark.parametrize("name", ["ltao_8m", "mcao_30m"])
@pytest.mark.parametrize("split", [1, 0])
def test_tomo_operators_match_reference(name, split, ref_proc):
    from conftest import get_system
    s = get_system(name)
    R = ref_proc
    R.call("setup", refbridge.system_desc(s, split=split))
    o = TomoOracle(s, split=split)
    rng = np.random.default_rng(11)
    x = rng.standard_normal(s.nx_total)
    g = rng.standard_normal(s.ngrad)
    # pupil/layer grids are stored like the reference's loc_t (x fastest)
    px, py = R.call("loc_coords", (s.pmap.nx, s.pmap.ny, s.pmap.dx, s.pmap.ox, s.pmap.oy))
    assert np.allclose(px, np.tile(s.pmap.xs(), s.pmap.ny))
    assert np.allclose(py, np.repeat(s.pmap.ys(), s.pmap.nx))
    for iw, w in enumerate(s.wfs):
        assert rel(o.hx(x)[iw], R.call("hx", iw, x)) < 1e-12
        if w.PTT is not None:
            assert rel(w.PTT, R.call("ptt", iw)) < 1e-12
    assert rel(o.tomo_R(g), R.call("tomoR", g)) < 1e-12
    assert rel(o.tomo_L(x), R.call("tomoL", x)) < 1e-12
    assert rel(o.tomo_L(x, alpha=-0.5), R.call("tomoL", x, -0.5)) < 1e-12


def fdpcg_system(name):
    """A preset with the FDPCG preconditioner: the 30 m system as configured,
    and the 8 m systems switched to FDPCG, whose clipped subaperture-selection
    spectrum keeps four frequencies (fdpcg_saselect, maos/fdpcg.c:71)."""
    from conftest import get_system
    if name == "mcao_30m":
        return get_system(name)
    from maos_b200 import config, geometry
    cfg = config.PRESETS[name]()
    cfg.tomo_precond = 1
    return geometry.build_tomo(cfg)


@pytest.mark.parametrize("name", ["mcao_30m", "ltao_8m", "scao_8m"])
def test_fdpcg_tables_and_apply_match_reference(ref_proc, name):
    s = fdpcg_system(name)
    R = ref_proc
    R.call("setup", refbridge.system_desc(s, split=1))
    fd = R.call("fdpcg_prepare")
    assert fd["scale"] == s.fdpcg.scale
    assert np.array_equal(fd["perm"], s.fdpcg.perm)
    assert rel(s.fdpcg.Mbinv, fd["Mbinv"]) < 1e-8  # SVD pseudo-inverses, FP64
    R.call("fdpcg_set", s.fdpcg.Mbinv, s.fdpcg.perm, s.fdpcg.scale)
    o = TomoOracle(s)
    r = np.random.default_rng(5).standard_normal(s.nx_total)
    assert rel(o.fdpcg_precond(r), R.call("fdpcg_precond", r)) < 1e-12


@pytest.mark.parametrize("name,warm", [("ltao_8m", False), ("mcao_30m", False), ("mcao_30m", True)])
def test_pcg_matches_reference(name, warm, ref_proc):
    from conftest import get_system
    s = get_system(name)
    R = ref_proc
    R.call("setup", refbridge.system_desc(s, split=1))
    if s.fdpcg is not None:
        R.call("fdpcg_set", s.fdpcg.Mbinv, s.fdpcg.perm, s.fdpcg.scale)
    o = TomoOracle(s)
    rng = np.random.default_rng(7)
    b = o.tomo_R(rng.standard_normal(s.ngrad))
    x0 = rng.standard_normal(s.nx_total) * 1e-3 if warm else None
    M = o.fdpcg_precond if s.fdpcg is not None else None
    x1, r1 = pcg(x0, o.tomo_L, M, b, warm, s.cfg.tomo_maxit)
    x2, r2 = R.call("pcg", b, x0, int(warm), s.cfg.tomo_maxit, int(s.fdpcg is not None))
    assert rel(x1, x2) < 1e-10
    assert abs(r1 - r2) <= 1e-10 * abs(r2)


def test_gradient_operator_matches_reference_mkg(ref_proc, ltao):
    s = ltao
    w = s.wfs[0]
    p, i, x, nr, nc = ref_proc.call("mkg", (s.pmap.nx, s.pmap.ny, s.pmap.dx, s.pmap.ox, s.pmap.oy),
                                    s.amp, w.salocx, w.salocy, w.dsa)
    import scipy.sparse as sps
    G = sps.csc_matrix((x, i, p), shape=(nr, nc)).toarray()
    assert G.shape == w.GP.shape
    assert np.abs(G - w.GP.toarray()).max() <= 1e-12 * np.abs(G).max()


@pytest.mark.parametrize("name", ["ltao_8m", "mcao_30m"])
def test_fit_operators_match_reference(name, ref_proc):
    """FitR/FitL/CG of the oracle vs the reference's FitR/FitL/pcg, whose HA
    and HXF the driver builds with the reference's own mkh, and whose slaving
    term comes from the reference's own slaving (lib/slaving.c)."""
    from conftest import get_system, get_fit
    from oracle.recon_oracle import FitOracle
    s = get_system(name)
    fs = get_fit(name)
    R = ref_proc
    R.call("setup", refbridge.system_desc(s, split=1))
    R.call("fit_setup", refbridge.fit_desc(fs))
    # the slaving term of FitL from the reference's own genactcpl + slaving
    assert R.call("fit_setup_slave", s.cfg.fit_actthres) == (fs.actslave is not None)
    fo = FitOracle(s, fs)
    rng = np.random.default_rng(21)
    x = rng.standard_normal(s.nx_total)
    a = rng.standard_normal(fs.nact)
    assert rel(fo.fit_R(x), R.call("fitR", x)) < 1e-12
    assert rel(fo.fit_L(a), R.call("fitL", a)) < 1e-12
    b = fo.fit_R(x)
    a1, r1 = pcg(None, fo.fit_L, None, b, False, fs.maxit)
    a2, r2 = R.call("fit_pcg", b, None, 0, fs.maxit)
    assert rel(a1, a2) < 1e-10


def test_fit_weighting_matches_reference_mkw_amp(ref_proc, ltao):
    import scipy.sparse as sps
    from maos_b200.fit_setup import mkw_amp
    from maos_b200.geometry import annulus_fraction
    g = ltao.pmap
    X, Y = np.meshgrid(g.xs() - g.dx / 2, g.ys() - g.dy / 2)
    amp = annulus_fraction(X.ravel(), Y.ravel(), g.dx, 0.5, 4.0, nsub=8)
    amp /= amp.sum()
    W0, W1 = mkw_amp(g, amp)
    p, i, x, w1 = ref_proc.call("mkw_amp", (g.nx, g.ny, g.dx, g.ox, g.oy), amp)
    Wr = sps.csc_matrix((x, i, p), shape=(g.n, g.n))
    assert abs(W0 - Wr).max() <= 1e-14 * abs(Wr).max()
    assert np.abs(W1 - w1).max() <= 1e-14 * np.abs(w1).max()
