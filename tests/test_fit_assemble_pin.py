"""The assembled DM fit (the reference's default: actuators inside the
metapupil, slaving, extrapolation, Tikhonov) against the reference's own code.

maos_b200.fit_assemble restates the reference's fit setup in numpy; here every
table it builds is compared with the reference compiled from its sources
(oracle/_ref), given the same inputs:

* floc and aloc points:   create_metapupil with square=0 (math/loc.c:1471)
* loc maps with ghosts:   loc_create_map_npad (math/loc.c:208)
* W0, W1:                 mkw_circular (lib/mkw.c:363)
* FR.M/U/V, FL.M/U/V,
  actinterp, actslave,
  actcpl, NW:             setup_fit (maos/setup_recon_fit.c:303)

and the oracle's assembled fit (FR, then CG on FL) with the reference's muv
and pcg (maos/recon.c:93 muv_solve).  All to FP64 round-off.
"""
import numpy as np
import pytest
import scipy.sparse as sps

from oracle import refbridge
from oracle.recon_oracle import SparseFitOracle, pcg

pytestmark = [pytest.mark.ref,
              pytest.mark.skipif(not refbridge.available(), reason="reference library not built")]


def rel(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def sp_rel(A, ref):
    p, i, x, nr, nc = ref
    B = sps.csc_matrix((x, i, p), shape=(nr, nc))
    assert A.shape == B.shape
    return float(abs(A - B).max() / abs(B).max())


@pytest.fixture(scope="module")
def ref_proc():
    with refbridge.RefProcess(nthread=4) as R:
        yield R


@pytest.mark.parametrize("name", ["ltao_8m", "mcao_30m"])
def test_assembled_fit_matches_reference_setup(name, ref_proc):
    from conftest import get_fit_assembled, get_system
    from maos_b200.geometry import all_dirs
    s = get_system(name)
    sf = get_fit_assembled(name)
    cfg = s.cfg
    R = ref_proc
    R.call("setup", refbridge.system_desc(s, split=1))
    dirs = all_dirs(cfg)
    dxr = cfg.atmr_dx / cfg.tomo_pos
    x, y = R.call("metapupil", dirs, cfg.D, 0.0, dxr, 0.0, cfg.tomo_guard * dxr, 0)
    assert np.array_equal(x, sf.floc.locx) and np.array_equal(y, sf.floc.locy)
    for k, d in enumerate(cfg.dms):
        off = d.offset + (int(round(d.order)) % 2) * 0.5
        x, y = R.call("metapupil", dirs, cfg.D, d.ht, d.dx, off, d.dx, 0)
        a = sf.alocs[k]
        assert np.array_equal(x, a.locx) and np.array_equal(y, a.locy)
        m, ox, oy = R.call("loc_map", a.locx, a.locy, a.dx, 1)
        assert np.array_equal(m, a.map) and ox == a.mox and oy == a.moy
    p, i, w0x, w1 = R.call("mkw_circular", sf.floc.locx, sf.floc.locy, sf.floc.dx, 1, 0.0, 0.0, cfg.D / 2)
    n = sf.floc.nloc
    assert sp_rel(sf.W0, (p, i, w0x, n, n)) < 1e-13
    assert rel(sf.W1, w1) < 1e-13
    R.call("fit_assemble", refbridge.fit_assembled_desc(sf, cfg))
    for which, mine in enumerate((sf.FRM, sf.FLM, sf.actinterp, sf.actslave)):
        ref = R.call("fitas_sparse", which)
        assert (ref is None) == (mine is None), which
        if mine is not None:
            assert sp_rel(mine, ref) < 1e-12, which
    for which, mine in enumerate((sf.FRU, sf.FRV, sf.FLU, sf.FLV, np.concatenate(sf.actcpl)[:, None], sf.NW)):
        ref = R.call("fitas_dense", which)
        assert ref.shape == mine.shape, which
        assert rel(mine, ref) < 1e-12, which
    # the operators and the CG of the oracle against muv / pcg of the reference
    fo = SparseFitOracle(s, sf)
    rng = np.random.default_rng(5)
    xl = rng.standard_normal(s.nx_total)
    a0 = rng.standard_normal(sf.nact)
    assert rel(fo.fit_R(xl), R.call("fitas_rhs", xl)) < 1e-12
    assert rel(fo.fit_L(a0), R.call("fitas_L", a0)) < 1e-12
    b = fo.fit_R(xl)
    for warm in (0, 1):
        a1, r1 = pcg(a0.copy() if warm else None, fo.fit_L, None, b, bool(warm), sf.maxit)
        a2, r2 = R.call("fitas_pcg", b, a0 if warm else None, warm, sf.maxit)
        assert rel(a1, a2) < 1e-10 and abs(r1 - r2) < 1e-10 * max(r2, 1e-30)


def test_assembled_fit_has_the_default_terms():
    """The 30 m system's assembled fit: in-pupil actuators (about 7,000, as the
    NFIRAOS-like configuration quotes), a slaving term, extrapolation to
    weakly coupled actuators and the Tikhonov diagonal tikcr*4/nact."""
    from conftest import get_fit_assembled
    sf = get_fit_assembled("mcao_30m")
    assert 6500 < sf.nact < 7500
    assert sf.actslave is not None and sf.actslave.nnz > 0
    assert (sf.actinterp != sps.identity(sf.nact)).nnz > 0
    assert sf.tikcr == 1e-7
    assert sf.FLU.shape[1] == len(sf.thetax) + sf.NW.shape[1]
