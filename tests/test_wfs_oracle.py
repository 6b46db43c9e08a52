"""Geometric-WFS oracle and tables on the CPU: the noise generator against the
published Philox4x32-10 known answers, the stencils' structure, and the
oracle's gradients of known wavefronts."""

import numpy as np
import pytest

from oracle import wfs_oracle


def test_philox_known_answers():
    # Salmon et al., "Parallel random numbers: as easy as 1, 2, 3" (SC 2011): Random123 test vectors
    cases = [([0, 0, 0, 0], [0, 0], [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]),
             ([0xffffffff] * 4, [0xffffffff] * 2, [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]),
             ([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344], [0xa4093822, 0x299f31d0],
              [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1])]
    for c, k, want in cases:
        out = wfs_oracle.philox4x32_10(np.array([c], dtype=np.uint32), np.array([k], dtype=np.uint32))[0]
        assert [int(v) for v in out] == want


def test_normals_are_standard():
    n1, n2 = wfs_oracle.geom_normals(1234, 7, 2, 0, 200000)
    for n in (n1, n2):
        assert abs(n.mean()) < 0.01 and abs(n.std() - 1.0) < 0.01
    assert abs(np.corrcoef(n1, n2)[0, 1]) < 0.01
    a, _ = wfs_oracle.geom_normals(1234, 8, 2, 0, 1000)
    assert not np.allclose(a, n1[:1000])


@pytest.fixture(scope="module")
def ltao_geom():
    from conftest import get_system
    from maos_b200 import wfs_setup
    s = get_system("ltao_8m")
    return s, wfs_setup.build_geom_wfs(s)


def test_stencils_shared_and_area_normalised(ltao_geom):
    s, geom = ltao_geom
    P = geom.powfs[0]
    assert P.nxsa == 26 and len(P.ix0) == s.wfs[0].nsa
    assert len(P.stencils) < len(P.ix0) // 2
    # x stencil of a full subaperture: a tilt of 1 rad in x gives gradient 1
    G = P.gs0()
    X, Y = np.meshgrid(P.grid.ox + np.arange(P.grid.nx) * P.grid.dx, P.grid.oy + np.arange(P.grid.ny) * P.grid.dy)
    gx = G @ X.ravel()
    gy = G @ Y.ravel()
    nsa = len(P.ix0)
    full = s.wfs[0].saa > 0.999
    assert np.allclose(gx[:nsa][full], 1.0, atol=1e-12) and np.allclose(gy[nsa:][full], 1.0, atol=1e-12)
    assert np.allclose(gx[nsa:][full], 0.0, atol=1e-12) and np.allclose(gy[:nsa][full], 0.0, atol=1e-12)


def test_oracle_gradients_of_a_tilted_layer(ltao_geom):
    s, geom = ltao_geom
    # a pure x tilt on a ground layer, periodic over the screen: gradient = tilt
    n, dx = 256, 0.125
    ox = -n * dx / 2
    xs = ox + np.arange(n) * dx
    scr = np.tile(1e-6 * xs, (n, 1))
    atm = [wfs_oracle.Screen(scr, ox, ox, dx, 0.0)]
    g = wfs_oracle.geom_grads(geom, atm, [], 0, 1 / 800.0)
    P = geom.powfs[0]
    nsa = len(P.ix0)
    full = s.wfs[0].saa > 0.999
    for iw in range(geom.nwfs):
        gw = g[2 * nsa * iw: 2 * nsa * (iw + 1)]
        scale = 1.0
        assert np.allclose(gw[:nsa][full], 1e-6 * scale, rtol=1e-9)
        assert np.allclose(gw[nsa:][full], 0.0, atol=1e-15)


def test_tables_and_ray_tracing_match_golden_vectors():
    """Against the reference's own GS0, amplitude and prop_grid of a small
    partially illuminated pupil (tests/golden/make_wfs_golden.py)."""
    import os
    import scipy.sparse as sps
    from maos_b200 import wfs_setup
    z = np.load(os.path.join(os.path.dirname(__file__), "golden", "wfs_cases.npz"))
    D, DIN, DSA, NXSA = z["params"]
    P = wfs_setup.build_geom_powfs(z["salocx"], z["salocy"], float(DSA), float(DSA) / int(NXSA), float(D), float(DIN))
    assert P.nxsa == int(NXSA)
    gx = np.rint((z["locx"] - P.grid.ox) / P.grid.dx).astype(np.int64)
    gy = np.rint((z["locy"] - P.grid.oy) / P.grid.dy).astype(np.int64)
    col = gy * P.grid.nx + gx
    assert np.array_equal(P.amp.ravel()[col], z["amp"])
    nr, nc = z["gs0_shape"]
    Gref = sps.csc_matrix((z["gs0_x"], z["gs0_i"], z["gs0_p"]), shape=(int(nr), int(nc)))
    G = P.gs0()
    assert G.nnz == Gref.nnz
    d = (G[:, col] - Gref).tocoo()
    assert (np.abs(d.data).max() if d.nnz else 0.0) <= 1e-14 * np.abs(Gref.data).max()
    nx, ny, dx, ox, oy = z["grid"]
    for wrap, key in ((True, "prop_wrap"), (False, "prop_nowrap")):
        ours = wfs_oracle.prop_grid(z["screen"], ox, oy, dx, z["px"], z["py"], 0.8, 0.4, -0.9, 0.9, wrap)
        assert np.abs(ours - z[key]).max() <= 1e-13 * np.abs(z[key]).max()
