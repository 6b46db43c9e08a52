"""GPU parity of the tomography path against the FP64 oracle.

The oracle (oracle/recon_oracle.py) is pinned to the reference's compiled CPU
code by test_oracle_pin.py.  Tolerances (relative L2, FP32 on the GPU):
  single operator applications: 5e-5
  full CG / FDPCG solve (30 iterations): 2e-3 on the layer OPD
"""
import numpy as np
import pytest

from oracle.recon_oracle import TomoOracle, tomo_solve

pytestmark = pytest.mark.gpu

OP_TOL = 5e-5
SOLVE_TOL = 2e-3


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(b))


def fdpcg_variant(name):
    """The 8 m LTAO system with the FDPCG preconditioner: its subaperture
    selection keeps four frequencies (the general fdpcg_saselect case)."""
    from maos_b200 import config, geometry
    cfg = config.PRESETS[name]()
    cfg.tomo_precond = 1
    return geometry.build_tomo(cfg)


@pytest.fixture(scope="module", params=["ltao_8m", "mcao_30m", "ltao_8m_fdpcg"])
def setup(request):
    from conftest import get_system
    from maos_b200.recon import Reconstructor
    name = request.param
    s = fdpcg_variant(name[:-6]) if name.endswith("_fdpcg") else get_system(name)
    R = Reconstructor(s, nbatch=2)
    yield s, R, TomoOracle(s)
    R.close()


def test_hx(setup):
    s, R, o = setup
    x = np.random.default_rng(1).standard_normal((2, s.nx_total)) * 1e-7
    got = R.apply_hx(x)
    for b in range(2):
        want = o.hx(x[b])
        for w in range(len(s.wfs)):
            assert rel(got[b, w], want[w]) < OP_TOL


def test_tomo_R(setup):
    s, R, o = setup
    g = np.random.default_rng(2).standard_normal((2, s.ngrad)) * 1e-6
    got = R.apply_R(g)
    for b in range(2):
        assert rel(got[b], o.tomo_R(g[b])) < OP_TOL


def test_tomo_L(setup):
    s, R, o = setup
    x = np.random.default_rng(3).standard_normal((2, s.nx_total)) * 1e-7
    got = R.apply_L(x)
    for b in range(2):
        assert rel(got[b], o.tomo_L(x[b])) < OP_TOL


def test_fdpcg(setup):
    s, R, o = setup
    if s.fdpcg is None:
        pytest.skip("plain CG configuration")
    x = np.random.default_rng(4).standard_normal((2, s.nx_total))
    got = R.apply_fdpcg(x)
    for b in range(2):
        assert rel(got[b], o.fdpcg_precond(x[b])) < OP_TOL


def test_solve_cold_then_warm(setup):
    s, R, o = setup
    rng = np.random.default_rng(5)
    g1 = rng.standard_normal((2, s.ngrad)) * 1e-6
    g2 = g1 + rng.standard_normal((2, s.ngrad)) * 1e-7
    R.reset()
    x1, r1 = R.tomo(g1)
    x2, r2 = R.tomo(g2)  # warm-started from x1
    for b in range(2):
        w1, res1 = tomo_solve(o, g1[b])
        w2, res2 = tomo_solve(o, g2[b], x0=w1)
        assert rel(x1[b], w1) < SOLVE_TOL
        assert rel(x2[b], w2) < SOLVE_TOL
        assert abs(r1[b] - res1) < 0.05 * res1 + 1e-6
        assert abs(r2[b] - res2) < 0.05 * res2 + 1e-6


def test_update_cn2_reaches_the_captured_step(setup):
    """gpu_update_recon_cn2 (cuda/gpu.h:50): new layer weights change the
    regularisation in both the operator and the captured graph step."""
    import dataclasses
    from maos_b200.config import TOMOSCALE
    from maos_b200.geometry import laplacian_coef
    s, R, o = setup
    # new Cn2 profile: the layer weights reversed; l2c as the setup derives it
    wt = np.asarray(s.wt, dtype=np.float64)[::-1].copy()
    l2c = np.array([(laplacian_coef(s.cfg.r0, w, g.dx) * 0.25) ** 2 * s.cfg.tomo_cxxscale * TOMOSCALE
                    for w, g in zip(wt, s.xmaps)])
    assert not np.allclose(l2c, s.l2c)
    s2 = dataclasses.replace(s, wt=wt, l2c=l2c)
    o2 = TomoOracle(s2)
    rng = np.random.default_rng(8)
    x = rng.standard_normal((2, s.nx_total)) * 1e-7
    g = rng.standard_normal((2, s.ngrad)) * 1e-6
    try:
        R.update_cn2(l2c, s.fdpcg)  # the preconditioner tables are re-sent with it (kept here)
        got = R.apply_L(x)
        R.reset()
        xs, _ = R.tomo(g)
        for b in range(2):
            assert rel(got[b], o2.tomo_L(x[b])) < OP_TOL
            want, _ = tomo_solve(o2, g[b])
            assert rel(xs[b], want) < SOLVE_TOL
    finally:
        R.update_cn2(np.asarray(s.l2c, dtype=np.float64), s.fdpcg)
        R.reset()


def test_update_cn2_rebuilds_fdpcg_on_device(setup):
    """mb_update_recon_cn2 without new tables: the FDPCG blocks for the new
    layer weights are rebuilt on the GPU from the data term kept at setup;
    they must act like the host fdpcg_prepare of the new weights, and a
    rebuild at the original weights must give back the original operator."""
    import dataclasses
    from maos_b200 import fdpcg_setup
    from maos_b200.config import TOMOSCALE
    from maos_b200.geometry import laplacian_coef
    s, R, o = setup
    if s.fdpcg is None:
        pytest.skip("plain CG configuration")
    wt = np.asarray(s.wt, dtype=np.float64)[::-1].copy()
    l2c = np.array([(laplacian_coef(s.cfg.r0, w, g.dx) * 0.25) ** 2 * s.cfg.tomo_cxxscale * TOMOSCALE
                    for w, g in zip(wt, s.xmaps)])
    s2 = dataclasses.replace(s, wt=wt, l2c=l2c)
    s2 = dataclasses.replace(s2, fdpcg=fdpcg_setup.fdpcg_prepare(s2))  # host tables of the new weights
    o2 = TomoOracle(s2)
    rng = np.random.default_rng(10)
    x = rng.standard_normal((2, s.nx_total))
    g = rng.standard_normal((2, s.ngrad)) * 1e-6
    try:
        R.update_cn2(l2c)  # no tables: rebuilt on the device
        z = R.apply_fdpcg(x)
        R.reset()
        xs, _ = R.tomo(g)
        for b in range(2):
            assert rel(z[b], o2.fdpcg_precond(x[b])) < OP_TOL
            want, _ = tomo_solve(o2, g[b])
            assert rel(xs[b], want) < SOLVE_TOL
    finally:
        R.update_cn2(np.asarray(s.l2c, dtype=np.float64))  # device rebuild at the setup weights
        R.reset()
    z0 = R.apply_fdpcg(x)
    for b in range(2):
        assert rel(z0[b], o.fdpcg_precond(x[b])) < OP_TOL


def test_batch_instances_are_independent(setup):
    s, R, o = setup
    from maos_b200.recon import Reconstructor
    R1 = Reconstructor(s, nbatch=1)
    g = np.random.default_rng(6).standard_normal((2, s.ngrad)) * 1e-6
    R.reset()
    xb, _ = R.tomo(g)
    x1, _ = R1.tomo(g[1:2])
    R1.close()
    assert rel(xb[1], x1[0]) < 1e-6


@pytest.mark.parametrize("name", ["ltao_8m", "mcao_30m"])
def test_integrated_tip_tilt_split0(name):
    """recon.split=0: the LHS carries the tip/tilt projection too."""
    from conftest import get_system
    from maos_b200.recon import Reconstructor
    s = get_system(name)
    o = TomoOracle(s, split=0)
    R = Reconstructor(s, nbatch=2, split=0)
    try:
        rng = np.random.default_rng(8)
        x = rng.standard_normal((2, s.nx_total)) * 1e-7
        got = R.apply_L(x)
        for b in range(2):
            assert rel(got[b], o.tomo_L(x[b])) < OP_TOL
        g = rng.standard_normal((2, s.ngrad)) * 1e-6
        xs, _ = R.tomo(g)
        for b in range(2):
            w, _ = tomo_solve(o, g[b])
            assert rel(xs[b], w) < SOLVE_TOL
    finally:
        R.close()


def test_autotune_keeps_results():
    """The autotuner changes blockings and launch shapes only: the pupil-row
    blocking changes no bit; the y-half CTA size changes the order of the
    FP64 p.Ap partial sums and the preconditioner's form changes FP32
    rounding, so the solution agrees to FP32 rounding."""
    from conftest import get_system
    from maos_b200.recon import Reconstructor
    s = get_system("mcao_30m")
    g = np.random.default_rng(9).standard_normal((4, s.ngrad)) * 1e-6
    R = Reconstructor(s, nbatch=4)
    try:
        x0, _ = R.tomo(g)
        rows, ms = R.autotune(reps=3)
        nyp = s.pmap.nx
        splits = {-(-nyp // k) for k in range(1, nyp + 1)}
        assert rows in ms or (1 <= rows <= 32 and rows in splits)  # 4/8/16 or an even split
        if rows in ms:
            assert ms[rows] == min(ms.values())
        if s.fdpcg is not None:
            R.fdpcg_mode(1)
        R.reset()
        x1, _ = R.tomo(g)
        assert rel(x1, x0) < SOLVE_TOL
    finally:
        R.close()


def test_fdpcg_batch_shape_keeps_results():
    """The three-kernel FDPCG form's batch shape (instances per block-solve
    CTA, mb_fdpcg_shape, chosen by the autotuner) changes no bit of the
    solution, at an instance count that leaves partial CTAs for most shapes."""
    from conftest import get_system
    from maos_b200.recon import Reconstructor
    s = get_system("mcao_30m")
    g = np.random.default_rng(19).standard_normal((5, s.ngrad)) * 1e-6
    R = Reconstructor(s, nbatch=5)
    try:
        R.fdpcg_mode(1)
        assert R.fdpcg_shape() == 8
        x0, _ = R.tomo(g)
        for ni in (2, 4, 16):
            assert R.fdpcg_shape(ni) == ni
            R.reset()
            x1, _ = R.tomo(g)
            assert np.array_equal(x0, x1), ni
    finally:
        R.close()


def test_fused_preconditioner_matches_the_oracle(setup):
    """The fused FDPCG step (mb_fdpcg_mode 2: one cluster kernel per CG step,
    the layers split over its CTAs) solves to the oracle's tolerance, agrees
    with the three-kernel form to FP32 rounding, and gives an instance the
    same result (bit for bit) alone and beside another."""
    s, R, o = setup
    if s.fdpcg is None:
        pytest.skip("plain CG configuration")
    from maos_b200.recon import Reconstructor
    rng = np.random.default_rng(15)
    g1 = rng.standard_normal((2, s.ngrad)) * 1e-6
    g2 = g1 + rng.standard_normal((2, s.ngrad)) * 1e-7
    xs = {}
    try:
        for mode in (1, 2):
            if R.fdpcg_mode(mode) != mode:
                pytest.skip("the fused cluster does not fit on this device")
            R.reset()
            x1, _ = R.tomo(g1)
            x2, r2 = R.tomo(g2)
            xs[mode] = (x1, x2)
        for b in range(2):
            w1, _ = tomo_solve(o, g1[b])
            w2, res2 = tomo_solve(o, g2[b], x0=w1)
            assert rel(xs[2][0][b], w1) < SOLVE_TOL
            assert rel(xs[2][1][b], w2) < SOLVE_TOL
            assert rel(xs[2][1][b], xs[1][1][b]) < SOLVE_TOL
        # alone and in a batch of two: identical bits
        R1 = Reconstructor(s, nbatch=1)
        try:
            assert R1.fdpcg_mode(2) == 2
            R1.reset()
            a1, _ = R1.tomo(g1[1:2])
            a2, _ = R1.tomo(g2[1:2])
        finally:
            R1.close()
        assert np.array_equal(a2[0], xs[2][1][1])
    finally:
        R.fdpcg_mode(1)


def test_fdpcg_data_term_formed_and_rebuilt_on_device(setup):
    """f2, the FDPCG part of gpu_update_recon on the device: the block
    matrices' data term (maos/fdpcg.c:427-480) is formed on the GPU from its
    geometry and equals the host setup's at FP64 round-off; after the noise of
    one WFS changes, mb_update_recon_nea + mb_update_recon_neam rebuild the
    data term and the blocks on the device, again equal to the host setup's
    at the new noise, and the preconditioner and the solve follow the oracle
    built at the new noise."""
    import dataclasses
    import time
    from maos_b200 import fdpcg_setup
    s, R, o = setup
    if s.fdpcg is None:
        pytest.skip("plain CG configuration")
    want = s.fdpcg.mhat_data
    got = R.fdpcg_data()
    assert np.abs(got - want).max() <= 1e-12 * np.abs(want).max()
    # the noise of WFS 1 rises by 1.5 (its PTT is unchanged by a uniform scale)
    sc = 1.5
    wfs = list(s.wfs)
    w = wfs[1]
    wfs[1] = dataclasses.replace(w, saneai=w.saneai / sc ** 2, sanea=w.sanea * sc ** 2, neam=w.neam * sc)
    s2 = dataclasses.replace(s, wfs=wfs, fdpcg=None)
    s2 = dataclasses.replace(s2, fdpcg=fdpcg_setup.fdpcg_prepare(s2))
    nsa = w.nsa

    def neai_of(wt):
        return np.stack([wt.saneai[:nsa], wt.saneai[nsa:], np.zeros(nsa)], axis=1).ravel()

    try:
        R.update_nea(1, neai_of(wfs[1]), w.PTT)
        R.lib.mb_kernel_launches(1)
        t0 = time.perf_counter()
        R.update_neam(s2.fdpcg.geom["neam"])
        dt = time.perf_counter() - t0
        got2 = R.fdpcg_data()
        want2 = s2.fdpcg.mhat_data
        assert np.abs(got2 - want2).max() <= 1e-12 * np.abs(want2).max()
        assert np.abs(want2 - want).max() > 1e-3 * np.abs(want).max()  # the change is real
        o2 = TomoOracle(s2)
        x = np.random.default_rng(8).standard_normal((2, s.nx_total))
        z = R.apply_fdpcg(x)
        for b in range(2):
            assert rel(z[b], o2.fdpcg_precond(x[b])) < OP_TOL
        g = np.random.default_rng(9).standard_normal((2, s.ngrad)) * 1e-6
        R.reset()
        xs, _ = R.tomo(g)
        for b in range(2):
            w2, _ = tomo_solve(o2, g[b])
            assert rel(xs[b], w2) < SOLVE_TOL
        print(f"device rebuild of the FDPCG data term and blocks: {dt * 1e3:.3f} ms")
    finally:
        R.update_nea(1, neai_of(w), w.PTT)
        R.update_neam(s.fdpcg.geom["neam"])
