"""GPU parity of the DM fit against the FP64 oracle, in both forms:

* grid form (cufit_grid, gpu.fit=2) with the slaving term, oracle FitOracle
  pinned to the reference's FitR/FitL/slaving/pcg by test_oracle_pin.py;
* assembled form (cusolve_sparse, gpu.fit=1, the reference default: in-pupil
  actuators, slaving, extrapolation, tikcr), oracle SparseFitOracle pinned to
  the reference's setup_fit/muv/pcg by test_fit_assemble_pin.py.

Tolerances (relative L2, FP32 on the GPU):
  FitR / FitL applications: 5e-5
  DM command vector after tomography + fit CG (same iteration counts as the
  oracle, warm start chained over two steps): 1e-4
"""
import numpy as np
import pytest

from oracle.recon_oracle import FitOracle, SparseFitOracle, TomoOracle, fit_solve, tomo_solve

pytestmark = pytest.mark.gpu

OP_TOL = 5e-5
SOLVE_TOL = 1e-4


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(b))


@pytest.fixture(scope="module", params=[("ltao_8m", "grid"), ("mcao_30m", "grid"), ("ltao_8m", "assembled"),
                                        ("mcao_30m", "assembled")], ids=lambda p: "-".join(p))
def setup(request):
    from conftest import get_fit, get_fit_assembled, get_system
    from maos_b200.recon import Reconstructor
    name, kind = request.param
    s = get_system(name)
    fs = get_fit(name) if kind == "grid" else get_fit_assembled(name)
    R = Reconstructor(s, nbatch=2, fit=fs)
    yield s, fs, R
    R.close()


def oracle_for(s, fs):
    return SparseFitOracle(s, fs) if hasattr(fs, "FLM") else FitOracle(s, fs)


def test_fit_R(setup):
    s, fs, R = setup
    fo = oracle_for(s, fs)
    x = np.random.default_rng(1).standard_normal((2, s.nx_total)) * 1e-7
    got = R.apply_fit_R(x)
    for b in range(2):
        assert rel(got[b], fo.fit_R(x[b])) < OP_TOL


def test_fit_L(setup):
    s, fs, R = setup
    fo = oracle_for(s, fs)
    a = np.random.default_rng(2).standard_normal((2, fs.nact)) * 1e-7
    got = R.apply_fit_L(a)
    for b in range(2):
        assert rel(got[b], fo.fit_L(a[b])) < OP_TOL


def test_tomo_then_fit_two_steps(setup):
    s, fs, R = setup
    to = TomoOracle(s)
    fo = oracle_for(s, fs)
    rng = np.random.default_rng(3)
    g1 = rng.standard_normal((2, s.ngrad)) * 1e-6
    g2 = g1 + rng.standard_normal((2, s.ngrad)) * 1e-7
    R.reset()
    R.tomo(g1)
    a1, r1 = R.fit()
    R.tomo(g2)
    a2, r2 = R.fit()
    for b in range(2):
        x1, _ = tomo_solve(to, g1[b])
        w1, _ = fit_solve(fo, x1)
        x2, _ = tomo_solve(to, g2[b], x0=x1)
        w2, res2 = fit_solve(fo, x2, a0=w1)
        assert rel(a1[b], w1) < SOLVE_TOL
        assert rel(a2[b], w2) < SOLVE_TOL
        assert abs(r2[b] - res2) < 0.05 * res2 + 1e-6


def test_grid_fit_carries_the_slaving_term(setup):
    """The grid-form FitL includes actslave (cufit_grid::L, cuda/fit.cu:232):
    the device result matches the oracle with the term and differs from the
    oracle without it."""
    s, fs, R = setup
    if hasattr(fs, "FLM") or fs.actslave is None:
        pytest.skip("grid form with a slaving term only")
    import dataclasses
    a = np.random.default_rng(4).standard_normal((2, fs.nact)) * 1e-7
    got = R.apply_fit_L(a)
    with_term = FitOracle(s, fs).fit_L(a[0])
    without = FitOracle(s, dataclasses.replace(fs, actslave=None)).fit_L(a[0])
    assert rel(got[0], with_term) < OP_TOL
    assert rel(without, with_term) > 10 * OP_TOL
