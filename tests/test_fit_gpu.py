"""GPU parity of the DM fit (grid form) against the FP64 oracle.

The fit oracle is pinned to the reference's FitR/FitL/pcg by
test_oracle_pin.py.  Tolerances (relative L2, FP32 on the GPU):
  FitR / FitL applications: 5e-5
  DM command vector after tomography + fit CG (same iteration counts as the
  oracle, warm start chained over two steps): 1e-4
"""
import numpy as np
import pytest

from oracle.recon_oracle import FitOracle, TomoOracle, fit_solve, tomo_solve

pytestmark = pytest.mark.gpu

OP_TOL = 5e-5
SOLVE_TOL = 1e-4


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / np.linalg.norm(b))


@pytest.fixture(scope="module", params=["ltao_8m", "mcao_30m"])
def setup(request):
    from conftest import get_fit, get_system
    from maos_b200.recon import Reconstructor
    s = get_system(request.param)
    fs = get_fit(request.param)
    R = Reconstructor(s, nbatch=2, fit=fs)
    yield s, fs, R
    R.close()


def test_fit_R(setup):
    s, fs, R = setup
    fo = FitOracle(s, fs)
    x = np.random.default_rng(1).standard_normal((2, s.nx_total)) * 1e-7
    got = R.apply_fit_R(x)
    for b in range(2):
        assert rel(got[b], fo.fit_R(x[b])) < OP_TOL


def test_fit_L(setup):
    s, fs, R = setup
    fo = FitOracle(s, fs)
    a = np.random.default_rng(2).standard_normal((2, fs.nact)) * 1e-7
    got = R.apply_fit_L(a)
    for b in range(2):
        assert rel(got[b], fo.fit_L(a[b])) < OP_TOL


def test_tomo_then_fit_two_steps(setup):
    s, fs, R = setup
    to = TomoOracle(s)
    fo = FitOracle(s, fs)
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
