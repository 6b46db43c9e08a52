"""Device servo filter against the reference's own servo_filter
(lib/servo.c): golden commands from tests/golden/make_servo_golden.py.
The device follows the reference's FP64 operation order (products and sums
rounded separately), so the commands agree to the last bits."""
import os
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
from make_servo_golden import CASES  # noqa: E402

GOLD = np.load(os.path.join(HERE, "golden", "servo_cases.npz"))


@pytest.mark.parametrize("name", sorted(CASES))
def test_servo_matches_reference(name):
    import torch
    from maos_b200.servo import Servo
    n, ap, al, dt, ep = CASES[name]
    merr, want = GOLD[name + "/merr"], GOLD[name + "/cmd"]
    s = Servo(n, ep=ep, ap=ap, al=al, dt=dt)
    try:
        for rep in range(2):  # the second pass after a reset must repeat the first
            for k in range(merr.shape[0]):
                got = s.filter(torch.tensor(merr[k], device="cuda")).cpu().numpy()
                scale = max(np.abs(want[k]).max(), 1e-300)
                assert np.abs(got - want[k]).max() <= 1e-14 * scale, (name, rep, k)
            s.reset()
    finally:
        s.close()


def test_servo_batched_instances_are_independent():
    """Type I with per-mode gains on 3 stacked instances equals 3 runs of one."""
    import torch
    from maos_b200.servo import Servo
    n, ap, al, dt, ep = CASES["typeI_per_mode"]
    rng = np.random.default_rng(5)
    merr = rng.standard_normal((20, 3 * n))
    big = Servo(3 * n, ep=ep, ap=ap, al=al, dt=dt)
    one = [Servo(n, ep=ep, ap=ap, al=al, dt=dt) for _ in range(3)]
    try:
        for k in range(20):
            g = big.filter(torch.tensor(merr[k], device="cuda")).cpu().numpy()
            for b in range(3):
                o = one[b].filter(torch.tensor(merr[k, b * n:(b + 1) * n], device="cuda")).cpu().numpy()
                assert np.array_equal(g[b * n:(b + 1) * n], o)
    finally:
        big.close()
        for s in one:
            s.close()
