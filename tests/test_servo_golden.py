"""The committed servo golden vectors are what the reference's servo_filter
(lib/servo.c, compiled in oracle/_ref) returns: regenerate and compare."""
import os
import sys

import numpy as np
import pytest

from oracle import refbridge

pytestmark = pytest.mark.skipif(not refbridge.available(), reason="reference library not built")

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "golden"))
from make_servo_golden import CASES  # noqa: E402


def test_golden_servo_vectors_are_the_reference():
    gold = np.load(os.path.join(HERE, "golden", "servo_cases.npz"))
    with refbridge.RefProcess(nthread=1) as R:
        for name, (n, ap, al, dt, ep) in CASES.items():
            cmds = R.call("servo_run", gold[name + "/merr"], ap, al, dt, ep)
            assert np.array_equal(cmds, gold[name + "/cmd"]), name
