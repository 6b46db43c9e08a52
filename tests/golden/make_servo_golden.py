"""Golden vectors for the device servo: the reference's own servo_new /
servo_filter (lib/servo.c, compiled in oracle/_ref) on seeded errors.

    python tests/golden/make_servo_golden.py   -> tests/golden/servo_cases.npz
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle import refbridge  # noqa: E402

# name: (n, ap, al, dt, ep as a column-major ep_nx x ep_ny array)
CASES = {
    "typeI": (12, None, 0, 1 / 800, np.array([[0.5]])),
    "typeI_delay2_ap": (12, np.array([0.95, 0.05]), 2, 1 / 800, np.array([[0.4]])),
    "typeI_per_mode": (6, None, 1, 1 / 800, np.array([[0.1, 0.2, 0.3, 0.4, 0.5, 0.6]])),
    "pid": (12, np.array([1.0, 0.0, 0.0]), 1, 1 / 800, np.array([[0.5], [0.2]])),
    "typeII": (12, None, 0, 1 / 800, np.array([[0.3], [3.0], [0.01]])),
    "typeII_per_mode_delay": (4, None, 2, 1 / 800, np.array([[0.3, 0.2, 0.1, 0.25], [3.0, 2.5, 2.0, 4.0],
                                                              [0.01, 0.02, 0.015, 0.005]])),
}
NSTEP = 40


def main():
    out = {}
    rng = np.random.default_rng(11)
    with refbridge.RefProcess(nthread=1) as R:
        for name, (n, ap, al, dt, ep) in CASES.items():
            merrs = rng.standard_normal((NSTEP, n))
            cmds = R.call("servo_run", merrs, ap, al, dt, ep)
            out[name + "/merr"] = merrs
            out[name + "/cmd"] = cmds
    np.savez_compressed(os.path.join(HERE, "servo_cases.npz"), **out)


if __name__ == "__main__":
    main()
