"""Golden vectors for the geometric WFS tables and ray tracing: the
reference's own ptsnew/pts2loc/locannular/mkg (GS0 and the amplitude of a
small partially illuminated pupil) and prop_grid (with and without
wrap-around), compiled in oracle/_ref.

    python tests/golden/make_wfs_golden.py   -> tests/golden/wfs_cases.npz
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
from oracle import refbridge  # noqa: E402

# a 6 x 6 subaperture pupil of 0.5 m subapertures, D = 2.9 m with a 0.6 m
# central obscuration (partial subapertures on both edges), 8 points across
D, DIN, DSA, NXSA = 2.9, 0.6, 0.5, 8


def subapertures():
    c = (np.arange(6) - 3.0) * DSA
    X, Y = np.meshgrid(c, c)
    return X.ravel().copy(), Y.ravel().copy()


def main():
    sx, sy = subapertures()
    rng = np.random.default_rng(21)
    screen = rng.standard_normal((23, 31))
    px = rng.uniform(-5.0, 5.0, 600)
    py = rng.uniform(-4.0, 4.0, 600)
    grid = (31, 23, 0.25, -3.6, -2.7)
    with refbridge.RefProcess(nthread=1) as R:
        lx, ly, amp, p, i, x, nr, nc = R.call("wfs_gs0", sx, sy, DSA, NXSA, D, DIN)
        props = [R.call("prop_grid", grid, screen, px, py, 0.8, 0.4, -0.9, 0.9, wrap) for wrap in (1, 0)]
    np.savez_compressed(os.path.join(HERE, "wfs_cases.npz"), salocx=sx, salocy=sy, locx=lx, locy=ly, amp=amp,
                        gs0_p=p, gs0_i=i, gs0_x=x, gs0_shape=np.array([nr, nc]), screen=screen, px=px, py=py,
                        grid=np.array(grid), prop_wrap=props[0], prop_nowrap=props[1],
                        params=np.array([D, DIN, DSA, NXSA]))


if __name__ == "__main__":
    main()
