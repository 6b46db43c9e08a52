"""maos .bin files: maos_b200.binio against the reference's own writer and
reader (math/cell.c writebin, read_by_id; compiled in oracle/_ref)."""
import os

import numpy as np
import pytest

from maos_b200 import binio
from oracle import refbridge

pytestmark = pytest.mark.skipif(not refbridge.available(), reason="reference library not built")


@pytest.fixture(scope="module")
def ref():
    with refbridge.RefProcess(nthread=1) as R:
        yield R


def test_read_what_the_reference_writes(ref, tmp_path):
    a = np.random.default_rng(0).standard_normal((7, 5))
    fn = str(tmp_path / "a.bin")
    ref.call("bin_write_dmat", fn, a, "r0=0.186\nL0=30")
    got, hdr = binio.read(fn, header=True)
    assert got.shape == (7, 5) and np.array_equal(got, a)
    assert "r0=0.186" in hdr and "L0=30" in hdr


def test_reference_reads_what_we_write(ref, tmp_path):
    a = np.random.default_rng(1).standard_normal((4, 9))
    fn = str(tmp_path / "b.bin")
    binio.write(fn, a, header="written by maos_b200")
    got, hdr = ref.call("bin_read_dmat", fn)
    assert np.array_equal(got, a) and hdr.startswith("written by maos_b200")
    fz = str(tmp_path / "b.bin.gz")  # gzip, as the reference's zfopen reads it
    binio.write(fz, a)
    got, _ = ref.call("bin_read_dmat", fz)
    assert np.array_equal(got, a)


def test_cells_both_ways(ref, tmp_path):
    rng = np.random.default_rng(2)
    a, b = rng.standard_normal((3, 2)), rng.standard_normal((6, 1))
    fn = str(tmp_path / "c.bin")
    ref.call("bin_write_dcell3", fn, a, b)
    c = binio.read(fn)
    assert c.shape == (3, 1) and c[1, 0] is None
    assert np.array_equal(c[0, 0], a) and np.array_equal(c[2, 0], b)
    fn2 = str(tmp_path / "d.bin")
    binio.write(fn2, [a, None, b])
    got = ref.call("bin_read_dcell", fn2)
    assert got[1] is None and np.array_equal(got[0], a) and np.array_equal(got[2], b)


def test_round_trip_other_types(tmp_path):
    rng = np.random.default_rng(3)
    for arr in (rng.standard_normal((5, 3)).astype(np.float32),
                (rng.standard_normal((2, 4)) + 1j * rng.standard_normal((2, 4))),
                (rng.standard_normal((3, 3)) + 1j * rng.standard_normal((3, 3))).astype(np.complex64),
                np.arange(12, dtype=np.int64).reshape(3, 4), np.arange(6, dtype=np.int32)):
        fn = str(tmp_path / "t.bin")
        binio.write(fn, arr)
        got = binio.read(fn)
        want = arr.reshape(-1, 1) if arr.ndim == 1 else arr
        assert got.dtype == arr.dtype and np.array_equal(got, want)
    assert os.path.getsize(fn) == 4 + 4 + 16 + 6 * 4
