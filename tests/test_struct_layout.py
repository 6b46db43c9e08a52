"""The ctypes mirrors in ``maos_b200.native`` match the C structs of
``include/maos_b200.h`` field by field (offset and size), as gcc lays them
out: a wrong mirror would pass garbage through the ABI silently."""
import os
import shutil
import subprocess
import tempfile

import pytest

from maos_b200 import native

HERE = os.path.dirname(os.path.abspath(__file__))
INC = os.path.join(HERE, "..", "include")

PAIRS = [("mb_grid", native.MbGrid), ("mb_wfs_desc", native.MbWfsDesc), ("mb_fdpcg_desc", native.MbFdpcgDesc),
         ("mb_fdpcg_geom", native.MbFdpcgGeom),
         ("mb_csc", native.MbCsc), ("mb_fit_desc", native.MbFitDesc),
         ("mb_fit_sparse_desc", native.MbFitSparseDesc), ("mb_recon_desc", native.MbReconDesc),
         ("mb_geom_wfs_desc", native.MbGeomWfsDesc)]


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no C compiler")
def test_ctypes_structs_match_header():
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "maos_b200.h"', "int main(void) {"]
    for cname, py in PAIRS:
        lines.append(f'printf("{cname} size %zu\\n", sizeof({cname}));')
        for f, _ in py._fields_:
            lines.append(f'printf("{cname} {f} %zu %zu\\n", offsetof({cname}, {f}), sizeof((({cname} *)0)->{f}));')
    lines.append("return 0; }")
    with tempfile.TemporaryDirectory() as d:
        src = os.path.join(d, "layout.c")
        exe = os.path.join(d, "layout")
        with open(src, "w") as fh:
            fh.write("\n".join(lines))
        subprocess.run(["gcc", "-I", INC, src, "-o", exe], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split("\n")
    got = {}
    for ln in out:
        parts = ln.split()
        if len(parts) == 3:
            got[(parts[0], "size")] = int(parts[2])
        elif len(parts) == 4:
            got[(parts[0], parts[1])] = (int(parts[2]), int(parts[3]))
    for cname, py in PAIRS:
        assert got[(cname, "size")] == C_sizeof(py), cname
        for f, t in py._fields_:
            off, size = got[(cname, f)]
            assert getattr(py, f).offset == off and getattr(py, f).size == size, (cname, f)


def C_sizeof(t):
    import ctypes
    return ctypes.sizeof(t)
