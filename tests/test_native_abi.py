"""The C-ABI library builds, loads, and exports every symbol include/maos_b200.h declares.

CPU only: no compute calls are made (there may be no GPU)."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", f) for f in os.listdir(os.path.join(ROOT, "include"))
           if f.endswith(".h")]


def declared_symbols():
    names = set()
    for h in HEADERS:
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w \*]*?\b(mb_\w+)\s*\(", src, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


@pytest.fixture(scope="module")
def lib():
    from maos_b200 import build, native
    build.build()
    return native.load()


def test_header_declares_entry_points():
    names = declared_symbols()
    for n in ("mb_setup_recon", "mb_tomo", "mb_recon_reset", "mb_update_recon_cn2",
              "mb_update_recon_nea", "mb_init", "mb_cleanup"):
        assert n in names


def test_library_exports_every_declared_symbol(lib):
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header(lib):
    from maos_b200 import native
    assert set(declared_symbols()) <= set(native.SIGNATURES)


def test_error_strings(lib):
    assert lib.mb_error_string(0) == b"ok"
    assert lib.mb_error_string(-5) == b"unsupported geometry"
    assert lib.mb_version() >= 1


def test_null_arguments_are_rejected_without_a_gpu(lib):
    # argument checks happen before any CUDA call
    assert lib.mb_setup_recon(None, None) == -1
    assert lib.mb_tomo(None, None, None, None) == -1
    assert lib.mb_recon_reset(None) == -1


def test_mvm_rejects_bad_arguments(lib):
    import numpy as np
    h = ctypes.c_void_p()
    M = np.zeros(4)
    P = ctypes.POINTER(ctypes.c_double)
    lib.mb_mvm_create.argtypes = [P, ctypes.c_long, ctypes.c_long, ctypes.c_int, ctypes.c_int,
                                  ctypes.POINTER(ctypes.c_void_p)]
    assert lib.mb_mvm_create(M.ctypes.data_as(P), 2, 2, 7, 1, ctypes.byref(h)) == -1
    assert lib.mb_mvm_create(None, 2, 2, 0, 1, ctypes.byref(h)) == -1
