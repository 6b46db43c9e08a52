"""Control-matrix MVM (FP32 / BF16 / FP8-E4M3 with per-row scales) on the GPU.

Each storage type is compared with an FP64 product of the same rounded
matrix (the rounding emulated on the CPU with torch's bf16 / float8_e4m3fn
casts); the only remaining difference is FP32 accumulation order, so the
tolerance is 1e-5 relative.  The storage error itself (vs FP64 M) is bounded
separately: BF16 < 1e-2, FP8 < 8e-2 relative on random matrices.
"""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def rounded(M, dtype):
    if dtype == 0:
        return M.astype(np.float32).astype(np.float64)
    if dtype == 1:
        return torch.from_numpy(M).to(torch.bfloat16).to(torch.float64).numpy()
    s = np.abs(M).max(axis=1, keepdims=True) / 448.0
    s[s == 0] = 1
    q = torch.from_numpy(M / s).to(torch.float8_e4m3fn).to(torch.float64).numpy()
    return q * s.astype(np.float32).astype(np.float64)


@pytest.mark.parametrize("dtype", [0, 1, 2])
@pytest.mark.parametrize("nbatch", [1, 3, 8, 20, 40])
def test_mvm_matches_rounded_product(dtype, nbatch):
    from maos_b200 import native
    lib = native.load()
    rng = np.random.default_rng(dtype * 10 + nbatch)
    nact, ngrad = 517, 4099  # ragged: not multiples of the tiles
    M = rng.standard_normal((nact, ngrad))
    g = rng.standard_normal((nbatch, ngrad))
    h = C.c_void_p()
    Mc = np.asfortranarray(M)
    native.check(lib.mb_mvm_create(Mc.ctypes.data_as(C.POINTER(C.c_double)), nact, ngrad, dtype,
                                   nbatch, C.byref(h)), "mb_mvm_create")
    out = np.empty((nbatch, nact))
    native.check(lib.mb_recon_mvm(h, g.ctypes.data_as(C.POINTER(C.c_double)),
                                  out.ctypes.data_as(C.POINTER(C.c_double))), "mb_recon_mvm")
    lib.mb_mvm_free(h)
    gf = g.astype(np.float32).astype(np.float64)
    want = gf @ rounded(M, dtype).T
    err = np.linalg.norm(out - want) / np.linalg.norm(want)
    assert err < 1e-5, err
    storage = np.linalg.norm(out - g @ M.T) / np.linalg.norm(g @ M.T)
    assert storage < (1e-5, 1e-2, 8e-2)[dtype]


@pytest.mark.parametrize("dtype", [1, 2])
def test_tensor_core_mvm_wide_dynamic_range(dtype):
    """Gradients spanning twelve decades within each instance, one instance all
    zero, on the tensor-core path (batch >= 4): the BF16 path's two terms and
    the FP8 path's four power-of-two-scaled E4M3 terms still give the product
    of the rounded matrix to 1e-5 per instance, and exactly zero for the zero
    instance."""
    from maos_b200 import native
    lib = native.load()
    rng = np.random.default_rng(40 + dtype)
    nact, ngrad, nbatch = 300, 2500, 12
    M = rng.standard_normal((nact, ngrad))
    g = rng.standard_normal((nbatch, ngrad)) * 10.0 ** rng.uniform(-6, 6, (nbatch, ngrad))
    g[0] = 0
    g[1] *= 1e-20  # small, still clear of FP32 subnormals in the BF16 low term
    h = C.c_void_p()
    Mc = np.asfortranarray(M)
    native.check(lib.mb_mvm_create(Mc.ctypes.data_as(C.POINTER(C.c_double)), nact, ngrad, dtype,
                                   nbatch, C.byref(h)), "mb_mvm_create")
    out = np.empty((nbatch, nact))
    native.check(lib.mb_recon_mvm(h, g.ctypes.data_as(C.POINTER(C.c_double)),
                                  out.ctypes.data_as(C.POINTER(C.c_double))), "mb_recon_mvm")
    lib.mb_mvm_free(h)
    want = g.astype(np.float32).astype(np.float64) @ rounded(M, dtype).T
    assert np.all(out[0] == 0)
    for b in range(1, nbatch):
        err = np.linalg.norm(out[b] - want[b]) / np.linalg.norm(want[b])
        assert err < 1e-5, (b, err)
