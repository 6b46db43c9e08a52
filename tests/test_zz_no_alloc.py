"""The allocation-free MVM entry point against the allocating one.

Callers such as a real-time control loop cannot allocate device memory
during operation (cudaMalloc can synchronise the device and take unbounded
time), so mb_mvm_apply_noalloc keeps its split-K partial sums in a static
device array instead.  This test calls it through the C ABI twice in a row
and compares each result with mb_mvm_apply_device (an mb_mvm built with FP32
storage) and with the FP64 product of the FP32-rounded matrix and gradients,
within the MVM tests' tolerance, 1e-5 relative.  It also checks that a request
too large for the static array is refused with a message, including sizes
whose product would overflow a 64-bit integer.
"""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

TOL = 1e-5


def test_noalloc_mvm_matches_allocating_entry_point():
    from maos_b200 import native
    lib = native.load()
    rng = np.random.default_rng(42)
    nact, ngrad, nbatch = 777, 5003, 3          # ragged sizes: tail paths exercised
    ldm = (ngrad + 3) // 4 * 4
    M = rng.standard_normal((nact, ngrad))
    g = torch.tensor(rng.standard_normal((nbatch, ngrad)), dtype=torch.float32, device="cuda")
    # existing entry point: mb_mvm built from the FP64 column-major matrix
    h = C.c_void_p()
    Mc = np.asfortranarray(M)
    native.check(lib.mb_mvm_create(Mc.ctypes.data_as(C.POINTER(C.c_double)), nact, ngrad, 0, nbatch,
                                   C.byref(h)), "mb_mvm_create")
    want = torch.empty(nbatch, nact, device="cuda")
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        native.check(lib.mb_mvm_apply_device(h, C.c_void_p(g.data_ptr()), C.c_void_p(want.data_ptr()),
                                             C.c_void_p(stream.cuda_stream)), "mb_mvm_apply_device")
    torch.cuda.synchronize()
    lib.mb_mvm_free(h)
    # the caller owns M, the gradients and the output on the device
    Md = torch.zeros(nact, ldm, dtype=torch.float32, device="cuda")
    Md[:, :ngrad] = torch.tensor(M, dtype=torch.float32, device="cuda")
    # FP64 product of the FP32-rounded operands
    want64 = g.double().cpu().numpy() @ M.astype(np.float32).astype(np.float64).T
    for call in range(2):
        out = torch.full((nbatch, nact), float("nan"), device="cuda")
        with torch.cuda.stream(stream):
            native.check(lib.mb_mvm_apply_noalloc(C.c_void_p(Md.data_ptr()), nact, ngrad, ldm,
                                                  C.c_void_p(g.data_ptr()), C.c_void_p(out.data_ptr()),
                                                  nbatch, C.c_void_p(stream.cuda_stream)),
                         f"mb_mvm_apply_noalloc call {call}")
        torch.cuda.synchronize()
        err = (torch.linalg.norm(out - want) / torch.linalg.norm(want)).item()
        assert err < TOL, (call, err)
        o64 = out.double().cpu().numpy()
        err64 = np.linalg.norm(o64 - want64) / np.linalg.norm(want64)
        assert err64 < TOL, (call, err64)


def test_noalloc_rejects_requests_beyond_the_static_scratch():
    from maos_b200 import native
    lib = native.load()
    M = torch.zeros(4, 4, device="cuda")
    g = torch.zeros(1, 4, device="cuda")
    out = torch.zeros(1, 4, device="cuda")
    # 2,000,000 rows need more partial sums than MB_NOALLOC_MAX_PARTIALS
    rc = lib.mb_mvm_apply_noalloc(C.c_void_p(M.data_ptr()), 2_000_000, 4, 4, C.c_void_p(g.data_ptr()),
                                  C.c_void_p(out.data_ptr()), 1, None)
    assert rc == -1
    assert b"static scratch holds" in lib.mb_last_error_message()
    # factors whose product overflows a signed 64-bit integer are refused too
    for nact, ngrad, nb in ((1 << 62, 4, 1), (1 << 40, 1 << 40, 1 << 20), (3, 1 << 62, 1)):
        rc = lib.mb_mvm_apply_noalloc(C.c_void_p(M.data_ptr()), nact, ngrad, 1 << 62, C.c_void_p(g.data_ptr()),
                                      C.c_void_p(out.data_ptr()), min(nb, 1 << 30), None)
        assert rc == -1, (nact, ngrad, nb)
