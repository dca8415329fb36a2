"""cud_mttkrp_noalloc -- the MTTKRP entry point for callers that cannot
allocate device memory (host callbacks, allocator hooks, frameworks that own
all device memory): it must give the same result as cud_mttkrp while taking
its workspace from the library's fixed device array, and must reject a
problem whose workspace would not fit.

Called through the C ABI with ctypes.  Collected last (file name) so that a
run stopping at the first failure has run every other test before it; it
also passes on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _noalloc(cd):
    lib = cd.library()
    f = lib.cud_mttkrp_noalloc
    f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_long),
                  ctypes.POINTER(ctypes.c_void_p), ctypes.c_int, ctypes.c_long, ctypes.c_void_p,
                  ctypes.c_int, ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f


def _call(cd, f, X, dims, U, mode, R, out, prec):
    d = (ctypes.c_long * len(dims))(*dims)
    p = (ctypes.c_void_p * len(U))(*[u.data_ptr() for u in U])
    return f(X.data_ptr(), len(dims), d, p, mode, R, out.data_ptr(), prec, None)


@pytest.mark.parametrize("prec", ["bf16x3", "fp32"])
def test_noalloc_matches_mttkrp_twice(cd, prec):
    f = _noalloc(cd)
    P = cd.PRECISIONS[prec]
    rng = np.random.default_rng(17)
    for call, (dims, R) in enumerate([((256, 96, 64), 32), ((120, 200, 36), 16)]):
        X = torch.from_numpy(rng.random(int(np.prod(dims))).astype(np.float32)).cuda()
        U = [torch.from_numpy(rng.random(d * R).astype(np.float32)).cuda() for d in dims]
        for mode in range(3):
            want = torch.empty(dims[mode] * R, device="cuda")
            cd.mttkrp(X, dims, U, mode, R, want, P)
            got = torch.full((dims[mode] * R,), float("nan"), device="cuda")
            st = _call(cd, f, X, dims, U, mode, R, got, P)
            assert st == 0, cd.library().cud_last_error_detail()
            torch.cuda.synchronize()
            g, w = got.double().cpu().numpy(), want.double().cpu().numpy()
            assert np.linalg.norm(g - w) <= 1e-6 * np.linalg.norm(w), (call, mode)


def test_noalloc_rejects_oversized_workspace(cd):
    f = _noalloc(cd)
    dims, R = (200000, 4, 4), 64   # one split of 200000 x 64 floats > 32 MiB
    X = torch.zeros(8, device="cuda")
    U = [torch.zeros(8, device="cuda") for _ in dims]
    out = torch.zeros(8, device="cuda")
    st = _call(cd, f, X, dims, U, 0, R, out, cd.PREC_BF16X3)
    assert st == cd.ERR_INVALID_ARGUMENT
    assert b"exceeds" in cd.library().cud_last_error_detail()
