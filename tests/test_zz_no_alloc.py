"""cud_mttkrp_noalloc -- the MTTKRP entry point for callers that cannot
allocate device memory (code inside a custom allocator's own hooks, where
cudaMalloc would re-enter the allocator; frameworks that own all device
memory): it must give the same result as cud_mttkrp while taking its
workspace from the library's fixed device array, and must reject a problem
whose workspace would not fit.

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


_FRESH = r'''
import ctypes, json, sys
import numpy as np
import torch
sys.path[:0] = [sys.argv[1]]
import cudecompose as cd
lib = cd.library()
f = lib.cud_mttkrp_noalloc
f.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.POINTER(ctypes.c_long),
              ctypes.POINTER(ctypes.c_void_p), ctypes.c_int, ctypes.c_long, ctypes.c_void_p,
              ctypes.c_int, ctypes.c_void_p]
f.restype = ctypes.c_int
rng = np.random.default_rng(5)
# small problem first, then one whose workspace (18 splits x 2048 x 32 floats,
# 4.7 MB) an allocating path would have to cudaMalloc
probs = []
for dims, R in (((256, 96, 64), 32), ((2048, 96, 64), 32)):
    X = torch.from_numpy(rng.random(int(np.prod(dims))).astype(np.float32)).cuda()
    U = [torch.from_numpy(rng.random(d * R).astype(np.float32)).cuda() for d in dims]
    probs.append((dims, R, X, U, torch.empty(dims[0] * R, device="cuda"), torch.empty(dims[0] * R, device="cuda")))
torch.cuda.synchronize()
free = [torch.cuda.mem_get_info()[0]]
sts = []
for dims, R, X, U, got, _ in probs:   # the library's first calls in this process
    d = (ctypes.c_long * 3)(*dims)
    p = (ctypes.c_void_p * 3)(*[u.data_ptr() for u in U])
    sts.append(f(X.data_ptr(), 3, d, p, 0, R, got.data_ptr(), cd.PREC_BF16X3, None))
    torch.cuda.synchronize()
    free.append(torch.cuda.mem_get_info()[0])
errs = []
for dims, R, X, U, got, want in probs:
    cd.mttkrp(X, dims, U, 0, R, want, cd.PREC_BF16X3)
    torch.cuda.synchronize()
    g, w = got.double().cpu().numpy(), want.double().cpu().numpy()
    errs.append(float(np.linalg.norm(g - w) / np.linalg.norm(w)))
print(json.dumps({"status": sts, "free": free, "errs": errs}))
'''


def test_noalloc_first_calls_allocate_nothing(tmp_path):
    """In a fresh process, before any other library call: the first call may
    load the module that holds the static array (committing its 32 MiB under
    lazy loading), but the second call -- whose workspace is larger than the
    first's -- must leave the device's free memory unchanged.  A workspace
    taken from an allocating arena would lower it by at least 4.7 MB (2 MiB
    cudaMalloc granularity); the bar is 2 MiB."""
    import json
    import os
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    script = tmp_path / "fresh_noalloc.py"
    script.write_text(_FRESH)
    r = subprocess.run([sys.executable, str(script), os.path.join(root, "first-project_b200")],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    res = json.loads(r.stdout.strip().splitlines()[-1])
    assert res["status"] == [0, 0], res
    free = res["free"]
    assert free[1] - free[2] < (2 << 20), free
    assert max(res["errs"]) <= 1e-6, res["errs"]
