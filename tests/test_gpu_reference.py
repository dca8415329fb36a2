"""Parity against the reference itself, run on the same GPU.

oracle/_ref/libref_cudecompose.so is the reference library compiled from its
own sources (recipe: oracle/Makefile `ref`).  Its C++ entry points are called
through their mangled names.  Only routines whose code is free of the
reference's known latent faults are called (not cp_als/cp_als4/
cp_tensorcore, which write past a one-int pivot buffer or free the caller's
buffers, nor the printing 4th-order/tensor-core Tucker variants).

Also runs tests/drivers/drop_in.cpp -- a program written against the
reference's header -- linked against this repository's drop-in archive.
"""
import ctypes
import os
import subprocess

import numpy as np
import pytest
import torch

import oracle

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def ref():
    if not os.path.exists(oracle.REF_LIB_PATH):
        pytest.skip("reference library not built (oracle/Makefile ref)")
    lib = ctypes.CDLL(oracle.REF_LIB_PATH)
    vp, l = ctypes.c_void_p, ctypes.c_long
    sigs = {
        "mttkrp": ("_Z6mttkrpPfS_S_S_lllll", [vp] * 4 + [l] * 5),
        "kr": ("_Z2krPfS_S_lll", [vp] * 3 + [l] * 3),
        "hadmard": ("_Z7hadmardPfS_S_ll", [vp] * 3 + [l] * 2),
        "t2m": ("_Z3t2mPfS_llll", [vp] * 2 + [l] * 4),
        "ttm": ("_Z3ttmPfS_S_lllll", [vp] * 3 + [l] * 5),
        "gencp": ("_Z5gencpPfS_S_S_llll", [vp] * 4 + [l] * 4),
        "gentucker": ("_Z9gentuckerPfS_S_S_S_llllll", [vp] * 5 + [l] * 6),
        "tucker_hosvd": ("_Z12tucker_hosvdPfS_S_S_S_llllll", [vp] * 5 + [l] * 6),
        "tensor_product": ("_Z14tensor_productPfS_S_llll", [vp] * 3 + [l] * 4),
    }
    out = {}
    for k, (sym, args) in sigs.items():
        f = getattr(lib, sym)
        f.argtypes = args
        f.restype = None
        out[k] = f
    return out


def dev_t(a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def rel(a, b):
    return np.linalg.norm(np.asarray(a, np.float64) - b) / max(np.linalg.norm(b), 1e-300)


def test_bandwidth_primitives_bit_exact_vs_reference(cd, ref):
    rng = np.random.default_rng(0)
    a, b, r = 57, 43, 6
    A = dev_t(rng.standard_normal(a * r)); B = dev_t(rng.standard_normal(b * r))
    o1 = torch.empty(a * b * r, device="cuda"); o2 = torch.empty_like(o1)
    ref["kr"](A.data_ptr(), B.data_ptr(), o1.data_ptr(), a, b, r)
    cd.kr(A, B, o2, a, b, r)
    np.testing.assert_array_equal(host(o1), host(o2))
    ref["hadmard"](A.data_ptr(), A.data_ptr(), o1.data_ptr(), a, r)
    cd.hadmard(A, A, o2, a, r)
    np.testing.assert_array_equal(host(o1)[: a * r], host(o2)[: a * r])
    m, n, k = 31, 17, 12
    T = dev_t(rng.standard_normal(m * n * k))
    t1 = torch.empty_like(T); t2 = torch.empty_like(T)
    for flag in (1, 2, 3):
        ref["t2m"](T.data_ptr(), t1.data_ptr(), flag, m, n, k)
        cd.t2m(T, t2, flag, m, n, k)
        np.testing.assert_array_equal(host(t1), host(t2))
    P = dev_t(rng.standard_normal(3 * 4)); Q = dev_t(rng.standard_normal(5 * 2))
    k1 = torch.empty(120, device="cuda"); k2 = torch.empty(120, device="cuda")
    ref["tensor_product"](P.data_ptr(), Q.data_ptr(), k1.data_ptr(), 3, 4, 5, 2)
    cd.tensor_product(P, Q, k2, 3, 4, 5, 2)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(host(k1), host(k2))


def test_mttkrp_vs_reference(cd, ref, golden):
    # integer fixture: exact for both
    X, A, B, C = (dev_t(golden[k]) for k in ("mt_X", "mt_A", "mt_B", "mt_C"))
    o1 = torch.empty(6, device="cuda"); o2 = torch.empty(6, device="cuda")
    for flag, (left, right) in ((1, (C, B)), (2, (C, A)), (3, (B, A))):
        ref["mttkrp"](X.data_ptr(), left.data_ptr(), right.data_ptr(), o1.data_ptr(), flag, 3, 3, 3, 2)
        cd.mttkrp_legacy(X, left, right, o2, flag, 3, 3, 3, 2)
        np.testing.assert_array_equal(host(o1), host(o2))
    # Random data, FP16 operand semantics on both sides (X and every whole
    # Khatri-Rao entry rounded to FP16 once, src/mttkrp.cu:21-25, 41-47,
    # 65-69).  A product of two FP16 values is exact in FP32, so the only
    # error left is the FP32 accumulation.  Bound for ours, independent of
    # the box: every value here is non-negative, so each rounding moves the
    # result by at most its own relative error.  The tensor core truncates;
    # one output accumulates at most 2*SEG = 32 K16 MMAs per segment
    # (SEG = 16 stages of K = 32), each allowed 2 ulps (2^-22), then at most
    # 8 round-to-nearest segment flushes and the final FP64 -> FP32 rounding
    # (2^-24 each): 32 * 2^-22 + 9 * 2^-24 = 8.2e-6.
    bound = 32 * 2.0 ** -22 + 9 * 2.0 ** -24
    rng = np.random.default_rng(1)
    m, n, k, r = 64, 48, 40, 16
    X = dev_t(rng.random(m * n * k)); A = dev_t(rng.random(m * r)); B = dev_t(rng.random(n * r))
    C = dev_t(rng.random(k * r))
    o1 = torch.empty(64 * r, device="cuda"); o2 = torch.empty(64 * r, device="cuda")
    for flag, (left, right) in ((1, (C, B)), (2, (C, A)), (3, (B, A))):
        q = {1: m, 2: n, 3: k}[flag]
        ref["mttkrp"](X.data_ptr(), left.data_ptr(), right.data_ptr(), o1.data_ptr(), flag, m, n, k, r)
        cd.mttkrp_legacy(X, left, right, o2, flag, m, n, k, r)
        ours, theirs = host(o2)[: q * r].astype(np.float64), host(o1)[: q * r].astype(np.float64)
        # against the reference (cuBLAS GemmEx; its own accumulation order)
        assert rel(ours, theirs) <= 5e-5, (flag, rel(ours, theirs))
        # against the exact FP16-operand result, at the analytic bound
        want = oracle.mttkrp_legacy(host(X), host(left), host(right), flag, m, n, k, r, round_fp16=True)
        assert rel(ours, want) <= bound, (flag, rel(ours, want), rel(theirs, want))


def test_ttm_and_generators_vs_reference(cd, ref):
    rng = np.random.default_rng(2)
    a, b, c, d = 20, 18, 16, 5
    X = dev_t(rng.random(a * b * c))
    for flag, In in ((1, a), (2, b), (3, c)):
        U = dev_t(rng.random(d * In))
        n = {1: d * b * c, 2: a * d * c, 3: a * b * d}[flag]
        o1 = torch.empty(n, device="cuda"); o2 = torch.empty(n, device="cuda")
        ref["ttm"](X.data_ptr(), U.data_ptr(), o1.data_ptr(), flag, a, b, c, d)
        cd.ttm(X, U, o2, flag, a, b, c, d, precision=cd.PREC_FP16)
        assert rel(host(o2), host(o1).astype(np.float64)) <= 1e-5
    r = 4
    A = dev_t(rng.random(a * r)); B = dev_t(rng.random(b * r)); C = dev_t(rng.random(c * r))
    o1 = torch.empty(a * b * c, device="cuda"); o2 = torch.empty_like(o1)
    ref["gencp"](o1.data_ptr(), A.data_ptr(), B.data_ptr(), C.data_ptr(), a, b, c, r)
    cd.gencp(o2, [A, B, C], (a, b, c), r)
    assert rel(host(o2), host(o1).astype(np.float64)) <= 1e-6
    G = dev_t(rng.random(2 * 3 * 2))
    A2 = dev_t(rng.random(a * 2)); B2 = dev_t(rng.random(b * 3)); C2 = dev_t(rng.random(c * 2))
    ref["gentucker"](o1.data_ptr(), G.data_ptr(), A2.data_ptr(), B2.data_ptr(), C2.data_ptr(), a, b, c, 2, 3, 2)
    cd.gentucker(o2, G, [A2, B2, C2], (a, b, c), (2, 3, 2))
    assert rel(host(o2), host(o1).astype(np.float64)) <= 1e-6


def test_hosvd_vs_reference(cd, ref):
    rng = np.random.default_rng(3)
    dims, ranks = (48, 40, 36), (5, 4, 3)
    core = rng.standard_normal(int(np.prod(ranks)))
    facs = [np.linalg.qr(rng.standard_normal((d, r)))[0].reshape(-1, order="F") for d, r in zip(dims, ranks)]
    X = oracle.gentucker(core, ranks, facs, dims)
    X = (X + 1e-3 * np.linalg.norm(X) / np.sqrt(X.size) * rng.standard_normal(X.size)).astype(np.float32)
    dX = dev_t(X)
    U1 = [torch.empty(d * r, device="cuda") for d, r in zip(dims, ranks)]
    U2 = [torch.empty(d * r, device="cuda") for d, r in zip(dims, ranks)]
    g1 = torch.empty(int(np.prod(ranks)), device="cuda"); g2 = torch.empty_like(g1)
    ref["tucker_hosvd"](dX.data_ptr(), g1.data_ptr(), *[u.data_ptr() for u in U1], *dims, *ranks)
    cd.tucker_hosvd(dX, dims, ranks, g2, U2)
    for u1, u2, d, r in zip(U1, U2, dims, ranks):
        a1 = host(u1).reshape(d, r, order="F").astype(np.float64)
        a2 = host(u2).reshape(d, r, order="F").astype(np.float64)
        assert np.linalg.norm(a1 @ a1.T - a2 @ a2.T) <= 1e-3
    assert abs(np.linalg.norm(host(g1)) - np.linalg.norm(host(g2))) <= 1e-4 * np.linalg.norm(host(g1))


def test_drop_in_program_runs(golden, tmp_path):
    exe = tmp_path / "drop_in"
    inc = os.path.join(ROOT, "include")
    arc = os.path.join(ROOT, "first-project_b200", "libcutensordecomposition.a")
    r = subprocess.run(["nvcc", "-o", str(exe), os.path.join(ROOT, "tests", "drivers", "drop_in.cpp"),
                        "-I", inc, arc, "-lcublas", "-lcusolver", "-lcurand"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stderr
    vals = {}
    for line in out.stdout.strip().splitlines():
        parts = line.split()
        vals[parts[0]] = np.array([float(x) for x in parts[1:]])
    np.testing.assert_array_equal(vals["mttkrp1"], golden["mt_out1"])
    np.testing.assert_array_equal(vals["mttkrp2"], golden["mt_out2"])
    np.testing.assert_array_equal(vals["mttkrp3"], golden["mt_out3"])
    X, A, B, C = (golden[k] for k in ("mt_X", "mt_A", "mt_B", "mt_C"))
    np.testing.assert_array_equal(vals["kr"], oracle.kr(A, B, 3, 3, 2))
    np.testing.assert_array_equal(vals["hadmard"], oracle.hadmard(A, B))
    np.testing.assert_array_equal(vals["t2m2"], oracle.t2m(X, 2, 3, 3, 3))
    np.testing.assert_array_equal(vals["t2m3"], oracle.t2m(X, 3, 3, 3, 3))
    np.testing.assert_array_equal(vals["gencp"], oracle.gencp((3, 3, 3), [A, B, C], 2))
    assert vals["status"][0] == 0


@pytest.mark.parametrize("dims,R", [((40, 36, 28), 8), ((12, 10, 9, 8), 5)])
def test_reference_gpu_mttkrp_harness(dims, R):
    """The baseline harness that times the reference's GPU MTTKRP (its
    Khatri-Rao + SGEMM calls) computes the MTTKRP: every mode against the
    FP64 oracle at the FP32 bar."""
    if not os.path.exists(oracle.REF_GPU_PATH):
        pytest.skip("baseline harness not built (make -C oracle)")
    rng = np.random.default_rng(sum(dims) + R)
    X = rng.random(int(np.prod(dims))).astype(np.float32)
    facs = [rng.random(d * R).astype(np.float32) for d in dims]
    h = oracle.RefGpuMttkrp(torch, dev_t(X), dims, [dev_t(f) for f in facs], R)
    try:
        for mode in range(len(dims)):
            h.run(mode)
            torch.cuda.synchronize()
            assert rel(h.result(mode), oracle.mttkrp(X, dims, facs, mode, R)) <= 1e-5, mode
    finally:
        h.close()


def test_print_tensor_same_text_as_reference(tmp_path):
    """printTensor (src/kr.cu:13-30): the same program linked against the
    drop-in archive and against the reference library prints the same
    bytes."""
    if not os.path.exists(oracle.REF_LIB_PATH):
        pytest.skip("reference library not built (oracle/Makefile ref)")
    src = os.path.join(ROOT, "tests", "drivers", "print_tensor.cpp")
    inc = os.path.join(ROOT, "include")
    ours, theirs = tmp_path / "print_ours", tmp_path / "print_ref"
    arc = os.path.join(ROOT, "first-project_b200", "libcutensordecomposition.a")
    r = subprocess.run(["nvcc", "-o", str(ours), src, "-I", inc, arc, "-lcublas", "-lcusolver", "-lcurand"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    refdir = os.path.dirname(oracle.REF_LIB_PATH)
    r = subprocess.run(["nvcc", "-o", str(theirs), src, "-I", inc, oracle.REF_LIB_PATH,
                        f"-Xlinker=-rpath,{refdir}", "-lcublas", "-lcusolver", "-lcurand"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    a = subprocess.run([str(ours)], capture_output=True, text=True, timeout=120)
    b = subprocess.run([str(theirs)], capture_output=True, text=True, timeout=120)
    assert a.returncode == 0 and b.returncode == 0, (a.stderr, b.stderr)
    assert a.stdout == b.stdout
    assert a.stdout.count("-----------------------------------") == 2


def test_tucker_tensorcore_vs_reference_and_fp64(cd, capfd):
    """tucker_tensorcore (src/tucker_tensorcore.cu:3-139) as a drop-in: the
    reference rounds X, the factors and the TTM chain to FP16 and leaves
    U1..U3 unwritten; ours runs three-term BF16 and writes them.  The core
    (sign-invariant norm) of both against the FP64 HOSVD's: ours at the
    FP32-level bar, the reference's at FP16's; our factors' subspaces against
    FP64 eigh.  The printed errors of both are close."""
    if not os.path.exists(oracle.REF_LIB_PATH):
        pytest.skip("reference library not built (oracle/Makefile ref)")
    rng = np.random.default_rng(31)
    dims, ranks = (64, 48, 40), (6, 5, 4)
    core0 = rng.standard_normal(int(np.prod(ranks)))
    facs = [np.linalg.qr(rng.standard_normal((d, r)))[0].reshape(-1, order="F") for d, r in zip(dims, ranks)]
    X = oracle.gentucker(core0, ranks, facs, dims)
    X = (X + 1e-3 * np.linalg.norm(X) / np.sqrt(X.size) * rng.standard_normal(X.size)).astype(np.float32)
    c64, f64 = oracle.tucker_hosvd(X, dims, ranks)
    n64 = np.linalg.norm(c64)
    vp, l = ctypes.c_void_p, ctypes.c_long
    out = {}
    for name, path in (("ours", cd.LIB_PATH), ("ref", oracle.REF_LIB_PATH)):
        lib = ctypes.CDLL(path)
        f = getattr(lib, "_Z17tucker_tensorcorePfS_S_S_S_llllll")
        f.argtypes = [vp] * 5 + [l] * 6
        f.restype = None
        dX = dev_t(X)
        core = torch.zeros(int(np.prod(ranks)), device="cuda")
        U = [torch.zeros(d * r, device="cuda") for d, r in zip(dims, ranks)]
        capfd.readouterr()
        f(dX.data_ptr(), core.data_ptr(), *[u.data_ptr() for u in U], *dims, *ranks)
        torch.cuda.synchronize()
        printed = float(capfd.readouterr().out.strip().splitlines()[-1])
        out[name] = (host(core).astype(np.float64), [host(u) for u in U], printed)
    core_o, U_o, err_o = out["ours"]
    core_r, _, err_r = out["ref"]
    assert abs(np.linalg.norm(core_o) - n64) <= 1e-5 * n64
    assert abs(np.linalg.norm(core_r) - n64) <= 2e-3 * n64
    for u, w, d, r in zip(U_o, f64, dims, ranks):
        a1 = u.reshape(d, r, order="F").astype(np.float64)
        a2 = w.reshape(d, r, order="F")
        assert np.linalg.norm(a1 @ a1.T - a2 @ a2.T) <= 1e-4
    # the printed relative error ||X - Xhat|| / ||X||: ours is the FP64
    # model's to 2 %; the reference's (FP16 core) is of the same magnitude
    rec = oracle.gentucker(c64, ranks, f64, dims)
    e64 = np.linalg.norm(X.astype(np.float64) - rec) / np.linalg.norm(X.astype(np.float64))
    assert abs(err_o - e64) <= 0.02 * e64, (err_o, e64)
    assert abs(err_o - err_r) <= 0.5 * max(err_o, err_r), (err_o, err_r)


def test_tucker_hosvd4_printed_error_vs_reference_and_fp64(cd, capfd):
    """tucker_hosvd4 (src/tucker4_hosvd.cu:3-141) prints the relative
    reconstruction error of its model (:123-129, gentucker4 + rse).  Ours and
    the reference's printed values against the FP64 HOSVD model's, and the
    cores' norms against each other."""
    if not os.path.exists(oracle.REF_LIB_PATH):
        pytest.skip("reference library not built (oracle/Makefile ref)")
    rng = np.random.default_rng(41)
    dims, ranks = (24, 20, 18, 16), (4, 3, 3, 2)
    core0 = rng.standard_normal(int(np.prod(ranks)))
    facs = [np.linalg.qr(rng.standard_normal((d, r)))[0].reshape(-1, order="F") for d, r in zip(dims, ranks)]
    X = oracle.gentucker(core0, ranks, facs, dims)
    X = (X + 1e-2 * np.linalg.norm(X) / np.sqrt(X.size) * rng.standard_normal(X.size)).astype(np.float32)
    c64, f64 = oracle.tucker_hosvd(X, dims, ranks)
    rec = oracle.gentucker(c64, ranks, f64, dims)
    e64 = np.linalg.norm(X.astype(np.float64) - rec) / np.linalg.norm(X.astype(np.float64))
    vp, l = ctypes.c_void_p, ctypes.c_long
    out = {}
    for name, path in (("ours", cd.LIB_PATH), ("ref", oracle.REF_LIB_PATH)):
        lib = ctypes.CDLL(path)
        f = getattr(lib, "_Z13tucker_hosvd4PfS_S_S_S_S_llllllll")
        f.argtypes = [vp] * 6 + [l] * 8
        f.restype = None
        dX = dev_t(X)
        core = torch.zeros(int(np.prod(ranks)), device="cuda")
        U = [torch.zeros(d * r, device="cuda") for d, r in zip(dims, ranks)]
        capfd.readouterr()
        f(dX.data_ptr(), core.data_ptr(), *[u.data_ptr() for u in U], *dims, *ranks)
        torch.cuda.synchronize()
        printed = float(capfd.readouterr().out.strip().splitlines()[-1])
        out[name] = (np.linalg.norm(host(core).astype(np.float64)), printed)
    (n_o, err_o), (n_r, err_r) = out["ours"], out["ref"]
    assert abs(n_o - n_r) <= 1e-4 * n_r
    assert abs(err_o - e64) <= 0.02 * e64, (err_o, e64)
    assert abs(err_r - e64) <= 0.02 * e64, (err_r, e64)
