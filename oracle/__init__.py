"""CPU oracle for the dense CP/Tucker path -- TEST INFRASTRUCTURE ONLY.

The checker the parity tests compare the CUDA library against.  It restates
the reference's algorithms (891922758/first-project, src/*.cu and the CPU
baseline decomposition/CPU/python/mycp.py) on the host: plain C in
oracle.c (loaded through ctypes) for the element-wise, MTTKRP, TTM and ALS
loops, and NumPy (LAPACK eigh) for the symmetric eigenproblems of HOSVD/HOOI.
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may use
it; the product library never does.

Pinning: tests/test_oracle_golden.py checks these functions against the exact
answers in tests/golden/ (generated by tests/golden/make_golden.py from the
reference drivers' integer fixtures).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
REF_LIB_PATH = os.path.join(_HERE, "_ref", "libref_cudecompose.so")


def build():
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


if not os.path.exists(LIB_PATH):
    build()
_lib = ctypes.CDLL(LIB_PATH)

_f = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_dp = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_u16 = np.ctypeslib.ndpointer(np.uint16, flags="C_CONTIGUOUS")
_l = ctypes.c_long


def _sig(name, args, res=None):
    fn = getattr(_lib, name)
    fn.argtypes = args
    fn.restype = res
    return fn


_sig("or_srand", [ctypes.c_uint])
_sig("or_fill_int", [_f, _l])
_sig("or_fill_frac", [_f, _l, ctypes.c_double])
_sig("or_fill_unit", [_f, _l])
_sig("or_hadmard", [_f, _f, _f, _l])
_sig("or_hadmard3", [_f, _f, _f, _f, _l])
_sig("or_tminust", [_f, _f, _l])
_sig("or_identity", [_f, _l])
_sig("or_kr", [_f, _f, _f, _l, _l, _l])
_sig("or_t2m", [_f, _f, _l, _l, _l, _l], ctypes.c_int)
_sig("or_tensor_product", [_f, _f, _f, _l, _l, _l, _l])
_sig("or_f2h", [_f, _u16, _l])
_sig("or_round_fp16", [_f, _f, _l])
_sig("or_round_bf16", [_f, _f, _l])
_sig("or_mttkrp", [_f, ctypes.c_int, ctypes.POINTER(_l), ctypes.POINTER(ctypes.c_void_p),
                   ctypes.c_int, _l, _dp])
_sig("or_mttkrp_legacy", [_f, _f, _f, _dp, _l, _l, _l, _l, _l, ctypes.c_int], ctypes.c_int)
_sig("or_ttm", [_f, _f, _dp, _l, _l, _l, _l, _l, ctypes.c_int], ctypes.c_int)
_sig("or_rse", [_f, _f, _l], ctypes.c_float)
_sig("or_gencp", [_dp, ctypes.c_int, ctypes.POINTER(_l), ctypes.POINTER(ctypes.c_void_p), _l])
_sig("or_mode_product", [_dp, ctypes.c_int, ctypes.POINTER(_l), ctypes.c_int, _dp, _l, _dp])
_sig("or_cp_als", [_f, ctypes.c_int, ctypes.POINTER(_l), _l, ctypes.POINTER(ctypes.c_void_p),
                   ctypes.c_int, ctypes.c_double, ctypes.c_int, _dp], ctypes.c_int)
_sig("or_unfold_gram", [_f, ctypes.c_int, ctypes.POINTER(_l), ctypes.c_int, _dp])


def _longs(xs):
    return (_l * len(xs))(*[int(x) for x in xs])


def _f32(x):
    return np.ascontiguousarray(x, dtype=np.float32).reshape(-1)


def _f64(x):
    return np.ascontiguousarray(x, dtype=np.float64).reshape(-1)


# ---------------------------------------------------------------- fixtures

def rand_int_fixture(seed: int, sizes):
    """glibc srand(seed) then the integer fill of test/test_mttkrp.cpp:27-39
    for consecutive arrays of the given sizes (X, A, B, C ...)."""
    _lib.or_srand(seed)
    out = []
    for n in sizes:
        a = np.zeros(int(n), np.float32)
        _lib.or_fill_int(a, int(n))
        out.append(a)
    return out


def rand_frac_fixture(seed: int | None, sizes, shift=0.0):
    """rand()*0.1/RAND_MAX (+shift) fill of test/test_t2m.cpp:12 /
    test/test_ttm.cpp:86; seed None keeps glibc's default seed (1)."""
    _lib.or_srand(1 if seed is None else seed)
    out = []
    for n in sizes:
        a = np.zeros(int(n), np.float32)
        _lib.or_fill_frac(a, int(n), float(shift))
        out.append(a)
    return out


def rand_unit_fixture(seed: int | None, sizes):
    _lib.or_srand(1 if seed is None else seed)
    out = []
    for n in sizes:
        a = np.zeros(int(n), np.float32)
        _lib.or_fill_unit(a, int(n))
        out.append(a)
    return out


# ---------------------------------------------------------------- primitives

def hadmard(A, B):
    A, B = _f32(A), _f32(B)
    C = np.empty_like(A)
    _lib.or_hadmard(A, B, C, A.size)
    return C


def hadmard3(A, B, K):
    A, B, K = _f32(A), _f32(B), _f32(K)
    D = np.empty_like(A)
    _lib.or_hadmard3(A, B, K, D, A.size)
    return D


def tminust(M, N):
    M, N = _f32(M), _f32(N).copy()
    _lib.or_tminust(M, N, M.size)
    return N


def identity(m):
    A = np.empty(m * m, np.float32)
    _lib.or_identity(A, m)
    return A


def kr(A, B, a, b, r):
    out = np.empty(a * b * r, np.float32)
    _lib.or_kr(_f32(A), _f32(B), out, a, b, r)
    return out


def t2m(T1, flag, m, n, k):
    T2 = np.zeros(m * n * k, np.float32)
    rc = _lib.or_t2m(_f32(T1), T2, flag, m, n, k)
    return T2 if rc == 0 else None


def tensor_product(A, B, a, b, c, d):
    C = np.empty(a * b * c * d, np.float32)
    _lib.or_tensor_product(_f32(A), _f32(B), C, a, b, c, d)
    return C


def f2h_bits(A):
    A = _f32(A)
    B = np.empty(A.size, np.uint16)
    _lib.or_f2h(A, B, A.size)
    return B


def round_fp16(A):
    A = _f32(A)
    B = np.empty_like(A)
    _lib.or_round_fp16(A, B, A.size)
    return B


def round_bf16(A):
    A = _f32(A)
    B = np.empty_like(A)
    _lib.or_round_bf16(A, B, A.size)
    return B


def rse(X, X1):
    """Returns (X - X1, ||X - X1|| / ||X||) as src/rse.cu:4-15."""
    X, X1 = _f32(X), _f32(X1).copy()
    e = _lib.or_rse(X, X1, X.size)
    return X1, float(e)


# ---------------------------------------------------------------- contractions

def mttkrp(X, dims, factors, mode, R):
    """FP64 MTTKRP of float X with the given factors (column-major)."""
    facs = [_f64(f) for f in factors]
    ptrs = (ctypes.c_void_p * len(facs))(*[f.ctypes.data for f in facs])
    out = np.zeros(int(dims[mode]) * int(R), np.float64)
    _lib.or_mttkrp(_f32(X), len(dims), _longs(dims), ptrs, mode, int(R), out)
    return out


def mttkrp_legacy(X, left, right, flag, m, n, k, r, round_fp16=True):
    q = {1: m, 2: n, 3: k}[flag]
    out = np.zeros(q * r, np.float64)
    _lib.or_mttkrp_legacy(_f32(X), _f32(left), _f32(right), out, flag, m, n, k, r,
                          1 if round_fp16 else 0)
    return out


def ttm(X, U, flag, a, b, c, d, round_fp16=False):
    n = {1: d * b * c, 2: a * d * c, 3: a * b * d}[flag]
    out = np.zeros(n, np.float64)
    _lib.or_ttm(_f32(X), _f32(U), out, flag, a, b, c, d, 1 if round_fp16 else 0)
    return out


def gencp(dims, factors, R):
    facs = [_f64(f) for f in factors]
    ptrs = (ctypes.c_void_p * len(facs))(*[f.ctypes.data for f in facs])
    n = int(np.prod(dims))
    out = np.zeros(n, np.float64)
    _lib.or_gencp(out, len(dims), _longs(dims), ptrs, int(R))
    return out


def mode_product(X, dims, mode, W, J):
    """Y = X x_mode W, W is J x dims[mode] column-major (FP64)."""
    X = _f64(X)
    out_dims = list(dims)
    out_dims[mode] = J
    Y = np.zeros(int(np.prod(out_dims)), np.float64)
    _lib.or_mode_product(X, len(dims), _longs(dims), mode, _f64(W), int(J), Y)
    return Y, out_dims


def gentucker(core, ranks, factors, dims):
    cur = list(ranks)
    Y = _f64(core)
    for m in range(len(dims)):
        Y, cur = mode_product(Y, cur, m, factors[m], dims[m])
    return Y


def unfold_gram(X, dims, mode):
    q = int(dims[mode])
    G = np.zeros(q * q, np.float64)
    _lib.or_unfold_gram(_f32(X), len(dims), _longs(dims), mode, G)
    return G.reshape(q, q)


# ---------------------------------------------------------------- decompositions

def cp_als(X, dims, R, init, max_sweeps, tol=0.0, use_lu=True):
    """CP-ALS of src/cp_als.cu:44-119 (any order), FP64, from `init`
    (list of column-major factors).  Returns (factors, fits, sweeps)."""
    facs = [_f64(f).copy() for f in init]
    ptrs = (ctypes.c_void_p * len(facs))(*[f.ctypes.data for f in facs])
    fits = np.zeros(max(1, max_sweeps), np.float64)
    sweeps = _lib.or_cp_als(_f32(X), len(dims), _longs(dims), int(R), ptrs, int(max_sweeps),
                            float(tol), 1 if use_lu else 0, fits)
    return facs, fits[:sweeps], sweeps


def cp_fit(X, dims, factors, R):
    rec = gencp(dims, factors, R)
    x = _f32(X).astype(np.float64)
    return 1.0 - np.linalg.norm(x - rec) / np.linalg.norm(x)


def _top_eigvecs(G, r):
    w, V = np.linalg.eigh(G)  # ascending, as syevdx
    return V[:, G.shape[0] - r:]


def tucker_hosvd(X, dims, ranks):
    """src/tucker_hosvd.cu:3-103 / src/tucker4_hosvd.cu:3-141 in FP64.
    Returns (core, factors) with column-major factors (dims[m] x ranks[m])."""
    facs = []
    for n in range(len(dims)):
        U = _top_eigvecs(unfold_gram(X, dims, n), ranks[n])
        facs.append(np.asfortranarray(U).reshape(-1, order="F"))
    core, _ = _project(X, dims, facs, ranks, skip=-1)
    return core, facs


def _project(X, dims, facs, ranks, skip):
    Y = _f32(X).astype(np.float64)
    cur = list(dims)
    for m in range(len(dims)):
        if m == skip:
            continue
        U = facs[m].reshape(dims[m], ranks[m], order="F")
        Y, cur = mode_product(Y, cur, m, np.asfortranarray(U.T).reshape(-1, order="F"), ranks[m])
    return Y, cur


def tucker_hooi(X, dims, ranks, sweeps=10):
    """decomposition/GPU/normal/tucker/tucker_hooi.cu:3-218 in FP64."""
    facs = [None] * len(dims)
    for n in range(1, len(dims)):
        U = _top_eigvecs(unfold_gram(X, dims, n), ranks[n])
        facs[n] = np.asfortranarray(U).reshape(-1, order="F")
    for _ in range(sweeps):
        for n in range(len(dims)):
            Y, cur = _project(X, dims, facs, ranks, skip=n)
            G = _gram64(Y, cur, n)
            U = _top_eigvecs(G, ranks[n])
            facs[n] = np.asfortranarray(U).reshape(-1, order="F")
    if sweeps == 0:
        facs[0] = np.asfortranarray(_top_eigvecs(unfold_gram(X, dims, 0), ranks[0])).reshape(-1, order="F")
    core, _ = _project(X, dims, facs, ranks, skip=-1)
    return core, facs


def _gram64(Y, dims, mode):
    T = np.asarray(Y, np.float64).reshape(tuple(reversed(dims)))
    T = np.moveaxis(T, len(dims) - 1 - mode, 0).reshape(dims[mode], -1)
    return T @ T.T


# ---------------------------------------------------------------- CPU baseline

def numpy_cp_als_sweep(X3, factors):
    """One sweep of the ALS of decomposition/CPU/python/mycp.py:10-20
    (Hadamard of Grams, MTTKRP through the KR product, solve), restated on
    NumPy arrays: X3 is the logical tensor (numpy, Fortran order), factors a
    list of (I_n x R) arrays, updated in place."""
    N = X3.ndim
    for n in range(N):
        V = np.ones((factors[0].shape[1],) * 2)
        for m in range(N):
            if m != n:
                V *= factors[m].T @ factors[m]
        M = unfolding_dot_khatri_rao(X3, factors, n)
        factors[n] = np.linalg.solve(V.T, M.T).T
    return factors


def unfolding_dot_khatri_rao(X3, factors, n):
    """X_(n) (KR of the other factors), column-major unfolding convention."""
    N = X3.ndim
    others = [m for m in range(N) if m != n]
    # KR with the earliest mode fastest
    K = factors[others[0]]
    for m in others[1:]:
        K = (factors[m][:, None, :] * K[None, :, :]).reshape(-1, K.shape[1])
    Xn = np.moveaxis(X3, n, 0).reshape(X3.shape[n], -1, order="F")
    return Xn @ K


# ---------------------------------------------------------------- learned warm start
# NumPy restatements of the workload generator and of the network's forward /
# backward pass (the library's csrc/warmstart.cu and gemm_tc.cu), for the
# warm-start parity tests.  The reference has no learned component; these pin
# the library's own generator and training kernels.

_M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def _mix64(z):
    """SplitMix64 finaliser (Steele, Lea and Flood, OOPSLA 2014), uint64
    arrays, wrapping arithmetic."""
    z = np.asarray(z, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def _hash3(seed, a, b):
    with np.errstate(over="ignore"):
        inner = _mix64(np.asarray(b, dtype=np.uint64) + np.uint64(0x632BE59BD9B4E019))
        mid = _mix64((np.asarray(a, dtype=np.uint64) * np.uint64(0x9E3779B97F4A7C15)) ^ inner)
    return _mix64(np.uint64(seed) ^ mid)


def _u01(h):
    return (np.asarray(h, dtype=np.uint64) >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def _normal2(h1, h2):
    u1 = 1.0 - _u01(h1)
    u2 = _u01(h2)
    return np.sqrt(-2.0 * np.log(u1)) * np.cos(np.pi * 2.0 * u2)


def ws_factors(gid, seed, I, R):
    """Generating factors of tensor `gid`: 3 column-major I x R matrices,
    columns sum_q a_q sin(2 pi w_q i / I + p_q)."""
    out = []
    i = np.arange(I, dtype=np.float64)
    for m in range(3):
        F = np.zeros((I, R))
        for r in range(R):
            col = m * R + r
            v = np.zeros(I)
            for q in range(3):
                b = col * 8 + q * 2
                w = 0.5 + 3.5 * _u01(_hash3(seed, gid, b * 4 + 0))
                p = 2.0 * np.pi * _u01(_hash3(seed, gid, b * 4 + 1))
                amp = _normal2(_hash3(seed, gid, b * 4 + 2), _hash3(seed, gid, b * 4 + 3))
                v += amp * np.sin(2.0 * np.pi * w * i / I + p)
            F[:, r] = v
        out.append(F.astype(np.float32).astype(np.float64))
    return out


def ws_tensor(gid, seed, I, R, noise):
    """The workload tensor (column-major, flattened) and its factors."""
    F = ws_factors(gid, seed, I, R)
    clean = np.einsum("ir,jr,kr->kji", *F).reshape(-1)  # element (i, j, k) at i + I j + I^2 k
    n = I ** 3
    norm2 = float(np.sum((F[0].T @ F[0]) * (F[1].T @ F[1]) * (F[2].T @ F[2])))
    sigma = noise * np.sqrt(norm2 / n)
    c = np.arange(n, dtype=np.uint64)
    s2 = np.uint64(seed) ^ np.uint64(0x5BD1E995)
    z = _normal2(_hash3(s2, gid, np.uint64(2) * c), _hash3(s2, gid, np.uint64(2) * c + np.uint64(1)))
    return (clean + sigma * z).astype(np.float32), F, norm2


def round_bf16_np(a):
    """Round-to-nearest-even to BF16, returned as float64 values."""
    x = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)
    lsb = (x >> np.uint32(16)) & np.uint32(1)
    r = (x + np.uint32(0x7FFF) + lsb) & np.uint32(0xFFFF0000)
    return r.view(np.float32).astype(np.float64)


def ws_mlp_grads(params, X, T):
    """Forward + backward of the warm-start MLP with the GPU path's rounding
    points: BF16 weights and activations, FP32 accumulation (here FP64), the
    MSE loss 1/(B D) sum (Y - T)^2.  Returns (loss, [gW1, gb1, gW2, gb2, gW3,
    gb3])."""
    W1, b1, W2, b2, W3, b3 = [np.asarray(p, np.float64) for p in params]
    W1h, W2h, W3h = round_bf16_np(W1), round_bf16_np(W2), round_bf16_np(W3)
    X = round_bf16_np(X)
    B, D = X.shape
    H1 = round_bf16_np(np.maximum(X @ W1h.T + b1, 0.0))
    H2 = round_bf16_np(np.maximum(H1 @ W2h.T + b2, 0.0))
    Y = (H2 @ W3h.T + b3).astype(np.float32).astype(np.float64)
    O = Y.shape[1]
    diff = (Y - T).astype(np.float32).astype(np.float64)
    loss = float(np.mean(diff ** 2))
    dY = round_bf16_np(diff * (2.0 / (B * O)))
    gW3, gb3 = dY.T @ H2, dY.sum(0)
    dH2 = round_bf16_np((dY @ W3h) * (H2 > 0))
    gW2, gb2 = dH2.T @ H1, dH2.sum(0)
    dH1 = round_bf16_np((dH2 @ W2h) * (H1 > 0))
    gW1, gb1 = dH1.T @ X, dH1.sum(0)
    return loss, [gW1, gb1, gW2, gb2, gW3, gb3]


# ---------------------------------------------------------------- reference GPU MTTKRP (baseline harness)

REF_GPU_PATH = os.path.join(_HERE, "_build", "libref_gpu.so")


class RefGpuMttkrp:
    """The reference's own GPU MTTKRP (its cuBLAS Khatri-Rao + SGEMM call
    sequence, oracle/ref_gpu.cu) on device buffers of one 3rd- or 4th-order
    problem.  Used as a timing baseline and checked against `mttkrp` by the
    GPU tests.  Arguments are raw device pointers (ints) and a stream handle.

    `factors` are the column-major dims[m] x R device buffers, `X` the flat
    column-major tensor.  Owns its scratch (the permuted copies the
    reference makes once, the Khatri-Rao matrices) through torch."""

    def __init__(self, torch, X, dims, factors, R, stream=None):
        self.torch = torch
        self.lib = ctypes.CDLL(REF_GPU_PATH)
        vp, l, i = ctypes.c_void_p, ctypes.c_long, ctypes.c_int
        self.lib.rg_create.argtypes = [ctypes.POINTER(vp), vp]
        self.lib.rg_destroy.argtypes = [vp]
        self.lib.rg_cp3_mttkrp.argtypes = [vp, i] + [vp] * 5 + [l] * 4 + [vp, vp]
        self.lib.rg_cp4_prepare.argtypes = [vp, vp, vp, vp, vp] + [l] * 4 + [vp]
        self.lib.rg_cp4_mttkrp.argtypes = [vp, i] + [vp] * 7 + [l] * 5 + [vp, vp, vp]
        self.dims, self.R = [int(d) for d in dims], int(R)
        self.X, self.U = X, list(factors)
        self.stream = stream
        h = vp()
        if self.lib.rg_create(ctypes.byref(h), stream) != 0:
            raise RuntimeError("cublasCreate failed")
        self.h = h
        dev = X.device
        n = X.numel()
        if len(dims) == 3:
            a, b, c = self.dims
            # X2: the mode-2 unfolding (b x ac), made once as the reference's
            # t2m does before its sweeps (src/cp_als.cu:28)
            self.X2 = X.view(c, b, a).permute(0, 2, 1).contiguous().view(-1)
            self.kr = torch.empty(max(b * c, a * c, a * b) * R, device=dev)
        elif len(dims) == 4:
            a, b, c, d = self.dims
            self.X2 = torch.empty(n, device=dev)
            self.X3 = torch.empty(n, device=dev)
            ident = torch.empty(a * b * a * b, device=dev)
            st = self.lib.rg_cp4_prepare(self.h, X.data_ptr(), self.X2.data_ptr(), self.X3.data_ptr(),
                                         ident.data_ptr(), a, b, c, d, stream)
            if st:
                raise RuntimeError("rg_cp4_prepare failed")
            torch.cuda.synchronize()
            del ident
            self.kr1 = torch.empty(max(c * d, a * b) * R, device=dev)
            self.kr = torch.empty(max(b * c * d, a * c * d, a * b * d, a * b * c) * R, device=dev)
        else:
            raise ValueError("the reference's CP-ALS has orders 3 and 4")
        self.out_t = torch.empty(max(self.dims) * R, device=dev)

    def run(self, mode):
        """Issue the mode's calls on the stream; the result (R x dims[mode],
        transposed, as the reference keeps it) lands in self.out_t.  In 4th
        order, modes 1 and 3 reuse the two-factor product that modes 0 and 2
        formed, as in the reference's sweep."""
        p = [u.data_ptr() for u in self.U]
        if len(self.dims) == 3:
            st = self.lib.rg_cp3_mttkrp(self.h, mode, self.X.data_ptr(), self.X2.data_ptr(), *p, *self.dims,
                                        self.R, self.kr.data_ptr(), self.out_t.data_ptr())
        else:
            st = self.lib.rg_cp4_mttkrp(self.h, mode, self.X.data_ptr(), self.X2.data_ptr(), self.X3.data_ptr(),
                                        *p, *self.dims, self.R, self.kr1.data_ptr(), self.kr.data_ptr(),
                                        self.out_t.data_ptr())
        if st:
            raise RuntimeError(f"reference MTTKRP mode {mode} failed")

    def result(self, mode):
        """dims[mode] x R column-major copy of the last result (host, FP64)."""
        q = self.dims[mode]
        t = self.out_t[: q * self.R].double().cpu().numpy()
        return t.reshape(self.R, q, order="F").T.reshape(-1, order="F")

    def close(self):
        if self.h:
            self.lib.rg_destroy(self.h)
            self.h = None


# ---------------------------------------------------------------- C++/OpenMP CPU baseline

CPU_ALS_PATH = os.path.join(_HERE, "_build", "libcpu_als.so")
_cpu = None


def _cpu_lib():
    global _cpu
    if _cpu is None:
        _cpu = ctypes.CDLL(CPU_ALS_PATH)
        vp, l, i, d = ctypes.c_void_p, ctypes.c_long, ctypes.c_int, ctypes.c_double
        for name in ("cpu_mttkrp_f32", "cpu_mttkrp_f64"):
            getattr(_cpu, name).argtypes = [vp, i, ctypes.POINTER(l), ctypes.POINTER(vp), i, l, vp, i]
        for name in ("cpu_cp_als_f32", "cpu_cp_als_f64"):
            getattr(_cpu, name).argtypes = [vp, i, ctypes.POINTER(l), l, ctypes.POINTER(vp), i, d, d, i, vp,
                                            ctypes.POINTER(i), ctypes.POINTER(d)]
        _cpu.cpu_max_threads.restype = i
    return _cpu


def cpu_threads():
    return int(_cpu_lib().cpu_max_threads())


def cpu_mttkrp(X, dims, factors, mode, R, threads=0):
    """The C++/OpenMP MTTKRP (oracle/cpu_als.cpp) in X's dtype (float32 or
    float64); returns dims[mode] x R column-major."""
    dt = np.float64 if np.asarray(X).dtype == np.float64 else np.float32
    X = np.ascontiguousarray(X, dt).reshape(-1)
    facs = [np.ascontiguousarray(f, dt).reshape(-1) for f in factors]
    out = np.zeros(int(dims[mode]) * int(R), dt)
    fn = _cpu_lib().cpu_mttkrp_f64 if dt == np.float64 else _cpu_lib().cpu_mttkrp_f32
    fn(X.ctypes.data, len(dims), _longs(dims), (ctypes.c_void_p * len(facs))(*[f.ctypes.data for f in facs]),
       int(mode), int(R), out.ctypes.data, int(threads))
    return out


def cpu_cp_als(X, dims, R, init, max_sweeps, tol=0.0, target_fit=0.0, threads=0):
    """The ALS of decomposition/CPU/python/mycp.py:7-22 in C++/OpenMP
    (oracle/cpu_als.cpp), in X's dtype, from `init`.  Returns (factors, fits,
    sweeps, seconds) -- seconds measured inside the C++ code."""
    dt = np.float64 if np.asarray(X).dtype == np.float64 else np.float32
    X = np.ascontiguousarray(X, dt).reshape(-1)
    facs = [np.array(f, dt).reshape(-1) for f in init]
    fits = np.zeros(max(1, max_sweeps), np.float64)
    sw, sec = ctypes.c_int(0), ctypes.c_double(0.0)
    fn = _cpu_lib().cpu_cp_als_f64 if dt == np.float64 else _cpu_lib().cpu_cp_als_f32
    st = fn(X.ctypes.data, len(dims), _longs(dims), int(R), (ctypes.c_void_p * len(facs))(*[f.ctypes.data for f in facs]),
            int(max_sweeps), float(tol), float(target_fit), int(threads), fits.ctypes.data, ctypes.byref(sw),
            ctypes.byref(sec))
    if st:
        raise RuntimeError(f"cpu_cp_als failed ({st})")
    return facs, fits[: sw.value], sw.value, sec.value
