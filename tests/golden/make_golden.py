"""Generates tests/golden/golden.npz: known-answer vectors for the hot path.

Inputs are the fixtures of the reference's own driver programs
(891922758/first-project, test/*.cpp and the hand-written tensors in
decomposition/GPU/normal/{cp,tucker}/de_*.cpp), regenerated here with glibc
rand() called through ctypes and the drivers' exact float expressions.
Expected outputs are computed independently of the oracle and of the
library: with Python integers / fractions where the data are integers, and
with IEEE single-rounding NumPy float32 arithmetic for the element-wise and
permutation primitives whose reference definition is one rounding per
element.

Run:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import ctypes
import os
from fractions import Fraction

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
libc = ctypes.CDLL("libc.so.6")
libc.rand.restype = ctypes.c_int
RAND_MAX = 2147483647
F32_RAND_MAX = np.float32(RAND_MAX)  # int -> float conversion in the C expressions


def srand(seed):
    libc.srand(ctypes.c_uint(seed))


def fill_int(n):
    # float(int(10*(((float) rand())/RAND_MAX - 0.5)))   test/test_mttkrp.cpp:29
    out = np.empty(n, np.float32)
    for i in range(n):
        f = np.float32(np.float32(libc.rand()) / F32_RAND_MAX)
        out[i] = np.float32(int(10.0 * (float(f) - 0.5)))
    return out


def fill_frac(n, shift=0.0):
    # rand()*0.1/(RAND_MAX) (- 0.5)    test/test_t2m.cpp:12, test/test_ttm.cpp:86
    out = np.empty(n, np.float32)
    for i in range(n):
        out[i] = np.float32(libc.rand() * 0.1 / RAND_MAX + shift)
    return out


def cm(a, shape):
    """flat column-major -> nested-index accessor (numpy Fortran view)."""
    return np.asarray(a).reshape(shape, order="F")


def exact_mttkrp(X, dims, factors, mode):
    """integer MTTKRP with Python ints."""
    Xi = cm(X, dims).astype(np.int64)
    facs = [None if f is None else cm(f, (d, -1)).astype(np.int64) for f, d in zip(factors, dims)]
    R = next(f.shape[1] for f in facs if f is not None)
    out = np.zeros((dims[mode], R), dtype=object)
    for idx in np.ndindex(*dims):
        x = int(Xi[idx])
        if x == 0:
            continue
        for r in range(R):
            w = x
            for m, i in enumerate(idx):
                if m != mode:
                    w *= int(facs[m][i, r])
            out[idx[mode], r] += w
    return np.asarray(out.reshape(-1, order="F"), dtype=np.float64)


def exact_gencp(dims, factors):
    facs = [cm(f, (d, -1)).astype(np.int64) for f, d in zip(factors, dims)]
    R = facs[0].shape[1]
    out = np.zeros(dims, dtype=object)
    for idx in np.ndindex(*dims):
        s = 0
        for r in range(R):
            p = 1
            for m, i in enumerate(idx):
                p *= int(facs[m][i, r])
            s += p
        out[idx] = s
    return np.asarray(out.reshape(-1, order="F"), dtype=np.float64)


def exact_gentucker(core, ranks, factors, dims):
    G = cm(core, ranks).astype(np.int64)
    facs = [cm(f, (d, r)).astype(np.int64) for f, d, r in zip(factors, dims, ranks)]
    out = np.zeros(dims, dtype=object)
    for idx in np.ndindex(*dims):
        s = 0
        for jdx in np.ndindex(*ranks):
            p = int(G[jdx])
            for m in range(len(dims)):
                p *= int(facs[m][idx[m], jdx[m]])
            s += p
        out[idx] = s
    return np.asarray(out.reshape(-1, order="F"), dtype=np.float64)


def exact_als_step(X, dims, factors, mode, R):
    """One exact ALS update of factor `mode` (rational arithmetic):
    U_n = MTTKRP_n * (Hadamard_{m != n} U_m^T U_m)^-1."""
    M = exact_mttkrp(X, dims, factors, mode).reshape(dims[mode], R, order="F")
    V = [[Fraction(1)] * R for _ in range(R)]
    for m, f in enumerate(factors):
        if m == mode:
            continue
        F = cm(f, (dims[m], R)).astype(np.int64)
        for a in range(R):
            for b in range(R):
                V[a][b] *= sum(int(F[i, a]) * int(F[i, b]) for i in range(dims[m]))
    # invert V (Gauss-Jordan over Fractions)
    n = R
    A = [row[:] + [Fraction(int(i == j)) for j in range(n)] for i, row in enumerate(V)]
    for c in range(n):
        p = next(r for r in range(c, n) if A[r][c] != 0)
        A[c], A[p] = A[p], A[c]
        pv = A[c][c]
        A[c] = [v / pv for v in A[c]]
        for r in range(n):
            if r != c and A[r][c] != 0:
                f = A[r][c]
                A[r] = [a - f * b for a, b in zip(A[r], A[c])]
    Vinv = [row[n:] for row in A]
    U = np.zeros((dims[mode], R), dtype=object)
    for i in range(dims[mode]):
        for c in range(R):
            U[i, c] = sum(Fraction(int(M[i, r])) * Vinv[r][c] for r in range(R))
    return np.array([float(v) for v in U.reshape(-1, order="F")], dtype=np.float64)


def main():
    g = {}

    # test/test_mttkrp.cpp:17-39 -- m=n=k=3, r=2; X, A, B, C from srand(2)
    srand(2)
    m = n = k = 3
    r = 2
    X = fill_int(m * n * k); A = fill_int(m * r); B = fill_int(n * r); C = fill_int(k * r)
    g.update(mt_X=X, mt_A=A, mt_B=B, mt_C=C)
    dims = (m, n, k)
    # mttkrp(X, C, B, .., 1), mttkrp(X, C, A, .., 2), mttkrp(X, B, A, .., 3)  (:60-62)
    g["mt_out1"] = exact_mttkrp(X, dims, [None, B, C], 0)
    g["mt_out2"] = exact_mttkrp(X, dims, [A, None, C], 1)
    g["mt_out3"] = exact_mttkrp(X, dims, [A, B, None], 2)

    # larger integer fixture, same generator: 20 x 12 x 10 (ragged vs tiles), R = 5
    srand(2)
    d2 = (20, 12, 10)
    r2 = 5
    X2 = fill_int(int(np.prod(d2)))
    F2 = [fill_int(d * r2) for d in d2]
    g.update(mt2_X=X2, mt2_dims=np.array(d2), mt2_R=np.array(r2))
    for i, f in enumerate(F2):
        g[f"mt2_U{i}"] = f
    for mode in range(3):
        facs = [None if j == mode else F2[j] for j in range(3)]
        g[f"mt2_out{mode}"] = exact_mttkrp(X2, d2, facs, mode)

    # 4th-order integer fixture 6 x 5 x 4 x 7, R = 3
    srand(3)
    d4 = (6, 5, 4, 7)
    r4 = 3
    X4 = fill_int(int(np.prod(d4)))
    F4 = [fill_int(d * r4) for d in d4]
    g.update(mt4_X=X4, mt4_dims=np.array(d4), mt4_R=np.array(r4))
    for i, f in enumerate(F4):
        g[f"mt4_U{i}"] = f
    for mode in range(4):
        facs = [None if j == mode else F4[j] for j in range(4)]
        g[f"mt4_out{mode}"] = exact_mttkrp(X4, d4, facs, mode)

    # test/test_gen.cpp:17-34 -- 2x2x2, r=2, core 2x2x2 from srand(2)
    srand(2)
    X = fill_int(8); A = fill_int(4); B = fill_int(4); C = fill_int(4); core = fill_int(8)
    g.update(gen_X=X, gen_A=A, gen_B=B, gen_C=C, gen_core=core)
    g["gen_cp"] = exact_gencp((2, 2, 2), [A, B, C])
    g["gen_tucker"] = exact_gentucker(core, (2, 2, 2), [A, B, C], (2, 2, 2))

    # decomposition/GPU/normal/tucker/de_tucker.cpp:11-22 (hand-written)
    tA = np.array([1, 3, 2, 0, -1, 2], np.float32)
    tB = np.array([2, 0, 4, 6, -1, 1, 1, 2], np.float32)
    tC = np.array([3, -1, 0, 2], np.float32)
    tG = np.array([-2, -1, 0, 3, 4, 1, 2, 3], np.float32)
    g.update(ht_A=tA, ht_B=tB, ht_C=tC, ht_G=tG)
    g["ht_rec"] = exact_gentucker(tG, (2, 2, 2), [tA, tB, tC], (3, 4, 2))

    # decomposition/GPU/normal/cp/de_cp.cpp:11-19 (hand-written): X = 0..11,
    # B, C given; the first A update of src/cp_als.cu:46-63, exact
    cX = np.arange(12, dtype=np.float32)
    cB = np.array([2, 1, 6, 3], np.float32)
    cC = np.array([0, 7, 1, 2], np.float32)
    g.update(hc_X=cX, hc_B=cB, hc_C=cC)
    g["hc_A1"] = exact_als_step(cX, (3, 2, 2), [np.zeros(6, np.float32), cB, cC], 0, 2)

    # test/test_t2m.cpp:9-13 -- 4x3x2, srand(2), rand()*0.1/RAND_MAX
    srand(2)
    T = fill_frac(24)
    Tl = cm(T, (4, 3, 2))
    g["t2m_T"] = T
    g["t2m_1"] = T.copy()
    g["t2m_2"] = np.concatenate([Tl[:, :, kk].T.reshape(-1, order="F") for kk in range(2)])
    g["t2m_3"] = T.reshape(12, 2, order="F").T.reshape(-1, order="F")

    # test/test_kr.cpp:21-31 -- unseeded (glibc default seed 1), a=b=3, r=2
    srand(1)
    kA = fill_frac(6); kB = fill_frac(6)
    g.update(kr_A=kA, kr_B=kB)
    out = np.empty(18, np.float32)
    for t in range(2):
        for y in range(3):
            for x in range(3):
                out[x + y * 3 + t * 9] = np.float32(kB[x + t * 3] * kA[y + t * 3])
    g["kr_out"] = out

    # test/test_hadmard.cpp:161-176 -- unseeded, a=b=2
    srand(1)
    hA = fill_frac(4); hB = fill_frac(4)
    g.update(hd_A=hA, hd_B=hB, hd_C=(hA * hB).astype(np.float32))

    # test/test_tensor_product.cpp:226-242 -- unseeded, A 2x2, B 3x3
    srand(1)
    pA = fill_frac(4); pB = fill_frac(9)
    g.update(tp_A=pA, tp_B=pB)
    g["tp_C"] = np.kron(cm(pA, (2, 2)), cm(pB, (3, 3))).astype(np.float32).reshape(-1, order="F")

    # test/test_ttm.cpp:73-96 -- srand(2), a=b=c=3, d=2, values rand()*0.1/RAND_MAX - 0.5
    srand(2)
    tX = fill_frac(27, -0.5); U1 = fill_frac(6, -0.5); U2 = fill_frac(6, -0.5); U3 = fill_frac(6, -0.5)
    g.update(ttm_X=tX, ttm_U1=U1, ttm_U2=U2, ttm_U3=U3)
    Xl = cm(tX, (3, 3, 3)).astype(np.float64)
    for flag, U in ((1, U1), (2, U2), (3, U3)):
        Ul = cm(U, (2, 3)).astype(np.float64)
        Y = np.moveaxis(np.tensordot(Ul, Xl, axes=([1], [flag - 1])), 0, flag - 1)
        g[f"ttm_out{flag}"] = Y.reshape(-1, order="F")

    np.savez_compressed(os.path.join(HERE, "golden.npz"), **g)
    print("wrote", os.path.join(HERE, "golden.npz"), len(g), "arrays")


if __name__ == "__main__":
    main()
