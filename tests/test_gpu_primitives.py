"""Bandwidth primitives on the GPU through the C ABI: bit-exact against the
golden vectors and the oracle (src/hadmard.cu, src/kr.cu,
src/tensor2matrix.cu, src/tensorproduct.cu, src/float2half.cu,
src/tminust.cu, src/rse.cu)."""
import numpy as np
import pytest
import torch

import oracle

pytestmark = pytest.mark.gpu


def dev_t(a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def test_golden_elementwise(cd, golden):
    A, B = dev_t(golden["hd_A"]), dev_t(golden["hd_B"])
    C = torch.empty_like(A)
    cd.hadmard(A, B, C, 2, 2)
    np.testing.assert_array_equal(host(C), golden["hd_C"])
    kA, kB = dev_t(golden["kr_A"]), dev_t(golden["kr_B"])
    out = torch.empty(18, device="cuda")
    cd.kr(kA, kB, out, 3, 3, 2)
    np.testing.assert_array_equal(host(out), golden["kr_out"])
    pA, pB = dev_t(golden["tp_A"]), dev_t(golden["tp_B"])
    pC = torch.empty(36, device="cuda")
    cd.tensor_product(pA, pB, pC, 2, 2, 3, 3)
    np.testing.assert_array_equal(host(pC), golden["tp_C"])


@pytest.mark.parametrize("flag", [1, 2, 3])
def test_golden_t2m(cd, golden, flag):
    T = dev_t(golden["t2m_T"])
    T2 = torch.empty_like(T)
    cd.t2m(T, T2, flag, 4, 3, 2)
    np.testing.assert_array_equal(host(T2), golden[f"t2m_{flag}"])


@pytest.mark.parametrize("shape", [(33, 17, 9), (128, 64, 40), (1, 1, 1), (5, 1, 70)])
@pytest.mark.parametrize("flag", [1, 2, 3])
def test_t2m_random_bit_exact(cd, shape, flag):
    rng = np.random.default_rng(sum(shape) + flag)
    m, n, k = shape
    T = rng.standard_normal(m * n * k).astype(np.float32)
    dT = dev_t(T)
    out = torch.empty_like(dT)
    cd.t2m(dT, out, flag, m, n, k)
    np.testing.assert_array_equal(host(out), oracle.t2m(T, flag, m, n, k))


@pytest.mark.parametrize("n", [1, 7, 4096, 1000003])
def test_hadmard_family_bit_exact(cd, n):
    rng = np.random.default_rng(n)
    A, B, K = (rng.standard_normal(n).astype(np.float32) for _ in range(3))
    dA, dB, dK = dev_t(A), dev_t(B), dev_t(K)
    out = torch.empty_like(dA)
    cd.hadmard(dA, dB, out, n, 1)
    np.testing.assert_array_equal(host(out), oracle.hadmard(A, B))
    cd.hadmard3(dA, dB, dK, out, 1, n)
    np.testing.assert_array_equal(host(out), oracle.hadmard3(A, B, K))
    cd.elepro3(dA, dB, dK, out, n)
    np.testing.assert_array_equal(host(out), oracle.hadmard3(A, B, K))
    N = dB.clone()
    cd.tminust(dA, N, n)
    np.testing.assert_array_equal(host(N), oracle.tminust(A, B))
    # unaligned (offset by one element) pointers take the scalar path
    if n > 8:
        out2 = torch.empty(n, device="cuda")
        cd.hadmard(dA[1:], dB[1:], out2[1:], n - 1, 1)
        np.testing.assert_array_equal(host(out2)[1:], oracle.hadmard(A[1:], B[1:]))


@pytest.mark.parametrize("a,b,r", [(3, 3, 2), (129, 67, 5), (512, 512, 4), (1, 300, 3)])
def test_kr_bit_exact(cd, a, b, r):
    rng = np.random.default_rng(a * b + r)
    A = rng.standard_normal(a * r).astype(np.float32)
    B = rng.standard_normal(b * r).astype(np.float32)
    out = torch.empty(a * b * r, device="cuda")
    cd.kr(dev_t(A), dev_t(B), out, a, b, r)
    np.testing.assert_array_equal(host(out), oracle.kr(A, B, a, b, r))


@pytest.mark.parametrize("a,b,c,d", [(2, 2, 3, 3), (17, 5, 9, 11), (1, 1, 1, 1)])
def test_tensor_product_bit_exact(cd, a, b, c, d):
    rng = np.random.default_rng(a + b + c + d)
    A = rng.standard_normal(a * b).astype(np.float32)
    B = rng.standard_normal(c * d).astype(np.float32)
    out = torch.empty(a * b * c * d, device="cuda")
    cd.tensor_product(dev_t(A), dev_t(B), out, a, b, c, d)
    np.testing.assert_array_equal(host(out), oracle.tensor_product(A, B, a, b, c, d))


def test_f2h_f2bf_bits(cd):
    rng = np.random.default_rng(5)
    A = np.concatenate([rng.standard_normal(10000) * 10 ** rng.uniform(-8, 5, 10000),
                        [0.0, -0.0, 65504.0, 65520.0, 1e-8, 6e-8, np.inf, -np.inf]]).astype(np.float32)
    dA = dev_t(A)
    h = torch.empty(A.size, dtype=torch.float16, device="cuda")
    cd.f2h(dA, h, A.size)
    np.testing.assert_array_equal(host(h).view(np.uint16), oracle.f2h_bits(A))
    bf = torch.empty(A.size, dtype=torch.bfloat16, device="cuda")
    cd.f2bf(dA, bf, A.size)
    np.testing.assert_array_equal(host(bf.float()), oracle.round_bf16(A))


def test_identity(cd):
    out = torch.empty(49, device="cuda")
    cd.initMat(out, 7)
    np.testing.assert_array_equal(host(out), oracle.identity(7))


@pytest.mark.parametrize("n", [27, 100000, 5000011])
def test_rse(cd, n):
    rng = np.random.default_rng(n)
    X = rng.standard_normal(n).astype(np.float32)
    X1 = (X + 1e-3 * rng.standard_normal(n)).astype(np.float32)
    dX, dX1 = dev_t(X), dev_t(X1)
    err = cd.rse(dX, dX1, n)
    diff, want = oracle.rse(X, X1)
    np.testing.assert_array_equal(host(dX1), diff)
    assert abs(err - want) <= 1e-6 * want
    assert abs(cd.norm2(dX) - float(np.dot(X.astype(np.float64), X))) <= 1e-12 * float(np.dot(X.astype(np.float64), X))
