"""MTTKRP on the GPU against the oracle.

Tolerances (relative Frobenius norm vs the FP64 oracle):
  fp32 / bf16x3 / default : 1e-5   (the FP32 bar of the reference GPU path)
  bf16                    : 2e-2   (8-bit operand mantissas)
  fp16                    : 2e-3   (11-bit operand mantissas)
Integer fixtures (the reference drivers' srand(2) data) are exact in every
precision and are compared bit for bit.
"""
import numpy as np
import pytest
import torch

import oracle

pytestmark = pytest.mark.gpu

TOL = {"fp32": 1e-5, "bf16x3": 1e-5, "default": 1e-5, "bf16": 2e-2, "fp16": 2e-3}


def dev_t(a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()


def run(cd, X, dims, facs, mode, R, prec):
    out = torch.empty(dims[mode] * R, device="cuda")
    cd.mttkrp(dev_t(X), dims, [dev_t(f) for f in facs], mode, R, out, cd.PRECISIONS[prec])
    torch.cuda.synchronize()
    return out.cpu().numpy().astype(np.float64)


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("prec", ["fp32", "bf16", "fp16", "bf16x3", "default"])
@pytest.mark.parametrize("prefix,order", [("mt2", 3), ("mt4", 4)])
def test_integer_fixtures_exact(cd, golden, prec, prefix, order):
    X = golden[f"{prefix}_X"]
    dims = tuple(int(d) for d in golden[f"{prefix}_dims"])
    R = int(golden[f"{prefix}_R"])
    facs = [golden[f"{prefix}_U{i}"] for i in range(order)]
    for mode in range(order):
        np.testing.assert_array_equal(run(cd, X, dims, facs, mode, R, prec), golden[f"{prefix}_out{mode}"])


def test_legacy_mttkrp_reference_fixture(cd, golden):
    """test/test_mttkrp.cpp:60-62 with the public FP16 mttkrp()."""
    X, A, B, C = (dev_t(golden[k]) for k in ("mt_X", "mt_A", "mt_B", "mt_C"))
    out = torch.empty(6, device="cuda")
    for flag, (left, right) in ((1, (C, B)), (2, (C, A)), (3, (B, A))):
        cd.mttkrp_legacy(X, left, right, out, flag, 3, 3, 3, 2)
        torch.cuda.synchronize()
        np.testing.assert_array_equal(out.cpu().numpy(), golden[f"mt_out{flag}"])


@pytest.mark.parametrize("prec", ["fp32", "bf16x3", "bf16", "fp16"])
@pytest.mark.parametrize("dims,R", [((64, 48, 40), 16), ((37, 130, 21), 7), ((130, 9, 66), 33),
                                    ((20, 18, 16, 14), 12), ((5, 6, 7, 8, 9), 3), ((700, 3, 2), 64)])
def test_random_vs_oracle(cd, prec, dims, R):
    rng = np.random.default_rng(int(np.prod(dims)) + R)
    X = rng.random(int(np.prod(dims))).astype(np.float32)
    facs = [rng.random(d * R).astype(np.float32) for d in dims]
    for mode in range(len(dims)):
        got = run(cd, X, dims, facs, mode, R, prec)
        want = oracle.mttkrp(X, dims, facs, mode, R)
        assert rel(got, want) <= TOL[prec], (mode, rel(got, want))


@pytest.mark.parametrize("prec", ["fp32", "bf16x3"])
def test_signed_data_vs_oracle(cd, prec):
    """Zero-mean data (cancellation) at the FP32 bar."""
    rng = np.random.default_rng(11)
    dims, R = (96, 80, 72), 32
    X = rng.standard_normal(int(np.prod(dims))).astype(np.float32)
    facs = [rng.standard_normal(d * R).astype(np.float32) for d in dims]
    for mode in range(3):
        got = run(cd, X, dims, facs, mode, R, prec)
        want = oracle.mttkrp(X, dims, facs, mode, R)
        assert rel(got, want) <= TOL[prec], (mode, rel(got, want))


def test_legacy_fp16_semantics_random(cd):
    """The public mttkrp() rounds X and each KR row to FP16 (src/mttkrp.cu:15-25)."""
    rng = np.random.default_rng(3)
    m, n, k, r = 40, 33, 27, 6
    X = rng.random(m * n * k).astype(np.float32)
    A, B, C = (rng.random(d * r).astype(np.float32) for d in (m, n, k))
    out = torch.empty(max(m, n, k) * r, device="cuda")
    for flag, (left, right) in ((1, (C, B)), (2, (C, A)), (3, (B, A))):
        cd.mttkrp_legacy(dev_t(X), dev_t(left), dev_t(right), out, flag, m, n, k, r)
        torch.cuda.synchronize()
        q = {1: m, 2: n, 3: k}[flag]
        got = out[: q * r].cpu().numpy().astype(np.float64)
        want = oracle.mttkrp_legacy(X, left, right, flag, m, n, k, r, round_fp16=True)
        assert rel(got, want) <= 1e-6


@pytest.mark.parametrize("dims,R", [((128, 96, 64), 16), ((64, 256, 96), 32)])
def test_fp16_rounds_whole_khatri_rao_entry(cd, dims, R):
    """FP16 at shapes whose fastest generating factor has a multiple of 32
    rows (>= 64): the tensor-core path must still round fp16(U0[x] * c[y]),
    the whole Khatri-Rao entry, as src/mttkrp.cu:21-25 does."""
    rng = np.random.default_rng(sum(dims) + R)
    X = rng.random(int(np.prod(dims))).astype(np.float32)
    facs = [rng.random(d * R).astype(np.float32) for d in dims]
    # mttkrp() flag f: (left, right) = the two other factors, slower first
    m, n, k = dims
    A, B, C = facs
    out = torch.empty(max(dims) * R, device="cuda")
    for flag, (left, right) in ((1, (C, B)), (2, (C, A)), (3, (B, A))):
        cd.mttkrp_legacy(dev_t(X), dev_t(left), dev_t(right), out, flag, m, n, k, R)
        torch.cuda.synchronize()
        q = dims[flag - 1]
        got = out[: q * R].cpu().numpy().astype(np.float64)
        want = oracle.mttkrp_legacy(X, left, right, flag, m, n, k, R, round_fp16=True)
        # non-negative data: at most 32 truncating K16 MMAs per segment (2
        # ulps each) plus 9 round-to-nearest flushes/roundings
        assert rel(got, want) <= 32 * 2.0 ** -22 + 9 * 2.0 ** -24, (flag, rel(got, want))


def test_bad_mode_rejected(cd):
    X = torch.zeros(8, device="cuda")
    out = torch.zeros(8, device="cuda")
    with pytest.raises(cd.CudError):
        cd.mttkrp(X, (2, 2, 2), [X, X, X], 3, 2, out)
