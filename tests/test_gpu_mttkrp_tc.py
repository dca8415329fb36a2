"""The tcgen05 tensor-core MTTKRP: the shapes that take it really take it
(cud_mttkrp_path), and its results match the oracle across ragged tiles
(rows not a multiple of 128, contraction not a multiple of the 32-deep
stage, ranks not a multiple of 16) for every precision.

Tolerances as tests/test_gpu_mttkrp.py: bf16x3 at the FP32 bar (1e-5
relative Frobenius vs FP64), bf16 2e-2, fp16 2e-3; integer data exact.
"""
import numpy as np
import pytest
import torch

import oracle

pytestmark = pytest.mark.gpu

TOL = {"bf16x3": 1e-5, "default": 1e-5, "bf16": 2e-2, "fp16": 2e-3}

# (dims, R): every mode of these takes the tensor-core path
TC_SHAPES = [
    ((128, 64, 32), 16),      # exact tiles
    ((700, 36, 20), 64),      # 6 row tiles (last ragged), S not a multiple of 32
    ((20, 52, 44), 12),       # P = 20 < 32: a partly empty stage
    ((96, 96, 96, 96), 32),   # 4th order, rows 96 < 128
    ((256, 4, 516), 128),     # R = 128 (largest MMA N built), thin middle mode
    ((8, 12, 16, 20, 24), 5), # 5th order, R < 16 padded
]


def dev_t(a):
    return torch.from_numpy(np.ascontiguousarray(a, np.float32)).cuda()


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("dims,R", TC_SHAPES)
def test_shapes_take_tensor_core_path(cd, dims, R):
    for mode in range(len(dims)):
        for prec in ("bf16x3", "bf16", "fp16"):
            assert cd.mttkrp_path(dims, mode, R, cd.PRECISIONS[prec]) == "tensor-core", (mode, prec)
        assert cd.mttkrp_path(dims, mode, R, cd.PREC_FP32) == "cuda-core"


def test_fallback_shapes_use_cuda_cores(cd):
    # rows of mode 0 not a multiple of 4 (TMA stride rule), R above 128
    assert cd.mttkrp_path((37, 8, 8), 0, 8) == "cuda-core"
    assert cd.mttkrp_path((37, 8, 8), 1, 8) == "cuda-core"
    assert cd.mttkrp_path((64, 64, 64), 0, 130) == "cuda-core"


@pytest.mark.parametrize("prec", ["bf16x3", "bf16", "fp16"])
@pytest.mark.parametrize("dims,R", TC_SHAPES)
def test_tensor_core_vs_oracle(cd, prec, dims, R):
    n = int(np.prod(dims))
    if n > 50_000_000:
        pytest.skip("oracle too slow")
    rng = np.random.default_rng(n % 9973 + R)
    X = rng.random(n).astype(np.float32)
    facs = [rng.random(d * R).astype(np.float32) for d in dims]
    dX = dev_t(X)
    dU = [dev_t(f) for f in facs]
    for mode in range(len(dims)):
        out = torch.empty(dims[mode] * R, device="cuda")
        cd.mttkrp(dX, dims, dU, mode, R, out, cd.PRECISIONS[prec])
        torch.cuda.synchronize()
        got = out.cpu().numpy().astype(np.float64)
        want = oracle.mttkrp(X, dims, facs, mode, R)
        assert rel(got, want) <= TOL[prec], (mode, rel(got, want))


@pytest.mark.parametrize("prec", ["bf16x3", "bf16", "fp16"])
def test_tensor_core_integer_exact(cd, prec):
    """Small integers are exact in every operand format: bit-exact result."""
    rng = np.random.default_rng(5)
    dims, R = (132, 40, 36), 20
    X = rng.integers(-4, 5, int(np.prod(dims))).astype(np.float32)
    facs = [rng.integers(-4, 5, d * R).astype(np.float32) for d in dims]
    for mode in range(3):
        assert cd.mttkrp_path(dims, mode, R, cd.PRECISIONS[prec]) == "tensor-core"
        out = torch.empty(dims[mode] * R, device="cuda")
        cd.mttkrp(dev_t(X), dims, [dev_t(f) for f in facs], mode, R, out, cd.PRECISIONS[prec])
        torch.cuda.synchronize()
        np.testing.assert_array_equal(out.cpu().numpy().astype(np.float64),
                                      oracle.mttkrp(X, dims, facs, mode, R))


def test_tensor_core_signed_cancellation(cd):
    rng = np.random.default_rng(8)
    dims, R = (128, 96, 80), 32
    X = rng.standard_normal(int(np.prod(dims))).astype(np.float32)
    facs = [rng.standard_normal(d * R).astype(np.float32) for d in dims]
    for mode in range(3):
        out = torch.empty(dims[mode] * R, device="cuda")
        cd.mttkrp(dev_t(X), dims, [dev_t(f) for f in facs], mode, R, out, cd.PREC_BF16X3)
        torch.cuda.synchronize()
        got = out.cpu().numpy().astype(np.float64)
        assert rel(got, oracle.mttkrp(X, dims, facs, mode, R)) <= 1e-5


def test_misaligned_tensor_falls_back(cd):
    """A tensor that does not start on a 16-byte boundary cannot be a TMA
    source: the call must still be right (CUDA-core path)."""
    rng = np.random.default_rng(9)
    dims, R = (64, 32, 16), 8
    n = int(np.prod(dims))
    X = rng.random(n + 1).astype(np.float32)
    facs = [rng.random(d * R).astype(np.float32) for d in dims]
    dX = dev_t(X)[1:]
    out = torch.empty(dims[0] * R, device="cuda")
    cd.mttkrp(dX, dims, [dev_t(f) for f in facs], 0, R, out, cd.PREC_BF16X3)
    torch.cuda.synchronize()
    assert rel(out.cpu().numpy().astype(np.float64), oracle.mttkrp(X[1:], dims, facs, 0, R)) <= 1e-5
