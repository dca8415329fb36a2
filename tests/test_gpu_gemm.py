"""BF16 tensor-core GEMM (cud_gemm_bf16): integer-valued operands are exact
in BF16 and their products and partial sums exact in FP32, so the tensor-core
result must equal an int64 matmul bit for bit -- across ragged tile edges,
the split-contraction path and every epilogue option.  Float operands are
checked against a float64 matmul of the same BF16 values."""
import pytest
import torch

pytestmark = pytest.mark.gpu


def ints(shape, lo=-4, hi=5, seed=0):
    g = torch.Generator(device="cpu").manual_seed(seed)
    return torch.randint(lo, hi, shape, generator=g)


@pytest.mark.parametrize("M,N,K", [(128, 128, 64), (200, 300, 1000), (1000, 64, 6144),
                                   (256, 512, 6144), (64, 1536, 512), (512, 512, 65536),
                                   (7, 9, 24),
                                   # skinny N, many rows: the persistent N <= 32 path
                                   (40000, 16, 128), (38000, 32, 512), (50001, 5, 1000), (45056, 32, 1024)])
def test_gemm_integer_exact(cd, M, N, K):
    A = ints((M, K), seed=M + K)
    B = ints((N, K), seed=N + 7 * K)
    want = (A @ B.T).to(torch.float32)
    C = torch.full((M, N), float("nan"), device="cuda")
    cd.gemm_bf16(A.to(torch.bfloat16).cuda(), B.to(torch.bfloat16).cuda(), out_f32=C)
    torch.cuda.synchronize()
    assert torch.equal(C.cpu(), want)


def test_gemm_epilogue_bias_relu_and_transposed_copies(cd):
    M, N, K = 300, 520, 2048
    A = ints((M, K), -2, 3, seed=1)
    B = ints((N, K), -2, 3, seed=2)
    bias = ints((N,), -8, 9, seed=3).float()
    ref = torch.relu(0.5 * (A @ B.T).float() + bias)
    Cf = torch.empty((N, M), device="cuda")                      # column-major FP32 (as C^T)
    H = torch.empty((M, N), device="cuda", dtype=torch.bfloat16)
    Ht = torch.empty((N, M), device="cuda", dtype=torch.bfloat16)
    cd.gemm_bf16(A.to(torch.bfloat16).cuda(), B.to(torch.bfloat16).cuda(), alpha=0.5,
                 bias=bias.cuda(), relu=True, out_f32=("T", Cf), out_bf16=H, out_bf16_2=("T", Ht))
    torch.cuda.synchronize()
    assert torch.equal(Cf.cpu().T, ref)
    assert torch.equal(H.cpu(), ref.to(torch.bfloat16))
    assert torch.equal(Ht.cpu().T, ref.to(torch.bfloat16))


def test_gemm_mask_and_accumulate(cd):
    M, N, K = 256, 200, 640
    A = ints((M, K), seed=5)
    B = ints((N, K), seed=6)
    mask = ints((M, N), -1, 2, seed=7).to(torch.bfloat16)
    prod = (A @ B.T).float()
    base = ints((M, N), -50, 50, seed=8).float()
    C = base.clone().cuda()
    cd.gemm_bf16(A.to(torch.bfloat16).cuda(), B.to(torch.bfloat16).cuda(), mask=mask.cuda(),
                 out_f32=C, accumulate=True)
    torch.cuda.synchronize()
    want = base + torch.where(mask.float() > 0, prod, torch.zeros_like(prod))
    assert torch.equal(C.cpu(), want)


def test_gemm_float_operands(cd):
    g = torch.Generator(device="cpu").manual_seed(11)
    A = torch.randn(384, 4096, generator=g).to(torch.bfloat16)
    B = torch.randn(640, 4096, generator=g).to(torch.bfloat16)
    want = A.double() @ B.double().T
    C = torch.empty((384, 640), device="cuda")
    cd.gemm_bf16(A.cuda(), B.cuda(), out_f32=C)
    torch.cuda.synchronize()
    err = (C.cpu().double() - want).norm() / want.norm()
    # FP32 accumulation of 4096 terms: 256 accumulator updates, each
    # truncating toward zero by up to an ulp of the running sum
    assert err < 2e-5


def test_gemm_rejects_bad_leading_dimension(cd):
    A = torch.zeros((16, 30), device="cuda", dtype=torch.bfloat16)   # row stride 30: not a multiple of 8
    B = torch.zeros((16, 30), device="cuda", dtype=torch.bfloat16)
    C = torch.empty((16, 16), device="cuda")
    with pytest.raises(cd.CudError):
        cd.gemm_bf16(A, B, out_f32=C)


def test_gemm_skinny_epilogue_strided_bf16(cd):
    """The persistent skinny path with the TTM epilogue: BF16 output with
    the rank index slowest (column-major C)."""
    M, N, K = 40960, 16, 256
    A = ints((M, K), -3, 4, seed=11)
    B = ints((N, K), -3, 4, seed=12)
    ref = (A @ B.T).float()
    Ct = torch.empty((N, M), device="cuda", dtype=torch.bfloat16)
    cd.gemm_bf16(A.to(torch.bfloat16).cuda(), B.to(torch.bfloat16).cuda(), out_bf16=("T", Ct))
    torch.cuda.synchronize()
    assert torch.equal(Ct.cpu().T.float(), ref.to(torch.bfloat16).float())
