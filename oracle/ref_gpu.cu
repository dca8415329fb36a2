// Baseline harness (test and benchmark infrastructure, not the product): the
// reference's own GPU MTTKRP, i.e. the cuBLAS calls its CP-ALS programs issue
// for one mode's right-hand side, so bench.py can time them on the same GPU
// as the library's kernels.  Each mode is the pair (or triple) of calls the
// reference makes, with the same operations, shapes, leading dimensions and
// batch strides, on a handle created once (as the reference creates one per
// cp_als call):
//   3rd order, src/cp_als.cu:
//     mode 0  Khatri-Rao C (.) B by rank-1 batched GEMM (:46), then
//             A^T(r x a) = KR^T X_(1)^T (:52)
//     mode 1  C (.) A (:66), then B^T = KR^T X2^T with X2 the mode-2
//             unfolding, made once before the sweeps by t2m (:28, :69)
//     mode 2  B (.) A (:85), then C^T = KR^T X (:88)
//   4th order, src/cp4_als.cu:
//     mode 0  D (.) C (:67), B (.) (D (.) C) (:68), A^T = KR^T X^T (:73)
//     mode 1  A (.) (D (.) C) (:91), B^T = KR^T X2^T (:96)
//     mode 2  B (.) A (:112), (B (.) A) (.) D (:113), C^T = KR^T X3^T (:117)
//     mode 3  (B (.) A) (.) C (:135), D^T = KR^T X (:138)
//   with X2 and X3 the permuted copies the program makes once by identity
//   GEMMs (:35-43).
// Outputs are the reference's transposed R x I_n right-hand sides.  The
// library under test never calls this file.
#include <cublas_v2.h>
#include <cuda_runtime.h>

namespace {

__global__ void k_identity(float *I, long n) {
    long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (t < n * n) I[t] = (t % n == t / n) ? 1.f : 0.f;
}

// One rank-1 batched GEMM forming a Khatri-Rao product the way the reference
// does: C_t (m x k) = U(:, t) * V(:, t)^T for each of the r columns t.
cublasStatus_t kr_batched(cublasHandle_t h, long m, long k, const float *U, long ldu, long su,
                          const float *V, long ldv, long sv, float *out, long ldo, long so, long r) {
    const float one = 1.f, zero = 0.f;
    return cublasSgemmStridedBatched(h, CUBLAS_OP_N, CUBLAS_OP_T, (int)m, (int)k, 1, &one, U, (int)ldu, su,
                                     V, (int)ldv, sv, &zero, out, (int)ldo, so, (int)r);
}

cublasStatus_t gemm(cublasHandle_t h, cublasOperation_t ta, cublasOperation_t tb, long m, long n, long k,
                    const float *A, long lda, const float *B, long ldb, float *C, long ldc) {
    const float one = 1.f, zero = 0.f;
    return cublasSgemm(h, ta, tb, (int)m, (int)n, (int)k, &one, A, (int)lda, B, (int)ldb, &zero, C, (int)ldc);
}

}  // namespace

extern "C" {

int rg_create(void **handle, void *stream) {
    cublasHandle_t h = nullptr;
    if (cublasCreate(&h) != CUBLAS_STATUS_SUCCESS) return 1;
    cublasSetStream(h, static_cast<cudaStream_t>(stream));
    *handle = h;
    return 0;
}

int rg_destroy(void *handle) { return cublasDestroy(static_cast<cublasHandle_t>(handle)) ? 1 : 0; }

// 3rd order.  kr holds (product of the two other dims) x r floats; out_t is
// r x dims[mode].
int rg_cp3_mttkrp(void *handle, int mode, const float *X, const float *X2, const float *A, const float *B,
                  const float *C, long a, long b, long c, long r, float *kr, float *out_t) {
    cublasHandle_t h = static_cast<cublasHandle_t>(handle);
    cublasStatus_t s;
    switch (mode) {
        case 0:
            s = kr_batched(h, b, c, B, b, b, C, c, c, kr, b, b * c, r);
            if (!s) s = gemm(h, CUBLAS_OP_T, CUBLAS_OP_T, r, a, b * c, kr, b * c, X, a, out_t, r);
            break;
        case 1:
            s = kr_batched(h, a, c, A, a, a, C, c, c, kr, a, a * c, r);
            if (!s) s = gemm(h, CUBLAS_OP_T, CUBLAS_OP_T, r, b, a * c, kr, a * c, X2, b, out_t, r);
            break;
        case 2:
            s = kr_batched(h, a, b, A, a, a, B, b, b, kr, a, a * b, r);
            if (!s) s = gemm(h, CUBLAS_OP_T, CUBLAS_OP_N, r, c, a * b, kr, a * b, X, a * b, out_t, r);
            break;
        default: return 2;
    }
    return s ? 1 : 0;
}

// 4th order: the permuted copies X2 (b x a x c x d) and X3 (for each d-slice
// the c x ab transpose) by identity GEMMs.  ident holds (ab)^2 floats.
int rg_cp4_prepare(void *handle, const float *X, float *X2, float *X3, float *ident, long a, long b, long c,
                   long d, void *stream) {
    cublasHandle_t h = static_cast<cublasHandle_t>(handle);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const float one = 1.f, zero = 0.f;
    k_identity<<<(unsigned)((a * a + 511) / 512), 512, 0, st>>>(ident, a);
    cublasStatus_t s = cublasSgemmStridedBatched(h, CUBLAS_OP_T, CUBLAS_OP_N, (int)b, (int)a, (int)a, &one, X,
                                                 (int)a, a * b, ident, (int)a, 0, &zero, X2, (int)b, a * b,
                                                 (int)(c * d));
    if (s) return 1;
    k_identity<<<(unsigned)((a * b * a * b + 511) / 512), 512, 0, st>>>(ident, a * b);
    s = cublasSgemmStridedBatched(h, CUBLAS_OP_T, CUBLAS_OP_N, (int)c, (int)(a * b), (int)(a * b), &one, X,
                                  (int)(a * b), a * b * c, ident, (int)(a * b), 0, &zero, X3, (int)c, a * b * c,
                                  (int)d);
    return s ? 1 : 0;
}

// 4th order, one mode.  kr1 holds the intermediate two-factor product
// (D (.) C for modes 0-1: c*d*r floats; B (.) A for modes 2-3: a*b*r) and is
// written by the mode that forms it (0 and 2) and read by the next (1, 3),
// as in the reference's sweep; kr holds the full Khatri-Rao matrix.
int rg_cp4_mttkrp(void *handle, int mode, const float *X, const float *X2, const float *X3, const float *A,
                  const float *B, const float *C, const float *D, long a, long b, long c, long d, long r,
                  float *kr1, float *kr, float *out_t) {
    cublasHandle_t h = static_cast<cublasHandle_t>(handle);
    cublasStatus_t s;
    switch (mode) {
        case 0:
            s = kr_batched(h, c, d, C, c, c, D, d, d, kr1, c, d * c, r);
            if (!s) s = kr_batched(h, b, c * d, B, b, b, kr1, c * d, c * d, kr, b, b * c * d, r);
            if (!s) s = gemm(h, CUBLAS_OP_T, CUBLAS_OP_T, r, a, b * c * d, kr, b * c * d, X, a, out_t, r);
            break;
        case 1:
            s = kr_batched(h, a, c * d, A, a, a, kr1, c * d, c * d, kr, a, a * c * d, r);
            if (!s) s = gemm(h, CUBLAS_OP_T, CUBLAS_OP_T, r, b, a * c * d, kr, a * c * d, X2, b, out_t, r);
            break;
        case 2:
            s = kr_batched(h, a, b, A, a, a, B, b, b, kr1, a, a * b, r);
            if (!s) s = kr_batched(h, b * a, d, kr1, a * b, a * b, D, d, d, kr, a * b, a * b * d, r);
            if (!s) s = gemm(h, CUBLAS_OP_T, CUBLAS_OP_T, r, c, a * b * d, kr, a * b * d, X3, c, out_t, r);
            break;
        case 3:
            s = kr_batched(h, b * a, c, kr1, a * b, a * b, C, c, c, kr, a * b, a * b * c, r);
            if (!s) s = gemm(h, CUBLAS_OP_T, CUBLAS_OP_N, r, d, a * b * c, kr, a * b * c, X, a * b * c, out_t, r);
            break;
        default: return 2;
    }
    return s ? 1 : 0;
}

}  // extern "C"
