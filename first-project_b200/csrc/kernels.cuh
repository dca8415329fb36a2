// Internal interfaces shared between the library's translation units.
#pragma once

#include "common.cuh"

namespace cud {

// General strided GEMM on CUDA cores (FP32 FMA):
//   C[b](m, n) = alpha * sum_{kin, kout} A(m, kin, kout) * B(kin, kout, n) + beta * C
// with element strides for every index, so unfoldings, mode products and
// unfolding Grams of column-major tensors are expressed without copies.
// `kout` is a second contraction index (it lets a contraction run over two
// non-adjacent tensor modes).  With out_f64 set, C is double and the partial
// sums over `splits` chunks of the contraction are reduced in FP64.
template <typename T>
struct GemmDescT {
    long M = 0, N = 0, Kin = 1, Kout = 1, batch = 1;
    const T *A = nullptr;
    long a_m = 0, a_kin = 0, a_kout = 0, a_b = 0;
    const T *B = nullptr;
    long b_kin = 0, b_kout = 0, b_n = 0, b_b = 0;
    void *C = nullptr;             // T, or double when out_f64
    long c_m = 0, c_n = 0, c_b = 0;
    T alpha = 1, beta = 0;
    bool out_f64 = false;
    int splits = 0;  // 0 = choose
};
using GemmDesc = GemmDescT<float>;
using GemmDesc64 = GemmDescT<double>;
int gemm_simt(const GemmDesc &d, cudaStream_t s);
int gemm_simt_f64(const GemmDesc64 &d, cudaStream_t s);  // FP64 operands and output

// Residual/norm helper (elementwise.cu).  Synchronises the stream.
int residual_norms(const float *X, float *X1, long n, int subtract, double *out, cudaStream_t s);

// Tensor views used by the contraction kernels: a column-major tensor seen as
// (P, Q, S) around mode n -- P = prod of the dims before n, Q = dims[n],
// S = prod of the dims after n.
struct ModeView {
    long P = 1, Q = 1, S = 1;
};
inline ModeView mode_view(int order, const long *dims, int mode) {
    ModeView v;
    for (int m = 0; m < mode; m++) v.P *= dims[m];
    v.Q = dims[mode];
    for (int m = mode + 1; m < order; m++) v.S *= dims[m];
    return v;
}

constexpr int kMaxOrder = 8;

// BF16 tensor-core GEMM with fused epilogue (gemm_tc.cu); ws holds
// gemm_tc_ws_bytes (split-contraction partials + error flag).
using GemmEpi = cud_gemm_epilogue;
size_t gemm_tc_ws_bytes(long M, long N, long K);
int gemm_tc_bf16(const __nv_bfloat16 *A, long lda, const __nv_bfloat16 *B, long ldb, long M, long N, long K,
                 const GemmEpi &e, void *ws, cudaStream_t s);

// Top-r eigenvectors of a symmetric PSD FP64 n x n matrix by subspace
// iteration (subspace.cu): U (n x r, FP32) in ascending eigenvalue order;
// CUD_ERR_NOT_CONVERGED if it did not settle within max_iters.  With U0
// (n x r, FP32, may alias U) the iteration starts from U0's columns instead
// of a random block, and falls back to the random start if they are
// numerically rank-deficient.
size_t subspace_ws_doubles(long n, long r);
int top_eigvecs_subspace(const double *G, long n, long r, float *U, double *ws, size_t ws_doubles, int max_iters,
                         cudaStream_t s, const float *U0 = nullptr);

// ||X - [[U]]||^2 and ||X||^2 into out2[0..1] (device, FP64), one pass
// over X (residual.cu); ws holds cp_residual_ws_bytes.
size_t cp_residual_ws_bytes(int order, const long *dims);
int cp_residual(const float *X, int order, const long *dims, const float *const *U, long R, double *out2,
                void *ws, cudaStream_t s);

// Factor set for on-the-fly Khatri-Rao rows: up to kMaxOrder-1 factor
// matrices (column-major rows x R) listed fastest-first.
struct KrFactors {
    int n = 0;
    const float *U[kMaxOrder];
    long rows[kMaxOrder];
};

// MTTKRP kernels take an explicit device workspace (split-contraction
// partials), so a captured CUDA graph can own its memory.
//
// CUDA-core path (mttkrp_simt.cu): FP32 FMA; with round = 1 (FP16) or 2
// (BF16) the operands -- X and each formed KR row -- are rounded first.
size_t mttkrp_simt_ws_bytes(int order, const long *dims, int mode, long R, int round);
int mttkrp_simt_rounded(const float *X, int order, const long *dims, const float *const *U,
                        int mode, long R, float *out, int round, void *ws, cudaStream_t s);
// The CUDA-core MTTKRP on FP64 data (FP64 CP-ALS); ws as sized below.
size_t mttkrp_simt_f64_ws_bytes(int order, const long *dims, int mode, long R);
int mttkrp_simt_f64(const double *X, int order, const long *dims, const double *const *U, int mode, long R,
                    double *out, void *ws, cudaStream_t s);
// Tensor-core path (mttkrp_tc.cu): CUD_OK and the workspace size when it
// applies to this shape/precision, CUD_ERR_UNSUPPORTED otherwise.
int mttkrp_tc_query(int order, const long *dims, int mode, long R, int precision, size_t *ws_bytes);
// Where an MTTKRP left its result: M(q, r) = the sum over z < splits of
// part[z zs + q qs + r rs], taken in FP64 in z order, or NaN everywhere when
// *error is set (a CTA whose bounded wait expired).
struct MttkrpParts {
    const float *part;
    long zs, qs, rs;
    int splits;
    const int *error;  // null: no flag
};
// With `parts` set, the split reduce is left to the caller: the partials'
// layout is returned there and `out` is not written.
int mttkrp_tc(const float *X, int order, const long *dims, const float *const *U, int mode,
              long R, float *out, int precision, void *ws, cudaStream_t s, MttkrpParts *parts = nullptr);
// Dispatcher (mttkrp.cu): tensor cores when they apply, else CUDA cores.
size_t mttkrp_ws_bytes(int order, const long *dims, int mode, long R, int precision);
int mttkrp_run(const float *X, int order, const long *dims, const float *const *U, int mode,
               long R, float *out, int precision, void *ws, cudaStream_t s);
// As mttkrp_run, for a consumer that sums the split partials itself: a
// tensor-core MTTKRP returns its partials in *parts (out not written); any
// other path writes out and describes it as one column-major split.
int mttkrp_run_parts(const float *X, int order, const long *dims, const float *const *U, int mode,
                     long R, float *out, int precision, void *ws, cudaStream_t s, MttkrpParts *parts);

// Exact CP residual pieces (residual.cu, residual_tc.cu): per-CTA partial
// pairs summed in a fixed order into out[0..1]; the tensor-core residual
// (order >= 3, R <= 64; the grid it launches, for sizing the partials).
int sum_pairs(const double *part, long n, double *out, cudaStream_t s);
bool residual_tc_plan(int order, const long *dims, long R, int *grid);
// need_x2 = false: out2[1] (||X||^2) is left 0 -- a caller that already has
// the norm saves the FP64 sum of squares (about a tenth of the kernel).
int residual_tc(const float *X, int order, const long *dims, const float *const *U, long R, double *part,
                double *out2, cudaStream_t s, bool need_x2 = true);
// ||X - [[U]]||^2 (and ||X||^2 when need_x2) to the host, synchronising s.
int cp_residual_host(const float *X, int order, const long *dims, const float *const *U, long R, bool need_x2,
                     double *res_norm2, double *x_norm2, cudaStream_t s);

// Mode product Y = X x_mode W (contract.cu); W is J x dims[mode], or its
// transpose when w_trans is set.
int mode_product(const float *X, int order, const long *dims, int mode, const float *W, long J,
                 float *Y, cudaStream_t s, bool w_trans = false);
// G (dims[mode]^2, FP64) = X_(mode) X_(mode)^T
int unfold_gram(const float *X, int order, const long *dims, int mode, double *G, cudaStream_t s);
// The same two on FP64 tensors (the FP64 Tucker path).
int mode_product_f64(const double *X, int order, const long *dims, int mode, const double *W, long J, double *Y,
                     cudaStream_t s, bool w_trans = false);
int unfold_gram_f64(const double *X, int order, const long *dims, int mode, double *G, cudaStream_t s);

// Symmetric eigensolver (eig.cu): A (n x n, FP64, destroyed) -> ascending W, V.
int syev_jacobi(double *A, long n, double *W, double *V, int max_sweeps, cudaStream_t s);

}  // namespace cud
