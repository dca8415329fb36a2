/*
 * cudecompose_c.h -- C ABI of the B200-native dense CP/Tucker library.
 *
 * Every entry point takes plain pointers and sizes: device pointers for
 * tensors and matrices (column-major, mode 1 fastest; factor matrices are
 * I_n x R column-major), `long` extents, and an optional CUDA stream passed as
 * `void *` (NULL = the legacy default stream).  Each returns a cud_status and
 * also records it as the calling thread's last status (cud_get_last_error),
 * the side channel the void-returning drop-in functions of cudecompose.h use.
 *
 * The comment above each declaration names the reference interface it
 * replaces (891922758/first-project, file:line).  Entry points marked
 * "extension" have no reference counterpart.
 */
#ifndef CUDECOMPOSE_C_H_
#define CUDECOMPOSE_C_H_

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status ----------------------------------------------------------- */

typedef enum cud_status {
    CUD_OK = 0,
    CUD_ERR_INVALID_ARGUMENT = 1, /* bad flag/mode, null pointer, bad extent  */
    CUD_ERR_CUDA = 2,             /* a CUDA runtime call failed                */
    CUD_ERR_NO_MEMORY = 3,        /* device workspace allocation failed        */
    CUD_ERR_NOT_CONVERGED = 4,    /* an iterative solver hit its sweep limit   */
    CUD_ERR_UNSUPPORTED = 5,      /* shape/precision combination not built     */
    CUD_ERR_SINGULAR = 6,         /* normal equations fell back to pinv        */
    CUD_ERR_DEVICE_TIMEOUT = 7    /* a bounded device-side wait gave up        */
} cud_status;

/* MTTKRP / TTM / Gram arithmetic. */
typedef enum cud_precision {
    CUD_PREC_FP32 = 0,   /* FP32 FMA on CUDA cores (plain FP32)                 */
    CUD_PREC_BF16 = 1,   /* BF16 operands, FP32 accumulate, tensor cores        */
    CUD_PREC_FP16 = 2,   /* FP16 operands, FP32 accumulate, tensor cores        */
    CUD_PREC_BF16X3 = 3, /* hi/lo BF16 split, 3 products, FP32-level accuracy   */
    CUD_PREC_DEFAULT = 4 /* BF16X3 where the tensor-core path applies, else FP32 */
} cud_precision;

/* Extension: the calling thread's last status (cudecomposeGetLastError). */
int cud_get_last_error(void);
/* Extension: a static message for a status code. */
const char *cud_status_string(int status);
/* Extension: the detail text (CUDA error name, failing call) of the thread's
 * last non-OK status, or "" */
const char *cud_last_error_detail(void);

/* ---- element-wise and permutation primitives -------------------------- */

/* inc/cudecompose.h:23, src/hadmard.cu:10-15: C = A .* B over a*b elements. */
int cud_hadmard(const float *A, const float *B, float *C, long a, long b, void *stream);

/* inc/cudecompose.h:50, src/hadmard.cu:25-30: D = A .* B .* C. */
int cud_hadmard3(const float *A, const float *B, const float *C, float *D, long a, long b,
                 void *stream);

/* inc/cudecompose.h:55, src/kernel.cu:3-9 elepro3: D = A .* B .* C over n. */
int cud_elepro3(const float *A, const float *B, const float *C, float *D, long n, void *stream);

/* inc/cudecompose.h:24, src/kr.cu:3-11: Khatri-Rao, out (a*b) x r with
 * out[x + y*b + t*a*b] = B[x,t]*A[y,t]. */
int cud_kr(const float *A, const float *B, float *AkrB, long a, long b, long r, void *stream);

/* inc/cudecompose.h:25, src/tensorproduct.cu:4-14: Kronecker product,
 * C (a*c) x (b*d) = A (a x b) (x) B (c x d). */
int cud_tensor_product(const float *A, const float *B, float *C, long a, long b, long c,
                       long d, void *stream);

/* inc/cudecompose.h:28, src/float2half.cu:14-18: FP32 -> FP16 (RN). */
int cud_f2h(const float *A, void *B_half, long n, void *stream);

/* Extension: FP32 -> BF16 (RN). */
int cud_f2bf(const float *A, void *B_bf16, long n, void *stream);

/* inc/cudecompose.h:35, src/tensor2matrix.cu:38-52: mode-n unfolding of an
 * m x n x k tensor (flag 1 copy, 2: n x (m*k), 3: k x (m*n)). */
int cud_t2m(const float *T1, float *T2, long flag, long m, long n, long k, void *stream);

/* inc/cudecompose.h:37, src/tminust.cu:10-15: N = M - N over m elements. */
int cud_tminust(const float *M, float *N, long m, void *stream);

/* inc/cudecompose.h:47, src/tminust.cu:31-36 initMat: m x m identity. */
int cud_init_identity(float *A, long m, void *stream);

/* inc/cudecompose.h:38, src/rse.cu:4-15: X1 <- X - X1 and
 * *err = ||X - X1|| / ||X|| (norms accumulated in FP64). err is a host pointer. */
int cud_rse(const float *X, float *X1, long n, float *err, void *stream);

/* Extension: sum of squares of x (FP64 accumulation), written to *out (host). */
int cud_norm2(const float *x, long n, double *out, void *stream);

/* ---- generators / reconstructions ------------------------------------- */

/* inc/cudecompose.h:39,52, src/rse.cu:17-30,53-73 gencp/gencp4, any order:
 * rec = sum_r U[0][:,r] o U[1][:,r] o ... ; U is a host array of `order`
 * device pointers, U[m] is dims[m] x R. */
int cud_gencp(float *rec, int order, const long *dims, const float *const *U, long R,
              void *stream);

/* inc/cudecompose.h:40,53, src/rse.cu:32-51,75-96 gentucker/gentucker4, any
 * order: rec = core x_1 U[0] x_2 U[1] ...; core is ranks[0] x ranks[1] x ...,
 * U[m] is dims[m] x ranks[m]. */
int cud_gentucker(float *rec, int order, const long *dims, const float *core,
                  const long *ranks, const float *const *U, void *stream);

/* ---- contractions ------------------------------------------------------ */

/* inc/cudecompose.h:29, src/ttm.cu:4-47: mode-`flag` product of the
 * a x b x c tensor X with U (d x I_flag, row = new index); XU is d x b x c,
 * a x d x c or a x b x d. */
int cud_ttm(const float *X, const float *U, float *XU, long flag, long a, long b, long c,
            long d, int precision, void *stream);

/* Extension: general-order mode product Y = X x_mode W, W is J x dims[mode]
 * (row = new index); Y has dims[mode] replaced by J. */
int cud_mode_product(const float *X, int order, const long *dims, int mode, const float *W,
                     long J, float *Y, int precision, void *stream);

/* inc/cudecompose.h:30, src/mttkrp.cu:3-80: MTTKRP of the m x n x k tensor
 * with the reference's operand convention (flag 1: left k x r, right n x r,
 * XU m x r; flag 2: left k x r, right m x r, XU n x r; flag 3: left n x r,
 * right m x r, XU k x r). */
int cud_mttkrp_legacy(const float *X, const float *left, const float *right, float *XU,
                      long flag, long m, long n, long k, long r, int precision, void *stream);

/* The FP32 MTTKRPs inside src/cp_als.cu:46-52,66-69,85-88 and
 * src/cp4_als.cu:67-73,91-96,112-117,135-138, any order, native layout:
 * out (dims[mode] x R) = X_(mode) * (KR of the other factors), with no
 * unfolding or Khatri-Rao matrix materialised. */
int cud_mttkrp(const float *X, int order, const long *dims, const float *const *U, int mode,
               long R, float *out, int precision, void *stream);

/* No counterpart in the reference.  cud_mttkrp for callers that cannot
 * allocate device memory (code inside a custom allocator's own hooks, where
 * cudaMalloc would re-enter the allocator, or under a framework that owns
 * all device memory): same arguments, kernels and results, but its
 * workspace is a fixed 32 MiB __device__ array inside the library, so it
 * calls no cudaMalloc/cudaFree.  It launches kernels on `stream`, so it must
 * not run inside a stream callback (CUDA forbids API calls there).  A call
 * needing more workspace is rejected (CUD_ERR_INVALID_ARGUMENT, message in
 * cud_last_error_detail).  All calls on a device share the array: calls that
 * overlap on the GPU race and must be serialised by the caller.  The first
 * call on a device loads the array's module (under lazy module loading, the
 * CUDA 12.2+ default, that commits the 32 MiB then) and resolves its
 * address: make it at start-up, with the memory free, and before any stream
 * capture. */
int cud_mttkrp_noalloc(const float *X, int order, const long *dims, const float *const *U,
                       int mode, long R, float *out, int precision, void *stream);

/* Extension (measurement; no counterpart in the reference): kernel timing
 * of the MTTKRP entry points.  With cud_prof_enable(1), every cud_mttkrp /
 * cud_mttkrp_legacy call records a pair of CUDA events on its stream around
 * its main kernel (the MTTKRP itself, not the B pack or the split reduce),
 * except while the stream is being captured into a graph; up to 256 pairs
 * are kept.  cud_prof_kernel_times synchronises on them, writes up to max_n
 * durations (ms) into ms, the number recorded into count, and clears them.
 * cud_prof_enable(0) turns it off. */
int cud_prof_enable(int on);
int cud_prof_kernel_times(float *ms, int max_n, int *count);

/* Extension: the kernel cud_mttkrp runs for these arguments (given a
 * 16-byte-aligned X): 1 = tcgen05 tensor cores, 0 = CUDA cores. */
int cud_mttkrp_path(int order, const long *dims, int mode, long R, int precision);

/* Extension: the unfolding Gram G = X_(mode) X_(mode)^T (dims[mode]^2),
 * written in FP64 -- the SGEMMs of src/tucker_hosvd.cu:27-29. */
int cud_unfold_gram(const float *X, int order, const long *dims, int mode, double *G,
                    int precision, void *stream);

/* Extension (the slice-pair SGEMMs of the reference's out-of-core HOSVD,
 * decomposition/GPU/large/slice_tucker_hosvd.cu:38-40): a block of a Gram
 * between two column sets, G[i + ldg j] = sum_p A[p + P i] B[p + P j] for
 * i < ma, j < mb, FP32 operands (column-major, P rows), FP64 output. */
int cud_cross_gram(const float *A, const float *B, long P, long ma, long mb, double *G, long ldg,
                   void *stream);

/* ---- symmetric eigensolver / small solves ------------------------------ */

/* Extension (replaces cusolverDnSsyevdx at src/tucker_hosvd.cu:43-61):
 * FP64 Jacobi eigensolver of the symmetric n x n matrix A (destroyed).
 * W receives the n eigenvalues in ascending order and V the eigenvectors
 * (column j pairs with W[j]).  max_sweeps bounds the iteration. */
int cud_syev_jacobi(double *A, long n, double *W, double *V, int max_sweeps, void *stream);

/* Extension (replaces the partial cusolverDnSsyevdx call at
 * src/tucker_hosvd.cu:43-61, which asks for the leading eigenpairs only):
 * the r leading eigenvectors of the symmetric positive semi-definite n x n
 * FP64 matrix G (column-major; G is not modified) by subspace iteration,
 * into U (n x r, FP32, column-major) in ascending eigenvalue order (the
 * largest last).  U0 (n x r, FP32; may be NULL or alias U) seeds the
 * iteration instead of a random block.  Returns CUD_ERR_NOT_CONVERGED when
 * the subspace did not settle within max_iters steps (U is then not
 * written) and CUD_ERR_UNSUPPORTED for r > 64. */
int cud_syev_top(const double *G, long n, long r, float *U, const float *U0, int max_iters, void *stream);

/* ---- decompositions ----------------------------------------------------- */

typedef struct cud_cp_options {
    int max_sweeps;   /* sweep limit (the reference's fixed L, src/cp_als.cu:42) */
    double tol;       /* stop when |fit - fit_prev| < tol; <= 0 disables       */
    int precision;    /* cud_precision of the MTTKRPs                          */
    int use_graph;    /* capture each sweep in a CUDA graph                    */
    int check_every;  /* read the fit back every this many sweeps (>= 1)       */
    double target_fit; /* also stop once the exact fit >= target_fit, checked */
                       /* every check_every sweeps (<= 0 disables)            */
    int sweep_layout;  /* 0: by size; 1: per mode, split reduce then update  */
                       /* with its Gram, V^-1 beside the MTTKRP; 2 (R <= 64):*/
                       /* the update sums the MTTKRP partials itself, the Gram*/
                       /* and the next V^-1 run beside the next MTTKRP, four  */
                       /* sweeps a graph.  Results agree to rounding.         */
} cud_cp_options;

typedef struct cud_cp_result {
    int sweeps;       /* sweeps run                                           */
    int fallbacks;    /* normal-equation solves that fell back to pinv        */
    double fit;       /* 1 - ||X - Xhat|| / ||X|| of the returned factors,     */
                      /* exact (cud_cp_residual, src/rse.cu:4)                 */
    double fit_prev;  /* sweep estimate of the fit one sweep earlier           */
    double seconds;   /* wall time of the sweeps on the stream                 */
    int kernels_per_sweep; /* kernel launches in one sweep (graph kernel nodes) */
    double fit_estimate; /* the last sweep's estimate ||X||^2 - 2<M,U> + ||Xhat||^2 */
                      /* (cheap, but it cancels when fit -> 1 and inherits the */
                      /* MTTKRP's rounding)                                    */
} cud_cp_result;

/* Extension: default options (500 sweeps, tol 0, CUD_PREC_DEFAULT, graph on). */
void cud_cp_default_options(cud_cp_options *opt);

/* src/cp_als.cu:3-134 (order 3) and src/cp4_als.cu:3-186 (order 4) as one
 * general-order entry: CP-ALS from the initial factors U (host array of
 * device pointers, U[m] is dims[m] x R, updated in place).  Update order
 * U[0], U[1], ...; normal equations (Hadamard of FP64 Grams) solved by an
 * FP64 Gauss-Jordan inverse with SPD pivots, with a Jacobi pseudo-inverse
 * fallback.  res may be NULL. */
int cud_cp_als(const float *X, int order, const long *dims, long R, float *const *U,
               const cud_cp_options *opt, cud_cp_result *res, void *stream);
/* Extension: cud_cp_als keeps its last plan (workspace and captured sweep
 * graph) for the next call on the same device with the same X and factor
 * pointers, dims, rank, precision and graph setting -- the data-dependent
 * state (||X||^2, the Grams, the fit history) is recomputed each call.  One
 * plan is kept; cud_cp_als_release frees it. */
int cud_cp_als_release(void);

/* The reference's FP64 variants decomposition/GPU/normal/dprice/cp_als.cu:3-212
 * (order 3) and dprice/4_cp_als.cu:3-229 (order 4), as one general-order
 * entry over device pointers: CP-ALS entirely in FP64 (CUDA-core MTTKRP,
 * FP64 Grams, Hadamard, inverse with pseudo-inverse fallback, fit from the
 * Gram identity each sweep).  X and U[m] (dims[m] x R, updated in place)
 * are double; opt's precision, use_graph and check_every are ignored;
 * R <= 160.  res may be NULL. */
int cud_cp_als_f64(const double *X, int order, const long *dims, long R, double *const *U,
                   const cud_cp_options *opt, cud_cp_result *res, void *stream);

/* FP64 MTTKRP (the Khatri-Rao DGEMMs of dprice/cp_als.cu:64,72), any order
 * and mode: out (dims[mode] x R, double) = X_(mode) (KR of the other
 * factors), on the CUDA cores with no Khatri-Rao matrix formed. */
int cud_mttkrp_f64(const double *X, int order, const long *dims, const double *const *U, int mode, long R,
                   double *out, void *stream);

/* The reference's FP64 Tucker programs decomposition/GPU/normal/dprice/
 * tucker_hosvd.cu:3-167 (order 3), 4_tucker_hosvd.cu:3-173 (order 4) and
 * tucker_hooi.cu:3-220, as general-order entries over double device
 * buffers: FP64 unfolding Grams (CUDA-core GEMMs), the FP64 Jacobi
 * eigensolver (the r_n leading eigenvectors in ascending eigenvalue order,
 * as syevd returns them) and an FP64 mode-product chain for the core.
 * Arguments as cud_tucker_hosvd / cud_tucker_hooi, without precision. */
int cud_tucker_hosvd_f64(const double *X, int order, const long *dims, const long *ranks, double *core,
                         double *const *U, void *stream);
int cud_tucker_hooi_f64(const double *X, int order, const long *dims, const long *ranks, double *core,
                        double *const *U, int sweeps, void *stream);

/* Extension: a reusable CP-ALS plan -- the workspace, the Grams and the
 * captured per-sweep CUDA graph for one (X, dims, R, factors) problem, so
 * sweeps can be enqueued without synchronisation (what cud_cp_als loops
 * over).  X and U must stay allocated while the plan lives. */
typedef struct cud_cp_plan_s *cud_cp_plan;

/* Creates the plan, computes ||X||^2 and the initial Grams on `stream`. */
int cud_cp_plan_create(const float *X, int order, const long *dims, long R, float *const *U,
                       const cud_cp_options *opt, void *stream, cud_cp_plan *plan);
/* Enqueues `sweeps` sweeps on `stream` (no host synchronisation). */
int cud_cp_plan_run(cud_cp_plan plan, int sweeps, void *stream);
/* Synchronises `stream` and reads the last two fits (either may be NULL). */
int cud_cp_plan_fit(cud_cp_plan plan, double *fit, double *fit_prev, void *stream);
/* Kernel launches per sweep and the pseudo-inverse fallbacks so far. */
int cud_cp_plan_info(cud_cp_plan plan, int *kernels_per_sweep, int *fallbacks);
int cud_cp_plan_destroy(cud_cp_plan plan);

/* Extension: the pieces of one CP-ALS mode update, for callers that
 * orchestrate sweeps themselves (e.g. one process per GPU with the tensor
 * sharded along its last mode and the partial MTTKRPs summed by NCCL).
 * G = U^T U (R x R, FP64) for U (I x R). */
int cud_factor_gram(const float *U, long I, long R, double *G, void *stream);
/* U (I x R) = M (I x R) * V^-1 with V = Hadamard_{m != mode} G[m] (FP64
 * Gauss-Jordan with SPD pivots, Jacobi pseudo-inverse fallback).  G is a host array of `order` device
 * pointers (R x R each); work holds 3 R^2 doubles + 16 bytes. */
int cud_cp_solve(const float *M, long I, long R, int order, const double *const *G, int mode,
                 float *U, double *work, void *stream);
/* cud_cp_solve in two halves, so the R x R inverse can run on another
 * stream beside the mode's MTTKRP (it needs only the other modes' Grams):
 * work (3 R^2 doubles + 16 bytes) receives V^-1 in its first R^2 doubles;
 * then U = M * V^-1 (FP64 accumulation) reads it. */
int cud_cp_normal_inverse(long R, int order, const double *const *G, int mode, double *work, void *stream);
int cud_cp_apply_inverse(const float *M, long I, long R, const double *work, float *U, void *stream);
/* Host results of the fit terms: inner = <M, U> (FP64) and
 * norm_hat2 = sum_{r,s} prod_m G[m][r,s]. */
int cud_cp_fit_terms(const float *M, const float *U, long IR, int order, const double *const *G,
                     long R, double *inner, double *norm_hat2, void *stream);

/* Extension (the reference runs one tensor per cp_als call,
 * src/cp_als.cu:3): CP-ALS of `ntensors` independent 3rd-order tensors
 * in one persistent kernel launch per sweep.  Tensor t is dims[3t..3t+2]
 * (each in [1, 96]) of rank ranks[t] (in [1, 16]), stored column-major at
 * X + x_offsets[t]; its factor m is dims[3t+m] x ranks[t] at
 * U + u_offsets[3t+m] (initial values in, result out).  opt: max_sweeps, tol
 * (per tensor), use_graph, check_every (= sweeps per captured graph).
 * fits / sweeps (host arrays of ntensors, may be NULL) receive each tensor's
 * final fit and sweep count; kernel_launches (may be NULL) the number of
 * sweep kernels launched. */
int cud_cp_als_batched(int ntensors, const long *dims, const long *ranks, const float *X,
                       const long *x_offsets, float *U, const long *u_offsets,
                       const cud_cp_options *opt, double *fits, int *sweeps, int *kernel_launches,
                       void *stream);

/* cud_cp_als_batched with a per-tensor stopping fit: tensor t is done once
 * its fit >= target_fits[t] (host array; <= 0 disables for that tensor). */
int cud_cp_als_batched_target(int ntensors, const long *dims, const long *ranks, const float *X,
                              const long *x_offsets, float *U, const long *u_offsets,
                              const cud_cp_options *opt, const double *target_fits, double *fits, int *sweeps,
                              int *kernel_launches, void *stream);

/* Extension: autotunes the batched sweep's launch shape (threads per CTA,
 * CTAs per SM, and the rows of the MTTKRP register tile, 2 or 4) for this
 * batch's shape class by timing two sweeps per candidate; U_scratch is a
 * copy of the factors (overwritten).  The choice is cached per shape class
 * and used by later cud_cp_als_batched calls; threads and ctas_per_sm
 * report the first two. */
int cud_cp_batched_tune(int ntensors, const long *dims, const long *ranks, const float *X,
                        const long *x_offsets, float *U_scratch, const long *u_offsets, int *threads,
                        int *ctas_per_sm, void *stream);

/* Extension (the reference calls cublasGemmEx with FP16 operands,
 * src/mttkrp.cu:40-72 and src/ttm.cu:20-39): BF16 tensor-core GEMM
 *     C[m, n] = epilogue(alpha * sum_k A[m, k] * B[n, k])
 * with A (M x K, row stride lda) and B (N x K, row stride ldb) BF16, K
 * contiguous, lda and ldb multiples of 8, A and B 16-byte aligned; FP32
 * accumulation.  The epilogue applies, in order: alpha, + bias[n], zero where
 * mask[m, n] <= 0 (a BF16 matrix, e.g. a ReLU output; NULL = none), ReLU,
 * then writes each non-NULL output at out + m * ldm + n * ldn (FP32, with
 * f32_accumulate adding to the old value; BF16 rounded to nearest).  */
typedef struct {
    float alpha;
    const float *bias;
    int relu;
    const void *mask;        /* BF16 */
    long mask_ldm, mask_ldn;
    float *out_f32;
    long f32_ldm, f32_ldn;
    int f32_accumulate;
    void *out_bf16;          /* BF16 */
    long bf16_ldm, bf16_ldn;
    void *out_bf16_2;        /* BF16, e.g. the transposed copy */
    long bf16_2_ldm, bf16_2_ldn;
} cud_gemm_epilogue;

int cud_gemm_bf16(const void *A, long lda, const void *B, long ldb, long M, long N, long K,
                  const cud_gemm_epilogue *epilogue, void *stream);

/* src/rse.cu:4-29 (gencp + rse, called from src/cp_als.cu:104-111): the
 * CP model's residual ||X - [[U_0..U_{order-1}]]||^2 and ||X||^2 (FP64, host
 * outputs; synchronous), computed in one pass over X without materialising
 * the reconstruction.  fit = 1 - sqrt(res_norm2 / x_norm2). */
int cud_cp_residual(const float *X, int order, const long *dims, const float *const *U, long R,
                    double *res_norm2, double *x_norm2, void *stream);

/* Extension: the exact fit (cud_cp_residual) of the plan's current factors,
 * independent of the fit estimate the sweep derives from its last MTTKRP. */
int cud_cp_plan_true_fit(cud_cp_plan plan, double *fit, void *stream);

/* ---------------------------------------------------------------- learned warm start
 * Extension (no counterpart in the reference): a multilayer perceptron
 * in -> hidden -> hidden -> out (ReLU) that maps random sketches of a
 * tensor's mode unfoldings to initial CP factors for src/cp_als.cu's ALS.
 * FP32 master weights, BF16 tensor-core GEMMs (cud_gemm_bf16) for the
 * forward and backward passes, Adam.  All sizes multiples of 8. */
typedef struct cud_ws_model_s *cud_ws_model;

int cud_ws_model_create(int in_dim, int hidden, int out_dim, int max_batch, unsigned long long seed,
                        cud_ws_model *model);
int cud_ws_model_destroy(cud_ws_model model);
/* When I, R > 0 (out_dim = 3 I R): the loss compares the prediction with
 * the targets' CP factors matched to it -- components reordered and signs
 * aligned (U_0, U_1 flipped, U_2 compensating) -- instead of their given
 * order.  I = R = 0 restores the plain loss. */
int cud_ws_model_align(cud_ws_model model, int I, int R);
/* host[k] (k = W1, b1, W2, b2, W3, b3; W row-major out x in; NULL skips):
 * set = 1 copies host -> model (and refreshes the BF16 copies), 0 the reverse */
int cud_ws_model_params(cud_ws_model model, float *const *host, int set);
/* the gradients of the last cud_ws_backward / cud_ws_train_step, same order */
int cud_ws_model_grads(cud_ws_model model, float *const *host);
/* in: batch x in_dim BF16 (row-major), in_t: its transpose, target: batch x
 * out_dim FP32.  Forward + backward of the MSE loss (loss may be NULL). */
int cud_ws_backward(cud_ws_model model, const void *in, const void *in_t, const float *target, int batch,
                    double *loss, void *stream);
/* cud_ws_backward followed by one Adam step (betas 0.9, 0.999) */
int cud_ws_train_step(cud_ws_model model, const void *in, const void *in_t, const float *target, int batch,
                      float lr, double *loss, void *stream);
/* forward pass: out = batch x out_dim FP32 */
int cud_ws_predict(cud_ws_model model, const void *in, int batch, float *out, void *stream);

/* Workload: ntensors I^3 tensors (column-major, X[t] at X + t I^3) whose
 * CP factors (F[t][m], I x R column-major, at F + (3t + m) I R) have
 * columns sum_{q<3} a_q sin(2 pi w_q i / I + p_q), w ~ U[0.5, 4],
 * p ~ U[0, 2 pi), a ~ N(0, 1), plus i.i.d. Gaussian noise of relative
 * Frobenius size `noise`; tensor ids id0.. with `seed` (counter-based: the
 * same (seed, id) always gives the same tensor).  clean_norm2[t] =
 * ||X_clean||^2.  I <= 128, R <= 16, ntensors <= 65535. */
int cud_ws_generate(long ntensors, long id0, unsigned long long seed, int I, int R, double noise, float *X,
                    float *F, double *clean_norm2, void *stream);
/* the three Gaussian projections Omega_m^T (S x I^2 each, BF16, N(0, 1)) */
int cud_ws_omega(int I, int S, unsigned long long seed, void *omega, void *stream);
/* features of each tensor: [X_(m) Omega_m for m = 0, 1, 2] / ||X|| (BF16,
 * ntensors x 3 I S, and its transpose in_t if not NULL); xnorm2 = ||X||^2 */
int cud_ws_features(const float *X, long ntensors, int I, const void *omega, int S, void *in, void *in_t,
                    double *xnorm2, void *stream);
/* canonical form of CP factors in place: unit columns of U_0, U_1 with
 * non-negative sums, weights and signs in U_2 / ||X||, columns by weight */
int cud_ws_canonical(float *F, const double *xnorm2, long ntensors, int I, int R, void *stream);
/* network output (canonical, ntensors x 3 I R) -> ALS initial factors */
int cud_ws_uncanonical(const float *Y, const double *xnorm2, float *F, long ntensors, int I, int R,
                       void *stream);
/* HOSVD initialisation (src/tucker_hosvd.cu:3-103 applied per tensor): the
 * R leading eigenvectors of each mode Gram X_(m) X_(m)^T (I <= 64, Jacobi
 * in FP32) as the initial factors F */
int cud_ws_hosvd_init(const float *X, long ntensors, int I, int R, float *F, void *stream);

/* src/cp_als.cu:20-24: the reference's initialisation -- cuRAND default
 * pseudo-random generator, seed 1234, uniform [0,1) into U[1], then U[2], ...
 * (U[0] is left as is; the first update overwrites it). */
int cud_cp_init_curand(int order, const long *dims, long R, float *const *U,
                       unsigned long long seed, void *stream);

/* src/tucker_hosvd.cu:3-103 (order 3), src/tucker4_hosvd.cu:3-141 (order 4):
 * HOSVD.  U[m] (dims[m] x ranks[m]) = eigenvectors of the r_m largest
 * eigenvalues of the FP64 unfolding Gram, in ascending eigenvalue order as
 * the reference's syevdx output; core = X x_1 U1^T x_2 U2^T ... */
int cud_tucker_hosvd(const float *X, int order, const long *dims, const long *ranks,
                     float *core, float *const *U, int precision, void *stream);

/* decomposition/GPU/normal/tucker/tucker_hooi.cu:3-218: HOOI, `sweeps`
 * sweeps from the HOSVD initialisation of modes 2..N, then the core. */
int cud_tucker_hooi(const float *X, int order, const long *dims, const long *ranks,
                    float *core, float *const *U, int sweeps, int precision, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* CUDECOMPOSE_C_H_ */
