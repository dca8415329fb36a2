// The R x R side of CP-ALS, all in FP64 on the device: factor Grams, the
// Hadamard product of Grams, its inverse by Gauss-Jordan elimination with
// symmetric positive pivots (a pseudo-inverse by Jacobi eigen when a pivot is
// not positive), the factor update U_n = M V^-1, and
// the fit from the Gram/MTTKRP identity.  Replaces the FP32 getrf/getrs +
// geam sequence of src/cp_als.cu:53-63 (and :73-82, :92-101).
#include <atomic>
#include "kernels.cuh"
#include "solve.cuh"
#include "tc_ptx.cuh"

namespace cud {

namespace {

// G = U^T U (R x R, FP64) for U (I x R, FP32 or FP64).  16x16 output tile
// per CTA, rows staged through shared memory in chunks of 64.
template <typename T>
__global__ void __launch_bounds__(256) k_factor_gram(const T *__restrict__ U, long I, long R,
                                                     double *__restrict__ G) {
    __shared__ double sa[64][17];
    __shared__ double sb[64][17];
    long a0 = blockIdx.x * 16L, b0 = blockIdx.y * 16L;
    int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    double acc = 0.0;
    for (long i0 = 0; i0 < I; i0 += 64) {
        for (int e = threadIdx.x; e < 64 * 16; e += 256) {
            int ii = e & 63, cc = e >> 6;
            long i = i0 + ii;
            sa[ii][cc] = (i < I && a0 + cc < R) ? (double)U[i + I * (a0 + cc)] : 0.0;
            sb[ii][cc] = (i < I && b0 + cc < R) ? (double)U[i + I * (b0 + cc)] : 0.0;
        }
        __syncthreads();
#pragma unroll 8
        for (int ii = 0; ii < 64; ii++) acc = fma(sa[ii][tx], sb[ii][ty], acc);
        __syncthreads();
    }
    long a = a0 + tx, b = b0 + ty;
    if (a < R && b < R) G[a + R * b] = acc;
}

// Cyclic Jacobi on the symmetric n x n matrix held in shared memory (A), with
// eigenvectors accumulated in Q (global).  One CTA; rotations of disjoint
// (p, q) pairs run in parallel in round-robin order.  Returns sweeps used.
__device__ int block_jacobi_smem(double *A, double *Q, int n, int max_sweeps, double tol) {
    const int tid = threadIdx.x + blockDim.x * threadIdx.y, nthr = blockDim.x * blockDim.y;
    __shared__ double s_cos[128], s_sin[128];
    __shared__ int s_p[128], s_q[128];
    __shared__ double s_off;
    int m = (n + 1) & ~1;  // even number of players (a dummy when n is odd)
    for (int e = tid; e < n * n; e += nthr) Q[e] = (e % n == e / n) ? 1.0 : 0.0;
    __syncthreads();
    int sweep;
    for (sweep = 0; sweep < max_sweeps; sweep++) {
        if (tid == 0) {
            double off = 0.0, dia = 0.0;
            for (int j = 0; j < n; j++)
                for (int i = 0; i < n; i++) {
                    double v = A[i + n * j] * A[i + n * j];
                    if (i == j) dia += v; else off += v;
                }
            s_off = (off <= tol * tol * (dia + off)) ? -1.0 : off;
        }
        __syncthreads();
        if (s_off < 0) break;
        for (int round = 0; round < m - 1; round++) {
            // round-robin pairing: player 0 fixed, others rotate
            for (int k = tid; k < m / 2; k += nthr) {
                int a = (k == 0) ? 0 : 1 + (k - 1 + round) % (m - 1);
                int b = 1 + (m - 2 - k + round) % (m - 1);
                int p = min(a, b), q = max(a, b);
                double c = 1.0, s = 0.0;
                if (q < n) {
                    double apq = A[p + n * q];
                    if (apq != 0.0) {
                        double app = A[p + n * p], aqq = A[q + n * q];
                        double theta = (aqq - app) / (2.0 * apq);
                        double tt = (theta >= 0 ? 1.0 : -1.0) /
                                    (fabs(theta) + sqrt(theta * theta + 1.0));
                        c = 1.0 / sqrt(tt * tt + 1.0);
                        s = tt * c;
                    }
                }
                s_p[k] = p; s_q[k] = q; s_cos[k] = c; s_sin[k] = s;
            }
            __syncthreads();
            // rows: A <- J^T A
            for (int e = tid; e < (m / 2) * n; e += nthr) {
                int k = e / n, col = e % n;
                int p = s_p[k], q = s_q[k];
                if (q >= n) continue;
                double c = s_cos[k], s = s_sin[k];
                double ap = A[p + n * col], aq = A[q + n * col];
                A[p + n * col] = c * ap - s * aq;
                A[q + n * col] = s * ap + c * aq;
            }
            __syncthreads();
            // columns: A <- A J, Q <- Q J
            for (int e = tid; e < (m / 2) * n; e += nthr) {
                int k = e / n, row = e % n;
                int p = s_p[k], q = s_q[k];
                if (q >= n) continue;
                double c = s_cos[k], s = s_sin[k];
                double ap = A[row + n * p], aq = A[row + n * q];
                A[row + n * p] = c * ap - s * aq;
                A[row + n * q] = s * ap + c * aq;
                double vp = Q[row + n * p], vq = Q[row + n * q];
                Q[row + n * p] = c * vp - s * vq;
                Q[row + n * q] = s * vp + c * vq;
            }
            __syncthreads();
        }
    }
    return sweep;
}

// Pseudo-inverse of V = Hadamard of the Grams except `mode`, for when a
// Gauss-Jordan pivot is not positive: V is rebuilt in shared memory (R x R),
// eigendecomposed by Jacobi (eigenvectors in a.work + R^2) and inverted on
// the eigenvalues above R eps lambda_max.  Every thread of the CTA calls it.
__device__ void pinv_fallback(const NormalArgs &a, double *V, const double *const *sG) {
    const int tid = threadIdx.x + blockDim.x * threadIdx.y, nthr = blockDim.x * blockDim.y;
    const int R = a.R;
    double *Q = a.work + R * R;
    for (int e = tid; e < R * R; e += nthr) {
        double v = 1.0;
        for (int m = 0; m < a.nG; m++)
            if (m != a.mode) v *= sG[m][e];
        V[e] = v;
    }
    __syncthreads();
    block_jacobi_smem(V, Q, R, 60, 1e-15);
    __syncthreads();
    double lmax = 0.0;
    for (int j = 0; j < R; j++) lmax = fmax(lmax, fabs(V[j + R * j]));
    double cut = lmax * (double)R * 2.2e-16;
    for (int e = tid; e < R * R; e += nthr) {
        const int i = e % R, j = e / R;
        double sacc = 0.0;
        for (int k = 0; k < R; k++) {
            double l = V[k + R * k];
            if (l > cut) sacc += Q[i + R * k] * Q[j + R * k] / l;
        }
        a.Vinv[e] = sacc;
    }
    if (tid == 0 && a.fallbacks) atomicAdd(a.fallbacks, 1);
}

// The same inverse for R <= 64 with V held in registers: 16 x 16 threads,
// thread (tx, ty) owning the entries (ty + 16 a, tx + 16 b), a, b < 4.  Per
// pivot k the owners of row k and of column k publish them to shared memory
// (double-buffered by the parity of k, so one barrier per pivot suffices:
// a buffer is rewritten two pivots later, after every thread has passed the
// barrier that follows its last read) and every thread updates its 16
// entries with the elimination step of k_normal_inverse below.  Same pivots,
// same fallback.
constexpr int NI_SMALL_R = 64;
__global__ void __launch_bounds__(256) k_normal_inverse_small(NormalArgs a) {
    extern __shared__ double Vs[];  // R x R: the result's transpose, or the fallback's V
    __shared__ double rowb[2][NI_SMALL_R], colb[2][NI_SMALL_R];
    __shared__ double pinv[2];  // 1 / pivot, published with the pivot row
    __shared__ const double *sG[kMaxOrder];
    __shared__ double s_maxdiag;
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int R = a.R;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int m = 0; m < kMaxOrder; m++) sG[m] = (m < a.nG) ? a.G[m] : nullptr;
    }
    __syncthreads();
    double v[4][4];
#pragma unroll
    for (int ai = 0; ai < 4; ai++)
#pragma unroll
        for (int bj = 0; bj < 4; bj++) v[ai][bj] = (ty + 16 * ai < R && tx + 16 * bj < R) ? 1.0 : 0.0;
    for (int m = 0; m < a.nG; m++) {
        if (m == a.mode) continue;
        const double *g = sG[m];
        double t[4][4];  // the 16 loads of one Gram go out together
#pragma unroll
        for (int ai = 0; ai < 4; ai++)
#pragma unroll
            for (int bj = 0; bj < 4; bj++) {
                const int i = ty + 16 * ai, j = tx + 16 * bj;
                t[ai][bj] = (i < R && j < R) ? g[i + R * j] : 0.0;
            }
#pragma unroll
        for (int ai = 0; ai < 4; ai++)
#pragma unroll
            for (int bj = 0; bj < 4; bj++) v[ai][bj] *= t[ai][bj];
    }
    // the largest |diagonal entry| (owned by tx == ty, a == b)
    if (tx == ty) {
#pragma unroll
        for (int ai = 0; ai < 4; ai++) colb[0][ty + 16 * ai] = v[ai][ai];
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double mx = 0.0;
        for (int j = 0; j < R; j++) mx = fmax(mx, fabs(colb[0][j]));
        s_maxdiag = mx;
    }
    __syncthreads();
    const double maxdiag = s_maxdiag;
    bool fail = false;
    // the owner of the next pivot takes its reciprocal (one division per
    // pivot, not one per thread)
    double inv_next = (threadIdx.x == 0) ? __drcp_rn(v[0][0]) : 0.0;
    for (int k = 0; k < R; k++) {
        const int kb = k >> 4, kk = k & 15, buf = k & 1;
        if (tx == kk && ty == kk) pinv[buf] = inv_next;
        if (ty == kk) {
#pragma unroll
            for (int ai = 0; ai < 4; ai++)
                if (ai == kb) {
#pragma unroll
                    for (int bj = 0; bj < 4; bj++) rowb[buf][tx + 16 * bj] = v[ai][bj];
                }
        }
        if (tx == kk) {
#pragma unroll
            for (int bj = 0; bj < 4; bj++)
                if (bj == kb) {
#pragma unroll
                    for (int ai = 0; ai < 4; ai++) colb[buf][ty + 16 * ai] = v[ai][bj];
                }
        }
        __syncthreads();
        const double piv = rowb[buf][k];
        if (!(piv > 1e-13 * maxdiag) || !isfinite(piv)) {  // same decision in every thread
            fail = true;
            break;
        }
        const double inv = pinv[buf];
#pragma unroll
        for (int bj = 0; bj < 4; bj++) {
            const int j = tx + 16 * bj;
            const double rj = (j == k ? 1.0 : rowb[buf][j]) * inv;
#pragma unroll
            for (int ai = 0; ai < 4; ai++) {
                const int i = ty + 16 * ai;
                const double old = (j == k) ? 0.0 : v[ai][bj];
                v[ai][bj] = (i == k) ? rj : old - colb[buf][i] * rj;
            }
        }
        // entry (k + 1, k + 1) is owned by tx == ty == (k + 1) & 15, a == b == (k + 1) >> 4
        const int k1 = k + 1;
        if (k1 < R && tx == (k1 & 15) && ty == (k1 & 15)) {
            const int a1 = k1 >> 4;  // (a select chain keeps v in registers)
            const double d = a1 == 0 ? v[0][0] : a1 == 1 ? v[1][1] : a1 == 2 ? v[2][2] : v[3][3];
            inv_next = __drcp_rn(d);  // correctly rounded, = 1.0 / d
        }
    }
    __syncthreads();
    if (!fail) {
#pragma unroll
        for (int ai = 0; ai < 4; ai++)
#pragma unroll
            for (int bj = 0; bj < 4; bj++) {
                const int i = ty + 16 * ai, j = tx + 16 * bj;
                if (i < R && j < R) Vs[i + R * j] = v[ai][bj];
            }
        __syncthreads();
        for (int e = threadIdx.x; e < R * R; e += 256) {
            const int i = e % R, j = e / R;
            a.Vinv[e] = 0.5 * (Vs[i + R * j] + Vs[j + R * i]);  // symmetrise
        }
    } else {
        pinv_fallback(a, Vs, sG);
    }
}

// The same inverse for R <= RW in one warp: lane j holds column j of V in
// registers; per pivot k the pivot and column k come from lane k by
// shuffles and every lane updates its column (no block barriers).  Same
// pivots, same elimination step, same fallback.  Used for R <= 16 (6.8 us
// against 11.6 for the 256-thread kernel on B200); at R = 32 the lone warp
// was slower, most of all beside an MTTKRP that fills the SM.
template <int RW>
__global__ void __launch_bounds__(32) k_normal_inverse_warp(NormalArgs a) {
    extern __shared__ double Vw[];  // 32 x 32: the transpose for the output, or the fallback's V
    __shared__ const double *sG[kMaxOrder];
    const int j = threadIdx.x;
    const int R = a.R;
    if (j == 0) {
#pragma unroll
        for (int m = 0; m < kMaxOrder; m++) sG[m] = (m < a.nG) ? a.G[m] : nullptr;  // static indices
    }
    __syncwarp();
    double v[RW];
#pragma unroll
    for (int i = 0; i < RW; i++) v[i] = (i < R && j < R) ? 1.0 : 0.0;
    for (int m = 0; m < a.nG; m++) {
        if (m == a.mode) continue;
        const double *g = sG[m];
        double t[RW];
#pragma unroll
        for (int i = 0; i < RW; i++) t[i] = (i < R && j < R) ? g[i + R * j] : 0.0;
#pragma unroll
        for (int i = 0; i < RW; i++) v[i] *= t[i];
    }
    double dg = 0.0;  // this lane's diagonal entry
#pragma unroll
    for (int i = 0; i < RW; i++)
        if (i == j) dg = v[i];
    double maxdiag = fabs(dg);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) maxdiag = fmax(maxdiag, __shfl_xor_sync(0xffffffffu, maxdiag, o));
    bool fail = false;
#pragma unroll
    for (int k = 0; k < RW; k++) {
        if (k >= R) break;
        const double piv = __shfl_sync(0xffffffffu, v[k], k);
        if (!(piv > 1e-13 * maxdiag) || !isfinite(piv)) {  // same decision in every lane
            fail = true;
            break;
        }
        const double inv = __drcp_rn(piv);  // correctly rounded, = 1.0 / piv
        const double rj = (j == k ? 1.0 : v[k]) * inv;
#pragma unroll
        for (int i = 0; i < RW; i++) {
            const double ck = __shfl_sync(0xffffffffu, v[i], k);  // column k, row i
            const double old = (j == k) ? 0.0 : v[i];
            v[i] = (i == k) ? rj : old - ck * rj;
        }
    }
    if (!fail) {
#pragma unroll
        for (int i = 0; i < RW; i++) Vw[i + 32 * j] = v[i];
        __syncwarp();
        for (int e = j; e < R * R; e += 32) {
            const int r = e % R, c = e / R;
            a.Vinv[e] = 0.5 * (Vw[r + 32 * c] + Vw[c + 32 * r]);  // symmetrise
        }
    } else {
        pinv_fallback(a, Vw, sG);
    }
}

// V = Hadamard of the Grams of all factors except `mode`; Vinv = V^-1 by
// in-place Gauss-Jordan elimination without pivoting (V is symmetric
// positive definite, so every pivot is a positive Schur complement -- the
// same pivots as its Cholesky factorisation), or, when a pivot is not
// positive, the pseudo-inverse from a Jacobi eigendecomposition.  One CTA,
// V in dynamic shared memory, two barriers per pivot.  `work` is global
// scratch of 2 R^2 doubles.
__global__ void __launch_bounds__(512) k_normal_inverse(NormalArgs a) {
    // 32 x 16 threads: element (i, j) of an R x R matrix visited as
    // i = tx, tx + 32, ...; j = ty, ty + 16, ... (no per-element division)
    extern __shared__ double V[];  // R x R
    __shared__ int s_fail;
    __shared__ double rowk[160], colk[160];
    __shared__ const double *sG[kMaxOrder];
    const int tx = threadIdx.x, ty = threadIdx.y, tid = tx + 32 * ty;
    const int R = a.R;
    if (tid == 0) {
#pragma unroll
        for (int m = 0; m < kMaxOrder; m++) sG[m] = (m < a.nG) ? a.G[m] : nullptr;
        s_fail = 0;
    }
    __syncthreads();
    for (int j = ty; j < R; j += 16)
        for (int i = tx; i < R; i += 32) {
            double v = 1.0;
            for (int m = 0; m < a.nG; m++)
                if (m != a.mode) v *= sG[m][i + R * j];
            V[i + R * j] = v;
        }
    __syncthreads();
    double maxdiag = 0.0;
    for (int j = 0; j < R; j++) maxdiag = fmax(maxdiag, fabs(V[j + R * j]));
    for (int k = 0; k < R; k++) {
        const double piv = V[k + R * k];
        if (!(piv > 1e-13 * maxdiag) || !isfinite(piv)) {  // same decision in every thread
            if (tid == 0) s_fail = 1;
            break;
        }
        const double inv = 1.0 / piv;
        for (int j = tid; j < R; j += 512) {
            rowk[j] = (j == k ? 1.0 : V[k + R * j]) * inv;
            colk[j] = V[j + R * k];
        }
        __syncthreads();
        for (int j = ty; j < R; j += 16) {
            const double rj = rowk[j];
            for (int i = tx; i < R; i += 32) {
                const double old = (j == k) ? 0.0 : V[i + R * j];
                V[i + R * j] = (i == k) ? rj : old - colk[i] * rj;
            }
        }
        __syncthreads();
    }
    __syncthreads();
    if (!s_fail) {
        for (int j = ty; j < R; j += 16)
            for (int i = tx; i < R; i += 32) a.Vinv[i + R * j] = 0.5 * (V[i + R * j] + V[j + R * i]);  // symmetrise
    } else {
        pinv_fallback(a, V, sG);
    }
}

// U (I x R, FP32) = M (I x R, FP32) * Vinv (R x R, FP64), FP64 accumulation.
__global__ void __launch_bounds__(256) k_apply_inverse(const float *__restrict__ M,
                                                       const double *__restrict__ Vinv, long I,
                                                       long R, float *__restrict__ U) {
    extern __shared__ double sV[];  // R x R when it fits, else read from global
    const bool in_smem = (R <= 64);
    if (in_smem) {
        for (long e = threadIdx.x; e < R * R; e += blockDim.x) sV[e] = Vinv[e];
        __syncthreads();
    }
    const double *Vp = in_smem ? sV : Vinv;
    long n = I * R;
    long tid = blockIdx.x * (long)blockDim.x + threadIdx.x;
    long stride = (long)gridDim.x * blockDim.x;
    for (long e = tid; e < n; e += stride) {
        long i = e % I, c = e / I;
        double s = 0.0;
        for (long r = 0; r < R; r++) s = fma((double)M[i + I * r], Vp[r + R * c], s);
        U[e] = (float)s;
    }
}

// fit = 1 - sqrt(max(||X||^2 - 2<M, U> + sum_{r,s} prod_m G_m[r,s], 0)) / ||X||
__global__ void __launch_bounds__(256) k_fit(FitArgs a) {
    __shared__ double sh[2][8];
    double inner = 0.0, hat = 0.0;
    for (long e = threadIdx.x; e < a.IR; e += blockDim.x) inner += (double)a.M[e] * (double)a.U[e];
    for (long e = threadIdx.x; e < (long)a.R * a.R; e += blockDim.x) {
        double p = 1.0;
        for (int m = 0; m < a.nG; m++) p *= a.G[m][e];
        hat += p;
    }
    for (int o = 16; o > 0; o >>= 1) {
        inner += __shfl_xor_sync(0xffffffffu, inner, o);
        hat += __shfl_xor_sync(0xffffffffu, hat, o);
    }
    int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) { sh[0][w] = inner; sh[1][w] = hat; }
    __syncthreads();
    if (threadIdx.x == 0) {
        double in = 0.0, h = 0.0;
        for (int i = 0; i < 8; i++) { in += sh[0][i]; h += sh[1][i]; }
        double res2 = a.normx2 - 2.0 * in + h;
        double fit = 1.0 - sqrt(res2 > 0.0 ? res2 : 0.0) / sqrt(a.normx2);
        a.out[1] = a.out[0];  // previous fit
        a.out[0] = fit;
        a.out[2] = in;
        a.out[3] = h;
    }
}

// Factor update in two passes, wide enough to occupy the GPU for the small
// I of CP factors.  Pass 1 (k_update_rows): each CTA takes a contiguous
// block of rows, 16 at a time staged in shared memory; U = M * Vinv with
// FP64 accumulation (skipped when Vinv is null: U = M), the CTA's partial
// Gram sum_i u_i u_i^T (upper triangle, e = q (q + 1) / 2 + p for p <= q)
// and its part of <M, U>, written as one partial per CTA.  Pass 2
// (k_update_reduce): one thread per triangle entry sums the partials in CTA
// order (deterministic), writes G (both halves), and, for the fit, each
// CTA's share of ||Xhat||^2 = sum_pq prod_m G_m[p, q] (off-diagonal entries
// twice); the last CTA (atomic ticket) combines those in order and writes
// the fit.
constexpr int UPD_RB = 16;
constexpr int UPD_STAGE_V = 64;    // V^-1 staged in shared memory up to this R
constexpr int SU_LD = UPD_RB + 1;  // sU column stride (odd: conflict-free Gram reads)
constexpr int UPD_RED = 256;       // threads of the reduce pass

// (p, q), p <= q, of upper-triangle entry e = q (q + 1) / 2 + p
__device__ __forceinline__ void tri_pq(long e, int &p, int &q) {
    q = (int)((sqrt(8.0 * (double)e + 1.0) - 1.0) * 0.5);
    while ((long)(q + 1) * (q + 2) / 2 <= e) q++;
    while ((long)q * (q + 1) / 2 > e) q--;
    p = (int)(e - (long)q * (q + 1) / 2);
}

template <int NT, int NACC, int UPT>
__global__ void __launch_bounds__(NT) k_update_rows(UpdateArgs a) {
    // shared: sU (SU_LD x R FP64), sM (UPD_RB x R FP32, this chunk of M),
    // sV (R x R FP64, V^-1 staged when R <= UPD_STAGE_V)
    extern __shared__ double smem_d[];
    __shared__ double s_red[NT / 32];
    const int R = a.R;
    const long I = a.I;
    double *sU = smem_d;
    float *sM = reinterpret_cast<float *>(sU + SU_LD * R);
    double *sV = sU + SU_LD * R + (UPD_RB * R + 1) / 2;
    const bool stage_v = a.Vinv && R <= UPD_STAGE_V;
    if (stage_v)
        for (int e0 = threadIdx.x; e0 < R * R; e0 += 8 * NT) {
            double t[8];
#pragma unroll
            for (int k = 0; k < 8; k++) t[k] = (e0 + k * NT < R * R) ? a.Vinv[e0 + k * NT] : 0.0;
#pragma unroll
            for (int k = 0; k < 8; k++)
                if (e0 + k * NT < R * R) sV[e0 + k * NT] = t[k];
        }
    const double *V = stage_v ? sV : a.Vinv;
    const long rpb = ((I + gridDim.x - 1) / gridDim.x + UPD_RB - 1) / UPD_RB * UPD_RB;
    const long r0 = blockIdx.x * rpb, r1 = min(I, r0 + rpb);
    // U = M V^-1: thread t owns column c = t % R of the rows i = g, g + ng,
    // ... (g = t / R, ng = NT / R groups; at most UPT rows): independent FMA
    // chains that share each V^-1 load
    const int ng = NT / R;
    const int cu = threadIdx.x % R, gu = threadIdx.x / R;
    double acc[NACC];
#pragma unroll
    for (int k = 0; k < NACC; k++) acc[k] = 0.0;
    int p0, q0;  // this thread's first triangle entry e = tid
    tri_pq(threadIdx.x, p0, q0);
    double inner = 0.0;
    for (long c0 = r0; c0 < r1; c0 += UPD_RB) {
        const int nr = (int)min((long)UPD_RB, r1 - c0);
        {
            constexpr int NB = (UPD_RB * 160 + NT - 1) / NT;  // loads per thread at the largest R
            float t[NB];
#pragma unroll
            for (int k = 0; k < NB; k++) {
                const int e = threadIdx.x + k * NT, i = e % UPD_RB, c = e / UPD_RB;
                t[k] = (e < UPD_RB * R && i < nr) ? a.M[c0 + i + I * c] : 0.f;
            }
#pragma unroll
            for (int k = 0; k < NB; k++)
                if (threadIdx.x + k * NT < UPD_RB * R) sM[threadIdx.x + k * NT] = t[k];
        }
        __syncthreads();
        if (a.Vinv) {
            if (gu < ng) {
                double u[UPT];
#pragma unroll
                for (int k = 0; k < UPT; k++) u[k] = 0.0;
                for (int r = 0; r < R; r++) {
                    // V^-1 is symmetric: column cu read along consecutive
                    // lanes, free of bank conflicts
                    const double v = V[cu + R * r];
#pragma unroll
                    for (int k = 0; k < UPT; k++)
                        if (gu + k * ng < UPD_RB) u[k] = fma((double)sM[gu + k * ng + UPD_RB * r], v, u[k]);
                }
#pragma unroll
                for (int k = 0; k < UPT; k++) {
                    const int i = gu + k * ng;
                    if (i < UPD_RB) {
                        double ud = 0.0;
                        if (i < nr) {
                            ud = (double)(float)u[k];
                            if (a.fit_out) inner += (double)sM[i + UPD_RB * cu] * ud;
                        }
                        sU[i + SU_LD * cu] = ud;
                    }
                }
            }
        } else {
            for (int e = threadIdx.x; e < UPD_RB * R; e += NT) {
                const int i = e % UPD_RB, c = e / UPD_RB;
                const double ud = (i < nr) ? (double)sM[e] : 0.0;
                if (a.fit_out) {
                    // <M, U> with the MTTKRP M given apart from U (the Gram's input)
                    const double m = a.Mfit ? ((i < nr) ? (double)a.Mfit[c0 + i + I * c] : 0.0) : (double)sM[e];
                    inner += m * ud;
                }
                sU[i + SU_LD * c] = ud;
            }
        }
        __syncthreads();
        // this chunk's rows of U, coalesced (16 consecutive rows per column)
        if (a.Vinv)
            for (int e = threadIdx.x; e < UPD_RB * R; e += NT) {
                const int i = e % UPD_RB, c = e / UPD_RB;
                if (i < nr) a.U[c0 + i + I * c] = (float)sU[i + SU_LD * c];
            }
        // triangle entries e = tid + NT k, (p, q) stepped incrementally
        {
            int p = p0, q = q0;
#pragma unroll
            for (int k = 0; k < NACC; k++) {
                if (q < R) {
                    double sacc = acc[k];
#pragma unroll
                    for (int i = 0; i < UPD_RB; i++) sacc = fma(sU[i + SU_LD * p], sU[i + SU_LD * q], sacc);
                    acc[k] = sacc;
                }
                p += NT;
                while (p > q && q < R) {
                    p -= q + 1;
                    q++;
                }
            }
        }
        __syncthreads();
    }
    const int T = R * (R + 1) / 2;
    const long stride = (long)T + 1;
    double *mine = a.gpart + blockIdx.x * stride;
#pragma unroll
    for (int k = 0; k < NACC; k++) {
        const int e = threadIdx.x + NT * k;
        if (e < T) mine[e] = acc[k];
    }
    for (int o = 16; o > 0; o >>= 1) inner += __shfl_xor_sync(0xffffffffu, inner, o);
    if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = inner;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < NT / 32; w++) t += s_red[w];
        mine[T] = t;
    }
}

// Gram partials of U (I x R, FP32, column-major; R <= 64) for the reduce
// pass below, with the partial layout of k_update_rows (entry e = q (q + 1)
// / 2 + p, stride T + 1, slot T = the CTA's part of <M, U> when fit_out is
// set).  CTA b takes rows [b rpc, (b + 1) rpc), staged GR_ROWS at a time in
// shared memory row-major (all of a stage's loads in flight together, along
// the rows: coalesced); thread t < R4 (R4 + 1) / 2 owns the 4 x 4 block
// (bp, bq), bp <= bq, of the upper triangle and accumulates its 16 products
// in FP64, two float4 shared-memory reads per row.
constexpr int GR_NT = 256, GR_ROWS = 128, GR_RMAX = 64;
__global__ void __launch_bounds__(GR_NT) k_gram_rows(UpdateArgs a, int rpc) {
    extern __shared__ __align__(16) float gsm[];  // GR_ROWS x RP
    __shared__ double s_red[GR_NT / 32];
    const int R = a.R, R4 = (R + 3) / 4, RP = 4 * R4 + 4;
    const long I = a.I;
    const long r0 = (long)blockIdx.x * rpc, r1 = min(I, r0 + rpc);
    const int nblk = R4 * (R4 + 1) / 2;
    int bp = 0, bq = 0;
    if ((int)threadIdx.x < nblk) tri_pq(threadIdx.x, bp, bq);
    double acc[4][4];
#pragma unroll
    for (int u = 0; u < 4; u++)
#pragma unroll
        for (int v = 0; v < 4; v++) acc[u][v] = 0.0;
    double inner = 0.0;
    const float *Mf = a.Mfit ? a.Mfit : a.M;
    for (long c0 = r0; c0 < r1; c0 += GR_ROWS) {
        const int nr = (int)min((long)GR_ROWS, r1 - c0);
        constexpr int NB = GR_ROWS * GR_RMAX / GR_NT;
        float t[NB];
#pragma unroll
        for (int k = 0; k < NB; k++) {
            const int e = threadIdx.x + k * GR_NT, i = e % GR_ROWS, c = e / GR_ROWS;
            t[k] = (c < R && i < nr) ? a.M[c0 + i + I * c] : 0.f;
        }
        if (a.fit_out) {
#pragma unroll
            for (int k = 0; k < NB; k++) {
                const int e = threadIdx.x + k * GR_NT, i = e % GR_ROWS, c = e / GR_ROWS;
                if (c < R && i < nr) inner += (double)Mf[c0 + i + I * c] * (double)t[k];
            }
        }
#pragma unroll
        for (int k = 0; k < NB; k++) {
            const int e = threadIdx.x + k * GR_NT, i = e % GR_ROWS, c = e / GR_ROWS;
            if (c < 4 * R4) gsm[i * RP + c] = t[k];
        }
        __syncthreads();
        if ((int)threadIdx.x < nblk) {
            for (int i = 0; i < nr; i++) {
                const float4 x = *reinterpret_cast<const float4 *>(gsm + i * RP + 4 * bp);
                const float4 y = *reinterpret_cast<const float4 *>(gsm + i * RP + 4 * bq);
                const double xv[4] = {x.x, x.y, x.z, x.w}, yv[4] = {y.x, y.y, y.z, y.w};
#pragma unroll
                for (int u = 0; u < 4; u++)
#pragma unroll
                    for (int v = 0; v < 4; v++) acc[u][v] = fma(xv[u], yv[v], acc[u][v]);
            }
        }
        __syncthreads();
    }
    const int T = R * (R + 1) / 2;
    double *mine = a.gpart + blockIdx.x * ((long)T + 1);
    if ((int)threadIdx.x < nblk) {
#pragma unroll
        for (int u = 0; u < 4; u++)
#pragma unroll
            for (int v = 0; v < 4; v++) {
                const int p = 4 * bp + u, q = 4 * bq + v;
                if (p <= q && q < R) mine[q * (q + 1) / 2 + p] = acc[u][v];
            }
    }
    for (int o = 16; o > 0; o >>= 1) inner += __shfl_xor_sync(0xffffffffu, inner, o);
    if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = inner;
    __syncthreads();
    if (threadIdx.x == 0) {
        double tt = 0.0;
        for (int w = 0; w < GR_NT / 32; w++) tt += s_red[w];
        mine[T] = tt;
    }
}

__global__ void __launch_bounds__(UPD_RED) k_update_reduce(UpdateArgs a, int nparts) {
    __shared__ double s_red[UPD_RED / 32];
    __shared__ int s_last;
    const int R = a.R;
    const int T = R * (R + 1) / 2;
    const long stride = (long)T + 1;
    const long e = blockIdx.x * (long)UPD_RED + threadIdx.x;
    double *hat_part = a.gpart + (size_t)nparts * stride;  // one per reduce CTA, then <M, U>
    double hat = 0.0;
    if (e < stride) {
        // fixed-order sum of the partials, 8 independent loads in flight
        double p8[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
        int b = 0;
        for (; b + 8 <= nparts; b += 8) {
#pragma unroll
            for (int j = 0; j < 8; j++) p8[j] += __ldcg(a.gpart + (b + j) * stride + e);
        }
#pragma unroll
        for (int j = 0; j < 8; j++)
            if (b + j < nparts) p8[j] += __ldcg(a.gpart + (b + j) * stride + e);
        const double sum = ((p8[0] + p8[1]) + (p8[2] + p8[3])) + ((p8[4] + p8[5]) + (p8[6] + p8[7]));
        if (e < T) {
            int p, q;
            tri_pq(e, p, q);
            a.G_out[p + R * q] = sum;
            a.G_out[q + R * p] = sum;
            if (a.fit_out) {
                double pr = 1.0;
                for (int m = 0; m < a.nG; m++) pr *= (m == a.mode) ? sum : a.Gall[m][p + R * q];
                hat = (p == q) ? pr : 2.0 * pr;
            }
        } else if (a.fit_out) {
            hat_part[gridDim.x] = sum;  // <M, U>
        }
    }
    if (!a.fit_out) return;
    for (int o = 16; o > 0; o >>= 1) hat += __shfl_xor_sync(0xffffffffu, hat, o);
    if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = hat;
    __syncthreads();
    if (threadIdx.x == 0) {
        double h = 0.0;
        for (int w = 0; w < UPD_RED / 32; w++) h += s_red[w];
        hat_part[blockIdx.x] = h;
        __threadfence();
        const unsigned ticket = atomicAdd(a.counter, 1u);
        s_last = (ticket == gridDim.x - 1);
    }
    __syncthreads();
    if (!s_last || threadIdx.x != 0) return;
    __threadfence();
    double h = 0.0;
    for (unsigned b = 0; b < gridDim.x; b++) h += __ldcg(hat_part + b);
    const double in = __ldcg(hat_part + gridDim.x);
    const double res2 = a.normx2 - 2.0 * in + h;
    const double fit = 1.0 - sqrt(res2 > 0.0 ? res2 : 0.0) / sqrt(a.normx2);
    a.fit_out[1] = a.fit_out[0];
    a.fit_out[0] = fit;
    a.fit_out[2] = in;
    a.fit_out[3] = h;
    atomicExch(a.counter, 0u);
}

// U = M V^-1 straight from an MTTKRP's split partials (the split reduce
// and the update in one kernel).  A CTA owns rb <= FU_RB consecutive rows:
//   * right after the grid-dependency wait (it runs as a programmatic
//     dependent of the MTTKRP) it starts the copy of V^-1 into shared memory
//     (cp.async, 16 B pieces) and issues all its partial loads, so both take
//     one round trip;
//   * the partials of an entry are summed over the splits in FP64 in split
//     order: split z by thread z mod T (T threads per float4 of a row, or per
//     element when the layout is not float4-able), the T sums combined in
//     thread order; M is rounded to FP32 and written;
//   * U = M V^-1 in FP64 (as k_update_rows), rounded to FP32.
constexpr int FU_NT = 256;
constexpr int FU_RB = 8;
constexpr int FU_LOADS = 16;   // partial loads per thread per batch (floats)
constexpr int FU_LOADS4 = 10;  // the same for float4 loads (two CTAs per SM)
struct FusedArgs {
    MttkrpParts pp;
    const double *Vinv;
    float *M, *U;
    long I;
    int R, rb;
    int vec;  // partial rows are float4-able: rs == 1, qs, zs multiples of 4, 16 B aligned
};

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_u32(smem)), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// sum over z = z0, z0 + dz, ... < nz of p[z zs], in z order, FP64; the loads
// go out in batches of FU_LOADS
__device__ __forceinline__ double split_sum(const float *p, long zs, int z0, int nz, int dz) {
    double sum = 0.0;
    for (int z = z0; z < nz; z += FU_LOADS * dz) {
        float t[FU_LOADS];
#pragma unroll
        for (int k = 0; k < FU_LOADS; k++) t[k] = (z + k * dz < nz) ? __ldcs(p + (long)(z + k * dz) * zs) : 0.f;
#pragma unroll
        for (int k = 0; k < FU_LOADS; k++)
            if (z + k * dz < nz) sum += (double)t[k];
    }
    return sum;
}

// the same for four consecutive entries (a float4 of a partial row)
__device__ __forceinline__ void split_sum4(const float *p, long zs, int z0, int nz, int dz, double s[4]) {
    s[0] = s[1] = s[2] = s[3] = 0.0;
    for (int z = z0; z < nz; z += FU_LOADS4 * dz) {
        float4 t[FU_LOADS4];
#pragma unroll
        for (int k = 0; k < FU_LOADS4; k++)
            t[k] = (z + k * dz < nz) ? __ldcs(reinterpret_cast<const float4 *>(p + (long)(z + k * dz) * zs))
                                     : make_float4(0.f, 0.f, 0.f, 0.f);
#pragma unroll
        for (int k = 0; k < FU_LOADS4; k++)
            if (z + k * dz < nz) {
                s[0] += (double)t[k].x;
                s[1] += (double)t[k].y;
                s[2] += (double)t[k].z;
                s[3] += (double)t[k].w;
            }
    }
}

__global__ void __launch_bounds__(FU_NT, 2) k_update_fused(FusedArgs a) {
    extern __shared__ __align__(16) double fsm[];
    const int R = a.R;
    double *sV = fsm;               // R x R
    double *sM = sV + R * R;        // rb x R, row-major (entry it = row R + c)
    double *sP = sM + FU_RB * R;    // 4 FU_NT split sums
    ptx::griddep_wait();
    {
        const int n16 = R * R / 2;  // 16-byte pieces of V^-1
        for (int e = threadIdx.x; e < n16; e += FU_NT) cp_async16(sV + 2 * e, a.Vinv + 2 * e);
        if ((R * R) & 1) {
            if (threadIdx.x == 0) sV[R * R - 1] = a.Vinv[R * R - 1];
        }
    }
    const long q0 = (long)blockIdx.x * a.rb;
    const int nr = (int)min((long)a.rb, a.I - q0);
    const bool bad = a.pp.error && *a.pp.error != 0;
    const double nan = __longlong_as_double(0x7ff8000000000000LL);
    if (a.vec) {
        const int R4 = (R + 3) / 4;
        const int items = nr * R4;  // float4 slots
        const int T = items >= FU_NT ? 1 : FU_NT / items;
        if (T == 1) {
            for (int it = threadIdx.x; it < items; it += FU_NT) {
                const int row = it / R4, c0 = 4 * (it - row * R4);
                double sv[4];
                split_sum4(a.pp.part + (q0 + row) * a.pp.qs + c0, a.pp.zs, 0, a.pp.splits, 1, sv);
#pragma unroll
                for (int k = 0; k < 4; k++)
                    if (c0 + k < R) sM[row * R + c0 + k] = bad ? nan : (double)(float)sv[k];
            }
        } else {
            const int it = threadIdx.x % items, zt = threadIdx.x / items;
            double sv[4] = {0.0, 0.0, 0.0, 0.0};
            if (zt < T) {
                const int row = it / R4, c0 = 4 * (it - row * R4);
                split_sum4(a.pp.part + (q0 + row) * a.pp.qs + c0, a.pp.zs, zt, a.pp.splits, T, sv);
            }
#pragma unroll
            for (int k = 0; k < 4; k++) sP[4 * threadIdx.x + k] = sv[k];
            __syncthreads();
            for (int e = threadIdx.x; e < nr * R; e += FU_NT) {
                const int row = e / R, c = e - row * R;
                const int slot = row * R4 + c / 4, k = c & 3;
                double t = 0.0;
                for (int z = 0; z < T; z++) t += sP[4 * (z * items + slot) + k];
                sM[e] = bad ? nan : (double)(float)t;
            }
        }
    } else {
        const int items = nr * R;
        const int T = items >= FU_NT ? 1 : FU_NT / items;
        if (T == 1) {
            for (int it = threadIdx.x; it < items; it += FU_NT) {
                const int row = it / R, c = it - row * R;
                const float *pp = a.pp.part + (q0 + row) * a.pp.qs + c * a.pp.rs;
                sM[it] = bad ? nan : (double)(float)split_sum(pp, a.pp.zs, 0, a.pp.splits, 1);
            }
        } else {
            const int it = threadIdx.x % items, zt = threadIdx.x / items;
            double sum = 0.0;
            if (zt < T) {
                const int row = it / R, c = it - row * R;
                const float *pp = a.pp.part + (q0 + row) * a.pp.qs + c * a.pp.rs;
                sum = split_sum(pp, a.pp.zs, zt, a.pp.splits, T);
            }
            sP[threadIdx.x] = sum;
            __syncthreads();
            if (threadIdx.x < items) {
                double t = 0.0;
                for (int k = 0; k < T; k++) t += sP[k * items + threadIdx.x];
                sM[threadIdx.x] = bad ? nan : (double)(float)t;
            }
        }
    }
    cp_async_wait_all();
    __syncthreads();
    for (int it = threadIdx.x; it < nr * R; it += FU_NT) {
        const int row = it / R, c = it - row * R;
        const double *mr = sM + row * R;
        double u = 0.0;
        // V^-1 is symmetric: column c read along consecutive lanes
#pragma unroll 8
        for (int r = 0; r < R; r++) u = fma(mr[r], sV[c + R * r], u);
        const long q = q0 + row;
        a.M[q + a.I * c] = (float)mr[c];
        a.U[q + a.I * c] = (float)u;
    }
}

}  // namespace

int update_from_parts(const MttkrpParts &pp, const double *Vinv, long I, int R, float *M, float *U,
                      cudaStream_t s) {
    if (R > FU_RMAX || I <= 0) return CUD_ERR_UNSUPPORTED;
    FusedArgs a;
    a.pp = pp;
    a.Vinv = Vinv;
    a.M = M;
    a.U = U;
    a.I = I;
    a.R = R;
    a.rb = (int)std::min<long>(FU_RB, std::max<long>(1, (I + 255) / 256));
    const uintptr_t al = reinterpret_cast<uintptr_t>(pp.part);
    a.vec = (pp.rs == 1 && pp.qs % 4 == 0 && pp.zs % 4 == 0 && (al & 15) == 0 &&
             pp.qs >= (R + 3) / 4 * 4) ? 1 : 0;
    if ((reinterpret_cast<uintptr_t>(Vinv) & 15) != 0) return CUD_ERR_UNSUPPORTED;
    const unsigned grid = (unsigned)((I + a.rb - 1) / a.rb);
    const size_t smem = sizeof(double) * ((size_t)R * R + (size_t)FU_RB * R + 4 * FU_NT);
    PdlLaunch l(grid, FU_NT, smem, s);
    CUD_CHECK(cudaLaunchKernelEx(&l.cfg, k_update_fused, a));
    CUD_CHECK_LAUNCH("update_from_parts");
    return CUD_OK;
}

// Pass-1 CTAs: 16-row chunks, at most two per SM, and few enough that the
// partial Grams stay within about 32 MB.
int update_blocks(long I, long R) {
    const long byrows = (I + UPD_RB - 1) / UPD_RB;
    const long cap = std::max(8L, 4000000L / (R * (R + 1) / 2 + 1));
    return (int)std::max(1L, std::min(std::min(byrows, 2L * kNumSMs), cap));
}

static long update_red_blocks(long R) { return (R * (R + 1) / 2 + 1 + UPD_RED - 1) / UPD_RED; }

size_t update_ws_doubles(long I, long R) {
    return (size_t)update_blocks(I, R) * (size_t)(R * (R + 1) / 2 + 1) + (size_t)update_red_blocks(R) + 2;
}

int factor_update(const UpdateArgs &a, cudaStream_t s) {
    if (!a.Vinv && a.R <= GR_RMAX) {
        // Gram only: 32 rows a CTA (at most max_blocks CTAs), then the reduce
        int nb = std::min<long>(update_blocks(a.I, a.R), (a.I + 31) / 32);
        if (a.max_blocks > 0) nb = std::min(nb, a.max_blocks);
        nb = std::max(nb, 1);
        const int rpc = (int)((a.I + nb - 1) / nb);
        const size_t smem = sizeof(float) * GR_ROWS * (4 * ((a.R + 3) / 4) + 4);
        k_gram_rows<<<nb, GR_NT, smem, s>>>(a, rpc);
        CUD_CHECK_LAUNCH("factor_update gram");
        k_update_reduce<<<(unsigned)update_red_blocks(a.R), UPD_RED, 0, s>>>(a, nb);
        CUD_CHECK_LAUNCH("factor_update reduce");
        return CUD_OK;
    }
    const int nb = a.max_blocks > 0 ? std::min(update_blocks(a.I, a.R), a.max_blocks) : update_blocks(a.I, a.R);
    const size_t smem = sizeof(double) * SU_LD * a.R + sizeof(float) * (UPD_RB * a.R + 2) +
                        (a.R <= UPD_STAGE_V ? sizeof(double) * a.R * a.R : 0);
    // NACC = ceil(R (R + 1) / 2 / NT) triangle entries per thread and
    // UPT = ceil(16 / (NT / R)) rows per thread of U = M V^-1, at the largest R
    if (a.R <= 32) k_update_rows<256, 3, 2><<<nb, 256, smem, s>>>(a);
    else if (a.R <= 64) k_update_rows<256, 9, 4><<<nb, 256, smem, s>>>(a);
    else if (a.R <= 160) k_update_rows<512, 26, 6><<<nb, 512, smem, s>>>(a);
    else return CUD_ERR_UNSUPPORTED;
    CUD_CHECK_LAUNCH("factor_update rows");
    k_update_reduce<<<(unsigned)update_red_blocks(a.R), UPD_RED, 0, s>>>(a, nb);
    CUD_CHECK_LAUNCH("factor_update reduce");
    return CUD_OK;
}

int factor_gram_f64(const double *U, long I, long R, double *G, cudaStream_t s) {
    dim3 grid((unsigned)((R + 15) / 16), (unsigned)((R + 15) / 16));
    k_factor_gram<double><<<grid, 256, 0, s>>>(U, I, R, G);
    CUD_CHECK_LAUNCH("factor_gram_f64");
    return CUD_OK;
}

int factor_gram(const float *U, long I, long R, double *G, cudaStream_t s) {
    if (R > 160) {
        dim3 grid((unsigned)((R + 15) / 16), (unsigned)((R + 15) / 16));
        k_factor_gram<float><<<grid, 256, 0, s>>>(U, I, R, G);
        CUD_CHECK_LAUNCH("factor_gram");
        return CUD_OK;
    }
    int st;
    size_t nd = update_ws_doubles(I, R);
    char *w = (char *)scratch(kSlotGram, 256 + sizeof(double) * nd, &st);
    if (!w) return st;
    UpdateArgs a;
    a.M = U;
    a.I = I;
    a.R = (int)R;
    a.G_out = G;
    a.counter = reinterpret_cast<unsigned *>(w);
    a.gpart = reinterpret_cast<double *>(w + 256);
    CUD_CHECK(cudaMemsetAsync(w, 0, 256, s));
    return factor_update(a, s);
}

int normal_inverse_prepare() {
    static std::atomic<bool> attr_set[64];  // per device; zero-initialised
    int dev = 0;
    CUD_CHECK(cudaGetDevice(&dev));
    if (dev >= 0 && dev < 64 && !attr_set[dev].load(std::memory_order_acquire)) {
        CUD_CHECK(cudaFuncSetAttribute(k_normal_inverse, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)(sizeof(double) * 160 * 160)));
        attr_set[dev].store(true, std::memory_order_release);
    }
    return CUD_OK;
}

int normal_inverse(const NormalArgs &a, cudaStream_t s) {
    size_t smem = sizeof(double) * (size_t)a.R * a.R;
    if (a.R > 160) return CUD_ERR_UNSUPPORTED;
    if (a.R <= 16) {
        k_normal_inverse_warp<16><<<1, 32, sizeof(double) * 32 * 32, s>>>(a);
        CUD_CHECK_LAUNCH("normal_inverse");
        return CUD_OK;
    }
    if (a.R <= NI_SMALL_R) {
        k_normal_inverse_small<<<1, 256, smem, s>>>(a);
        CUD_CHECK_LAUNCH("normal_inverse");
        return CUD_OK;
    }
    int st = normal_inverse_prepare();
    if (st) return st;
    k_normal_inverse<<<1, dim3(32, 16), smem, s>>>(a);
    CUD_CHECK_LAUNCH("normal_inverse");
    return CUD_OK;
}

int apply_inverse(const float *M, const double *Vinv, long I, long R, float *U, cudaStream_t s) {
    size_t smem = (R <= 64) ? sizeof(double) * R * R : 0;
    k_apply_inverse<<<blocks_for(I * R, 256, 148L * 4), 256, smem, s>>>(M, Vinv, I, R, U);
    CUD_CHECK_LAUNCH("apply_inverse");
    return CUD_OK;
}

int fit_eval(const FitArgs &a, cudaStream_t s) {
    k_fit<<<1, 256, 0, s>>>(a);
    CUD_CHECK_LAUNCH("fit_eval");
    return CUD_OK;
}

}  // namespace cud
