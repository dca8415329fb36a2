// MTTKRP on CUDA cores in FP32 (the "plain FP32" path and the fallback for
// shapes the tensor-core path does not take), and the same kernel in FP64
// for the FP64 CP-ALS.  Native layout, no unfolding,
// no materialised Khatri-Rao matrix.
//
// Around mode n the tensor is a (P, Q, S) array (P = prod of dims before n,
// Q = dims[n], S = prod after).  With L the Khatri-Rao product of the factors
// before n and Rt that of the factors after n,
//     M[q, r] = sum_s Rt[s, r] * sum_p X[p + P q + P Q s] * L[p, r].
// Mode 0 (P = 1) is one GEMM  X(Q x S) * Rt(S x R);  other modes are, for
// each s, a GEMM  X_s^T (Q x P) * L(P x R)  scaled by the row Rt[s, :].  The
// KR rows (B operand) are generated per 16-deep slice into shared memory; the
// contraction is split across CTAs and the FP32 partials reduced in FP64.
#include <type_traits>

#include "kernels.cuh"

namespace cud {

namespace {

constexpr int BQ = 64, BR = 64, BK = 16, NT = 256;

// The same kernel serves FP32 (KrFactors) and FP64 (KrFactors64) data.
struct KrFactors64 {
    int n = 0;
    const double *U[kMaxOrder];
    long rows[kMaxOrder];
};
template <typename T> struct KrOf;
template <> struct KrOf<float> { using type = KrFactors; };
template <> struct KrOf<double> { using type = KrFactors64; };

template <typename T>
struct SimtArgs {
    const T *X;
    long P, Q, S, R;
    int round;        // 0: operands as given; 1: round X and KR rows to FP16; 2: to BF16 (FP32 only)
    typename KrOf<T>::type gen;    // factors generating the B operand (fastest first)
    typename KrOf<T>::type outer;  // factors generating the per-s scale (P > 1), fastest first
    long ksteps;      // BK-steps per s
    long steps;       // total steps = (P > 1 ? S : 1) * ksteps
    long chunk;       // steps per split
    T *part;          // [split][R][Q]
};

template <typename KR>
__device__ __forceinline__ auto kr_value(const KR &f, const long *idx, long r) {
    using V = std::remove_cv_t<std::remove_pointer_t<std::remove_reference_t<decltype(f.U[0])>>>;
    V v = 1;
    for (int i = 0; i < f.n; i++) v *= f.U[i][idx[i] + r * f.rows[i]];
    return v;
}

__device__ __forceinline__ float round_to(float v, int mode) {
    if (mode == 1) return __half2float(__float2half_rn(v));
    if (mode == 2) return __bfloat162float(__float2bfloat16_rn(v));
    return v;
}
__device__ __forceinline__ double round_to(double v, int) { return v; }

__device__ __forceinline__ float fma_t(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double fma_t(double a, double b, double c) { return fma(a, b, c); }

__device__ __forceinline__ void load4(const float *p, float *x) {
    const float4 v = *reinterpret_cast<const float4 *>(p);
    x[0] = v.x; x[1] = v.y; x[2] = v.z; x[3] = v.w;
}
__device__ __forceinline__ void load4(const double *p, double *x) {
    const double2 a = *reinterpret_cast<const double2 *>(p), b = *reinterpret_cast<const double2 *>(p + 2);
    x[0] = a.x; x[1] = a.y; x[2] = b.x; x[3] = b.y;
}

template <typename KR>
__device__ __forceinline__ void decompose(const KR &f, long lin, long *idx) {
    for (int i = 0; i < f.n; i++) {
        long d = f.rows[i];
        idx[i] = lin % d;
        lin /= d;
    }
}

// kKind 0: mode 0, A(q, k) = X[q + Q k], B = KR of the factors after it.
// kKind 1: other modes, factored -- per s a GEMM over p with B = KR of the
//          factors before the mode, scaled by the KR row of those after it.
// kKind 2: other modes, flattened contraction k = p + P s with B = KR of all
//          other factors formed (and rounded) as one product, as the
//          reference's public mttkrp() does before its FP16 GEMM.
template <int kKind, typename T>
__global__ void __launch_bounds__(NT) k_mttkrp_simt(SimtArgs<T> a) {
    constexpr bool kModeZero = (kKind != 1);
    __shared__ __align__(16) T As[BK][BQ];
    __shared__ __align__(16) T Bs[BK][BR];
    __shared__ long kidx[BK][kMaxOrder];

    const int t = threadIdx.x;
    const long qtiles = (a.Q + BQ - 1) / BQ;
    const long q0 = (blockIdx.x % qtiles) * BQ;
    const long z = blockIdx.x / qtiles;
    const long r0 = (long)blockIdx.y * BR;
    const long sbeg = z * a.chunk;
    const long send = min(a.steps, sbeg + a.chunk);
    const int tx = t & 15, ty = t >> 4;

    T acc[4][4], tot[4][4];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) { acc[i][j] = 0; tot[i][j] = 0; }

    const long K = (kKind == 0) ? a.S : (kKind == 1) ? a.P : a.P * a.S;
    long cur_s = -1;

    for (long st = sbeg; st < send; st++) {
        long s = kModeZero ? 0 : st / a.ksteps;
        long k0 = (st % a.ksteps) * BK;
        if (!kModeZero && s != cur_s) {
            if (cur_s >= 0) {
                // flush: tot += acc * Rt[cur_s, r]
                long oidx[kMaxOrder];
                decompose(a.outer, cur_s, oidx);
#pragma unroll
                for (int j = 0; j < 4; j++) {
                    long r = r0 + ty * 4 + j;
                    T w = (r < a.R) ? kr_value(a.outer, oidx, r) : T(0);
#pragma unroll
                    for (int i = 0; i < 4; i++) { tot[i][j] = fma_t(acc[i][j], w, tot[i][j]); acc[i][j] = 0; }
                }
            }
            cur_s = s;
        }
        // index table for the BK generated KR rows of this slice
        if (t < BK) {
            long k = k0 + t;
            if (k < K) decompose(a.gen, k, kidx[t]);
        }
        // A tile: As[kk][qq] = X(q, k)
#pragma unroll
        for (int i = 0; i < 4; i++) {
            int e = t + NT * i;
            int qq, kk;
            if (kModeZero) { qq = e % BQ; kk = e / BQ; }
            else { kk = e % BK; qq = e / BK; }
            long q = q0 + qq, k = k0 + kk;
            T v = 0;
            if (q < a.Q && k < K) {
                if (kKind == 0) v = a.X[q + a.Q * k];
                else if (kKind == 1) v = a.X[k + a.P * (q + a.Q * s)];
                else v = a.X[(k % a.P) + a.P * (q + a.Q * (k / a.P))];
                v = round_to(v, a.round);
            }
            As[kk][qq] = v;
        }
        __syncthreads();
        // B tile: Bs[kk][rr] = KR(k, r)
#pragma unroll
        for (int i = 0; i < 4; i++) {
            int e = t + NT * i;
            int rr = e % BR, kk = e / BR;
            long r = r0 + rr, k = k0 + kk;
            T v = 0;
            if (r < a.R && k < K) v = round_to(kr_value(a.gen, kidx[kk], r), a.round);
            Bs[kk][rr] = v;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < BK; kk++) {
            T x[4], y[4];
            load4(&As[kk][tx * 4], x);
            load4(&Bs[kk][ty * 4], y);
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) acc[i][j] = fma_t(x[i], y[j], acc[i][j]);
        }
        __syncthreads();
    }
    if (kModeZero) {
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
            for (int j = 0; j < 4; j++) tot[i][j] = acc[i][j];
    } else if (cur_s >= 0) {
        long oidx[kMaxOrder];
        decompose(a.outer, cur_s, oidx);
#pragma unroll
        for (int j = 0; j < 4; j++) {
            long r = r0 + ty * 4 + j;
            T w = (r < a.R) ? kr_value(a.outer, oidx, r) : T(0);
#pragma unroll
            for (int i = 0; i < 4; i++) tot[i][j] = fma_t(acc[i][j], w, tot[i][j]);
        }
    }
    T *P = a.part + z * a.R * a.Q;
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) {
            long q = q0 + tx * 4 + i, r = r0 + ty * 4 + j;
            if (q < a.Q && r < a.R) P[q + a.Q * r] = tot[i][j];
        }
}

// ---------------------------------------------------------------------------
// Plain FP32 on the FFMA pipe, for the shapes that allow it (the fastest
// generating factor U0 has a multiple of FK rows, the tensor is 16-byte
// aligned and its contiguous index a multiple of 4).  An SGEMM-style kernel:
//   * a CTA owns FQ = 128 rows q and BR (32 or 64) ranks, 128 threads, each
//     accumulating an 8 x BR/8 register tile (8 q values x BR/8 ranks);
//   * the contraction runs in FK = 32-deep stages, double-buffered in shared
//     memory with register staging: stage i+1's global loads are in flight
//     while stage i is multiplied, one barrier per stage;
//   * A = the 128 x 32 tile of X in its native layout, 16-byte loads; for
//     mode 0 it is stored as is ([k][q], q contiguous), for the other modes
//     (p contiguous) it is transposed on the way into shared memory; the
//     tile's columns are XOR-swizzled in 4-float groups (column q of row k
//     lives at q ^ (k & 28)), which makes the transposing stores
//     conflict-free and keeps the 16-byte reads aligned;
//   * B = the stage's 32 Khatri-Rao rows.  A stage covers 32 consecutive rows
//     of U0 while the other factors contribute one constant row c, so B is
//     U0's rows (pre-packed once per call into a row-major copy, ranks
//     contiguous) times c, formed in FP32 as the reference's Khatri-Rao
//     matrix is (one rounding per entry).  Each thread stores the same 4
//     ranks every stage and computes c for them itself at a block boundary,
//     so the constant row needs no shared memory and no extra barrier.
// Partials [split][r][q] are summed in FP64 by k_sum_partials.
constexpr int FQ = 128, FK = 32, FT = 128;

struct FfmaArgs {
    const float *X;
    long P, Q, S;
    int R, kind;        // kind 0: mode 0 (q contiguous); 1: other modes (p contiguous)
    const float *U0p;   // U0 row-major, rows0 x Rp (zero beyond R)
    int rows0, Rp;
    KrFactors gen;      // generating factors, fastest first (gen.U[0] = U0, read through U0p)
    KrFactors outer;    // kind 1: the factors after the mode (per-s scale), fastest first
    long psteps;        // kind 1: stages per s
    long steps, chunk;  // total stages, stages per split
    float *part;        // [split][R][Q]
};

__device__ __forceinline__ int swz(int q, int k) { return q ^ (k & 28); }

// The constant Khatri-Rao row at stage st for ranks r..r+3: the product of
// the non-fastest generating factors' rows (digits of the block index) and,
// for kind 1, the outer factors' rows (digits of s).
__device__ __forceinline__ float4 ffma_const_row(const FfmaArgs &a, long st, int r) {
    uint32_t blk, s = 0;
    if (a.kind == 0) {
        blk = (uint32_t)((st * FK) / a.rows0);
    } else {
        s = (uint32_t)(st / a.psteps);
        blk = (uint32_t)(((st - (long)s * a.psteps) * FK) / a.rows0);
    }
    float4 c = make_float4(1.f, 1.f, 1.f, 1.f);
    auto mul = [&](const float *U, long rows, uint32_t row) {
        const float *p = U + row;
        if (r + 0 < a.R) c.x *= __ldg(p + (long)(r + 0) * rows); else c.x = 0.f;
        if (r + 1 < a.R) c.y *= __ldg(p + (long)(r + 1) * rows); else c.y = 0.f;
        if (r + 2 < a.R) c.z *= __ldg(p + (long)(r + 2) * rows); else c.z = 0.f;
        if (r + 3 < a.R) c.w *= __ldg(p + (long)(r + 3) * rows); else c.w = 0.f;
    };
    for (int f = 1; f < a.gen.n; f++) {
        const uint32_t d = (uint32_t)a.gen.rows[f], qd = blk / d;
        mul(a.gen.U[f], a.gen.rows[f], blk - qd * d);
        blk = qd;
    }
    if (a.kind == 1) {
        for (int f = 0; f < a.outer.n; f++) {
            const uint32_t d = (uint32_t)a.outer.rows[f], qd = s / d;
            mul(a.outer.U[f], a.outer.rows[f], s - qd * d);
            s = qd;
        }
    }
    return c;
}

template <int BR>
__global__ void __launch_bounds__(FT, 2) k_mttkrp_ffma(FfmaArgs a) {
    constexpr int TR = BR / 8;          // ranks per thread
    constexpr int NB = BR * FK / 4 / FT;  // B float4 per thread per stage (4 or 2)
    __shared__ __align__(16) float As[2][FK][FQ];
    __shared__ __align__(16) float Bs[2][FK][BR];

    const int t = threadIdx.x;
    const int tq = t >> 3, tr = t & 7;  // 16 x 8 threads
    const long qtiles = (a.Q + FQ - 1) / FQ;
    const long q0 = (blockIdx.x % qtiles) * FQ;
    const long z = blockIdx.x / qtiles;
    const int r0 = blockIdx.y * BR;
    const long sbeg = z * a.chunk;
    const long send = min(a.steps, sbeg + a.chunk);

    // this thread's B float4 slots: rank group rv (fixed), rows kb + i * kstep
    const int rv = t % (BR / 4);
    const int kb = t / (BR / 4);
    constexpr int kstep = FT / (BR / 4);

    float acc[8][TR];
#pragma unroll
    for (int i = 0; i < 8; i++)
#pragma unroll
        for (int j = 0; j < TR; j++) acc[i][j] = 0.f;

    float4 ra[8], rb[NB], cr = make_float4(0.f, 0.f, 0.f, 0.f);
    const int blk_stages = a.rows0 / FK;

    auto load = [&](long st) {
        long i0;  // row of U0 at the stage's first contraction index
        if (a.kind == 0) {
            const long k0 = st * FK;
            i0 = k0 % a.rows0;
#pragma unroll
            for (int i = 0; i < 8; i++) {
                const int e = t + FT * i, k = e >> 5, qv = e & 31;
                const long q = q0 + 4 * qv;
                ra[i] = (q < a.Q) ? __ldg(reinterpret_cast<const float4 *>(a.X + q + a.Q * (k0 + k)))
                                  : make_float4(0.f, 0.f, 0.f, 0.f);
            }
        } else {
            const long s = st / a.psteps;
            const long p0 = (st - s * a.psteps) * FK;
            i0 = p0 % a.rows0;
            const float *base = a.X + p0 + a.P * (a.Q * s);
#pragma unroll
            for (int i = 0; i < 8; i++) {
                const int e = t + FT * i, pv = e & 7, q = e >> 3;
                ra[i] = (q0 + q < a.Q)
                            ? __ldg(reinterpret_cast<const float4 *>(base + 4 * pv + a.P * (q0 + q)))
                            : make_float4(0.f, 0.f, 0.f, 0.f);
            }
        }
        const float *ub = a.U0p + (size_t)i0 * a.Rp + r0 + 4 * rv;
#pragma unroll
        for (int i = 0; i < NB; i++) rb[i] = __ldg(reinterpret_cast<const float4 *>(ub + (size_t)(kb + kstep * i) * a.Rp));
        if (st == sbeg || (st % blk_stages) == 0) cr = ffma_const_row(a, st, r0 + 4 * rv);
    };
    auto store = [&](int buf) {
        if (a.kind == 0) {
#pragma unroll
            for (int i = 0; i < 8; i++) {
                const int e = t + FT * i, k = e >> 5, qv = e & 31;
                *reinterpret_cast<float4 *>(&As[buf][k][swz(4 * qv, k)]) = ra[i];
            }
        } else {
#pragma unroll
            for (int i = 0; i < 8; i++) {
                const int e = t + FT * i, pv = e & 7, q = e >> 3;
                const int k = 4 * pv;
                As[buf][k + 0][swz(q, k + 0)] = ra[i].x;
                As[buf][k + 1][swz(q, k + 1)] = ra[i].y;
                As[buf][k + 2][swz(q, k + 2)] = ra[i].z;
                As[buf][k + 3][swz(q, k + 3)] = ra[i].w;
            }
        }
#pragma unroll
        for (int i = 0; i < NB; i++) {
            float4 v = rb[i];
            v.x *= cr.x; v.y *= cr.y; v.z *= cr.z; v.w *= cr.w;
            *reinterpret_cast<float4 *>(&Bs[buf][kb + kstep * i][4 * rv]) = v;
        }
    };

    if (sbeg < send) {
        load(sbeg);
        store(0);
        __syncthreads();
    }
    for (long st = sbeg; st < send; st++) {
        const int cur = (int)((st - sbeg) & 1);
        const bool more = st + 1 < send;
        if (more) load(st + 1);
#pragma unroll 4
        for (int k = 0; k < FK; k++) {
            const float4 x0 = *reinterpret_cast<const float4 *>(&As[cur][k][swz(8 * tq, k)]);
            const float4 x1 = *reinterpret_cast<const float4 *>(&As[cur][k][swz(8 * tq + 4, k)]);
            const float x[8] = {x0.x, x0.y, x0.z, x0.w, x1.x, x1.y, x1.z, x1.w};
            float y[TR];
            const float4 y0 = *reinterpret_cast<const float4 *>(&Bs[cur][k][TR * tr]);
            y[0] = y0.x; y[1] = y0.y; y[2] = y0.z; y[3] = y0.w;
            if constexpr (TR == 8) {
                const float4 y1 = *reinterpret_cast<const float4 *>(&Bs[cur][k][TR * tr + 4]);
                y[4] = y1.x; y[5] = y1.y; y[6] = y1.z; y[7] = y1.w;
            }
#pragma unroll
            for (int i = 0; i < 8; i++)
#pragma unroll
                for (int j = 0; j < TR; j++) acc[i][j] = fmaf(x[i], y[j], acc[i][j]);
        }
        if (more) store(cur ^ 1);
        __syncthreads();
    }
    float *P = a.part + z * (long)a.R * a.Q;
#pragma unroll
    for (int j = 0; j < TR; j++) {
        const int r = r0 + TR * tr + j;
        if (r >= a.R) continue;
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const long q = q0 + 8 * tq + i;
            if (q < a.Q) P[q + a.Q * r] = acc[i][j];
        }
    }
}

// U0 (rows x R, column-major) -> row-major rows x Rp, zero beyond R.
__global__ void k_pack_rows(const float *__restrict__ U, long rows, int R, int Rp, float *__restrict__ out) {
    const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (e >= rows * Rp) return;
    const long i = e / Rp;
    const int r = (int)(e - i * Rp);
    out[e] = (r < R) ? U[i + rows * r] : 0.f;
}

template <typename T>
__global__ void k_sum_partials(const T *__restrict__ part, int splits, long n, T *__restrict__ out) {
    long tid = blockIdx.x * (long)blockDim.x + threadIdx.x;
    long stride = (long)gridDim.x * blockDim.x;
    for (long e = tid; e < n; e += stride) {
        double s = 0.0;
        for (int z = 0; z < splits; z++) s += (double)part[(long)z * n + e];
        out[e] = (T)s;
    }
}

}  // namespace

namespace {

struct SimtPlan {
    int kind;
    long ksteps, steps, chunk, splits, qtiles, rtiles;
};

SimtPlan simt_plan(const ModeView &v, int mode, long R, int round) {
    SimtPlan p;
    p.kind = (mode == 0) ? 0 : (round ? 2 : 1);
    long K = (p.kind == 0) ? v.S : (p.kind == 1) ? v.P : v.P * v.S;
    p.ksteps = (K + BK - 1) / BK;
    p.steps = (p.kind == 1 ? v.S : 1) * p.ksteps;
    p.qtiles = (v.Q + BQ - 1) / BQ;
    p.rtiles = (R + BR - 1) / BR;
    long tiles = p.qtiles * p.rtiles;
    long want = (3L * kNumSMs + tiles - 1) / tiles;
    long splits = std::max(1L, std::min(want, p.steps));
    p.chunk = (p.steps + splits - 1) / splits;
    p.splits = (p.steps + p.chunk - 1) / p.chunk;
    return p;
}

// Launch plan of the FFMA kernel; ok = false when the shape does not allow it
// (the fastest generating factor's rows not a multiple of FK, mode 0 rows not
// a multiple of 4, or extents beyond its 32-bit digit arithmetic).
struct FfmaPlan {
    bool ok = false;
    int BR = 64, kind = 0, rows0 = 0, Rp = 0;
    long qtiles = 0, rtiles = 0, psteps = 0, steps = 0, chunk = 0, splits = 0;
    size_t part_bytes = 0, pack_bytes = 0;
};

FfmaPlan ffma_plan(int order, const long *dims, int mode, long R) {
    FfmaPlan p;
    if (order < 2 || R <= 0) return p;
    ModeView v = mode_view(order, dims, mode);
    p.kind = (mode == 0) ? 0 : 1;
    const long rows0 = (mode == 0) ? dims[1] : dims[0];
    if (rows0 % FK != 0 || rows0 > 0x7fffffffL) return p;
    if (p.kind == 0 && v.Q % 4 != 0) return p;
    if (v.Q > 0x7fffffffL || v.S > 0xffffffffL || v.P > 0x7fffffffL || R > 0x7fffffffL) return p;
    for (int m = 0; m < order; m++)
        if (dims[m] > 0x7fffffffL) return p;
    p.rows0 = (int)rows0;
    p.BR = (R <= 32) ? 32 : 64;
    p.rtiles = (R + p.BR - 1) / p.BR;
    if (p.rtiles > 65535) return p;
    p.Rp = (int)(p.rtiles * p.BR);
    p.qtiles = (v.Q + FQ - 1) / FQ;
    p.psteps = (p.kind == 1) ? v.P / FK : 0;
    p.steps = (p.kind == 1) ? v.S * p.psteps : v.S / FK;
    if (p.steps * (long)FK / rows0 > 0xffffffffL) return p;  // block index in 32 bits
    const long tiles = p.qtiles * p.rtiles;
    const long want = (2L * kNumSMs + tiles - 1) / tiles;  // two CTAs per SM
    p.splits = std::max(1L, std::min(want, p.steps));
    p.chunk = (p.steps + p.splits - 1) / p.splits;
    p.splits = (p.steps + p.chunk - 1) / p.chunk;
    if (p.qtiles * p.splits > 0x7fffffffL) return p;
    p.part_bytes = (sizeof(float) * (size_t)p.splits * R * v.Q + 255) & ~size_t(255);
    p.pack_bytes = sizeof(float) * (size_t)rows0 * p.Rp;
    p.ok = true;
    return p;
}

}  // namespace

size_t mttkrp_simt_ws_bytes(int order, const long *dims, int mode, long R, int round) {
    ModeView v = mode_view(order, dims, mode);
    SimtPlan p = simt_plan(v, mode, R, round);
    size_t b = sizeof(float) * (size_t)p.splits * R * v.Q;
    if (round == 0) {
        FfmaPlan f = ffma_plan(order, dims, mode, R);
        if (f.ok) b = std::max(b, f.part_bytes + f.pack_bytes);
    }
    return b;
}

namespace {

template <typename T>
int mttkrp_simt_impl(const T *X, int order, const long *dims, const T *const *U, int mode, long R, T *out,
                     int round, void *ws, cudaStream_t s) {
    ModeView v = mode_view(order, dims, mode);
    SimtPlan p = simt_plan(v, mode, R, round);
    SimtArgs<T> a;
    a.X = X;
    a.P = v.P; a.Q = v.Q; a.S = v.S; a.R = R;
    a.round = round;
    const int kind = p.kind;
    bool mode_zero = (kind != 1);
    // Generated (B-operand) factors: for mode 0 the factors after it; for
    // other modes the factors before it, with those after it as the per-s
    // scale.  Both lists run fastest mode first.
    a.gen.n = 0;
    a.outer.n = 0;
    for (int m = 0; m < order; m++) {
        if (m == mode) continue;
        auto &f = (mode_zero || m < mode) ? a.gen : a.outer;
        f.U[f.n] = U[m];
        f.rows[f.n] = dims[m];
        f.n++;
    }
    a.ksteps = p.ksteps;
    a.steps = p.steps;
    a.chunk = p.chunk;
    long splits = p.splits, qtiles = p.qtiles, rtiles = p.rtiles;
    a.part = (T *)ws;
    if (!a.part) return CUD_ERR_INVALID_ARGUMENT;
    if constexpr (std::is_same<T, float>::value) {
        // plain FP32: the FFMA kernel where the shape and alignment allow
        const FfmaPlan f = (round == 0) ? ffma_plan(order, dims, mode, R) : FfmaPlan();
        if (f.ok && (reinterpret_cast<uintptr_t>(X) & 15) == 0) {
            FfmaArgs fa;
            fa.X = X;
            fa.P = v.P; fa.Q = v.Q; fa.S = v.S;
            fa.R = (int)R;
            fa.kind = f.kind;
            fa.rows0 = f.rows0;
            fa.Rp = f.Rp;
            fa.gen = a.gen;
            fa.outer = a.outer;
            fa.psteps = f.psteps;
            fa.steps = f.steps;
            fa.chunk = f.chunk;
            fa.part = reinterpret_cast<float *>(ws);
            float *packed = reinterpret_cast<float *>(static_cast<char *>(ws) + f.part_bytes);
            fa.U0p = packed;
            const long items = (long)f.rows0 * f.Rp;
            k_pack_rows<<<(unsigned)((items + 255) / 256), 256, 0, s>>>(a.gen.U[0], f.rows0, (int)R, f.Rp, packed);
            CUD_CHECK_LAUNCH("mttkrp_ffma pack");
            dim3 grid((unsigned)(f.qtiles * f.splits), (unsigned)f.rtiles);
            const int pk = prof_begin(s);
            if (f.BR == 32) k_mttkrp_ffma<32><<<grid, FT, 0, s>>>(fa);
            else k_mttkrp_ffma<64><<<grid, FT, 0, s>>>(fa);
            prof_end(pk, s);
            CUD_CHECK_LAUNCH("mttkrp_ffma");
            k_sum_partials<float><<<blocks_for(R * v.Q, 256), 256, 0, s>>>(fa.part, (int)f.splits, R * v.Q, out);
            CUD_CHECK_LAUNCH("mttkrp_ffma reduce");
            return CUD_OK;
        }
    }
    if (rtiles > 65535 || qtiles * splits > 0x7fffffffL) return CUD_ERR_UNSUPPORTED;
    dim3 grid((unsigned)(qtiles * splits), (unsigned)rtiles);
    const int pk = prof_begin(s);
    if (kind == 0) k_mttkrp_simt<0, T><<<grid, NT, 0, s>>>(a);
    else if (kind == 1) k_mttkrp_simt<1, T><<<grid, NT, 0, s>>>(a);
    else k_mttkrp_simt<2, T><<<grid, NT, 0, s>>>(a);
    prof_end(pk, s);
    CUD_CHECK_LAUNCH("mttkrp_simt");
    k_sum_partials<T><<<blocks_for(R * v.Q, 256), 256, 0, s>>>(a.part, (int)splits, R * v.Q, out);
    CUD_CHECK_LAUNCH("mttkrp_simt reduce");
    return CUD_OK;
}

}  // namespace

int mttkrp_simt_rounded(const float *X, int order, const long *dims, const float *const *U,
                        int mode, long R, float *out, int round, void *ws, cudaStream_t s) {
    return mttkrp_simt_impl<float>(X, order, dims, U, mode, R, out, round, ws, s);
}

size_t mttkrp_simt_f64_ws_bytes(int order, const long *dims, int mode, long R) {
    return 2 * mttkrp_simt_ws_bytes(order, dims, mode, R, 0);
}

int mttkrp_simt_f64(const double *X, int order, const long *dims, const double *const *U, int mode, long R,
                    double *out, void *ws, cudaStream_t s) {
    return mttkrp_simt_impl<double>(X, order, dims, U, mode, R, out, 0, ws, s);
}

}  // namespace cud
