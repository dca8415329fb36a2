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

}  // namespace

size_t mttkrp_simt_ws_bytes(int order, const long *dims, int mode, long R, int round) {
    ModeView v = mode_view(order, dims, mode);
    SimtPlan p = simt_plan(v, mode, R, round);
    return sizeof(float) * (size_t)p.splits * R * v.Q;
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
    if (rtiles > 65535 || qtiles * splits > 0x7fffffffL) return CUD_ERR_UNSUPPORTED;
    dim3 grid((unsigned)(qtiles * splits), (unsigned)rtiles);
    if (kind == 0) k_mttkrp_simt<0, T><<<grid, NT, 0, s>>>(a);
    else if (kind == 1) k_mttkrp_simt<1, T><<<grid, NT, 0, s>>>(a);
    else k_mttkrp_simt<2, T><<<grid, NT, 0, s>>>(a);
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
