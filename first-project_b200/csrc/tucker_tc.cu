// Tucker HOSVD / HOOI on the tensor cores: the unfolding Grams and the TTM
// chains are BF16 GEMMs with FP32 accumulation (gemm_tc.cu); the Gram
// eigenproblems stay in FP64 (eig.cu).  Same algorithm and factor convention
// as tucker.cu (src/tucker_hosvd.cu:3-103, src/tucker4_hosvd.cu:3-141,
// decomposition/GPU/normal/tucker/tucker_hooi.cu:3-218); the reference runs
// its Grams as FP32 SGEMMs and its TTMs as FP16 GemmEx (src/ttm.cu:4-47).
//
// Layout trick: the GEMM wants its contraction index contiguous.  A TTM over
// the fastest mode of a column-major tensor is such a GEMM as it stands, and
// writing its output with the new rank index slowest -- (d_1, ..., d_N-1, r_0)
// -- makes the next mode the fastest one.  So the HOSVD core is N GEMMs over a
// BF16 copy of X with no transposes, and each HOOI projection is one rotating
// copy of X followed by N-1 such GEMMs.  Gram operands X_(n) (rows = mode n,
// the other modes contiguous) come from one convert-and-unfold kernel.
//
// Precision: BF16 -> Grams from one BF16 GEMM and single-term BF16 TTM
// chains.  BF16X3 / DEFAULT -> FP32-level accuracy throughout: Grams from
// the three-term split (hi hi + hi lo + lo hi, the last term the transpose
// of the middle one), and every TTM step three-term as well, T U ~ Th Uh +
// Th Ul + Tl Uh (one GEMM of Th against [Uh | Ul], one of Tl against Uh,
// FP32 accumulation), with the chain's intermediates kept as hi/lo pairs
// and the HOOI projection's Gram three-term.
#include <cuda_bf16.h>

#include "kernels.cuh"

namespace cud {

namespace {

__device__ __forceinline__ void put_split(__nv_bfloat16 *hi, __nv_bfloat16 *lo, long o, float x) {
    const __nv_bfloat16 h = __float2bfloat16_rn(x);
    hi[o] = h;
    if (lo) lo[o] = __float2bfloat16_rn(x - __bfloat162float(h));
}

// View X as (Q, S) with q fastest (a (P = 1, Q, S) mode view): out[q*S + s],
// 32 x 32 tiles through shared memory (coalesced on both sides).
__global__ void __launch_bounds__(256) k_unfold_t(const float *__restrict__ X, long Q, long S,
                                                  __nv_bfloat16 *hi, __nv_bfloat16 *lo) {
    __shared__ float tile[32][33];
    const long tq = (Q + 31) / 32, ts = (S + 31) / 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    for (long t = blockIdx.x; t < tq * ts; t += gridDim.x) {
        const long q0 = (t % tq) * 32, s0 = (t / tq) * 32;
        __syncthreads();
        for (int k = ty; k < 32; k += 8) {
            const long q = q0 + tx, s = s0 + k;
            tile[k][tx] = (q < Q && s < S) ? X[q + Q * s] : 0.f;
        }
        __syncthreads();
        for (int k = ty; k < 32; k += 8) {
            const long q = q0 + k, s = s0 + tx;
            if (q < Q && s < S) put_split(hi, lo, q * S + s, tile[tx][k]);
        }
    }
}

// The same (Q, S) transpose for Q % 4 == 0, S % 8 == 0 and 16-byte aligned
// buffers: 64 x 64 tiles, 16-byte loads (a warp reads two 256-byte column
// runs) and 16-byte stores of 8 BF16 values (lane pairs fill 32-byte
// sectors of 16 output rows).  Row stride 68 keeps the float4 shared stores
// conflict-free; the column reads are at most 2-way.
__global__ void __launch_bounds__(256) k_unfold_t64(const float *__restrict__ X, long Q, long S,
                                                    __nv_bfloat16 *__restrict__ hi, __nv_bfloat16 *__restrict__ lo) {
    __shared__ __align__(16) float tile[64][68];
    const long tq = (Q + 63) / 64, ts = (S + 63) / 64;
    const int t = threadIdx.x;
    for (long tt = blockIdx.x; tt < tq * ts; tt += gridDim.x) {
        const long q0 = (tt % tq) * 64, s0 = (tt / tq) * 64;
        const int q4 = (t & 15) * 4;
        const bool qin = q0 + q4 < Q;
        float4 v[4];
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const int sl = (t >> 4) + 16 * i;
            v[i] = (qin && s0 + sl < S) ? __ldcs(reinterpret_cast<const float4 *>(X + q0 + q4 + Q * (s0 + sl)))
                                        : make_float4(0.f, 0.f, 0.f, 0.f);
        }
        __syncthreads();
#pragma unroll
        for (int i = 0; i < 4; i++) *reinterpret_cast<float4 *>(&tile[(t >> 4) + 16 * i][q4]) = v[i];
        __syncthreads();
#pragma unroll
        for (int i = 0; i < 2; i++) {
            const int u = t + 256 * i, p = u >> 1;
            const int ql = p & 63, c = 2 * (p >> 6) + (u & 1);
            const long q = q0 + ql, sb = s0 + 8 * c;
            if (q >= Q || sb >= S) continue;
            uint32_t h[4], l[4];
#pragma unroll
            for (int j = 0; j < 4; j++) {
                const float a = tile[8 * c + 2 * j][ql], b = tile[8 * c + 2 * j + 1][ql];
                const __nv_bfloat162 hh = __floats2bfloat162_rn(a, b);
                const float2 hf = __bfloat1622float2(hh);
                const __nv_bfloat162 ll = __floats2bfloat162_rn(a - hf.x, b - hf.y);
                h[j] = *reinterpret_cast<const uint32_t *>(&hh);
                l[j] = *reinterpret_cast<const uint32_t *>(&ll);
            }
            *reinterpret_cast<uint4 *>(hi + q * S + sb) = make_uint4(h[0], h[1], h[2], h[3]);
            if (lo) *reinterpret_cast<uint4 *>(lo + q * S + sb) = make_uint4(l[0], l[1], l[2], l[3]);
        }
    }
}

// View X as (P, Q, S), P > 1: out[q*(P*S) + p + P*s] = X[p + P*q + P*Q*s];
// each (q, s) pair is a run of P contiguous values on both sides.
__global__ void __launch_bounds__(256) k_unfold_runs(const float *__restrict__ X, long P, long Q, long S,
                                                     __nv_bfloat16 *hi, __nv_bfloat16 *lo) {
    const long rows = Q * S;
    for (long qs = blockIdx.y; qs < rows; qs += gridDim.y) {
        const long q = qs / S, s = qs - q * S;
        const float *src = X + P * q + P * Q * s;
        const long o = q * (P * S) + P * s;
        for (long p = blockIdx.x * 256L + threadIdx.x; p < P; p += (long)gridDim.x * 256L)
            put_split(hi, lo, o + p, src[p]);
    }
}

// A BF16 (Q, S) matrix with q fastest -> rows of q with s contiguous, row
// stride Sp >= S, the pad columns S..Sp-1 zero.
__global__ void __launch_bounds__(256) k_transpose_bf16(const __nv_bfloat16 *__restrict__ X, long Q, long S,
                                                        long Sp, __nv_bfloat16 *__restrict__ out) {
    __shared__ __nv_bfloat16 tile[32][34];
    const long tq = (Q + 31) / 32, ts = (Sp + 31) / 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    for (long t = blockIdx.x; t < tq * ts; t += gridDim.x) {
        const long q0 = (t % tq) * 32, s0 = (t / tq) * 32;
        __syncthreads();
        for (int k = ty; k < 32; k += 8) {
            const long q = q0 + tx, s = s0 + k;
            tile[k][tx] = (q < Q && s < S) ? X[q + Q * s] : __float2bfloat16_rn(0.f);
        }
        __syncthreads();
        for (int k = ty; k < 32; k += 8) {
            const long q = q0 + k, s = s0 + tx;
            if (q < Q && s < Sp) out[q * Sp + s] = tile[tx][k];
        }
    }
}

__global__ void k_f32_to_f64(const float *__restrict__ a, double *__restrict__ b, long n) {
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x)
        b[e] = (double)a[e];
}

__global__ void k_take_top_f32(const double *__restrict__ V, long n, long r, float *__restrict__ U) {
    const long total = n * r;
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
        const long i = e % n, j = e / n;
        U[e] = (float)V[i + n * (n - r + j)];
    }
}

__global__ void k_to_bf16(const float *__restrict__ a, __nv_bfloat16 *__restrict__ b, long n) {
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x)
        b[e] = __float2bfloat16_rn(a[e]);
}

unsigned gfor(long n) { return (unsigned)std::min<long>((n + 255) / 256, 16L * kNumSMs); }

// a (n floats) -> hi (bf16(a)) and lo (bf16(a - hi)).
__global__ void k_split_bf16(const float *__restrict__ a, __nv_bfloat16 *__restrict__ hi,
                             __nv_bfloat16 *__restrict__ lo, long n) {
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x)
        put_split(hi, lo, e, a[e]);
}

// Three-term TTM finish: v = F2[e] + F2[e + n] + F3[e] (Th Uh, Th Ul and
// Tl Uh, each GEMM's plain FP32 output), written as FP32 (fout) or split
// into the next step's hi/lo operands.
__global__ void k_ttm3_finish(const float *__restrict__ F2, const float *__restrict__ F3, long n,
                              float *__restrict__ fout, __nv_bfloat16 *__restrict__ hi,
                              __nv_bfloat16 *__restrict__ lo) {
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) {
        const float v = (F2[e] + F2[e + n]) + F3[e];
        if (fout) fout[e] = v;
        else put_split(hi, lo, e, v);
    }
}

// An FP32 (Q, S) matrix with q fastest -> rows of q with s contiguous, row
// stride Sp >= S, split into BF16 hi and lo; pad columns S..Sp-1 zero.
__global__ void __launch_bounds__(256) k_transpose_split(const float *__restrict__ X, long Q, long S, long Sp,
                                                         __nv_bfloat16 *__restrict__ hi,
                                                         __nv_bfloat16 *__restrict__ lo) {
    __shared__ float tile[32][33];
    const long tq = (Q + 31) / 32, ts = (Sp + 31) / 32;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    for (long t = blockIdx.x; t < tq * ts; t += gridDim.x) {
        const long q0 = (t % tq) * 32, s0 = (t / tq) * 32;
        __syncthreads();
        for (int k = ty; k < 32; k += 8) {
            const long q = q0 + tx, s = s0 + k;
            tile[k][tx] = (q < Q && s < S) ? X[q + Q * s] : 0.f;
        }
        __syncthreads();
        for (int k = ty; k < 32; k += 8) {
            const long q = q0 + k, s = s0 + tx;
            if (q < Q && s < Sp) put_split(hi, lo, q * Sp + s, tile[tx][k]);
        }
    }
}

// X viewed as (P, Q, S) -> X_(view) rows of Q, the rest contiguous (BF16).
// Same unfolding for P a multiple of 8, in the source's memory order: item
// (u, c) = 8 consecutive floats c of source row u = q + Q s (two 16-byte
// loads, coalesced), written as 8 BF16 hi (and lo) values to row q, column
// block s of the unfolding (one 16-byte store each).  32-bit index
// arithmetic (the caller checks that the item count fits).
__global__ void __launch_bounds__(256) k_unfold_runs8(const float *__restrict__ X, unsigned P8, unsigned Q,
                                                      unsigned S, unsigned items, __nv_bfloat16 *hi,
                                                      __nv_bfloat16 *lo) {
    const unsigned long P = 8ul * P8;
    for (unsigned it = blockIdx.x * 256u + threadIdx.x; it < items; it += gridDim.x * 256u) {
        const unsigned u = it / P8, c = it - u * P8;
        const unsigned sidx = u / Q, q = u - sidx * Q;
        const float4 *src = reinterpret_cast<const float4 *>(X + (unsigned long)u * P + 8ul * c);
        const float4 a = __ldcs(src), b = __ldcs(src + 1);
        const float v[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
        uint32_t h[4], l[4];
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const __nv_bfloat162 hh = __floats2bfloat162_rn(v[2 * j], v[2 * j + 1]);
            const float2 hf = __bfloat1622float2(hh);
            const __nv_bfloat162 ll = __floats2bfloat162_rn(v[2 * j] - hf.x, v[2 * j + 1] - hf.y);
            h[j] = *reinterpret_cast<const uint32_t *>(&hh);
            l[j] = *reinterpret_cast<const uint32_t *>(&ll);
        }
        const unsigned long o = (unsigned long)q * P * S + (unsigned long)sidx * P + 8ul * c;
        *reinterpret_cast<uint4 *>(hi + o) = make_uint4(h[0], h[1], h[2], h[3]);
        if (lo) *reinterpret_cast<uint4 *>(lo + o) = make_uint4(l[0], l[1], l[2], l[3]);
    }
}

int unfold_bf16(const float *X, long P, long Q, long S, __nv_bfloat16 *hi, __nv_bfloat16 *lo, cudaStream_t s) {
    const long items = P / 8 * Q * S;
    const bool aligned = ((reinterpret_cast<uintptr_t>(X) | reinterpret_cast<uintptr_t>(hi) |
                           reinterpret_cast<uintptr_t>(lo)) & 15) == 0;
    if (P > 1 && P % 8 == 0 && aligned && items < 0xffffffffL && Q < 0xffffffffL && S < 0xffffffffL) {
        const unsigned grid = (unsigned)std::min<long>((items + 255) / 256, 16L * kNumSMs);
        k_unfold_runs8<<<grid, 256, 0, s>>>(X, (unsigned)(P / 8), (unsigned)Q, (unsigned)S, (unsigned)items, hi, lo);
        CUD_CHECK_LAUNCH("unfold_bf16");
        return CUD_OK;
    }
    if (P == 1 && Q % 4 == 0 && S % 8 == 0 && aligned) {
        const long tiles = ((Q + 63) / 64) * ((S + 63) / 64);
        k_unfold_t64<<<(unsigned)std::min<long>(tiles, 8L * kNumSMs), 256, 0, s>>>(X, Q, S, hi, lo);
    } else if (P == 1) {
        const long tiles = ((Q + 31) / 32) * ((S + 31) / 32);
        k_unfold_t<<<(unsigned)std::min<long>(tiles, 16L * kNumSMs), 256, 0, s>>>(X, Q, S, hi, lo);
    } else {
        const unsigned gx = (unsigned)std::min<long>((P + 255) / 256, 64);
        const unsigned gy = (unsigned)std::min<long>(Q * S, 65535);
        k_unfold_runs<<<dim3(gx, gy), 256, 0, s>>>(X, P, Q, S, hi, lo);
    }
    CUD_CHECK_LAUNCH("unfold_bf16");
    return CUD_OK;
}

struct TcWork {
    __nv_bfloat16 *xb = nullptr;       // X in BF16 (rotated as needed), total
    __nv_bfloat16 *uh = nullptr, *ul = nullptr;  // Gram operands, total each
    __nv_bfloat16 *z0 = nullptr, *z1 = nullptr;  // chain intermediates
    __nv_bfloat16 *ub = nullptr;       // a factor in BF16 (three-term: hi then lo, 2 K r)
    __nv_bfloat16 *zl0 = nullptr, *zl1 = nullptr;  // three-term: low parts of the intermediates
    float *f2 = nullptr;               // three-term: FP32 TTM partials, 2 zmax
    float *f3 = nullptr;               // three-term: FP32 partial Tl Uh, zmax
    float *yf = nullptr;               // three-term: the projection Y in FP32, zmax
    float *g32 = nullptr;              // Gram FP32
    double *g64 = nullptr, *W = nullptr, *V = nullptr;
    void *gws = nullptr;               // GEMM workspace
    size_t gws_bytes = 0;
};

int tc_alloc(int order, const long *dims, const long *ranks, bool three, TcWork &w) {
    long total = 1, maxd = 0, maxr = 0;
    for (int m = 0; m < order; m++) {
        total *= dims[m];
        maxd = std::max(maxd, dims[m]);
        maxr = std::max(maxr, ranks[m]);
    }
    // largest chain intermediate: X with one mode reduced to its rank
    long zmax = 0;
    for (int m = 0; m < order; m++) zmax = std::max(zmax, total / dims[m] * ranks[m]);
    // GEMM workspace: the largest of the Gram and TTM shapes used
    size_t gw = 0;
    for (int m = 0; m < order; m++) {
        gw = std::max(gw, gemm_tc_ws_bytes(dims[m], dims[m], total / dims[m]));
        gw = std::max(gw, gemm_tc_ws_bytes(total / dims[m], ranks[m], dims[m]));
        if (three) gw = std::max(gw, gemm_tc_ws_bytes(total / dims[m], 2 * ranks[m], dims[m]));
        long rest = 1;
        for (int q = 0; q < order; q++)
            if (q != m) rest *= ranks[q];
        gw = std::max(gw, gemm_tc_ws_bytes(dims[m], dims[m], (rest + 7) / 8 * 8));
    }
    auto up = [](size_t b) { return (b + 255) & ~size_t(255); };
    size_t off = 0;
    const size_t o_xb = off; off += up(2 * (size_t)total);
    const size_t o_uh = off; off += up(2 * (size_t)total);
    const size_t o_ul = off; off += three ? up(2 * (size_t)total) : 0;
    const size_t o_z0 = off; off += up(2 * (size_t)zmax);
    const size_t o_z1 = off; off += up(2 * (size_t)zmax);
    const size_t o_ub = off; off += up(2 * 2 * (size_t)maxd * maxr);
    const size_t o_zl0 = off; off += three ? up(2 * (size_t)zmax) : 0;
    const size_t o_zl1 = off; off += three ? up(2 * (size_t)zmax) : 0;
    const size_t o_f2 = off; off += three ? up(4 * 2 * (size_t)zmax) : 0;
    const size_t o_yf = off; off += three ? up(4 * (size_t)zmax) : 0;
    const size_t o_f3 = off; off += three ? up(4 * (size_t)zmax) : 0;
    const size_t o_g32 = off; off += up(4 * (size_t)maxd * maxd);
    const size_t o_g64 = off; off += up(8 * (size_t)maxd * maxd);
    const size_t o_W = off; off += up(8 * (size_t)maxd);
    const size_t o_V = off; off += up(8 * (size_t)maxd * maxd);
    const size_t o_gws = off; off += up(gw);
    int st;
    char *p = static_cast<char *>(scratch(kSlotTmp1, off, &st));
    if (!p) return st;
    w.xb = (__nv_bfloat16 *)(p + o_xb);
    w.uh = (__nv_bfloat16 *)(p + o_uh);
    w.ul = three ? (__nv_bfloat16 *)(p + o_ul) : nullptr;
    w.z0 = (__nv_bfloat16 *)(p + o_z0);
    w.z1 = (__nv_bfloat16 *)(p + o_z1);
    w.ub = (__nv_bfloat16 *)(p + o_ub);
    w.zl0 = three ? (__nv_bfloat16 *)(p + o_zl0) : nullptr;
    w.zl1 = three ? (__nv_bfloat16 *)(p + o_zl1) : nullptr;
    w.f2 = three ? (float *)(p + o_f2) : nullptr;
    w.yf = three ? (float *)(p + o_yf) : nullptr;
    w.f3 = three ? (float *)(p + o_f3) : nullptr;
    w.g32 = (float *)(p + o_g32);
    w.g64 = (double *)(p + o_g64);
    w.W = (double *)(p + o_W);
    w.V = (double *)(p + o_V);
    w.gws = p + o_gws;
    w.gws_bytes = gw;
    return CUD_OK;
}

GemmEpi epi_f32(float *out, long ldm, long ldn, int accumulate) {
    GemmEpi e;
    memset(&e, 0, sizeof(e));
    e.alpha = 1.f;
    e.out_f32 = out; e.f32_ldm = ldm; e.f32_ldn = ldn; e.f32_accumulate = accumulate;
    return e;
}

// Gram (I x I, FP64 into w.g64) of the rows of the I x K BF16 operands:
// hi hi^T, plus hi lo^T + lo hi^T when use_lo.
// g64 = HH + P + P^T in FP64 (P = hi lo^T; its transpose is lo hi^T).
__global__ void k_gram_finish(const float *__restrict__ HH, const float *__restrict__ P, long I,
                              double *__restrict__ g64) {
    const long n2 = I * I;
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n2; e += (long)gridDim.x * blockDim.x) {
        const long m = e / I, n = e - m * I;
        g64[e] = (double)HH[e] + (double)P[e] + (double)P[n * I + m];
    }
}

// The Gram of the unfolding in FP64.  BF16x3: hi hi^T + hi lo^T + lo hi^T,
// where the last term is the transpose of the middle one, so two GEMMs
// (one pass less over the operands) and a finishing sum; P goes to w.V,
// which the eigensolver only uses afterwards.
int gram_tc(const TcWork &w, long I, long K, bool use_lo, cudaStream_t s) {
    if (gemm_tc_ws_bytes(I, I, K) > w.gws_bytes) return CUD_ERR_INVALID_ARGUMENT;
    int st = gemm_tc_bf16(w.uh, K, w.uh, K, I, I, K, epi_f32(w.g32, I, 1, 0), w.gws, s);
    if (st) return st;
    if (use_lo && w.ul) {
        float *P = reinterpret_cast<float *>(w.V);
        if ((st = gemm_tc_bf16(w.uh, K, w.ul, K, I, I, K, epi_f32(P, I, 1, 0), w.gws, s))) return st;
        k_gram_finish<<<gfor(I * I), 256, 0, s>>>(w.g32, P, I, w.g64);
    } else {
        k_f32_to_f64<<<gfor(I * I), 256, 0, s>>>(w.g32, w.g64, I * I);
    }
    CUD_CHECK_LAUNCH("gram_tc");
    return CUD_OK;
}

// U (I x r, FP32) = eigenvectors of the r largest eigenvalues of w.g64:
// subspace iteration (fast when the Gram has a gap after its r-th
// eigenvalue), else the full FP64 Jacobi eigensolver.  warm: start the
// subspace iteration from U's current columns.
int top_vectors(const TcWork &w, long I, long r, float *U, cudaStream_t s, bool warm = false) {
    if (subspace_ws_doubles(I, r) <= (size_t)I * I) {
        const int sst = top_eigvecs_subspace(w.g64, I, r, U, w.V, (size_t)I * I, 300, s, warm ? U : nullptr);
        if (sst == CUD_OK) return CUD_OK;
        if (sst != CUD_ERR_NOT_CONVERGED && sst != CUD_ERR_UNSUPPORTED) return sst;
    }
    int st = syev_jacobi(w.g64, I, w.W, w.V, 60, s);
    if (st != CUD_OK && st != CUD_ERR_NOT_CONVERGED) return st;
    k_take_top_f32<<<gfor(I * r), 256, 0, s>>>(w.V, I, r, U);
    CUD_CHECK_LAUNCH("top_vectors");
    return st;
}

// One TTM over the fastest mode: T (K x rest, K fastest, BF16) times U
// (K x r, FP32) -> (rest x r) with r slowest: BF16 into zout, or FP32 into
// fout.  Returns the GEMM status.
int ttm_fast(const TcWork &w, const __nv_bfloat16 *T, long K, long rest, const float *U, long r,
             __nv_bfloat16 *zout, float *fout, cudaStream_t s) {
    if (gemm_tc_ws_bytes(rest, r, K) > w.gws_bytes) return CUD_ERR_INVALID_ARGUMENT;
    k_to_bf16<<<gfor(K * r), 256, 0, s>>>(U, w.ub, K * r);
    CUD_CHECK_LAUNCH("ttm factor bf16");
    GemmEpi e;
    memset(&e, 0, sizeof(e));
    e.alpha = 1.f;
    if (fout) { e.out_f32 = fout; e.f32_ldm = 1; e.f32_ldn = rest; }
    else { e.out_bf16 = zout; e.bf16_ldm = 1; e.bf16_ldn = rest; }
    return gemm_tc_bf16(T, K, w.ub, K, rest, r, K, e, w.gws, s);
}

// Three-term TTM over the fastest mode: (Th + Tl) (K x rest, K fastest) times
// U (K x r, FP32) ~ Th Uh + Th Ul + Tl Uh -> (rest x r), r slowest, as FP32
// into fout or as the hi/lo pair (zh, zl).  With 2 r <= 32 (the skinny GEMM's
// width) Th is read once, against [Uh | Ul]; wider ranks take two GEMMs of
// width r over Th.  Every GEMM writes its own plain FP32 output (the fast
// epilogue) and one pass adds the three terms.
int ttm3_fast(const TcWork &w, const __nv_bfloat16 *Th, const __nv_bfloat16 *Tl, long K, long rest, const float *U,
              long r, __nv_bfloat16 *zh, __nv_bfloat16 *zl, float *fout, cudaStream_t s) {
    if (gemm_tc_ws_bytes(rest, 2 * r, K) > w.gws_bytes) return CUD_ERR_INVALID_ARGUMENT;
    const __nv_bfloat16 *Uh = w.ub, *Ul = w.ub + K * r;
    k_split_bf16<<<gfor(K * r), 256, 0, s>>>(U, w.ub, w.ub + K * r, K * r);
    CUD_CHECK_LAUNCH("ttm3 factor split");
    int st;
    if (2 * r <= 32) {
        if ((st = gemm_tc_bf16(Th, K, Uh, K, rest, 2 * r, K, epi_f32(w.f2, 1, rest, 0), w.gws, s))) return st;
    } else {
        if ((st = gemm_tc_bf16(Th, K, Uh, K, rest, r, K, epi_f32(w.f2, 1, rest, 0), w.gws, s))) return st;
        if ((st = gemm_tc_bf16(Th, K, Ul, K, rest, r, K, epi_f32(w.f2 + rest * r, 1, rest, 0), w.gws, s)))
            return st;
    }
    if ((st = gemm_tc_bf16(Tl, K, Uh, K, rest, r, K, epi_f32(w.f3, 1, rest, 0), w.gws, s))) return st;
    k_ttm3_finish<<<gfor(rest * r), 256, 0, s>>>(w.f2, w.f3, rest * r, fout, zh, zl);
    CUD_CHECK_LAUNCH("ttm3 finish");
    return CUD_OK;
}

// Contracts modes `first`, first+1, ... (cyclically) of T -- laid out with
// mode `first` fastest, cyclic order -- except mode `skip` (or none when
// skip < 0, all `order` modes).  Returns the BF16 buffer holding the result
// (or writes FP32 `final_out` at the last step) and its element count.
int chain(const TcWork &w, const __nv_bfloat16 *T, int order, const long *dims, const long *ranks,
          float *const *U, int first, int skip, float *final_out, const __nv_bfloat16 **res, cudaStream_t s,
          const __nv_bfloat16 *Tlo = nullptr) {
    long cur[2 * kMaxOrder];  // sizes in layout order
    for (int k = 0; k < order; k++) cur[k] = dims[(first + k) % order];
    long total = 1;
    for (int k = 0; k < order; k++) total *= cur[k];
    const int nsteps = (skip < 0) ? order : order - 1;
    const __nv_bfloat16 *src = T;
    for (int step = 0; step < nsteps; step++) {
        const int m = (first + step) % order;  // the fastest mode now
        const long K = cur[step];
        const long rest = total / K;
        const bool last = (step == nsteps - 1);
        __nv_bfloat16 *dst = (step & 1) ? w.z1 : w.z0;
        int st;
        if (Tlo) {
            // three-term: the intermediates carry their low parts along
            __nv_bfloat16 *dlo = (step & 1) ? w.zl1 : w.zl0;
            st = ttm3_fast(w, src, Tlo, K, rest, U[m], ranks[m], dst, dlo, (last && final_out) ? final_out : nullptr,
                           s);
            Tlo = dlo;
        } else {
            st = ttm_fast(w, src, K, rest, U[m], ranks[m], dst, (last && final_out) ? final_out : nullptr, s);
        }
        if (st) return st;
        cur[order + step] = ranks[m];
        total = rest * ranks[m];
        src = dst;
    }
    *res = src;
    return CUD_OK;
}

bool tc_ok(int order, const long *dims, const long *ranks) {
    if (order < 2 || order > kMaxOrder) return false;
    for (int m = 0; m < order; m++)
        if (dims[m] % 8 != 0) return false;  // GEMM leading dimensions
    long total = 1;
    for (int m = 0; m < order; m++) total *= dims[m];
    return total / dims[order - 1] % 8 == 0;
}

}  // namespace

bool tucker_tc_supported(int order, const long *dims, const long *ranks) { return tc_ok(order, dims, ranks); }

// The HOSVD factors of the given modes (U[n] for n in [n0, order)) from BF16
// Gram GEMMs.
int tucker_tc_factors(const float *X, int order, const long *dims, const long *ranks, float *const *U, int n0,
                      bool three, cudaStream_t s, int *worst) {
    TcWork w;
    int st = tc_alloc(order, dims, ranks, three, w);
    if (st) return st;
    long total = 1;
    for (int m = 0; m < order; m++) total *= dims[m];
    for (int n = n0; n < order; n++) {
        long P = 1, S = 1;
        for (int m = 0; m < n; m++) P *= dims[m];
        for (int m = n + 1; m < order; m++) S *= dims[m];
        if ((st = unfold_bf16(X, P, dims[n], S, w.uh, w.ul, s))) return st;
        if ((st = gram_tc(w, dims[n], total / dims[n], three, s))) return st;
        st = top_vectors(w, dims[n], ranks[n], U[n], s);
        if (st == CUD_ERR_NOT_CONVERGED) *worst = st;
        else if (st) return st;
    }
    return CUD_OK;
}

// core = X x_0 U_0^T x_1 ... (ranks in mode order), BF16 TTM chain.
int tucker_tc_core(const float *X, int order, const long *dims, const long *ranks, float *const *U, float *core,
                   bool three, cudaStream_t s) {
    TcWork w;
    int st = tc_alloc(order, dims, ranks, three, w);
    if (st) return st;
    long total = 1;
    for (int m = 0; m < order; m++) total *= dims[m];
    // plain BF16 copy (three-term: hi into xb, lo into ul)
    if ((st = unfold_bf16(X, total, 1, 1, w.xb, three ? w.ul : nullptr, s))) return st;
    const __nv_bfloat16 *res;
    return chain(w, w.xb, order, dims, ranks, U, 0, -1, core, &res, s, three ? w.ul : nullptr);
}

// One HOOI sweep: for each mode n, U_n = top eigenvectors of the Gram of
// Y = X x_{m != n} U_m^T.  The eigensolver starts from the current U_n (the
// previous sweep's, or the HOSVD one), which is already close to the new
// subspace; U_0 is not set before the first sweep (u0_set false).
int tucker_tc_hooi_sweep(const float *X, int order, const long *dims, const long *ranks, float *const *U,
                         bool three, bool u0_set, cudaStream_t s, int *worst) {
    TcWork w;
    int st = tc_alloc(order, dims, ranks, three, w);
    if (st) return st;
    long total = 1;
    for (int m = 0; m < order; m++) total *= dims[m];
    for (int n = 0; n < order; n++) {
        // rotate X so mode n+1 is fastest: (P = prod_{m<=n} d_m) x rest transposed
        long Pn = 1;
        for (int m = 0; m <= n; m++) Pn *= dims[m];
        const long rest = total / Pn;
        const int first = (n + 1) % order;
        // three-term: the low part of X goes to ul (not otherwise used here)
        __nv_bfloat16 *xlo = three ? w.ul : nullptr;
        if (rest == 1) st = unfold_bf16(X, total, 1, 1, w.xb, xlo, s);
        else st = unfold_bf16(X, 1, Pn, rest, w.xb, xlo, s);
        if (st) return st;
        const __nv_bfloat16 *Y;
        if ((st = chain(w, w.xb, order, dims, ranks, U, first, n, three ? w.yf : nullptr, &Y, s, xlo))) return st;
        // Y: mode n fastest, then the other modes' ranks -> rows of mode n
        long R = 1;
        for (int m = 0; m < order; m++)
            if (m != n) R *= ranks[m];
        // Y has mode n fastest: a tiled transpose gives the Gram operand's
        // rows (single-term: Y is already BF16; three-term: Y is FP32 and
        // is split into hi/lo on the way)
        // rows padded to a multiple of 8 (the GEMM's leading-dimension rule)
        const long Rp = (R + 7) / 8 * 8;
        const long tiles = ((dims[n] + 31) / 32) * ((Rp + 31) / 32);
        const unsigned tg = (unsigned)std::min<long>(tiles, 16L * kNumSMs);
        if (three) {
            // Y in FP32 (the chain's last step) -> hi/lo Gram operands; X's
            // low part in ul is no longer needed
            k_transpose_split<<<tg, 256, 0, s>>>(w.yf, dims[n], R, Rp, w.uh, w.ul);
        } else {
            k_transpose_bf16<<<tg, 256, 0, s>>>(Y, dims[n], R, Rp, w.uh);
        }
        CUD_CHECK_LAUNCH("hooi transpose");
        if ((st = gram_tc(w, dims[n], Rp, three, s))) return st;
        st = top_vectors(w, dims[n], ranks[n], U[n], s, n > 0 || u0_set);
        if (st == CUD_ERR_NOT_CONVERGED) *worst = st;
        else if (st) return st;
    }
    return CUD_OK;
}

}  // namespace cud
