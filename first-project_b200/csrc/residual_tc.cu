// Exact CP residual on the tensor cores: ||X - [[U_0, ..., U_{N-1}]]||^2 and
// ||X||^2 in one pass over X, the reconstruction formed in TMEM by
// tcgen05 BF16x3 products (order >= 3, R <= 64).
//
// The reference measures the model's error by reconstructing the tensor and
// taking the norm of the difference (src/rse.cu:4-15 with gencp,
// src/rse.cu:17-29).  With X viewed as I_0 x I_1 x K (K = the product of the
// slower modes, index k), the reconstruction's frontal slice k is
//     Xh[:, :, k] = (U_0 * diag(c_k)) U_1^T,   c_k[r] = prod_{m >= 2} U_m[digit_m(k), r],
// a 128-row tile of which is one MMA per 128 columns of U_1 with contraction
// length R.  A CTA owns one 128-row tile of mode 0 and a contiguous range of
// k; per k:
//   * four builder warps form A' = U_0 rows times c_k (each thread holds its
//     row of U_0 in registers), split it into BF16 hi and lo and store both
//     in TMEM (double-buffered over k);
//   * one thread issues, per 128-column chunk of U_1, the three products
//     A'_hi B_hi + A'_hi B_lo + A'_lo B_hi into a TMEM accumulator
//     (double-buffered over chunks); B = U_1 split into hi and lo once per CTA
//     and resident in shared memory in the canonical K-major layout;
//   * one thread streams the matching X tiles (128 rows x 32 columns,
//     TMA, a ring as deep as the shared memory beside U_1 allows, 2-12
//     tiles) -- X is read exactly once;
//   * eight epilogue warps (two per TMEM lane quarter, each half of the
//     columns) read the accumulator row by row (tcgen05.ld) and the X tile
//     from shared memory and add (x - xh)^2 (per tile in FP32) and x^2 (in
//     FP64) into FP64 totals, four independent sums each.
// Rows past I_0 and columns past I_1 are zero in A' and B and in the X tiles
// (the TMA fill), so they add nothing.  Per-CTA totals are summed in a fixed
// order by k_sum_pairs (deterministic).  Every wait is bounded; a CTA that
// gives up writes NaN totals, so the result cannot pass for a value.
//
// Accuracy: the BF16x3 products carry about 16 significand bits per
// operand, so each reconstructed entry is within a few 1e-6 of its FP32
// value (relative); the residual of a model at fit 0.99 then moves by about
// 1e-6 relative, far inside the 1e-4 fit margins it is used for.
#include <atomic>
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>
#include "kernels.cuh"
#include "tc_ptx.cuh"

namespace cud {

namespace {

constexpr int RT_ROWS = 128;    // mode-0 rows per tile (TMEM lanes, MMA M)
constexpr int RT_NJ = 128;      // U_1 rows per MMA (N) = one accumulator buffer
constexpr int RT_XJ = 32;       // U_1 rows (X columns) per X tile
// Deepest X ring; the shared memory left after U_1 bounds it (6 tiles at
// 512^3 R64).  Rings of 5, 8 and 12 tiles timed the same: the kernel is
// bound by its per-slice chain (A' build -> MMA -> epilogue), not by the
// bytes in flight.
constexpr int RT_XSMAX = 12;
constexpr int RT_THREADS = 448; // warp 0 TMA, 1 MMA, 2-5 builders, 6-13 epilogue
constexpr int RT_EPI = 8;       // epilogue warps: two per TMEM lane quarter, 16 of every 32 columns each
constexpr uint32_t RT_XBYTES = RT_ROWS * RT_XJ * 4;
constexpr int RT_RMAX = 64;
constexpr int RT_BMAX = 128 * 1024;  // U_1 hi + lo in shared memory
constexpr uint32_t RT_TMEM_COLS = 512;  // 2 accumulators x 128, then 2 A' buffers x 64

struct RtArgs {
    const float *U0, *U1;
    KrFactors f;          // U_2 .. U_{N-1}, fastest first (the digits of k)
    long I0, I1, K;
    int R, Rpad, nq;      // rank, rank rounded to 16, chunks of 128 U_1 rows
    int cpt;              // CTAs per row tile (they split k)
    int xs;               // X ring depth
    int need_x2;          // also sum x^2 (the caller may know ||X||^2 already)
    double *part;         // [grid][2]
};

struct RtCtrl {
    uint64_t x_full[RT_XSMAX], x_empty[RT_XSMAX];
    uint64_t a_full[2], a_free[2], d_full[2], d_free[2], done;
    uint32_t tmem_base;
    int abort;
    const float *fU[kMaxOrder];
    long frows[kMaxOrder];
    float cvec[4][RT_RMAX];
    double red[2][RT_EPI];
};
constexpr size_t RT_CTRL_BYTES = (sizeof(RtCtrl) + 1023) & ~size_t(1023);

__host__ __device__ constexpr size_t rt_b_bytes(int Rpad, int nq) { return (size_t)nq * RT_NJ * Rpad * 2; }
__host__ __device__ constexpr size_t rt_smem_bytes(int Rpad, int nq, int xs) {
    return 1024 + RT_CTRL_BYTES + 2 * rt_b_bytes(Rpad, nq) + (size_t)xs * RT_XBYTES;
}
constexpr size_t RT_SMEM_MAX = 232448;
// the deepest X ring that fits beside U_1
int rt_ring(int Rpad, int nq) {
    int xs = RT_XSMAX;
    while (xs > 2 && rt_smem_bytes(Rpad, nq, xs) > RT_SMEM_MAX) xs--;
    return xs;
}

__device__ __forceinline__ uint32_t rt_pack_bf16(float a, float b) {
    __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<uint32_t *>(&h);
}

// hi = bf16(x), lo = bf16(x - hi), for a pair of values (one 32-bit word each)
__device__ __forceinline__ void rt_split_pair(float a, float b, uint32_t &hi, uint32_t &lo) {
    __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    const float2 f = __bfloat1622float2(h);
    hi = *reinterpret_cast<uint32_t *>(&h);
    lo = rt_pack_bf16(a - f.x, b - f.y);
}

__global__ void __launch_bounds__(RT_THREADS, 1)
    k_residual_tc(const __grid_constant__ CUtensorMap tmap, RtArgs a) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t *base = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    RtCtrl &sm = *reinterpret_cast<RtCtrl *>(base);
    uint8_t *b_hi = base + RT_CTRL_BYTES;
    uint8_t *b_lo = b_hi + rt_b_bytes(a.Rpad, a.nq);
    uint8_t *xring = b_lo + rt_b_bytes(a.Rpad, a.nq);  // 1024-aligned: the B sizes are multiples of 4 KB
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int tile = blockIdx.x / a.cpt, zc = blockIdx.x % a.cpt;
    const long i0 = (long)tile * RT_ROWS;
    const long k_beg = a.K * zc / a.cpt, k_end = a.K * (zc + 1) / a.cpt;
    const long nk = k_end - k_beg;
    const long nchunks = nk * a.nq;
    volatile int *abort = &sm.abort;

    if (threadIdx.x == 0) {
        for (int i = 0; i < RT_XSMAX; i++) {
            ptx::mbar_init(&sm.x_full[i], 1);
            ptx::mbar_init(&sm.x_empty[i], RT_EPI);  // the epilogue warps
        }
        for (int b = 0; b < 2; b++) {
            ptx::mbar_init(&sm.a_full[b], 4);   // the builder warps
            ptx::mbar_init(&sm.a_free[b], 1);   // tcgen05.commit
            ptx::mbar_init(&sm.d_full[b], 1);   // tcgen05.commit
            ptx::mbar_init(&sm.d_free[b], RT_EPI);   // the epilogue warps
        }
        ptx::mbar_init(&sm.done, 1);
        sm.abort = 0;
#pragma unroll
        for (int m = 0; m < kMaxOrder; m++) {  // constant indices: no local copy of the parameter
            sm.fU[m] = m < a.f.n ? a.f.U[m] : nullptr;
            sm.frows[m] = m < a.f.n ? a.f.rows[m] : 1;
        }
        ptx::fence_mbar_init();
        ptx::prefetch_tmap(&tmap);
    }
    if (warp == 0) {
        ptx::tmem_alloc(&sm.tmem_base, RT_TMEM_COLS);
        ptx::tmem_relinquish();
    }
    // B = U_1 in BF16 hi and lo, K-major, no swizzle: chunk q holds rows
    // 128 q .. 128 q + 127; the 8 values r = 8 kc .. 8 kc + 7 of local row jr
    // form one 16-byte word at jr * 16 + kc * 2048 (descriptor: 8-row groups
    // 128 B apart, K chunks 2048 B apart)
    {
        const int kcs = a.Rpad / 8;
        const long items = (long)a.nq * RT_NJ * kcs;
        for (long it = threadIdx.x; it < items; it += RT_THREADS) {
            const int jr = (int)(it % RT_NJ);
            const long rest = it / RT_NJ;
            const int kc = (int)(rest % kcs), q = (int)(rest / kcs);
            const long j = (long)q * RT_NJ + jr;
            float v[8];
#pragma unroll
            for (int e = 0; e < 8; e++) {
                const int r = 8 * kc + e;
                v[e] = (j < a.I1 && r < a.R) ? a.U1[j + a.I1 * r] : 0.f;
            }
            uint4 h, l;
            rt_split_pair(v[0], v[1], h.x, l.x);
            rt_split_pair(v[2], v[3], h.y, l.y);
            rt_split_pair(v[4], v[5], h.z, l.z);
            rt_split_pair(v[6], v[7], h.w, l.w);
            const size_t off = (size_t)q * RT_NJ * a.Rpad * 2 + (size_t)jr * 16 + (size_t)kc * RT_NJ * 16;
            *reinterpret_cast<uint4 *>(b_hi + off) = h;
            *reinterpret_cast<uint4 *>(b_lo + off) = l;
        }
    }
    ptx::fence_proxy_async_smem();  // B, written by threads, is read by the tensor cores
    ptx::tc_fence_before();
    __syncthreads();
    ptx::tc_fence_after();
    const uint32_t tbase = sm.tmem_base;
    const uint32_t lane_off = (uint32_t)((warp & 3) * 32) << 16;  // a warp's TMEM lane quarter
    const int row = (warp & 3) * 32 + lane;                       // tile row of builder / epilogue threads

    long issued_x = 0;
    double s_res = 0.0, s_x = 0.0;
    if (warp == 0) {
        // ------------------------------------------------------------ TMA producer
        if (lane == 0) {
            long xi = 0;
            for (long kl = 0; kl < nk && !*abort; kl++) {
                for (int q = 0; q < a.nq && !*abort; q++) {
                    for (int s = 0; s < RT_NJ / RT_XJ; s++, xi++) {
                        const int slot = (int)(xi % a.xs);
                        const long use = xi / a.xs;
                        if (use > 0 && !ptx::mbar_wait(&sm.x_empty[slot], (uint32_t)((use - 1) & 1), abort)) break;
                        ptx::mbar_arrive_expect_tx(&sm.x_full[slot], RT_XBYTES);
                        ptx::tma_load_3d(xring + (size_t)slot * RT_XBYTES, &tmap, &sm.x_full[slot], (int)i0,
                                         q * RT_NJ + s * RT_XJ, (int)(k_beg + kl));
                        issued_x = xi + 1;
                    }
                }
            }
        }
    } else if (warp == 1) {
        // ------------------------------------------------------------ MMA issuer
        if (lane == 0) {
            const uint32_t idesc = ptx::idesc_f16(1, RT_ROWS, RT_NJ);
            const uint32_t lbo = RT_NJ * 16;  // K chunks of 8 values
            const size_t chunk_bytes = (size_t)RT_NJ * a.Rpad * 2;
            long ci = 0;
            for (long kl = 0; kl < nk && !*abort; kl++) {
                const int b = (int)(kl & 1);
                if (!ptx::mbar_wait(&sm.a_full[b], (uint32_t)((kl >> 1) & 1), abort)) break;
                ptx::tc_fence_after();
                const uint32_t a_hi = tbase + 2u * RT_NJ + (uint32_t)b * 64u, a_lo = a_hi + 32u;
                for (int q = 0; q < a.nq; q++, ci++) {
                    const int db = (int)(ci & 1);
                    if (ci >= 2 && !ptx::mbar_wait(&sm.d_free[db], (uint32_t)(((ci >> 1) - 1) & 1), abort)) break;
                    ptx::tc_fence_after();
                    const uint32_t d = tbase + (uint32_t)db * RT_NJ;
                    const uint32_t bh = ptx::smem_addr(b_hi + (size_t)q * chunk_bytes);
                    const uint32_t bl = ptx::smem_addr(b_lo + (size_t)q * chunk_bytes);
                    for (int kk = 0; kk < a.Rpad / 16; kk++) {
                        const uint64_t dh = ptx::smem_desc_kmajor_noswizzle(bh + 2u * kk * lbo, lbo, 128);
                        const uint64_t dl = ptx::smem_desc_kmajor_noswizzle(bl + 2u * kk * lbo, lbo, 128);
                        ptx::mma_ts_f16(d, a_hi + 8u * kk, dh, idesc, kk > 0 ? 1u : 0u);
                        ptx::mma_ts_f16(d, a_hi + 8u * kk, dl, idesc, 1u);
                        ptx::mma_ts_f16(d, a_lo + 8u * kk, dh, idesc, 1u);
                    }
                    ptx::mma_commit(&sm.d_full[db]);
                }
                ptx::mma_commit(&sm.a_free[b]);
            }
            // every MMA issued has completed before the accumulators go away
            ptx::mma_commit(&sm.done);
            for (long it = 0; it < 40000 && !ptx::mbar_try_wait_hint(&sm.done, 0, 100000u); it++) {
            }
        }
    } else if (warp < 6) {
        // ------------------------------------------------------------ A' builders
        const long i = i0 + row;
        float u0[RT_RMAX];
#pragma unroll
        for (int r = 0; r < RT_RMAX; r++) u0[r] = (i < a.I0 && r < a.R) ? a.U0[i + a.I0 * r] : 0.f;
        float *cv = sm.cvec[warp - 2];
        for (long kl = 0; kl < nk && !*abort; kl++) {
            const int b = (int)(kl & 1);
            // c_k for r = lane, lane + 32: the slower factors' rows of k
            const long k = k_beg + kl;
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int r = lane + 32 * h;
                float c = 0.f;
                if (r < a.R) {
                    c = 1.f;
                    long rem = k;
                    for (int f = 0; f < a.f.n; f++) {
                        const long d = rem % sm.frows[f];
                        rem /= sm.frows[f];
                        c *= sm.fU[f][d + sm.frows[f] * r];
                    }
                }
                cv[r] = c;
            }
            __syncwarp();
            if (kl >= 2 && !*abort) ptx::mbar_wait(&sm.a_free[b], (uint32_t)(((kl >> 1) - 1) & 1), abort);
            const bool ok = __all_sync(0xffffffffu, *abort == 0);  // warp-uniform exit before tcgen05.st
            if (!ok) break;
            ptx::tc_fence_after();
            const uint32_t a_hi = tbase + lane_off + 2u * RT_NJ + (uint32_t)b * 64u, a_lo = a_hi + 32u;
#pragma unroll
            for (int g = 0; g < RT_RMAX / 16; g++) {
                if (g < a.Rpad / 16) {
                    uint32_t hi[8], lo[8];
#pragma unroll
                    for (int c = 0; c < 8; c++) {
                        const int r = 16 * g + 2 * c;
                        rt_split_pair(u0[r] * cv[r], u0[r + 1] * cv[r + 1], hi[c], lo[c]);
                    }
                    ptx::tmem_st8(a_hi + 8u * g, hi);
                    ptx::tmem_st8(a_lo + 8u * g, lo);
                }
            }
            ptx::tmem_wait_st();
            ptx::tc_fence_before();
            __syncwarp();
            if (lane == 0) ptx::mbar_arrive(&sm.a_full[b]);
        }
    } else {
        // ------------------------------------------------------------ epilogue
        const int hcol = ((warp - 6) >> 2) * (RT_XJ / 2);  // this warp's 16 columns of each tile
        double sr[4] = {0.0, 0.0, 0.0, 0.0}, sx[4] = {0.0, 0.0, 0.0, 0.0};
        long ci = 0, xi = 0;
        for (; ci < nchunks && !*abort; ci++) {
            const int db = (int)(ci & 1);
            if (!*abort) ptx::mbar_wait(&sm.d_full[db], (uint32_t)((ci >> 1) & 1), abort);
            const bool ok = __all_sync(0xffffffffu, *abort == 0);  // warp-uniform exit before tcgen05.ld
            if (!ok) break;
            ptx::tc_fence_after();
            // the chunk's accumulator columns of this warp, four loads and one wait
            uint32_t v[RT_NJ / RT_XJ][16];
#pragma unroll
            for (int s = 0; s < RT_NJ / RT_XJ; s++)
                ptx::tmem_ld16(tbase + lane_off + (uint32_t)db * RT_NJ + (uint32_t)(s * RT_XJ + hcol), v[s]);
            ptx::tmem_wait_ld();
            bool stop = false;
#pragma unroll
            for (int s = 0; s < RT_NJ / RT_XJ; s++, xi++) {
                const int slot = (int)(xi % a.xs);
                if (!*abort) ptx::mbar_wait(&sm.x_full[slot], (uint32_t)((xi / a.xs) & 1), abort);
                if (!__all_sync(0xffffffffu, *abort == 0)) {
                    stop = true;
                    break;
                }
                const float *xs = reinterpret_cast<const float *>(xring + (size_t)slot * RT_XBYTES) + hcol * RT_ROWS;
                // (x - xh)^2 per tile in FP32; x^2 in FP64 (exact products of
                // FP32 values), so ||X||^2 matches an FP64 sum; four chains
                // each.  (FP32 tile sums for x^2 too measured 10 % faster at
                // 512^3 R64 -- 0.159 against 0.176 ms -- for a 1e-9 error.)
                float fr[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
                for (int jj = 0; jj < RT_XJ / 2; jj++) {
                    const float x = xs[jj * RT_ROWS + row];
                    const float dv = x - __uint_as_float(v[s][jj]);
                    fr[jj & 3] = fmaf(dv, dv, fr[jj & 3]);
                    if (a.need_x2) sx[jj & 3] = fma((double)x, (double)x, sx[jj & 3]);
                }
#pragma unroll
                for (int c = 0; c < 4; c++) sr[c] += (double)fr[c];
                __syncwarp();
                if (lane == 0) ptx::mbar_arrive(&sm.x_empty[slot]);
            }
            if (stop) break;
            ptx::tc_fence_before();
            __syncwarp();
            if (lane == 0) ptx::mbar_arrive(&sm.d_free[db]);
        }
        s_res = (sr[0] + sr[1]) + (sr[2] + sr[3]);
        s_x = (sx[0] + sx[1]) + (sx[2] + sx[3]);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            s_res += __shfl_xor_sync(0xffffffffu, s_res, o);
            s_x += __shfl_xor_sync(0xffffffffu, s_x, o);
        }
        if (lane == 0) {
            sm.red[0][warp - 6] = s_res;
            sm.red[1][warp - 6] = s_x;
        }
    }

    // ------------------------------------------------------------ teardown
    if (threadIdx.x == 0 && *abort) {
        // copies still in flight land before the CTA's shared memory is released
        for (long x = (issued_x > a.xs ? issued_x - a.xs : 0); x < issued_x; x++) {
            const uint32_t par = (uint32_t)((x / a.xs) & 1);
            for (long it = 0; it < 20000 && !ptx::mbar_try_wait_hint(&sm.x_full[x % a.xs], par, 100000u); it++) {
            }
        }
    }
    ptx::tc_fence_before();
    __syncthreads();
    ptx::tc_fence_after();
    if (warp == 0) ptx::tmem_dealloc(tbase, RT_TMEM_COLS);
    if (threadIdx.x == 0) {
        double r = 0.0, x = 0.0;
        for (int w = 0; w < RT_EPI; w++) {
            r += sm.red[0][w];
            x += sm.red[1][w];
        }
        if (*abort) r = x = __longlong_as_double(0x7ff8000000000000LL);
        a.part[2 * blockIdx.x] = r;
        a.part[2 * blockIdx.x + 1] = x;
    }
}

PFN_cuTensorMapEncodeTiled_v12000 rt_encode_fn() {
    // resolved once (thread-safe static initialisation)
    static const PFN_cuTensorMapEncodeTiled_v12000 fn = []() -> PFN_cuTensorMapEncodeTiled_v12000 {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        return nullptr;
    }();
    return fn;
}

}  // namespace

// The tensor-core path applies to order >= 3, R <= 64, I_0 a multiple of 4
// (16-byte row strides for the TMA), U_1 resident in shared memory (its hi
// and lo at most 128 KB), and a slower-mode index within 32 bits.
bool residual_tc_plan(int order, const long *dims, long R, int *grid) {
    if (order < 3 || R <= 0 || R > RT_RMAX || dims[0] % 4 != 0) return false;
    const int Rpad = (int)((R + 15) / 16 * 16);
    const long nq = (dims[1] + RT_NJ - 1) / RT_NJ;
    if (2 * rt_b_bytes(Rpad, (int)nq) > (size_t)RT_BMAX) return false;
    if (rt_smem_bytes(Rpad, (int)nq, 2) > RT_SMEM_MAX) return false;
    long K = 1;
    for (int m = 2; m < order; m++) K *= dims[m];
    if (K > 0x7fffffffL || dims[0] > 0x7fffffffL || dims[1] > 0x7fffffffL) return false;
    const long tiles = (dims[0] + RT_ROWS - 1) / RT_ROWS;
    const long cpt = std::max(1L, std::min(K, (long)kNumSMs / tiles));
    if (grid) *grid = (int)(tiles * cpt);
    return true;
}

int residual_tc(const float *X, int order, const long *dims, const float *const *U, long R, double *part,
                double *out2, cudaStream_t s, bool need_x2) {
    int grid = 0;
    if (!residual_tc_plan(order, dims, R, &grid)) return CUD_ERR_UNSUPPORTED;
    if ((reinterpret_cast<uintptr_t>(X) & 15) != 0) return CUD_ERR_UNSUPPORTED;
    auto encode = rt_encode_fn();
    if (!encode) return CUD_ERR_UNSUPPORTED;
    long K = 1;
    for (int m = 2; m < order; m++) K *= dims[m];
    CUtensorMap tmap;
    cuuint64_t gdim[3] = {(cuuint64_t)dims[0], (cuuint64_t)dims[1], (cuuint64_t)K};
    cuuint64_t gstride[2] = {(cuuint64_t)dims[0] * 4, (cuuint64_t)dims[0] * dims[1] * 4};
    cuuint32_t box[3] = {RT_ROWS, RT_XJ, 1};
    cuuint32_t estr[3] = {1, 1, 1};
    if (encode(&tmap, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float *>(X), gdim, gstride, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return CUD_ERR_UNSUPPORTED;
    RtArgs a;
    a.U0 = U[0];
    a.U1 = U[1];
    a.f.n = 0;
    for (int m = 2; m < order; m++) {
        a.f.U[a.f.n] = U[m];
        a.f.rows[a.f.n] = dims[m];
        a.f.n++;
    }
    a.I0 = dims[0];
    a.I1 = dims[1];
    a.K = K;
    a.R = (int)R;
    a.Rpad = (int)((R + 15) / 16 * 16);
    a.nq = (int)((dims[1] + RT_NJ - 1) / RT_NJ);
    const long tiles = (dims[0] + RT_ROWS - 1) / RT_ROWS;
    a.cpt = (int)(grid / tiles);
    a.part = part;
    a.need_x2 = need_x2 ? 1 : 0;
    a.xs = rt_ring(a.Rpad, a.nq);
    const size_t smem = rt_smem_bytes(a.Rpad, a.nq, a.xs);
    static std::atomic<bool> attr[64];  // per device; zero-initialised
    int dev = 0;
    CUD_CHECK(cudaGetDevice(&dev));
    if (dev >= 0 && dev < 64 && !attr[dev].load(std::memory_order_acquire)) {
        CUD_CHECK(cudaFuncSetAttribute(k_residual_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)RT_SMEM_MAX));
        attr[dev].store(true, std::memory_order_release);
    }
    const int pk = prof_begin(s);
    k_residual_tc<<<(unsigned)grid, RT_THREADS, smem, s>>>(tmap, a);
    prof_end(pk, s);
    CUD_CHECK_LAUNCH("cp_residual tc");
    return sum_pairs(part, grid, out2, s);
}

}  // namespace cud
