// MTTKRP on the 5th-generation tensor cores (tcgen05, sm_100a).
//
// Around mode n the FP32 tensor is a (P, Q, S) array; the result is
// M[q, r] = sum_kappa X(q, kappa) * KR(kappa, r), with kappa running over the
// other modes.  Per CTA: one tile of 128 rows q (the MMA's M) and a
// contiguous range of 32-deep contraction stages, pipelined NST deep between
// four warp roles:
//   * warp 0 (TMA): the 128 x 32 FP32 tile of X, in its native layout, into
//     shared memory (mode 0: rows contiguous, a 2-D box over (q, s); other
//     modes: kappa contiguous, a 3-D box over (p, q, s) with 128-byte
//     swizzle);
//   * warps 2-5 (A converters): each thread reads its row (= its TMEM lane),
//     splits every value into BF16 hi + lo (x = hi + lo + O(2^-16 x)) and
//     stores both into tensor memory as the MMA's A operand -- X crosses
//     shared memory once;
//   * warps 6-7 (KR producers): the stage's 32 Khatri-Rao rows.  The stage's
//     kappa run over 32 consecutive rows of the fastest generating factor
//     while the other factors contribute one constant row, so each thread
//     loads two 128-bit vectors of one factor column (prefetched a stage
//     ahead), scales, splits and stores 16 bytes per operand into the K-major
//     canonical B layout.  They only wait for the slot to be free, so they
//     run up to NST stages ahead of the MMA;
//   * warp 1 (MMA): tcgen05.mma kind::f16, FP32 accumulation in TMEM:
//     D += Xhi*KRhi + Xhi*KRlo + Xlo*KRhi  (BF16X3), or one product (BF16,
//     FP16).
// The tensor core's FP32 accumulation truncates, so long accumulation chains
// drift low; the CTA's stage range is therefore cut into segments of SEG
// stages, each accumulated in its own TMEM buffer (two, alternating), and
// the A converters add each finished segment into the CTA's FP32 partial in
// global memory with round-to-nearest reductions (`red.add`, fire and
// forget; each partial element has one owning thread, so the order of the
// adds is fixed and the result deterministic).  A small second kernel sums the
// partials over the contraction splits in FP64.  The unfolding and the KR
// matrix are never materialised: X is read from HBM exactly once.
//
// Every wait is bounded: an expired wait raises a CTA-wide abort flag, the
// roles drain and the TMEM is freed before the CTA exits, and the kernel's
// error flag is set.
#include <cuda.h>
#include <cudaTypedefs.h>

#include "kernels.cuh"
#include "tc_ptx.cuh"

namespace cud {

namespace {

constexpr int BQ = 128;          // rows per CTA tile (MMA M)
constexpr int BKS = 32;          // contraction depth per stage (two MMA K-steps of 16)
constexpr int NST = 4;           // pipeline stages
#ifndef CUD_TC_SEG
#define CUD_TC_SEG 16
#endif
constexpr int SEG = CUD_TC_SEG;  // stages per TMEM accumulation segment
constexpr int NTHREADS = 256;    // w0 TMA, w1 MMA, w2-5 A converters, w6-7 KR producers
constexpr int NCONV = 128;       // A converter threads
constexpr int NKR = 64;          // KR producer threads
constexpr int X_STAGE_BYTES = BQ * BKS * 4;  // 16 KB
constexpr int RPAD_MAX = 128;

struct TcArgs {
    long P, Q, S, R;
    int Rpad;          // R rounded up to a multiple of 16 (MMA N)
    int kind;          // 0: mode 0 (rows contiguous); 1: other modes (kappa contiguous)
    int prec;          // CUD_PREC_BF16 / FP16 / BF16X3 / DEFAULT
    int fast;          // stages never cross a row block of the fastest generating factor
    uint32_t tmem_cols;
    long psteps;       // stages per s (kind 1) = ceil(P / 32)
    long stages;       // total stages
    long chunk;        // stages per CTA
    long qtiles;
    KrFactors gen;     // kind 0: factors after mode 0; kind 1: factors before the mode
    KrFactors outer;   // kind 1: factors after the mode (one constant row per stage)
    float *part;       // [split][R][Q]
    int *error;        // device flag
};

struct TcCtrl {
    uint64_t full_x[NST], empty_x[NST], full_a[NST], empty_a[NST];
    uint64_t d_full[2], d_free[2], done;
    const float *gU[kMaxOrder];
    const float *oU[kMaxOrder];
    long grows[kMaxOrder], orows[kMaxOrder];
    uint32_t tmem_base;
    int abort;
};

constexpr size_t CTRL_BYTES = (sizeof(TcCtrl) + 1023) & ~size_t(1023);

__host__ __device__ constexpr size_t b_tile_bytes(int Rpad) { return (size_t)Rpad * BKS * 2; }

__host__ __device__ constexpr size_t tc_smem_bytes(int Rpad) {
    return 1024 + CTRL_BYTES + (size_t)NST * X_STAGE_BYTES + (size_t)NST * 2 * b_tile_bytes(Rpad);
}

__device__ __forceinline__ uint32_t pack_bf16(float a, float b) {
    __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<uint32_t *>(&h);
}

__device__ __forceinline__ uint32_t pack_f16(float a, float b) {
    __half2 h = __floats2half2_rn(a, b);
    return *reinterpret_cast<uint32_t *>(&h);
}

// hi/lo BF16 split of a pair: hi = bf16(x), lo = bf16(x - hi).
__device__ __forceinline__ void split_pair(float a, float b, uint32_t &hi, uint32_t &lo) {
    __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    float2 f = __bfloat1622float2(h);
    hi = *reinterpret_cast<uint32_t *>(&h);
    lo = pack_bf16(a - f.x, b - f.y);
}

// B tile (Rpad x 32 16-bit values, K-major, no swizzle): core matrix
// (n/8, k/8) -- 8 rows x 16 bytes -- at (n/8)*128 + (k/8)*Rpad*16, so the
// 8 values k = 8c..8c+7 of row n form one 16-byte chunk at n*16 + c*Rpad*16.
// Descriptor: SBO (8-row groups) = 128 B, LBO (K chunks) = Rpad*16 B.

// The Khatri-Rao values one producer thread makes per stage: KIPT items,
// each (row r, chunk kc) = 8 consecutive kappa of one column r.
template <int KIPT>
struct KrRegs {
    float f[KIPT][8];
    float c[KIPT];
};

// Loads (fast path) or computes (general path) this thread's KR items for
// stage g into registers.  `cache_key` / `cc` memoise the constant row,
// which only changes when the stage crosses a row block of the fastest
// generating factor or (kind 1) a slab.
template <int KIPT>
__device__ __forceinline__ void kr_load(const TcArgs &a, const TcCtrl &sm, long g, int kt,
                                        KrRegs<KIPT> &o, long &cache_key, float (&cc)[KIPT]) {
    long k0, kmax, s;
    if (a.kind == 0) { k0 = g * BKS; kmax = a.S; s = 0; }
    else { s = g / a.psteps; k0 = (g % a.psteps) * BKS; kmax = a.P; }
    const int ng = a.gen.n, no = a.outer.n;
    const long rows0 = sm.grows[0];
    const long rest = k0 / rows0;
    const long i0 = k0 - rest * rows0;
    const long key = rest * 2147483647L + s;
    const bool refresh = (key != cache_key);
    cache_key = key;
#pragma unroll
    for (int it = 0; it < KIPT; it++) {
        const int id = kt + NKR * it;
        const int kc = id & 3;
        const int r = id >> 2;
#pragma unroll
        for (int j = 0; j < 8; j++) o.f[it][j] = 0.f;
        o.c[it] = 0.f;
        if (r >= a.R) continue;
        if (refresh) {
            // the constant row: the digits of s over the outer factors and
            // (fast path) of `rest` over the slower generating factors,
            // recomputed per item so no index array lives in local memory
            float c = 1.f;
            long lin = s;
            for (int f = 0; f < no; f++) {
                const long d = sm.orows[f];
                const long idx = lin % d;
                lin /= d;
                c *= __ldg(sm.oU[f] + idx + r * d);
            }
            if (a.fast) {
                lin = rest;
                for (int f = 1; f < ng; f++) {
                    const long d = sm.grows[f];
                    const long idx = lin % d;
                    lin /= d;
                    c *= __ldg(sm.gU[f] + idx + r * d);
                }
            }
            cc[it] = c;
        }
        o.c[it] = cc[it];
        if (a.fast) {
            const float4 *src = reinterpret_cast<const float4 *>(sm.gU[0] + i0 + kc * 8 + r * rows0);
            float4 v0 = __ldg(src), v1 = __ldg(src + 1);
            o.f[it][0] = v0.x; o.f[it][1] = v0.y; o.f[it][2] = v0.z; o.f[it][3] = v0.w;
            o.f[it][4] = v1.x; o.f[it][5] = v1.y; o.f[it][6] = v1.z; o.f[it][7] = v1.w;
        } else {
#pragma unroll
            for (int j = 0; j < 8; j++) {
                long k = k0 + kc * 8 + j;
                if (k >= kmax) continue;
                float v = 1.f;
                long lin = k;
                for (int f = 0; f < ng; f++) {
                    long d = sm.grows[f];
                    v *= __ldg(sm.gU[f] + (lin % d) + r * d);
                    lin /= d;
                }
                o.f[it][j] = v;
            }
        }
    }
}

template <int KIPT, int MINB>
__global__ void __launch_bounds__(NTHREADS, MINB)
    k_mttkrp_tc(const __grid_constant__ CUtensorMap tmap, TcArgs a) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t *base = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    TcCtrl &sm = *reinterpret_cast<TcCtrl *>(base);
    float *xst = reinterpret_cast<float *>(base + CTRL_BYTES);
    uint8_t *bst = base + CTRL_BYTES + (size_t)NST * X_STAGE_BYTES;
    const uint32_t bbytes = (uint32_t)b_tile_bytes(a.Rpad);
    const uint32_t a_col0 = 2u * (uint32_t)a.Rpad;  // two D buffers first, then the A stages
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long qtile = blockIdx.x % a.qtiles;
    const long z = blockIdx.x / a.qtiles;
    const long q0 = qtile * BQ;
    const long st_beg = z * a.chunk;
    const long st_end = min(a.stages, st_beg + a.chunk);
    const long nst = st_end - st_beg;
    const long nseg = (nst + SEG - 1) / SEG;
    volatile int *abort = &sm.abort;

    if (threadIdx.x == 0) {
        for (int i = 0; i < NST; i++) {
            ptx::mbar_init(&sm.full_x[i], 1);
            // producer barriers count warps: lane 0 arrives for its warp
            // after __syncwarp, so each stage costs 6 arrivals, not 192
            ptx::mbar_init(&sm.empty_x[i], NCONV / 32);
            ptx::mbar_init(&sm.full_a[i], (NCONV + NKR) / 32);
            ptx::mbar_init(&sm.empty_a[i], 1);
        }
        for (int b = 0; b < 2; b++) {
            ptx::mbar_init(&sm.d_full[b], 1);
            ptx::mbar_init(&sm.d_free[b], NCONV / 32);
        }
        ptx::mbar_init(&sm.done, 1);
        sm.abort = 0;
        for (int f = 0; f < kMaxOrder; f++) {
            sm.gU[f] = f < a.gen.n ? a.gen.U[f] : nullptr;
            sm.grows[f] = f < a.gen.n ? a.gen.rows[f] : 1;
            sm.oU[f] = f < a.outer.n ? a.outer.U[f] : nullptr;
            sm.orows[f] = f < a.outer.n ? a.outer.rows[f] : 1;
        }
        ptx::fence_mbar_init();
        ptx::prefetch_tmap(&tmap);
    }
    if (warp == 0) {
        ptx::tmem_alloc(&sm.tmem_base, a.tmem_cols);
        ptx::tmem_relinquish();
    }
    ptx::tc_fence_before();
    __syncthreads();
    ptx::tc_fence_after();
    const uint32_t tbase = sm.tmem_base;

    const bool three = (a.prec == CUD_PREC_BF16X3 || a.prec == CUD_PREC_DEFAULT);
    const bool f16 = (a.prec == CUD_PREC_FP16);

    long issued = 0;  // TMA loads issued (producer thread)
    if (warp == 0) {
        // ------------------------------------------------------------ TMA producer
        if (lane == 0) {
            for (long i = 0; i < nst && !*abort; i++) {
                const int slot = (int)(i % NST);
                const long use = i / NST;
                if (use > 0 && !ptx::mbar_wait(&sm.empty_x[slot], (uint32_t)((use - 1) & 1), abort)) break;
                const long g = st_beg + i;
                issued = i + 1;
                ptx::mbar_arrive_expect_tx(&sm.full_x[slot], X_STAGE_BYTES);
                float *dst = xst + (size_t)slot * BQ * BKS;
                if (a.kind == 0) {
                    ptx::tma_load_2d(dst, &tmap, &sm.full_x[slot], (int)q0, (int)(g * BKS));
                } else {
                    const long s = g / a.psteps, p0 = (g % a.psteps) * BKS;
                    ptx::tma_load_3d(dst, &tmap, &sm.full_x[slot], (int)p0, (int)q0, (int)s);
                }
            }
        }
    } else if (warp == 1) {
        // ------------------------------------------------------------ MMA issuer
        if (lane == 0) {
            const uint32_t idesc = ptx::idesc_f16(f16 ? 0u : 1u, BQ, (uint32_t)a.Rpad);
            const uint32_t lbo = (uint32_t)a.Rpad * 16u;
            for (long i = 0; i < nst; i++) {
                const int slot = (int)(i % NST);
                const long use = i / NST;
                const long seg = i / SEG;
                const int b = (int)(seg & 1);
                const bool seg_first = (i % SEG) == 0;
                // the segment's D buffer must have been drained (segment seg-2)
                if (seg_first && seg >= 2 &&
                    !ptx::mbar_wait(&sm.d_free[b], (uint32_t)(((seg >> 1) - 1) & 1), abort)) break;
                if (!ptx::mbar_wait(&sm.full_a[slot], (uint32_t)(use & 1), abort)) break;
                ptx::tc_fence_after();
                const uint32_t d = tbase + (uint32_t)b * (uint32_t)a.Rpad;
                const uint32_t a_hi = tbase + a_col0 + (uint32_t)slot * 32u;
                const uint32_t a_lo = a_hi + 16u;
                const uint32_t b_hi = ptx::smem_addr(bst + (size_t)(2 * slot) * bbytes);
                const uint32_t b_lo = b_hi + bbytes;
                uint32_t acc = seg_first ? 0u : 1u;
#pragma unroll
                for (int j = 0; j < 2; j++) {
                    uint64_t dh = ptx::smem_desc_kmajor_noswizzle(b_hi + 2 * j * lbo, lbo, 128);
                    ptx::mma_ts_f16(d, a_hi + j * 8, dh, idesc, acc);
                    acc = 1;
                    if (three) {
                        uint64_t dl = ptx::smem_desc_kmajor_noswizzle(b_lo + 2 * j * lbo, lbo, 128);
                        ptx::mma_ts_f16(d, a_hi + j * 8, dl, idesc, 1);
                        ptx::mma_ts_f16(d, a_lo + j * 8, dh, idesc, 1);
                    }
                }
                ptx::mma_commit(&sm.empty_a[slot]);
                if ((i % SEG) == SEG - 1 || i == nst - 1) ptx::mma_commit(&sm.d_full[b]);
            }
            // `done` completes when every MMA issued above has; waiting on it
            // here (bounded, even after an abort) keeps TMEM alive until then
            ptx::mma_commit(&sm.done);
            for (long it = 0; it < 40000 && !ptx::mbar_try_wait_hint(&sm.done, 0, 100000u); it++) {
            }
        }
    } else if (warp < 6) {
        // ------------------------------------------------------------ A converters
        const int sub = warp & 3;                 // TMEM sub-partition of this warp
        const int row = sub * 32 + lane;          // row within the tile (= TMEM lane)
        const uint32_t lane_off = (uint32_t)(sub * 32) << 16;
        const long q = q0 + row;
        float *P = a.part + z * a.R * a.Q;
        long flushed = 0;  // segments already added into the partial
        // Adds finished segment `seg` (TMEM buffer seg & 1) into the partial.
        auto flush = [&](long seg) {
            const int b = (int)(seg & 1);
            if (!*abort) ptx::mbar_wait(&sm.d_full[b], (uint32_t)((seg >> 1) & 1), abort);
            const bool ok = __all_sync(0xffffffffu, *abort == 0);  // warp-uniform tcgen05.ld
            if (ok) {
                ptx::tc_fence_after();
                const uint32_t d = tbase + lane_off + (uint32_t)b * (uint32_t)a.Rpad;
                for (int c0 = 0; c0 < a.Rpad; c0 += 32) {
                    uint32_t v[2][16];
                    const bool two = c0 + 16 < a.Rpad;  // warp-uniform
                    ptx::tmem_ld16(d + (uint32_t)c0, v[0]);
                    if (two) ptx::tmem_ld16(d + (uint32_t)c0 + 16u, v[1]);
                    ptx::tmem_wait_ld();
                    if (q < a.Q) {
                        float *p = P + q + a.Q * c0;
#pragma unroll
                        for (int j = 0; j < 32; j++) {
                            if (c0 + j < a.R) {
                                const float val = __uint_as_float(v[j >> 4][j & 15]);
                                if (seg == 0) p[a.Q * j] = val;
                                else atomicAdd(p + a.Q * j, val);  // red.global.add.f32, RN
                            }
                        }
                    }
                }
                ptx::tc_fence_before();
            }
            __syncwarp();
            if (lane == 0) ptx::mbar_arrive(&sm.d_free[b]);
        };
        for (long i = 0; i < nst; i++) {
            const int slot = (int)(i % NST);
            const long use = i / NST;
            // After an abort the loop keeps running (without waiting) so every
            // converter thread reaches the same warp-aligned tcgen05 instructions.
            if (use > 0 && !*abort) ptx::mbar_wait(&sm.empty_a[slot], (uint32_t)((use - 1) & 1), abort);
            if (!*abort) ptx::mbar_wait(&sm.full_x[slot], (uint32_t)(use & 1), abort);
            __syncwarp();
            float x[BKS];
            const float *xs = xst + (size_t)slot * BQ * BKS;
            if (a.kind == 0) {
#pragma unroll
                for (int k = 0; k < BKS; k++) x[k] = xs[k * BQ + row];
            } else {
                const float4 *r4 = reinterpret_cast<const float4 *>(xs + row * BKS);
#pragma unroll
                for (int c = 0; c < 8; c++) {
                    float4 v = r4[c ^ (row & 7)];
                    x[4 * c] = v.x; x[4 * c + 1] = v.y; x[4 * c + 2] = v.z; x[4 * c + 3] = v.w;
                }
            }
            __syncwarp();
            if (lane == 0) ptx::mbar_arrive(&sm.empty_x[slot]);
            uint32_t hi[16], lo[16];
            if (f16) {
#pragma unroll
                for (int c = 0; c < 16; c++) hi[c] = pack_f16(x[2 * c], x[2 * c + 1]);
            } else if (three) {
#pragma unroll
                for (int c = 0; c < 16; c++) split_pair(x[2 * c], x[2 * c + 1], hi[c], lo[c]);
            } else {
#pragma unroll
                for (int c = 0; c < 16; c++) hi[c] = pack_bf16(x[2 * c], x[2 * c + 1]);
            }
            const uint32_t ta = tbase + lane_off + a_col0 + (uint32_t)slot * 32u;
            ptx::tmem_st16(ta, hi);
            if (three) ptx::tmem_st16(ta + 16, lo);
            ptx::tmem_wait_st();
            ptx::tc_fence_before();
            __syncwarp();
            if (lane == 0) ptx::mbar_arrive(&sm.full_a[slot]);
            // a segment just ended: drain the one before it (long finished)
            if ((i % SEG) == SEG - 1 && i / SEG >= 1) flush(flushed++);
        }
        while (flushed < nseg) flush(flushed++);
    } else {
        // ------------------------------------------------------------ KR producers
        const int kt = threadIdx.x - 192;  // 0..63
        long ckey = -1;
        float cc[KIPT];
#pragma unroll
        for (int it = 0; it < KIPT; it++) cc[it] = 0.f;
        KrRegs<KIPT> nxt;
        if (nst > 0) kr_load<KIPT>(a, sm, st_beg, kt, nxt, ckey, cc);
        for (long i = 0; i < nst; i++) {
            const int slot = (int)(i % NST);
            const long use = i / NST;
            KrRegs<KIPT> cur = nxt;
            if (i + 1 < nst) kr_load<KIPT>(a, sm, st_beg + i + 1, kt, nxt, ckey, cc);
            if (use > 0 && !*abort) ptx::mbar_wait(&sm.empty_a[slot], (uint32_t)((use - 1) & 1), abort);
            uint8_t *bh = bst + (size_t)(2 * slot) * bbytes;
            uint8_t *bl = bh + bbytes;
#pragma unroll
            for (int it = 0; it < KIPT; it++) {
                const int id = kt + NKR * it;
                const int r = id >> 2, kc = id & 3;
                if (r >= a.Rpad) continue;
                const uint32_t off = (uint32_t)r * 16u + (uint32_t)kc * (uint32_t)a.Rpad * 16u;
                float v[8];
#pragma unroll
                for (int j = 0; j < 8; j++) v[j] = cur.f[it][j] * cur.c[it];
                uint4 h, l;
                if (f16) {
                    h.x = pack_f16(v[0], v[1]); h.y = pack_f16(v[2], v[3]);
                    h.z = pack_f16(v[4], v[5]); h.w = pack_f16(v[6], v[7]);
                } else if (three) {
                    split_pair(v[0], v[1], h.x, l.x); split_pair(v[2], v[3], h.y, l.y);
                    split_pair(v[4], v[5], h.z, l.z); split_pair(v[6], v[7], h.w, l.w);
                    *reinterpret_cast<uint4 *>(bl + off) = l;
                } else {
                    h.x = pack_bf16(v[0], v[1]); h.y = pack_bf16(v[2], v[3]);
                    h.z = pack_bf16(v[4], v[5]); h.w = pack_bf16(v[6], v[7]);
                }
                *reinterpret_cast<uint4 *>(bh + off) = h;
            }
            ptx::fence_proxy_async_smem();  // generic-proxy B writes -> tensor core
            __syncwarp();
            if (lane == 0) ptx::mbar_arrive(&sm.full_a[slot]);
        }
    }

    // ------------------------------------------------------------ teardown
    if (threadIdx.x == 0 && *abort) {
        // drain: the last load issued into each slot must land before the
        // CTA's shared memory goes away (bounded, abort flag ignored)
        for (long i = (issued > NST ? issued - NST : 0); i < issued; i++) {
            const uint32_t par = (uint32_t)((i / NST) & 1);
            for (long it = 0; it < 20000 && !ptx::mbar_try_wait_hint(&sm.full_x[i % NST], par, 100000u); it++) {
            }
        }
        atomicExch(a.error, 1);
    }
    ptx::tc_fence_before();
    __syncthreads();
    ptx::tc_fence_after();
    if (warp == 0) ptx::tmem_dealloc(tbase, a.tmem_cols);
}

// out[e] = sum_z part[z][e] in FP64: 64 outputs per CTA, the splits spread
// over 4 lanes per output (coalesced rows of 64), combined in fixed order.
__global__ void __launch_bounds__(256) k_sum_tc_partials(const float *__restrict__ part, int splits,
                                                         long n, float *__restrict__ out) {
    __shared__ double red[4][64];
    const int o = threadIdx.x & 63, lanez = threadIdx.x >> 6;
    const long e = blockIdx.x * 64L + o;
    double s = 0.0;
    if (e < n)
        for (int z = lanez; z < splits; z += 4) s += (double)__ldcs(part + (long)z * n + e);
    red[lanez][o] = s;
    __syncthreads();
    if (lanez == 0 && e < n) out[e] = (float)(((red[0][o] + red[1][o]) + red[2][o]) + red[3][o]);
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

struct TcPlan {
    int kind;
    long P, Q, S, Rpad, psteps, stages, qtiles, splits, chunk;
};

bool tc_plan(int order, const long *dims, int mode, long R, int precision, TcPlan &p) {
    if (!(precision == CUD_PREC_BF16 || precision == CUD_PREC_FP16 || precision == CUD_PREC_BF16X3 ||
          precision == CUD_PREC_DEFAULT))
        return false;
    if (order < 2 || order > kMaxOrder || R <= 0 || R > RPAD_MAX) return false;
    ModeView v = mode_view(order, dims, mode);
    p.P = v.P; p.Q = v.Q; p.S = v.S;
    p.kind = (mode == 0) ? 0 : 1;
    if (p.kind == 0 && (v.Q % 4 != 0)) return false;
    if (p.kind == 1 && (v.P % 4 != 0)) return false;
    if (v.Q > 0x7fffffffL || v.S > 0x7fffffffL || v.P > 0x7fffffffL) return false;
    for (int m = 0; m < order; m++)
        if (dims[m] > 0x7fffffffL) return false;
    p.Rpad = std::max(16L, (R + 15) / 16 * 16);
    p.psteps = (p.kind == 0) ? 1 : (v.P + BKS - 1) / BKS;
    p.stages = (p.kind == 0) ? (v.S + BKS - 1) / BKS : v.S * p.psteps;
    if (p.kind == 0 && p.stages * BKS > 0x7fffffffL) return false;
    p.qtiles = (v.Q + BQ - 1) / BQ;
    long want = std::max(1L, (2L * kNumSMs) / p.qtiles);
    p.splits = std::min(want, p.stages);
    p.chunk = (p.stages + p.splits - 1) / p.splits;
    p.splits = (p.stages + p.chunk - 1) / p.chunk;
    return true;
}

template <int KIPT, int MINB>
int launch_tc(const CUtensorMap &tmap, const TcArgs &a, unsigned grid, cudaStream_t s) {
    static bool attr[64] = {false};
    int dev = 0;
    CUD_CHECK(cudaGetDevice(&dev));
    if (dev >= 0 && dev < 64 && !attr[dev]) {
        CUD_CHECK(cudaFuncSetAttribute(k_mttkrp_tc<KIPT, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)tc_smem_bytes(RPAD_MAX)));
        attr[dev] = true;
    }
    k_mttkrp_tc<KIPT, MINB><<<grid, NTHREADS, tc_smem_bytes(a.Rpad), s>>>(tmap, a);
    CUD_CHECK_LAUNCH("mttkrp_tc");
    return CUD_OK;
}

}  // namespace

int mttkrp_tc_query(int order, const long *dims, int mode, long R, int precision, size_t *ws_bytes) {
    TcPlan p;
    if (!tc_plan(order, dims, mode, R, precision, p)) return CUD_ERR_UNSUPPORTED;
    if (!encode_fn()) return CUD_ERR_UNSUPPORTED;
    if (ws_bytes) *ws_bytes = sizeof(float) * (size_t)p.splits * R * p.Q + 256;
    return CUD_OK;
}

int mttkrp_tc(const float *X, int order, const long *dims, const float *const *U, int mode, long R,
              float *out, int precision, void *ws, cudaStream_t s) {
    TcPlan p;
    if (!tc_plan(order, dims, mode, R, precision, p)) return CUD_ERR_UNSUPPORTED;
    if ((reinterpret_cast<uintptr_t>(X) & 15) != 0) return CUD_ERR_UNSUPPORTED;
    auto encode = encode_fn();
    if (!encode) return CUD_ERR_UNSUPPORTED;
    CUtensorMap tmap;
    CUresult cr;
    if (p.kind == 0) {
        cuuint64_t gdim[2] = {(cuuint64_t)p.Q, (cuuint64_t)p.S};
        cuuint64_t gstride[1] = {(cuuint64_t)p.Q * 4};
        cuuint32_t box[2] = {BQ, BKS};
        cuuint32_t estr[2] = {1, 1};
        cr = encode(&tmap, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float *>(X), gdim, gstride, box,
                    estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    } else {
        cuuint64_t gdim[3] = {(cuuint64_t)p.P, (cuuint64_t)p.Q, (cuuint64_t)p.S};
        cuuint64_t gstride[2] = {(cuuint64_t)p.P * 4, (cuuint64_t)p.P * p.Q * 4};
        cuuint32_t box[3] = {BKS, BQ, 1};
        cuuint32_t estr[3] = {1, 1, 1};
        cr = encode(&tmap, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<float *>(X), gdim, gstride, box,
                    estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
                    CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    }
    if (cr != CUDA_SUCCESS) return CUD_ERR_UNSUPPORTED;

    TcArgs a;
    a.P = p.P; a.Q = p.Q; a.S = p.S; a.R = R;
    a.Rpad = (int)p.Rpad;
    a.kind = p.kind;
    a.prec = precision;
    a.psteps = p.psteps;
    a.stages = p.stages;
    a.chunk = p.chunk;
    a.qtiles = p.qtiles;
    a.gen.n = 0;
    a.outer.n = 0;
    for (int m = 0; m < order; m++) {
        if (m == mode) continue;
        KrFactors &f = (p.kind == 0 || m < mode) ? a.gen : a.outer;
        f.U[f.n] = U[m];
        f.rows[f.n] = dims[m];
        f.n++;
    }
    // Fast KR path: every stage covers 32 consecutive rows of the fastest
    // generating factor (its row count is a multiple of 32) and that
    // factor's columns can be read as aligned 128-bit vectors.
    a.fast = (a.gen.rows[0] % BKS == 0) && ((reinterpret_cast<uintptr_t>(a.gen.U[0]) & 15) == 0);
    char *w = static_cast<char *>(ws);
    a.error = reinterpret_cast<int *>(w);
    a.part = reinterpret_cast<float *>(w + 256);
    CUD_CHECK(cudaMemsetAsync(a.error, 0, sizeof(int), s));
    // two D buffers + NST A stages of 32 columns, rounded to a power of two
    a.tmem_cols = (2 * p.Rpad + NST * 32 <= 256) ? 256u : 512u;
    unsigned grid = (unsigned)(p.qtiles * p.splits);
    // KR items (row, 8-kappa chunk) per producer thread: 4 Rpad / 64
    int kipt = (int)((4 * p.Rpad + NKR - 1) / NKR);
    int st;
    if (kipt <= 1) st = launch_tc<1, 2>(tmap, a, grid, s);
    else if (kipt <= 2) st = launch_tc<2, 2>(tmap, a, grid, s);
    else if (kipt <= 4) st = launch_tc<4, 2>(tmap, a, grid, s);
    else st = launch_tc<8, 1>(tmap, a, grid, s);
    if (st) return st;
    long n = R * p.Q;
    k_sum_tc_partials<<<(unsigned)((n + 63) / 64), 256, 0, s>>>(a.part, (int)p.splits, n, out);
    CUD_CHECK_LAUNCH("mttkrp_tc reduce");
    return CUD_OK;
}

}  // namespace cud
