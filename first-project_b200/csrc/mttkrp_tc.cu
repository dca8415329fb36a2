// MTTKRP on the 5th-generation tensor cores (tcgen05, sm_100a).
//
// Around mode n the FP32 tensor is a (P, Q, S) array; the result is
// M[q, r] = sum_kappa X(q, kappa) * KR(kappa, r), with kappa running over the
// other modes.  Per CTA: one tile of 128 rows q (the MMA's M) and a
// contiguous range of 32-deep contraction stages.  Per stage:
//   * TMA brings the 128 x 32 FP32 tile of X, in its native layout, into
//     shared memory (mode 0: rows contiguous, a 2-D box over (q, s); other
//     modes: kappa contiguous, a 3-D box over (p, q, s) with 128-byte
//     swizzle);
//   * four converter warps read their rows, split each value into BF16
//     hi + lo (x = hi + lo + O(2^-16 x)), and store both into tensor memory
//     as the MMA's A operand (one TMEM lane per row);
//   * the same warps form the 32 Khatri-Rao rows of the stage from the factor
//     matrices, split them the same way, and write them to shared memory in
//     the K-major canonical layout (the B operand);
//   * one thread issues tcgen05.mma (kind::f16, FP32 accumulation in TMEM):
//     D += Xhi*KRhi + Xhi*KRlo + Xlo*KRhi  (BF16X3), or one product for
//     BF16 / FP16.
// The unfolding and the KR matrix are never materialised: X is read from HBM
// exactly once.  After the last stage the converter warps read D from TMEM
// and write the CTA's FP32 partial; a second small kernel sums the partials
// over the contraction splits in FP64.
//
// Every wait is bounded: an expired wait raises a CTA-wide abort flag, the
// roles drain and the TMEM is freed before the CTA exits; the host sees the
// error flag and returns CUD_ERR_DEVICE_TIMEOUT.
#include <cuda.h>
#include <cudaTypedefs.h>

#include "kernels.cuh"
#include "tc_ptx.cuh"

namespace cud {

namespace {

constexpr int BQ = 128;      // rows per CTA tile (MMA M)
constexpr int BKS = 32;      // contraction depth per stage (two MMA K-steps of 16)
constexpr int NST = 4;       // pipeline stages
constexpr int NTHREADS = 192;  // warp 0 TMA, warp 1 MMA, warps 2..5 converters
constexpr int NCONV = 128;
constexpr uint32_t TMEM_COLS = 256;
constexpr uint32_t A_COL0 = 128;  // A stages start at this TMEM column
constexpr int X_STAGE_BYTES = BQ * BKS * 4;  // 16 KB

struct TcArgs {
    long P, Q, S, R;
    int Rpad;          // R rounded up to a multiple of 16 (MMA N)
    int kind;          // 0: mode 0 (rows contiguous); 1: other modes (kappa contiguous)
    int prec;          // CUD_PREC_BF16 / FP16 / BF16X3
    long psteps;       // stages per s (kind 1) = ceil(P / 32)
    long stages;       // total stages
    long chunk;        // stages per CTA
    long qtiles;
    KrFactors gen;     // kind 0: factors after mode 0; kind 1: factors before the mode
    KrFactors outer;   // kind 1: factors after the mode (per-stage constant row)
    float *part;       // [split][R][Q]
    int *error;        // device flag
};

// Shared memory: control block first, then (1024-byte aligned) the NST X
// stages of 16 KB, then the NST pairs of B tiles of Rpad x 32 16-bit values.
struct TcCtrl {
    uint64_t full_x[NST], empty_x[NST], full_a[NST], empty_a[NST], done;
    int tab[BKS][kMaxOrder];   // KR row indices of the current stage
    int rt[kMaxOrder];         // row index of the outer factors (per stage constant)
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

// Byte offset of element (n, k) (16-bit) in a K-major, no-swizzle B tile of
// 32 columns: core matrix (n/8, k/8) at (n/8)*512 + (k/8)*128.
__device__ __forceinline__ uint32_t b_offset(int n, int k) {
    return (uint32_t)((n >> 3) * 512 + (k >> 3) * 128 + (n & 7) * 16 + (k & 7) * 2);
}

__global__ void __launch_bounds__(NTHREADS, 2)
    k_mttkrp_tc(const __grid_constant__ CUtensorMap tmap, TcArgs a) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t *base = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    TcCtrl &sm = *reinterpret_cast<TcCtrl *>(base);
    float *xst = reinterpret_cast<float *>(base + CTRL_BYTES);
    uint8_t *bst = base + CTRL_BYTES + (size_t)NST * X_STAGE_BYTES;
    const size_t bbytes = b_tile_bytes(a.Rpad);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long qtile = blockIdx.x % a.qtiles;
    const long z = blockIdx.x / a.qtiles;
    const long q0 = qtile * BQ;
    const long st_beg = z * a.chunk;
    const long st_end = min(a.stages, st_beg + a.chunk);
    const long nst = st_end - st_beg;
    volatile int *abort = &sm.abort;

    if (threadIdx.x == 0) {
        for (int i = 0; i < NST; i++) {
            ptx::mbar_init(&sm.full_x[i], 1);
            ptx::mbar_init(&sm.empty_x[i], NCONV);
            ptx::mbar_init(&sm.full_a[i], NCONV);
            ptx::mbar_init(&sm.empty_a[i], 1);
        }
        ptx::mbar_init(&sm.done, 1);
        sm.abort = 0;
        ptx::fence_mbar_init();
        ptx::prefetch_tmap(&tmap);
    }
    if (warp == 0) {
        ptx::tmem_alloc(&sm.tmem_base, TMEM_COLS);
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
                int slot = (int)(i % NST);
                long use = i / NST;
                if (use > 0 && !ptx::mbar_wait(&sm.empty_x[slot], (uint32_t)((use - 1) & 1), abort)) break;
                long g = st_beg + i;
                issued = i + 1;
                ptx::mbar_arrive_expect_tx(&sm.full_x[slot], X_STAGE_BYTES);
                if (a.kind == 0) {
                    ptx::tma_load_2d((xst + (size_t)slot * BQ * BKS), &tmap, &sm.full_x[slot], (int)q0, (int)(g * BKS));
                } else {
                    long s = g / a.psteps, p0 = (g % a.psteps) * BKS;
                    ptx::tma_load_3d((xst + (size_t)slot * BQ * BKS), &tmap, &sm.full_x[slot], (int)p0, (int)q0, (int)s);
                }
            }
        }
    } else if (warp == 1) {
        // ------------------------------------------------------------ MMA issuer
        if (lane == 0) {
            const uint32_t idesc = ptx::idesc_f16(f16 ? 0u : 1u, BQ, (uint32_t)a.Rpad);
            uint32_t acc = 0;
            for (long i = 0; i < nst; i++) {
                int slot = (int)(i % NST);
                long use = i / NST;
                if (!ptx::mbar_wait(&sm.full_a[slot], (uint32_t)(use & 1), abort)) break;
                ptx::tc_fence_after();
                const uint32_t a_hi = tbase + A_COL0 + (uint32_t)slot * 32u;
                const uint32_t a_lo = a_hi + 16u;
                const uint32_t b_hi = ptx::smem_addr(bst + (size_t)(2 * slot) * bbytes);
                const uint32_t b_lo = ptx::smem_addr(bst + (size_t)(2 * slot + 1) * bbytes);
#pragma unroll
                for (int j = 0; j < 2; j++) {
                    uint64_t dh = ptx::smem_desc_kmajor_noswizzle(b_hi + j * 256, 128, 512);
                    ptx::mma_ts_f16(tbase, a_hi + j * 8, dh, idesc, acc);
                    acc = 1;
                    if (three) {
                        uint64_t dl = ptx::smem_desc_kmajor_noswizzle(b_lo + j * 256, 128, 512);
                        ptx::mma_ts_f16(tbase, a_hi + j * 8, dl, idesc, 1);
                        ptx::mma_ts_f16(tbase, a_lo + j * 8, dh, idesc, 1);
                    }
                }
                ptx::mma_commit(&sm.empty_a[slot]);
            }
            // `done` completes when every MMA issued above has; waiting on it
            // here (bounded, even after an abort) keeps TMEM alive until then
            ptx::mma_commit(&sm.done);
            for (long it = 0; it < (1L << 24) && !ptx::mbar_try_wait(&sm.done, 0); it++) __nanosleep(32);
        }
    } else {
        // ------------------------------------------------------------ converters
        const int sub = warp & 3;                 // TMEM sub-partition of this warp
        const int row = sub * 32 + lane;          // row within the tile (= TMEM lane)
        const int ct = threadIdx.x - 64;          // 0..127 among converters
        const uint32_t lane_off = (uint32_t)(sub * 32) << 16;
        for (long i = 0; i < nst; i++) {
            int slot = (int)(i % NST);
            long use = i / NST;
            long g = st_beg + i;
            // stage decode
            long s = 0, p0 = 0;
            if (a.kind == 1) { s = g / a.psteps; p0 = (g % a.psteps) * BKS; }
            long k0 = (a.kind == 0) ? g * BKS : p0;  // first contraction index of the stage
            long kmax = (a.kind == 0) ? a.S : a.P;
            // KR index table for this stage (threads 0..31), outer row (thread 32)
            if (ct < BKS) {
                long k = k0 + ct;
                if (k < kmax) {
                    long lin = k;
                    for (int f = 0; f < a.gen.n; f++) {
                        sm.tab[ct][f] = (int)(lin % a.gen.rows[f]);
                        lin /= a.gen.rows[f];
                    }
                } else {
                    sm.tab[ct][0] = -1;
                }
            } else if (ct == BKS && a.kind == 1) {
                long lin = s;
                for (int f = 0; f < a.outer.n; f++) {
                    sm.rt[f] = (int)(lin % a.outer.rows[f]);
                    lin /= a.outer.rows[f];
                }
            }
            // The slot's TMEM A stage and B tile are free once the MMAs of its
            // previous use completed.  After an abort the loop keeps running
            // (without waiting) so every converter thread reaches the same
            // warp-aligned tcgen05 instructions and named barriers.
            if (use > 0 && !*abort) ptx::mbar_wait(&sm.empty_a[slot], (uint32_t)((use - 1) & 1), abort);
            if (!*abort) ptx::mbar_wait(&sm.full_x[slot], (uint32_t)(use & 1), abort);
            __syncwarp();
            // ---- A operand: this thread's row, 32 values
            float x[BKS];
            const float *xs = (xst + (size_t)slot * BQ * BKS);
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
            ptx::mbar_arrive(&sm.empty_x[slot]);
            {
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
                const uint32_t ta = tbase + lane_off + A_COL0 + (uint32_t)slot * 32u;
                ptx::tmem_st16(ta, hi);
                if (three) ptx::tmem_st16(ta + 16, lo);
            }
            // ---- B operand: the stage's 32 KR rows, Rpad columns
            ptx::named_bar_sync(1, NCONV);  // index table ready
            {
                uint8_t *bh = bst + (size_t)(2 * slot) * bbytes;
                uint8_t *bl = bst + (size_t)(2 * slot + 1) * bbytes;
                const int npairs = a.Rpad * (BKS / 2);
                for (int e = ct; e < npairs; e += NCONV) {
                    int r = e % a.Rpad, kp = e / a.Rpad;
                    float v0 = 0.f, v1 = 0.f;
                    if (r < a.R) {
                        float w = 1.0f;
                        if (a.kind == 1)
                            for (int f = 0; f < a.outer.n; f++)
                                w *= __ldg(a.outer.U[f] + sm.rt[f] + r * a.outer.rows[f]);
                        const int *t0 = sm.tab[2 * kp];
                        const int *t1 = sm.tab[2 * kp + 1];
                        if (t0[0] >= 0) {
                            v0 = 1.0f;
                            for (int f = 0; f < a.gen.n; f++) v0 *= __ldg(a.gen.U[f] + t0[f] + r * a.gen.rows[f]);
                            v0 *= w;
                        }
                        if (t1[0] >= 0) {
                            v1 = 1.0f;
                            for (int f = 0; f < a.gen.n; f++) v1 *= __ldg(a.gen.U[f] + t1[f] + r * a.gen.rows[f]);
                            v1 *= w;
                        }
                    }
                    uint32_t off = b_offset(r, 2 * kp);
                    if (f16) {
                        *reinterpret_cast<uint32_t *>(bh + off) = pack_f16(v0, v1);
                    } else if (three) {
                        uint32_t h, l;
                        split_pair(v0, v1, h, l);
                        *reinterpret_cast<uint32_t *>(bh + off) = h;
                        *reinterpret_cast<uint32_t *>(bl + off) = l;
                    } else {
                        *reinterpret_cast<uint32_t *>(bh + off) = pack_bf16(v0, v1);
                    }
                }
            }
            ptx::fence_proxy_async_smem();  // generic-proxy B writes -> tensor core
            ptx::tmem_wait_st();
            ptx::tc_fence_before();
            ptx::mbar_arrive(&sm.full_a[slot]);
            ptx::named_bar_sync(2, NCONV);  // table slot reuse guard
        }
        // ---- epilogue: D (128 x Rpad FP32) -> partial
        if (!*abort) ptx::mbar_wait(&sm.done, 0, abort);
        // warp-uniform decision: tcgen05.ld is a warp-aligned instruction
        const bool epi = __all_sync(0xffffffffu, *abort == 0);
        if (epi) {
            ptx::tc_fence_after();
            long q = q0 + row;
            float *P = a.part + z * a.R * a.Q;
            for (int c0 = 0; c0 < a.Rpad; c0 += 16) {
                uint32_t v[16];
                ptx::tmem_ld16(tbase + lane_off + (uint32_t)c0, v);
                ptx::tmem_wait_ld();
                if (q < a.Q) {
#pragma unroll
                    for (int j = 0; j < 16; j++) {
                        int r = c0 + j;
                        if (r < a.R) P[q + a.Q * r] = __uint_as_float(v[j]);
                    }
                }
            }
        }
    }

    // ------------------------------------------------------------ teardown
    if (threadIdx.x == 0 && *abort) {
        // drain: the last load issued into each slot must land before the
        // CTA's shared memory goes away (bounded polls, abort flag ignored)
        for (long i = (issued > NST ? issued - NST : 0); i < issued; i++) {
            uint32_t par = (uint32_t)((i / NST) & 1);
            for (long it = 0; it < (1L << 22) && !ptx::mbar_try_wait(&sm.full_x[i % NST], par); it++)
                __nanosleep(32);
        }
        atomicExch(a.error, 1);
    }
    ptx::tc_fence_before();
    __syncthreads();
    ptx::tc_fence_after();
    if (warp == 0) ptx::tmem_dealloc(tbase, TMEM_COLS);
}

__global__ void k_sum_tc_partials(const float *__restrict__ part, int splits, long n,
                                  float *__restrict__ out) {
    long tid = blockIdx.x * (long)blockDim.x + threadIdx.x;
    long stride = (long)gridDim.x * blockDim.x;
    for (long e = tid; e < n; e += stride) {
        double s = 0.0;
        for (int z = 0; z < splits; z++) s += (double)part[(long)z * n + e];
        out[e] = (float)s;
    }
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
    if (order < 2 || R <= 0 || R > 128) return false;
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
    char *w = static_cast<char *>(ws);
    a.error = reinterpret_cast<int *>(w);
    a.part = reinterpret_cast<float *>(w + 256);
    size_t smem = tc_smem_bytes(a.Rpad);
    static bool attr[64] = {false};
    int dev = 0;
    CUD_CHECK(cudaGetDevice(&dev));
    if (dev >= 0 && dev < 64 && !attr[dev]) {
        CUD_CHECK(cudaFuncSetAttribute(k_mttkrp_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        attr[dev] = true;
    }
    CUD_CHECK(cudaMemsetAsync(a.error, 0, sizeof(int), s));
    k_mttkrp_tc<<<(unsigned)(p.qtiles * p.splits), NTHREADS, smem, s>>>(tmap, a);
    CUD_CHECK_LAUNCH("mttkrp_tc");
    long n = R * p.Q;
    k_sum_tc_partials<<<blocks_for(n, 256), 256, 0, s>>>(a.part, (int)p.splits, n, out);
    CUD_CHECK_LAUNCH("mttkrp_tc reduce");
    return CUD_OK;
}

}  // namespace cud
