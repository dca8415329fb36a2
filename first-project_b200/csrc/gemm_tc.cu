// BF16 GEMM on the 5th-generation tensor cores (tcgen05, sm_100a):
//
//     C[m, n] = epilogue( alpha * sum_k A[m, k] * B[n, k] )
//
// A (M x K) and B (N x K) are BF16 with K contiguous ("TN"); both reach
// shared memory by TMA in 128-byte-swizzled K-major tiles, the MMA issues
// from shared memory (tcgen05.mma kind::f16, FP32 accumulation in TMEM), and
// four epilogue warps drain TMEM.  The epilogue is fused: scale, bias per n,
// ReLU, multiply by a ReLU mask (backward), and up to three outputs with
// their own (m, n) strides -- FP32 (optionally accumulated) and two BF16
// copies, so a layer can write its activation and its transpose in one pass.
//
// Tile 128 x BN (BN = 128 or 256) x 64 per stage, 4 stages; one CTA per SM.
// When the tiles alone cannot fill the GPU the contraction is split over
// gridDim.z and a second kernel sums the FP32 partials in a fixed order and
// applies the same epilogue.  Every wait is bounded (abort flag, drained
// copies, TMEM freed, error flag set).
#include <atomic>
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>

#include "kernels.cuh"
#include "tc_ptx.cuh"

namespace cud {

namespace {

constexpr int GBM = 128;
constexpr int GBK = 64;        // one 128-byte swizzle row of BF16
constexpr int GST = 4;         // pipeline stages
constexpr int GTHREADS = 192;  // w0 TMA, w1 MMA, w2-5 epilogue

struct GemmArgs {
    long M, N, K;
    long kb_per_split;  // 64-deep blocks per split
    long kblocks;
    GemmEpi e;
    float *part;        // [split][N][M] when split (m fastest), else null
    int *error;
};

struct GemmCtrl {
    uint64_t full[GST], empty[GST], done;
    uint32_t tmem_base;
    int abort;
};

constexpr size_t GCTRL_BYTES = 1024;

__host__ __device__ constexpr size_t gemm_stage_bytes(int BN) { return (size_t)(GBM + BN) * GBK * 2; }
__host__ __device__ constexpr size_t gemm_smem_bytes(int BN) { return 1024 + GCTRL_BYTES + GST * gemm_stage_bytes(BN); }

// The fused epilogue for one element (m, n) with accumulator value v.
__device__ __forceinline__ void epi_store(const GemmEpi &e, long m, long n, float v) {
    v *= e.alpha;
    if (e.bias) v += e.bias[n];
    if (e.mask) {
        const __nv_bfloat16 *mk = static_cast<const __nv_bfloat16 *>(e.mask);
        if (!(__bfloat162float(mk[m * e.mask_ldm + n * e.mask_ldn]) > 0.f)) v = 0.f;
    }
    if (e.relu) v = fmaxf(v, 0.f);
    if (e.out_f32) {
        float *p = e.out_f32 + m * e.f32_ldm + n * e.f32_ldn;
        *p = e.f32_accumulate ? *p + v : v;
    }
    if (e.out_bf16)
        static_cast<__nv_bfloat16 *>(e.out_bf16)[m * e.bf16_ldm + n * e.bf16_ldn] = __float2bfloat16_rn(v);
    if (e.out_bf16_2)
        static_cast<__nv_bfloat16 *>(e.out_bf16_2)[m * e.bf16_2_ldm + n * e.bf16_2_ldn] = __float2bfloat16_rn(v);
}

template <int BN>
__global__ void __launch_bounds__(GTHREADS, 1)
    k_gemm_tc(const __grid_constant__ CUtensorMap ta, const __grid_constant__ CUtensorMap tb, GemmArgs g) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t *base = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    GemmCtrl &sm = *reinterpret_cast<GemmCtrl *>(base);
    uint8_t *stages = base + GCTRL_BYTES;
    constexpr uint32_t A_BYTES = GBM * GBK * 2;
    constexpr uint32_t STAGE = (uint32_t)gemm_stage_bytes(BN);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long m0 = (long)blockIdx.x * GBM, n0 = (long)blockIdx.y * BN;
    const long kb0 = (long)blockIdx.z * g.kb_per_split;
    const long kb1 = min(g.kblocks, kb0 + g.kb_per_split);
    const long nkb = kb1 - kb0;
    volatile int *abort = &sm.abort;

    if (threadIdx.x == 0) {
        for (int i = 0; i < GST; i++) {
            ptx::mbar_init(&sm.full[i], 1);
            ptx::mbar_init(&sm.empty[i], 1);
        }
        ptx::mbar_init(&sm.done, 1);
        sm.abort = 0;
        ptx::fence_mbar_init();
        ptx::prefetch_tmap(&ta);
        ptx::prefetch_tmap(&tb);
    }
    if (warp == 1) {
        ptx::tmem_alloc(&sm.tmem_base, (uint32_t)BN);
        ptx::tmem_relinquish();
    }
    ptx::tc_fence_before();
    __syncthreads();
    ptx::tc_fence_after();
    const uint32_t tbase = sm.tmem_base;

    long issued = 0;
    if (warp == 0) {
        if (lane == 0) {
            for (long i = 0; i < nkb && !*abort; i++) {
                const int slot = (int)(i % GST);
                const long use = i / GST;
                if (use > 0 && !ptx::mbar_wait(&sm.empty[slot], (uint32_t)((use - 1) & 1), abort)) break;
                issued = i + 1;
                uint8_t *st = stages + (size_t)slot * STAGE;
                ptx::mbar_arrive_expect_tx(&sm.full[slot], STAGE);
                const int kx = (int)((kb0 + i) * GBK);
                ptx::tma_load_2d(st, &ta, &sm.full[slot], kx, (int)m0);
                ptx::tma_load_2d(st + A_BYTES, &tb, &sm.full[slot], kx, (int)n0);
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            const uint32_t idesc = ptx::idesc_f16(1u, GBM, (uint32_t)BN);
            for (long i = 0; i < nkb; i++) {
                const int slot = (int)(i % GST);
                const long use = i / GST;
                if (!ptx::mbar_wait(&sm.full[slot], (uint32_t)(use & 1), abort)) break;
                ptx::tc_fence_after();
                const uint32_t sa = ptx::smem_addr(stages + (size_t)slot * STAGE);
                const uint32_t sb = sa + A_BYTES;
#pragma unroll
                for (int j = 0; j < GBK / 16; j++) {
                    const uint64_t da = ptx::smem_desc_kmajor_sw128(sa + 32u * j, 1024u);
                    const uint64_t db = ptx::smem_desc_kmajor_sw128(sb + 32u * j, 1024u);
                    ptx::mma_ss_f16(tbase, da, db, idesc, (i > 0 || j > 0) ? 1u : 0u);
                }
                ptx::mma_commit(&sm.empty[slot]);
            }
            ptx::mma_commit(&sm.done);
        }
    } else {
        // epilogue: warp w reads TMEM lanes 32 (w % 4) .. +31
        const int sub = warp & 3;
        const long m = m0 + sub * 32 + lane;
        const uint32_t lane_off = (uint32_t)(sub * 32) << 16;
        bool ok = true;
        if (!*abort) ok = ptx::mbar_wait(&sm.done, 0u, abort);
        ok = __all_sync(0xffffffffu, ok && *abort == 0 && nkb > 0);
        if (ok) {
            ptx::tc_fence_after();
            for (int c0 = 0; c0 < BN; c0 += 32) {
                uint32_t v[32];
                ptx::tmem_ld32(tbase + lane_off + (uint32_t)c0, v);
                ptx::tmem_wait_ld();
                if (m < g.M) {
#pragma unroll
                    for (int j = 0; j < 32; j++) {
                        const long n = n0 + c0 + j;
                        if (n < g.N) {
                            const float val = __uint_as_float(v[j]);
                            if (g.part) g.part[((long)blockIdx.z * g.N + n) * g.M + m] = val;
                            else epi_store(g.e, m, n, val);
                        }
                    }
                }
            }
            ptx::tc_fence_before();
        }
    }

    // ------------------------------------------------------------ teardown
    if (threadIdx.x == 32 && *abort) {
        // the MMAs issued before the abort must finish before TMEM is freed
        for (long it = 0; it < 20000 && !ptx::mbar_try_wait_hint(&sm.done, 0u, 100000u); it++) {
        }
    }
    if (threadIdx.x == 0 && *abort) {
        for (long i = (issued > GST ? issued - GST : 0); i < issued; i++) {
            const uint32_t par = (uint32_t)((i / GST) & 1);
            for (long it = 0; it < 20000 && !ptx::mbar_try_wait_hint(&sm.full[i % GST], par, 100000u); it++) {
            }
        }
        atomicExch(g.error, 1);
    }
    ptx::tc_fence_before();
    __syncthreads();
    ptx::tc_fence_after();
    if (warp == 1) ptx::tmem_dealloc(tbase, (uint32_t)BN);
}

// ---------------------------------------------------------------- skinny N
// N <= 32 with many rows (the TTM chain's products, N = rank): one CTA per
// SM loops over 128-row tiles; the whole B (N x K, K <= SK_KMAX) is loaded
// once into shared memory, A streams through an SK_ST-deep ring, and the
// accumulators alternate between two TMEM buffers so the epilogue of one
// tile overlaps the MMAs of the next.
constexpr int SK_BN = 32;
constexpr int SK_ST = 8;
constexpr int SK_KMAX = 1024;

struct SkCtrl {
    uint64_t full[SK_ST], empty[SK_ST], b_full, d_full[2], d_free[2];
    uint32_t tmem_base;
    int abort;
};

__host__ __device__ constexpr size_t sk_smem_bytes(long kblocks) {
    return 1024 + GCTRL_BYTES + (size_t)kblocks * SK_BN * GBK * 2 + (size_t)SK_ST * GBM * GBK * 2;
}

__global__ void __launch_bounds__(GTHREADS, 1)
    k_gemm_skinny(const __grid_constant__ CUtensorMap ta, const __grid_constant__ CUtensorMap tb, GemmArgs g,
                  long mt) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t *base = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    SkCtrl &sm = *reinterpret_cast<SkCtrl *>(base);
    constexpr uint32_t A_BYTES = GBM * GBK * 2;
    constexpr uint32_t B_BYTES = SK_BN * GBK * 2;
    const long nkb = g.kblocks;
    uint8_t *bsm = base + GCTRL_BYTES;                    // nkb B tiles
    uint8_t *aring = bsm + (size_t)nkb * B_BYTES;          // SK_ST A tiles (1024-aligned: B_BYTES is)
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    volatile int *abort = &sm.abort;
    // this CTA's tiles: t = blockIdx.x + gridDim.x * j
    const long ntile = (mt - blockIdx.x + gridDim.x - 1) / gridDim.x;

    if (threadIdx.x == 0) {
        for (int i = 0; i < SK_ST; i++) {
            ptx::mbar_init(&sm.full[i], 1);
            ptx::mbar_init(&sm.empty[i], 1);
        }
        ptx::mbar_init(&sm.b_full, 1);
        for (int b = 0; b < 2; b++) {
            ptx::mbar_init(&sm.d_full[b], 1);
            ptx::mbar_init(&sm.d_free[b], 4);  // the four epilogue warps
        }
        sm.abort = 0;
        ptx::fence_mbar_init();
        ptx::prefetch_tmap(&ta);
        ptx::prefetch_tmap(&tb);
    }
    if (warp == 1) {
        ptx::tmem_alloc(&sm.tmem_base, 2 * SK_BN);
        ptx::tmem_relinquish();
    }
    ptx::tc_fence_before();
    __syncthreads();
    ptx::tc_fence_after();
    const uint32_t tbase = sm.tmem_base;

    long issued = 0;
    if (warp == 0) {
        if (lane == 0) {
            ptx::mbar_arrive_expect_tx(&sm.b_full, (uint32_t)(nkb * B_BYTES));
            for (long kb = 0; kb < nkb; kb++)
                ptx::tma_load_2d(bsm + (size_t)kb * B_BYTES, &tb, &sm.b_full, (int)(kb * GBK), 0);
            long i = 0;  // stage counter over all tiles
            for (long j = 0; j < ntile && !*abort; j++) {
                const long m0 = (blockIdx.x + gridDim.x * j) * GBM;
                for (long kb = 0; kb < nkb && !*abort; kb++, i++) {
                    const int slot = (int)(i % SK_ST);
                    const long use = i / SK_ST;
                    if (use > 0 && !ptx::mbar_wait(&sm.empty[slot], (uint32_t)((use - 1) & 1), abort)) break;
                    ptx::mbar_arrive_expect_tx(&sm.full[slot], A_BYTES);
                    ptx::tma_load_2d(aring + (size_t)slot * A_BYTES, &ta, &sm.full[slot], (int)(kb * GBK), (int)m0);
                    issued = i + 1;
                }
            }
        }
    } else if (warp == 1) {
        if (lane == 0) {
            const uint32_t idesc = ptx::idesc_f16(1u, GBM, (uint32_t)SK_BN);
            bool ok = ptx::mbar_wait(&sm.b_full, 0u, abort);
            long i = 0;
            for (long j = 0; j < ntile && ok; j++) {
                const int b = (int)(j & 1);
                // the buffer's previous tile (j - 2) must have been drained
                if (j >= 2 && !ptx::mbar_wait(&sm.d_free[b], (uint32_t)(((j >> 1) - 1) & 1), abort)) break;
                const uint32_t d = tbase + (uint32_t)b * SK_BN;
                for (long kb = 0; kb < nkb; kb++, i++) {
                    const int slot = (int)(i % SK_ST);
                    const long use = i / SK_ST;
                    if (!ptx::mbar_wait(&sm.full[slot], (uint32_t)(use & 1), abort)) { ok = false; break; }
                    ptx::tc_fence_after();
                    const uint32_t sa = ptx::smem_addr(aring + (size_t)slot * A_BYTES);
                    const uint32_t sb = ptx::smem_addr(bsm + (size_t)kb * B_BYTES);
#pragma unroll
                    for (int k = 0; k < GBK / 16; k++) {
                        const uint64_t da = ptx::smem_desc_kmajor_sw128(sa + 32u * k, 1024u);
                        const uint64_t db = ptx::smem_desc_kmajor_sw128(sb + 32u * k, 1024u);
                        ptx::mma_ss_f16(d, da, db, idesc, (kb > 0 || k > 0) ? 1u : 0u);
                    }
                    ptx::mma_commit(&sm.empty[slot]);
                }
                if (!ok) break;
                ptx::mma_commit(&sm.d_full[b]);
            }
        }
    } else {
        // epilogue: warp w reads TMEM lanes 32 (w % 4) .. +31
        const int sub = warp & 3;
        const uint32_t lane_off = (uint32_t)(sub * 32) << 16;
        const bool plain = g.e.alpha == 1.f && !g.e.bias && !g.e.mask && !g.e.relu && !g.e.out_bf16_2;
        const bool simple_bf16 = plain && g.e.out_bf16 && !g.e.out_f32;
        const bool simple_f32 = plain && g.e.out_f32 && !g.e.f32_accumulate && !g.e.out_bf16;
        for (long j = 0; j < ntile; j++) {
            const int b = (int)(j & 1);
            const long m = (blockIdx.x + gridDim.x * j) * GBM + sub * 32 + lane;
            bool ok = true;
            if (!*abort) ok = ptx::mbar_wait(&sm.d_full[b], (uint32_t)((j >> 1) & 1), abort);
            ok = __all_sync(0xffffffffu, ok && *abort == 0);
            if (!ok) break;
            ptx::tc_fence_after();
            uint32_t v[32];
            ptx::tmem_ld32(tbase + lane_off + (uint32_t)b * SK_BN, v);
            ptx::tmem_wait_ld();
            ptx::tc_fence_before();
            __syncwarp();
            if (lane == 0) ptx::mbar_arrive(&sm.d_free[b]);  // the values are in registers
            if (m < g.M) {
                if (simple_bf16) {
                    // plain BF16 output: walk the row's outputs by pointer
                    __nv_bfloat16 *p = static_cast<__nv_bfloat16 *>(g.e.out_bf16) + m * g.e.bf16_ldm;
                    const long step = g.e.bf16_ldn;
#pragma unroll
                    for (int n = 0; n < SK_BN; n++) {
                        if (n < g.N) *p = __float2bfloat16_rn(__uint_as_float(v[n]));
                        p += step;
                    }
                } else if (simple_f32) {
                    float *p = g.e.out_f32 + m * g.e.f32_ldm;
                    const long step = g.e.f32_ldn;
#pragma unroll
                    for (int n = 0; n < SK_BN; n++) {
                        if (n < g.N) *p = __uint_as_float(v[n]);
                        p += step;
                    }
                } else {
#pragma unroll
                    for (int n = 0; n < SK_BN; n++)
                        if (n < g.N) epi_store(g.e, m, n, __uint_as_float(v[n]));
                }
            }
        }
    }

    // ------------------------------------------------------------ teardown
    if (threadIdx.x == 0 && *abort) {
        for (long i = (issued > SK_ST ? issued - SK_ST : 0); i < issued; i++) {
            const uint32_t par = (uint32_t)((i / SK_ST) & 1);
            for (long it = 0; it < 20000 && !ptx::mbar_try_wait_hint(&sm.full[i % SK_ST], par, 100000u); it++) {
            }
        }
        for (long it = 0; it < 20000 && !ptx::mbar_try_wait_hint(&sm.b_full, 0u, 100000u); it++) {
        }
        atomicExch(g.error, 1);
    }
    if (threadIdx.x == 32) {
        // every MMA issued must finish before TMEM is freed (bounded)
        ptx::mma_commit(&sm.b_full);  // b_full phase 1 completes once the issued MMAs have
        for (long it = 0; it < 20000 && !ptx::mbar_try_wait_hint(&sm.b_full, 1u, 100000u); it++) {
        }
    }
    ptx::tc_fence_before();
    __syncthreads();
    ptx::tc_fence_after();
    if (warp == 1) ptx::tmem_dealloc(tbase, 2 * SK_BN);
}

// Sums the split partials (fixed order) and applies the epilogue.
__global__ void __launch_bounds__(256) k_gemm_splitk_epi(const float *__restrict__ part, int splits, long M, long N,
                                                          GemmEpi e) {
    const long total = M * N;
    for (long idx = blockIdx.x * 256L + threadIdx.x; idx < total; idx += (long)gridDim.x * 256L) {
        const long n = idx / M, m = idx - n * M;
        float s = 0.f;
        for (int z = 0; z < splits; z++) s += part[(long)z * total + idx];
        epi_store(e, m, n, s);
    }
}

PFN_cuTensorMapEncodeTiled_v12000 gemm_encode_fn() {
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

bool encode_bf16_kmajor(CUtensorMap &map, const void *ptr, long rows, long K, long ld, int box_rows) {
    auto enc = gemm_encode_fn();
    if (!enc) return false;
    cuuint64_t gdim[2] = {(cuuint64_t)K, (cuuint64_t)rows};
    cuuint64_t gstride[1] = {(cuuint64_t)ld * 2};
    cuuint32_t box[2] = {(cuuint32_t)GBK, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    return enc(&map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(ptr), gdim, gstride, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

struct GemmPlan {
    int BN;
    long mt, nt, kblocks, splits, kb_per_split;
};

GemmPlan gemm_plan(long M, long N, long K) {
    GemmPlan p;
    p.BN = (N > 128) ? 256 : 128;
    p.mt = (M + GBM - 1) / GBM;
    p.nt = (N + p.BN - 1) / p.BN;
    p.kblocks = (K + GBK - 1) / GBK;
    const long tiles = p.mt * p.nt;
    long want = std::max(1L, kNumSMs / tiles);
    // a split keeps at least 4 blocks of 64 so the pipeline fills
    want = std::min(want, std::max(1L, p.kblocks / 4));
    p.kb_per_split = (p.kblocks + want - 1) / want;
    p.splits = (p.kblocks + p.kb_per_split - 1) / p.kb_per_split;
    return p;
}

// The skinny path: N <= 32, K <= SK_KMAX, and at least two tiles per SM.
bool skinny_ok(long M, long N, long K) {
#ifdef CUD_GEMM_NO_SKINNY
    return false;
#endif
    return N <= SK_BN && K <= SK_KMAX && (M + GBM - 1) / GBM >= 2 * kNumSMs;
}

template <int BN>
int launch_gemm(const CUtensorMap &ta, const CUtensorMap &tb, const GemmArgs &g, dim3 grid, cudaStream_t s) {
    static std::atomic<bool> attr[64];  // per device; zero-initialised
    int dev = 0;
    CUD_CHECK(cudaGetDevice(&dev));
    if (dev >= 0 && dev < 64 && !attr[dev].load(std::memory_order_acquire)) {
        CUD_CHECK(cudaFuncSetAttribute(k_gemm_tc<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)gemm_smem_bytes(BN)));
        attr[dev].store(true, std::memory_order_release);
    }
    k_gemm_tc<BN><<<grid, GTHREADS, gemm_smem_bytes(BN), s>>>(ta, tb, g);
    CUD_CHECK_LAUNCH("gemm_tc");
    return CUD_OK;
}

}  // namespace

size_t gemm_tc_ws_bytes(long M, long N, long K) {
    GemmPlan p = gemm_plan(M, N, K);
    size_t b = 256;
    if (p.splits > 1 && !skinny_ok(M, N, K)) b += sizeof(float) * (size_t)p.splits * M * N;
    return b;
}

int gemm_tc_bf16(const __nv_bfloat16 *A, long lda, const __nv_bfloat16 *B, long ldb, long M, long N, long K,
                 const GemmEpi &e, void *ws, cudaStream_t s) {
    if (M <= 0 || N <= 0 || K <= 0 || !A || !B || !ws) return CUD_ERR_INVALID_ARGUMENT;
    if (lda < K || ldb < K || (lda % 8) || (ldb % 8)) return CUD_ERR_INVALID_ARGUMENT;
    if ((reinterpret_cast<uintptr_t>(A) & 15) || (reinterpret_cast<uintptr_t>(B) & 15)) return CUD_ERR_INVALID_ARGUMENT;
    if (M > 0x7fffffffL || N > 0x7fffffffL || K > 0x7fffffffL) return CUD_ERR_UNSUPPORTED;
    GemmPlan p = gemm_plan(M, N, K);
    CUtensorMap ta, tb;
    if (skinny_ok(M, N, K)) {
        if (!encode_bf16_kmajor(ta, A, M, K, lda, GBM) || !encode_bf16_kmajor(tb, B, N, K, ldb, SK_BN))
            return CUD_ERR_UNSUPPORTED;
        GemmArgs g;
        g.M = M; g.N = N; g.K = K;
        g.kblocks = (K + GBK - 1) / GBK;
        g.kb_per_split = g.kblocks;
        g.e = e;
        g.error = reinterpret_cast<int *>(ws);
        g.part = nullptr;
        CUD_CHECK(cudaMemsetAsync(g.error, 0, sizeof(int), s));
        const long mt = (M + GBM - 1) / GBM;
        const size_t smem = sk_smem_bytes(g.kblocks);
        static std::atomic<bool> attr[64];  // per device; zero-initialised
        int dev = 0;
        CUD_CHECK(cudaGetDevice(&dev));
        if (dev >= 0 && dev < 64 && !attr[dev].load(std::memory_order_acquire)) {
            CUD_CHECK(cudaFuncSetAttribute(k_gemm_skinny, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)sk_smem_bytes(SK_KMAX / GBK)));
            attr[dev].store(true, std::memory_order_release);
        }
        k_gemm_skinny<<<(unsigned)std::min<long>(mt, kNumSMs), GTHREADS, smem, s>>>(ta, tb, g, mt);
        CUD_CHECK_LAUNCH("gemm_tc skinny");
        return CUD_OK;
    }
    if (!encode_bf16_kmajor(ta, A, M, K, lda, GBM) || !encode_bf16_kmajor(tb, B, N, K, ldb, p.BN))
        return CUD_ERR_UNSUPPORTED;
    GemmArgs g;
    g.M = M; g.N = N; g.K = K;
    g.kblocks = p.kblocks;
    g.kb_per_split = p.kb_per_split;
    g.e = e;
    char *w = static_cast<char *>(ws);
    g.error = reinterpret_cast<int *>(w);
    g.part = (p.splits > 1) ? reinterpret_cast<float *>(w + 256) : nullptr;
    CUD_CHECK(cudaMemsetAsync(g.error, 0, sizeof(int), s));
    dim3 grid((unsigned)p.mt, (unsigned)p.nt, (unsigned)p.splits);
    int st = (p.BN == 256) ? launch_gemm<256>(ta, tb, g, grid, s) : launch_gemm<128>(ta, tb, g, grid, s);
    if (st) return st;
    if (p.splits > 1) {
        const long total = M * N;
        const unsigned blocks = (unsigned)std::min<long>((total + 255) / 256, 4L * kNumSMs);
        k_gemm_splitk_epi<<<blocks, 256, 0, s>>>(g.part, (int)p.splits, M, N, e);
        CUD_CHECK_LAUNCH("gemm_tc split-k epilogue");
    }
    return CUD_OK;
}

}  // namespace cud

using namespace cud;

extern "C" int cud_gemm_bf16(const void *A, long lda, const void *B, long ldb, long M, long N, long K,
                             const cud_gemm_epilogue *epilogue, void *stream) {
    if (!epilogue) return set_status(CUD_ERR_INVALID_ARGUMENT);
    int st;
    void *ws = scratch(kSlotTmp2, gemm_tc_ws_bytes(M, N, K), &st);
    if (!ws) return set_status(st);
    st = gemm_tc_bf16(static_cast<const __nv_bfloat16 *>(A), lda, static_cast<const __nv_bfloat16 *>(B), ldb, M, N,
                      K, *epilogue, ws, as_stream(stream));
    return set_status(st);
}
