// MTTKRP on the 5th-generation tensor cores (tcgen05, sm_100a).
//
// Around mode n the FP32 tensor is a (P, Q, S) array; the result is
// M[q, r] = sum_kappa X(q, kappa) * KR(kappa, r), with kappa running over the
// other modes.  Per CTA: one tile of 128 rows q (the MMA's M) and a
// contiguous range of 32-deep contraction stages, pipelined 3-6 deep between
// warp roles:
//   * a TMA warp: the 128 x 32 FP32 tile of X, in its native layout, into
//     shared memory (mode 0: rows contiguous, a 2-D box over (q, s); other
//     modes: kappa contiguous, a 3-D box over (p, q, s) with 128-byte
//     swizzle);
//   * eight A-converter warps in two stage-parity groups (one warp per TMEM
//     lane quarter each): a thread reads its row (= its TMEM lane), splits
//     every value into BF16 hi + lo (x = hi + lo + O(2^-16 x)) and stores
//     both into tensor memory as the MMA's A operand -- X crosses shared
//     memory once;
//   * the B operand (the stage's 32 Khatri-Rao rows), two ways.  The stage's
//     kappa run over 32 consecutive rows of the fastest generating factor U0
//     while the other factors contribute one constant row c.  Pre-packed B
//     path (k_mttkrp_pb): c is applied per accumulation segment at the flush,
//     so B is U0's unscaled rows, packed once per call into the MMA's layout
//     and bulk-copied per stage.  Khatri-Rao path (k_mttkrp_tc, the other
//     shapes): Khatri-Rao warps and the converters build B each stage;
//   * an MMA warp: tcgen05.mma kind::f16, FP32 accumulation in TMEM:
//     D += Xhi*KRhi + Xhi*KRlo + Xlo*KRhi  (BF16X3), or one product (BF16,
//     FP16).
// The tensor core's FP32 accumulation truncates, so long accumulation chains
// drift low; the CTA's stage range is therefore cut into segments of at most
// SEG stages, each accumulated in its own TMEM buffer (two, alternating), and
// the converters add each finished segment into the CTA's FP32 partial in
// global memory with round-to-nearest reductions (`red.add`, fire and
// forget; each partial element has one owning thread, so the order of the
// adds is fixed and the result deterministic).  A small second kernel sums the
// partials over the contraction splits in FP64.  The unfolding and the KR
// matrix are never materialised: X is read from HBM exactly once.
//
// Every wait is bounded: an expired wait raises a CTA-wide abort flag, the
// roles drain and the TMEM is freed before the CTA exits, and the kernel's
// error flag is set (the reduce then writes NaN).
#include <atomic>
#include <cuda.h>
#include <cudaTypedefs.h>

#include "kernels.cuh"
#include "tc_ptx.cuh"

namespace cud {

namespace {

constexpr int BQ = 128;          // rows per CTA tile (MMA M)
constexpr int BKS = 32;          // contraction depth per stage (two MMA K-steps of 16)
constexpr int NXMAX = 8;         // X tiles in flight (deep: hides DRAM latency)
constexpr int NBMAX = 4;         // U / B / A stages (shallow: feeds the MMA)
#ifndef CUD_TC_SEG
#define CUD_TC_SEG 16
#endif
constexpr int SEG = CUD_TC_SEG;  // stages per TMEM accumulation segment
#ifndef CUD_TC_KR_ITEMS
#define CUD_TC_KR_ITEMS 64  // B items per stage made by the KR warp (two CTAs per SM; twice that with one)
#endif
constexpr int NTHREADS = 384;    // w0 TMA, w1 MMA, w2-9 A converters, w10-11 KR producers
constexpr int NCONV = 256;       // A converter threads: two groups of one warp per TMEM lane quarter
constexpr int GROUPS = 2;        // converter groups (stages i with i % GROUPS == group)
constexpr int GCONV = NCONV / GROUPS;  // converter threads per stage
constexpr int FLUSH_GRP = (CUD_TC_SEG - 1) % GROUPS;  // converts each segment's last stage
static_assert(CUD_TC_SEG % GROUPS == 0, "segments hold whole converter rounds");
constexpr int NKR = 64;          // KR producer threads: one warp per stage parity
constexpr int KRW = NKR / GROUPS;  // KR producer threads per stage
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
    int nx, nb;        // X ring and U/B/A ring depths of this launch
    int nkri;          // B items (row, 8-kappa chunk) made by the KR warps; the converters make the rest
    long Rp;           // partial row width: R rounded up to a multiple of 4
    KrFactors gen;     // kind 0: factors after mode 0; kind 1: factors before the mode
    KrFactors outer;   // kind 1: factors after the mode (one constant row per stage)
    float *part;       // [split][Q][Rp]
    int *error;        // device flag
    const uint8_t *pb; // pre-packed B path: blk B tiles (hi, lo) of the folded factors' Khatri-Rao rows
    long blk;          // stages per constant-row block (folded rows / 32)
    int fold;          // pre-packed B path: factors folded into B, counted along gen then outer
    long frows;        // pre-packed B path: product of the folded factors' rows (= 32 * blk)
    int pack_pdl;      // pre-packed B path: the pack was launched programmatically (may overlap
                       // the kernel before it), so factor reads wait for the pack grid
};

struct TcCtrl {
    uint64_t full_x[NXMAX], empty_x[NXMAX];                       // X tiles
    uint64_t full_u[NBMAX], empty_u[NBMAX], full_a[NBMAX], empty_a[NBMAX];  // U tiles, A + B operands
    uint64_t d_full[2], d_free[2], done;
    const float *gU[kMaxOrder];
    const float *oU[kMaxOrder];
    long grows[kMaxOrder], orows[kMaxOrder];
    uint32_t tmem_base;
    int abort;
};

constexpr size_t CTRL_BYTES = (sizeof(TcCtrl) + 1023) & ~size_t(1023);

__host__ __device__ constexpr size_t b_tile_bytes(int Rpad) { return (size_t)Rpad * BKS * 2; }

// one U/B stage: (fast path) the U tile of Rpad x 32 FP32, B hi + lo
__host__ __device__ constexpr size_t tc_ub_bytes(int Rpad, bool fast) {
    return (fast ? (size_t)Rpad * 128 : 0) + 2 * b_tile_bytes(Rpad);
}

__host__ __device__ constexpr size_t tc_smem_bytes(int Rpad, bool fast, int nx, int nb) {
    return 1024 + CTRL_BYTES + (size_t)nx * X_STAGE_BYTES + (size_t)nb * tc_ub_bytes(Rpad, fast);
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

// Per-stage Khatri-Rao values of one producer item (row r, 8-kappa chunk kc)
// on the general path (any factor shapes): computed from global memory.
// Indices fit 32 bits (tc_plan checks every extent), so the digit
// arithmetic uses 32-bit unsigned division.
__device__ __forceinline__ void kr_general(const TcArgs &a, const TcCtrl &sm, long g, int r, int kc, float (&v)[8]) {
    const uint32_t gs = (uint32_t)g, ps = (uint32_t)a.psteps;
    uint32_t k0, kmax, s;
    if (a.kind == 0) { k0 = gs * BKS; kmax = (uint32_t)a.S; s = 0; }
    else { s = gs / ps; k0 = (gs - s * ps) * BKS; kmax = (uint32_t)a.P; }
    float c = 1.f;
    uint32_t lin = s;
    for (int f = 0; f < a.outer.n; f++) {
        const uint32_t d = (uint32_t)sm.orows[f];
        const uint32_t qd = lin / d;
        c *= __ldg(sm.oU[f] + (lin - qd * d) + (long)r * d);
        lin = qd;
    }
#pragma unroll
    for (int j = 0; j < 8; j++) {
        const uint32_t k = k0 + kc * 8 + j;
        float x = 0.f;
        if (k < kmax) {
            x = c;
            uint32_t l2 = k;
            for (int f = 0; f < a.gen.n; f++) {
                const uint32_t d = (uint32_t)sm.grows[f];
                const uint32_t qd = l2 / d;
                x *= __ldg(sm.gU[f] + (l2 - qd * d) + (long)r * d);
                l2 = qd;
            }
        }
        v[j] = x;
    }
}

// B item `id` -> (row r, 8-kappa chunk kc): 32 consecutive ids cover 8 rows x
// 4 chunks, so a quarter-warp stores 128 contiguous bytes of the B tile.
// Position in a ring of n slots: stage i sits in slot i % n for the
// (i / n)-th time, advanced by one per stage without dividing.
struct Ring {
    int slot, n;
    long use;
    __device__ explicit Ring(int n_) : slot(0), n(n_), use(0) {}
    __device__ __forceinline__ void next() {
        if (++slot == n) {
            slot = 0;
            ++use;
        }
    }
    // advance by `step` stages (step <= n)
    __device__ __forceinline__ void next(int step) {
        slot += step;
        if (slot >= n) {
            slot -= n;
            ++use;
        }
    }
    // parity of the slot's previous phase (the one a producer waits out)
    __device__ __forceinline__ uint32_t prev_parity() const { return (uint32_t)((use - 1) & 1); }
};

// Parity waits and ring depths.  A consumer that visits every GROUPS-th
// stage waits on a slot whose phases, with an odd ring depth, alternate
// between it and the other group; a parity wait is only exact when the
// barrier has already completed the phase before the awaited one.  Every
// consumer therefore first waits for the MMA of stage i - nb (empty_a): that
// MMA ran after the other group's full_a arrival for stage i - nb, which came
// after its own full_x / full_u waits for that stage, so the X and U slots'
// previous phases are complete (the X ring is as deep as the A/B ring).

__device__ __forceinline__ void b_item(int id, int &r, int &kc) {
    r = ((id >> 5) << 3) | (id & 7);
    kc = (id >> 3) & 3;
}

// The 8 raw Khatri-Rao inputs of B item (r, kc) from the stage's U tile in
// shared memory (128-byte swizzled: row r's 16-byte chunk c at c ^ (r & 7)).
__device__ __forceinline__ void load_u_item(const float *us, int r, int kc, float4 &u0, float4 &u1) {
    u0 = *reinterpret_cast<const float4 *>(us + r * BKS + (((2 * kc) ^ (r & 7)) << 2));
    u1 = *reinterpret_cast<const float4 *>(us + r * BKS + (((2 * kc + 1) ^ (r & 7)) << 2));
}

// Packs 16 consecutive contraction values x[k0..k0+15] of an A row into 8
// hi words (and, for BF16x3, 8 lo words), two values per word.
__device__ __forceinline__ void split_half(const float (&x)[BKS], int k0, uint32_t (&hi)[8], uint32_t (&lo)[8],
                                           bool three, bool f16) {
#pragma unroll
    for (int c = 0; c < 8; c++) {
        const float a0 = x[k0 + 2 * c], a1 = x[k0 + 2 * c + 1];
        lo[c] = 0u;
        if (f16) hi[c] = pack_f16(a0, a1);
        else if (three) split_pair(a0, a1, hi[c], lo[c]);
        else hi[c] = pack_bf16(a0, a1);
    }
}

// Rounds / splits the 8 Khatri-Rao values of a B item into its hi (and, for
// BF16x3, lo) words.
__device__ __forceinline__ void pack_b_item(const float (&v)[8], uint4 &h, uint4 &l, bool three, bool f16) {
    l = make_uint4(0u, 0u, 0u, 0u);
    if (f16) {
        h.x = pack_f16(v[0], v[1]); h.y = pack_f16(v[2], v[3]);
        h.z = pack_f16(v[4], v[5]); h.w = pack_f16(v[6], v[7]);
    } else if (three) {
        split_pair(v[0], v[1], h.x, l.x); split_pair(v[2], v[3], h.y, l.y);
        split_pair(v[4], v[5], h.z, l.z); split_pair(v[6], v[7], h.w, l.w);
    } else {
        h.x = pack_bf16(v[0], v[1]); h.y = pack_bf16(v[2], v[3]);
        h.z = pack_bf16(v[4], v[5]); h.w = pack_bf16(v[6], v[7]);
    }
}

// Fast path: the words of B item (r, kc) from the U values u0, u1 times the
// constant row c.
__device__ __forceinline__ void fast_b_item(float c, float4 u0, float4 u1, uint4 &h, uint4 &l, bool three,
                                            bool f16) {
    const float v[8] = {u0.x * c, u0.y * c, u0.z * c, u0.w * c, u1.x * c, u1.y * c, u1.z * c, u1.w * c};
    pack_b_item(v, h, l, three, f16);
}

// Stores B item (r, kc) into the canonical (K-major, no swizzle) B layout.
__device__ __forceinline__ void store_b_item(const TcArgs &a, int r, int kc, uint4 h, uint4 l, uint8_t *bh,
                                             uint8_t *bl, bool three) {
    const uint32_t off = (uint32_t)r * 16u + (uint32_t)kc * (uint32_t)a.Rpad * 16u;
    *reinterpret_cast<uint4 *>(bh + off) = h;
    if (three) *reinterpret_cast<uint4 *>(bl + off) = l;
}

// General path: B item (r, kc) of stage g from the factors in global memory.
__device__ __forceinline__ void general_b_item(const TcArgs &a, const TcCtrl &sm, long g, int r, int kc,
                                               uint8_t *bh, uint8_t *bl, bool three, bool f16) {
    float v[8];
    if (r < a.R) {
        kr_general(a, sm, g, r, kc, v);
    } else {
#pragma unroll
        for (int j = 0; j < 8; j++) v[j] = 0.f;
    }
    uint4 h, l;
    pack_b_item(v, h, l, three, f16);
    store_b_item(a, r, kc, h, l, bh, bl, three);
}

// The constant row of the fast path for the block of stages starting at g:
// the product over the slower generating factors (digits of kappa / rows0)
// and the outer factors (digits of s) of their row for column r (32-bit
// digit arithmetic, as above).
template <class Ctrl>
__device__ __forceinline__ float kr_const_row(const TcArgs &a, const Ctrl &sm, long g, int r) {
    const uint32_t gs = (uint32_t)g, ps = (uint32_t)a.psteps;
    uint32_t k0, s;
    if (a.kind == 0) { k0 = gs * BKS; s = 0; }
    else { s = gs / ps; k0 = (gs - s * ps) * BKS; }
    float c = 1.f;
    uint32_t lin = k0 / (uint32_t)sm.grows[0];
    for (int f = 1; f < a.gen.n; f++) {
        const uint32_t d = (uint32_t)sm.grows[f];
        const uint32_t qd = lin / d;
        c *= __ldg(sm.gU[f] + (lin - qd * d) + (long)r * d);
        lin = qd;
    }
    lin = s;
    for (int f = 0; f < a.outer.n; f++) {
        const uint32_t d = (uint32_t)sm.orows[f];
        const uint32_t qd = lin / d;
        c *= __ldg(sm.oU[f] + (lin - qd * d) + (long)r * d);
        lin = qd;
    }
    return c;
}

template <int KIPT, int CIPT, int MINB>
__global__ void __launch_bounds__(NTHREADS, MINB)
    k_mttkrp_tc(const __grid_constant__ CUtensorMap tmap, const __grid_constant__ CUtensorMap umap, TcArgs a) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t *base = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    TcCtrl &sm = *reinterpret_cast<TcCtrl *>(base);
    const int nx = a.nx, nb = a.nb;
    uint8_t *xring = base + CTRL_BYTES;                        // nx X tiles
    uint8_t *ubring = xring + (size_t)nx * X_STAGE_BYTES;      // nb (U tile, B hi, B lo)
    const uint32_t ubytes = a.fast ? (uint32_t)a.Rpad * 128u : 0u;   // U tile: Rpad x 32 FP32
    const uint32_t bbytes = (uint32_t)b_tile_bytes(a.Rpad);          // one B operand (hi or lo)
    const uint32_t ubstage = ubytes + 2u * bbytes;
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
        // consumer / producer counts are warps: lane 0 arrives for its warp
        // after __syncwarp
        for (int i = 0; i < NXMAX; i++) {
            ptx::mbar_init(&sm.full_x[i], 1);
            ptx::mbar_init(&sm.empty_x[i], GCONV / 32);
        }
        for (int i = 0; i < NBMAX; i++) {
            ptx::mbar_init(&sm.full_u[i], 1);
            ptx::mbar_init(&sm.empty_u[i], KRW / 32 + (CIPT > 0 ? GCONV / 32 : 0));
            ptx::mbar_init(&sm.full_a[i], (GCONV + KRW) / 32);
            ptx::mbar_init(&sm.empty_a[i], 1);
        }
        for (int b = 0; b < 2; b++) {
            ptx::mbar_init(&sm.d_full[b], 1);
            ptx::mbar_init(&sm.d_free[b], 4);  // the flushing group's four warps
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
        if (a.fast) ptx::prefetch_tmap(&umap);
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

    long issued_x = 0, issued_u = 0;  // TMA loads issued (producer thread)
    if (warp == 0) {
        // ------------------------------------------------------------ TMA producer
        if (lane == 0) {
            // stage coordinates advance by counters (no division in the loop):
            // kind 1 stage g = s * psteps + p; uk = first kappa of the stage
            // modulo the fastest generating factor's rows
            Ring xr(nx), ur(nb);
            long ks = (a.kind == 0) ? 0 : st_beg / a.psteps;
            long kp = (a.kind == 0) ? st_beg : st_beg % a.psteps;
            const long rows0 = sm.grows[0];
            long uk = a.fast ? (kp * BKS) % rows0 : 0;
            for (long i = 0; i < nst && !*abort; i++) {
                {
                    if (xr.use > 0 && !ptx::mbar_wait(&sm.empty_x[xr.slot], xr.prev_parity(), abort)) break;
                    uint8_t *dst = xring + (size_t)xr.slot * X_STAGE_BYTES;
                    ptx::mbar_arrive_expect_tx(&sm.full_x[xr.slot], (uint32_t)X_STAGE_BYTES);
                    if (a.kind == 0) {
                        ptx::tma_load_2d(dst, &tmap, &sm.full_x[xr.slot], (int)q0, (int)(kp * BKS));
                    } else {
                        ptx::tma_load_3d(dst, &tmap, &sm.full_x[xr.slot], (int)(kp * BKS), (int)q0, (int)ks);
                    }
                    issued_x = i + 1;
                }
                if (a.fast) {
                    if (ur.use > 0 && !ptx::mbar_wait(&sm.empty_u[ur.slot], ur.prev_parity(), abort)) break;
                    ptx::mbar_arrive_expect_tx(&sm.full_u[ur.slot], ubytes);
                    ptx::tma_load_2d(ubring + (size_t)ur.slot * ubstage, &umap, &sm.full_u[ur.slot], (int)uk, 0);
                    issued_u = i + 1;
                }
                xr.next();
                ur.next();
                kp++;
                uk += BKS;
                if (uk == rows0) uk = 0;
                if (a.kind != 0 && kp == a.psteps) {
                    kp = 0;
                    ks++;
                    uk = 0;  // rows0 divides P = psteps * BKS on the fast path
                }
            }
        }
    } else if (warp == 1) {
        // ------------------------------------------------------------ MMA issuer
        if (lane == 0) {
            const uint32_t idesc = ptx::idesc_f16(f16 ? 0u : 1u, BQ, (uint32_t)a.Rpad);
            const uint32_t lbo = (uint32_t)a.Rpad * 16u;
            Ring ar(nb);
            for (long i = 0; i < nst; i++, ar.next()) {
                const int slot = ar.slot;
                const long use = ar.use;
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
                const uint32_t b_hi = ptx::smem_addr(ubring + (size_t)slot * ubstage + ubytes);
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
    } else if (warp < 10) {
        // ------------------------------------------------------------ A converters
        // Two groups of four warps (one warp per TMEM lane quarter); group
        // grp converts the stages i with i % 2 == grp, all 32 contraction
        // values of its row, so two stages are converted at a time.
        const int sub = warp & 3;                 // TMEM sub-partition of this warp
        const int grp = (warp - 2) >> 2;          // stage parity of this warp's group
        const int row = sub * 32 + lane;          // row within the tile (= TMEM lane)
        const uint32_t lane_off = (uint32_t)(sub * 32) << 16;
        const long q = q0 + row;
        const int ct = row;  // converter thread within its group, 0..127
        const long blk = a.fast ? (long)(sm.grows[0] / BKS) : 1;
        long pos = a.fast ? (st_beg + grp) % blk : 0;  // stage index within its row block
        float ccv[CIPT > 0 ? CIPT : 1];
#pragma unroll
        for (int j = 0; j < (CIPT > 0 ? CIPT : 1); j++) ccv[j] = 0.f;
        float *P = a.part + (z * a.Q + q) * a.Rp;  // this row's partial (Rp floats)
        long flushed = 0;  // segments already added into the partial
        // Adds finished segment `seg` (TMEM buffer seg & 1) into the partial.
        auto flush = [&](long seg) {
            const int b = (int)(seg & 1);
            if (!*abort) ptx::mbar_wait(&sm.d_full[b], (uint32_t)((seg >> 1) & 1), abort);
            const bool ok = __all_sync(0xffffffffu, *abort == 0);  // warp-uniform tcgen05.ld
            if (ok) {
                ptx::tc_fence_after();
                const uint32_t d = tbase + lane_off + (uint32_t)b * (uint32_t)a.Rpad;
                for (int c0 = 0; c0 < a.Rpad; c0 += 16) {
                    uint32_t v[16];
                    ptx::tmem_ld16(d + (uint32_t)c0, v);
                    ptx::tmem_wait_ld();
                    if (q < a.Q) {
#pragma unroll
                        for (int j4 = 0; j4 < 4; j4++) {
                            const int c = c0 + 4 * j4;
                            if (c < a.R) {  // columns R..Rp-1 of D are zero (zero B rows)
                                const uint32_t *w = &v[j4 * 4];
                                float4 val = make_float4(__uint_as_float(w[0]), __uint_as_float(w[1]),
                                                         __uint_as_float(w[2]), __uint_as_float(w[3]));
                                float *pp = P + c;
                                if (seg == 0) *reinterpret_cast<float4 *>(pp) = val;
                                else asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(pp),
                                                  "f"(val.x), "f"(val.y), "f"(val.z), "f"(val.w)
                                                  : "memory");  // RN
                            }
                        }
                    }
                }
                ptx::tc_fence_before();
            }
            __syncwarp();
            if (lane == 0) ptx::mbar_arrive(&sm.d_free[b]);
        };
        Ring xr(nx), ar(nb);
        if (grp) {
            xr.next();
            ar.next();
        }
        for (long i = grp; i < nst; i += GROUPS, xr.next(GROUPS), ar.next(GROUPS)) {
            const int xslot = xr.slot, slot = ar.slot;
            const long xuse = xr.use, use = ar.use;
            // After an abort the loop keeps running (without waiting) so every
            // converter thread reaches the same warp-aligned tcgen05 instructions.
            if (use > 0 && !*abort) ptx::mbar_wait(&sm.empty_a[slot], (uint32_t)((use - 1) & 1), abort);
            if (!*abort) ptx::mbar_wait(&sm.full_x[xslot], (uint32_t)(xuse & 1), abort);
            if (CIPT > 0 && a.fast && !*abort) ptx::mbar_wait(&sm.full_u[slot], (uint32_t)(use & 1), abort);
            __syncwarp();
            float x[BKS];
            const float *xs = reinterpret_cast<const float *>(xring + (size_t)xslot * X_STAGE_BYTES);
            if (a.kind == 0) {
#pragma unroll
                for (int k = 0; k < BKS; k++) x[k] = xs[k * BQ + row];
            } else {
                const float4 *r4 = reinterpret_cast<const float4 *>(xs + row * BKS);
#pragma unroll
                for (int c = 0; c < BKS / 4; c++) {
                    float4 v = r4[c ^ (row & 7)];
                    x[4 * c] = v.x; x[4 * c + 1] = v.y; x[4 * c + 2] = v.z; x[4 * c + 3] = v.w;
                }
            }
            // A stage: hi in columns 0-15, lo in 16-31 (2 values per column),
            // as two halves of 16 contraction values
            uint32_t hi0[8], lo0[8], hi1[8], lo1[8];
            split_half(x, 0, hi0, lo0, three, f16);
            split_half(x, 16, hi1, lo1, three, f16);
            // A release must follow the instructions that consume the loaded
            // values: an arrive issued while a shared-memory load is still in
            // flight lets the next TMA overwrite the data under it.  The split
            // above reads every X value.
            __syncwarp();
            if (lane == 0) ptx::mbar_arrive(&sm.empty_x[xslot]);  // the X tile is consumed
            const uint32_t ta = tbase + lane_off + a_col0 + (uint32_t)slot * 32u;
            ptx::tmem_st8(ta, hi0);
            ptx::tmem_st8(ta + 8u, hi1);
            if (three) {
                ptx::tmem_st8(ta + 16u, lo0);
                ptx::tmem_st8(ta + 24u, lo1);
            }
            // this thread's share of the B tile
            if (CIPT > 0) {
                const long g = st_beg + i;
                // the constant row changed since this group's previous stage
                if (a.fast && (i == grp || pos < GROUPS)) {
#pragma unroll
                    for (int j = 0; j < CIPT; j++) {
                        const int id = a.nkri + ct + GCONV * j;
                        int r, kc;
                        b_item(id, r, kc);
                        ccv[j] = (id < 4 * a.Rpad && r < a.R) ? kr_const_row(a, sm, g, r) : 0.f;
                    }
                }
                uint8_t *bh = ubring + (size_t)slot * ubstage + ubytes;
                if (a.fast) {
                    // the items' words from the U tile; they consume every U
                    // value read, so the tile can be released after them
                    const float *us = reinterpret_cast<const float *>(ubring + (size_t)slot * ubstage);
                    uint4 ch[CIPT > 0 ? CIPT : 1], cl[CIPT > 0 ? CIPT : 1];
#pragma unroll
                    for (int j = 0; j < CIPT; j++) {
                        const int id = a.nkri + ct + GCONV * j;
                        int r, kc;
                        b_item(id < 4 * a.Rpad ? id : 0, r, kc);
                        float4 u0, u1;
                        load_u_item(us, r, kc, u0, u1);
                        fast_b_item(ccv[j], u0, u1, ch[j], cl[j], three, f16);
                    }
                    __syncwarp();
                    if (lane == 0) ptx::mbar_arrive(&sm.empty_u[slot]);
#pragma unroll
                    for (int j = 0; j < CIPT; j++) {
                        const int id = a.nkri + ct + GCONV * j;
                        if (id < 4 * a.Rpad) {
                            int r, kc;
                            b_item(id, r, kc);
                            store_b_item(a, r, kc, ch[j], cl[j], bh, bh + bbytes, three);
                        }
                    }
                } else {
#pragma unroll
                    for (int j = 0; j < CIPT; j++) {
                        const int id = a.nkri + ct + GCONV * j;
                        if (id < 4 * a.Rpad) {
                            int r, kc;
                            b_item(id, r, kc);
                            general_b_item(a, sm, g, r, kc, bh, bh + bbytes, three, f16);
                        }
                    }
                }
                ptx::fence_proxy_async_smem();  // generic-proxy B writes -> tensor core
            }
            if (a.fast) {
                pos += GROUPS;
                while (pos >= blk) pos -= blk;
            }
            ptx::tmem_wait_st();
            ptx::tc_fence_before();
            __syncwarp();
            if (lane == 0) ptx::mbar_arrive(&sm.full_a[slot]);
            // a segment just ended: drain the one before it (long finished);
            // the group converting each segment's last stage does the flushes
            if (grp == FLUSH_GRP && (i % SEG) == SEG - 1 && i / SEG >= 1) flush(flushed++);
        }
        if (grp == FLUSH_GRP)
            while (flushed < nseg) flush(flushed++);
    } else {
        // ------------------------------------------------------------ KR producers
        // one warp per stage parity, like the converter groups
        const int kgrp = warp - 10;
        const int kt = lane;
        // fast path: the stage's 32 rows of the fastest generating factor
        // arrive by TMA with X; the constant row changes every `blk` stages
        const long blk = a.fast ? (long)(sm.grows[0] / BKS) : 1;
        long pos = a.fast ? (st_beg + kgrp) % blk : 0;  // stage index within its block
        float cc[KIPT];
#pragma unroll
        for (int it = 0; it < KIPT; it++) cc[it] = 0.f;
        Ring ar(nb);
        if (kgrp) ar.next();
        for (long i = kgrp; i < nst; i += GROUPS, ar.next(GROUPS)) {
            const int slot = ar.slot;
            const long use = ar.use;
            const long g = st_beg + i;
            // the constant row changed since this warp's previous stage
            if (a.fast && (i == kgrp || pos < GROUPS)) {
#pragma unroll
                for (int it = 0; it < KIPT; it++) {
                    const int id = kt + KRW * it;
                    int r, kc;
                    b_item(id, r, kc);
                    cc[it] = (id < a.nkri && r < a.R) ? kr_const_row(a, sm, g, r) : 0.f;
                }
            }
            uint8_t *st = ubring + (size_t)slot * ubstage;
            // the slot's B tile is free once the MMA of stage i - nb is done
            if (use > 0 && !*abort) ptx::mbar_wait(&sm.empty_a[slot], (uint32_t)((use - 1) & 1), abort);
            uint4 kh[KIPT], kl[KIPT];
            if (a.fast) {
                // the U tile: make this thread's items' words (they consume
                // every U value read), then release the tile
                if (!*abort) ptx::mbar_wait(&sm.full_u[slot], (uint32_t)(use & 1), abort);
                const float *us = reinterpret_cast<const float *>(st);
#pragma unroll
                for (int it = 0; it < KIPT; it++) {
                    const int id = kt + KRW * it;
                    int r, kc;
                    b_item(id < a.nkri ? id : 0, r, kc);
                    float4 u0, u1;
                    load_u_item(us, r, kc, u0, u1);
                    fast_b_item(cc[it], u0, u1, kh[it], kl[it], three, f16);
                }
                __syncwarp();
                if (lane == 0) ptx::mbar_arrive(&sm.empty_u[slot]);
            }
            uint8_t *bh = st + ubytes;
#pragma unroll
            for (int it = 0; it < KIPT; it++) {
                const int id = kt + KRW * it;
                if (id < a.nkri) {
                    int r, kc;
                    b_item(id, r, kc);
                    if (a.fast) store_b_item(a, r, kc, kh[it], kl[it], bh, bh + bbytes, three);
                    else general_b_item(a, sm, g, r, kc, bh, bh + bbytes, three, f16);
                }
            }
            ptx::fence_proxy_async_smem();  // generic-proxy B writes -> tensor core
            __syncwarp();
            if (lane == 0) ptx::mbar_arrive(&sm.full_a[slot]);
            if (a.fast) {
                pos += GROUPS;
                while (pos >= blk) pos -= blk;
            }
        }
    }

    // ------------------------------------------------------------ teardown
    if (threadIdx.x == 0 && *abort) {
        // drain: the last load issued into each slot must land before the
        // CTA's shared memory goes away (bounded, abort flag ignored)
        for (long i = (issued_x > nx ? issued_x - nx : 0); i < issued_x; i++) {
            const uint32_t par = (uint32_t)((i / nx) & 1);
            for (long it = 0; it < 20000 && !ptx::mbar_try_wait_hint(&sm.full_x[i % nx], par, 100000u); it++) {
            }
        }
        for (long i = (issued_u > nb ? issued_u - nb : 0); i < issued_u; i++) {
            const uint32_t par = (uint32_t)((i / nb) & 1);
            for (long it = 0; it < 20000 && !ptx::mbar_try_wait_hint(&sm.full_u[i % nb], par, 100000u); it++) {
            }
        }
        atomicExch(a.error, 1);
    }
    ptx::tc_fence_before();
    __syncthreads();
    ptx::tc_fence_after();
    if (warp == 0) ptx::tmem_dealloc(tbase, a.tmem_cols);
}

// ---------------------------------------------------------------- pre-packed B path
//
// On the fast path the stage's Khatri-Rao rows are U0's 32 rows for the
// stage times one constant row c (the other factors), and c only changes
// from one block of blk = rows0 / 32 stages to the next.  With segments
// that never straddle a block, the segment's accumulation can use the
// unscaled U0 rows as B and apply c once, when the segment is flushed:
// partial[q][r] += c[r] * T[q][r].  The unscaled B tiles (one per stage
// position in a block, hi + lo, already in the MMA's canonical layout) are
// packed once per call by k_pack_b and copied into shared memory per stage
// by one bulk copy, so no warp builds B per stage.  Roles:
//   * warp 0: TMA of the X tile and bulk copy of the stage's B tile;
//   * warp 1: MMA issuer (as above);
//   * warps 2-9: A converters in two stage-parity groups (as above), the
//     odd group flushing segments, scaled by c;
//   * warp 10: the constant row c of each segment into shared memory.
constexpr int PB_THREADS = 352;

// The contraction position of stage g runs over l = 32 g .. 32 g + 31, with
// digits over the factor list F = gen followed by outer (kind 1: l = p + P s
// and P = 32 psteps).  The first `fold` factors of F are folded into the
// packed B; the constant row is the product of the remaining factors' rows
// at the digits of l / frows.
template <class Ctrl>
__device__ __forceinline__ float pb_const_row(const TcArgs &a, const Ctrl &sm, long g, int r) {
    // the block index fits 32 bits: stages < 2^31, so 32 g / frows < 2^31
    uint32_t lin = (uint32_t)(((long)g * BKS) / a.frows);
    float c = 1.f;
    for (int f = a.fold; f < a.gen.n; f++) {
        const uint32_t d = (uint32_t)sm.grows[f], qd = lin / d;
        c *= __ldg(sm.gU[f] + (lin - qd * d) + (long)r * d);
        lin = qd;
    }
    for (int f = (a.fold > a.gen.n ? a.fold - a.gen.n : 0); f < a.outer.n; f++) {
        const uint32_t d = (uint32_t)sm.orows[f], qd = lin / d;
        c *= __ldg(sm.oU[f] + (lin - qd * d) + (long)r * d);
        lin = qd;
    }
    return c;
}
constexpr int PB_RING = 6;  // deepest X ring = A/B ring

struct PbCtrl {
    uint64_t full_x[PB_RING], empty_x[PB_RING], full_a[PB_RING], empty_a[PB_RING];
    uint64_t d_full[2], d_free[2], c_full[2], done;
    const float *gU[kMaxOrder];
    const float *oU[kMaxOrder];
    long grows[kMaxOrder], orows[kMaxOrder];
    alignas(16) float cvec[2][RPAD_MAX];  // constant row of the segment in D buffer b
    uint32_t tmem_base;
    int abort;
};

constexpr size_t PB_CTRL_BYTES = (sizeof(PbCtrl) + 1023) & ~size_t(1023);

// Segmentation of a CTA's stages on the pre-packed B path: a segment ends at
// the end of every constant-row block, at every SEG-th stage of a block, and
// at the CTA's last stage, so no segment straddles a block and none is
// longer than SEG.  step() advances over one stage and tells whether it
// ends a segment.
struct SegTrack {
    uint32_t pos, blk;  // position of the next stage in its block (blk < 2^31)
    long ended;         // segments ended so far
    __device__ SegTrack(long st_beg, long blk_) : pos((uint32_t)(st_beg % blk_)), blk((uint32_t)blk_), ended(0) {}
    __device__ __forceinline__ bool step(long i, long nst) {
        static_assert((SEG & (SEG - 1)) == 0, "SEG is a power of two");
        const bool end = (pos == blk - 1) || ((pos & (SEG - 1)) == SEG - 1) || (i == nst - 1);
        if (++pos == blk) pos = 0;
        if (end) ended++;
        return end;
    }
};

__host__ __device__ constexpr size_t pb_smem_bytes(int Rpad, int n) {
    return 1024 + PB_CTRL_BYTES + (size_t)n * (X_STAGE_BYTES + 2 * b_tile_bytes(Rpad));
}

// B tiles of the pre-packed path: tile t holds the Khatri-Rao rows
// 32t..32t+31 of the folded factors (fastest first; one factor: U0's rows)
// for every column r (zero for r >= R), hi then lo, each in the canonical
// layout above.  A row's entries are formed as one FP32 product, the way the
// Khatri-Rao matrix of the reference is.  One thread per (tile, 8-row chunk
// kc, column r); consecutive threads write consecutive 16-byte chunks.
__global__ void __launch_bounds__(256) k_pack_b(KrFactors fold, long R, int Rpad, long blk, int prec,
                                                uint8_t *__restrict__ pb, int *error) {
    const long n = blk * 4 * Rpad;
    const long id = blockIdx.x * 256L + threadIdx.x;
    // this grid may have started early (launched programmatically after the
    // previous kernel, e.g. the previous mode's factor update): the factors
    // it reads and the tiles it writes wait for that kernel first
    ptx::griddep_wait();
    // the MTTKRP kernel may start now: it waits for this grid only before it
    // reads the packed tiles, and its other reads (X, the factors' constant
    // rows) need nothing from this grid -- the factors are final, since this
    // grid has passed its wait
    ptx::griddep_launch();
    if (id == 0) *error = 0;
    if (id >= n) return;
    const long t = id / (4 * Rpad);
    const int rem = (int)(id - t * 4 * Rpad);
    const int kc = rem / Rpad, r = rem - kc * Rpad;
    float v[8];
    if (fold.n == 1) {
        // U0's own rows (no index arithmetic)
#pragma unroll
        for (int j = 0; j < 8; j++) v[j] = (r < R) ? __ldg(fold.U[0] + 32 * t + 8 * kc + j + (long)r * fold.rows[0]) : 0.f;
    } else if (fold.rows[0] % 8 == 0 && (reinterpret_cast<uintptr_t>(fold.U[0]) & 15) == 0) {
        // the 8 rows 8 (4 t + kc) .. + 7 share every digit but the fastest
        // (8 divides its extent): one row of each slower factor, and 8
        // consecutive rows of the fastest as two 16-byte loads (its column r
        // starts at r * rows_0, a multiple of 8 floats).  With three or more
        // folded factors the product is formed in another order than below
        // (U_0 (U_1 U_2) against (U_0 U_1) U_2): the same value to FP32
        // rounding, ahead of the BF16 split.
        const uint32_t d0 = (uint32_t)fold.rows[0];
        uint32_t lin = (uint32_t)(32 * t + 8 * kc);  // < frows < 2^31 (the plan's bound)
        uint32_t q = lin / d0;
        const uint32_t x0 = lin - q * d0;
        float c = 1.f;
        for (int f = 1; f < fold.n; f++) {
            const uint32_t d = (uint32_t)fold.rows[f], qd = q / d;
            c *= (r < R) ? __ldg(fold.U[f] + (q - qd * d) + (long)r * d) : 0.f;
            q = qd;
        }
        float4 u0 = make_float4(0.f, 0.f, 0.f, 0.f), u1 = u0;
        if (r < R) {
            const float4 *src = reinterpret_cast<const float4 *>(fold.U[0] + x0 + (long)r * d0);
            u0 = __ldg(src);
            u1 = __ldg(src + 1);
        }
        v[0] = u0.x * c; v[1] = u0.y * c; v[2] = u0.z * c; v[3] = u0.w * c;
        v[4] = u1.x * c; v[5] = u1.y * c; v[6] = u1.z * c; v[7] = u1.w * c;
    } else {
#pragma unroll
        for (int j = 0; j < 8; j++) {
            uint32_t lin = (uint32_t)(32 * t + 8 * kc + j);  // < frows < 2^31 (the plan's bound)
            float p = 1.f;
            for (int f = 0; f < fold.n; f++) {
                const uint32_t d = (uint32_t)fold.rows[f], qd = lin / d;
                p *= (r < R) ? __ldg(fold.U[f] + (lin - qd * d) + (long)r * d) : 0.f;
                lin = qd;
            }
            v[j] = (r < R) ? p : 0.f;
        }
    }
    const bool three = (prec == CUD_PREC_BF16X3 || prec == CUD_PREC_DEFAULT);
    uint4 h, l;
    pack_b_item(v, h, l, three, prec == CUD_PREC_FP16);
    const size_t bbytes = b_tile_bytes(Rpad);
    uint8_t *tile = pb + (size_t)t * 2 * bbytes;
    const size_t off = (size_t)r * 16 + (size_t)kc * Rpad * 16;
    *reinterpret_cast<uint4 *>(tile + off) = h;
    *reinterpret_cast<uint4 *>(tile + bbytes + off) = l;
}

template <int MINB>
__global__ void __launch_bounds__(PB_THREADS, MINB)
    k_mttkrp_pb(const __grid_constant__ CUtensorMap tmap, TcArgs a) {
    extern __shared__ uint8_t smem_raw[];
    uint8_t *base = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    PbCtrl &sm = *reinterpret_cast<PbCtrl *>(base);
    const int nx = a.nx, nb = a.nb;  // equal: see the parity note at the converters
    uint8_t *xring = base + PB_CTRL_BYTES;                 // nx X tiles
    uint8_t *bring = xring + (size_t)nx * X_STAGE_BYTES;   // nb B tiles (hi, lo)
    const uint32_t bbytes = (uint32_t)b_tile_bytes(a.Rpad);
    const uint32_t bstage = 2u * bbytes;
    const uint32_t a_col0 = 2u * (uint32_t)a.Rpad;  // two D buffers first, then the A stages
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long qtile = blockIdx.x % a.qtiles;
    const long z = blockIdx.x / a.qtiles;
    const long q0 = qtile * BQ;
    const long st_beg = z * a.chunk;
    const long st_end = min(a.stages, st_beg + a.chunk);
    const long nst = st_end - st_beg;
    volatile int *abort = &sm.abort;

    if (threadIdx.x == 0) {
        for (int i = 0; i < PB_RING; i++) {
            ptx::mbar_init(&sm.full_x[i], 1);
            ptx::mbar_init(&sm.empty_x[i], GCONV / 32);
            ptx::mbar_init(&sm.full_a[i], GCONV / 32 + 1);  // converter group + the B copy
            ptx::mbar_init(&sm.empty_a[i], 1);
        }
        for (int b = 0; b < 2; b++) {
            ptx::mbar_init(&sm.d_full[b], 1);
            ptx::mbar_init(&sm.d_free[b], 4);  // the flushing group's four warps
            ptx::mbar_init(&sm.c_full[b], 1);
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

    long issued_x = 0, issued_b = 0;  // copies issued (producer thread)
    if (warp == 0) {
        // ------------------------------------------------------------ TMA producer
        if (lane == 0) {
            Ring xr(nx), br(nb);
            long ks = (a.kind == 0) ? 0 : st_beg / a.psteps;
            long kp = (a.kind == 0) ? st_beg : st_beg % a.psteps;
            long pos = st_beg % a.blk;  // stage position in its block = B tile
            bool packed = false;        // the pack kernel's tiles are visible
            for (long i = 0; i < nst && !*abort; i++) {
                if (xr.use > 0 && !ptx::mbar_wait(&sm.empty_x[xr.slot], xr.prev_parity(), abort)) break;
                uint8_t *dst = xring + (size_t)xr.slot * X_STAGE_BYTES;
                ptx::mbar_arrive_expect_tx(&sm.full_x[xr.slot], (uint32_t)X_STAGE_BYTES);
                if (a.kind == 0) ptx::tma_load_2d(dst, &tmap, &sm.full_x[xr.slot], (int)q0, (int)(kp * BKS));
                else ptx::tma_load_3d(dst, &tmap, &sm.full_x[xr.slot], (int)(kp * BKS), (int)q0, (int)ks);
                issued_x = i + 1;
                // the slot's B tile is free once the MMA of stage i - nb is done
                if (br.use > 0 && !ptx::mbar_wait(&sm.empty_a[br.slot], br.prev_parity(), abort)) break;
                if (!packed) {
                    ptx::griddep_wait();
                    packed = true;
                }
                ptx::mbar_arrive_expect_tx(&sm.full_a[br.slot], bstage);
                ptx::bulk_load(bring + (size_t)br.slot * bstage, a.pb + (size_t)pos * bstage, bstage,
                               &sm.full_a[br.slot]);
                issued_b = i + 1;
                xr.next();
                br.next();
                kp++;
                if (a.kind != 0 && kp == a.psteps) {
                    kp = 0;
                    ks++;
                }
                if (++pos == a.blk) pos = 0;  // blk divides psteps on the fast path
            }
        }
    } else if (warp == 1) {
        // ------------------------------------------------------------ MMA issuer
        if (lane == 0) {
            const uint32_t idesc = ptx::idesc_f16(f16 ? 0u : 1u, BQ, (uint32_t)a.Rpad);
            const uint32_t lbo = (uint32_t)a.Rpad * 16u;
            Ring ar(nb);
            SegTrack tr(st_beg, a.blk);
            bool seg_first = true;
            for (long i = 0; i < nst; i++) {
                const int slot = ar.slot;
                const long use = ar.use;
                const long si = tr.ended;  // segment of this stage
                const int b = (int)(si & 1);
                // the segment's D buffer must have been drained (segment si - 2)
                if (seg_first && si >= 2 &&
                    !ptx::mbar_wait(&sm.d_free[b], (uint32_t)(((si >> 1) - 1) & 1), abort)) break;
                if (!ptx::mbar_wait(&sm.full_a[slot], (uint32_t)(use & 1), abort)) break;
                ptx::tc_fence_after();
                const uint32_t d = tbase + (uint32_t)b * (uint32_t)a.Rpad;
                const uint32_t a_hi = tbase + a_col0 + (uint32_t)slot * 32u;
                const uint32_t a_lo = a_hi + 16u;
                const uint32_t b_hi = ptx::smem_addr(bring + (size_t)slot * bstage);
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
                seg_first = tr.step(i, nst);
                if (seg_first) ptx::mma_commit(&sm.d_full[b]);
                ar.next();
            }
            ptx::mma_commit(&sm.done);
            for (long it = 0; it < 40000 && !ptx::mbar_try_wait_hint(&sm.done, 0, 100000u); it++) {
            }
        }
    } else if (warp < 10) {
        // ------------------------------------------------------------ A converters
        // Two groups of four warps, group grp converting the stages i with
        // i % 2 == grp.  Parity waits: every wait here comes after the wait
        // for the MMA of stage i - nb, which ran after the other group's
        // full_x wait for that stage; with nx == nb the X slot's previous
        // phase is therefore complete and the parity is exact.
        const int sub = warp & 3;
        const int grp = (warp - 2) >> 2;
        const int row = sub * 32 + lane;
        const uint32_t lane_off = (uint32_t)(sub * 32) << 16;
        const long q = q0 + row;
        float *P = a.part + (z * a.Q + q) * a.Rp;
        long flushed = 0;
        // Adds finished segment `sg` (TMEM buffer sg & 1) times its constant
        // row into the partial.
        auto flush = [&](long sg) {
            const int b = (int)(sg & 1);
            if (!*abort) ptx::mbar_wait(&sm.d_full[b], (uint32_t)((sg >> 1) & 1), abort);
            if (!*abort) ptx::mbar_wait(&sm.c_full[b], (uint32_t)((sg >> 1) & 1), abort);
            const bool ok = __all_sync(0xffffffffu, *abort == 0);  // warp-uniform tcgen05.ld
            if (ok) {
                ptx::tc_fence_after();
                const uint32_t d = tbase + lane_off + (uint32_t)b * (uint32_t)a.Rpad;
                for (int c0 = 0; c0 < a.Rpad; c0 += 16) {
                    uint32_t v[16];
                    ptx::tmem_ld16(d + (uint32_t)c0, v);
                    ptx::tmem_wait_ld();
                    if (q < a.Q) {
#pragma unroll
                        for (int j4 = 0; j4 < 4; j4++) {
                            const int c = c0 + 4 * j4;
                            if (c < a.R) {
                                const float4 cv = *reinterpret_cast<const float4 *>(&sm.cvec[b][c]);
                                const uint32_t *w = &v[j4 * 4];
                                float4 val = make_float4(__uint_as_float(w[0]) * cv.x, __uint_as_float(w[1]) * cv.y,
                                                         __uint_as_float(w[2]) * cv.z, __uint_as_float(w[3]) * cv.w);
                                float *pp = P + c;
                                if (sg == 0) *reinterpret_cast<float4 *>(pp) = val;
                                else asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(pp),
                                                  "f"(val.x), "f"(val.y), "f"(val.z), "f"(val.w)
                                                  : "memory");  // RN
                            }
                        }
                    }
                }
                ptx::tc_fence_before();
            }
            __syncwarp();
            if (lane == 0) ptx::mbar_arrive(&sm.d_free[b]);
        };
        Ring xr(nx), ar(nb);
        // the flushing group follows the segmentation of every stage
        SegTrack tr(st_beg, a.blk);
        long tracked = 0;  // stages the tracker has passed
        if (grp) {
            xr.next();
            ar.next();
        }
        for (long i = grp; i < nst; i += GROUPS, xr.next(GROUPS), ar.next(GROUPS)) {
            const int xslot = xr.slot, slot = ar.slot;
            const long xuse = xr.use, use = ar.use;
            if (use > 0 && !*abort) ptx::mbar_wait(&sm.empty_a[slot], (uint32_t)((use - 1) & 1), abort);
            if (!*abort) ptx::mbar_wait(&sm.full_x[xslot], (uint32_t)(xuse & 1), abort);
            __syncwarp();
            float x[BKS];
            const float *xs = reinterpret_cast<const float *>(xring + (size_t)xslot * X_STAGE_BYTES);
            if (a.kind == 0) {
#pragma unroll
                for (int k = 0; k < BKS; k++) x[k] = xs[k * BQ + row];
            } else {
                const float4 *r4 = reinterpret_cast<const float4 *>(xs + row * BKS);
#pragma unroll
                for (int c = 0; c < BKS / 4; c++) {
                    float4 v = r4[c ^ (row & 7)];
                    x[4 * c] = v.x; x[4 * c + 1] = v.y; x[4 * c + 2] = v.z; x[4 * c + 3] = v.w;
                }
            }
            uint32_t hi0[8], lo0[8], hi1[8], lo1[8];
            split_half(x, 0, hi0, lo0, three, f16);
            split_half(x, 16, hi1, lo1, three, f16);
            // released after the split, which reads every loaded X value
            __syncwarp();
            if (lane == 0) ptx::mbar_arrive(&sm.empty_x[xslot]);
            const uint32_t ta = tbase + lane_off + a_col0 + (uint32_t)slot * 32u;
            ptx::tmem_st8(ta, hi0);
            ptx::tmem_st8(ta + 8u, hi1);
            if (three) {
                ptx::tmem_st8(ta + 16u, lo0);
                ptx::tmem_st8(ta + 24u, lo1);
            }
            ptx::tmem_wait_st();
            ptx::tc_fence_before();
            __syncwarp();
            if (lane == 0) ptx::mbar_arrive(&sm.full_a[slot]);
            // drain every segment whose successor has ended by now: its MMAs
            // were all issued, and the issuer waits for this drain before it
            // reuses the buffer two segments on
            if (grp == FLUSH_GRP) {
                for (; tracked <= i; tracked++) tr.step(tracked, nst);
                while (flushed + 1 < tr.ended) flush(flushed++);
            }
        }
        if (grp == FLUSH_GRP) {
            for (; tracked < nst; tracked++) tr.step(tracked, nst);
            while (flushed < tr.ended) flush(flushed++);
        }
    } else {
        // ------------------------------------------------------------ constant rows
        // after a programmatic pack launch the factors may come from a kernel
        // that ran just before the B pack (a factor update): read them only
        // once the pack grid, which waited for that kernel, has completed
        if (a.pack_pdl) ptx::griddep_wait();
        SegTrack tr(st_beg, a.blk);
        bool seg_first = true;
        for (long i = 0; i < nst; i++) {
            if (seg_first) {
                const long sg = tr.ended;
                const int b = (int)(sg & 1);
                // buffer b's previous segment (sg - 2) must have been drained
                if (sg >= 2 && !*abort) ptx::mbar_wait(&sm.d_free[b], (uint32_t)(((sg >> 1) - 1) & 1), abort);
                for (int r = lane; r < a.Rpad; r += 32)
                    sm.cvec[b][r] = (r < a.R) ? pb_const_row(a, sm, st_beg + i, r) : 0.f;
                __syncwarp();
                if (lane == 0) ptx::mbar_arrive(&sm.c_full[b]);
            }
            seg_first = tr.step(i, nst);
        }
    }

    // ------------------------------------------------------------ teardown
    if (threadIdx.x == 0 && *abort) {
        for (long i = (issued_x > nx ? issued_x - nx : 0); i < issued_x; i++) {
            const uint32_t par = (uint32_t)((i / nx) & 1);
            for (long it = 0; it < 20000 && !ptx::mbar_try_wait_hint(&sm.full_x[i % nx], par, 100000u); it++) {
            }
        }
        for (long i = (issued_b > nb ? issued_b - nb : 0); i < issued_b; i++) {
            const uint32_t par = (uint32_t)((i / nb) & 1);
            for (long it = 0; it < 20000 && !ptx::mbar_try_wait_hint(&sm.full_a[i % nb], par, 100000u); it++) {
            }
        }
        ptx::griddep_wait();  // after the pack kernel's clearing of the flag
        atomicExch(a.error, 1);
    }
    ptx::tc_fence_before();
    __syncthreads();
    ptx::tc_fence_after();
    if (warp == 0) ptx::tmem_dealloc(tbase, a.tmem_cols);
    // the split reduce may launch once every CTA got here (it waits for the
    // whole grid before reading the partials)
    ptx::griddep_launch();
}

// The same sum with one warp per output (lane l takes z = l, l + 32, ...,
// then a fixed shuffle tree), for outputs too few to fill the GPU with the
// 8-lane layout below (96 x 32 outputs at 96^4 rank 32: 96 CTAs of 37
// sequential loads each).
__global__ void __launch_bounds__(256) k_sum_tc_partials_w(const float *__restrict__ part, int splits, long Q,
                                                           long R, long Rp, const int *__restrict__ error,
                                                           float *__restrict__ out) {
    ptx::griddep_wait();  // the MTTKRP grid's partials
    const int lane = threadIdx.x & 31;
    const long e = blockIdx.x * 8L + (threadIdx.x >> 5);  // q * Rp + r
    const long n = Q * Rp;
    if (e >= n) return;  // warp-uniform
    double sum = 0.0;
#pragma unroll 4
    for (int z = lane; z < splits; z += 32) sum += (double)__ldcs(part + (long)z * n + e);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    if (lane == 0) {
        const long q = e / Rp, r = e - q * Rp;
        if (*error) sum = __longlong_as_double(0x7ff8000000000000LL);
        if (r < R) out[q + Q * r] = (float)sum;
    }
}

// Launches the split reduce in the layout that fills the GPU.
void sum_tc_partials(const float *part, int splits, long Q, long R, long Rp, const int *error, float *out,
                     cudaStream_t s);

// out[q + Q r] = sum_z part[z][q][r] in FP64, fixed order.  A CTA owns 32
// consecutive (q, r) slots of the padded partial rows (coalesced reads), each
// summed by 8 lanes over the splits z = lane, lane + 8, ..., then combined
// in lane order.
__global__ void __launch_bounds__(256) k_sum_tc_partials(const float *__restrict__ part, int splits, long Q,
                                                         long R, long Rp, const int *__restrict__ error,
                                                         float *__restrict__ out) {
    __shared__ double red[8][32];
    ptx::griddep_wait();  // the MTTKRP grid's partials
    const int o = threadIdx.x & 31, zl = threadIdx.x >> 5;
    const long e = blockIdx.x * 32L + o;  // q * Rp + r
    const long n = Q * Rp;
    double sum = 0.0;
    if (e < n) {
#pragma unroll 16
        for (int z = zl; z < splits; z += 8) sum += (double)__ldcs(part + (long)z * n + e);
    }
    red[zl][o] = sum;
    __syncthreads();
    if (zl == 0 && e < n) {
        double t = red[0][o];
        for (int k = 1; k < 8; k++) t += red[k][o];
        const long q = e / Rp, r = e - q * Rp;
        // a CTA whose bounded wait expired left its partial incomplete: the
        // output becomes NaN so the failure cannot pass for a result
        if (*error) t = __longlong_as_double(0x7ff8000000000000LL);
        if (r < R) out[q + Q * r] = (float)t;
    }
}

void sum_tc_partials(const float *part, int splits, long Q, long R, long Rp, const int *error, float *out,
                     cudaStream_t s) {
    const long n = Q * Rp;
    if ((n + 31) / 32 < 2L * kNumSMs && splits > 32) {
        PdlLaunch l((unsigned)((n + 7) / 8), 256, 0, s);
        cudaLaunchKernelEx(&l.cfg, k_sum_tc_partials_w, part, splits, Q, R, Rp, error, out);
    } else {
        PdlLaunch l((unsigned)((n + 31) / 32), 256, 0, s);
        cudaLaunchKernelEx(&l.cfg, k_sum_tc_partials, part, splits, Q, R, Rp, error, out);
    }
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
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

struct TcPlan {
    int kind;
    long P, Q, S, Rpad, psteps, stages, qtiles, splits, chunk;
    bool fast;
    int nx, nb, ctas_per_sm;
    bool pb;    // pre-packed B path
    long blk;   // stages per constant-row block (fast path)
    int fold;   // pre-packed B path: factors folded into B (along gen, then outer)
    long frows; // their rows' product (= 32 blk)
};

// Pre-packed B path launch shape: the deepest rings (X and A/B equal, at
// most PB_RING) whose shared memory and TMEM fit two CTAs per SM, else one
// CTA; contraction splits filling one wave.
void pb_shape(TcPlan &p) {
    constexpr size_t kTwoCtaSmem = 115712;
    constexpr size_t kOneCtaSmem = 232448;
    p.ctas_per_sm = 0;
    for (int n = PB_RING; n >= 3 && !p.ctas_per_sm; n--)
        if (pb_smem_bytes((int)p.Rpad, n) <= kTwoCtaSmem && 2 * p.Rpad + 32 * n <= 256) {
            p.ctas_per_sm = 2;
            p.nx = p.nb = n;
        }
    for (int n = PB_RING; n >= 3 && !p.ctas_per_sm; n--)
        if (pb_smem_bytes((int)p.Rpad, n) <= kOneCtaSmem && 2 * p.Rpad + 32 * n <= 512) {
            p.ctas_per_sm = 1;
            p.nx = p.nb = n;
        }
    long want = std::max(1L, (p.ctas_per_sm * (long)kNumSMs - 2) / p.qtiles);
    p.splits = std::min(want, p.stages);
    p.chunk = (p.stages + p.splits - 1) / p.splits;
    p.splits = (p.stages + p.chunk - 1) / p.chunk;
}

// Launch shape: two CTAs per SM when their shared memory and TMEM (two D
// buffers + 32 columns per A stage, at most 256 each) fit with 3 or 4
// stages in both rings, else one CTA with 4; then enough contraction splits
// to fill every SM.  (The X ring and the U/B/A ring are separate and could
// differ in depth; a deeper X ring measured slower here.)
void tc_shape(TcPlan &p) {
    constexpr size_t kTwoCtaSmem = 115712;   // (228 KB - 2 x 1 KB reserved) / 2
    p.ctas_per_sm = 1;
    p.nx = p.nb = 4;
    for (int n = 4; n >= 3; n--) {
        if (tc_smem_bytes((int)p.Rpad, p.fast, n, n) <= kTwoCtaSmem && 2 * p.Rpad + 32 * n <= 256) {
            p.ctas_per_sm = 2;
            p.nx = p.nb = n;
            break;
        }
    }
    // one wave of CTAs, minus two slots: a sweep runs the R x R solve on a
    // second stream beside the MTTKRP, and a grid that needs every slot
    // would push one CTA into a second wave behind it
    long want = std::max(1L, (p.ctas_per_sm * (long)kNumSMs - 2) / p.qtiles);
    p.splits = std::min(want, p.stages);
    p.chunk = (p.stages + p.splits - 1) / p.splits;
    p.splits = (p.stages + p.chunk - 1) / p.chunk;
}

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
    if (p.stages > 0x7fffffffL) return false;  // 32-bit stage / digit arithmetic in the kernel
    p.qtiles = (v.Q + BQ - 1) / BQ;
    // fast KR path: the fastest generating factor's row count is a multiple
    // of 32, so each stage covers 32 of its rows (one TMA box)
    const long rows0 = (mode == 0) ? dims[1] : dims[0];
    p.fast = (rows0 % BKS == 0);
    p.blk = p.fast ? rows0 / BKS : 1;
    p.fold = 1;
    p.frows = rows0;
    // pre-packed B path: blocks of at least 2 stages (each segment flush
    // adds a whole 128 x R partial tile, at least every other stage).  Not
    // for FP16: the public mttkrp rounds each whole Khatri-Rao entry,
    // fp16(U0[x] * c[y]) (src/mttkrp.cu:21-25, 41-47, 65-69), while the
    // packed tiles hold fp16(U0[x]) and apply c in FP32 at the flush; the
    // Khatri-Rao-building kernel forms the product first and rounds it once.
    // When U0's own blocks are shorter than a segment (96 rows: a flush of
    // the whole 128 x R partial tile every 3 stages), fold the next factors
    // of the contraction (gen, then outer) into the packed B as long as the
    // packed tiles stay within kFoldBytes: the constant row then changes
    // every frows / 32 stages.
    if (p.fast && precision != CUD_PREC_FP16) {
        constexpr long kFoldBytes = 8L << 20;
        long fl[2 * kMaxOrder];
        int nf = 0;
        for (int m = 0; m < order; m++)
            if (m != mode && (p.kind == 0 || m < mode)) fl[nf++] = dims[m];
        for (int m = mode + 1; p.kind == 1 && m < order; m++) fl[nf++] = dims[m];
        while (p.frows / BKS < SEG && p.fold < nf &&
               p.frows * fl[p.fold] * p.Rpad * 4 <= kFoldBytes && p.frows * fl[p.fold] <= 0x7fffffffL) {
            p.frows *= fl[p.fold];
            p.fold++;
        }
        p.blk = p.frows / BKS;
    }
    p.pb = p.fast && p.blk >= 2 && precision != CUD_PREC_FP16;
#ifdef CUD_TC_NO_PB
    p.pb = false;
#endif
    if (p.pb) pb_shape(p);
    else tc_shape(p);
    return true;
}

// Workspace: error flag, partials [splits][Q][Rp], then (pre-packed B path)
// the packed B tiles.
size_t tc_part_bytes(const TcPlan &p, long R) {
    return (sizeof(float) * (size_t)p.splits * ((R + 3) / 4 * 4) * p.Q + 255) & ~size_t(255);
}
size_t tc_pb_bytes(const TcPlan &p) { return p.pb ? (size_t)p.blk * 2 * b_tile_bytes((int)p.Rpad) : 0; }

template <int KIPT, int CIPT, int MINB>
int launch_tc(const CUtensorMap &tmap, const CUtensorMap &umap, const TcArgs &a, size_t smem, unsigned grid,
              cudaStream_t s) {
    static std::atomic<bool> attr[64];  // per device; zero-initialised
    int dev = 0;
    CUD_CHECK(cudaGetDevice(&dev));
    if (dev >= 0 && dev < 64 && !attr[dev].load(std::memory_order_acquire)) {
        CUD_CHECK(cudaFuncSetAttribute(k_mttkrp_tc<KIPT, CIPT, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       232448));
        attr[dev].store(true, std::memory_order_release);
    }
    k_mttkrp_tc<KIPT, CIPT, MINB><<<grid, NTHREADS, smem, s>>>(tmap, umap, a);
    CUD_CHECK_LAUNCH("mttkrp_tc");
    return CUD_OK;
}

template <int MINB>
int launch_pb(const CUtensorMap &tmap, const TcArgs &a, size_t smem, unsigned grid, cudaStream_t s) {
    static std::atomic<bool> attr[64];  // per device; zero-initialised
    int dev = 0;
    CUD_CHECK(cudaGetDevice(&dev));
    if (dev >= 0 && dev < 64 && !attr[dev].load(std::memory_order_acquire)) {
        CUD_CHECK(cudaFuncSetAttribute(k_mttkrp_pb<MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize, 232448));
        attr[dev].store(true, std::memory_order_release);
    }
    PdlLaunch l(grid, PB_THREADS, smem, s);  // overlaps the B pack (see griddep_wait)
    CUD_CHECK(cudaLaunchKernelEx(&l.cfg, k_mttkrp_pb<MINB>, tmap, a));
    CUD_CHECK_LAUNCH("mttkrp_pb");
    return CUD_OK;
}

}  // namespace

int mttkrp_tc_query(int order, const long *dims, int mode, long R, int precision, size_t *ws_bytes) {
    TcPlan p;
    if (!tc_plan(order, dims, mode, R, precision, p)) return CUD_ERR_UNSUPPORTED;
    if (!encode_fn()) return CUD_ERR_UNSUPPORTED;
    if (ws_bytes) *ws_bytes = 256 + tc_part_bytes(p, R) + tc_pb_bytes(p);
    return CUD_OK;
}

int mttkrp_tc(const float *X, int order, const long *dims, const float *const *U, int mode, long R,
              float *out, int precision, void *ws, cudaStream_t s, MttkrpParts *parts) {
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
    const float *U0 = U[(mode == 0) ? 1 : 0];
    // A misaligned fastest factor takes the general KR path; the launch shape
    // (stages, splits, shared memory) stays the planned one, so the workspace
    // sized by mttkrp_tc_query still holds.
    const bool fast = p.fast && (p.pb || (reinterpret_cast<uintptr_t>(U0) & 15) == 0);
    CUtensorMap umap;
    memset(&umap, 0, sizeof(umap));
    if (fast && !p.pb) {
        // the fastest generating factor (rows0 x R, column-major): a box of
        // 32 rows x Rpad columns per stage; columns >= R read as zero
        const long rows0 = (mode == 0) ? dims[1] : dims[0];
        cuuint64_t gdim[2] = {(cuuint64_t)rows0, (cuuint64_t)R};
        cuuint64_t gstride[1] = {(cuuint64_t)rows0 * 4};
        cuuint32_t box[2] = {BKS, (cuuint32_t)p.Rpad};
        cuuint32_t estr[2] = {1, 1};
        cr = encode(&umap, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float *>(U0), gdim, gstride, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (cr != CUDA_SUCCESS) return CUD_ERR_UNSUPPORTED;
    }

    TcArgs a;
    a.P = p.P; a.Q = p.Q; a.S = p.S; a.R = R;
    a.Rpad = (int)p.Rpad;
    a.kind = p.kind;
    a.prec = precision;
    a.psteps = p.psteps;
    a.stages = p.stages;
    a.chunk = p.chunk;
    a.qtiles = p.qtiles;
    a.nx = p.nx;
    a.nb = p.nb;
    a.Rp = (R + 3) / 4 * 4;
    // B items: 4 per padded row; the stage's KR warp makes the first nkri
    // (64 with two CTAs per SM, 128 with one), the stage's converter group
    // the rest
    const int ni = 4 * (int)p.Rpad;
    a.nkri = std::min(ni, p.ctas_per_sm == 2 ? CUD_TC_KR_ITEMS : 2 * CUD_TC_KR_ITEMS);
    const int kipt_need = (a.nkri + KRW - 1) / KRW;
    const int cipt_need = (ni - a.nkri + GCONV - 1) / GCONV;
    a.gen.n = 0;
    a.outer.n = 0;
    for (int m = 0; m < order; m++) {
        if (m == mode) continue;
        KrFactors &f = (p.kind == 0 || m < mode) ? a.gen : a.outer;
        f.U[f.n] = U[m];
        f.rows[f.n] = dims[m];
        f.n++;
    }
    a.fast = fast ? 1 : 0;
    char *w = static_cast<char *>(ws);
    a.error = reinterpret_cast<int *>(w);
    a.part = reinterpret_cast<float *>(w + 256);
    a.blk = p.blk;
    a.fold = p.fold;
    a.frows = p.frows;
    a.pb = reinterpret_cast<const uint8_t *>(w + 256 + tc_part_bytes(p, R));
    if (p.pb) {
        // the pack kernel also clears the error flag (no separate memset)
        KrFactors fold;  // the first p.fold factors of gen ++ outer
        fold.n = 0;
        for (int f = 0; f < a.gen.n && fold.n < p.fold; f++, fold.n++) {
            fold.U[fold.n] = a.gen.U[f];
            fold.rows[fold.n] = a.gen.rows[f];
        }
        for (int f = 0; f < a.outer.n && fold.n < p.fold; f++, fold.n++) {
            fold.U[fold.n] = a.outer.U[f];
            fold.rows[fold.n] = a.outer.rows[f];
        }
        const long items = p.blk * 4 * p.Rpad;
        const unsigned pgrid = (unsigned)((items + 255) / 256);
        // Below 64 MiB of X the MTTKRP is short enough that the pack's launch
        // gap shows (128^3, R = 16: 4 % of a sweep), so the pack launches
        // programmatically behind the kernel before it; above, the constant-row
        // warp's early start is worth more than the hidden launch.
        a.pack_pdl = (p.P * p.Q * p.S * 4 < (64L << 20)) ? 1 : 0;
        if (a.pack_pdl) {
            PdlLaunch l(pgrid, 256, 0, s);
            CUD_CHECK(cudaLaunchKernelEx(&l.cfg, k_pack_b, fold, R, (int)p.Rpad, p.blk, precision,
                                         const_cast<uint8_t *>(a.pb), a.error));
        } else {
            k_pack_b<<<pgrid, 256, 0, s>>>(fold, R, (int)p.Rpad, p.blk, precision, const_cast<uint8_t *>(a.pb),
                                           a.error);
        }
        CUD_CHECK_LAUNCH("mttkrp_pb pack");
        a.tmem_cols = (2 * p.Rpad + p.nb * 32 <= 256) ? 256u : 512u;
        const unsigned grid = (unsigned)(p.qtiles * p.splits);
        const size_t smem = pb_smem_bytes((int)p.Rpad, p.nb);
        const int pk = prof_begin(s);
        int st = (p.ctas_per_sm == 2) ? launch_pb<2>(tmap, a, smem, grid, s) : launch_pb<1>(tmap, a, smem, grid, s);
        prof_end(pk, s);
        if (st) return st;
        if (parts) {
            *parts = MttkrpParts{a.part, p.Q * a.Rp, a.Rp, 1, (int)p.splits, a.error};
            return CUD_OK;
        }
        sum_tc_partials(a.part, (int)p.splits, p.Q, R, a.Rp, a.error, out, s);
        CUD_CHECK_LAUNCH("mttkrp_tc reduce");
        return CUD_OK;
    }
    CUD_CHECK(cudaMemsetAsync(a.error, 0, sizeof(int), s));
    // two D buffers + nst A stages of 32 columns, rounded to a power of two
    a.tmem_cols = (2 * p.Rpad + p.nb * 32 <= 256) ? 256u : 512u;
    unsigned grid = (unsigned)(p.qtiles * p.splits);
    const size_t smem = tc_smem_bytes((int)p.Rpad, p.fast, p.nx, p.nb);
    int st;
    const int pk = prof_begin(s);
    if (p.ctas_per_sm == 2) {
        if (kipt_need <= 2 && cipt_need <= 0) st = launch_tc<2, 0, 2>(tmap, umap, a, smem, grid, s);
        else if (kipt_need <= 2 && cipt_need <= 1) st = launch_tc<2, 1, 2>(tmap, umap, a, smem, grid, s);
        else if (kipt_need <= 2 && cipt_need <= 2) st = launch_tc<2, 2, 2>(tmap, umap, a, smem, grid, s);
        else return CUD_ERR_UNSUPPORTED;  // two CTAs per SM only hold Rpad <= 80 (TMEM)
    } else {
        if (kipt_need <= 4 && cipt_need <= 3) st = launch_tc<4, 3, 1>(tmap, umap, a, smem, grid, s);
        else return CUD_ERR_UNSUPPORTED;  // Rpad <= 128 needs at most 4 / 3
    }
    prof_end(pk, s);
    if (st) return st;
    if (parts) {
        *parts = MttkrpParts{a.part, p.Q * a.Rp, a.Rp, 1, (int)p.splits, a.error};
        return CUD_OK;
    }
    sum_tc_partials(a.part, (int)p.splits, p.Q, R, a.Rp, a.error, out, s);
    CUD_CHECK_LAUNCH("mttkrp_tc reduce");
    return CUD_OK;
}

}  // namespace cud
