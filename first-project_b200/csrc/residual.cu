// Exact CP residual: ||X - [[U_0, ..., U_{N-1}]]||^2 and ||X||^2 in one pass
// over X, without materialising the reconstruction.
//
// The reference measures a CP model's error by reconstructing the full
// tensor and taking the norm of the difference (src/rse.cu:4-15 with
// gencp, src/rse.cu:17-29; the call sits in src/cp_als.cu:104-111).  Here
// the reconstruction is formed tile by tile in registers: a CTA owns TI = 128
// rows of mode 0 and walks chunks of TJ = 32 consecutive "rest" indices (the
// other modes, mode 1 fastest).  Per chunk it builds the Khatri-Rao rows
// W[r][j] = prod_{m>=1} U_m[digit_m(rest0 + j), r] in shared memory (each
// thread decomposes one rest index and fills 8 ranks of it), each thread
// forms 2 x 8 reconstructed entries xh = sum_r U_0[i, r] W[r][j] in FP32 and
// accumulates (x - xh)^2 and x^2 in FP64.  X is read once, coalesced
// along mode 0.  Per-CTA partials are summed in a fixed order by a second
// kernel, so the result is deterministic.
//
// Shapes that allow it take an FFMA-tiled fast path (k_residual_ffma below).
//
// Unlike the fit the ALS sweep derives from its last MTTKRP
// (||X||^2 - 2<M, U> + ||Xh||^2, which cancels catastrophically when the fit
// is close to 1 and inherits the MTTKRP's rounding), this value depends only
// on X and the factors.
#include "kernels.cuh"

namespace cud {

namespace {

constexpr int TI = 128;     // mode-0 rows per CTA (two per thread)
constexpr int TJ = 32;      // rest indices per chunk
constexpr int RC = 64;      // ranks per shared-memory pass
constexpr int NT = 256;     // 64 row pairs x 4 lanes, each lane 8 rest indices

struct ResArgs {
    const float *X;
    const float *U0;
    long I0, rest, R;
    KrFactors f;            // U_1 .. U_{N-1}, fastest first
    double *part;           // [grid][2]
};

__global__ void __launch_bounds__(NT) k_cp_residual(ResArgs a) {
    __shared__ float U0s[RC][TI];
    __shared__ __align__(16) float Ws[RC][TJ];
    __shared__ double red[2][NT / 32];
    __shared__ const float *fU[kMaxOrder];
    __shared__ long fRows[kMaxOrder];
    const int nf = a.f.n;
    if (threadIdx.x == 0) {
        // staged in shared memory with constant indices: a dynamically
        // indexed kernel-parameter array would be copied to local memory
#pragma unroll
        for (int m = 0; m < kMaxOrder; m++) {
            fU[m] = m < nf ? a.f.U[m] : nullptr;
            fRows[m] = m < nf ? a.f.rows[m] : 1;
        }
    }
    __syncthreads();
    const int ti = threadIdx.x % 64;  // rows ti and ti + 64 of the tile
    const int rl = threadIdx.x / 64;  // 0..3, warp-uniform
    const long i0 = blockIdx.x * (long)TI + ti, i1 = i0 + 64;
    // KR-row builder role of this thread: rest index wj, ranks wg + 8t
    const int wj = threadIdx.x % TJ, wg = threadIdx.x / TJ;
    const long nchunks = (a.rest + TJ - 1) / TJ;
    const bool one_pass = a.R <= RC;  // U_0's tile fits: load it once
    double acc = 0.0, xx = 0.0;
    if (one_pass) {
        for (int e = threadIdx.x; e < RC * TI; e += NT) {
            const int r = e / TI, t = e % TI;
            const long i = blockIdx.x * (long)TI + t;
            U0s[r][t] = (r < a.R && i < a.I0) ? a.U0[i + a.I0 * r] : 0.f;
        }
    }
    for (long ch = blockIdx.y; ch < nchunks; ch += gridDim.y) {
        const long rest0 = ch * TJ;
        float x0[8], x1[8], h0[8], h1[8];
#pragma unroll
        for (int c = 0; c < 8; c++) {
            const long j = rest0 + rl * 8 + c;
            const bool okj = j < a.rest;
            x0[c] = (okj && i0 < a.I0) ? __ldcs(a.X + i0 + a.I0 * j) : 0.f;
            x1[c] = (okj && i1 < a.I0) ? __ldcs(a.X + i1 + a.I0 * j) : 0.f;
            h0[c] = 0.f;
            h1[c] = 0.f;
        }
        // this thread's factor rows for rest index rest0 + wj (digits once)
        const float *wb[kMaxOrder];
        long ws[kMaxOrder];
        const bool wok = rest0 + wj < a.rest;
        {
            long lin = rest0 + wj;
#pragma unroll
            for (int m = 0; m < kMaxOrder; m++) {
                wb[m] = nullptr;
                ws[m] = 0;
                if (m < nf) {
                    const long d = fRows[m];
                    wb[m] = fU[m] + (lin % d);
                    ws[m] = d;
                    lin /= d;
                }
            }
        }
        for (long rc = 0; rc < a.R; rc += RC) {
            __syncthreads();
            if (!one_pass) {
                for (int e = threadIdx.x; e < RC * TI; e += NT) {
                    const int r = e / TI, t = e % TI;
                    const long i = blockIdx.x * (long)TI + t;
                    U0s[r][t] = (rc + r < a.R && i < a.I0) ? a.U0[i + a.I0 * (rc + r)] : 0.f;
                }
            }
#pragma unroll
            for (int t = 0; t < RC / 8; t++) {
                const int r = wg + 8 * t;
                const long rr = rc + r;
                float w = 0.f;
                if (wok && rr < a.R) {
                    w = 1.f;
#pragma unroll
                    for (int m = 0; m < kMaxOrder; m++)
                        if (m < nf) w *= __ldg(wb[m] + ws[m] * rr);
                }
                Ws[r][wj] = w;
            }
            __syncthreads();
#pragma unroll 4
            for (int r = 0; r < RC; r++) {
                const float u0 = U0s[r][ti], u1 = U0s[r][ti + 64];
                const float4 w0 = *reinterpret_cast<const float4 *>(&Ws[r][rl * 8]);
                const float4 w1 = *reinterpret_cast<const float4 *>(&Ws[r][rl * 8 + 4]);
                const float w[8] = {w0.x, w0.y, w0.z, w0.w, w1.x, w1.y, w1.z, w1.w};
#pragma unroll
                for (int c = 0; c < 8; c++) {
                    h0[c] = fmaf(u0, w[c], h0[c]);
                    h1[c] = fmaf(u1, w[c], h1[c]);
                }
            }
        }
#pragma unroll
        for (int c = 0; c < 8; c++) {
            const double d0 = (double)x0[c] - (double)h0[c];
            const double d1 = (double)x1[c] - (double)h1[c];
            acc = fma(d0, d0, fma(d1, d1, acc));
            xx = fma((double)x0[c], (double)x0[c], fma((double)x1[c], (double)x1[c], xx));
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        acc += __shfl_xor_sync(0xffffffffu, acc, o);
        xx += __shfl_xor_sync(0xffffffffu, xx, o);
    }
    if ((threadIdx.x & 31) == 0) {
        red[0][threadIdx.x >> 5] = acc;
        red[1][threadIdx.x >> 5] = xx;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double s0 = 0.0, s1 = 0.0;
        for (int w = 0; w < NT / 32; w++) { s0 += red[0][w]; s1 += red[1][w]; }
        const long b = blockIdx.y * (long)gridDim.x + blockIdx.x;
        a.part[2 * b] = s0;
        a.part[2 * b + 1] = s1;
    }
}

// out[0..1] = sum over the n partial pairs, fixed order (one CTA).
__global__ void __launch_bounds__(256) k_sum_pairs(const double *part, long n, double *out) {
    __shared__ double red[2][256];
    double s0 = 0.0, s1 = 0.0;
    for (long b = threadIdx.x; b < n; b += 256) { s0 += part[2 * b]; s1 += part[2 * b + 1]; }
    red[0][threadIdx.x] = s0;
    red[1][threadIdx.x] = s1;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) {
            red[0][threadIdx.x] += red[0][threadIdx.x + w];
            red[1][threadIdx.x] += red[1][threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) { out[0] = red[0][0]; out[1] = red[1][0]; }
}

}  // namespace

int sum_pairs(const double *part, long n, double *out, cudaStream_t s) {
    k_sum_pairs<<<1, 256, 0, s>>>(part, n, out);
    CUD_CHECK_LAUNCH("cp_residual sum");
    return CUD_OK;
}

namespace {

// ---------------------------------------------------------------------------
// FFMA fast path (R <= 64, mode-0 rows a multiple of 4, U_1's rows a
// multiple of 32, X and U_1 16-byte aligned): the SGEMM-style tile of the
// plain FP32 MTTKRP, transposed.  A CTA owns RQ = 128 rows q of mode 0 with
// their U_0 rows staged once in shared memory (rank-major), and walks a
// contiguous range of RK = 32-column stages of the "rest" index; a stage's
// 32 Khatri-Rao columns are 32 consecutive rows of U_1 times one constant
// row c (the other factors' rows, fixed for a block of rows_1 / 32 stages),
// formed in FP32 into a double-buffered shared tile.  Each of the 128
// threads rebuilds an 8 x 4 patch of the reconstruction in registers
// (xh = sum_r U_0[q, r] KR[col, r], FP32, r in order), takes the difference
// with the matching X values (16-byte loads, prefetched one stage ahead)
// and adds (x - xh)^2 and x^2 of the stage in FP32 to FP64 totals.
// Per-CTA totals go to the partial pairs summed by k_sum_pairs.
constexpr int RQ = 128, RK = 32, RTH = 128, RRMAX = 64;

struct ResFArgs {
    const float *X;
    const float *U0;
    long I0, rest;
    int R, rows1;
    KrFactors f;    // U_1 .. U_{N-1}, fastest first (f.U[0] = U_1)
    long stages, chunk;
    double *part;   // [grid][2]
};

__global__ void __launch_bounds__(RTH, 3) k_residual_ffma(ResFArgs a) {
    __shared__ __align__(16) float As[RRMAX][RQ];
    __shared__ __align__(16) float Bs[2][RRMAX][RK];
    // the end-of-kernel reduction reuses the B tiles (after the last barrier)
    double(*red)[RTH / 32] = reinterpret_cast<double(*)[RTH / 32]>(&Bs[0][0][0]);
    const int t = threadIdx.x, tq = t >> 3, tk = t & 7;
    const long qtiles = (a.I0 + RQ - 1) / RQ;
    const long q0 = (blockIdx.x % qtiles) * RQ;
    const long z = blockIdx.x / qtiles;
    const long sbeg = z * a.chunk, send = min(a.stages, sbeg + a.chunk);
    const int R = a.R;
    for (int e = t; e < RRMAX * RQ; e += RTH) {
        const int r = e / RQ, q = e - r * RQ;
        As[r][q] = (r < R && q0 + q < a.I0) ? a.U0[q0 + q + a.I0 * r] : 0.f;
    }
    const int blk_stages = a.rows1 / RK;
    const long qa = q0 + 8 * tq;          // this thread's rows qa .. qa + 7
    const bool ok0 = qa < a.I0, ok1 = qa + 4 < a.I0;
    float4 rb[4], xv[4][2], xn[4][2];
    float cr[4] = {0.f, 0.f, 0.f, 0.f};
    // B slots of this thread: ranks tq + 16 i, columns 4 tk .. 4 tk + 3
    auto loadB = [&](long st) {
        const long k0 = st * RK;
        const long i1 = k0 % a.rows1;
#pragma unroll
        for (int i = 0; i < 4; i++) {
            const int r = tq + 16 * i;
            rb[i] = (r < R) ? __ldg(reinterpret_cast<const float4 *>(a.f.U[0] + i1 + 4 * tk + (long)a.rows1 * r))
                            : make_float4(0.f, 0.f, 0.f, 0.f);
        }
        if (st == sbeg || (st % blk_stages) == 0) {
            // the constant row: digits of the block index over U_2, U_3, ...
            uint32_t lin = (uint32_t)(k0 / a.rows1);
#pragma unroll
            for (int i = 0; i < 4; i++) cr[i] = (tq + 16 * i < R) ? 1.f : 0.f;
            for (int m = 1; m < a.f.n; m++) {
                const uint32_t d = (uint32_t)a.f.rows[m], qd = lin / d;
                const float *row = a.f.U[m] + (lin - qd * d);
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    const int r = tq + 16 * i;
                    if (r < R) cr[i] *= __ldg(row + (long)d * r);
                }
                lin = qd;
            }
        }
    };
    auto loadX = [&](long st, float4 (&x)[4][2]) {
        const long c0 = st * RK + 4 * tk;
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const float *p = a.X + qa + a.I0 * (c0 + c);
            x[c][0] = ok0 ? __ldcs(reinterpret_cast<const float4 *>(p)) : make_float4(0.f, 0.f, 0.f, 0.f);
            x[c][1] = ok1 ? __ldcs(reinterpret_cast<const float4 *>(p + 4)) : make_float4(0.f, 0.f, 0.f, 0.f);
        }
    };
    auto storeB = [&](int buf) {
#pragma unroll
        for (int i = 0; i < 4; i++) {
            float4 v = rb[i];
            v.x *= cr[i]; v.y *= cr[i]; v.z *= cr[i]; v.w *= cr[i];
            *reinterpret_cast<float4 *>(&Bs[buf][tq + 16 * i][4 * tk]) = v;
        }
    };
    double acc = 0.0, xx = 0.0;
    if (sbeg < send) {
        loadB(sbeg);
        storeB(0);
        loadX(sbeg, xv);
    }
    __syncthreads();
    for (long st = sbeg; st < send; st++) {
        const int cur = (int)((st - sbeg) & 1);
        const bool more = st + 1 < send;
        if (more) {
            loadB(st + 1);
            loadX(st + 1, xn);
        }
        float h[8][4];
#pragma unroll
        for (int i = 0; i < 8; i++)
#pragma unroll
            for (int c = 0; c < 4; c++) h[i][c] = 0.f;
#pragma unroll 4
        for (int r = 0; r < R; r++) {
            const float4 a0 = *reinterpret_cast<const float4 *>(&As[r][8 * tq]);
            const float4 a1 = *reinterpret_cast<const float4 *>(&As[r][8 * tq + 4]);
            const float4 b = *reinterpret_cast<const float4 *>(&Bs[cur][r][4 * tk]);
            const float av[8] = {a0.x, a0.y, a0.z, a0.w, a1.x, a1.y, a1.z, a1.w};
            const float bv[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
            for (int i = 0; i < 8; i++)
#pragma unroll
                for (int c = 0; c < 4; c++) h[i][c] = fmaf(av[i], bv[c], h[i][c]);
        }
        float sr = 0.f, sx = 0.f;
#pragma unroll
        for (int c = 0; c < 4; c++) {
            const float x[8] = {xv[c][0].x, xv[c][0].y, xv[c][0].z, xv[c][0].w,
                                xv[c][1].x, xv[c][1].y, xv[c][1].z, xv[c][1].w};
#pragma unroll
            for (int i = 0; i < 8; i++) {
                const float d = x[i] - h[i][c];
                sr = fmaf(d, d, sr);
                sx = fmaf(x[i], x[i], sx);
            }
        }
        // rows past I0 read zeros: their h is zero too (U_0 rows zero)
        acc += (double)sr;
        xx += (double)sx;
        if (more) {
            storeB(cur ^ 1);
#pragma unroll
            for (int c = 0; c < 4; c++) { xv[c][0] = xn[c][0]; xv[c][1] = xn[c][1]; }
        }
        __syncthreads();
    }
    for (int o = 16; o > 0; o >>= 1) {
        acc += __shfl_xor_sync(0xffffffffu, acc, o);
        xx += __shfl_xor_sync(0xffffffffu, xx, o);
    }
    if ((t & 31) == 0) {
        red[0][t >> 5] = acc;
        red[1][t >> 5] = xx;
    }
    __syncthreads();
    if (t == 0) {
        double s0 = 0.0, s1 = 0.0;
        for (int w = 0; w < RTH / 32; w++) { s0 += red[0][w]; s1 += red[1][w]; }
        a.part[2 * blockIdx.x] = s0;
        a.part[2 * blockIdx.x + 1] = s1;
    }
}

// Launch plan of the fast path; false when the shape or R does not allow it.
bool residual_ffma_plan(int order, const long *dims, long R, long &qtiles, long &stages, long &chunk,
                        long &splits) {
    if (order < 2 || R <= 0 || R > RRMAX) return false;
    const long I0 = dims[0], rows1 = dims[1];
    if (I0 % 4 != 0 || rows1 % RK != 0 || I0 > 0x7fffffffL) return false;
    long rest = 1;
    for (int m = 1; m < order; m++) {
        if (dims[m] > 0x7fffffffL) return false;
        rest *= dims[m];
    }
    qtiles = (I0 + RQ - 1) / RQ;
    stages = rest / RK;
    if (rest / rows1 > 0xffffffffL) return false;  // block index in 32 bits
    const long want = (3L * kNumSMs + qtiles - 1) / qtiles;
    splits = std::max(1L, std::min(want, stages));
    chunk = (stages + splits - 1) / splits;
    splits = (stages + chunk - 1) / chunk;
    return qtiles * splits <= 0x7fffffffL;
}

void residual_grid(long I0, long rest, unsigned &gx, unsigned &gy) {
    gx = (unsigned)((I0 + TI - 1) / TI);
    const long nchunks = (rest + TJ - 1) / TJ;
    long want = std::max(1L, (8L * kNumSMs) / (long)gx);
    gy = (unsigned)std::min(std::min(want, nchunks), 65535L);
}

}  // namespace

size_t cp_residual_ws_bytes(int order, const long *dims) {
    long rest = 1;
    for (int m = 1; m < order; m++) rest *= dims[m];
    unsigned gx, gy;
    residual_grid(dims[0], rest, gx, gy);
    size_t parts = (size_t)gx * gy;
    long qt, st, ch, sp;
    // the fast path's grid, for any rank (the partials are all it needs)
    if (residual_ffma_plan(order, dims, 1, qt, st, ch, sp)) parts = std::max(parts, (size_t)(qt * sp));
    int tcg = 0;  // the tensor-core path's grid, for any rank it takes
    if (residual_tc_plan(order, dims, 1, &tcg)) parts = std::max(parts, (size_t)tcg);
    return sizeof(double) * (2 * parts + 2);
}

int cp_residual(const float *X, int order, const long *dims, const float *const *U, long R, double *out2,
                void *ws, cudaStream_t s, bool need_x2 = true) {
    if (order < 1 || order > kMaxOrder || R <= 0) return CUD_ERR_INVALID_ARGUMENT;
    ResArgs a;
    a.X = X;
    a.U0 = U[0];
    a.I0 = dims[0];
    a.R = R;
    a.rest = 1;
    a.f.n = 0;
    for (int m = 1; m < order; m++) {
        a.rest *= dims[m];
        a.f.U[a.f.n] = U[m];
        a.f.rows[a.f.n] = dims[m];
        a.f.n++;
    }
    a.part = static_cast<double *>(ws);
    {
        const int st = residual_tc(X, order, dims, U, R, a.part, out2, s, need_x2);
        if (st != CUD_ERR_UNSUPPORTED) return st;
    }
    long qt, stg, ch, sp;
    if (residual_ffma_plan(order, dims, R, qt, stg, ch, sp) && ((reinterpret_cast<uintptr_t>(X) |
                                                               reinterpret_cast<uintptr_t>(U[1])) & 15) == 0) {
        ResFArgs f;
        f.X = X;
        f.U0 = U[0];
        f.I0 = dims[0];
        f.rest = a.rest;
        f.R = (int)R;
        f.rows1 = (int)dims[1];
        f.f = a.f;
        f.stages = stg;
        f.chunk = ch;
        f.part = a.part;
        k_residual_ffma<<<(unsigned)(qt * sp), RTH, 0, s>>>(f);
        CUD_CHECK_LAUNCH("cp_residual ffma");
        k_sum_pairs<<<1, 256, 0, s>>>(a.part, qt * sp, out2);
        CUD_CHECK_LAUNCH("cp_residual sum");
        return CUD_OK;
    }
    unsigned gx, gy;
    residual_grid(a.I0, a.rest, gx, gy);
    k_cp_residual<<<dim3(gx, gy), NT, 0, s>>>(a);
    CUD_CHECK_LAUNCH("cp_residual");
    k_sum_pairs<<<1, 256, 0, s>>>(a.part, (long)gx * gy, out2);
    CUD_CHECK_LAUNCH("cp_residual sum");
    return CUD_OK;
}

int cp_residual_host(const float *X, int order, const long *dims, const float *const *U, long R, bool need_x2,
                     double *res_norm2, double *x_norm2, cudaStream_t s) {
    int st;
    const size_t bytes = cp_residual_ws_bytes(order, dims);
    double *ws = static_cast<double *>(scratch(kSlotReduce, bytes, &st));
    if (!ws) return st;
    double *out = ws + (bytes / sizeof(double) - 2);
    st = cp_residual(X, order, dims, U, R, out, ws, s, need_x2);
    if (st) return st;
    double *h = pinned_scalars();
    if (!h) return CUD_ERR_NO_MEMORY;
    CUD_CHECK(cudaMemcpyAsync(h, out, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
    CUD_CHECK(cudaStreamSynchronize(s));
    if (res_norm2) *res_norm2 = h[0];
    if (x_norm2) *x_norm2 = h[1];
    return CUD_OK;
}

}  // namespace cud

using namespace cud;

extern "C" int cud_cp_residual(const float *X, int order, const long *dims, const float *const *U, long R,
                               double *res_norm2, double *x_norm2, void *stream) {
    if (!X || !dims || !U || order < 1 || order > kMaxOrder || R <= 0) return set_status(CUD_ERR_INVALID_ARGUMENT);
    for (int m = 0; m < order; m++)
        if (dims[m] <= 0 || !U[m]) return set_status(CUD_ERR_INVALID_ARGUMENT);
    return set_status(cp_residual_host(X, order, dims, U, R, true, res_norm2, x_norm2, as_stream(stream)));
}
