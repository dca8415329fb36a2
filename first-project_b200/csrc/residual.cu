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
    return sizeof(double) * (2 * (size_t)gx * gy + 2);
}

int cp_residual(const float *X, int order, const long *dims, const float *const *U, long R, double *out2,
                void *ws, cudaStream_t s) {
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
    unsigned gx, gy;
    residual_grid(a.I0, a.rest, gx, gy);
    k_cp_residual<<<dim3(gx, gy), NT, 0, s>>>(a);
    CUD_CHECK_LAUNCH("cp_residual");
    k_sum_pairs<<<1, 256, 0, s>>>(a.part, (long)gx * gy, out2);
    CUD_CHECK_LAUNCH("cp_residual sum");
    return CUD_OK;
}

}  // namespace cud

using namespace cud;

extern "C" int cud_cp_residual(const float *X, int order, const long *dims, const float *const *U, long R,
                               double *res_norm2, double *x_norm2, void *stream) {
    if (!X || !dims || !U || order < 1 || order > kMaxOrder || R <= 0) return set_status(CUD_ERR_INVALID_ARGUMENT);
    for (int m = 0; m < order; m++)
        if (dims[m] <= 0 || !U[m]) return set_status(CUD_ERR_INVALID_ARGUMENT);
    cudaStream_t s = as_stream(stream);
    int st;
    const size_t bytes = cp_residual_ws_bytes(order, dims);
    double *ws = static_cast<double *>(scratch(kSlotReduce, bytes, &st));
    if (!ws) return set_status(st);
    double *out = ws + (bytes / sizeof(double) - 2);
    st = cp_residual(X, order, dims, U, R, out, ws, s);
    if (st) return set_status(st);
    double *h = pinned_scalars();
    if (!h) return set_status(CUD_ERR_NO_MEMORY);
    CUD_CHECK(cudaMemcpyAsync(h, out, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
    CUD_CHECK(cudaStreamSynchronize(s));
    if (res_norm2) *res_norm2 = h[0];
    if (x_norm2) *x_norm2 = h[1];
    return set_status(CUD_OK);
}
