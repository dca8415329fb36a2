// FP64 CP-ALS: the reference's double-precision variants
// decomposition/GPU/normal/dprice/cp_als.cu:3-212 (order 3) and
// dprice/4_cp_als.cu:3-229 (order 4) -- the same ALS sweep as src/cp_als.cu
// (MTTKRP through a Khatri-Rao DGEMM, Hadamard of the factor Grams, LU
// solve) with `typedef double dt` -- as one general-order entry over device
// pointers, like cud_cp_als.
//
// Per mode: the CUDA-core MTTKRP on FP64 data (mttkrp_simt.cu, no
// Khatri-Rao matrix), V = Hadamard of the other FP64 Grams and its inverse
// (solve.cu's normal_inverse: Gauss-Jordan with Cholesky's pivots, Jacobi
// pseudo-inverse fallback), U = M V^-1 and the new factor's Gram.  The fit
// after each sweep comes from the Gram identity
//     ||X - Xhat||^2 = ||X||^2 - 2 <M_N, U_N> + sum_rs prod_m G_m[r, s],
// every sum formed in a fixed order (deterministic), and drives the Δfit /
// target-fit stops.  Everything stays FP64; there is no reduced-precision
// path here.
#include <chrono>

#include "kernels.cuh"
#include "solve.cuh"

namespace cud {

namespace {

constexpr int F64_PARTS = 296;  // CTAs of the dot-product partial pass

// U (I x R) = M (I x R) Vinv (R x R), column-major, FP64.
__global__ void k_apply_inverse_f64(const double *__restrict__ M, const double *__restrict__ Vinv, long I, long R,
                                    double *__restrict__ U) {
    const long n = I * R;
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) {
        const long i = e % I, c = e / I;
        double s = 0.0;
        for (long r = 0; r < R; r++) s = fma(M[i + I * r], Vinv[r + R * c], s);
        U[e] = s;
    }
}

// part[b] = sum over this CTA's grid-stride elements of a[e] b[e] (the
// warps' sums added in warp order).
__global__ void __launch_bounds__(256) k_dot_parts(const double *__restrict__ a, const double *__restrict__ b,
                                                   long n, double *__restrict__ part) {
    __shared__ double red[8];
    double t = 0.0;
    for (long e = blockIdx.x * 256L + threadIdx.x; e < n; e += (long)gridDim.x * 256L) t = fma(a[e], b[e], t);
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < 8; w++) s += red[w];
        part[blockIdx.x] = s;
    }
}

struct GramList {
    const double *G[kMaxOrder];
    int n;
};

// out[0] = sum of the nparts partials in order; out[1] = sum_rs prod_m
// G_m[r, s] (when gl.n > 0).  One CTA.
__global__ void __launch_bounds__(256) k_fit_terms_f64(const double *__restrict__ part, int nparts, GramList gl,
                                                       long R, double *__restrict__ out) {
    __shared__ double red[8];
    double h = 0.0;
    for (long e = threadIdx.x; e < R * R; e += 256) {
        double p = 1.0;
        for (int m = 0; m < gl.n; m++) p *= gl.G[m][e];
        h += p;
    }
    for (int o = 16; o > 0; o >>= 1) h += __shfl_xor_sync(0xffffffffu, h, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = h;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int b = 0; b < nparts; b++) s += part[b];
        double hh = 0.0;
        for (int w = 0; w < 8; w++) hh += red[w];
        out[0] = s;
        out[1] = hh;
    }
}

int dot_f64(const double *a, const double *b, long n, double *part, double *out, cudaStream_t s) {
    k_dot_parts<<<F64_PARTS, 256, 0, s>>>(a, b, n, part);
    GramList none;
    none.n = 0;
    k_fit_terms_f64<<<1, 256, 0, s>>>(part, F64_PARTS, none, 1, out);
    CUD_CHECK_LAUNCH("dot_f64");
    return CUD_OK;
}

}  // namespace

}  // namespace cud

using namespace cud;

extern "C" int cud_mttkrp_f64(const double *X, int order, const long *dims, const double *const *U, int mode,
                              long R, double *out, void *stream) {
    if (order < 2 || order > kMaxOrder || !dims || mode < 0 || mode >= order || R <= 0 || !X || !U || !out)
        return set_status(CUD_ERR_INVALID_ARGUMENT);
    for (int m = 0; m < order; m++) {
        if (dims[m] <= 0) return set_status(CUD_ERR_INVALID_ARGUMENT);
        if (m != mode && !U[m]) return set_status(CUD_ERR_INVALID_ARGUMENT);
    }
    int st;
    void *ws = scratch(kSlotMttkrp, mttkrp_simt_f64_ws_bytes(order, dims, mode, R), &st);
    if (!ws) return set_status(st);
    return set_status(mttkrp_simt_f64(X, order, dims, U, mode, R, out, ws, as_stream(stream)));
}

extern "C" int cud_cp_als_f64(const double *X, int order, const long *dims, long R, double *const *U,
                              const cud_cp_options *opt_in, cud_cp_result *res, void *stream) {
    if (order < 2 || order > kMaxOrder || !dims || R <= 0 || R > 160 || !X || !U)
        return set_status(CUD_ERR_INVALID_ARGUMENT);
    long total = 1, maxd = 0;
    for (int m = 0; m < order; m++) {
        if (dims[m] <= 0 || !U[m]) return set_status(CUD_ERR_INVALID_ARGUMENT);
        total *= dims[m];
        maxd = std::max(maxd, dims[m]);
    }
    cud_cp_options opt;
    cud_cp_default_options(&opt);
    if (opt_in) opt = *opt_in;
    if (opt.max_sweeps < 0) return set_status(CUD_ERR_INVALID_ARGUMENT);
    cudaStream_t s = as_stream(stream);

    // workspace: MTTKRP partials | M | Grams | Vinv | inverse scratch | dot partials | scalars
    size_t mws = 0;
    for (int m = 0; m < order; m++) mws = std::max(mws, mttkrp_simt_f64_ws_bytes(order, dims, m, R));
    auto up = [](size_t b) { return (b + 255) & ~size_t(255); };
    const size_t o_m = up(mws), o_g = o_m + up(8 * (size_t)maxd * R), o_v = o_g + up(8 * (size_t)order * R * R),
                 o_w = o_v + up(8 * (size_t)R * R), o_p = o_w + up(8 * (size_t)2 * R * R + 64),
                 o_s = o_p + up(8 * (size_t)F64_PARTS), bytes = o_s + 256;
    int st;
    char *w = static_cast<char *>(scratch(kSlotTmp2, bytes, &st));
    if (!w) return set_status(st);
    double *M = reinterpret_cast<double *>(w + o_m), *G = reinterpret_cast<double *>(w + o_g),
           *Vinv = reinterpret_cast<double *>(w + o_v), *work = reinterpret_cast<double *>(w + o_w),
           *part = reinterpret_cast<double *>(w + o_p), *sc = reinterpret_cast<double *>(w + o_s);
    int *fallbacks = reinterpret_cast<int *>(work + 2 * R * R);
    double *h = pinned_scalars();
    if (!h) return set_status(CUD_ERR_NO_MEMORY);
    CUD_CHECK(cudaMemsetAsync(fallbacks, 0, sizeof(int), s));

    const auto t0 = std::chrono::steady_clock::now();
    for (int m = 0; m < order; m++)
        if ((st = factor_gram_f64(U[m], dims[m], R, G + (size_t)m * R * R, s))) return set_status(st);
    if ((st = dot_f64(X, X, total, part, sc + 2, s))) return set_status(st);  // sc[2] = ||X||^2
    CUD_CHECK(cudaMemcpyAsync(h, sc + 2, sizeof(double), cudaMemcpyDeviceToHost, s));
    CUD_CHECK(cudaStreamSynchronize(s));
    const double normx2 = h[0];

    const double *Uc[kMaxOrder];
    for (int m = 0; m < order; m++) Uc[m] = U[m];
    double fit = 0.0, fit_prev = 0.0;
    int sweeps = 0;
    for (int sw = 0; sw < opt.max_sweeps; sw++) {
        for (int mode = 0; mode < order; mode++) {
            void *mw = w;  // MTTKRP partials at the start of the workspace
            if ((st = mttkrp_simt_f64(X, order, dims, Uc, mode, R, M, mw, s))) return set_status(st);
            NormalArgs na;
            for (int m = 0; m < order; m++) na.G[m] = G + (size_t)m * R * R;
            na.nG = order;
            na.mode = mode;
            na.R = (int)R;
            na.Vinv = Vinv;
            na.work = work;
            na.fallbacks = fallbacks;
            if ((st = normal_inverse(na, s))) return set_status(st);
            const long n = dims[mode] * R;
            k_apply_inverse_f64<<<(unsigned)std::min<long>((n + 255) / 256, 4L * kNumSMs), 256, 0, s>>>(
                M, Vinv, dims[mode], R, U[mode]);
            CUD_CHECK_LAUNCH("cp_als_f64 update");
            if ((st = factor_gram_f64(U[mode], dims[mode], R, G + (size_t)mode * R * R, s))) return set_status(st);
        }
        sweeps = sw + 1;
        // fit of the factors just computed: M holds the last mode's MTTKRP
        k_dot_parts<<<F64_PARTS, 256, 0, s>>>(M, U[order - 1], dims[order - 1] * R, part);
        GramList gl;
        gl.n = order;
        for (int m = 0; m < order; m++) gl.G[m] = G + (size_t)m * R * R;
        k_fit_terms_f64<<<1, 256, 0, s>>>(part, F64_PARTS, gl, R, sc);
        CUD_CHECK_LAUNCH("cp_als_f64 fit");
        CUD_CHECK(cudaMemcpyAsync(h, sc, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
        CUD_CHECK(cudaStreamSynchronize(s));
        const double res2 = normx2 - 2.0 * h[0] + h[1];
        fit_prev = fit;
        fit = 1.0 - std::sqrt(res2 > 0.0 ? res2 : 0.0) / std::sqrt(normx2);
        if (opt.tol > 0.0 && sw > 0 && std::fabs(fit - fit_prev) < opt.tol) break;
        if (opt.target_fit > 0.0 && fit >= opt.target_fit) break;
    }
    CUD_CHECK(cudaMemcpyAsync(h, fallbacks, sizeof(int), cudaMemcpyDeviceToHost, s));
    CUD_CHECK(cudaStreamSynchronize(s));
    if (res) {
        res->sweeps = sweeps;
        res->fallbacks = *reinterpret_cast<int *>(h);
        res->fit = fit;
        res->fit_prev = fit_prev;
        res->fit_estimate = fit;
        res->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        res->kernels_per_sweep = order * 5 + 2;
    }
    return set_status(CUD_OK);
}
