// Tucker decompositions: HOSVD (src/tucker_hosvd.cu:3-103,
// src/tucker4_hosvd.cu:3-141) and HOOI
// (decomposition/GPU/normal/tucker/tucker_hooi.cu:3-218), any order.
//
// Factor n = eigenvectors of the r_n largest eigenvalues of the FP64
// unfolding Gram, taken as the last r_n columns of the ascending
// eigendecomposition (the reference copies d_Xn_Xn + (I_n - r_n) I_n).
// The core is the chain X x_1 U_1^T x_2 U_2^T ... in mode order.
//
// The CUDA-core path is written once for FP32 and FP64 data: the FP64
// instantiation is the reference's decomposition/GPU/normal/dprice/
// tucker_hosvd.cu:3-167, 4_tucker_hosvd.cu:3-173 and tucker_hooi.cu:3-220
// (cud_tucker_hosvd_f64 / cud_tucker_hooi_f64).
#include "kernels.cuh"

namespace cud {

namespace {

template <typename T>
__global__ void k_take_top(const double *__restrict__ V, long n, long r, T *__restrict__ U) {
    long total = n * r;
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
        long i = e % n, j = e / n;
        U[e] = (T)V[i + n * (n - r + j)];
    }
}

struct TuckerWork {
    double *G = nullptr, *W = nullptr, *V = nullptr;
    void *buf0 = nullptr, *buf1 = nullptr;  // chain intermediates (FP32 or FP64)
    size_t bufn = 0;
};

int mp(const float *X, int order, const long *dims, int mode, const float *W, long J, float *Y, cudaStream_t s) {
    return mode_product(X, order, dims, mode, W, J, Y, s, true);
}
int mp(const double *X, int order, const long *dims, int mode, const double *W, long J, double *Y,
       cudaStream_t s) {
    return mode_product_f64(X, order, dims, mode, W, J, Y, s, true);
}
int ug(const float *X, int order, const long *dims, int mode, double *G, cudaStream_t s) {
    return unfold_gram(X, order, dims, mode, G, s);
}
int ug(const double *X, int order, const long *dims, int mode, double *G, cudaStream_t s) {
    return unfold_gram_f64(X, order, dims, mode, G, s);
}

int alloc_work(int order, const long *dims, const long *ranks, TuckerWork &w, size_t elem = sizeof(float)) {
    long maxd = 0;
    for (int m = 0; m < order; m++) maxd = std::max(maxd, dims[m]);
    // largest intermediate of any contraction chain: X with one mode reduced
    size_t maxn = 0;
    for (int m = 0; m < order; m++) {
        size_t n = 1;
        for (int q = 0; q < order; q++) n *= (q == m) ? ranks[q] : dims[q];
        maxn = std::max(maxn, n);
    }
    size_t gbytes = sizeof(double) * (size_t)maxd * maxd;
    size_t off_W = (gbytes + 255) & ~size_t(255);
    size_t off_V = off_W + ((sizeof(double) * maxd + 255) & ~size_t(255));
    size_t off_B = off_V + ((gbytes + 255) & ~size_t(255));
    size_t bytes = off_B + elem * maxn * 2 + 512;
    int st;
    char *p = (char *)scratch(kSlotTmp0, bytes, &st);
    if (!p) return st;
    w.G = (double *)p;
    w.W = (double *)(p + off_W);
    w.V = (double *)(p + off_V);
    w.buf0 = p + off_B;
    w.buf1 = p + off_B + elem * maxn;
    w.bufn = maxn;
    return CUD_OK;
}

// U_out (I x r) = top-r eigenvectors of G (I x I, destroyed).
template <typename T>
int top_eigvecs(double *G, long I, long r, const TuckerWork &w, T *U, cudaStream_t s) {
    int st = syev_jacobi(G, I, w.W, w.V, 60, s);
    if (st != CUD_OK && st != CUD_ERR_NOT_CONVERGED) return st;
    k_take_top<T><<<blocks_for(I * r, 256), 256, 0, s>>>(w.V, I, r, U);
    CUD_CHECK_LAUNCH("top_eigvecs");
    return st;
}

// Y = X x_{m in modes, m != skip} U_m^T, ascending mode order; result dims in
// `cur`.  Uses the two work buffers; returns the pointer holding Y.
template <typename T>
int project_all_but(const T *X, int order, const long *dims, const long *ranks, T *const *U, int skip,
                    const TuckerWork &w, long *cur, const T **Y, T *final_out, cudaStream_t s) {
    for (int m = 0; m < order; m++) cur[m] = dims[m];
    const T *src = X;
    int nsteps = 0;
    for (int m = 0; m < order; m++)
        if (m != skip) nsteps++;
    int step = 0;
    for (int m = 0; m < order; m++) {
        if (m == skip) continue;
        step++;
        T *dst = (step == nsteps && final_out) ? final_out : static_cast<T *>((step & 1) ? w.buf0 : w.buf1);
        int st = mp(src, order, cur, m, U[m], ranks[m], dst, s);
        if (st) return st;
        cur[m] = ranks[m];
        src = dst;
    }
    *Y = src;
    return CUD_OK;
}

template <typename T>
bool valid(int order, const long *dims, const long *ranks, T *const *U, const T *X, const T *core) {
    if (order < 2 || order > kMaxOrder || !dims || !ranks || !U || !X || !core) return false;
    for (int m = 0; m < order; m++)
        if (dims[m] <= 0 || ranks[m] <= 0 || ranks[m] > dims[m] || !U[m]) return false;
    return true;
}

}  // namespace

// tucker_tc.cu
bool tucker_tc_supported(int order, const long *dims, const long *ranks);
int tucker_tc_factors(const float *X, int order, const long *dims, const long *ranks, float *const *U, int n0,
                      bool three, cudaStream_t s, int *worst);
int tucker_tc_core(const float *X, int order, const long *dims, const long *ranks, float *const *U, float *core,
                   bool three, cudaStream_t s);
int tucker_tc_hooi_sweep(const float *X, int order, const long *dims, const long *ranks, float *const *U,
                         bool three, bool u0_set, cudaStream_t s, int *worst);

}  // namespace cud

using namespace cud;

namespace {

// Tensor cores for every precision but FP32 (CUD_PREC_BF16: one-term Grams;
// BF16X3 / DEFAULT: three-term Grams; TTMs BF16), when the extents allow.
bool use_tc(int precision, int order, const long *dims, const long *ranks) {
    return precision != CUD_PREC_FP32 && precision != CUD_PREC_FP16 && tucker_tc_supported(order, dims, ranks);
}

}  // namespace

namespace {

// HOSVD on the CUDA cores (FP64 Grams and eigensolver; data FP32 or FP64).
template <typename T>
int hosvd_plain(const T *X, int order, const long *dims, const long *ranks, T *core, T *const *U,
                cudaStream_t s) {
    TuckerWork w;
    int st = alloc_work(order, dims, ranks, w, sizeof(T));
    if (st) return st;
    int worst = CUD_OK;
    for (int n = 0; n < order; n++) {
        if ((st = ug(X, order, dims, n, w.G, s))) return st;
        st = top_eigvecs(w.G, dims[n], ranks[n], w, U[n], s);
        if (st == CUD_ERR_NOT_CONVERGED) worst = st;
        else if (st) return st;
    }
    long cur[kMaxOrder];
    const T *Y;
    if ((st = project_all_but(X, order, dims, ranks, U, -1, w, cur, &Y, core, s))) return st;
    CUD_CHECK(cudaStreamSynchronize(s));
    return worst;
}

// HOOI on the CUDA cores: U_2..U_N from the unfolding Grams
// (tucker_hooi.cu:45-75), then `sweeps` sweeps of U_n = top eigenvectors of
// the Gram of X x_{m != n} U_m^T, then the core.
template <typename T>
int hooi_plain(const T *X, int order, const long *dims, const long *ranks, T *core, T *const *U, int sweeps,
               cudaStream_t s) {
    TuckerWork w;
    int st = alloc_work(order, dims, ranks, w, sizeof(T));
    if (st) return st;
    int worst = CUD_OK;
    for (int n = 1; n < order; n++) {
        if ((st = ug(X, order, dims, n, w.G, s))) return st;
        st = top_eigvecs(w.G, dims[n], ranks[n], w, U[n], s);
        if (st == CUD_ERR_NOT_CONVERGED) worst = st;
        else if (st) return st;
    }
    long cur[kMaxOrder];
    const T *Y;
    for (int it = 0; it < sweeps; it++) {
        for (int n = 0; n < order; n++) {
            if ((st = project_all_but(X, order, dims, ranks, U, n, w, cur, &Y, (T *)nullptr, s))) return st;
            if ((st = ug(Y, order, cur, n, w.G, s))) return st;
            st = top_eigvecs(w.G, dims[n], ranks[n], w, U[n], s);
            if (st == CUD_ERR_NOT_CONVERGED) worst = st;
            else if (st) return st;
        }
    }
    if (sweeps == 0) {
        // no sweep: U_1 from its Gram as in HOSVD
        if ((st = ug(X, order, dims, 0, w.G, s))) return st;
        st = top_eigvecs(w.G, dims[0], ranks[0], w, U[0], s);
        if (st && st != CUD_ERR_NOT_CONVERGED) return st;
    }
    if ((st = project_all_but(X, order, dims, ranks, U, -1, w, cur, &Y, core, s))) return st;
    CUD_CHECK(cudaStreamSynchronize(s));
    return worst;
}

}  // namespace

extern "C" int cud_tucker_hosvd(const float *X, int order, const long *dims, const long *ranks,
                                float *core, float *const *U, int precision, void *stream) {
    if (!valid(order, dims, ranks, U, X, core)) return set_status(CUD_ERR_INVALID_ARGUMENT);
    cudaStream_t s = as_stream(stream);
    if (use_tc(precision, order, dims, ranks)) {
        const bool three = precision != CUD_PREC_BF16;
        int worst = CUD_OK;
        int st = tucker_tc_factors(X, order, dims, ranks, U, 0, three, s, &worst);
        if (st == CUD_OK) st = tucker_tc_core(X, order, dims, ranks, U, core, three, s);
        if (st) return set_status(st);
        CUD_CHECK(cudaStreamSynchronize(s));
        return set_status(worst);
    }
    return set_status(hosvd_plain<float>(X, order, dims, ranks, core, U, s));
}

extern "C" int cud_tucker_hooi(const float *X, int order, const long *dims, const long *ranks,
                               float *core, float *const *U, int sweeps, int precision, void *stream) {
    if (!valid(order, dims, ranks, U, X, core) || sweeps < 0) return set_status(CUD_ERR_INVALID_ARGUMENT);
    cudaStream_t s = as_stream(stream);
    if (use_tc(precision, order, dims, ranks)) {
        const bool three = precision != CUD_PREC_BF16;
        int worst = CUD_OK;
        // initial U_2..U_N from the Grams (tucker_hooi.cu:45-75), U_1 too when no sweep runs
        int st = tucker_tc_factors(X, order, dims, ranks, U, sweeps > 0 ? 1 : 0, three, s, &worst);
        for (int it = 0; it < sweeps && st == CUD_OK; it++)
            st = tucker_tc_hooi_sweep(X, order, dims, ranks, U, three, it > 0, s, &worst);
        if (st == CUD_OK) st = tucker_tc_core(X, order, dims, ranks, U, core, three, s);
        if (st) return set_status(st);
        CUD_CHECK(cudaStreamSynchronize(s));
        return set_status(worst);
    }
    return set_status(hooi_plain<float>(X, order, dims, ranks, core, U, sweeps, s));
}

extern "C" int cud_tucker_hosvd_f64(const double *X, int order, const long *dims, const long *ranks,
                                    double *core, double *const *U, void *stream) {
    if (!valid(order, dims, ranks, U, X, core)) return set_status(CUD_ERR_INVALID_ARGUMENT);
    return set_status(hosvd_plain<double>(X, order, dims, ranks, core, U, as_stream(stream)));
}

extern "C" int cud_tucker_hooi_f64(const double *X, int order, const long *dims, const long *ranks,
                                   double *core, double *const *U, int sweeps, void *stream) {
    if (!valid(order, dims, ranks, U, X, core) || sweeps < 0) return set_status(CUD_ERR_INVALID_ARGUMENT);
    return set_status(hooi_plain<double>(X, order, dims, ranks, core, U, sweeps, as_stream(stream)));
}
