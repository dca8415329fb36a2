// Mode products (TTM), unfolding Grams and the CP/Tucker reconstructions,
// expressed as strided GEMMs over the column-major tensor -- no unfolding is
// ever materialised.
#include <vector>

#include "kernels.cuh"

using namespace cud;

namespace cud {

namespace {

__global__ void k_round_copy(const float *__restrict__ in, float *__restrict__ out, long n, int mode) {
    long tid = blockIdx.x * (long)blockDim.x + threadIdx.x;
    long stride = (long)gridDim.x * blockDim.x;
    for (long i = tid; i < n; i += stride) {
        float v = in[i];
        if (mode == 1) v = __half2float(__float2half_rn(v));
        else if (mode == 2) v = __bfloat162float(__float2bfloat16_rn(v));
        out[i] = v;
    }
}

}  // namespace

// Y = X x_mode W  (W: J x dims[mode], row = new index).  With w_trans set,
// W is given as its transpose (dims[mode] x J, e.g. a factor matrix U, so
// that Y = X x_mode U^T).  FP32 or FP64 (gemm_simt / gemm_simt_f64).
template <typename T>
int mode_product_t(const T *X, int order, const long *dims, int mode, const T *W, long J, T *Y, cudaStream_t s,
                   bool w_trans) {
    auto run = [&](const GemmDescT<T> &d) {
        if constexpr (sizeof(T) == 8) return gemm_simt_f64(d, s);
        else return gemm_simt(d, s);
    };
    ModeView v = mode_view(order, dims, mode);
    GemmDescT<T> d;
    if (v.P == 1) {
        d.M = J; d.N = v.S; d.Kin = v.Q;
        d.A = W;
        if (w_trans) { d.a_m = v.Q; d.a_kin = 1; } else { d.a_m = 1; d.a_kin = J; }
        d.B = X; d.b_kin = 1; d.b_n = v.Q;
        d.C = Y; d.c_m = 1; d.c_n = J;
        d.splits = 1;
        return run(d);
    }
    for (long s0 = 0; s0 < v.S; s0 += 65535) {
        long nb = std::min(65535L, v.S - s0);
        d = GemmDescT<T>();
        d.M = v.P; d.N = J; d.Kin = v.Q; d.batch = nb;
        d.A = X + s0 * v.P * v.Q; d.a_m = 1; d.a_kin = v.P; d.a_b = v.P * v.Q;
        d.B = W; d.b_b = 0;
        if (w_trans) { d.b_kin = 1; d.b_n = v.Q; } else { d.b_kin = J; d.b_n = 1; }
        d.C = Y + s0 * v.P * J; d.c_m = 1; d.c_n = v.P; d.c_b = v.P * J;
        d.splits = 1;
        int st = run(d);
        if (st) return st;
    }
    return CUD_OK;
}

int mode_product(const float *X, int order, const long *dims, int mode, const float *W, long J,
                 float *Y, cudaStream_t s, bool w_trans) {
    return mode_product_t<float>(X, order, dims, mode, W, J, Y, s, w_trans);
}

int mode_product_f64(const double *X, int order, const long *dims, int mode, const double *W, long J, double *Y,
                     cudaStream_t s, bool w_trans) {
    return mode_product_t<double>(X, order, dims, mode, W, J, Y, s, w_trans);
}

// G (Q x Q, FP64) = X_(mode) X_(mode)^T; for FP64 X the split-K partials
// are FP64 as well.
template <typename T>
GemmDescT<T> gram_desc(const T *X, int order, const long *dims, int mode, double *G) {
    ModeView v = mode_view(order, dims, mode);
    GemmDescT<T> d;
    d.M = v.Q; d.N = v.Q;
    d.A = X; d.B = X;
    if (v.P == 1) {
        d.Kin = v.S; d.Kout = 1;
        d.a_m = 1; d.a_kin = v.Q;
        d.b_n = 1; d.b_kin = v.Q;
    } else {
        d.Kin = v.P; d.Kout = v.S;
        d.a_m = v.P; d.a_kin = 1; d.a_kout = v.P * v.Q;
        d.b_n = v.P; d.b_kin = 1; d.b_kout = v.P * v.Q;
    }
    d.C = G; d.c_m = 1; d.c_n = v.Q;
    return d;
}

int unfold_gram(const float *X, int order, const long *dims, int mode, double *G, cudaStream_t s) {
    GemmDesc d = gram_desc<float>(X, order, dims, mode, G);
    d.out_f64 = true;
    return gemm_simt(d, s);
}

int unfold_gram_f64(const double *X, int order, const long *dims, int mode, double *G, cudaStream_t s) {
    return gemm_simt_f64(gram_desc<double>(X, order, dims, mode, G), s);
}

int round_copy(const float *in, float *out, long n, int mode, cudaStream_t s) {
    k_round_copy<<<blocks_for(n, 256), 256, 0, s>>>(in, out, n, mode);
    CUD_CHECK_LAUNCH("round_copy");
    return CUD_OK;
}

}  // namespace cud

extern "C" int cud_mode_product(const float *X, int order, const long *dims, int mode,
                                const float *W, long J, float *Y, int precision, void *stream) {
    if (order < 1 || order > kMaxOrder || !dims || mode < 0 || mode >= order || J <= 0 || !X ||
        !W || !Y)
        return set_status(CUD_ERR_INVALID_ARGUMENT);
    long total = 1;
    for (int m = 0; m < order; m++) {
        if (dims[m] <= 0) return set_status(CUD_ERR_INVALID_ARGUMENT);
        total *= dims[m];
    }
    cudaStream_t s = as_stream(stream);
    int rmode = precision == CUD_PREC_FP16 ? 1 : precision == CUD_PREC_BF16 ? 2 : 0;
    if (rmode == 0) return set_status(mode_product(X, order, dims, mode, W, J, Y, s));
    int st;
    long wn = J * dims[mode];
    float *buf = (float *)scratch(kSlotTmp1, sizeof(float) * (total + wn), &st);
    if (!buf) return set_status(st);
    if ((st = round_copy(X, buf, total, rmode, s))) return set_status(st);
    if ((st = round_copy(W, buf + total, wn, rmode, s))) return set_status(st);
    return set_status(mode_product(buf, order, dims, mode, buf + total, J, Y, s));
}

extern "C" int cud_ttm(const float *X, const float *U, float *XU, long flag, long a, long b,
                       long c, long d, int precision, void *stream) {
    if (flag < 1 || flag > 3) return set_status(CUD_ERR_INVALID_ARGUMENT);
    long dims[3] = {a, b, c};
    return cud_mode_product(X, 3, dims, (int)flag - 1, U, d, XU, precision, stream);
}

extern "C" int cud_unfold_gram(const float *X, int order, const long *dims, int mode, double *G,
                               int precision, void *stream) {
    (void)precision;
    if (order < 1 || order > kMaxOrder || !dims || mode < 0 || mode >= order || !X || !G)
        return set_status(CUD_ERR_INVALID_ARGUMENT);
    for (int m = 0; m < order; m++)
        if (dims[m] <= 0) return set_status(CUD_ERR_INVALID_ARGUMENT);
    return set_status(unfold_gram(X, order, dims, mode, G, as_stream(stream)));
}

extern "C" int cud_cross_gram(const float *A, const float *B, long P, long ma, long mb, double *G, long ldg,
                              void *stream) {
    if (!A || !B || !G || P <= 0 || ma <= 0 || mb <= 0 || ldg < ma) return set_status(CUD_ERR_INVALID_ARGUMENT);
    GemmDesc d;
    d.M = ma; d.N = mb; d.Kin = P;
    d.A = A; d.a_m = P; d.a_kin = 1;
    d.B = B; d.b_n = P; d.b_kin = 1;
    d.C = G; d.c_m = 1; d.c_n = ldg;
    d.out_f64 = true;
    return set_status(gemm_simt(d, as_stream(stream)));
}

extern "C" int cud_gencp(float *rec, int order, const long *dims, const float *const *U, long R,
                         void *stream) {
    if (order < 1 || order > kMaxOrder || !dims || !U || !rec || R <= 0)
        return set_status(CUD_ERR_INVALID_ARGUMENT);
    long rest = 1;
    for (int m = 0; m < order; m++) {
        if (dims[m] <= 0 || !U[m]) return set_status(CUD_ERR_INVALID_ARGUMENT);
        if (m > 0) rest *= dims[m];
    }
    cudaStream_t s = as_stream(stream);
    int st;
    if (order == 1) {
        // rec[i] = sum_r U0[i, r]
        float *ones = (float *)scratch(kSlotTmp1, sizeof(float) * R, &st);
        if (!ones) return set_status(st);
        std::vector<float> h(R, 1.0f);
        CUD_CHECK(cudaMemcpyAsync(ones, h.data(), sizeof(float) * R, cudaMemcpyHostToDevice, s));
        GemmDesc d;
        d.M = dims[0]; d.N = 1; d.Kin = R;
        d.A = U[0]; d.a_m = 1; d.a_kin = dims[0];
        d.B = ones; d.b_kin = 1; d.b_n = R;
        d.C = rec; d.c_m = 1; d.c_n = dims[0];
        d.splits = 1;
        st = gemm_simt(d, s);
        if (st == CUD_OK) st = cudaStreamSynchronize(s) == cudaSuccess ? CUD_OK : CUD_ERR_CUDA;
        return set_status(st);
    }
    // KR of U[1..], fastest first, materialised like src/rse.cu:24-25 (then
    // one GEMM against U[0]).  Two buffers ping-pong for order > 3.
    float *kr = (float *)scratch(kSlotTmp1, sizeof(float) * rest * R * (order > 3 ? 2 : 1), &st);
    if (!kr) return set_status(st);
    const float *cur = U[1];
    long rows = dims[1];
    float *bufs[2] = {kr, kr + rest * R};
    int which = 0;
    for (int m = 2; m < order; m++) {
        float *dst = bufs[which];
        if ((st = cud_kr(U[m], cur, dst, dims[m], rows, R, stream))) return set_status(st);
        cur = dst;
        rows *= dims[m];
        which ^= 1;
    }
    GemmDesc d;
    d.M = dims[0]; d.N = rest; d.Kin = R;
    d.A = U[0]; d.a_m = 1; d.a_kin = dims[0];
    d.B = cur; d.b_kin = rest; d.b_n = 1;
    d.C = rec; d.c_m = 1; d.c_n = dims[0];
    d.splits = 1;
    return set_status(gemm_simt(d, s));
}

extern "C" int cud_gentucker(float *rec, int order, const long *dims, const float *core,
                             const long *ranks, const float *const *U, void *stream) {
    if (order < 1 || order > kMaxOrder || !dims || !ranks || !U || !rec || !core)
        return set_status(CUD_ERR_INVALID_ARGUMENT);
    long cur[kMaxOrder];
    size_t maxn = 0;
    for (int m = 0; m < order; m++) {
        if (dims[m] <= 0 || ranks[m] <= 0 || !U[m]) return set_status(CUD_ERR_INVALID_ARGUMENT);
        cur[m] = ranks[m];
    }
    // sizes after each step
    {
        long c2[kMaxOrder];
        for (int m = 0; m < order; m++) c2[m] = ranks[m];
        for (int m = 0; m < order; m++) {
            c2[m] = dims[m];
            size_t n = 1;
            for (int q = 0; q < order; q++) n *= c2[q];
            maxn = std::max(maxn, n);
        }
    }
    cudaStream_t s = as_stream(stream);
    int st;
    float *buf = (float *)scratch(kSlotTmp1, sizeof(float) * maxn * 2, &st);
    if (!buf) return set_status(st);
    const float *src = core;
    // rec = core x_1 U0 x_2 U1 ... (src/rse.cu:43-45: mode 1, then 2, then 3)
    for (int m = 0; m < order; m++) {
        float *dst = (m == order - 1) ? rec : buf + (m & 1) * maxn;
        if ((st = mode_product(src, order, cur, m, U[m], dims[m], dst, s))) return set_status(st);
        cur[m] = dims[m];
        src = dst;
    }
    return set_status(CUD_OK);
}
