// MTTKRP dispatch and the public MTTKRP entry points.
//
// CUD_PREC_FP32 runs the CUDA-core kernel; every other precision runs the
// tcgen05 tensor-core kernel where it applies (shape, alignment, rank) and
// otherwise the CUDA-core kernel with the same operand rounding
// (BF16X3/DEFAULT fall back to plain FP32, which is at least as accurate).
#include "kernels.cuh"

namespace cud {

namespace {
int round_mode(int precision) {
    return precision == CUD_PREC_FP16 ? 1 : precision == CUD_PREC_BF16 ? 2 : 0;
}
}  // namespace

// Sized for both paths, so a call may fall back (e.g. a misaligned X) with
// the same workspace.
size_t mttkrp_ws_bytes(int order, const long *dims, int mode, long R, int precision) {
    size_t b = mttkrp_simt_ws_bytes(order, dims, mode, R, round_mode(precision));
    size_t t = 0;
    if (precision != CUD_PREC_FP32 && mttkrp_tc_query(order, dims, mode, R, precision, &t) == CUD_OK)
        b = std::max(b, t);
    return b;
}

int mttkrp_run(const float *X, int order, const long *dims, const float *const *U, int mode, long R,
               float *out, int precision, void *ws, cudaStream_t s) {
    if (precision != CUD_PREC_FP32) {
        size_t b = 0;
        if (mttkrp_tc_query(order, dims, mode, R, precision, &b) == CUD_OK) {
            int st = mttkrp_tc(X, order, dims, U, mode, R, out, precision, ws, s);
            if (st != CUD_ERR_UNSUPPORTED) return st;
        }
    }
    return mttkrp_simt_rounded(X, order, dims, U, mode, R, out, round_mode(precision), ws, s);
}

int mttkrp_run_parts(const float *X, int order, const long *dims, const float *const *U, int mode, long R,
                     float *out, int precision, void *ws, cudaStream_t s, MttkrpParts *parts) {
    if (precision != CUD_PREC_FP32) {
        size_t b = 0;
        if (mttkrp_tc_query(order, dims, mode, R, precision, &b) == CUD_OK) {
            int st = mttkrp_tc(X, order, dims, U, mode, R, out, precision, ws, s, parts);
            if (st != CUD_ERR_UNSUPPORTED) return st;
        }
    }
    int st = mttkrp_simt_rounded(X, order, dims, U, mode, R, out, round_mode(precision), ws, s);
    if (st == CUD_OK) *parts = MttkrpParts{out, 0, 1, dims[mode], 1, nullptr};
    return st;
}

}  // namespace cud

using namespace cud;

extern "C" int cud_mttkrp(const float *X, int order, const long *dims, const float *const *U,
                          int mode, long R, float *out, int precision, void *stream) {
    if (order < 2 || order > kMaxOrder || !dims || mode < 0 || mode >= order || R <= 0 || !X ||
        !U || !out || precision < 0 || precision > CUD_PREC_DEFAULT)
        return set_status(CUD_ERR_INVALID_ARGUMENT);
    for (int m = 0; m < order; m++) {
        if (dims[m] <= 0) return set_status(CUD_ERR_INVALID_ARGUMENT);
        if (m != mode && !U[m]) return set_status(CUD_ERR_INVALID_ARGUMENT);
    }
    int st;
    void *ws = scratch(kSlotMttkrp, mttkrp_ws_bytes(order, dims, mode, R, precision), &st);
    if (!ws) return set_status(st);
    return set_status(mttkrp_run(X, order, dims, U, mode, R, out, precision, ws, as_stream(stream)));
}

extern "C" int cud_mttkrp_path(int order, const long *dims, int mode, long R, int precision) {
    if (order < 2 || order > kMaxOrder || !dims || mode < 0 || mode >= order || R <= 0) return 0;
    if (precision == CUD_PREC_FP32) return 0;
    size_t b = 0;
    return mttkrp_tc_query(order, dims, mode, R, precision, &b) == CUD_OK ? 1 : 0;
}

extern "C" int cud_mttkrp_legacy(const float *X, const float *left, const float *right, float *XU,
                                 long flag, long m, long n, long k, long r, int precision,
                                 void *stream) {
    if (flag < 1 || flag > 3) return set_status(CUD_ERR_INVALID_ARGUMENT);
    long dims[3] = {m, n, k};
    const float *U[3] = {nullptr, nullptr, nullptr};
    // src/mttkrp.cu:12,32,55: the KR row is right[x] * left[y], right fastest
    if (flag == 1) { U[1] = right; U[2] = left; }
    else if (flag == 2) { U[0] = right; U[2] = left; }
    else { U[0] = right; U[1] = left; }
    return cud_mttkrp(X, 3, dims, U, (int)flag - 1, r, XU, precision, stream);
}
