// Device-side FP64 normal-equation machinery for CP-ALS (solve.cu).
#pragma once

#include "kernels.cuh"

namespace cud {

struct NormalArgs {
    const double *G[kMaxOrder];  // factor Grams, R x R each
    int nG = 0;                  // number of factors (tensor order)
    int mode = 0;                // excluded factor
    int R = 0;
    double *Vinv = nullptr;      // out: R x R
    double *work = nullptr;      // scratch: 2 R^2 doubles
    int *fallbacks = nullptr;    // incremented when the pseudo-inverse is used
};

struct FitArgs {
    const float *M = nullptr;    // last mode's MTTKRP
    const float *U = nullptr;    // last mode's updated factor
    long IR = 0;
    const double *G[kMaxOrder];
    int nG = 0;
    int R = 0;
    double normx2 = 0.0;
    double *out = nullptr;       // [fit, fit_prev, inner, ||Xhat||^2]
};

struct UpdateArgs {
    const float *M = nullptr;      // I x R
    const double *Vinv = nullptr;  // R x R, or null: U = M, Gram only
    float *U = nullptr;            // I x R out (when Vinv is set)
    long I = 0;
    int R = 0;
    double *G_out = nullptr;       // R x R Gram of U
    double *gpart = nullptr;       // update_ws_doubles(I, R) doubles
    unsigned *counter = nullptr;   // zero; left zero on return
    // optional fit (when fit_out is set): Gall[m] for m != mode, G_out for mode
    const double *Gall[kMaxOrder];
    int nG = 0, mode = 0;
    double normx2 = 0.0;
    double *fit_out = nullptr;     // [fit, fit_prev, inner, ||Xhat||^2]
    // with Vinv null and fit_out set: the MTTKRP result paired with U = M in
    // <M, U> (null: M itself)
    const float *Mfit = nullptr;
    // at most this many row-pass CTAs (0: as many as fill the GPU); a small
    // cap keeps a Gram beside a full-GPU kernel from taking its CTA slots
    int max_blocks = 0;
};
// Fused U = M Vinv, G = U^T U (+ fit), deterministic multi-CTA reduction.
int factor_update(const UpdateArgs &a, cudaStream_t s);
// U = M V^-1 from an MTTKRP's split partials in one kernel (M, rounded to
// FP32, is written too); CUD_ERR_UNSUPPORTED above FU_RMAX.
constexpr int FU_RMAX = 64;
int update_from_parts(const MttkrpParts &pp, const double *Vinv, long I, int R, float *M, float *U,
                      cudaStream_t s);
size_t update_ws_doubles(long I, long R);

int factor_gram(const float *U, long I, long R, double *G, cudaStream_t s);
int factor_gram_f64(const double *U, long I, long R, double *G, cudaStream_t s);
int normal_inverse(const NormalArgs &a, cudaStream_t s);
// Per-device kernel attributes for normal_inverse; call before stream capture.
int normal_inverse_prepare();
int apply_inverse(const float *M, const double *Vinv, long I, long R, float *U, cudaStream_t s);
int fit_eval(const FitArgs &a, cudaStream_t s);

}  // namespace cud
