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

int factor_gram(const float *U, long I, long R, double *G, cudaStream_t s);
int normal_inverse(const NormalArgs &a, cudaStream_t s);
// Per-device kernel attributes for normal_inverse; call before stream capture.
int normal_inverse_prepare();
int apply_inverse(const float *M, const double *Vinv, long I, long R, float *U, cudaStream_t s);
int fit_eval(const FitArgs &a, cudaStream_t s);

}  // namespace cud
