// The drop-in C++ entry points of cudecompose.h: the reference's free
// functions (inc/cudecompose.h:22-57) with their exact signatures, each a
// thin host-synchronous wrapper over the C ABI.  Status goes to the
// thread-local side channel (cudecomposeGetLastError) instead of stdout.
#include <iostream>
#include <vector>
#include <cmath>

#include "../../include/cudecompose.h"
#include "common.cuh"

namespace {

void sync_after(int st) {
    cudaError_t e = cudaDeviceSynchronize();
    if (st == CUD_OK && e != cudaSuccess) cud::cuda_status(e, "cudaDeviceSynchronize");
}

// Relative error ||X - Xhat|| / ||X|| of a CP model from its fit.
void print_error(double fit) { std::cout << (float)(1.0 - fit) << std::endl; }

}  // namespace

void hadmard(dt *d_A, dt *d_B, dt *d_C, long a, long b) { sync_after(cud_hadmard(d_A, d_B, d_C, a, b, nullptr)); }

void hadmard3(dt *d_A, dt *d_B, dt *d_C, dt *d_ABC, long a, long b) {
    sync_after(cud_hadmard3(d_A, d_B, d_C, d_ABC, a, b, nullptr));
}

void kr(dt *d_A, dt *d_B, dt *d_AkrB, long a, long b, long r) {
    sync_after(cud_kr(d_A, d_B, d_AkrB, a, b, r, nullptr));
}

void tensor_product(dt *d_A, dt *d_B, dt *d_C, long a, long b, long c, long d) {
    sync_after(cud_tensor_product(d_A, d_B, d_C, a, b, c, d, nullptr));
}

void printTensor(dt *A, long a, long b, long c) {
    std::vector<float> h((size_t)(a * b * c));
    if (cudaMemcpy(h.data(), A, sizeof(float) * h.size(), cudaMemcpyDeviceToHost) != cudaSuccess) {
        cud::cuda_status(cudaGetLastError(), "printTensor");
        return;
    }
    // same layout as src/kr.cu:19-27: slice by slice, row by row
    for (long i = 0; i < c; i++) {
        for (long j = 0; j < a; j++) {
            for (long k = 0; k < b; k++) std::cout << h[i * a * b + k * a + j] << "  ";
            std::cout << std::endl;
        }
        std::cout << "-----------------------------------" << std::endl;
    }
    std::cout << std::endl;
}

void f2h(dt *A, half *B, long num) { cud_f2h(A, B, num, nullptr); }

void ttm(dt *d_X, dt *d_U, dt *d_XU, long flag, long a, long b, long c, long d) {
    // FP16 operands, FP32 result, as src/ttm.cu:15-37
    sync_after(cud_ttm(d_X, d_U, d_XU, flag, a, b, c, d, CUD_PREC_FP16, nullptr));
}

void mttkrp(dt *d_X, dt *left, dt *d_right, dt *d_XU, long flag, long m, long n, long k, long r) {
    // FP16 operands, FP32 accumulation, as src/mttkrp.cu:15-25
    sync_after(cud_mttkrp_legacy(d_X, left, d_right, d_XU, flag, m, n, k, r, CUD_PREC_FP16, nullptr));
}

void t2m(dt *d_T1, dt *d_T2, long flag, long m, long n, long k) {
    cud_t2m(d_T1, d_T2, flag, m, n, k, nullptr);
}

void tminust(dt *d_left, dt *d_right, long m) { sync_after(cud_tminust(d_left, d_right, m, nullptr)); }

void initMat(dt *d_A, long m) { sync_after(cud_init_identity(d_A, m, nullptr)); }

void rse(dt *d_X, dt *d_X1, long m, dt *error) { sync_after(cud_rse(d_X, d_X1, m, error, nullptr)); }

void gencp(dt *d_rec, dt *d_A, dt *d_B, dt *d_C, long a, long b, long c, long r) {
    long dims[3] = {a, b, c};
    const float *U[3] = {d_A, d_B, d_C};
    sync_after(cud_gencp(d_rec, 3, dims, U, r, nullptr));
}

void gencp4(dt *d_T, dt *d_AA, dt *d_BB, dt *d_CC, dt *d_DD, long a, long b, long c, long d, long r) {
    long dims[4] = {a, b, c, d};
    const float *U[4] = {d_AA, d_BB, d_CC, d_DD};
    sync_after(cud_gencp(d_T, 4, dims, U, r, nullptr));
}

void gentucker(dt *d_rec, dt *d_core, dt *d_A, dt *d_B, dt *d_C, long a, long b, long c, long r1,
               long r2, long r3) {
    long dims[3] = {a, b, c}, ranks[3] = {r1, r2, r3};
    const float *U[3] = {d_A, d_B, d_C};
    sync_after(cud_gentucker(d_rec, 3, dims, d_core, ranks, U, nullptr));
}

void gentucker4(dt *d_T, dt *d_G, dt *d_A, dt *d_B, dt *d_C, dt *d_D, long a, long b, long c, long d,
                long r1, long r2, long r3, long r4) {
    long dims[4] = {a, b, c, d}, ranks[4] = {r1, r2, r3, r4};
    const float *U[4] = {d_A, d_B, d_C, d_D};
    sync_after(cud_gentucker(d_T, 4, dims, d_G, ranks, U, nullptr));
}

void cp_als(dt *d_X, dt *d_A, dt *d_B, dt *d_C, long a, long b, long c, long r) {
    long dims[3] = {a, b, c};
    float *U[3] = {d_A, d_B, d_C};
    if (cud_cp_init_curand(3, dims, r, U, 1234ULL, nullptr) != CUD_OK) return;
    cud_cp_options opt;
    cud_cp_default_options(&opt);
    cud_cp_result res;
    sync_after(cud_cp_als(d_X, 3, dims, r, U, &opt, &res, nullptr));
}

void cp_als4(dt *d_X, dt *d_A, dt *d_B, dt *d_C, dt *d_D, long a, long b, long c, long d, long r) {
    long dims[4] = {a, b, c, d};
    float *U[4] = {d_A, d_B, d_C, d_D};
    if (cud_cp_init_curand(4, dims, r, U, 1234ULL, nullptr) != CUD_OK) return;
    cud_cp_options opt;
    cud_cp_default_options(&opt);
    cud_cp_result res;
    int st = cud_cp_als(d_X, 4, dims, r, U, &opt, &res, nullptr);
    sync_after(st);
    if (st == CUD_OK) print_error(res.fit);  // src/cp4_als.cu:154-162 prints the error
}

void cp_tensorcore(dt *d_X, dt *d_A, dt *d_B, dt *d_C, long a, long b, long c, long r) {
    long dims[3] = {a, b, c};
    float *U[3] = {d_A, d_B, d_C};
    if (cud_cp_init_curand(3, dims, r, U, 1234ULL, nullptr) != CUD_OK) return;
    cud_cp_options opt;
    cud_cp_default_options(&opt);
    opt.precision = CUD_PREC_FP16;  // FP16 MTTKRP operands, src/tensorcore_cp.cu:69-70
    cud_cp_result res;
    int st = cud_cp_als(d_X, 3, dims, r, U, &opt, &res, nullptr);
    sync_after(st);
    if (st == CUD_OK) print_error(res.fit);  // src/tensorcore_cp.cu:110-118
}

namespace {

// ||X - Xhat|| / ||X|| of a Tucker model, printed as the reference does
// (src/tucker_tensorcore.cu:114-121, src/tucker4_hosvd.cu:123-130): the
// model is reconstructed into a temporary tensor and the residual taken
// element by element.  (The shortcut ||X||^2 - ||core||^2 cancels: at a
// relative error of 1e-3 it subtracts two numbers that agree to six digits.)
void print_tucker_error(const float *X, int order, const long *dims, const float *core, const long *ranks,
                        float *const *U) {
    long n = 1;
    for (int m = 0; m < order; m++) n *= dims[m];
    float *rec = nullptr;
    if (cudaMalloc(&rec, sizeof(float) * (size_t)n) != cudaSuccess) {
        cud::cuda_status(cudaGetLastError(), "cudaMalloc");
        return;
    }
    float err = 0.0f;
    if (cud_gentucker(rec, order, dims, core, ranks, U, nullptr) == CUD_OK &&
        cud_rse(X, rec, n, &err, nullptr) == CUD_OK)
        std::cout << err << std::endl;
    cudaFree(rec);
}

}  // namespace

void tucker_hosvd(dt *d_X, dt *d_core, dt *d_U1, dt *d_U2, dt *d_U3, long a, long b, long c, long r1,
                  long r2, long r3) {
    long dims[3] = {a, b, c}, ranks[3] = {r1, r2, r3};
    float *U[3] = {d_U1, d_U2, d_U3};
    sync_after(cud_tucker_hosvd(d_X, 3, dims, ranks, d_core, U, CUD_PREC_FP32, nullptr));
}

void tucker_hosvd4(dt *d_X, dt *d_core, dt *d_U1, dt *d_U2, dt *d_U3, dt *d_U4, long a, long b, long c,
                   long d, long r1, long r2, long r3, long r4) {
    long dims[4] = {a, b, c, d}, ranks[4] = {r1, r2, r3, r4};
    float *U[4] = {d_U1, d_U2, d_U3, d_U4};
    int st = cud_tucker_hosvd(d_X, 4, dims, ranks, d_core, U, CUD_PREC_FP32, nullptr);
    sync_after(st);
    if (st == CUD_OK) print_tucker_error(d_X, 4, dims, d_core, ranks, U);
}

// The reference rounds X, the factors and the chain's intermediates to FP16
// for its Gram and TTM GEMMs (src/tucker_tensorcore.cu:27-44, 85-108); this
// drop-in runs them on the tensor cores as three-term BF16 products
// (FP32-level accuracy, closer to the exact result than FP16) and also
// writes U1..U3.
void tucker_tensorcore(dt *d_X, dt *d_core, dt *d_U1, dt *d_U2, dt *d_U3, long a, long b, long c,
                       long r1, long r2, long r3) {
    long dims[3] = {a, b, c}, ranks[3] = {r1, r2, r3};
    float *U[3] = {d_U1, d_U2, d_U3};
    int st = cud_tucker_hosvd(d_X, 3, dims, ranks, d_core, U, CUD_PREC_BF16X3, nullptr);
    sync_after(st);
    if (st == CUD_OK) print_tucker_error(d_X, 3, dims, d_core, ranks, U);
}

void tucker_hooi(dt *d_X, dt *d_core, dt *d_U1, dt *d_U2, dt *d_U3, long a, long b, long c, long r1,
                 long r2, long r3) {
    long dims[3] = {a, b, c}, ranks[3] = {r1, r2, r3};
    float *U[3] = {d_U1, d_U2, d_U3};
    // 10 sweeps, decomposition/GPU/normal/tucker/tucker_hooi.cu:102
    sync_after(cud_tucker_hooi(d_X, 3, dims, ranks, d_core, U, 10, CUD_PREC_FP32, nullptr));
}

int cudecomposeGetLastError(void) { return cud_get_last_error(); }
