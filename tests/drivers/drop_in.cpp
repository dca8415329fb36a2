// A program written against the reference's public header
// (inc/cudecompose.h of 891922758/first-project), built unchanged against
// this repository's include/cudecompose.h and libcutensordecomposition.a.
// It prints each result as "name v0 v1 ..." for tests/test_drop_in.py.
#include "cudecompose.h"
#include <vector>

static void fill_int(float *h, long n) {
    for (long i = 0; i < n; i++) h[i] = float(int(10 * (((float)rand()) / RAND_MAX - 0.5)));
}

static void dump(const char *name, const float *d, long n) {
    std::vector<float> h(n);
    cudaMemcpy(h.data(), d, sizeof(float) * n, cudaMemcpyDeviceToHost);
    printf("%s", name);
    for (long i = 0; i < n; i++) printf(" %.9g", h[i]);
    printf("\n");
}

static float *upload(const float *h, long n) {
    float *d;
    cudaMalloc((void **)&d, sizeof(float) * n);
    cudaMemcpy(d, h, sizeof(float) * n, cudaMemcpyHostToDevice);
    return d;
}

int main() {
    const long m = 3, n = 3, k = 3, r = 2;
    float X[27], A[6], B[6], C[6];
    srand(2);
    fill_int(X, 27); fill_int(A, 6); fill_int(B, 6); fill_int(C, 6);
    float *dX = upload(X, 27), *dA = upload(A, 6), *dB = upload(B, 6), *dC = upload(C, 6);
    float *out;
    cudaMalloc((void **)&out, sizeof(float) * 1024);

    mttkrp(dX, dC, dB, out, 1, m, n, k, r); dump("mttkrp1", out, m * r);
    mttkrp(dX, dC, dA, out, 2, m, n, k, r); dump("mttkrp2", out, n * r);
    mttkrp(dX, dB, dA, out, 3, m, n, k, r); dump("mttkrp3", out, k * r);
    kr(dA, dB, out, m, n, r); dump("kr", out, m * n * r);
    hadmard(dA, dB, out, m, r); dump("hadmard", out, m * r);
    hadmard3(dA, dB, dC, out, m, r); dump("hadmard3", out, m * r);
    t2m(dX, out, 2, m, n, k); cudaDeviceSynchronize(); dump("t2m2", out, 27);
    t2m(dX, out, 3, m, n, k); cudaDeviceSynchronize(); dump("t2m3", out, 27);
    tensor_product(dA, dB, out, m, r, n, r); cudaDeviceSynchronize(); dump("kron", out, 36);
    gencp(out, dA, dB, dC, m, n, k, r); dump("gencp", out, 27);
    float G[8];
    fill_int(G, 8);
    float *dG = upload(G, 8);
    gentucker(out, dG, dA, dB, dC, m, n, k, 2, 2, 2); dump("gentucker", out, 27);
    float *rec = upload(X, 27);
    gencp(rec, dA, dB, dC, m, n, k, r);
    float err = 0.f;
    rse(dX, rec, 27, &err);
    printf("rse %.9g\n", err);
    dump("rse_diff", rec, 27);
    initMat(out, 4); dump("identity", out, 16);
    printf("status %d\n", cudecomposeGetLastError());
    return 0;
}
