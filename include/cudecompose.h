/*
 * cudecompose.h -- drop-in header for the B200-native libcutensordecomposition.
 *
 * Declares the same free functions, with the same C++ signatures (and so the
 * same mangled link names), as the reference header inc/cudecompose.h:20-57 of
 * 891922758/first-project, so programs written against it compile and link
 * unchanged.  The functions keep the reference's semantics (device pointers
 * in and out, column-major, `long` extents, host-synchronous) and record a
 * status retrievable with cudecomposeGetLastError() instead of printing.
 * The stream-taking, status-returning C ABI is in cudecompose_c.h.
 *
 * Differences from the reference, by design: cp_tensorcore does not free the
 * caller's buffers (src/tensorcore_cp.cu:136-139), cp_als4 does not reset
 * the device (src/cp4_als.cu:184), tucker_tensorcore writes U1..U3
 * (src/tucker_tensorcore.cu:84-108 leaves them unwritten) and computes in
 * three-term BF16 on the tensor cores where the reference rounds to FP16
 * (closer to the exact result), and the
 * normal-equation solve is an FP64 Gauss-Jordan inverse with SPD pivots (a
 * Jacobi pseudo-inverse when a pivot is not positive) rather than FP32 LU.
 */
#ifndef GUARD_cudecompose_h
#define GUARD_cudecompose_h
#include <iostream>
#include <fstream>
#include <cuda_runtime.h>
#include <cuda_fp16.h>
#include <time.h>
#include <stdio.h>
using namespace std;  /* the reference header does this; its drivers rely on it */

#include "cudecompose_c.h"

typedef float dt;

#ifdef __CUDACC__
/* Kernels the reference exports (inc/cudecompose.h:22,27,31-33,35,45,47,55-57),
 * one thread per element, same arguments. */
extern __global__ void hardm(dt *M, dt *N, dt *res, long m, long n);
extern __global__ void floattohalf(dt *AA, half *BB, long m);
extern __global__ void tensorTomat1(dt *T1, dt *T2, long m, long n, long k);
extern __global__ void tensorTomat2(dt *T1, dt *T2, long m, long n, long k);
extern __global__ void tensorTomat3(dt *T1, dt *T2, long m, long n, long k);
extern __global__ void t_t(dt *M, dt *N, long m);
extern __global__ void initIdeMat(dt *AA, long m);
extern __global__ void hardm3(dt *M, dt *N, dt *K, dt *res, long m, long n);
extern __global__ void elepro3(dt *AA, dt *BB, dt *CC, dt *DD, int m);
extern __global__ void initIdeMat(dt *AA, int m);
extern __global__ void elemin(dt *A, dt *B, long n);
#endif

void hadmard(dt *d_A, dt *d_B, dt *d_C, long a, long b);
void kr(dt *d_A, dt *d_B, dt *d_AkrB, long a, long b, long r);
void tensor_product(dt *d_A, dt *d_B, dt *d_C, long a, long b, long c, long d);
void printTensor(dt *A, long a, long b, long c);
void f2h(dt *A, half *B, long num);
void ttm(dt *d_X, dt *d_U, dt *d_XU, long flag, long a, long b, long c, long d);
void mttkrp(dt *d_X, dt *left, dt *d_right, dt *d_XU, long flag, long m, long n, long k, long r);
void t2m(dt *d_T1, dt *d_T2, long flag, long m, long n, long k);
void tminust(dt *d_left, dt *d_right, long m);
void rse(dt *d_X, dt *d_X1, long m, dt *error);
void gencp(dt *d_rec, dt *d_A, dt *d_B, dt *d_C, long a, long b, long c, long r);
void gentucker(dt *d_rec, dt *d_core, dt *d_A, dt *d_B, dt *d_C, long a, long b, long c,
               long r1, long r2, long r3);
void cp_als(dt *d_X, dt *d_A, dt *d_B, dt *d_C, long a, long b, long c, long r);
void tucker_hosvd(dt *d_X, dt *d_core, dt *d_U1, dt *d_U2, dt *d_U3, long a, long b, long c,
                  long r1, long r2, long r3);
void cp_tensorcore(dt *d_X, dt *d_A, dt *d_B, dt *d_C, long a, long b, long c, long r);
void tucker_tensorcore(dt *d_X, dt *d_core, dt *d_U1, dt *d_U2, dt *d_U3, long a, long b,
                       long c, long r1, long r2, long r3);
void initMat(dt *d_A, long m);
void hadmard3(dt *d_A, dt *d_B, dt *d_C, dt *d_ABC, long a, long b);
void cp_als4(dt *d_X, dt *d_A, dt *d_B, dt *d_C, dt *d_D, long a, long b, long c, long d,
             long r);
void tucker_hosvd4(dt *d_X, dt *d_core, dt *d_U1, dt *d_U2, dt *d_U3, dt *d_U4, long a,
                   long b, long c, long d, long r1, long r2, long r3, long r4);
void gencp4(dt *d_T, dt *d_AA, dt *d_BB, dt *d_CC, dt *d_DD, long a, long b, long c, long d,
            long r);
void gentucker4(dt *d_T, dt *d_G, dt *d_A, dt *d_B, dt *d_C, dt *d_D, long a, long b, long c,
                long d, long r1, long r2, long r3, long r4);

/* Extension: HOOI as a drop-in style entry
 * (decomposition/GPU/normal/tucker/tucker_hooi.cu:3, there with host
 * pointers; here device pointers like the rest of this header). */
void tucker_hooi(dt *d_X, dt *d_core, dt *d_U1, dt *d_U2, dt *d_U3, long a, long b, long c,
                 long r1, long r2, long r3);

/* Extension: last status recorded by this thread (0 = OK). */
int cudecomposeGetLastError(void);

#endif
