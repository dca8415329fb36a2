/*
 * CPU oracle for the dense CP/Tucker path -- TEST INFRASTRUCTURE ONLY.
 *
 * This file restates, in plain C on the host, the arithmetic of the reference
 * library's hot path (891922758/first-project, src/*.cu).  It is the checker
 * the parity tests compare the CUDA library against; nothing in the product
 * (first-project_b200/) links or calls it.  Only tests/, the smoke check and
 * the CPU-baseline leg of bench.py may load it.
 *
 * Conventions (as in the reference, inc/cudecompose.h:20 and
 * src/tensor2matrix.cu:7-10): column-major, mode 1 fastest, element (i,j,k)
 * of an a x b x c tensor at i + j*a + k*a*b; factor matrices I_n x R
 * column-major.
 *
 * Pinning: the integer fixtures of the reference's drivers
 * (test/test_mttkrp.cpp:27-39, test/test_gen.cpp:19-34) are regenerated here
 * with glibc rand() exactly as those drivers do, and the exact answers on them
 * are checked by tests/test_oracle_golden.py against tests/golden/.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------ */
/* Fixture generators: restate the reference drivers' input loops.          */
/* ------------------------------------------------------------------------ */

void or_srand(unsigned seed) { srand(seed); }

/* test/test_mttkrp.cpp:29 / test/test_gen.cpp:20:
 *   X[i] = float(int(10*(((float) rand())/RAND_MAX - 0.5)));              */
void or_fill_int(float *dst, long n) {
    for (long i = 0; i < n; i++)
        dst[i] = (float)(int)(10 * (((float)rand()) / RAND_MAX - 0.5));
}

/* test/test_t2m.cpp:12, test/test_kr.cpp:27:  A[i] = rand()*0.1/(RAND_MAX) */
void or_fill_frac(float *dst, long n, double shift) {
    for (long i = 0; i < n; i++)
        dst[i] = (float)(rand() * 0.1 / (RAND_MAX) + shift);
}

/* test/test_cp.cpp:18: A[i] = ((float)rand()/RAND_MAX)                       */
void or_fill_unit(float *dst, long n) {
    for (long i = 0; i < n; i++) dst[i] = ((float)rand() / RAND_MAX);
}

/* ------------------------------------------------------------------------ */
/* Element-wise and permutation primitives (bit-exact targets).              */
/* ------------------------------------------------------------------------ */

/* src/hadmard.cu:2-8 hardm: res[i] = M[i]*N[i] over m*n elements. */
void or_hadmard(const float *A, const float *B, float *C, long n) {
    for (long i = 0; i < n; i++) C[i] = A[i] * B[i];
}

/* src/hadmard.cu:17-23 hardm3: res = M*N*K, evaluated left to right. */
void or_hadmard3(const float *A, const float *B, const float *K, float *D, long n) {
    for (long i = 0; i < n; i++) D[i] = A[i] * B[i] * K[i];
}

/* src/tminust.cu:2-8 t_t: N[i] = M[i] - N[i]. */
void or_tminust(const float *M, float *N, long n) {
    for (long i = 0; i < n; i++) N[i] = M[i] - N[i];
}

/* src/tminust.cu:17-29 initIdeMat: m x m identity. */
void or_identity(float *A, long m) {
    for (long j = 0; j < m; j++)
        for (long i = 0; i < m; i++) A[i + j * m] = (i == j) ? 1.0f : 0.0f;
}

/* src/kr.cu:9: cublasSgemmStridedBatched(N,T,b,a,1, B,b,b, A,a,a, out,b,ab, r)
 * gives out[x + y*b + t*a*b] = B[x,t] * A[y,t] (one rounding).            */
void or_kr(const float *A, const float *B, float *out, long a, long b, long r) {
    for (long t = 0; t < r; t++)
        for (long y = 0; y < a; y++)
            for (long x = 0; x < b; x++)
                out[x + y * b + t * a * b] = B[x + t * b] * A[y + t * a];
}

/* src/tensor2matrix.cu:38-52.  Returns 0, or -1 for a flag outside 1..3
 * (the reference prints and does nothing then).                             */
int or_t2m(const float *T1, float *T2, long flag, long m, long n, long k) {
    if (flag < 1 || flag > 3) return -1;
    for (long tube = 0; tube < k; tube++)
        for (long col = 0; col < n; col++)
            for (long row = 0; row < m; row++) {
                float v = T1[tube * m * n + col * m + row];
                if (flag == 1) T2[tube * m * n + col * m + row] = v;          /* :10 */
                else if (flag == 2) T2[tube * m * n + row * n + col] = v;     /* :22 */
                else T2[k * (col * m + row) + tube] = v;                      /* :33 */
            }
    return 0;
}

/* src/tensorproduct.cu:9-11: C = A (a x b) kron B (c x d), (a*c) x (b*d):
 * C[x + c*y, t + d*i] = A[y,i] * B[x,t].                                    */
void or_tensor_product(const float *A, const float *B, float *C, long a, long b,
                       long c, long d) {
    long ld = a * c;
    for (long i = 0; i < b; i++)
        for (long t = 0; t < d; t++)
            for (long y = 0; y < a; y++)
                for (long x = 0; x < c; x++)
                    C[(x + c * y) + ld * (t + d * i)] = A[y + a * i] * B[x + c * t];
}

/* IEEE binary16 round-to-nearest-even, as __float2half (src/float2half.cu:8). */
uint16_t or_f2h_one(float f) {
    uint32_t x;
    memcpy(&x, &f, 4);
    uint32_t sign = (x >> 16) & 0x8000u;
    uint32_t exp = (x >> 23) & 0xffu;
    uint32_t man = x & 0x7fffffu;
    if (exp == 0xff) return (uint16_t)(sign | 0x7c00u | (man ? 0x200u : 0u));
    int e = (int)exp - 127 + 15;
    if (e >= 31) return (uint16_t)(sign | 0x7c00u);
    if (e <= 0) {
        if (e < -10) return (uint16_t)sign;
        man |= 0x800000u;
        int shift = 14 - e;
        uint32_t half = man >> shift;
        uint32_t rem = man & ((1u << shift) - 1u);
        uint32_t mid = 1u << (shift - 1);
        if (rem > mid || (rem == mid && (half & 1u))) half++;
        return (uint16_t)(sign | half);
    }
    uint32_t h = (uint32_t)e << 10 | (man >> 13);
    uint32_t rem = man & 0x1fffu;
    if (rem > 0x1000u || (rem == 0x1000u && (h & 1u))) h++;
    return (uint16_t)(sign | h);
}

float or_h2f_one(uint16_t h) {
    uint32_t sign = (uint32_t)(h & 0x8000u) << 16;
    uint32_t exp = (h >> 10) & 0x1fu;
    uint32_t man = h & 0x3ffu;
    uint32_t x;
    if (exp == 0) {
        if (man == 0) x = sign;
        else {
            int e = -1;
            do { man <<= 1; e++; } while (!(man & 0x400u));
            x = sign | (uint32_t)(127 - 15 - e) << 23 | (man & 0x3ffu) << 13;
        }
    } else if (exp == 0x1f) x = sign | 0x7f800000u | man << 13;
    else x = sign | (exp - 15 + 127) << 23 | man << 13;
    float f;
    memcpy(&f, &x, 4);
    return f;
}

void or_f2h(const float *A, uint16_t *B, long n) {
    for (long i = 0; i < n; i++) B[i] = or_f2h_one(A[i]);
}

/* bfloat16 round-to-nearest-even (used by the mixed-precision variants). */
uint16_t or_f2bf_one(float f) {
    uint32_t x;
    memcpy(&x, &f, 4);
    if ((x & 0x7fffffffu) > 0x7f800000u) return (uint16_t)((x >> 16) | 0x40u);
    uint32_t lsb = (x >> 16) & 1u;
    x += 0x7fffu + lsb;
    return (uint16_t)(x >> 16);
}

float or_bf2f_one(uint16_t h) {
    uint32_t x = (uint32_t)h << 16;
    float f;
    memcpy(&f, &x, 4);
    return f;
}

void or_round_fp16(const float *A, float *B, long n) {
    for (long i = 0; i < n; i++) B[i] = or_h2f_one(or_f2h_one(A[i]));
}

void or_round_bf16(const float *A, float *B, long n) {
    for (long i = 0; i < n; i++) B[i] = or_bf2f_one(or_f2bf_one(A[i]));
}

/* ------------------------------------------------------------------------ */
/* MTTKRP, general order, FP64 accumulation.                                  */
/* ------------------------------------------------------------------------ */

/* out[q, r] = sum over all other indices of X[...] * prod_{m != mode} U_m[i_m, r]
 * (the math of src/mttkrp.cu:11-73 and of the FP32 MTTKRPs inside
 * src/cp_als.cu:46-52,66-69,85-88).  U[m] are column-major dims[m] x R.
 * X is float (the library's storage type); U and out are double.           */
void or_mttkrp(const float *X, int order, const long *dims, const double *const *U,
               int mode, long R, double *out) {
    long total = 1;
    for (int m = 0; m < order; m++) total *= dims[m];
    long Q = dims[mode];
    memset(out, 0, sizeof(double) * Q * R);
    long idx[16] = {0};
    double *w = (double *)malloc(sizeof(double) * R);
    for (long lin = 0; lin < total; lin++) {
        double x = X[lin];
        if (x != 0.0) {
            for (long r = 0; r < R; r++) w[r] = x;
            for (int m = 0; m < order; m++) {
                if (m == mode) continue;
                const double *um = U[m] + idx[m];
                for (long r = 0; r < R; r++) w[r] *= um[r * dims[m]];
            }
            double *o = out + idx[mode];
            for (long r = 0; r < R; r++) o[r * Q] += w[r];
        }
        for (int m = 0; m < order; m++) {
            if (++idx[m] < dims[m]) break;
            idx[m] = 0;
        }
    }
    free(w);
}

/* The public mttkrp() of src/mttkrp.cu:3-80 on a 3-way m x n x k tensor.
 * flag 1: left k x r, right n x r -> XU m x r  (:12,21-25)
 * flag 2: left k x r, right m x r -> XU n x r  (:32,41-47)
 * flag 3: left n x r, right m x r -> XU k x r  (:55,65-69)
 * The Khatri-Rao row is formed in FP32 (one rounding, :21/:41/:65), then X
 * and the KR are rounded to FP16 when round_fp16 is set (:15,23,45-46,59,67);
 * the products and sums are taken in FP64 here.                             */
int or_mttkrp_legacy(const float *X, const float *left, const float *right, double *out,
                     long flag, long m, long n, long k, long r, int round_fp16) {
    long Q = flag == 1 ? m : flag == 2 ? n : flag == 3 ? k : -1;
    if (Q < 0) return -1;
    memset(out, 0, sizeof(double) * Q * r);
    for (long kk = 0; kk < k; kk++)
        for (long jj = 0; jj < n; jj++)
            for (long ii = 0; ii < m; ii++) {
                float x = X[ii + jj * m + kk * m * n];
                if (round_fp16) x = or_h2f_one(or_f2h_one(x));
                long q, li, ri;
                if (flag == 1) { q = ii; li = kk; ri = jj; }
                else if (flag == 2) { q = jj; li = kk; ri = ii; }
                else { q = kk; li = jj; ri = ii; }
                long ldl = (flag == 3) ? n : k;
                long ldr = (flag == 1) ? n : m;
                for (long t = 0; t < r; t++) {
                    float w = right[ri + t * ldr] * left[li + t * ldl];
                    if (round_fp16) w = or_h2f_one(or_f2h_one(w));
                    out[q + t * Q] += (double)x * (double)w;
                }
            }
    return 0;
}

/* src/ttm.cu:4-47, U is d x I_n (row = new index):
 * flag 1: XU (d x b x c) = U * X_(1)                            (:21)
 * flag 2: XU (a x d x c), XU(:,:,k) = X(:,:,k) * U^T              (:29)
 * flag 3: XU (a x b x d) = X(ab x c) * U^T                         (:37)
 * FP16-rounded inputs when round_fp16 is set, FP64 sums.                    */
int or_ttm(const float *X, const float *U, double *XU, long flag, long a, long b, long c,
           long d, int round_fp16) {
    if (flag < 1 || flag > 3) return -1;
    long outn = (flag == 1) ? d * b * c : (flag == 2) ? a * d * c : a * b * d;
    memset(XU, 0, sizeof(double) * outn);
    long In = (flag == 1) ? a : (flag == 2) ? b : c;
    for (long kk = 0; kk < c; kk++)
        for (long jj = 0; jj < b; jj++)
            for (long ii = 0; ii < a; ii++) {
                double x = X[ii + jj * a + kk * a * b];
                if (round_fp16) x = or_h2f_one(or_f2h_one((float)x));
                for (long t = 0; t < d; t++) {
                    long src = (flag == 1) ? ii : (flag == 2) ? jj : kk;
                    double u = U[t + d * src];
                    if (round_fp16) u = or_h2f_one(or_f2h_one((float)u));
                    long o;
                    if (flag == 1) o = t + d * (jj + b * kk);
                    else if (flag == 2) o = ii + a * (t + d * kk);
                    else o = ii + a * (jj + b * t);
                    XU[o] += x * u;
                }
            }
    (void)In;
    return 0;
}

/* src/rse.cu:4-15: X1 <- X - X1, returns ||X - X1|| / ||X|| (norms in FP64). */
float or_rse(const float *X, float *X1, long n) {
    double s1 = 0.0, s2 = 0.0;
    for (long i = 0; i < n; i++) {
        X1[i] = X[i] - X1[i];
        s1 += (double)X1[i] * X1[i];
        s2 += (double)X[i] * X[i];
    }
    return (float)(sqrt(s1) / sqrt(s2));
}

/* src/rse.cu:17-30 gencp and :53-73 gencp4: the CP reconstruction
 * sum_r U1[:,r] o U2[:,r] o ... (general order), FP64.                      */
void or_gencp(double *rec, int order, const long *dims, const double *const *U, long R) {
    long total = 1;
    for (int m = 0; m < order; m++) total *= dims[m];
    long idx[16] = {0};
    for (long lin = 0; lin < total; lin++) {
        double s = 0.0;
        for (long r = 0; r < R; r++) {
            double p = 1.0;
            for (int m = 0; m < order; m++) p *= U[m][idx[m] + r * dims[m]];
            s += p;
        }
        rec[lin] = s;
        for (int m = 0; m < order; m++) {
            if (++idx[m] < dims[m]) break;
            idx[m] = 0;
        }
    }
}

/* Mode-n product Y = X x_n W with W (J x I_n) applied to mode n, general
 * order, FP64 (the TTM chains of src/rse.cu:32-51,75-96 and
 * src/tucker_hosvd.cu:78-80 are sequences of these).                        */
void or_mode_product(const double *X, int order, const long *dims, int mode,
                     const double *W, long J, double *Y) {
    long before = 1, after = 1;
    for (int m = 0; m < mode; m++) before *= dims[m];
    for (int m = mode + 1; m < order; m++) after *= dims[m];
    long In = dims[mode];
    memset(Y, 0, sizeof(double) * before * J * after);
    for (long s = 0; s < after; s++)
        for (long q = 0; q < In; q++)
            for (long p = 0; p < before; p++) {
                double x = X[p + before * (q + In * s)];
                if (x == 0.0) continue;
                for (long j = 0; j < J; j++)
                    Y[p + before * (j + J * s)] += x * W[j + J * q];
            }
}

/* ------------------------------------------------------------------------ */
/* Small dense linear algebra used by the CP-ALS restatement.                 */
/* ------------------------------------------------------------------------ */

/* Solve S * Z = Bt for Z, S is R x R, Bt is R x nrhs (column-major), by LU
 * with partial pivoting -- the getrf/getrs pair of src/cp_als.cu:58-61.
 * Returns 0, or the 1-based index of a zero pivot.                          */
int or_lu_solve(double *S, long R, double *Bt, long nrhs) {
    long *piv = (long *)malloc(sizeof(long) * R);
    int info = 0;
    for (long j = 0; j < R; j++) {
        long p = j;
        double best = fabs(S[j + j * R]);
        for (long i = j + 1; i < R; i++)
            if (fabs(S[i + j * R]) > best) { best = fabs(S[i + j * R]); p = i; }
        piv[j] = p;
        if (best == 0.0) { if (!info) info = (int)j + 1; continue; }
        if (p != j)
            for (long c = 0; c < R; c++) {
                double t = S[j + c * R]; S[j + c * R] = S[p + c * R]; S[p + c * R] = t;
            }
        for (long i = j + 1; i < R; i++) {
            double l = S[i + j * R] / S[j + j * R];
            S[i + j * R] = l;
            for (long c = j + 1; c < R; c++) S[i + c * R] -= l * S[j + c * R];
        }
    }
    if (!info) {
        for (long col = 0; col < nrhs; col++) {
            double *b = Bt + col * R;
            for (long j = 0; j < R; j++)
                if (piv[j] != j) { double t = b[j]; b[j] = b[piv[j]]; b[piv[j]] = t; }
            for (long i = 0; i < R; i++)
                for (long j = 0; j < i; j++) b[i] -= S[i + j * R] * b[j];
            for (long i = R - 1; i >= 0; i--) {
                for (long j = i + 1; j < R; j++) b[i] -= S[i + j * R] * b[j];
                b[i] /= S[i + i * R];
            }
        }
    }
    free(piv);
    return info;
}

/* CP-ALS of src/cp_als.cu:44-119 (3rd order) and src/cp4_als.cu:64-164
 * (4th order), generalised to any order: for n = 0..order-1 in turn,
 *   V = Hadamard_{m != n} (U_m^T U_m),  M = MTTKRP_n,  U_n = M V^{-1}
 * with the solve by LU (use_lu=1, the reference's getrf/getrs) or by
 * Cholesky (use_lu=0).  No column normalisation (the reference has none).
 * Stops after max_sweeps sweeps or when |fit - fit_prev| < tol (tol <= 0
 * disables the test, as in the reference's fixed L=500).  fit = 1 -
 * ||X - Xhat|| / ||X||, evaluated after each sweep from the Gram/MTTKRP
 * identity.  Returns the number of sweeps run; fit_hist (may be NULL)
 * receives one fit per sweep.                                               */
int or_cp_als(const float *X, int order, const long *dims, long R, double **U,
              int max_sweeps, double tol, int use_lu, double *fit_hist) {
    long total = 1, maxd = 0;
    for (int m = 0; m < order; m++) { total *= dims[m]; if (dims[m] > maxd) maxd = dims[m]; }
    double normx2 = 0.0;
    for (long i = 0; i < total; i++) normx2 += (double)X[i] * X[i];
    double **G = (double **)malloc(sizeof(double *) * order);
    for (int m = 0; m < order; m++) G[m] = (double *)malloc(sizeof(double) * R * R);
    double *V = (double *)malloc(sizeof(double) * R * R);
    double *M = (double *)malloc(sizeof(double) * maxd * R);
    double *Bt = (double *)malloc(sizeof(double) * maxd * R);
    for (int m = 0; m < order; m++) {
        long I = dims[m];
        for (long a = 0; a < R; a++)
            for (long b = 0; b < R; b++) {
                double s = 0.0;
                for (long i = 0; i < I; i++) s += U[m][i + a * I] * U[m][i + b * I];
                G[m][a + b * R] = s;
            }
    }
    double fit_prev = 0.0;
    int sweep;
    for (sweep = 0; sweep < max_sweeps; sweep++) {
        double inner = 0.0;
        for (int n = 0; n < order; n++) {
            long I = dims[n];
            for (long e = 0; e < R * R; e++) V[e] = 1.0;
            for (int m = 0; m < order; m++)
                if (m != n)
                    for (long e = 0; e < R * R; e++) V[e] *= G[m][e];
            or_mttkrp(X, order, dims, (const double *const *)U, n, R, M);
            /* solve V * U_n^T = M^T */
            for (long i = 0; i < I; i++)
                for (long r = 0; r < R; r++) Bt[r + i * R] = M[i + r * I];
            if (use_lu) {
                or_lu_solve(V, R, Bt, I);
            } else {
                /* Cholesky V = L L^T */
                for (long j = 0; j < R; j++) {
                    double d = V[j + j * R];
                    for (long k = 0; k < j; k++) d -= V[j + k * R] * V[j + k * R];
                    d = sqrt(d > 0 ? d : 0);
                    V[j + j * R] = d;
                    for (long i = j + 1; i < R; i++) {
                        double s = V[i + j * R];
                        for (long k = 0; k < j; k++) s -= V[i + k * R] * V[j + k * R];
                        V[i + j * R] = d > 0 ? s / d : 0.0;
                    }
                }
                for (long col = 0; col < I; col++) {
                    double *b = Bt + col * R;
                    for (long i = 0; i < R; i++) {
                        for (long k = 0; k < i; k++) b[i] -= V[i + k * R] * b[k];
                        b[i] = V[i + i * R] > 0 ? b[i] / V[i + i * R] : 0.0;
                    }
                    for (long i = R - 1; i >= 0; i--) {
                        for (long k = i + 1; k < R; k++) b[i] -= V[k + i * R] * b[k];
                        b[i] = V[i + i * R] > 0 ? b[i] / V[i + i * R] : 0.0;
                    }
                }
            }
            for (long i = 0; i < I; i++)
                for (long r = 0; r < R; r++) U[n][i + r * I] = Bt[r + i * R];
            for (long a = 0; a < R; a++)
                for (long b = 0; b < R; b++) {
                    double s = 0.0;
                    for (long i = 0; i < I; i++) s += U[n][i + a * I] * U[n][i + b * I];
                    G[n][a + b * R] = s;
                }
            if (n == order - 1) {
                inner = 0.0;
                for (long e = 0; e < I * R; e++) inner += U[n][e] * M[e];
            }
        }
        double nrm2 = 0.0;
        for (long e = 0; e < R * R; e++) {
            double p = 1.0;
            for (int m = 0; m < order; m++) p *= G[m][e];
            nrm2 += p;
        }
        double res2 = normx2 - 2.0 * inner + nrm2;
        double fit = 1.0 - sqrt(res2 > 0 ? res2 : 0.0) / sqrt(normx2);
        if (fit_hist) fit_hist[sweep] = fit;
        if (tol > 0 && sweep > 0 && fabs(fit - fit_prev) < tol) { sweep++; break; }
        fit_prev = fit;
    }
    for (int m = 0; m < order; m++) free(G[m]);
    free(G); free(V); free(M); free(Bt);
    return sweep;
}

/* Gram of the mode-n unfolding, G = X_(n) X_(n)^T (I_n x I_n), FP64 -- the
 * SGEMMs of src/tucker_hosvd.cu:27-29 and src/tucker4_hosvd.cu:40-46.       */
void or_unfold_gram(const float *X, int order, const long *dims, int mode, double *G) {
    long before = 1, after = 1;
    for (int m = 0; m < mode; m++) before *= dims[m];
    for (int m = mode + 1; m < order; m++) after *= dims[m];
    long In = dims[mode];
    memset(G, 0, sizeof(double) * In * In);
    double *col = (double *)malloc(sizeof(double) * In);
    for (long s = 0; s < after; s++)
        for (long p = 0; p < before; p++) {
            for (long q = 0; q < In; q++) col[q] = X[p + before * (q + In * s)];
            for (long b = 0; b < In; b++) {
                double xb = col[b];
                if (xb == 0.0) continue;
                for (long a = b; a < In; a++) G[a + b * In] += col[a] * xb;
            }
        }
    for (long b = 0; b < In; b++)
        for (long a = b + 1; a < In; a++) G[b + a * In] = G[a + b * In];
    free(col);
}
