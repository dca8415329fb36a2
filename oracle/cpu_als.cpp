// CPU baseline (test and benchmark infrastructure, not the product): the ALS
// of the reference's CPU path, decomposition/CPU/python/mycp.py:7-22, in C++
// with OpenMP, FP32 or FP64 arithmetic.  Per sweep, for each mode n in turn
// (mycp.py:10-20):
//   V = Hadamard product of the other factors' Grams U_m^T U_m      (:10,14,18)
//   M = unfolding_dot_khatri_rao(X, factors, n)  = X_(n) (KR others) (:11,15,19)
//   U_n = M V^-1, solved as the transposed system V^T U_n^T = M^T     (:12,16,20)
// (LU with partial pivoting, as numpy.linalg.solve behind tl.solve), then
// the fit from ||X||^2 - 2 <M_N, U_N> + sum prod G (after the last mode).
// Any order; column-major tensors and factors (dims[m] x R), as the GPU
// library.  mycp.py runs a fixed 10 iterations; here max_sweeps, a delta-fit
// tolerance and a target fit set the stop, as the GPU runs they are timed
// against.
//
// The MTTKRP streams X once in its native layout around mode n, viewed as
// (P, Q, S): with L = KR of the factors before n (P x R) and T = KR of the
// factors after n (S x R), M[q, :] = sum_s T[s, :] * sum_p X[p, q, s] L[p, :].
// OpenMP splits the work items (chunks of s for mode 0, (s, chunk of p)
// otherwise) across threads with private accumulators, summed in thread
// order.
#include <math.h>
#include <omp.h>
#include <stdlib.h>
#include <string.h>

#include <vector>

namespace {

template <typename T>
void kr_rows(const std::vector<const T *> &U, const std::vector<long> &rows, long R, std::vector<T> &out,
             long &n) {
    // out (n x R, row-major: rank contiguous) = Khatri-Rao rows, first factor fastest
    n = 1;
    for (long d : rows) n *= d;
    out.assign((size_t)n * R, T(1));
#pragma omp parallel for schedule(static)
    for (long i = 0; i < n; i++) {
        long lin = i;
        T *o = &out[(size_t)i * R];
        for (size_t f = 0; f < U.size(); f++) {
            const long d = rows[f], ix = lin % d;
            lin /= d;
            for (long r = 0; r < R; r++) o[r] *= U[f][ix + d * r];
        }
    }
}

// Register tile of the MTTKRP micro-kernel: 4 rows q x RB ranks (two AVX2
// registers of FP32 per row, or two of FP64 for half as many ranks).
template <typename T> struct Tile;
template <> struct Tile<float> { static constexpr long RB = 16; };
template <> struct Tile<double> { static constexpr long RB = 8; };

template <typename T>
void mttkrp(const T *X, int order, const long *dims, T *const *U, int mode, long R, T *out, int threads) {
    constexpr long RB = Tile<T>::RB;
    long P = 1, S = 1;
    const long Q = dims[mode];
    std::vector<const T *> lu, tu;
    std::vector<long> lr, tr;
    for (int m = 0; m < mode; m++) { P *= dims[m]; lu.push_back(U[m]); lr.push_back(dims[m]); }
    for (int m = mode + 1; m < order; m++) { S *= dims[m]; tu.push_back(U[m]); tr.push_back(dims[m]); }
    std::vector<T> L0, Tt;
    long nl, nt;
    kr_rows(lu, lr, R, L0, nl);
    kr_rows(tu, tr, R, Tt, nt);
    // L with its rows padded to Rp = a multiple of RB ranks (zeros)
    const long Rp = (R + RB - 1) / RB * RB;
    std::vector<T> L((size_t)P * Rp, T(0));
#pragma omp parallel for schedule(static)
    for (long p = 0; p < P; p++)
        for (long r = 0; r < R; r++) L[(size_t)p * Rp + r] = L0[(size_t)p * R + r];
    const int nth = threads > 0 ? threads : omp_get_max_threads();
    std::vector<T> acc((size_t)nth * Q * R, T(0));
    if (P == 1) {
        // mode 0: M = X_(0) T, a GEMM over s with X's rows q contiguous.
        // Items: chunks of SC values of s; micro-kernel: 8 rows q (one
        // vector of x) x 8 ranks held in registers over the chunk.  Static
        // schedule: the summation order is fixed.
        constexpr long SC = 512, QV = 8, RV = 8;
        const long items = (S + SC - 1) / SC;
#pragma omp parallel num_threads(nth)
        {
            T *a = &acc[(size_t)omp_get_thread_num() * Q * R];
#pragma omp for schedule(static)
            for (long it = 0; it < items; it++) {
                const long s0 = it * SC, s1 = s0 + SC < S ? s0 + SC : S;
                for (long q0 = 0; q0 < Q; q0 += QV) {
                    const long nq = Q - q0 < QV ? Q - q0 : QV;
                    for (long r0 = 0; r0 < R; r0 += RV) {
                        const long nr = R - r0 < RV ? R - r0 : RV;
                        T c[RV][QV];
                        for (long r = 0; r < RV; r++)
                            for (long i = 0; i < QV; i++) c[r][i] = T(0);
                        if (nq == QV && nr == RV) {
                            for (long ss = s0; ss < s1; ss++) {
                                const T *x = X + q0 + Q * ss;
                                const T *w = &Tt[(size_t)ss * R + r0];
                                for (long r = 0; r < RV; r++) {
                                    const T wr = w[r];
#pragma omp simd
                                    for (long i = 0; i < QV; i++) c[r][i] += x[i] * wr;
                                }
                            }
                        } else {
                            for (long ss = s0; ss < s1; ss++)
                                for (long r = 0; r < nr; r++)
                                    for (long i = 0; i < nq; i++) c[r][i] += X[q0 + i + Q * ss] * Tt[(size_t)ss * R + r0 + r];
                        }
                        for (long r = 0; r < nr; r++)
                            for (long i = 0; i < nq; i++) a[(size_t)(q0 + i) * R + r0 + r] += c[r][i];
                    }
                }
            }
        }
    } else {
        // other modes: items (s, chunk of PC values of p) covering every row
        // q, so L streams through the caches once per s; micro-kernel: 4 rows
        // q x RB ranks held in registers over the chunk, scaled by T's row s
        // when added.  Static schedule: the summation order is fixed.
        constexpr long PC = 4096;
        const long nch = (P + PC - 1) / PC;
        const long items = S * nch;
#pragma omp parallel num_threads(nth)
        {
            T *a = &acc[(size_t)omp_get_thread_num() * Q * R];
            const T zero[1] = {T(0)};
#pragma omp for schedule(static)
            for (long it = 0; it < items; it++) {
                const long s = it / nch, p0 = (it % nch) * PC;
                const long p1 = p0 + PC < P ? p0 + PC : P;
                const T *ts = &Tt[(size_t)s * R];
                for (long qq = 0; qq < Q; qq += 4) {
                    // rows past Q read a zero and add nothing
                    const T *x[4];
                    long inc[4];
                    for (int i = 0; i < 4; i++) {
                        const bool ok = qq + i < Q;
                        x[i] = ok ? X + P * (qq + i + Q * s) : zero;
                        inc[i] = ok ? 1 : 0;
                    }
                    for (long r0 = 0; r0 < Rp; r0 += RB) {
                        T c[4][RB];
                        for (int i = 0; i < 4; i++)
                            for (long rr = 0; rr < RB; rr++) c[i][rr] = T(0);
                        for (long p = p0; p < p1; p++) {
                            const T *l = &L[(size_t)p * Rp + r0];
                            const T x0 = x[0][p * inc[0]], x1 = x[1][p * inc[1]], x2 = x[2][p * inc[2]],
                                    x3 = x[3][p * inc[3]];
#pragma omp simd
                            for (long rr = 0; rr < RB; rr++) {
                                c[0][rr] += x0 * l[rr];
                                c[1][rr] += x1 * l[rr];
                                c[2][rr] += x2 * l[rr];
                                c[3][rr] += x3 * l[rr];
                            }
                        }
                        for (int i = 0; i < 4 && qq + i < Q; i++) {
                            T *ar = a + (size_t)(qq + i) * R;
                            for (long rr = 0; rr < RB && r0 + rr < R; rr++) ar[r0 + rr] += c[i][rr] * ts[r0 + rr];
                        }
                    }
                }
            }
        }
    }
    // sum the threads' accumulators in thread order; out is column-major Q x R
#pragma omp parallel for num_threads(nth) schedule(static)
    for (long q = 0; q < Q; q++)
        for (long r = 0; r < R; r++) {
            T sum = T(0);
            for (int k = 0; k < nth; k++) sum += acc[(size_t)k * Q * R + (size_t)q * R + r];
            out[q + Q * r] = sum;
        }
}

template <typename T>
void gram(const T *U, long I, long R, double *G) {
    for (long a = 0; a < R; a++)
        for (long b = 0; b < R; b++) {
            double s = 0.0;
            for (long i = 0; i < I; i++) s += (double)U[i + I * a] * (double)U[i + I * b];
            G[a + R * b] = s;
        }
}

// Solves A^T Y^T = B^T for Y (I x R) with A (R x R) by LU with partial pivoting
// (A^T factored once, I right-hand sides).  Returns 0, or 1 when singular.
template <typename T>
int solve_rows(const double *A, long R, const T *B, long I, T *Y, int threads) {
    std::vector<double> F((size_t)R * R);
    std::vector<long> piv(R);
    for (long i = 0; i < R; i++)
        for (long j = 0; j < R; j++) F[i + R * j] = A[j + R * i];  // A^T
    for (long k = 0; k < R; k++) {
        long p = k;
        for (long i = k + 1; i < R; i++)
            if (fabs(F[i + R * k]) > fabs(F[p + R * k])) p = i;
        piv[k] = p;
        if (F[p + R * k] == 0.0) return 1;
        if (p != k)
            for (long j = 0; j < R; j++) { double t = F[k + R * j]; F[k + R * j] = F[p + R * j]; F[p + R * j] = t; }
        for (long i = k + 1; i < R; i++) {
            F[i + R * k] /= F[k + R * k];
            for (long j = k + 1; j < R; j++) F[i + R * j] -= F[i + R * k] * F[k + R * j];
        }
    }
#pragma omp parallel for num_threads(threads) schedule(static)
    for (long i = 0; i < I; i++) {
        std::vector<double> x((size_t)R);
        for (long r = 0; r < R; r++) x[r] = (double)B[i + I * r];
        for (long k = 0; k < R; k++)
            if (piv[k] != k) { double t = x[k]; x[k] = x[piv[k]]; x[piv[k]] = t; }
        for (long k = 0; k < R; k++)
            for (long j = 0; j < k; j++) x[k] -= F[k + R * j] * x[j];
        for (long k = R - 1; k >= 0; k--) {
            for (long j = k + 1; j < R; j++) x[k] -= F[k + R * j] * x[j];
            x[k] /= F[k + R * k];
        }
        for (long r = 0; r < R; r++) Y[i + I * r] = (T)x[r];
    }
    return 0;
}

template <typename T>
int cp_als(const T *X, int order, const long *dims, long R, T *const *U, int max_sweeps, double tol,
           double target_fit, int threads, double *fits, int *sweeps_out, double *seconds) {
    if (order < 2 || order > 8 || R <= 0) return 2;
    const int nth = threads > 0 ? threads : omp_get_max_threads();
    const double t0 = omp_get_wtime();
    long n = 1, maxd = 0;
    for (int m = 0; m < order; m++) { n *= dims[m]; maxd = dims[m] > maxd ? dims[m] : maxd; }
    double nx2 = 0.0;
#pragma omp parallel for num_threads(nth) reduction(+ : nx2) schedule(static)
    for (long e = 0; e < n; e++) nx2 += (double)X[e] * (double)X[e];
    std::vector<double> G((size_t)order * R * R), V((size_t)R * R);
    for (int m = 0; m < order; m++) gram(U[m], dims[m], R, &G[(size_t)m * R * R]);
    std::vector<T> M((size_t)maxd * R);
    double fit_prev = 0.0;
    int sw = 0;
    for (; sw < max_sweeps;) {
        double inner = 0.0;
        for (int mode = 0; mode < order; mode++) {
            for (long e = 0; e < R * R; e++) {
                double v = 1.0;
                for (int m = 0; m < order; m++)
                    if (m != mode) v *= G[(size_t)m * R * R + e];
                V[e] = v;
            }
            mttkrp(X, order, dims, U, mode, R, M.data(), nth);
            if (solve_rows(V.data(), R, M.data(), dims[mode], U[mode], nth)) return 1;
            gram(U[mode], dims[mode], R, &G[(size_t)mode * R * R]);
            if (mode == order - 1)
                for (long e = 0; e < dims[mode] * R; e++) inner += (double)M[e] * (double)U[mode][e];
        }
        double hat = 0.0;
        for (long e = 0; e < R * R; e++) {
            double v = 1.0;
            for (int m = 0; m < order; m++) v *= G[(size_t)m * R * R + e];
            hat += v;
        }
        const double res2 = nx2 - 2.0 * inner + hat;
        const double fit = 1.0 - sqrt(res2 > 0.0 ? res2 : 0.0) / sqrt(nx2);
        if (fits) fits[sw] = fit;
        sw++;
        if (target_fit > 0.0 && fit >= target_fit) break;
        if (tol > 0.0 && sw >= 2 && fabs(fit - fit_prev) < tol) break;
        fit_prev = fit;
    }
    if (sweeps_out) *sweeps_out = sw;
    if (seconds) *seconds = omp_get_wtime() - t0;
    return 0;
}

}  // namespace

extern "C" {

int cpu_mttkrp_f32(const float *X, int order, const long *dims, float *const *U, int mode, long R, float *out,
                   int threads) {
    mttkrp<float>(X, order, dims, U, mode, R, out, threads);
    return 0;
}

int cpu_mttkrp_f64(const double *X, int order, const long *dims, double *const *U, int mode, long R, double *out,
                   int threads) {
    mttkrp<double>(X, order, dims, U, mode, R, out, threads);
    return 0;
}

int cpu_cp_als_f32(const float *X, int order, const long *dims, long R, float *const *U, int max_sweeps,
                   double tol, double target_fit, int threads, double *fits, int *sweeps, double *seconds) {
    return cp_als<float>(X, order, dims, R, U, max_sweeps, tol, target_fit, threads, fits, sweeps, seconds);
}

int cpu_cp_als_f64(const double *X, int order, const long *dims, long R, double *const *U, int max_sweeps,
                   double tol, double target_fit, int threads, double *fits, int *sweeps, double *seconds) {
    return cp_als<double>(X, order, dims, R, U, max_sweeps, tol, target_fit, threads, fits, sweeps, seconds);
}

int cpu_max_threads(void) { return omp_get_max_threads(); }

}  // extern "C"
