// FP64 blocked two-sided Jacobi eigensolver for the symmetric I_n x I_n
// unfolding Grams of HOSVD/HOOI (replaces cusolverDnSsyevdx at
// src/tucker_hosvd.cu:43-61).
//
// The matrix is cut into blocks of BS rows/columns.  One sweep visits every
// pair of blocks once in round-robin order; in each round the nb/2 disjoint
// pairs are processed in parallel:
//   1. each pair (I, J) diagonalises its 2BS x 2BS principal submatrix in
//      shared memory (inner cyclic Jacobi), giving an orthogonal Q_IJ;
//   2. columns:  A[:, IJ] <- A[:, IJ] Q_IJ,   V[:, IJ] <- V[:, IJ] Q_IJ;
//   3. rows:     A[IJ, :] <- Q_IJ^T A[IJ, :].
// One cooperative launch runs all sweeps; the phases are separated by a grid
// barrier whose spin is bounded (an expired wait sets an error flag and every
// CTA returns).  Convergence: off(A) <= tol^2 * ||A||_F^2, tested at the start
// of each sweep from per-CTA partial sums reduced in a fixed order.
#include <vector>
#include <algorithm>

#include "kernels.cuh"

namespace cud {

namespace {

constexpr int BS = 16;          // block size
constexpr int M2 = 2 * BS;      // pair submatrix size
constexpr int NT = 256;
constexpr long kSpinLimit = 1L << 24;
constexpr double kInnerTol = 4e-15 * M2;  // relative off-norm at which a pair block counts as diagonal

struct EigArgs {
    double *A;          // n x n, destroyed
    double *V;          // n x n, eigenvectors (unsorted)
    double *Q;          // npairs x M2 x M2
    double *part;       // gridDim partial sums (2 per CTA)
    unsigned *bar;      // [count, generation]
    int *status;        // [error, sweeps]
    int n, nb, max_sweeps;
    double tol;
};

__device__ bool grid_barrier(const EigArgs &a) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        volatile unsigned *gen = a.bar + 1;
        unsigned g = *gen;
        __threadfence();
        unsigned arrived = atomicAdd(a.bar, 1u);
        if (arrived == gridDim.x - 1) {
            atomicExch(a.bar, 0u);
            __threadfence();
            atomicAdd(a.bar + 1, 1u);
        } else {
            long it = 0;
            while (*gen == g) {
                if (++it > kSpinLimit) { atomicExch(a.status, 1); break; }
                __nanosleep(64);
            }
        }
        __threadfence();
        s_ok = (*(volatile int *)a.status == 0);
    }
    __syncthreads();
    return s_ok;
}

__device__ __forceinline__ void pair_blocks(int k, int round, int nb, int &I, int &J) {
    int a = (k == 0) ? 0 : 1 + (k - 1 + round) % (nb - 1);
    int b = 1 + (nb - 2 - k + round) % (nb - 1);
    I = min(a, b);
    J = max(a, b);
}

__device__ __forceinline__ int pair_index(int I, int J, int jj) {
    return (jj < BS) ? I * BS + jj : J * BS + (jj - BS);
}

// Cyclic Jacobi on S (M2 x M2, shared), accumulating Q (shared).
__device__ void inner_jacobi(double *S, double *Q, double tol) {
    __shared__ double c_[M2 / 2], s_[M2 / 2];
    __shared__ int p_[M2 / 2], q_[M2 / 2];
    __shared__ int s_go;
    for (int e = threadIdx.x; e < M2 * M2; e += blockDim.x) Q[e] = (e % M2 == e / M2) ? 1.0 : 0.0;
    __syncthreads();
    for (int sweep = 0; sweep < 12; sweep++) {
        if (threadIdx.x < 32) {
            double off = 0.0, tot = 0.0;
            for (int e = threadIdx.x; e < M2 * M2; e += 32) {
                double v = S[e] * S[e];
                tot += v;
                if (e % M2 != e / M2) off += v;
            }
            for (int o = 16; o > 0; o >>= 1) {
                off += __shfl_xor_sync(0xffffffffu, off, o);
                tot += __shfl_xor_sync(0xffffffffu, tot, o);
            }
            if (threadIdx.x == 0) s_go = (off > tol * tol * tot) && tot > 0.0;
        }
        __syncthreads();
        if (!s_go) break;
        for (int round = 0; round < M2 - 1; round++) {
            if (threadIdx.x < M2 / 2) {
                int k = threadIdx.x;
                int a = (k == 0) ? 0 : 1 + (k - 1 + round) % (M2 - 1);
                int b = 1 + (M2 - 2 - k + round) % (M2 - 1);
                int p = min(a, b), q = max(a, b);
                double apq = S[p + M2 * q], app = S[p + M2 * p], aqq = S[q + M2 * q];
                double c = 1.0, s = 0.0;
                if (fabs(apq) > 1e-300 && fabs(apq) > 1e-17 * sqrt(fabs(app * aqq))) {
                    double theta = (aqq - app) / (2.0 * apq);
                    double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                    c = 1.0 / sqrt(t * t + 1.0);
                    s = t * c;
                }
                p_[k] = p; q_[k] = q; c_[k] = c; s_[k] = s;
            }
            __syncthreads();
            for (int e = threadIdx.x; e < (M2 / 2) * M2; e += blockDim.x) {
                int k = e / M2, col = e % M2;
                int p = p_[k], q = q_[k];
                double c = c_[k], s = s_[k];
                double ap = S[p + M2 * col], aq = S[q + M2 * col];
                S[p + M2 * col] = c * ap - s * aq;
                S[q + M2 * col] = s * ap + c * aq;
            }
            __syncthreads();
            for (int e = threadIdx.x; e < (M2 / 2) * M2; e += blockDim.x) {
                int k = e / M2, row = e % M2;
                int p = p_[k], q = q_[k];
                double c = c_[k], s = s_[k];
                double ap = S[row + M2 * p], aq = S[row + M2 * q];
                S[row + M2 * p] = c * ap - s * aq;
                S[row + M2 * q] = s * ap + c * aq;
                double vp = Q[row + M2 * p], vq = Q[row + M2 * q];
                Q[row + M2 * p] = c * vp - s * vq;
                Q[row + M2 * q] = s * vp + c * vq;
            }
            __syncthreads();
        }
    }
}

__global__ void __launch_bounds__(NT) k_block_jacobi(EigArgs a) {
    __shared__ double S[M2 * M2];
    __shared__ double Qs[M2 * M2];
    __shared__ double red[2][NT / 32];
    const int n = a.n, nb = a.nb, npairs = nb / 2;
    const long nn = (long)n * n;

    // V = I
    for (long e = blockIdx.x * (long)NT + threadIdx.x; e < nn; e += (long)gridDim.x * NT)
        a.V[e] = (e % n == e / n) ? 1.0 : 0.0;
    if (!grid_barrier(a)) return;

    int sweep = 0;
    for (;; sweep++) {
        // convergence test: per-CTA partials, reduced in fixed order by all
        double off = 0.0, tot = 0.0;
        for (long e = blockIdx.x * (long)NT + threadIdx.x; e < nn; e += (long)gridDim.x * NT) {
            double v = a.A[e] * a.A[e];
            tot += v;
            if (e % n != e / n) off += v;
        }
        for (int o = 16; o > 0; o >>= 1) {
            off += __shfl_xor_sync(0xffffffffu, off, o);
            tot += __shfl_xor_sync(0xffffffffu, tot, o);
        }
        if ((threadIdx.x & 31) == 0) { red[0][threadIdx.x >> 5] = off; red[1][threadIdx.x >> 5] = tot; }
        __syncthreads();
        if (threadIdx.x == 0) {
            double o2 = 0.0, t2 = 0.0;
            for (int w = 0; w < NT / 32; w++) { o2 += red[0][w]; t2 += red[1][w]; }
            a.part[2 * blockIdx.x] = o2;
            a.part[2 * blockIdx.x + 1] = t2;
        }
        if (!grid_barrier(a)) return;
        double offs = 0.0, tots = 0.0;
        for (int b = 0; b < (int)gridDim.x; b++) {
            offs += ((volatile double *)a.part)[2 * b];
            tots += ((volatile double *)a.part)[2 * b + 1];
        }
        if (!(offs > a.tol * a.tol * tots) || tots == 0.0) break;
        if (sweep >= a.max_sweeps) {
            if (blockIdx.x == 0 && threadIdx.x == 0) a.status[0] = 2;
            break;
        }
        if (!grid_barrier(a)) return;  // everyone has read part before it is rewritten

        for (int round = 0; round < nb - 1; round++) {
            // phase 1: diagonalise each pair's 2BS x 2BS block
            for (int k = blockIdx.x; k < npairs; k += gridDim.x) {
                int I, J;
                pair_blocks(k, round, nb, I, J);
                for (int e = threadIdx.x; e < M2 * M2; e += NT) {
                    int ii = e % M2, jj = e / M2;
                    int gi = pair_index(I, J, ii), gj = pair_index(I, J, jj);
                    S[e] = (gi < n && gj < n) ? a.A[gi + (long)n * gj] : 0.0;
                }
                __syncthreads();
                inner_jacobi(S, Qs, kInnerTol);
                double *Qg = a.Q + (long)k * M2 * M2;
                for (int e = threadIdx.x; e < M2 * M2; e += NT) Qg[e] = Qs[e];
                __syncthreads();
            }
            if (!grid_barrier(a)) return;
            // phase 2: columns of A and V
            {
                int rchunks = (n + NT - 1) / NT;
                for (int task = blockIdx.x; task < npairs * rchunks; task += gridDim.x) {
                    int k = task % npairs, rc = task / npairs;
                    int I, J;
                    pair_blocks(k, round, nb, I, J);
                    const double *Qg = a.Q + (long)k * M2 * M2;
                    __syncthreads();
                    for (int e = threadIdx.x; e < M2 * M2; e += NT) Qs[e] = Qg[e];
                    __syncthreads();
                    int r = rc * NT + threadIdx.x;
                    if (r < n) {
                        for (int which = 0; which < 2; which++) {
                            double *Mx = which ? a.V : a.A;
                            double x[M2];
#pragma unroll
                            for (int jj = 0; jj < M2; jj++) {
                                int g = pair_index(I, J, jj);
                                x[jj] = (g < n) ? Mx[r + (long)n * g] : 0.0;
                            }
#pragma unroll 4
                            for (int jj = 0; jj < M2; jj++) {
                                int g = pair_index(I, J, jj);
                                if (g >= n) continue;
                                double s = 0.0;
#pragma unroll
                                for (int ii = 0; ii < M2; ii++) s = fma(x[ii], Qs[ii + M2 * jj], s);
                                Mx[r + (long)n * g] = s;
                            }
                        }
                    }
                }
            }
            if (!grid_barrier(a)) return;
            // phase 3: rows of A
            {
                int cchunks = (n + NT - 1) / NT;
                for (int task = blockIdx.x; task < npairs * cchunks; task += gridDim.x) {
                    int k = task % npairs, cc = task / npairs;
                    int I, J;
                    pair_blocks(k, round, nb, I, J);
                    const double *Qg = a.Q + (long)k * M2 * M2;
                    __syncthreads();
                    for (int e = threadIdx.x; e < M2 * M2; e += NT) Qs[e] = Qg[e];
                    __syncthreads();
                    int c = cc * NT + threadIdx.x;
                    if (c < n) {
                        double x[M2];
#pragma unroll
                        for (int ii = 0; ii < M2; ii++) {
                            int g = pair_index(I, J, ii);
                            x[ii] = (g < n) ? a.A[g + (long)n * c] : 0.0;
                        }
#pragma unroll 4
                        for (int jj = 0; jj < M2; jj++) {
                            int g = pair_index(I, J, jj);
                            if (g >= n) continue;
                            double s = 0.0;
#pragma unroll
                            for (int ii = 0; ii < M2; ii++) s = fma(Qs[ii + M2 * jj], x[ii], s);
                            a.A[g + (long)n * c] = s;
                        }
                    }
                }
            }
            if (!grid_barrier(a)) return;
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) a.status[1] = sweep;
}

// W ascending with V's columns permuted to match.
__global__ void k_sort_eig(const double *__restrict__ A, const double *__restrict__ Vin, int n,
                           double *__restrict__ W, double *__restrict__ Vout, int *__restrict__ perm) {
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        for (int i = 0; i < n; i++) perm[i] = i;
        // insertion sort by eigenvalue (n is at most a few thousand)
        for (int i = 1; i < n; i++) {
            int p = perm[i];
            double v = A[p + (long)n * p];
            int j = i - 1;
            while (j >= 0 && A[perm[j] + (long)n * perm[j]] > v) { perm[j + 1] = perm[j]; j--; }
            perm[j + 1] = p;
        }
        for (int i = 0; i < n; i++) W[i] = A[perm[i] + (long)n * perm[i]];
    }
}

__global__ void k_permute_cols(const double *__restrict__ Vin, const int *__restrict__ perm, int n,
                               double *__restrict__ Vout) {
    long nn = (long)n * n;
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < nn; e += (long)gridDim.x * blockDim.x) {
        long r = e % n, c = e / n;
        Vout[e] = Vin[r + (long)n * perm[c]];
    }
}

}  // namespace

int syev_jacobi(double *A, long n, double *W, double *V, int max_sweeps, cudaStream_t s) {
    if (n <= 0) return CUD_OK;
    if (n > 32768) return CUD_ERR_UNSUPPORTED;
    int nb = (int)((n + BS - 1) / BS);
    if (nb < 2) nb = 2;
    if (nb & 1) nb++;
    int npairs = nb / 2;
    int dev = 0, occ = 0;
    CUD_CHECK(cudaGetDevice(&dev));
    CUD_CHECK(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, k_block_jacobi, NT, 0));
    int sms = 0;
    CUD_CHECK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    int grid = std::max(1, std::min(occ * sms, std::max(npairs, sms)));
    size_t bytes_Q = sizeof(double) * (size_t)npairs * M2 * M2;
    size_t bytes_V = sizeof(double) * (size_t)n * n;
    size_t off_part = bytes_Q;
    size_t off_bar = off_part + sizeof(double) * 2 * grid;
    size_t off_st = off_bar + 64;
    size_t off_Vt = (off_st + 64 + 255) & ~size_t(255);
    size_t off_perm = off_Vt + bytes_V;
    int st;
    char *w = (char *)scratch(kSlotEig, off_perm + sizeof(int) * n + 64, &st);
    if (!w) return st;
    EigArgs a;
    a.A = A;
    a.V = (double *)(w + off_Vt);
    a.Q = (double *)w;
    a.part = (double *)(w + off_part);
    a.bar = (unsigned *)(w + off_bar);
    a.status = (int *)(w + off_st);
    a.n = (int)n;
    a.nb = nb;
    a.max_sweeps = max_sweeps > 0 ? max_sweeps : 40;
    // off(A) can only be driven to the rounding floor of the rotations,
    // about n * eps relative to ||A||_F, and no lower than the pair blocks'
    // own stop (kInnerTol of each block's norm): with a tighter outer test a
    // clustered spectrum (a near low-rank Gram) never met it
    a.tol = std::max(4.0 * 2.22e-16 * (double)std::max(16L, n), kInnerTol);
    CUD_CHECK(cudaMemsetAsync(w + off_bar, 0, 128, s));
    void *args[] = {&a};
    CUD_CHECK(cudaLaunchCooperativeKernel((void *)k_block_jacobi, grid, NT, args, 0, s));
    CUD_CHECK_LAUNCH("syev_jacobi");
    int *perm = (int *)(w + off_perm);
    k_sort_eig<<<1, 32, 0, s>>>(A, a.V, (int)n, W, V, perm);
    k_permute_cols<<<blocks_for(n * n, 256), 256, 0, s>>>(a.V, perm, (int)n, V);
    CUD_CHECK_LAUNCH("syev_jacobi sort");
    int hst[2] = {0, 0};
    CUD_CHECK(cudaMemcpyAsync(hst, a.status, sizeof(hst), cudaMemcpyDeviceToHost, s));
    CUD_CHECK(cudaStreamSynchronize(s));
    if (hst[0] == 1) return CUD_ERR_DEVICE_TIMEOUT;
    if (hst[0] == 2) return CUD_ERR_NOT_CONVERGED;
    return CUD_OK;
}

}  // namespace cud

extern "C" int cud_syev_jacobi(double *A, long n, double *W, double *V, int max_sweeps, void *stream) {
    if (n < 0 || (n > 0 && (!A || !W || !V))) return cud::set_status(CUD_ERR_INVALID_ARGUMENT);
    return cud::set_status(cud::syev_jacobi(A, n, W, V, max_sweeps, cud::as_stream(stream)));
}
