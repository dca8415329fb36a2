// Leading eigenvectors of a symmetric positive semi-definite FP64 matrix by
// subspace iteration, for the Tucker factors (the r_n leading eigenvectors
// of an I_n x I_n unfolding Gram; the reference asks cuSOLVER's syevdx for
// them, src/tucker_hosvd.cu:38-56).
//
//   V <- orth(G V)   (CholQR, applied twice for orthogonality),
//
// from a seeded Gaussian start, until the subspace stops moving
// (r - ||V_old^T V_new||_F^2 = sum of squared sines of the principal angles
// below a tolerance), then Rayleigh-Ritz: the r x r matrix V^T G V is
// diagonalised by Jacobi in shared memory and its eigenvectors rotate V.
// The iteration converges at the rate lambda_{r+1} / lambda_r, i.e. in a few
// steps when the Gram has a gap after its r-th eigenvalue (a low-rank-plus-
// noise tensor); callers fall back to the full Jacobi eigensolver when it
// does not converge.
#include "kernels.cuh"

namespace cud {

namespace {

constexpr int SI_RMAX = 64;

__device__ __forceinline__ unsigned long long si_mix(unsigned long long z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

// V (n x r) = i.i.d. standard normal (Box-Muller over a counter hash).
__global__ void k_si_init(double *V, long n, int r) {
    const long total = n * r;
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
        const double u1 = 1.0 - (double)(si_mix(2 * e + 0x51) >> 11) * (1.0 / 9007199254740992.0);
        const double u2 = (double)(si_mix(2 * e + 0x52) >> 11) * (1.0 / 9007199254740992.0);
        V[e] = sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
    }
}

// Y (n x r) = G (n x n) V (n x r), column-major.
__global__ void __launch_bounds__(256) k_si_apply(const double *__restrict__ G, const double *__restrict__ V,
                                                  long n, int r, double *__restrict__ Y) {
    const long total = n * r;
    for (long e = blockIdx.x * 256L + threadIdx.x; e < total; e += (long)gridDim.x * 256L) {
        const long i = e % n, c = e / n;
        double s = 0.0;
        for (long k = 0; k < n; k++) s = fma(G[i + n * k], V[k + n * c], s);
        Y[e] = s;
    }
}

// In place Y <- Y L^-T with L L^T = Y^T Y (Cholesky QR), one CTA.  Sets
// *fail when Y^T Y is not numerically positive definite.
__global__ void __launch_bounds__(256) k_si_cholqr(double *Y, long n, int r, int *fail) {
    __shared__ double C[SI_RMAX * SI_RMAX];
    __shared__ int bad;
    for (int e = threadIdx.x; e < r * r; e += blockDim.x) {
        const int a = e % r, b = e / r;
        double s = 0.0;
        if (a >= b)
            for (long i = 0; i < n; i++) s = fma(Y[i + n * a], Y[i + n * b], s);
        C[e] = s;
    }
    if (threadIdx.x == 0) bad = 0;
    __syncthreads();
    // Cholesky (lower, column by column), small: one column per step
    for (int j = 0; j < r; j++) {
        if (threadIdx.x == 0) {
            double d = C[j + r * j];
            for (int k = 0; k < j; k++) d -= C[j + r * k] * C[j + r * k];
            if (!(d > 0.0) || !isfinite(d)) { bad = 1; d = 1.0; }
            C[j + r * j] = sqrt(d);
        }
        __syncthreads();
        for (int i = j + 1 + threadIdx.x; i < r; i += blockDim.x) {
            double s = C[i + r * j];
            for (int k = 0; k < j; k++) s -= C[i + r * k] * C[j + r * k];
            C[i + r * j] = s / C[j + r * j];
        }
        __syncthreads();
    }
    if (bad) {
        if (threadIdx.x == 0) *fail = 1;
        return;
    }
    // rows of Y: y_i <- L^-1 y_i (forward substitution), i.e. Y <- Y L^-T
    for (long i = threadIdx.x; i < n; i += blockDim.x) {
        double z[SI_RMAX];
        for (int a = 0; a < r; a++) {
            double s = Y[i + n * a];
            for (int k = 0; k < a; k++) s -= C[a + r * k] * z[k];
            z[a] = s / C[a + r * a];
        }
        for (int a = 0; a < r; a++) Y[i + n * a] = z[a];
    }
}

// out = r - ||A^T B||_F^2 (A, B n x r orthonormal), one CTA.
__global__ void __launch_bounds__(256) k_si_gap(const double *A, const double *B, long n, int r, double *out) {
    __shared__ double red[256];
    double acc = 0.0;
    for (int e = threadIdx.x; e < r * r; e += blockDim.x) {
        const int a = e % r, b = e / r;
        double s = 0.0;
        for (long i = 0; i < n; i++) s = fma(A[i + n * a], B[i + n * b], s);
        acc += s * s;
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[0] = (double)r - red[0];
}

// Rayleigh-Ritz: H = V^T Y (Y = G V), Jacobi on H in shared memory, then
// U[:, j] = V w_j for the eigenvalues in ascending order (FP32 out).  One CTA.
__global__ void __launch_bounds__(256) k_si_ritz(const double *V, const double *Y, long n, int r, float *U,
                                                 double *W) {
    __shared__ double H[SI_RMAX * SI_RMAX];  // W (r x r rotations) lives in global scratch
    __shared__ double cs[SI_RMAX / 2], sn[SI_RMAX / 2];
    __shared__ int pp[SI_RMAX / 2], qq[SI_RMAX / 2], ord[SI_RMAX];
    __shared__ double off_s;
    for (int e = threadIdx.x; e < r * r; e += blockDim.x) {
        const int a = e % r, b = e / r;
        double s = 0.0;
        for (long i = 0; i < n; i++) s = fma(V[i + n * a], Y[i + n * b], s);
        H[e] = s;
        W[e] = (a == b) ? 1.0 : 0.0;
    }
    __syncthreads();
    for (int e = threadIdx.x; e < r * r; e += blockDim.x) {  // symmetrise
        const int a = e % r, b = e / r;
        if (a < b) {
            const double m = 0.5 * (H[a + r * b] + H[b + r * a]);
            H[a + r * b] = m;
            H[b + r * a] = m;
        }
    }
    __syncthreads();
    const int m = (r + 1) & ~1;
    for (int sweep = 0; sweep < 40; sweep++) {
        if (threadIdx.x == 0) {
            double off = 0.0, tot = 0.0;
            for (int e = 0; e < r * r; e++) {
                tot += H[e] * H[e];
                if (e % r != e / r) off += H[e] * H[e];
            }
            off_s = (off <= 1e-30 * tot) ? -1.0 : off;
        }
        __syncthreads();
        if (off_s < 0) break;
        for (int round = 0; round < m - 1; round++) {
            if (threadIdx.x < m / 2) {
                const int k = threadIdx.x;
                int a = (k == 0) ? m - 1 : (round + k) % (m - 1);
                int b = (k == 0) ? round % (m - 1) : (round + m - 1 - k) % (m - 1);
                const int p = min(a, b), q = max(a, b);
                double c = 1.0, s = 0.0;
                if (q < r && H[p + r * q] != 0.0) {
                    const double theta = (H[q + r * q] - H[p + r * p]) / (2.0 * H[p + r * q]);
                    const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                    c = 1.0 / sqrt(t * t + 1.0);
                    s = t * c;
                }
                cs[k] = c; sn[k] = s; pp[k] = p; qq[k] = q;
            }
            __syncthreads();
            for (int e = threadIdx.x; e < (m / 2) * r; e += blockDim.x) {
                const int k = e / r, col = e % r, p = pp[k], q = qq[k];
                if (q >= r) continue;
                const double hp = H[p + r * col], hq = H[q + r * col];
                H[p + r * col] = cs[k] * hp - sn[k] * hq;
                H[q + r * col] = sn[k] * hp + cs[k] * hq;
            }
            __syncthreads();
            for (int e = threadIdx.x; e < (m / 2) * r; e += blockDim.x) {
                const int k = e / r, row = e % r, p = pp[k], q = qq[k];
                if (q >= r) continue;
                const double hp = H[row + r * p], hq = H[row + r * q];
                H[row + r * p] = cs[k] * hp - sn[k] * hq;
                H[row + r * q] = sn[k] * hp + cs[k] * hq;
                const double wp = W[row + r * p], wq = W[row + r * q];
                W[row + r * p] = cs[k] * wp - sn[k] * wq;
                W[row + r * q] = sn[k] * wp + cs[k] * wq;
            }
            __syncthreads();
        }
    }
    if (threadIdx.x == 0) {  // ascending eigenvalues
        for (int j = 0; j < r; j++) ord[j] = j;
        for (int a = 1; a < r; a++)
            for (int b = a; b > 0 && H[ord[b] + r * ord[b]] < H[ord[b - 1] + r * ord[b - 1]]; b--) {
                const int t = ord[b]; ord[b] = ord[b - 1]; ord[b - 1] = t;
            }
    }
    __syncthreads();
    for (long e = threadIdx.x; e < n * r; e += blockDim.x) {
        const long i = e % n;
        const int j = (int)(e / n), c = ord[j];
        double s = 0.0;
        for (int a = 0; a < r; a++) s = fma(V[i + n * a], W[a + r * c], s);
        U[e] = (float)s;
    }
}

}  // namespace

size_t subspace_ws_doubles(long n, long r) { return 3 * (size_t)n * r + 8; }  // V, Y, W (r*r <= n*r), scalars

int top_eigvecs_subspace(const double *G, long n, long r, float *U, double *ws, int max_iters, cudaStream_t s) {
    if (r <= 0 || r > SI_RMAX || r > n) return CUD_ERR_UNSUPPORTED;
    double *V = ws, *Y = ws + n * r, *Wr = ws + 2 * n * r, *scal = ws + 3 * n * r;
    int *fail = reinterpret_cast<int *>(scal + 2);
    double *h = pinned_scalars();
    if (!h) return CUD_ERR_NO_MEMORY;
    const unsigned gb = (unsigned)std::min<long>((n * r + 255) / 256, 4L * kNumSMs);
    CUD_CHECK(cudaMemsetAsync(fail, 0, sizeof(int), s));
    k_si_init<<<gb, 256, 0, s>>>(V, n, (int)r);
    k_si_cholqr<<<1, 256, 0, s>>>(V, n, (int)r, fail);
    k_si_cholqr<<<1, 256, 0, s>>>(V, n, (int)r, fail);
    CUD_CHECK_LAUNCH("subspace init");
    int extra = -1;  // iterations still to run after the tolerance is met
    for (int it = 0; it < max_iters; it++) {
        k_si_apply<<<gb, 256, 0, s>>>(G, V, n, (int)r, Y);
        k_si_cholqr<<<1, 256, 0, s>>>(Y, n, (int)r, fail);
        k_si_cholqr<<<1, 256, 0, s>>>(Y, n, (int)r, fail);
        k_si_gap<<<1, 256, 0, s>>>(V, Y, n, (int)r, scal);
        CUD_CHECK_LAUNCH("subspace step");
        std::swap(V, Y);
        CUD_CHECK(cudaMemcpyAsync(h, scal, 3 * sizeof(double), cudaMemcpyDeviceToHost, s));
        CUD_CHECK(cudaStreamSynchronize(s));
        if (reinterpret_cast<int *>(h + 2)[0]) return CUD_ERR_NOT_CONVERGED;  // rank-deficient iterate
        if (extra < 0 && h[0] < 1e-13 * (double)r) extra = 2;
        if (extra >= 0 && extra-- == 0) {
            k_si_apply<<<gb, 256, 0, s>>>(G, V, n, (int)r, Y);
            k_si_ritz<<<1, 256, 0, s>>>(V, Y, n, (int)r, U, Wr);
            CUD_CHECK_LAUNCH("subspace ritz");
            return CUD_OK;
        }
    }
    return CUD_ERR_NOT_CONVERGED;
}

}  // namespace cud
