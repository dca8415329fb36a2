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

// V (n x r) = the given FP32 start block.
__global__ void k_si_init_from(const float *__restrict__ U0, double *V, long n, int r) {
    const long total = n * r;
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x)
        V[e] = (double)U0[e];
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
    // stop at a relative off-diagonal norm of 1e-13: rounding alone keeps it
    // near r * eps, so a test at eps itself would run every sweep
    for (int sweep = 0; sweep < 40; sweep++) {
        if (threadIdx.x == 0) {
            double off = 0.0, tot = 0.0;
            for (int e = 0; e < r * r; e++) {
                tot += H[e] * H[e];
                if (e % r != e / r) off += H[e] * H[e];
            }
            off_s = (off <= 1e-26 * tot) ? -1.0 : off;
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

// ---------------------------------------------------------------- fast path
// r <= SI_FR and the n x r iterate fits in one CTA's shared memory.  One
// step is two launches: the product G V split over k across CTAs
// (k_si_apply_split, partial products per k slice), then one CTA that sums
// the partials in slice order (deterministic), runs both CholQR passes on
// the iterate held in shared memory and measures the subspace gap against
// the previous iterate (k_si_orth).  The Rayleigh-Ritz step reuses the same
// shape (k_si_ritz_smem).
constexpr int SI_FR = 32;
constexpr int SI_OT = 512;    // threads of the one-CTA kernels
constexpr int SI_VCH = 64;    // rows of the previous iterate staged per chunk

__host__ __device__ inline long si_ld(long n) { return n | 1; }  // odd column stride in shared memory

// part[y] (n x r) = G[:, ks_y] V[ks_y, :] for k slice y (kchunk rows of V);
// one thread per row of G, V's rows staged 64 at a time.  V is given as the
// sum of nin slices of n x r (a previous product's partials), summed in
// slice order while staging.
__global__ void __launch_bounds__(128) k_si_apply_split(const double *__restrict__ G, const double *__restrict__ V,
                                                        int nin, long n, int r, long kchunk,
                                                        double *__restrict__ part) {
    __shared__ double sv[64][SI_FR];
    const long i = blockIdx.x * 128L + threadIdx.x;
    const long k0 = blockIdx.y * kchunk, k1 = min(n, k0 + kchunk);
    double acc[SI_FR];
#pragma unroll
    for (int c = 0; c < SI_FR; c++) acc[c] = 0.0;
    for (long kb = k0; kb < k1; kb += 64) {
        const int nk = (int)min(64L, k1 - kb);
        __syncthreads();
        for (int e = threadIdx.x; e < 64 * SI_FR; e += 128) {
            const int kk = e / SI_FR, c = e % SI_FR;
            double v = 0.0;
            if (kk < nk && c < r)
                for (int y = 0; y < nin; y++) v += V[(long)y * n * r + (kb + kk) + n * c];
            sv[kk][c] = v;
        }
        __syncthreads();
        if (i < n)
            for (int kk = 0; kk < nk; kk++) {
                const double g = G[i + n * (kb + kk)];
#pragma unroll
                for (int c = 0; c < SI_FR; c++) acc[c] = fma(g, sv[kk][c], acc[c]);
            }
    }
    if (i < n)
        for (int c = 0; c < r; c++) part[(long)blockIdx.y * n * r + i + n * c] = acc[c];
}

// ys (shared, column stride si_ld(n)) = sum over the nks slices of part.
__device__ void si_load_sum(const double *__restrict__ part, int nks, long n, int r, double *ys) {
    const long ld = si_ld(n), nr = n * r;
    for (long e = threadIdx.x; e < nr; e += blockDim.x) {
        double t = 0.0;
        for (int y = 0; y < nks; y++) t += part[(long)y * nr + e];
        ys[e % n + ld * (e / n)] = t;
    }
}

// out (r x r, shared) = A^T ys with A (n x r) in global memory, staged
// SI_VCH rows at a time; one entry (a, b) per thread (r * r <= blockDim).
__device__ void si_cross(const double *__restrict__ A, long n, int r, const double *ys, double *vs, double *out) {
    const long ld = si_ld(n);
    // entries e = tid and tid + blockDim (r * r <= 2 * blockDim)
    const int e0 = threadIdx.x, e1 = threadIdx.x + blockDim.x;
    const int a0 = e0 % r, b0 = e0 / r, a1 = e1 % r, b1 = e1 / r;
    double acc0 = 0.0, acc1 = 0.0;
    for (long i0 = 0; i0 < n; i0 += SI_VCH) {
        const int nn = (int)min((long)SI_VCH, n - i0);
        __syncthreads();
        for (int e = threadIdx.x; e < SI_VCH * r; e += blockDim.x) {
            const int ii = e % SI_VCH, c = e / SI_VCH;
            vs[ii + (SI_VCH + 1) * c] = (ii < nn) ? A[i0 + ii + n * c] : 0.0;
        }
        __syncthreads();
        if (b0 < r)
            for (int ii = 0; ii < nn; ii++) acc0 = fma(vs[ii + (SI_VCH + 1) * a0], ys[i0 + ii + ld * b0], acc0);
        if (b1 < r)
            for (int ii = 0; ii < nn; ii++) acc1 = fma(vs[ii + (SI_VCH + 1) * a1], ys[i0 + ii + ld * b1], acc1);
    }
    __syncthreads();
    if (b0 < r) out[a0 + r * b0] = acc0;
    if (b1 < r) out[a1 + r * b1] = acc1;
    __syncthreads();
}

// One CholQR pass on ys in shared memory: C = ys^T ys = L L^T, then
// ys <- ys L^-T.  C (r x r, lower) lives in shared memory; gp is scratch
// for the Gram's row-group partials (SI_GRP * 36 * 16 doubles).  The loops
// are rolled on purpose: this code runs once per launch, and fully unrolled
// r x r loops ran from the instruction cache's misses.  Returns false (every
// thread) when C is not numerically positive definite.
constexpr int SI_GRP = 8;  // row groups of the Gram
__device__ bool si_cholqr_smem(double *ys, long n, int r, double *C, double *gp, int *bad) {
    const long ld = si_ld(n);
    // Gram: 4 x 4 tiles of the lower triangle, each over one of SI_GRP row
    // groups, partials summed in group order
    const int nt = (r + 3) / 4, ntiles = nt * (nt + 1) / 2;
    const int w = threadIdx.x;
    if (w < ntiles * SI_GRP) {
        const int tile = w % ntiles, g = w / ntiles;
        int ta = 0, rem = tile;
        while (rem > ta) {
            rem -= ta + 1;
            ta++;
        }
        const int tb = rem;  // ta >= tb
        const long i0 = (long)g * n / SI_GRP, i1 = (long)(g + 1) * n / SI_GRP;
        double acc[4][4];
#pragma unroll
        for (int u = 0; u < 4; u++)
#pragma unroll
            for (int v = 0; v < 4; v++) acc[u][v] = 0.0;
        for (long i = i0; i < i1; i++) {
            double ya[4], yb[4];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                ya[u] = (4 * ta + u < r) ? ys[i + ld * (4 * ta + u)] : 0.0;
                yb[u] = (4 * tb + u < r) ? ys[i + ld * (4 * tb + u)] : 0.0;
            }
#pragma unroll
            for (int u = 0; u < 4; u++)
#pragma unroll
                for (int v = 0; v < 4; v++) acc[u][v] = fma(ya[u], yb[v], acc[u][v]);
        }
#pragma unroll
        for (int u = 0; u < 4; u++)
#pragma unroll
            for (int v = 0; v < 4; v++) gp[(g * ntiles + tile) * 16 + 4 * u + v] = acc[u][v];
    }
    if (threadIdx.x == 0) *bad = 0;
    __syncthreads();
    for (int e = threadIdx.x; e < ntiles * 16; e += blockDim.x) {
        const int tile = e / 16, u = (e / 4) % 4, v = e % 4;
        int ta = 0, rem = tile;
        while (rem > ta) {
            rem -= ta + 1;
            ta++;
        }
        const int a = 4 * ta + u, b = 4 * rem + v;
        double t = 0.0;
        for (int g = 0; g < SI_GRP; g++) t += gp[(g * ntiles + tile) * 16 + 4 * u + v];
        if (a < r && b < r && a >= b) C[a + r * b] = t;
    }
    __syncthreads();
    // right-looking Cholesky over the block, one column per step
    for (int j = 0; j < r; j++) {
        if (threadIdx.x == 0) {
            const double d = C[j + r * j];
            const bool ok = (d > 0.0) && isfinite(d);
            if (!ok) *bad = 1;
            C[j + r * j] = ok ? sqrt(d) : 1.0;
        }
        __syncthreads();
        const double inv = 1.0 / C[j + r * j];
        for (int i = j + 1 + threadIdx.x; i < r; i += blockDim.x) C[i + r * j] *= inv;
        __syncthreads();
        const int m = r - j - 1;
        for (int e = threadIdx.x; e < m * m; e += blockDim.x) {
            const int i = j + 1 + e % m, k = j + 1 + e / m;
            if (i >= k) C[i + r * k] = fma(-C[i + r * j], C[k + r * j], C[i + r * k]);
        }
        __syncthreads();
    }
    if (*bad) return false;
    // rows of ys: y_i <- L^-1 y_i, forward substitution in place
    for (long i = threadIdx.x; i < n; i += blockDim.x) {
        for (int a = 0; a < r; a++) {
            double t = ys[i + ld * a];
            for (int k = 0; k < a; k++) t = fma(-C[a + r * k], ys[i + ld * k], t);
            ys[i + ld * a] = t / C[a + r * a];
        }
    }
    __syncthreads();
    return true;
}

// Y = orth(sum of the partials) by `passes` CholQR passes; with Vold, also
// scal[0] = r - ||Vold^T Y||_F^2.  One CTA.
__global__ void __launch_bounds__(SI_OT) k_si_orth(const double *__restrict__ part, int nks, const double *Vold,
                                                   long n, int r, int passes, double *__restrict__ Y, double *scal,
                                                   int *fail) {
    extern __shared__ double sm_si[];
    __shared__ double C[SI_FR * SI_FR];
    __shared__ double red[SI_OT / 32];
    __shared__ int bad;
    const long ld = si_ld(n);
    double *ys = sm_si, *vs = sm_si + ld * r, *gp = vs + (SI_VCH + 1) * r;
    si_load_sum(part, nks, n, r, ys);
    __syncthreads();
    for (int pass = 0; pass < passes; pass++)
        if (!si_cholqr_smem(ys, n, r, C, gp, &bad)) {
            if (threadIdx.x == 0) *fail = 1;
            return;
        }
    if (Vold) {
        si_cross(Vold, n, r, ys, vs, C);
        double t = 0.0;
        for (int e = threadIdx.x; e < r * r; e += blockDim.x) t += C[e] * C[e];
        for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = t;
        __syncthreads();
        if (threadIdx.x == 0) {
            double g = 0.0;
            for (int w = 0; w < SI_OT / 32; w++) g += red[w];
            scal[0] = (double)r - g;
        }
    }
    for (long e = threadIdx.x; e < n * r; e += blockDim.x) Y[e] = ys[e % n + ld * (e / n)];
}

// Rayleigh-Ritz: H = V^T (G V) (G V = sum of the partials), Jacobi on H in
// shared memory, U[:, j] = V w_j for the eigenvalues in ascending order.
__global__ void __launch_bounds__(SI_OT) k_si_ritz_smem(const double *__restrict__ part, int nks,
                                                        const double *__restrict__ V, long n, int r, float *U) {
    extern __shared__ double sm_si[];
    __shared__ double H[SI_FR * SI_FR], W[SI_FR * SI_FR];
    __shared__ double cs[SI_FR / 2], sn[SI_FR / 2];
    __shared__ double cs_red[2 * SI_OT / 32];
    __shared__ int pp[SI_FR / 2], qq[SI_FR / 2], ord[SI_FR];
    __shared__ double off_s;
    const long ld = si_ld(n);
    double *ys = sm_si, *vs = sm_si + ld * r;
    si_load_sum(part, nks, n, r, ys);
    __syncthreads();
    si_cross(V, n, r, ys, vs, H);
    for (int e = threadIdx.x; e < r * r; e += blockDim.x) {
        const int a = e % r, b = e / r;
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
    // stop at a relative off-diagonal norm of 1e-13: rounding alone keeps it
    // near r * eps, so a test at eps itself would run every sweep
    for (int sweep = 0; sweep < 40; sweep++) {
        // off-diagonal and total squared norms, reduced over the block
        {
            double off = 0.0, tot = 0.0;
            for (int e = threadIdx.x; e < r * r; e += blockDim.x) {
                const double hv = H[e];
                tot += hv * hv;
                if (e % r != e / r) off += hv * hv;
            }
            for (int o = 16; o > 0; o >>= 1) {
                off += __shfl_xor_sync(0xffffffffu, off, o);
                tot += __shfl_xor_sync(0xffffffffu, tot, o);
            }
            if ((threadIdx.x & 31) == 0) {
                cs_red[threadIdx.x >> 5] = off;
                cs_red[SI_OT / 32 + (threadIdx.x >> 5)] = tot;
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                double o2 = 0.0, t2 = 0.0;
                for (int w = 0; w < SI_OT / 32; w++) {
                    o2 += cs_red[w];
                    t2 += cs_red[SI_OT / 32 + w];
                }
                off_s = (o2 <= 1e-26 * t2) ? -1.0 : o2;
            }
            __syncthreads();
        }
        if (off_s < 0) break;
        for (int round = 0; round < m - 1; round++) {
            if (threadIdx.x < m / 2) {
                const int k = threadIdx.x;
                int a = (k == 0) ? m - 1 : (round + k) % (m - 1);
                int b = (k == 0) ? round % (m - 1) : (round + m - 1 - k) % (m - 1);
                const int p = min(a, b), q = max(a, b);
                double c = 1.0, sv = 0.0;
                if (q < r && H[p + r * q] != 0.0) {
                    const double theta = (H[q + r * q] - H[p + r * p]) / (2.0 * H[p + r * q]);
                    const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                    c = 1.0 / sqrt(t * t + 1.0);
                    sv = t * c;
                }
                cs[k] = c; sn[k] = sv; pp[k] = p; qq[k] = q;
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
        double t = 0.0;
        for (int a = 0; a < r; a++) t = fma(V[i + n * a], W[a + r * c], t);
        U[e] = (float)t;
    }
}

size_t si_fast_smem(long n, long r) {
    return sizeof(double) * (size_t)(si_ld(n) * r + (SI_VCH + 1) * r + SI_GRP * 36 * 16);
}

}  // namespace

size_t subspace_ws_doubles(long n, long r) { return 3 * (size_t)n * r + 8; }  // V, Y, W (r*r <= n*r), scalars

// Fast path (r <= 32, iterate in one CTA's shared memory): ws holds V, Y
// (n x r each) and two sets of nks partial products, nks as many as
// ws_doubles allows (at most 8).  Each step forms G^2 V (two split
// products), then orthonormalises and measures the subspace change.
static int top_eigvecs_fast(const double *G, long n, long r, float *U, double *ws, size_t ws_doubles,
                            int max_iters, cudaStream_t s, const float *U0) {
    const long nr = n * r;
    const long room = ((long)ws_doubles - 2 * nr - 8) / (2 * nr);
    const int nks = (int)std::max(0L, std::min(8L, room));
    if (nks < 1) return CUD_ERR_UNSUPPORTED;
    const size_t smem = si_fast_smem(n, r);
    {
        static bool attr[64] = {false};
        int dev = 0;
        CUD_CHECK(cudaGetDevice(&dev));
        if (dev >= 0 && dev < 64 && !attr[dev]) {
            CUD_CHECK(cudaFuncSetAttribute(k_si_orth, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
            CUD_CHECK(cudaFuncSetAttribute(k_si_ritz_smem, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
            attr[dev] = true;
        }
    }
    double *V = ws, *Y = ws + nr, *part = ws + 2 * nr, *part2 = ws + (2 + nks) * nr,
           *scal = ws + (2 + 2 * nks) * nr;
    int *fail = reinterpret_cast<int *>(scal + 2);
    double *h = pinned_scalars();
    if (!h) return CUD_ERR_NO_MEMORY;
    const long kchunk = (n + nks - 1) / nks;
    const dim3 ga((unsigned)((n + 127) / 128), (unsigned)nks);
    const unsigned gi = (unsigned)std::min<long>((nr + 255) / 256, 4L * kNumSMs);
    CUD_CHECK(cudaMemsetAsync(fail, 0, sizeof(int), s));
    if (U0) k_si_init_from<<<gi, 256, 0, s>>>(U0, Y, n, (int)r);
    else k_si_init<<<gi, 256, 0, s>>>(Y, n, (int)r);
    k_si_orth<<<1, SI_OT, smem, s>>>(Y, 1, nullptr, n, (int)r, 2, V, scal, fail);
    CUD_CHECK_LAUNCH("subspace init");
    int extra = -1;  // iterations still to run after the tolerance is met
    for (int it = 0; it < max_iters; it++) {
        // two products per orthonormalisation (G^2 V): the columns' condition
        // grows by (lambda_1 / lambda_r)^2 per step, well inside CholQR2's range
        k_si_apply_split<<<ga, 128, 0, s>>>(G, V, 1, n, (int)r, kchunk, part2);
        k_si_apply_split<<<ga, 128, 0, s>>>(G, part2, nks, n, (int)r, kchunk, part);
        k_si_orth<<<1, SI_OT, smem, s>>>(part, nks, V, n, (int)r, 2, Y, scal, fail);
        CUD_CHECK_LAUNCH("subspace step");
        std::swap(V, Y);
        CUD_CHECK(cudaMemcpyAsync(h, scal, 3 * sizeof(double), cudaMemcpyDeviceToHost, s));
        CUD_CHECK(cudaStreamSynchronize(s));
        if (reinterpret_cast<int *>(h + 2)[0]) return CUD_ERR_NOT_CONVERGED;  // rank-deficient iterate
        if (extra < 0 && h[0] < 1e-13 * (double)r) extra = 1;
        if (extra >= 0 && extra-- == 0) {
            k_si_apply_split<<<ga, 128, 0, s>>>(G, V, 1, n, (int)r, kchunk, part);
            k_si_ritz_smem<<<1, SI_OT, smem, s>>>(part, nks, V, n, (int)r, U);
            CUD_CHECK_LAUNCH("subspace ritz");
            return CUD_OK;
        }
    }
    return CUD_ERR_NOT_CONVERGED;
}

static int subspace_run(const double *G, long n, long r, float *U, double *ws, size_t ws_doubles, int max_iters,
                        cudaStream_t s, const float *U0) {
    if (r <= SI_FR && n <= 4 * SI_OT && si_fast_smem(n, r) <= 200 * 1024) {
        const int st = top_eigvecs_fast(G, n, r, U, ws, ws_doubles, max_iters, s, U0);
        if (st != CUD_ERR_UNSUPPORTED) return st;
    }
    double *V = ws, *Y = ws + n * r, *Wr = ws + 2 * n * r, *scal = ws + 3 * n * r;
    int *fail = reinterpret_cast<int *>(scal + 2);
    double *h = pinned_scalars();
    if (!h) return CUD_ERR_NO_MEMORY;
    const unsigned gb = (unsigned)std::min<long>((n * r + 255) / 256, 4L * kNumSMs);
    CUD_CHECK(cudaMemsetAsync(fail, 0, sizeof(int), s));
    if (U0) k_si_init_from<<<gb, 256, 0, s>>>(U0, V, n, (int)r);
    else k_si_init<<<gb, 256, 0, s>>>(V, n, (int)r);
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

int top_eigvecs_subspace(const double *G, long n, long r, float *U, double *ws, size_t ws_doubles, int max_iters,
                         cudaStream_t s, const float *U0) {
    if (r <= 0 || r > SI_RMAX || r > n) return CUD_ERR_UNSUPPORTED;
    if (U0) {
        // U is written only on success: a failed warm start (a rank-
        // deficient start block) retries from the random block
        const int st = subspace_run(G, n, r, U, ws, ws_doubles, max_iters, s, U0);
        if (st != CUD_ERR_NOT_CONVERGED) return st;
    }
    return subspace_run(G, n, r, U, ws, ws_doubles, max_iters, s, nullptr);
}

}  // namespace cud
