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
#include <cooperative_groups.h>

#include <atomic>
#include <mutex>

#include "kernels.cuh"

namespace cud {

namespace cg = cooperative_groups;

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
// r <= 32 and n <= 2048.  One step is two launches of the product G V
// (k_si_apply_cols; the k range split in slices whose partial products are
// kept apart) and one launch of a cluster of CL_N CTAs that owns the n x r
// iterate by row blocks (k_si_orth_cl): the partial products summed in
// slice order, two CholQR passes, and the subspace gap against the previous
// iterate.  Each r x r Gram or cross product is the sum of the CTAs' row-
// block contributions, read through distributed shared memory and added in
// rank order; every CTA forms the same sum, so the small factorisations run
// redundantly in each CTA with identical results and need no broadcast.
// The Rayleigh-Ritz step (k_si_ritz_cl) has the same shape.  The r x r
// work -- the factorisation with its triangular inverse, the Jacobi sweeps
// -- keeps the matrix cells in registers across all threads and takes a
// fixed number of block barriers per step; the n x r work -- partial sums,
// row-block Grams, Y L^-T, V W -- is spread over the rows.
constexpr int SI_FR = 32;
constexpr int CL_N = 8;    // CTAs per cluster
constexpr int CL_T = 256;  // threads per CTA
constexpr int CL_RS = 33;  // row stride (doubles) of the row-major blocks in shared memory
constexpr size_t CL_SMEM_MAX = 200 * 1024;

// Dynamic shared memory of the cluster kernels (offsets in doubles): two
// row blocks (nl x 32, zero beyond column r), the two r x r buffers the
// peers read, the 4 x 4 tile partials, two 32 x 32 matrices.
struct ClLayout {
    int nl;  // rows per CTA
    size_t ya, yb, red, gp, C, T, total;
};
__host__ __device__ inline ClLayout cl_layout(long n) {
    ClLayout L;
    L.nl = (int)((n + CL_N - 1) / CL_N);
    const size_t blk = (size_t)L.nl * CL_RS;
    L.ya = 0;
    L.yb = L.ya + blk;
    L.red = L.yb + blk;
    L.gp = L.red + 2 * 32 * 32;
    L.C = L.gp + (size_t)CL_T * 16;
    L.T = L.C + 32 * CL_RS;
    L.total = L.T + 32 * CL_RS;
    return L;
}

// dst (nl x 32 row-major) = rows i0 .. i0 + nl - 1 of the sum of the nks
// column-major n x r slices of src, summed in slice order; columns r..31 zero.
__device__ void cl_load_rows(const double *__restrict__ src, int nks, long n, int r, long i0, int nl, double *dst) {
    const long nr = n * r;
#pragma unroll 4
    for (int e = threadIdx.x; e < nl * 32; e += CL_T) {
        const int a = e / nl, i = e - a * nl;
        double t = 0.0;
        if (a < r) {
            const double *p = src + (i0 + i) + n * a;
            for (int y = 0; y < nks; y++) t += p[(long)y * nr];
        }
        dst[i * CL_RS + a] = t;
    }
}

__device__ __forceinline__ void cl_tile(int tile, int nt, bool sym, int &ta, int &tb) {
    if (sym) {  // lower-triangle tiles in row order
        ta = 0;
        int rem = tile;
        while (rem > ta) {
            rem -= ta + 1;
            ta++;
        }
        tb = rem;
    } else {
        ta = tile / nt;
        tb = tile - ta * nt;
    }
}

// out (32 x 32 row-major) = this CTA's rows' part of A^T B (lower triangle
// when sym, with the diagonal tiles whole): 4 x 4 tiles, the rows split in
// groups whose partials are added in group order.  Ends on a block barrier.
__device__ void cl_cross(const double *A, const double *B, int nl, int r, bool sym, double *gp, double *out) {
    const int nt = (r + 3) / 4;
    const int ntiles = sym ? nt * (nt + 1) / 2 : nt * nt;
    const int ng = min(8, CL_T / ntiles);
    if ((int)threadIdx.x < ntiles * ng) {
        const int tile = threadIdx.x % ntiles, g = threadIdx.x / ntiles;
        int ta, tb;
        cl_tile(tile, nt, sym, ta, tb);
        const int i0 = g * nl / ng, i1 = (g + 1) * nl / ng;
        double acc[4][4];
#pragma unroll
        for (int u = 0; u < 4; u++)
#pragma unroll
            for (int v = 0; v < 4; v++) acc[u][v] = 0.0;
        for (int i = i0; i < i1; i++) {
            const double *ra = A + i * CL_RS + 4 * ta, *rb = B + i * CL_RS + 4 * tb;
            double xa[4], xb[4];
#pragma unroll
            for (int u = 0; u < 4; u++) {
                xa[u] = ra[u];
                xb[u] = rb[u];
            }
#pragma unroll
            for (int u = 0; u < 4; u++)
#pragma unroll
                for (int v = 0; v < 4; v++) acc[u][v] = fma(xa[u], xb[v], acc[u][v]);
        }
#pragma unroll
        for (int u = 0; u < 4; u++)
#pragma unroll
            for (int v = 0; v < 4; v++) gp[(g * ntiles + tile) * 16 + 4 * u + v] = acc[u][v];
    }
    __syncthreads();
    for (int e = threadIdx.x; e < ntiles * 16; e += CL_T) {
        const int tile = e >> 4, u = (e >> 2) & 3, v = e & 3;
        int ta, tb;
        cl_tile(tile, nt, sym, ta, tb);
        double t = 0.0;
        for (int g = 0; g < ng; g++) t += gp[(g * ntiles + tile) * 16 + 4 * u + v];
        out[(4 * ta + u) * 32 + 4 * tb + v] = t;
    }
    __syncthreads();
}

// dst (32 x CL_RS) = sum over the cluster's CTAs, in rank order, of their
// buffer `red` (entries a, b < r, a >= b when sym; zero elsewhere).  The
// caller has synchronised the cluster after the buffers were written.
__device__ void cl_sum(cg::cluster_group &cl, double *red, int r, bool sym, double *dst) {
    for (int e = threadIdx.x; e < 32 * 32; e += CL_T) {
        const int a = e >> 5, b = e & 31;
        double t = 0.0;
        if (a < r && b < r && (!sym || a >= b))
            for (int q = 0; q < CL_N; q++) t += cl.map_shared_rank(red, q)[e];
        dst[a * CL_RS + b] = t;
    }
    __syncthreads();
}

// CholQR's r x r factor work on all threads: C (lower triangle valid, in
// shared memory) = L D L^T with unit L by right-looking elimination, and in
// the same steps R = L^-1 (row k of R is final once step k-1 is done);
// then T = (L D^1/2)^-1 = D^-1/2 R (32 x 32, zero outside the lower r x r
// triangle).  Thread t keeps the cells (t / 32 + 8q, t % 32), q < 4, in
// registers; step k's pivot column and row k of R are published through
// shared memory, double-buffered, so a step takes one block barrier (a
// sequential loop through shared memory would wait on every load).
// Returns on every thread whether every pivot was positive and finite.
__device__ __forceinline__ bool cl_chol_inv(const double *C, double *T, int r, double *pub, double *dsh) {
    const int x = threadIdx.x & 31, w = threadIdx.x >> 5;
    double a[4], rr[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const int i = w + 8 * q;
        a[q] = (i < r && x < r && i >= x) ? C[i * CL_RS + x] : 0.0;
        rr[q] = (i == x) ? 1.0 : 0.0;
        if (x == 0 && i < r) pub[i] = a[q];  // column 0, buffer 0
    }
    __syncthreads();
    bool ok = true;
    for (int k = 0; k < r; k++) {
        const double *col = pub + 64 * (k & 1), *row = col + 32;
        double *ncol = pub + 64 * ((k + 1) & 1), *nrow = ncol + 32;
        const double akk = col[k];
        const bool good = akk > 0.0 && isfinite(akk);
        ok = ok && good;
        const double inv = good ? 1.0 / akk : 0.0;
        if (threadIdx.x == 0) dsh[k] = good ? akk : 1.0;
        const double cx = (x > k && x < r) ? col[x] * inv : 0.0;
        const double rx = (x < k) ? row[x] : 1.0;
#pragma unroll
        for (int q = 0; q < 4; q++) {
            const int i = w + 8 * q;
            if (i < r && x < r) {
                if (x > k && i >= x) a[q] = fma(-col[i], cx, a[q]);                // a_ix -= a_ik a_xk / a_kk
                else if (i > k && x <= k) rr[q] = fma(-col[i] * inv, rx, rr[q]);   // R_ix -= (a_ik / a_kk) R_kx
                if (x == k + 1 && i >= k + 1) ncol[i] = a[q];
                if (i == k + 1 && x <= k) nrow[x] = rr[q];
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const int i = w + 8 * q;
        T[i * CL_RS + x] = (i < r && x <= i) ? rr[q] / sqrt(dsh[i]) : 0.0;
    }
    __syncthreads();
    return ok;
}

// dst[i][a] = sum_k M[a][k] src[i][k] over the nl rows (M 32 x 32, row
// stride CL_RS; its zero rows beyond r keep dst's padding columns zero).
// Four threads per row, eight outputs each (a = s, s + 4, ...).
__device__ void cl_transform(const double *src, const double *M, int nl, double *dst) {
    for (int it = threadIdx.x; it < nl * 4; it += CL_T) {
        const int i = it >> 2, s = it & 3;
        const double *y = src + i * CL_RS;
        double acc[8];
#pragma unroll
        for (int j = 0; j < 8; j++) acc[j] = 0.0;
#pragma unroll 4
        for (int k = 0; k < 32; k++) {
            const double yk = y[k];
#pragma unroll
            for (int j = 0; j < 8; j++) acc[j] = fma(M[(s + 4 * j) * CL_RS + k], yk, acc[j]);
        }
#pragma unroll
        for (int j = 0; j < 8; j++) dst[i * CL_RS + s + 4 * j] = acc[j];
    }
}

// Cyclic Jacobi on all threads (round-robin pairs, m/2 disjoint rotations
// per round) on the symmetric H (r x r in Hs, row stride CL_RS), the
// rotations accumulated in W.  Thread t keeps the cells (t / 32 + 8q,
// t % 32), q < 4, of H and W in registers: a round's column rotations pair
// lanes of one warp (shuffles), its row rotations read the partner row of
// H J through shared memory (Mb).  Stops at a relative off-diagonal norm of
// 1e-13 (rounding alone keeps it near r * eps, so a test at eps itself
// would run every sweep).  On return Hs holds the rotated H, Ws = W (row
// stride CL_RS) and ord the eigenvalue order, ascending.  Ends on a block
// barrier.
__device__ __forceinline__ void cl_jacobi(double *Hs, double *Mb, double *Ws, int r, double *cval, double *sval,
                                          int *pt, int *role, int *ord, double *wred) {
    const int x = threadIdx.x & 31, w = threadIdx.x >> 5;
    double h[4], wv[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
        const int i = w + 8 * q;
        h[q] = (i < r && x < r) ? 0.5 * (Hs[i * CL_RS + x] + Hs[x * CL_RS + i]) : 0.0;
        wv[q] = (i == x && i < r) ? 1.0 : 0.0;
    }
    if (threadIdx.x < 32) {  // unpaired indices rotate by the identity
        pt[x] = x;
        role[x] = 0;
        cval[x] = 1.0;
        sval[x] = 0.0;
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 4; q++) Hs[(w + 8 * q) * CL_RS + x] = h[q];
    __syncthreads();
    const int m = (r + 1) & ~1;
    for (int sweep = 0; sweep < 40; sweep++) {
        double off = 0.0, tot = 0.0;
#pragma unroll
        for (int q = 0; q < 4; q++) {
            tot = fma(h[q], h[q], tot);
            if (w + 8 * q != x) off = fma(h[q], h[q], off);
        }
        for (int o = 16; o > 0; o >>= 1) {
            off += __shfl_xor_sync(0xffffffffu, off, o);
            tot += __shfl_xor_sync(0xffffffffu, tot, o);
        }
        if (x == 0) {
            wred[w] = off;
            wred[8 + w] = tot;
        }
        __syncthreads();
        double o2 = 0.0, t2 = 0.0;
        for (int v = 0; v < CL_T / 32; v++) {  // same order on every thread
            o2 += wred[v];
            t2 += wred[8 + v];
        }
        __syncthreads();  // wred is rewritten next sweep
        if (o2 <= 1e-26 * t2) break;
        for (int round = 0; round < m - 1; round++) {
            if ((int)threadIdx.x < m / 2) {
                const int k = threadIdx.x;
                const int a = (k == 0) ? m - 1 : (round + k) % (m - 1);
                const int b = (k == 0) ? round % (m - 1) : (round + m - 1 - k) % (m - 1);
                const int p = min(a, b), q = max(a, b);
                double c = 1.0, sv = 0.0;
                if (q < r) {
                    const double hpq = Hs[p * CL_RS + q];
                    if (hpq != 0.0) {
                        const double theta = (Hs[q * CL_RS + q] - Hs[p * CL_RS + p]) / (2.0 * hpq);
                        const double t = (theta >= 0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
                        c = 1.0 / sqrt(t * t + 1.0);
                        sv = t * c;
                    }
                    pt[p] = q;
                    pt[q] = p;
                    role[q] = 1;
                } else {
                    pt[p] = p;
                    pt[q] = q;
                    role[q] = 0;
                }
                role[p] = 0;
                cval[p] = c;
                cval[q] = c;
                sval[p] = sv;
                sval[q] = sv;
            }
            __syncthreads();
            {  // H J and W J: columns x and pt[x] live in lanes of the same warp
                const int px = pt[x], rx = role[x];
                const double cx = cval[x], sx = rx ? sval[x] : -sval[x];
#pragma unroll
                for (int q = 0; q < 4; q++) {
                    const double ho = __shfl_sync(0xffffffffu, h[q], px);
                    const double wo = __shfl_sync(0xffffffffu, wv[q], px);
                    h[q] = fma(sx, ho, cx * h[q]);
                    wv[q] = fma(sx, wo, cx * wv[q]);
                    Mb[(w + 8 * q) * CL_RS + x] = h[q];
                }
            }
            __syncthreads();
#pragma unroll
            for (int q = 0; q < 4; q++) {  // J^T (H J): row i against its partner row
                const int i = w + 8 * q;
                const int pi = pt[i];
                const double ci = cval[i], si = role[i] ? sval[i] : -sval[i];
                h[q] = fma(si, Mb[pi * CL_RS + x], ci * h[q]);
                Hs[i * CL_RS + x] = h[q];
            }
            __syncthreads();
        }
    }
#pragma unroll
    for (int q = 0; q < 4; q++) Ws[(w + 8 * q) * CL_RS + x] = wv[q];
    if (threadIdx.x < 32) {  // ascending order by rank (ties by index); a
                             // non-permutation (NaN eigenvalues) falls back
                             // to the identity order
        int rk = 0;
        if (x < r) {
            const double d = Hs[x * CL_RS + x];
            for (int b = 0; b < r; b++) {
                const double e = Hs[b * CL_RS + b];
                rk += (e < d) || (e == d && b < x);
            }
        }
        const unsigned bits = __reduce_or_sync(0xffffffffu, x < r ? 1u << rk : 0u);
        const unsigned want = (r == 32) ? 0xffffffffu : ((1u << r) - 1u);
        if (x < r) ord[bits == want ? rk : x] = x;
    }
    __syncthreads();
}

// Y (n x r) = orth(sum of the nks partial slices) by two CholQR passes;
// with Vold, also scal[0] = r - ||Vold^T Y||_F^2.  *fail = 1 (and Y not
// written) when a Gram is not numerically positive definite.
//
// With st (a step of the iteration), the convergence test runs here, so
// the host can queue several steps and read the state once: st[0] done
// (later launches return at once), st[1] the steps still to run after the
// gap first fell below the tolerance, plus one (0: not yet), st[2] steps
// taken, st[3] the step whose iterate is final.  The state is read on entry
// by every CTA and written by CTA 0 only after the cluster's last barrier,
// so all CTAs of a launch see the same value.
__global__ void __cluster_dims__(CL_N, 1, 1) __launch_bounds__(CL_T)
    k_si_orth_cl(const double *__restrict__ part, int nks, const double *__restrict__ Vold, long n, int r,
                 double *__restrict__ Y, double *scal, int *fail, int *st) {
    if (st && st[0]) return;
    cg::cluster_group cl = cg::this_cluster();
    extern __shared__ double smc[];
    __shared__ double pub[128], dsh[32], wred[CL_T / 32];
    const ClLayout L = cl_layout(n);
    const int rank = (int)cl.block_rank();
    const long i0 = (long)rank * L.nl;
    const int nl = (int)max(0L, min((long)L.nl, n - i0));
    double *ya = smc + L.ya, *yb = smc + L.yb, *red = smc + L.red, *gp = smc + L.gp, *C = smc + L.C,
           *T = smc + L.T;
    cl_load_rows(part, nks, n, r, i0, nl, ya);
    __syncthreads();
    for (int pass = 0; pass < 2; pass++) {
        double *src = pass ? yb : ya, *dst = pass ? ya : yb, *rb = red + pass * 32 * 32;
        cl_cross(src, src, nl, r, true, gp, rb);
        cl.sync();
        cl_sum(cl, rb, r, true, C);
        if (!cl_chol_inv(C, T, r, pub, dsh)) {  // the same verdict in every CTA
            cl.sync();                              // peers may still read this CTA's buffers
            if (rank == 0 && threadIdx.x == 0) {
                *fail = 1;
                if (st) st[0] = 1;
            }
            return;
        }
        cl_transform(src, T, nl, dst);
        __syncthreads();
    }
    if (Vold) {
        cl_load_rows(Vold, 1, n, r, i0, nl, yb);
        __syncthreads();
        cl_cross(yb, ya, nl, r, false, gp, red);  // buffer 0: its readers all passed the last cluster barrier
        cl.sync();
        if (rank == 0) {
            cl_sum(cl, red, r, false, C);
            double t = 0.0;
            for (int e = threadIdx.x; e < 32 * 32; e += CL_T) {
                const double v = C[(e >> 5) * CL_RS + (e & 31)];
                t = fma(v, v, t);
            }
            for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
            if ((threadIdx.x & 31) == 0) wred[threadIdx.x >> 5] = t;
            __syncthreads();
            if (threadIdx.x == 0) {
                double g = 0.0;
                for (int w = 0; w < CL_T / 32; w++) g += wred[w];
                scal[0] = (double)r - g;
            }
        }
    }
    for (int e = threadIdx.x; e < nl * r; e += CL_T) {
        const int a = e / nl, i = e - a * nl;
        Y[(i0 + i) + n * a] = ya[i * CL_RS + a];
    }
    cl.sync();  // keep this CTA's buffers alive until every peer has read them
    if (st && rank == 0 && threadIdx.x == 0) {
        // one more step after the gap first falls below the tolerance
        const int step = st[2] + 1;
        int extra = st[1] - 1;
        if (extra < 0 && scal[0] < 1e-13 * (double)r) extra = 1;
        if (extra >= 0 && extra-- == 0) {
            st[0] = 1;
            st[3] = step;
        }
        st[1] = extra + 1;
        st[2] = step;
    }
}

// Rayleigh-Ritz: H = V^T (G V) (G V = the sum of the partial slices),
// Jacobi on H, U[:, j] = V w_ord[j] with the eigenvalues ascending.
__global__ void __cluster_dims__(CL_N, 1, 1) __launch_bounds__(CL_T)
    k_si_ritz_cl(const double *__restrict__ part, int nks, const double *__restrict__ V, long n, int r,
                 float *__restrict__ U) {
    cg::cluster_group cl = cg::this_cluster();
    extern __shared__ double smc[];
    __shared__ double cval[32], sval[32], wred[16];
    __shared__ int pt[32], role[32], ord[32];
    const ClLayout L = cl_layout(n);
    const int rank = (int)cl.block_rank();
    const long i0 = (long)rank * L.nl;
    const int nl = (int)max(0L, min((long)L.nl, n - i0));
    double *ya = smc + L.ya, *yb = smc + L.yb, *red = smc + L.red, *gp = smc + L.gp, *H = smc + L.C,
           *W = smc + L.T;
    cl_load_rows(part, nks, n, r, i0, nl, ya);
    cl_load_rows(V, 1, n, r, i0, nl, yb);
    __syncthreads();
    cl_cross(yb, ya, nl, r, false, gp, red);
    cl.sync();
    cl_sum(cl, red, r, false, H);
    cl_jacobi(H, gp, W, r, cval, sval, pt, role, ord, wred);
    double *M = gp + 32 * CL_RS;  // M[j][a] = W[a][ord[j]]
    for (int e = threadIdx.x; e < 32 * 32; e += CL_T) {
        const int j = e >> 5, a = e & 31;
        M[j * CL_RS + a] = (j < r && a < r) ? W[a * CL_RS + ord[j]] : 0.0;
    }
    __syncthreads();
    cl_transform(yb, M, nl, ya);
    __syncthreads();
    for (int e = threadIdx.x; e < nl * r; e += CL_T) {
        const int j = e / nl, i = e - j * nl;
        U[(i0 + i) + n * j] = (float)ya[i * CL_RS + j];
    }
    cl.sync();  // keep this CTA's buffers alive until every peer has read them
}

// part[y] (n x r) = G[:, slice y] V[slice y, :] for the k slices of kchunk
// rows (V given as the sum of nin n x r slices, summed in slice order).  A
// CTA takes 32 rows of G (one per lane) and one k slice; warp w forms
// columns 4w .. 4w+3, so each output has one owner and no cross-warp sum.
constexpr int AP_KB = 64;  // rows of V staged per pass
__global__ void __launch_bounds__(256) k_si_apply_cols(const double *__restrict__ G, const double *__restrict__ V,
                                                       int nin, long n, int r, long kchunk,
                                                       double *__restrict__ part, const int *st) {
    if (st && st[0]) return;  // the iteration has converged (k_si_orth_cl)
    __shared__ double sv[AP_KB][SI_FR + 1];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const long i = blockIdx.x * 32L + lane;
    const long k0 = blockIdx.y * kchunk, k1 = min(n, k0 + kchunk);
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (long kb = k0; kb < k1; kb += AP_KB) {
        const int nk = (int)min((long)AP_KB, k1 - kb);
        __syncthreads();
        for (int e = threadIdx.x; e < AP_KB * SI_FR; e += 256) {
            const int kk = e % AP_KB, c = e / AP_KB;
            double v = 0.0;
            if (kk < nk && c < r)
                for (int y = 0; y < nin; y++) v += V[(long)y * n * r + (kb + kk) + n * c];
            sv[kk][c] = v;
        }
        __syncthreads();
        if (i < n && 4 * w < r) {
            const double *g = G + i + n * kb;
#pragma unroll 16
            for (int kk = 0; kk < nk; kk++) {
                const double gv = g[n * kk];
#pragma unroll
                for (int u = 0; u < 4; u++) acc[u] = fma(gv, sv[kk][4 * w + u], acc[u]);
            }
        }
    }
    if (i < n)
#pragma unroll
        for (int u = 0; u < 4; u++) {
            const int c = 4 * w + u;
            if (c < r) part[(long)blockIdx.y * n * r + i + n * c] = acc[u];
        }
}

// After each batch of steps in the loop graph: whether its WHILE node runs
// another batch -- the host loop's rule (stop once the iteration has
// converged or failed, or max_iters steps have run; every step of a batch
// that has not converged runs, so st[2] counts the steps queued).
__global__ void k_si_loop_cond(cudaGraphConditionalHandle h, const int *fail, const int *st, int max_iters) {
    if (threadIdx.x != 0) return;
    const bool more = *fail == 0 && st[0] == 0 && st[2] < max_iters;
    cudaGraphSetConditional(h, more ? 1u : 0u);
}

constexpr int SI_BATCH = 4;  // steps queued between two reads of the state

// One batch of SI_BATCH fast-path steps from V = buffer 0 (ws), as the host
// loop queues it; SI_BATCH is even, so the batch ends with V in buffer 0
// again and every batch is the same launch sequence.
struct SiSteps {
    const double *G;
    long n;
    int r, nks;
    long kchunk;
    dim3 ga;
    size_t smem;
    double *ws, *part, *part2, *scal;
    int *fail, *st;
    void enqueue(int steps, cudaStream_t s) const {
        const long nr = n * (long)r;
        double *V = ws, *Y = ws + nr;
        for (int b = 0; b < steps; b++) {
            // two products per orthonormalisation (G^2 V): the columns' condition
            // grows by (lambda_1 / lambda_r)^2 per step, well inside CholQR2's range
            k_si_apply_cols<<<ga, 256, 0, s>>>(G, V, 1, n, r, kchunk, part2, st);
            k_si_apply_cols<<<ga, 256, 0, s>>>(G, part2, nks, n, r, kchunk, part, st);
            k_si_orth_cl<<<CL_N, CL_T, smem, s>>>(part, nks, V, n, r, Y, scal, fail, st);
            std::swap(V, Y);
        }
    }
};

// Loop graphs of the fast path, one per (device, G, n, r, ws, nks,
// max_iters): a WHILE node whose body is one batch and k_si_loop_cond, so a
// call reads the state once instead of once per batch.  The key holds the
// exact pointers the captured launches use.  A few entries (the Tucker
// drivers call with one Gram and one workspace per plan), never replaced,
// since another thread may be launching one: once all are taken, new keys
// keep the host loop.
struct SiGraph {
    int dev = -1;
    const double *G = nullptr, *ws = nullptr;
    long n = 0;
    int r = 0, nks = 0, max_iters = 0;
    cudaGraphExec_t ex = nullptr;
};
constexpr int SI_GRAPHS = 8;
std::mutex g_si_mu;
SiGraph g_si[SI_GRAPHS];
int g_si_used = 0;
bool g_si_refused[64] = {};  // per device: the driver refused a loop graph once; keep the host loop

// Capture the loop graph on a private stream (capturing records the
// launches without running them); null when the driver refuses any step,
// and the caller keeps the host loop.
cudaGraphExec_t si_build_loop(const SiSteps &k, int max_iters) {
    cudaStream_t cs = nullptr;
    if (cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking) != cudaSuccess) {
        (void)cudaGetLastError();
        return nullptr;
    }
    cudaGraph_t g = nullptr;
    cudaGraphExec_t ex = nullptr;
    bool ok = cudaGraphCreate(&g, 0) == cudaSuccess;
    cudaGraphConditionalHandle h = 0;
    cudaGraph_t body = nullptr;
    if (ok) ok = cudaGraphConditionalHandleCreate(&h, g, 1, cudaGraphCondAssignDefault) == cudaSuccess;
    if (ok) {
        cudaGraphNodeParams np = {};
        np.type = cudaGraphNodeTypeConditional;
        np.conditional.handle = h;
        np.conditional.type = cudaGraphCondTypeWhile;
        np.conditional.size = 1;
        cudaGraphNode_t node;
        ok = cudaGraphAddNode(&node, g, nullptr, 0, &np) == cudaSuccess;
        if (ok) body = np.conditional.phGraph_out[0];
    }
    if (ok) ok = cudaStreamBeginCaptureToGraph(cs, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal) ==
                 cudaSuccess;
    if (ok) {
        k.enqueue(SI_BATCH, cs);
        k_si_loop_cond<<<1, 32, 0, cs>>>(h, k.fail, k.st, max_iters);
        const bool launched = cudaGetLastError() == cudaSuccess;
        cudaGraph_t captured = nullptr;
        ok = cudaStreamEndCapture(cs, &captured) == cudaSuccess && launched;
    }
    if (ok) ok = cudaGraphInstantiate(&ex, g, 0) == cudaSuccess;
    (void)cudaGetLastError();
    if (!ok && ex) {
        cudaGraphExecDestroy(ex);
        ex = nullptr;
    }
    if (g) cudaGraphDestroy(g);  // the executable graph keeps what it needs
    cudaStreamDestroy(cs);
    return ex;
}

cudaGraphExec_t si_loop_graph(int dev, const SiSteps &k, int max_iters) {
    std::lock_guard<std::mutex> lk(g_si_mu);
    for (const SiGraph &e : g_si)
        if (e.ex && e.dev == dev && e.G == k.G && e.ws == k.ws && e.n == k.n && e.r == k.r && e.nks == k.nks &&
            e.max_iters == max_iters)
            return e.ex;
    if (g_si_used == SI_GRAPHS || g_si_refused[dev]) return nullptr;
    cudaGraphExec_t ex = si_build_loop(k, max_iters);
    if (!ex) {
        g_si_refused[dev] = true;
        return nullptr;
    }
    SiGraph &slot = g_si[g_si_used++];
    slot.dev = dev; slot.G = k.G; slot.ws = k.ws; slot.n = k.n; slot.r = k.r; slot.nks = k.nks;
    slot.max_iters = max_iters;
    slot.ex = ex;
    return ex;
}

}  // namespace

size_t subspace_ws_doubles(long n, long r) { return 3 * (size_t)n * r + 8; }  // V, Y, W (r*r <= n*r), scalars

// Fast path (r <= 32, n <= 2048): ws holds V, Y (n x r each) and two sets
// of nks partial products, nks as many as ws_doubles allows (at most 8).
// Each step forms G^2 V (two split products), then orthonormalises and
// measures the subspace change.
static int top_eigvecs_fast(const double *G, long n, long r, float *U, double *ws, size_t ws_doubles,
                            int max_iters, cudaStream_t s, const float *U0) {
    const long nr = n * r;
    const long room = ((long)ws_doubles - 2 * nr - 8) / (2 * nr);
    const int nks = (int)std::max(0L, std::min(8L, room));
    if (nks < 1) return CUD_ERR_UNSUPPORTED;
    const size_t smem = cl_layout(n).total * sizeof(double);
    int dev = 0;
    CUD_CHECK(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return CUD_ERR_UNSUPPORTED;
    {
        // once per device: the shared-memory opt-in, and whether a cluster
        // of this size can be resident at all
        static std::atomic<int> ready[64];  // 0 unknown, 1 usable, 2 not; zero-initialised
        if (!ready[dev]) {
            CUD_CHECK(cudaFuncSetAttribute(k_si_orth_cl, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)CL_SMEM_MAX));
            CUD_CHECK(cudaFuncSetAttribute(k_si_ritz_cl, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)CL_SMEM_MAX));
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = dim3(CL_N);
            cfg.blockDim = dim3(CL_T);
            cfg.dynamicSmemBytes = CL_SMEM_MAX;
            int nc = 0;
            const cudaError_t e1 = cudaOccupancyMaxActiveClusters(&nc, k_si_orth_cl, &cfg);
            int nc2 = 0;
            const cudaError_t e2 = cudaOccupancyMaxActiveClusters(&nc2, k_si_ritz_cl, &cfg);
            ready[dev] = (e1 == cudaSuccess && e2 == cudaSuccess && nc > 0 && nc2 > 0) ? 1 : 2;
            (void)cudaGetLastError();
        }
        if (ready[dev] != 1) return CUD_ERR_UNSUPPORTED;
    }
    double *V = ws, *Y = ws + nr, *part = ws + 2 * nr, *part2 = ws + (2 + nks) * nr,
           *scal = ws + (2 + 2 * nks) * nr;
    int *fail = reinterpret_cast<int *>(scal + 2);
    int *st = reinterpret_cast<int *>(scal + 3);  // 4 ints: done, extra + 1, steps, final step
    double *h = pinned_scalars();
    if (!h) return CUD_ERR_NO_MEMORY;
    const long kchunk = (n + nks - 1) / nks;
    const dim3 ga((unsigned)((n + 31) / 32), (unsigned)nks);
    const unsigned gi = (unsigned)std::min<long>((nr + 255) / 256, 4L * kNumSMs);
    CUD_CHECK(cudaMemsetAsync(fail, 0, 3 * sizeof(double), s));  // fail and the state
    if (U0) k_si_init_from<<<gi, 256, 0, s>>>(U0, Y, n, (int)r);
    else k_si_init<<<gi, 256, 0, s>>>(Y, n, (int)r);
    k_si_orth_cl<<<CL_N, CL_T, smem, s>>>(Y, 1, nullptr, n, (int)r, V, scal, fail, nullptr);
    CUD_CHECK_LAUNCH("subspace init");
    // Steps are queued SI_BATCH at a time and the launches after convergence
    // return at once.  Step j (from 1) writes buffer j % 2 (buffer 0 = the
    // initial V).  When max_iters is a whole number of batches, the batches
    // run in the loop graph and the state is read once; otherwise the host
    // reads it after every batch.
    const SiSteps k{G, n, (int)r, nks, kchunk, ga, smem, ws, part, part2, scal, fail, st};
    const cudaGraphExec_t loop = (max_iters % SI_BATCH == 0) ? si_loop_graph(dev, k, max_iters) : nullptr;
    for (int queued = 0; queued < max_iters;) {
        if (loop) {
            CUD_CHECK(cudaGraphLaunch(loop, s));
            queued = max_iters;
        } else {
            const int nb = std::min(SI_BATCH, max_iters - queued);
            k.enqueue(nb, s);
            CUD_CHECK_LAUNCH("subspace steps");
            queued += nb;
        }
        CUD_CHECK(cudaMemcpyAsync(h, scal + 2, 3 * sizeof(double), cudaMemcpyDeviceToHost, s));
        CUD_CHECK(cudaStreamSynchronize(s));
        const int *hs = reinterpret_cast<const int *>(h);  // fail, pad, done, extra + 1, steps, final
        if (hs[0]) return CUD_ERR_NOT_CONVERGED;          // rank-deficient iterate
        if (hs[2]) {
            const double *Vf = ws + ((hs[5] % 2) ? nr : 0);
            k_si_apply_cols<<<ga, 256, 0, s>>>(G, Vf, 1, n, (int)r, kchunk, part, nullptr);
            k_si_ritz_cl<<<CL_N, CL_T, smem, s>>>(part, nks, Vf, n, (int)r, U);
            CUD_CHECK_LAUNCH("subspace ritz");
            return CUD_OK;
        }
    }
    return CUD_ERR_NOT_CONVERGED;
}

static int subspace_run(const double *G, long n, long r, float *U, double *ws, size_t ws_doubles, int max_iters,
                        cudaStream_t s, const float *U0) {
    if (r <= SI_FR && n <= 2048 && cl_layout(n).total * sizeof(double) <= CL_SMEM_MAX) {
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

extern "C" int cud_syev_top(const double *G, long n, long r, float *U, const float *U0, int max_iters,
                            void *stream) {
    if (n <= 0 || r <= 0 || r > n || !G || !U || max_iters <= 0) return cud::set_status(CUD_ERR_INVALID_ARGUMENT);
    // room for the fast path's eight k slices of partial products
    const size_t wsd = std::max(cud::subspace_ws_doubles(n, r), (size_t)18 * (size_t)n * (size_t)r + 8);
    int st;
    double *ws = static_cast<double *>(cud::scratch(cud::kSlotEig, wsd * sizeof(double), &st));
    if (!ws) return cud::set_status(st);
    return cud::set_status(cud::top_eigvecs_subspace(G, n, r, U, ws, wsd, max_iters, cud::as_stream(stream), U0));
}
