// Learned warm start for CP-ALS: the device side.
//
// A small MLP maps random sketches of a tensor's three mode unfoldings to
// initial CP factors.  This file holds everything of it that is not a GEMM
// (the GEMMs -- sketches, forward and backward layers -- run on the tcgen05
// kernel in gemm_tc.cu):
//   * a seeded generator of the smooth-factor workload: 3rd-order tensors
//     whose factor columns are sums of three sinusoids, plus relative
//     Gaussian noise (random numbers from a counter-based hash, so any tensor
//     of any batch can be regenerated from (seed, tensor id));
//   * the mode-n unfolding of each tensor in BF16, rows K-contiguous, the
//     sketch GEMM's A operand;
//   * feature packing (sketches scaled by 1/||X||, plus the transpose the
//     weight-gradient GEMM reads);
//   * target canonicalisation of CP factors (unit columns, fixed signs,
//     columns ordered by weight);
//   * the MSE loss and its gradient, bias gradients, and Adam on FP32 master
//     weights with BF16 working copies (and their transposes).
// The reference has no learned component; the ALS it warm-starts is
// src/cp_als.cu.
#include <cuda_bf16.h>

#include "kernels.cuh"

namespace cud {

namespace {

// SplitMix64 finaliser (Steele, Lea and Flood, "Fast splittable pseudorandom
// number generators", OOPSLA 2014): a bijective 64-bit mix.
__host__ __device__ __forceinline__ unsigned long long mix64(unsigned long long z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

// Counter-based stream: the k-th 64-bit value of stream (seed, a, b).
__host__ __device__ __forceinline__ unsigned long long hash3(unsigned long long seed, unsigned long long a,
                                                             unsigned long long b) {
    return mix64(seed ^ mix64(a * 0x9e3779b97f4a7c15ULL ^ mix64(b + 0x632be59bd9b4e019ULL)));
}

__device__ __forceinline__ double u01(unsigned long long h) { return (double)(h >> 11) * (1.0 / 9007199254740992.0); }

// Standard normal from two counter values (Box-Muller, cosine branch).
__device__ __forceinline__ double normal2(unsigned long long h1, unsigned long long h2) {
    const double u1 = 1.0 - u01(h1);  // (0, 1]
    const double u2 = u01(h2);
    return sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
}

constexpr double kTwoPi = 6.283185307179586;

}  // namespace

// ---------------------------------------------------------------- generator

// Factors of tensor t (global id = id0 + t): mode m, column r, entry i of an
// I x R column-major matrix at F + t*(3*I*R) + m*I*R:
//   f(i) = sum_{q<3} a_q sin(2 pi w_q i / I + p_q),
//   w_q ~ U[0.5, 4], p_q ~ U[0, 2 pi), a_q ~ N(0, 1)   (per column).
// Also ||X_clean||^2 = sum_{r,s} prod_m (U_m^T U_m)[r, s] into norm2[t].
__global__ void __launch_bounds__(256) k_ws_factors(float *F, double *norm2, int I, int R, long id0,
                                                    unsigned long long seed) {
    extern __shared__ float fs[];  // 3 * I * R
    const long t = blockIdx.x;
    const long gid = id0 + t;
    const int per = I * R;
    for (int e = threadIdx.x; e < 3 * per; e += blockDim.x) {
        const int m = e / per, rem = e % per, r = rem / I, i = rem % I;
        const unsigned long long col = (unsigned long long)(m * R + r);
        double v = 0.0;
        for (int q = 0; q < 3; q++) {
            const unsigned long long b = col * 8 + q * 2;
            const double w = 0.5 + 3.5 * u01(hash3(seed, gid, b * 4 + 0));
            const double p = kTwoPi * u01(hash3(seed, gid, b * 4 + 1));
            const double amp = normal2(hash3(seed, gid, b * 4 + 2), hash3(seed, gid, b * 4 + 3));
            v += amp * sin(kTwoPi * w * (double)i / (double)I + p);
        }
        fs[e] = (float)v;
        F[t * 3 * per + e] = (float)v;
    }
    __syncthreads();
    // ||X_clean||^2 from the Grams (FP64), one thread per (r, s) pair
    __shared__ double red[256];
    double acc = 0.0;
    for (int rs = threadIdx.x; rs < R * R; rs += blockDim.x) {
        const int r = rs % R, s = rs / R;
        double prod = 1.0;
        for (int m = 0; m < 3; m++) {
            const float *U = fs + m * per;
            double g = 0.0;
            for (int i = 0; i < I; i++) g += (double)U[i + I * r] * (double)U[i + I * s];
            prod *= g;
        }
        acc += prod;
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) norm2[t] = red[0];
}

// X[t] (I^3, column-major) = [[U_0, U_1, U_2]] + noise * ||X_clean|| / sqrt(I^3) * N(0, 1).
__global__ void __launch_bounds__(256) k_ws_tensor(const float *F, const double *norm2, float *X, int I, int R,
                                                   long id0, unsigned long long seed, double noise) {
    __shared__ float fs[3 * 128 * 16];
    const long t = blockIdx.y;
    const long gid = id0 + t;
    const int per = I * R;
    for (int e = threadIdx.x; e < 3 * per; e += blockDim.x) fs[e] = F[t * 3 * per + e];
    __syncthreads();
    const long n = (long)I * I * I;
    const double sigma = noise * sqrt(norm2[t] / (double)n);
    float *Xt = X + t * n;
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) {
        const int i = (int)(e % I), j = (int)((e / I) % I), k = (int)(e / ((long)I * I));
        float v = 0.f;
        for (int r = 0; r < R; r++) v = fmaf(fs[i + I * r] * fs[per + j + I * r], fs[2 * per + k + I * r], v);
        const unsigned long long c = (unsigned long long)e;
        const double z = normal2(hash3(seed ^ 0x5bd1e995ULL, gid, 2 * c), hash3(seed ^ 0x5bd1e995ULL, gid, 2 * c + 1));
        Xt[e] = v + (float)(sigma * z);
    }
}

// Mode-n unfolding in BF16 with the contraction index contiguous:
// out[t][row][kappa] = X[t] element with index `row` along mode n and the
// other two modes (first before second) forming kappa.
__global__ void __launch_bounds__(256) k_ws_unfold_bf16(const float *X, __nv_bfloat16 *out, int I, int mode,
                                                        long ntensors) {
    const long n = (long)I * I * I;
    const long total = n * ntensors;
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
        const long t = e / n, rem = e % n;
        const long row = rem / ((long)I * I), kap = rem % ((long)I * I);
        const long a = kap % I, b = kap / I;  // the other modes, in order
        long i, j, k;
        if (mode == 0) { i = row; j = a; k = b; }
        else if (mode == 1) { i = a; j = row; k = b; }
        else { i = a; j = b; k = row; }
        out[e] = __float2bfloat16_rn(X[t * n + i + I * (j + (long)I * k)]);
    }
}

// Features: in[t][m*I*S + i*S + c] = sketch_m[t*I + i][c] / ||X_t||, BF16,
// and the transposed copy inT[feature][t].  S = sketch width.
struct Sketches {
    const float *m[3];
};
__global__ void __launch_bounds__(256) k_ws_pack(Sketches sk, const double *xnorm2, __nv_bfloat16 *in,
                                                 __nv_bfloat16 *inT, int I, int S, long ntensors) {
    const long nf = 3L * I * S;
    const long total = nf * ntensors;
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
        const long t = e / nf, f = e % nf;
        const int m = (int)(f / ((long)I * S)), rem = (int)(f % ((long)I * S)), i = rem / S, c = rem % S;
        const float scale = (float)(1.0 / sqrt(xnorm2[t] > 0.0 ? xnorm2[t] : 1.0));
        const float *src = (m == 0) ? sk.m[0] : (m == 1 ? sk.m[1] : sk.m[2]);
        const __nv_bfloat16 v = __float2bfloat16_rn(src[(t * I + i) * S + c] * scale);
        in[e] = v;
        if (inT) inT[f * ntensors + t] = v;
    }
}

// ||X_t||^2 of each tensor (FP64), one CTA per tensor.
__global__ void __launch_bounds__(256) k_ws_norms(const float *X, long n, double *out) {
    __shared__ double red[256];
    const float *x = X + (long)blockIdx.x * n;
    double s = 0.0;
    for (long e = threadIdx.x; e < n; e += 256) s += (double)x[e] * (double)x[e];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[blockIdx.x] = red[0];
}

// Canonical CP factors of tensor t (3 column-major I x R factors, in place):
// columns of U_0 and U_1 scaled to unit norm with non-negative sums, the
// scales and signs moved into U_2, which is then divided by ||X_t||; columns
// ordered by the norm of their U_2 column, largest first.  One CTA per
// tensor.
__global__ void __launch_bounds__(128) k_ws_canonical(float *F, const double *xnorm2, int I, int R) {
    __shared__ float fs[3 * 128 * 16];
    __shared__ float w[16];
    __shared__ int order[16];
    const long t = blockIdx.x;
    const int per = I * R;
    float *Ft = F + t * 3 * per;
    for (int e = threadIdx.x; e < 3 * per; e += blockDim.x) fs[e] = Ft[e];
    __syncthreads();
    if (threadIdx.x < R) {
        const int r = threadIdx.x;
        double scale = 1.0 / sqrt(xnorm2[t] > 0.0 ? xnorm2[t] : 1.0);
        for (int m = 0; m < 2; m++) {
            float *c = fs + m * per + I * r;
            double n2 = 0.0, sum = 0.0;
            for (int i = 0; i < I; i++) { n2 += (double)c[i] * c[i]; sum += c[i]; }
            const double nrm = sqrt(n2);
            const double sg = (sum < 0.0) ? -1.0 : 1.0;
            if (nrm > 0.0)
                for (int i = 0; i < I; i++) c[i] = (float)(c[i] * sg / nrm);
            scale *= nrm * sg;
        }
        float *c2 = fs + 2 * per + I * r;
        double n2 = 0.0;
        for (int i = 0; i < I; i++) {
            c2[i] = (float)(c2[i] * scale);
            n2 += (double)c2[i] * c2[i];
        }
        w[r] = (float)sqrt(n2);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int r = 0; r < R; r++) order[r] = r;
        for (int a = 1; a < R; a++)  // insertion sort, largest first, stable
            for (int b = a; b > 0 && w[order[b]] > w[order[b - 1]]; b--) {
                const int tmp = order[b]; order[b] = order[b - 1]; order[b - 1] = tmp;
            }
    }
    __syncthreads();
    for (int e = threadIdx.x; e < 3 * per; e += blockDim.x) {
        const int m = e / per, rem = e % per, r = rem / I, i = rem % I;
        Ft[e] = fs[m * per + I * order[r] + i];
    }
}

// Predicted factors (rows of Y, canonical form) -> ALS initial factors:
// U_m = Y[t][m*I*R ...] with U_2 scaled back by ||X_t||.
__global__ void __launch_bounds__(256) k_ws_uncanon(const float *Y, const double *xnorm2, float *F, int I, int R,
                                                    long ntensors) {
    const long per3 = 3L * I * R;
    const long total = per3 * ntensors;
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < total; e += (long)gridDim.x * blockDim.x) {
        const long t = e / per3, f = e % per3;
        const double s = (f >= 2L * I * R) ? sqrt(xnorm2[t]) : 1.0;
        F[e] = (float)(Y[e] * s);
    }
}

// Aligns each sample's target factors to the prediction (in place): the
// target's rank-1 terms are matched to the predicted ones greedily by
// |<a, a'> <b, b'> <c, c'>| (columns normalised), reordered into the
// prediction's order, and sign-aligned -- the target's U_0 and U_1 columns
// flipped to agree with the prediction, U_2 compensating so each rank-1
// term is unchanged.  Removes the loss's dependence on the arbitrary order
// and signs of CP components.  One CTA (R*R <= 256 threads) per sample.
__global__ void __launch_bounds__(256) k_ws_align(const float *Y, float *T, int I, int R) {
    __shared__ float sim[16][16], sga[16][16], sgb[16][16];
    __shared__ int match[16];
    __shared__ float tmp[3 * 128 * 16];
    const long t = blockIdx.x;
    const int per = I * R;
    const float *y = Y + t * 3 * per;
    float *tt = T + t * 3 * per;
    const int p = threadIdx.x / R, q = threadIdx.x % R;  // predicted p, target q
    if (threadIdx.x < R * R) {
        float prod = 1.f, sa = 1.f, sb = 1.f;
        for (int m = 0; m < 3; m++) {
            const float *yp = y + m * per + p * I, *tq = tt + m * per + q * I;
            float d = 0.f, ny = 0.f, nt = 0.f;
            for (int i = 0; i < I; i++) { d += yp[i] * tq[i]; ny += yp[i] * yp[i]; nt += tq[i] * tq[i]; }
            const float c = d / sqrtf(fmaxf(ny * nt, 1e-30f));
            prod *= c;
            if (m == 0) sa = (d < 0.f) ? -1.f : 1.f;
            if (m == 1) sb = (d < 0.f) ? -1.f : 1.f;
        }
        sim[p][q] = fabsf(prod);
        sga[p][q] = sa;
        sgb[p][q] = sb;
    }
    for (int e = threadIdx.x; e < 3 * per; e += blockDim.x) tmp[e] = tt[e];
    __syncthreads();
    if (threadIdx.x == 0) {
        bool used_p[16] = {}, used_q[16] = {};
        for (int k = 0; k < R; k++) {  // greedy: the best remaining pair, fixed tie order
            float best = -1.f;
            int bp = 0, bq = 0;
            for (int a = 0; a < R; a++)
                for (int b = 0; b < R; b++)
                    if (!used_p[a] && !used_q[b] && sim[a][b] > best) { best = sim[a][b]; bp = a; bq = b; }
            used_p[bp] = used_q[bq] = true;
            match[bp] = bq;
        }
    }
    __syncthreads();
    for (int e = threadIdx.x; e < 3 * per; e += blockDim.x) {
        const int m = e / per, rem = e % per, r = rem / I, i = rem % I;
        const int qq = match[r];
        const float sa = sga[r][qq], sb = sgb[r][qq];
        const float sg = (m == 0) ? sa : (m == 1 ? sb : sa * sb);
        tt[e] = sg * tmp[m * per + qq * I + i];
    }
}

// MSE loss 1/(B*D) sum (Y - T)^2 and its gradient dY = 2 (Y - T) / (B*D) as
// BF16 (B x D) and its transpose (D x B).  loss2[0] += partial sums.
__global__ void __launch_bounds__(256) k_ws_mse(const float *Y, const float *T, long B, long D,
                                                __nv_bfloat16 *dY, __nv_bfloat16 *dYt, double *loss) {
    __shared__ double red[256];
    const long total = B * D;
    const float scale = (float)(2.0 / (double)total);
    double s = 0.0;
    for (long e = blockIdx.x * 256L + threadIdx.x; e < total; e += (long)gridDim.x * 256L) {
        const float d = Y[e] - T[e];
        s += (double)d * d;
        const __nv_bfloat16 g = __float2bfloat16_rn(d * scale);
        dY[e] = g;
        const long b = e / D, j = e % D;
        dYt[j * B + b] = g;
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) red[threadIdx.x] += red[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) atomicAdd(loss, red[0] / (double)total);
}

// db[n] = sum_m G[m][n] (G row-major B x N, BF16), fixed order per n.
__global__ void __launch_bounds__(256) k_ws_colsum(const __nv_bfloat16 *G, long B, long N, float *db) {
    const long n = blockIdx.x * 256L + threadIdx.x;
    if (n >= N) return;
    float s = 0.f;
    for (long m = 0; m < B; m++) s += __bfloat162float(G[m * N + n]);
    db[n] = s;
}

// Adam step on FP32 master weights W (rows x cols, row-major) with gradient
// g; writes the BF16 working copy and (if Wt) its transpose.
__global__ void __launch_bounds__(256) k_ws_adam(float *W, const float *g, float *m1, float *m2, long rows,
                                                 long cols, float lr, float b1, float b2, float eps, float c1,
                                                 float c2, __nv_bfloat16 *Wh, __nv_bfloat16 *Wt) {
    const long total = rows * cols;
    for (long e = blockIdx.x * 256L + threadIdx.x; e < total; e += (long)gridDim.x * 256L) {
        const float gr = g[e];
        const float a = b1 * m1[e] + (1.f - b1) * gr;
        const float b = b2 * m2[e] + (1.f - b2) * gr * gr;
        m1[e] = a;
        m2[e] = b;
        const float w = W[e] - lr * (a / c1) / (sqrtf(b / c2) + eps);
        W[e] = w;
        const __nv_bfloat16 h = __float2bfloat16_rn(w);
        if (Wh) Wh[e] = h;
        if (Wt) {
            const long r = e / cols, c = e % cols;
            Wt[c * rows + r] = h;
        }
    }
}

}  // namespace cud

// ---------------------------------------------------------------- batched HOSVD init

namespace cud {

namespace {

// Gram of the mode-m unfolding of tensor t (I^3, column-major), FP32 SIMT:
// G[t][m] (I x I) = X_(m) X_(m)^T, one CTA per (t, m), I <= 64.
__global__ void __launch_bounds__(256) k_ws_gram(const float *X, float *G, int I) {
    __shared__ float slab[64 * 65];
    const long t = blockIdx.x / 3;
    const int m = (int)(blockIdx.x % 3);
    const long n = (long)I * I * I;
    const float *x = X + t * n;
    const int tx = threadIdx.x % 16, ty = threadIdx.x / 16;  // 16 x 16 threads, 4 x 4 outputs each
    float acc[4][4] = {};
    // the other two modes index kappa = (a, b); stage one b-slice (I x I
    // matrix of rows = mode-m index, columns = a) at a time
    for (int b = 0; b < I; b++) {
        __syncthreads();
        for (int e = threadIdx.x; e < I * I; e += 256) {
            const int row = e % I, a = e / I;
            long idx;
            if (m == 0) idx = row + (long)I * (a + (long)I * b);
            else if (m == 1) idx = a + (long)I * (row + (long)I * b);
            else idx = a + (long)I * (b + (long)I * row);
            slab[row * 65 + a] = x[idx];
        }
        __syncthreads();
        for (int a = 0; a < I; a++) {
            float u[4], v[4];
#pragma unroll
            for (int q = 0; q < 4; q++) {
                const int r1 = ty * 4 + q, r2 = tx * 4 + q;
                u[q] = r1 < I ? slab[r1 * 65 + a] : 0.f;
                v[q] = r2 < I ? slab[r2 * 65 + a] : 0.f;
            }
#pragma unroll
            for (int p = 0; p < 4; p++)
#pragma unroll
                for (int q = 0; q < 4; q++) acc[p][q] = fmaf(u[p], v[q], acc[p][q]);
        }
    }
    float *g = G + (t * 3 + m) * (long)I * I;
    for (int p = 0; p < 4; p++)
        for (int q = 0; q < 4; q++) {
            const int r1 = ty * 4 + p, r2 = tx * 4 + q;
            if (r1 < I && r2 < I) g[r1 + (long)I * r2] = acc[p][q];
        }
}

// Top-R eigenvectors of each symmetric I x I matrix (I <= 64, even or odd),
// cyclic Jacobi with the round-robin pairing (I/2 disjoint rotations per
// round, all applied in parallel), FP32 in shared memory.  Writes the
// eigenvectors of the R largest eigenvalues, largest first, as the I x R
// column-major factor at F + (t*3 + m) * I * R.
__global__ void __launch_bounds__(256) k_ws_jacobi_top(const float *G, float *F, int I, int R, int max_sweeps) {
    __shared__ float A[64][65];
    __shared__ float V[64][65];
    __shared__ float cs[32], sn[32];
    __shared__ int pp[32], qq[32];
    __shared__ int perm[64];
    __shared__ float off_red[256];
    const int n = (I + 1) / 2 * 2;  // padded to even: a dummy index decouples
    const float *g = G + (long)blockIdx.x * I * I;
    for (int e = threadIdx.x; e < n * n; e += 256) {
        const int r = e % n, c = e / n;
        A[r][c] = (r < I && c < I) ? g[r + (long)I * c] : 0.f;
        V[r][c] = (r == c) ? 1.f : 0.f;
    }
    __syncthreads();
    float norm = 0.f;
    for (int e = 0; e < n; e++) norm = fmaxf(norm, fabsf(A[e][e]));
    // the cyclic sweeps converge quadratically down to FP32's rounding floor
    // and then stall: stop at the tolerance, or once a sweep no longer
    // halves the off-diagonal mass
    float prev_off = 3.4e38f;
    for (int sweep = 0; sweep < max_sweeps; sweep++) {
        // off-diagonal mass
        float s = 0.f;
        for (int e = threadIdx.x; e < n * n; e += 256) {
            const int r = e % n, c = e / n;
            if (r != c) s += A[r][c] * A[r][c];
        }
        off_red[threadIdx.x] = s;
        __syncthreads();
        for (int w = 128; w > 0; w >>= 1) {
            if (threadIdx.x < w) off_red[threadIdx.x] += off_red[threadIdx.x + w];
            __syncthreads();
        }
        const float off = off_red[0];
        __syncthreads();
        if (!(off > 1e-12f * norm * norm)) break;
        if (sweep >= 2 && off > 0.5f * prev_off) break;
        prev_off = off;
        for (int round = 0; round < n - 1; round++) {
            if (threadIdx.x < n / 2) {
                // round-robin: index n-1 fixed, the others rotate
                const int k = threadIdx.x;
                int a = (k == 0) ? n - 1 : (round + k) % (n - 1);
                int b = (round + n - 1 - k) % (n - 1);
                if (k == 0) b = round % (n - 1);
                const int p = min(a, b), q = max(a, b);
                const float apq = A[p][q];
                float c = 1.f, sgn = 0.f;
                if (fabsf(apq) > 1e-30f) {
                    const float theta = (A[q][q] - A[p][p]) / (2.f * apq);
                    const float tt = copysignf(1.f, theta) / (fabsf(theta) + sqrtf(theta * theta + 1.f));
                    c = rsqrtf(tt * tt + 1.f);
                    sgn = tt * c;
                }
                cs[k] = c; sn[k] = sgn; pp[k] = p; qq[k] = q;
            }
            __syncthreads();
            // A <- J^T A (rows p, q), then A <- A J (columns p, q), V <- V J
            for (int e = threadIdx.x; e < (n / 2) * n; e += 256) {
                const int k = e / n, col = e % n;
                const int p = pp[k], q = qq[k];
                const float c = cs[k], s = sn[k];
                const float ap = A[p][col], aq = A[q][col];
                A[p][col] = c * ap - s * aq;
                A[q][col] = s * ap + c * aq;
            }
            __syncthreads();
            for (int e = threadIdx.x; e < (n / 2) * n; e += 256) {
                const int k = e / n, row = e % n;
                const int p = pp[k], q = qq[k];
                const float c = cs[k], s = sn[k];
                const float ap = A[row][p], aq = A[row][q];
                A[row][p] = c * ap - s * aq;
                A[row][q] = s * ap + c * aq;
                const float vp = V[row][p], vq = V[row][q];
                V[row][p] = c * vp - s * vq;
                V[row][q] = s * vp + c * vq;
            }
            __syncthreads();
        }
    }
    if (threadIdx.x == 0) {
        for (int e = 0; e < n; e++) perm[e] = e;
        for (int a = 1; a < n; a++)  // eigenvalues descending (diagonal), dummy index last
            for (int b = a; b > 0; b--) {
                const int x = perm[b], y = perm[b - 1];
                const float vx = x < I ? A[x][x] : -3.4e38f, vy = y < I ? A[y][y] : -3.4e38f;
                if (vx > vy) { perm[b] = y; perm[b - 1] = x; } else break;
            }
    }
    __syncthreads();
    float *f = F + (long)blockIdx.x * I * R;
    for (int e = threadIdx.x; e < I * R; e += 256) {
        const int i = e % I, r = e / I;
        f[e] = (r < n) ? V[i][perm[r]] : 0.f;
    }
}

// Omega_m^T (S x I^2, BF16, K-major): i.i.d. N(0, 1) from the hash stream.
__global__ void __launch_bounds__(256) k_ws_omega(__nv_bfloat16 *om, long n, unsigned long long seed) {
    for (long e = blockIdx.x * 256L + threadIdx.x; e < n; e += (long)gridDim.x * 256L)
        om[e] = __float2bfloat16_rn((float)normal2(hash3(seed, 0x0e, 2 * (unsigned long long)e),
                                                   hash3(seed, 0x0e, 2 * (unsigned long long)e + 1)));
}

__global__ void __launch_bounds__(256) k_ws_init_uniform(float *W, long n, float bound, unsigned long long seed) {
    for (long e = blockIdx.x * 256L + threadIdx.x; e < n; e += (long)gridDim.x * 256L)
        W[e] = (float)((2.0 * u01(hash3(seed, 0x77, (unsigned long long)e)) - 1.0) * bound);
}

__global__ void __launch_bounds__(256) k_ws_to_bf16(const float *W, long rows, long cols, __nv_bfloat16 *Wh,
                                                    __nv_bfloat16 *Wt) {
    const long total = rows * cols;
    for (long e = blockIdx.x * 256L + threadIdx.x; e < total; e += (long)gridDim.x * 256L) {
        const __nv_bfloat16 h = __float2bfloat16_rn(W[e]);
        if (Wh) Wh[e] = h;
        if (Wt) Wt[(e % cols) * rows + e / cols] = h;
    }
}

unsigned grid_for(long n) { return (unsigned)std::min<long>((n + 255) / 256, 8L * kNumSMs); }

}  // namespace
}  // namespace cud

// ---------------------------------------------------------------- model

struct cud_ws_model_s {
    int in = 0, hid = 0, out = 0, maxb = 0;
    char *mem = nullptr;
    size_t bytes = 0;
    // FP32 master parameters, Adam moments and gradients: 6 tensors each
    float *P[6] = {}, *M1[6] = {}, *M2[6] = {}, *G[6] = {};
    long rows[6] = {}, cols[6] = {};
    __nv_bfloat16 *W1h = nullptr, *W2h = nullptr, *W2t = nullptr, *W3h = nullptr, *W3t = nullptr;
    __nv_bfloat16 *H1 = nullptr, *H1t = nullptr, *H2 = nullptr, *H2t = nullptr;
    __nv_bfloat16 *dY = nullptr, *dYt = nullptr, *dH2 = nullptr, *dH2t = nullptr, *dH1 = nullptr, *dH1t = nullptr;
    float *Y = nullptr;
    double *loss = nullptr;
    void *ws = nullptr;
    size_t ws_bytes = 0;
    long step = 0;
    int align_I = 0, align_R = 0;  // when set, targets are aligned to the prediction (k_ws_align)
    float *Ta = nullptr;           // the aligned copy of the targets
};

using namespace cud;

namespace {

int ws_gemm(cud_ws_model m, const __nv_bfloat16 *A, long lda, const __nv_bfloat16 *B, long ldb, long M, long N,
            long K, const GemmEpi &e, cudaStream_t s) {
    if (gemm_tc_ws_bytes(M, N, K) > m->ws_bytes) return CUD_ERR_INVALID_ARGUMENT;
    return gemm_tc_bf16(A, lda, B, ldb, M, N, K, e, m->ws, s);
}

GemmEpi epi0() {
    GemmEpi e;
    memset(&e, 0, sizeof(e));
    e.alpha = 1.f;
    return e;
}

int ws_refresh_bf16(cud_ws_model m, cudaStream_t s) {
    k_ws_to_bf16<<<grid_for(m->rows[0] * m->cols[0]), 256, 0, s>>>(m->P[0], m->rows[0], m->cols[0], m->W1h, nullptr);
    k_ws_to_bf16<<<grid_for(m->rows[2] * m->cols[2]), 256, 0, s>>>(m->P[2], m->rows[2], m->cols[2], m->W2h, m->W2t);
    k_ws_to_bf16<<<grid_for(m->rows[4] * m->cols[4]), 256, 0, s>>>(m->P[4], m->rows[4], m->cols[4], m->W3h, m->W3t);
    CUD_CHECK_LAUNCH("ws bf16 copies");
    return CUD_OK;
}

// Forward pass of a batch; keeps H1, H2 (and transposes) for the backward.
int ws_forward(cud_ws_model m, const __nv_bfloat16 *in, long B, float *Y, cudaStream_t s) {
    const long H = m->hid;
    GemmEpi e = epi0();
    e.bias = m->P[1]; e.relu = 1;
    e.out_bf16 = m->H1; e.bf16_ldm = H; e.bf16_ldn = 1;
    e.out_bf16_2 = m->H1t; e.bf16_2_ldm = 1; e.bf16_2_ldn = B;
    int st = ws_gemm(m, in, m->in, m->W1h, m->in, B, H, m->in, e, s);
    if (st) return st;
    e = epi0();
    e.bias = m->P[3]; e.relu = 1;
    e.out_bf16 = m->H2; e.bf16_ldm = H; e.bf16_ldn = 1;
    e.out_bf16_2 = m->H2t; e.bf16_2_ldm = 1; e.bf16_2_ldn = B;
    st = ws_gemm(m, m->H1, H, m->W2h, H, B, H, H, e, s);
    if (st) return st;
    e = epi0();
    e.bias = m->P[5];
    e.out_f32 = Y; e.f32_ldm = m->out; e.f32_ldn = 1;
    return ws_gemm(m, m->H2, H, m->W3h, H, B, m->out, H, e, s);
}

int ws_backward(cud_ws_model m, const __nv_bfloat16 *in, const __nv_bfloat16 *inT, const float *target, long B,
                cudaStream_t s) {
    const long H = m->hid, O = m->out, D = m->in;
    int st = ws_forward(m, in, B, m->Y, s);
    if (st) return st;
    CUD_CHECK(cudaMemsetAsync(m->loss, 0, sizeof(double), s));
    if (m->align_I > 0) {
        CUD_CHECK(cudaMemcpyAsync(m->Ta, target, sizeof(float) * B * O, cudaMemcpyDeviceToDevice, s));
        k_ws_align<<<(unsigned)B, 256, 0, s>>>(m->Y, m->Ta, m->align_I, m->align_R);
        CUD_CHECK_LAUNCH("ws align");
        target = m->Ta;
    }
    k_ws_mse<<<grid_for(B * O), 256, 0, s>>>(m->Y, target, B, O, m->dY, m->dYt, m->loss);
    CUD_CHECK_LAUNCH("ws mse");
    // layer 3
    GemmEpi e = epi0();
    e.out_f32 = m->G[4]; e.f32_ldm = H; e.f32_ldn = 1;
    if ((st = ws_gemm(m, m->dYt, B, m->H2t, B, O, H, B, e, s))) return st;
    k_ws_colsum<<<(unsigned)((O + 255) / 256), 256, 0, s>>>(m->dY, B, O, m->G[5]);
    e = epi0();
    e.mask = m->H2; e.mask_ldm = H; e.mask_ldn = 1;
    e.out_bf16 = m->dH2; e.bf16_ldm = H; e.bf16_ldn = 1;
    e.out_bf16_2 = m->dH2t; e.bf16_2_ldm = 1; e.bf16_2_ldn = B;
    if ((st = ws_gemm(m, m->dY, O, m->W3t, O, B, H, O, e, s))) return st;
    // layer 2
    e = epi0();
    e.out_f32 = m->G[2]; e.f32_ldm = H; e.f32_ldn = 1;
    if ((st = ws_gemm(m, m->dH2t, B, m->H1t, B, H, H, B, e, s))) return st;
    k_ws_colsum<<<(unsigned)((H + 255) / 256), 256, 0, s>>>(m->dH2, B, H, m->G[3]);
    e = epi0();
    e.mask = m->H1; e.mask_ldm = H; e.mask_ldn = 1;
    e.out_bf16 = m->dH1; e.bf16_ldm = H; e.bf16_ldn = 1;
    e.out_bf16_2 = m->dH1t; e.bf16_2_ldm = 1; e.bf16_2_ldn = B;
    if ((st = ws_gemm(m, m->dH2, H, m->W2t, H, B, H, H, e, s))) return st;
    // layer 1
    e = epi0();
    e.out_f32 = m->G[0]; e.f32_ldm = D; e.f32_ldn = 1;
    if ((st = ws_gemm(m, m->dH1t, B, inT, B, H, D, B, e, s))) return st;
    k_ws_colsum<<<(unsigned)((H + 255) / 256), 256, 0, s>>>(m->dH1, B, H, m->G[1]);
    CUD_CHECK_LAUNCH("ws colsum");
    return CUD_OK;
}

}  // namespace

extern "C" int cud_ws_model_create(int in_dim, int hidden, int out_dim, int max_batch, unsigned long long seed,
                                   cud_ws_model *out) {
    if (!out || in_dim <= 0 || hidden <= 0 || out_dim <= 0 || max_batch <= 0 || (in_dim % 8) || (hidden % 8) ||
        (out_dim % 8) || (max_batch % 8))
        return set_status(CUD_ERR_INVALID_ARGUMENT);
    cud_ws_model m = new cud_ws_model_s();
    m->in = in_dim; m->hid = hidden; m->out = out_dim; m->maxb = max_batch;
    const long rows[6] = {hidden, 1, hidden, 1, out_dim, 1};
    const long cols[6] = {in_dim, hidden, hidden, hidden, hidden, out_dim};
    size_t f32 = 0;
    for (int k = 0; k < 6; k++) { m->rows[k] = rows[k]; m->cols[k] = cols[k]; f32 += 4 * (size_t)rows[k] * cols[k]; }
    const long H = hidden, O = out_dim, D = in_dim, B = max_batch;
    const size_t bf = 2 * ((size_t)H * D + 2 * H * H + 2 * O * H + 4 * B * H + 2 * B * O + 4 * B * H);
    const size_t wsb = std::max({gemm_tc_ws_bytes(B, H, D), gemm_tc_ws_bytes(B, H, H), gemm_tc_ws_bytes(B, O, H),
                                 gemm_tc_ws_bytes(O, H, B), gemm_tc_ws_bytes(B, H, O), gemm_tc_ws_bytes(H, H, B),
                                 gemm_tc_ws_bytes(H, D, B)});
    // + 256-byte rounding of each of the 41 buffers carved below
    m->bytes = 4 * f32 + bf + 8 * (size_t)B * O + 256 + wsb + 48 * 256;
    if (cudaMalloc(&m->mem, m->bytes) != cudaSuccess) {
        cudaGetLastError();
        delete m;
        return set_status(CUD_ERR_NO_MEMORY);
    }
    cudaMemset(m->mem, 0, m->bytes);
    char *p = m->mem;
    auto take = [&](size_t b) { char *q = p; p += (b + 255) / 256 * 256; return q; };
    for (int k = 0; k < 6; k++) {
        const size_t b = 4 * (size_t)rows[k] * cols[k];
        m->P[k] = (float *)take(b); m->M1[k] = (float *)take(b); m->M2[k] = (float *)take(b); m->G[k] = (float *)take(b);
    }
    m->W1h = (__nv_bfloat16 *)take(2 * H * D);
    m->W2h = (__nv_bfloat16 *)take(2 * H * H); m->W2t = (__nv_bfloat16 *)take(2 * H * H);
    m->W3h = (__nv_bfloat16 *)take(2 * O * H); m->W3t = (__nv_bfloat16 *)take(2 * O * H);
    m->H1 = (__nv_bfloat16 *)take(2 * B * H); m->H1t = (__nv_bfloat16 *)take(2 * B * H);
    m->H2 = (__nv_bfloat16 *)take(2 * B * H); m->H2t = (__nv_bfloat16 *)take(2 * B * H);
    m->dY = (__nv_bfloat16 *)take(2 * B * O); m->dYt = (__nv_bfloat16 *)take(2 * B * O);
    m->dH2 = (__nv_bfloat16 *)take(2 * B * H); m->dH2t = (__nv_bfloat16 *)take(2 * B * H);
    m->dH1 = (__nv_bfloat16 *)take(2 * B * H); m->dH1t = (__nv_bfloat16 *)take(2 * B * H);
    m->Y = (float *)take(4 * (size_t)B * O);
    m->Ta = (float *)take(4 * (size_t)B * O);
    m->loss = (double *)take(64);
    m->ws_bytes = wsb;
    m->ws = take(wsb);
    if ((size_t)(p - m->mem) > m->bytes) {
        cudaFree(m->mem);
        delete m;
        return set_status(CUD_ERR_INVALID_ARGUMENT);
    }
    // He-uniform hidden weights (fan-in), zero biases, and a zero output
    // layer: the network starts at the zero prediction and its first
    // gradients into the hidden layers are small.  (He-initialised output
    // weights made the first Adam steps drive nearly all of the second
    // layer's ReLUs dead, leaving a constant predictor.)
    const float b1 = sqrtf(6.f / (float)D), b2 = sqrtf(6.f / (float)H);
    k_ws_init_uniform<<<grid_for(H * D), 256>>>(m->P[0], H * D, b1, seed);
    k_ws_init_uniform<<<grid_for(H * H), 256>>>(m->P[2], H * H, b2, seed + 1);
    cudaMemsetAsync(m->P[4], 0, sizeof(float) * (size_t)O * H, 0);  // checked by the synchronise below
    int st = ws_refresh_bf16(m, nullptr);
    if (st == CUD_OK && cudaDeviceSynchronize() != cudaSuccess) st = CUD_ERR_CUDA;
    if (st) {
        cudaFree(m->mem);
        delete m;
        return set_status(st);
    }
    *out = m;
    return set_status(CUD_OK);
}

extern "C" int cud_ws_model_align(cud_ws_model m, int I, int R) {
    if (!m || I < 0 || R < 0 || R > 16 || I > 128 || (I > 0 && 3 * I * R != m->out))
        return set_status(CUD_ERR_INVALID_ARGUMENT);
    m->align_I = I;
    m->align_R = R;
    return set_status(CUD_OK);
}

extern "C" int cud_ws_model_destroy(cud_ws_model m) {
    if (!m) return set_status(CUD_ERR_INVALID_ARGUMENT);
    cudaFree(m->mem);
    delete m;
    return set_status(CUD_OK);
}

extern "C" int cud_ws_model_params(cud_ws_model m, float *const *host, int set) {
    if (!m || !host) return set_status(CUD_ERR_INVALID_ARGUMENT);
    for (int k = 0; k < 6; k++) {
        if (!host[k]) continue;
        const size_t b = 4 * (size_t)m->rows[k] * m->cols[k];
        CUD_CHECK(set ? cudaMemcpy(m->P[k], host[k], b, cudaMemcpyHostToDevice)
                      : cudaMemcpy(host[k], m->P[k], b, cudaMemcpyDeviceToHost));
    }
    if (set) {
        int st = ws_refresh_bf16(m, nullptr);
        if (st) return set_status(st);
        CUD_CHECK(cudaDeviceSynchronize());
    }
    return set_status(CUD_OK);
}

extern "C" int cud_ws_model_grads(cud_ws_model m, float *const *host) {
    if (!m || !host) return set_status(CUD_ERR_INVALID_ARGUMENT);
    CUD_CHECK(cudaDeviceSynchronize());
    for (int k = 0; k < 6; k++)
        if (host[k]) CUD_CHECK(cudaMemcpy(host[k], m->G[k], 4 * (size_t)m->rows[k] * m->cols[k], cudaMemcpyDeviceToHost));
    return set_status(CUD_OK);
}

extern "C" int cud_ws_backward(cud_ws_model m, const void *in, const void *inT, const float *target, int batch,
                               double *loss, void *stream) {
    if (!m || !in || !inT || !target || batch <= 0 || batch > m->maxb || (batch % 8))
        return set_status(CUD_ERR_INVALID_ARGUMENT);
    cudaStream_t s = as_stream(stream);
    int st = ws_backward(m, static_cast<const __nv_bfloat16 *>(in), static_cast<const __nv_bfloat16 *>(inT), target,
                         batch, s);
    if (st) return set_status(st);
    if (loss) {
        CUD_CHECK(cudaMemcpyAsync(loss, m->loss, sizeof(double), cudaMemcpyDeviceToHost, s));
        CUD_CHECK(cudaStreamSynchronize(s));
    }
    return set_status(CUD_OK);
}

extern "C" int cud_ws_train_step(cud_ws_model m, const void *in, const void *inT, const float *target, int batch,
                                 float lr, double *loss, void *stream) {
    int st = cud_ws_backward(m, in, inT, target, batch, nullptr, stream);
    if (st) return st;
    cudaStream_t s = as_stream(stream);
    m->step++;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.f - powf(b1, (float)m->step), c2 = 1.f - powf(b2, (float)m->step);
    for (int k = 0; k < 6; k++) {
        __nv_bfloat16 *Wh = nullptr, *Wt = nullptr;
        if (k == 0) Wh = m->W1h;
        if (k == 2) { Wh = m->W2h; Wt = m->W2t; }
        if (k == 4) { Wh = m->W3h; Wt = m->W3t; }
        const long n = m->rows[k] * m->cols[k];
        k_ws_adam<<<grid_for(n), 256, 0, s>>>(m->P[k], m->G[k], m->M1[k], m->M2[k], m->rows[k], m->cols[k], lr, b1,
                                              b2, 1e-8f, c1, c2, Wh, Wt);
    }
    CUD_CHECK_LAUNCH("ws adam");
    if (loss) {
        CUD_CHECK(cudaMemcpyAsync(loss, m->loss, sizeof(double), cudaMemcpyDeviceToHost, s));
        CUD_CHECK(cudaStreamSynchronize(s));
    }
    return set_status(CUD_OK);
}

extern "C" int cud_ws_predict(cud_ws_model m, const void *in, int batch, float *out, void *stream) {
    if (!m || !in || !out || batch <= 0 || batch > m->maxb) return set_status(CUD_ERR_INVALID_ARGUMENT);
    return set_status(ws_forward(m, static_cast<const __nv_bfloat16 *>(in), batch, out, as_stream(stream)));
}

// ---------------------------------------------------------------- data entry points

extern "C" int cud_ws_generate(long ntensors, long id0, unsigned long long seed, int I, int R, double noise,
                               float *X, float *F, double *clean_norm2, void *stream) {
    if (ntensors <= 0 || ntensors > 65535 || I <= 0 || I > 128 || R <= 0 || R > 16 || !X || !F || !clean_norm2)
        return set_status(CUD_ERR_INVALID_ARGUMENT);
    cudaStream_t s = as_stream(stream);
    k_ws_factors<<<(unsigned)ntensors, 256, 3 * I * R * sizeof(float), s>>>(F, clean_norm2, I, R, id0, seed);
    const long n = (long)I * I * I;
    const unsigned bx = (unsigned)std::min<long>((n + 255) / 256, 64);
    k_ws_tensor<<<dim3(bx, (unsigned)ntensors), 256, 0, s>>>(F, clean_norm2, X, I, R, id0, seed, noise);
    CUD_CHECK_LAUNCH("ws generate");
    return set_status(CUD_OK);
}

extern "C" int cud_ws_omega(int I, int S, unsigned long long seed, void *omega, void *stream) {
    if (I <= 0 || S <= 0 || !omega) return set_status(CUD_ERR_INVALID_ARGUMENT);
    const long n = 3L * S * I * I;
    k_ws_omega<<<grid_for(n), 256, 0, as_stream(stream)>>>(static_cast<__nv_bfloat16 *>(omega), n, seed);
    CUD_CHECK_LAUNCH("ws omega");
    return set_status(CUD_OK);
}

extern "C" int cud_ws_features(const float *X, long ntensors, int I, const void *omega, int S, void *in, void *in_t,
                               double *xnorm2, void *stream) {
    if (!X || ntensors <= 0 || I <= 0 || (I * I) % 8 || !omega || S <= 0 || !in || !xnorm2)
        return set_status(CUD_ERR_INVALID_ARGUMENT);
    cudaStream_t s = as_stream(stream);
    const long n = (long)I * I * I, K = (long)I * I, M = ntensors * I;
    int st;
    __nv_bfloat16 *unf = static_cast<__nv_bfloat16 *>(scratch(kSlotTmp0, sizeof(__nv_bfloat16) * n * ntensors, &st));
    if (!unf) return set_status(st);
    float *sk = static_cast<float *>(scratch(kSlotTmp1, sizeof(float) * 3 * M * S, &st));
    if (!sk) return set_status(st);
    void *ws = scratch(kSlotTmp2, gemm_tc_ws_bytes(M, S, K), &st);
    if (!ws) return set_status(st);
    k_ws_norms<<<(unsigned)ntensors, 256, 0, s>>>(X, n, xnorm2);
    CUD_CHECK_LAUNCH("ws norms");
    Sketches sks;
    for (int m = 0; m < 3; m++) {
        k_ws_unfold_bf16<<<grid_for(n * ntensors), 256, 0, s>>>(X, unf, I, m, ntensors);
        CUD_CHECK_LAUNCH("ws unfold");
        GemmEpi e = epi0();
        e.out_f32 = sk + (long)m * M * S; e.f32_ldm = S; e.f32_ldn = 1;
        st = gemm_tc_bf16(unf, K, static_cast<const __nv_bfloat16 *>(omega) + (long)m * S * K, K, M, S, K, e, ws, s);
        if (st) return set_status(st);
        sks.m[m] = sk + (long)m * M * S;
    }
    k_ws_pack<<<grid_for(3L * I * S * ntensors), 256, 0, s>>>(sks, xnorm2, static_cast<__nv_bfloat16 *>(in),
                                                              static_cast<__nv_bfloat16 *>(in_t), I, S, ntensors);
    CUD_CHECK_LAUNCH("ws pack");
    return set_status(CUD_OK);
}

extern "C" int cud_ws_canonical(float *F, const double *xnorm2, long ntensors, int I, int R, void *stream) {
    if (!F || !xnorm2 || ntensors <= 0 || I <= 0 || I > 128 || R <= 0 || R > 16)
        return set_status(CUD_ERR_INVALID_ARGUMENT);
    k_ws_canonical<<<(unsigned)ntensors, 128, 0, as_stream(stream)>>>(F, xnorm2, I, R);
    CUD_CHECK_LAUNCH("ws canonical");
    return set_status(CUD_OK);
}

extern "C" int cud_ws_uncanonical(const float *Y, const double *xnorm2, float *F, long ntensors, int I, int R,
                                  void *stream) {
    if (!Y || !xnorm2 || !F || ntensors <= 0 || I <= 0 || R <= 0) return set_status(CUD_ERR_INVALID_ARGUMENT);
    k_ws_uncanon<<<grid_for(3L * I * R * ntensors), 256, 0, as_stream(stream)>>>(Y, xnorm2, F, I, R, ntensors);
    CUD_CHECK_LAUNCH("ws uncanonical");
    return set_status(CUD_OK);
}

extern "C" int cud_ws_hosvd_init(const float *X, long ntensors, int I, int R, float *F, void *stream) {
    if (!X || !F || ntensors <= 0 || I <= 0 || I > 64 || R <= 0 || R > I) return set_status(CUD_ERR_INVALID_ARGUMENT);
    cudaStream_t s = as_stream(stream);
    int st;
    float *G = static_cast<float *>(scratch(kSlotTmp0, sizeof(float) * 3 * ntensors * I * I, &st));
    if (!G) return set_status(st);
    k_ws_gram<<<(unsigned)(3 * ntensors), 256, 0, s>>>(X, G, I);
    k_ws_jacobi_top<<<(unsigned)(3 * ntensors), 256, 0, s>>>(G, F, I, R, 30);
    CUD_CHECK_LAUNCH("ws hosvd init");
    return set_status(CUD_OK);
}
