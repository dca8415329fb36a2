// Batched CP-ALS: thousands of small, independent 3rd-order tensors of uneven
// shape and rank, one persistent kernel launch per ALS sweep for the whole
// batch (sized for 4096 tensors with dims in [16, 96] and ranks in [4, 16]).
//
// Each CTA pulls tensors from a work queue (largest first) and runs one full
// sweep of that tensor on its own, everything on-chip except X:
//   * the three factor matrices live in shared memory (<= 96 x 16 each);
//   * each MTTKRP streams X through shared memory one frontal slice
//     (I x J) at a time and contracts it with register-blocked FMA (the
//     ranks are too small for tensor cores to pay): mode 1 over j, modes 2
//     and 3 over i, with the slice's C row as the per-slice weight (mode 3
//     reduces the slice to one row of M);
//   * the R x R normal equations (Hadamard of the FP64 Grams) are inverted
//     by Gauss-Jordan in shared memory (FP64), with a tiny diagonal shift
//     retried when a pivot is not positive;
//   * the fit comes from ||X||^2 - 2 <M_3, C> + sum prod G (FP64), per
//     tensor; a tensor whose fit changed by less than `tol` is marked
//     converged and skipped by later sweeps.
// The host captures `sweeps_per_graph` sweeps (queue reset + kernel) in one
// CUDA graph and replays it until every tensor has converged or hit the
// sweep limit.  The CTA size, the CTAs per SM and the MTTKRP register tile's
// height come from a small autotuner
// (batched_tune) that times one sweep per candidate on the batch itself and
// caches the winner per batch shape class.
#include <atomic>
#include <map>
#include <mutex>
#include <vector>
#include <algorithm>

#include "kernels.cuh"

namespace cud {

namespace {

constexpr int BMAXD = 96;    // largest mode size handled (smem sizing)
constexpr int BMAXR = 16;    // largest rank handled
constexpr int B_RED3 = 2 * BMAXR * BMAXD;  // mode-3 partials: 2 RT groups x ranks x BMAXD / RT row groups

__device__ __forceinline__ void cp_async4(void *dst, const void *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

struct TensorMeta {
    long xoff;          // offset of X (elements) in the packed tensor buffer
    long uoff[3];       // offsets of the factors in the packed factor buffer
    int dims[3];
    int R;
    int done;
    int sweeps;
    double normx2;
    double fit, fit_prev;
    double target;      // stop once fit >= target (<= 0: no target)
    double G[3][BMAXR * BMAXR];  // factor Grams (FP64)
};

struct BatchArgs {
    TensorMeta *meta;
    const int *order;   // processing order (largest first)
    int ntensors;
    const float *X;
    float *U;
    unsigned *queue;    // work counter, zero at kernel start
    int *ndone;         // tensors marked converged so far
    int max_sweeps;
    double tol;
    int *fallbacks;
};

// shared memory layout (floats / doubles), sized for BMAXD x BMAXR
struct BatchSmem {
    float F[3][BMAXD * BMAXR];       // factors, column-major I_m x R
    float slice[2][BMAXD * (BMAXD + 1) + 4];  // two frontal slices (double buffer), row stride I + 1
    float M[BMAXD * BMAXR];          // MTTKRP result of the current mode
    float red3[B_RED3];              // mode-3 per-slice partials (group x rank x row group)
    double V[BMAXR * BMAXR];         // normal matrix / its inverse
    double rowk[BMAXR], colk[BMAXR];
    double red[32];
    int tensor;
    int fail;
};

template <int NT>
__device__ void load_factors(BatchSmem &sm, const BatchArgs &a, const TensorMeta &t) {
    for (int m = 0; m < 3; m++) {
        const float *src = a.U + t.uoff[m];
        const int n = t.dims[m] * t.R;
        for (int e = threadIdx.x; e < n; e += NT) sm.F[m][e] = src[e];
    }
}

// M (I_mode x R) = MTTKRP of mode `mode` with the factors in shared memory.
// Thread items: (RT consecutive rows, 4 ranks) with rows = i (mode 1) or j
// (modes 2, 3) -- an RT x 4 register tile, RT x 4 FMAs per RT + 4 shared
// loads; RT (2 or 4) is the autotuner's tile height.  The loads are not
// guarded: rows past the mode's end read the slice's padding column or the
// next column, ranks past R read the factor arrays' spare columns (all
// inside the buffers since BMAXD is a multiple of RT), and those products
// only reach accumulators that are never stored.  When the items leave
// threads idle, S <= 2 RT groups of threads split the inner contraction
// (over j, or over i) and their partials are added at the end (modes 1, 2)
// or per slice (mode 3) in group order.  The frontal slices stream through
// two shared-memory buffers with cp.async: slice k + 1 loads while slice k
// is contracted.  (A deeper ring measured slower: the contraction's
// instruction issue, not the load latency, sets the pace.)
template <int NT, int RT>
__device__ void mttkrp_small(BatchSmem &sm, const BatchArgs &a, const TensorMeta &t, int mode) {
    constexpr int GS = 2 * RT;          // most groups splitting one contraction
    constexpr int NGM = BMAXD / RT;     // row groups at most
    constexpr int IPB = (NGM * (BMAXR / 4) + NT - 1) / NT;
    static_assert(BMAXD % RT == 0, "row tiles must divide BMAXD");
    static_assert(GS * BMAXR * NGM <= B_RED3, "mode-3 partials");
    const int I = t.dims[0], J = t.dims[1], K = t.dims[2], R = t.R;
    const int ld = I + 1;
    const float *X = a.X + t.xoff;
    const int Q = t.dims[mode];
    const int rows = (mode == 0) ? I : J;
    const int ngrp = (rows + RT - 1) / RT;
    const int rq = (R + 3) / 4;
    const int items = ngrp * rq;
    const int S = max(1, min(GS, NT / max(1, items)));
    const int L = (mode == 0) ? J : I;  // contraction length within a slice
    // this thread: item it = tid % items' (u = 0 when split), group g
    const int g = (S > 1) ? (int)threadIdx.x / items : 0;
    const int l0 = g * L / S, l1 = (g + 1) * L / S;
    float acc[IPB][RT][4];
#pragma unroll
    for (int u = 0; u < IPB; u++)
#pragma unroll
        for (int v = 0; v < RT; v++)
#pragma unroll
            for (int c = 0; c < 4; c++) acc[u][v][c] = 0.f;
    auto issue = [&](int k) {  // slice k into buffer k & 1, as one cp.async group
        const float *src = X + (long)k * I * J;
        float *dst = sm.slice[k & 1];
        int i = threadIdx.x % I, j = threadIdx.x / I;
        const int di = NT % I, dj = NT / I;
        for (int e = threadIdx.x; e < I * J; e += NT) {
            cp_async4(&dst[i + ld * j], src + e);
            i += di;
            j += dj;
            if (i >= I) { i -= I; j++; }
        }
        cp_async_commit();
    };
    __syncthreads();  // the previous user of the slice buffers is done
    issue(0);
    for (int k = 0; k < K; k++) {
        if (k + 1 < K) {
            issue(k + 1);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        const float *sl = sm.slice[k & 1];
#pragma unroll
        for (int u = 0; u < IPB; u++) {
            const int it = (S > 1) ? ((u == 0 && (int)threadIdx.x < S * items) ? (int)threadIdx.x % items : items)
                                   : (int)threadIdx.x + NT * u;
            if (it >= items) continue;
            const int rg = it % ngrp;
            const int rp = rg * RT;
            const int r0 = (it / ngrp) * 4;
            float t2[RT][4];
#pragma unroll
            for (int v = 0; v < RT; v++)
#pragma unroll
                for (int c = 0; c < 4; c++) t2[v][c] = 0.f;
            if (mode == 0) {
                // T[i, r] = sum_j X[i, j] B[j, r]
                const float *xp = sl + rp;
                const float *bp = sm.F[1] + J * r0;
#pragma unroll 2
                for (int j = l0; j < l1; j++) {
                    float x[RT], b[4];
#pragma unroll
                    for (int v = 0; v < RT; v++) x[v] = xp[v + ld * j];
#pragma unroll
                    for (int c = 0; c < 4; c++) b[c] = bp[j + J * c];
#pragma unroll
                    for (int v = 0; v < RT; v++)
#pragma unroll
                        for (int c = 0; c < 4; c++) t2[v][c] = fmaf(x[v], b[c], t2[v][c]);
                }
            } else {
                // T[j, r] = sum_i X[i, j] A[i, r]
                const float *xp = sl + ld * rp;
                const float *ap = sm.F[0] + I * r0;
#pragma unroll 2
                for (int i = l0; i < l1; i++) {
                    float x[RT], av[4];
#pragma unroll
                    for (int v = 0; v < RT; v++) x[v] = xp[i + ld * v];
#pragma unroll
                    for (int c = 0; c < 4; c++) av[c] = ap[i + I * c];
#pragma unroll
                    for (int v = 0; v < RT; v++)
#pragma unroll
                        for (int c = 0; c < 4; c++) t2[v][c] = fmaf(x[v], av[c], t2[v][c]);
                }
            }
            if (mode < 2) {
                const float *cp = sm.F[2] + K * r0 + k;
#pragma unroll
                for (int c = 0; c < 4; c++) {
                    const float w = cp[K * c];
#pragma unroll
                    for (int v = 0; v < RT; v++) acc[u][v][c] = fmaf(t2[v][c], w, acc[u][v][c]);
                }
            } else {
                // this row group's (and thread group's) share of M[k, r] = sum_j T[j, r] B[j, r]
                const float *Bf = sm.F[1];
#pragma unroll
                for (int c = 0; c < 4; c++) {
                    const int r = r0 + c;
                    float v = 0.f;
                    if (r < R)
#pragma unroll
                        for (int w = 0; w < RT; w++)
                            if (rp + w < J) v = fmaf(t2[w][c], Bf[rp + w + J * r], v);
                    sm.red3[(g * BMAXR + r0 + c) * NGM + rg] = v;
                }
            }
        }
        if (mode == 2) {
            // sum over groups and row groups: one warp per rank, lanes over
            // the row groups, then a fixed shuffle tree (deterministic)
            __syncthreads();
            const int lane = threadIdx.x & 31;
            for (int r = threadIdx.x >> 5; r < R; r += NT / 32) {
                float v = 0.f;
                for (int gg = 0; gg < S; gg++)
                    for (int p2 = lane; p2 < ngrp; p2 += 32) v += sm.red3[(gg * BMAXR + r) * NGM + p2];
                for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
                if (lane == 0) sm.M[k + K * r] = v;
            }
        }
        __syncthreads();  // slice k's buffer is refilled by the next issue
    }
    if (mode < 2) {
        // groups' partials added in group order: group 0 writes, the others
        // add in turn
        for (int gg = 0; gg < S; gg++) {
#pragma unroll
            for (int u = 0; u < IPB; u++) {
                const int it = (S > 1) ? ((u == 0 && (int)threadIdx.x < S * items) ? (int)threadIdx.x % items : items)
                                       : (int)threadIdx.x + NT * u;
                if (it >= items || g != gg) continue;
                const int rp = (it % ngrp) * RT;
                const int r0 = (it / ngrp) * 4;
#pragma unroll
                for (int c = 0; c < 4; c++) {
                    const int r = r0 + c;
                    if (r < R)
#pragma unroll
                        for (int v = 0; v < RT; v++)
                            if (rp + v < Q) {
                                if (gg == 0) sm.M[rp + v + Q * r] = acc[u][v][c];
                                else sm.M[rp + v + Q * r] += acc[u][v][c];
                            }
                }
            }
            __syncthreads();
        }
    }
    __syncthreads();
}

// V = Hadamard of the Grams other than `mode`; V <- V^-1 (Gauss-Jordan).
// Leaves sm.fail set when both attempts met a non-positive pivot (V is then
// not an inverse and the caller keeps the old factor).
template <int NT>
__device__ void normal_inverse_small(BatchSmem &sm, const BatchArgs &a, const TensorMeta &t, int mode) {
    const int R = t.R;
    for (int attempt = 0; attempt < 2; attempt++) {
        for (int e = threadIdx.x; e < R * R; e += NT) {
            double v = 1.0;
            for (int m = 0; m < 3; m++)
                if (m != mode) v *= t.G[m][e];
            sm.V[e] = v;
        }
        if (threadIdx.x == 0) sm.fail = 0;
        __syncthreads();
        double maxdiag = 0.0;
        for (int j = 0; j < R; j++) maxdiag = fmax(maxdiag, fabs(sm.V[j + R * j]));
        if (attempt == 1) {
            __syncthreads();
            for (int j = threadIdx.x; j < R; j += NT) sm.V[j + R * j] += 1e-10 * maxdiag + 1e-300;
            __syncthreads();
        }
        for (int k = 0; k < R; k++) {
            const double piv = sm.V[k + R * k];
            if (!(piv > 1e-14 * maxdiag) || !isfinite(piv)) {
                if (threadIdx.x == 0) sm.fail = 1;
                break;
            }
            const double inv = 1.0 / piv;
            for (int j = threadIdx.x; j < R; j += NT) {
                sm.rowk[j] = (j == k ? 1.0 : sm.V[k + R * j]) * inv;
                sm.colk[j] = sm.V[j + R * k];
            }
            __syncthreads();
            for (int e = threadIdx.x; e < R * R; e += NT) {
                const int i = e % R, j = e / R;
                const double old = (j == k) ? 0.0 : sm.V[e];
                sm.V[e] = (i == k) ? sm.rowk[j] : old - sm.colk[i] * sm.rowk[j];
            }
            __syncthreads();
        }
        __syncthreads();
        if (!sm.fail) return;
        if (threadIdx.x == 0 && attempt == 0) atomicAdd(a.fallbacks, 1);
        __syncthreads();
    }
}

template <int NT, int RT>
__global__ void __launch_bounds__(NT) k_batch_sweep(BatchArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    BatchSmem &sm = *reinterpret_cast<BatchSmem *>(smem_raw);
    for (;;) {
        if (threadIdx.x == 0) {
            unsigned w = atomicAdd(a.queue, 1u);
            sm.tensor = (w < (unsigned)a.ntensors) ? a.order[w] : -1;
        }
        __syncthreads();
        const int ti = sm.tensor;
        __syncthreads();
        if (ti < 0) return;
        TensorMeta &t = a.meta[ti];
        if (t.done) continue;
        const int R = t.R;
        load_factors<NT>(sm, a, t);
        __syncthreads();
        double inner = 0.0;
        for (int mode = 0; mode < 3; mode++) {
            mttkrp_small<NT, RT>(sm, a, t, mode);
            normal_inverse_small<NT>(sm, a, t, mode);
            // U_mode = M V^-1 (FP64 accumulation), into shared and global memory
            const int Q = t.dims[mode];
            float *Ug = a.U + t.uoff[mode];
            const bool keep = sm.fail != 0;  // singular twice: keep the old factor
            double part = 0.0;
            for (int e = threadIdx.x; e < Q * R; e += NT) {
                const int q = e % Q, c = e / Q;
                float u = sm.F[mode][e];
                if (!keep) {
                    double s = 0.0;
                    for (int r = 0; r < R; r++) s = fma((double)sm.M[q + Q * r], sm.V[r + R * c], s);
                    u = (float)s;
                    sm.F[mode][e] = u;
                    Ug[e] = u;
                }
                if (mode == 2) part += (double)sm.M[e] * (double)u;
            }
            __syncthreads();
            // Gram of the new factor
            for (int e = threadIdx.x; e < R * R; e += NT) {
                const int p = e % R, q2 = e / R;
                double s = 0.0;
                for (int i = 0; i < Q; i++) s = fma((double)sm.F[mode][i + Q * p], (double)sm.F[mode][i + Q * q2], s);
                t.G[mode][e] = s;
            }
            if (mode == 2) {
                for (int o = 16; o > 0; o >>= 1) part += __shfl_xor_sync(0xffffffffu, part, o);
                if ((threadIdx.x & 31) == 0) sm.red[threadIdx.x >> 5] = part;
            }
            __syncthreads();
            if (mode == 2 && threadIdx.x == 0) {
                for (int w = 0; w < NT / 32; w++) inner += sm.red[w];
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            double hat = 0.0;
            for (int e = 0; e < R * R; e++) hat += t.G[0][e] * t.G[1][e] * t.G[2][e];
            const double res2 = t.normx2 - 2.0 * inner + hat;
            const double fit = 1.0 - sqrt(res2 > 0.0 ? res2 : 0.0) / sqrt(t.normx2);
            t.fit_prev = t.fit;
            t.fit = fit;
            t.sweeps += 1;
            if ((a.tol > 0 && t.sweeps >= 2 && fabs(t.fit - t.fit_prev) < a.tol) || t.sweeps >= a.max_sweeps ||
                (t.target > 0.0 && t.fit >= t.target)) {
                t.done = 1;
                atomicAdd(a.ndone, 1);
            }
        }
        __syncthreads();
    }
}

// Per-tensor ||X||^2 and the initial Grams.
__global__ void __launch_bounds__(256) k_batch_setup(TensorMeta *meta, int ntensors, const float *X,
                                                     const float *U) {
    __shared__ double red[8];
    for (int ti = blockIdx.x; ti < ntensors; ti += gridDim.x) {
        TensorMeta &t = meta[ti];
        const long n = (long)t.dims[0] * t.dims[1] * t.dims[2];
        double s = 0.0;
        for (long e = threadIdx.x; e < n; e += 256) {
            const double x = X[t.xoff + e];
            s += x * x;
        }
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
        __syncthreads();
        if (threadIdx.x == 0) {
            double tot = 0.0;
            for (int w = 0; w < 8; w++) tot += red[w];
            t.normx2 = tot;
            t.fit = 0.0;
            t.fit_prev = 0.0;
            t.sweeps = 0;
            t.done = 0;
        }
        const int R = t.R;
        for (int m = 0; m < 3; m++) {
            const float *F = U + t.uoff[m];
            const int I = t.dims[m];
            for (int e = threadIdx.x; e < R * R; e += 256) {
                const int p = e % R, q = e / R;
                double g = 0.0;
                for (int i = 0; i < I; i++) g = fma((double)F[i + I * p], (double)F[i + I * q], g);
                t.G[m][e] = g;
            }
        }
        __syncthreads();
    }
}

struct BatchState {
    TensorMeta *meta = nullptr;
    int *order = nullptr;
    unsigned *queue = nullptr;
    int *fallbacks = nullptr;
};

template <int NT, int RT>
int launch_sweep(const BatchArgs &a, int ctas_per_sm, cudaStream_t s) {
    static std::atomic<bool> attr[64];  // per device; zero-initialised
    int dev = 0;
    CUD_CHECK(cudaGetDevice(&dev));
    if (dev >= 0 && dev < 64 && !attr[dev].load(std::memory_order_acquire)) {
        CUD_CHECK(cudaFuncSetAttribute(k_batch_sweep<NT, RT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)sizeof(BatchSmem)));
        attr[dev].store(true, std::memory_order_release);
    }
    CUD_CHECK(cudaMemsetAsync(a.queue, 0, sizeof(unsigned), s));
    k_batch_sweep<NT, RT><<<kNumSMs * ctas_per_sm, NT, sizeof(BatchSmem), s>>>(a);
    CUD_CHECK_LAUNCH("batched sweep");
    return CUD_OK;
}

// Launch shape: threads per CTA, CTAs per SM, rows of the MTTKRP register
// tile.
struct BatchCfg {
    int threads, ctas, rt;
};

int launch_cfg(const BatchArgs &a, const BatchCfg &c, cudaStream_t s) {
    if (c.rt == 4)
        return c.threads == 128 ? launch_sweep<128, 4>(a, c.ctas, s) : launch_sweep<256, 4>(a, c.ctas, s);
    return c.threads == 128 ? launch_sweep<128, 2>(a, c.ctas, s) : launch_sweep<256, 2>(a, c.ctas, s);
}

// Autotuner cache: shape class -> launch shape
std::mutex g_tune_mu;
std::map<long, BatchCfg> g_tune;

long shape_class(int n, const int *dims, const int *ranks) {
    // bucket the mean element count and mean rank; plus the batch size order
    double e = 0.0, r = 0.0;
    for (int t = 0; t < n; t++) {
        e += (double)dims[3 * t] * dims[3 * t + 1] * dims[3 * t + 2];
        r += ranks[t];
    }
    e /= std::max(1, n);
    r /= std::max(1, n);
    long eb = (long)log2(std::max(1.0, e)), rb = (long)r / 4, nb = (long)log2(std::max(1, n));
    return eb * 10000 + rb * 100 + nb;
}

}  // namespace

}  // namespace cud

using namespace cud;

namespace {

int batched_impl(int ntensors, const long *dims, const long *ranks, const float *X, const long *x_offsets, float *U,
                 const long *u_offsets, const cud_cp_options *opt_in, const double *targets, double *fits,
                 int *sweeps, int *kernel_launches, void *stream) {
    if (ntensors <= 0 || !dims || !ranks || !X || !x_offsets || !U || !u_offsets)
        return set_status(CUD_ERR_INVALID_ARGUMENT);
    cud_cp_options opt;
    cud_cp_default_options(&opt);
    if (opt_in) opt = *opt_in;
    if (opt.max_sweeps < 1) return set_status(CUD_ERR_INVALID_ARGUMENT);
    cudaStream_t s = as_stream(stream);
    std::vector<TensorMeta> hm(ntensors);
    std::vector<int> hd(3 * ntensors), hr(ntensors);
    std::vector<std::pair<double, int>> work(ntensors);
    for (int t = 0; t < ntensors; t++) {
        TensorMeta &m = hm[t];
        memset(&m, 0, sizeof(TensorMeta));
        for (int k = 0; k < 3; k++) {
            if (dims[3 * t + k] < 1 || dims[3 * t + k] > BMAXD) return set_status(CUD_ERR_UNSUPPORTED);
            m.dims[k] = (int)dims[3 * t + k];
            m.uoff[k] = u_offsets[3 * t + k];
            hd[3 * t + k] = m.dims[k];
        }
        if (ranks[t] < 1 || ranks[t] > BMAXR) return set_status(CUD_ERR_UNSUPPORTED);
        m.R = (int)ranks[t];
        hr[t] = m.R;
        m.xoff = x_offsets[t];
        m.target = targets ? targets[t] : 0.0;
        work[t] = {-(double)m.dims[0] * m.dims[1] * m.dims[2] * m.R, t};
    }
    std::sort(work.begin(), work.end());
    std::vector<int> order(ntensors);
    for (int t = 0; t < ntensors; t++) order[t] = work[t].second;

    int st;
    size_t bytes = sizeof(TensorMeta) * ntensors + sizeof(int) * ntensors + 256;
    char *w = (char *)scratch(kSlotTmp1, bytes, &st);
    if (!w) return set_status(st);
    BatchArgs a;
    a.meta = reinterpret_cast<TensorMeta *>(w);
    a.order = reinterpret_cast<int *>(w + sizeof(TensorMeta) * ntensors);
    a.queue = reinterpret_cast<unsigned *>(w + sizeof(TensorMeta) * ntensors + sizeof(int) * ntensors);
    a.fallbacks = reinterpret_cast<int *>(a.queue + 16);
    a.ndone = reinterpret_cast<int *>(a.queue + 32);
    a.ntensors = ntensors;
    a.X = X;
    a.U = U;
    a.max_sweeps = opt.max_sweeps;
    a.tol = opt.tol;
    CUD_CHECK(cudaMemcpyAsync(a.meta, hm.data(), sizeof(TensorMeta) * ntensors, cudaMemcpyHostToDevice, s));
    CUD_CHECK(cudaMemcpyAsync(const_cast<int *>(a.order), order.data(), sizeof(int) * ntensors,
                              cudaMemcpyHostToDevice, s));
    CUD_CHECK(cudaMemsetAsync(a.queue, 0, 256, s));
    k_batch_setup<<<std::min(ntensors, kNumSMs * 4), 256, 0, s>>>(a.meta, ntensors, X, U);
    CUD_CHECK_LAUNCH("batched setup");

    // launch shape from the autotuner (threads per CTA, CTAs per SM, tile rows)
    long key = shape_class(ntensors, hd.data(), hr.data());
    BatchCfg cfg{256, 2, 4};
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        auto it = g_tune.find(key);
        if (it != g_tune.end()) cfg = it->second;
    }
    // sweeps: graph of `per` sweeps replayed; the done-count read back between
    const int per = std::max(1, std::min(opt.check_every > 1 ? opt.check_every : 5, opt.max_sweeps));
    cudaStream_t cs = s;
    bool own = false;
    if (s == nullptr || s == cudaStreamLegacy || s == cudaStreamPerThread) {
        CUD_CHECK(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
        own = true;
        CUD_CHECK(cudaStreamSynchronize(s));
    }
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    st = CUD_OK;
    if (opt.use_graph) {
        if (cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) != cudaSuccess) st = CUD_ERR_CUDA;
        for (int i = 0; i < per && st == CUD_OK; i++) st = launch_cfg(a, cfg, cs);
        cudaError_t e = cudaStreamEndCapture(cs, &graph);
        if (st == CUD_OK && e != cudaSuccess) st = cuda_status(e, "batched capture");
        if (st == CUD_OK) {
            e = cudaGraphInstantiate(&exec, graph, 0);
            if (e != cudaSuccess) st = cuda_status(e, "batched instantiate");
        }
    }
    int launched = 0, done_sweeps = 0;
    double *hs = pinned_scalars();  // slot 63: the converged count
    int *ndone_h = hs ? reinterpret_cast<int *>(hs + 63) : nullptr;
    while (st == CUD_OK && done_sweeps < opt.max_sweeps) {
        if (exec) {
            if (cudaGraphLaunch(exec, cs) != cudaSuccess) { st = CUD_ERR_CUDA; break; }
        } else {
            for (int i = 0; i < per && st == CUD_OK; i++) st = launch_cfg(a, cfg, cs);
        }
        launched += per;
        done_sweeps += per;
        // convergence check: the count of converged tensors (4 bytes)
        if (!ndone_h || cudaMemcpyAsync(ndone_h, a.ndone, sizeof(int), cudaMemcpyDeviceToHost, cs) != cudaSuccess ||
            cudaStreamSynchronize(cs) != cudaSuccess) { st = CUD_ERR_CUDA; break; }
        if (*ndone_h >= ntensors) break;
    }
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    std::vector<TensorMeta> out;
    if (st == CUD_OK && (fits || sweeps)) {
        out.resize(ntensors);
        if (cudaMemcpyAsync(out.data(), a.meta, sizeof(TensorMeta) * ntensors, cudaMemcpyDeviceToHost, cs) != cudaSuccess ||
            cudaStreamSynchronize(cs) != cudaSuccess)
            st = CUD_ERR_CUDA;
    }
    if (st == CUD_OK) {
        for (int t = 0; t < ntensors; t++) {
            if (fits) fits[t] = out[t].fit;
            if (sweeps) sweeps[t] = out[t].sweeps;
        }
        if (kernel_launches) *kernel_launches = launched;
    }
    if (own) {
        cudaStreamSynchronize(cs);
        cudaStreamDestroy(cs);
    }
    return set_status(st);
}

}  // namespace

extern "C" int cud_cp_als_batched(int ntensors, const long *dims, const long *ranks, const float *X,
                                  const long *x_offsets, float *U, const long *u_offsets,
                                  const cud_cp_options *opt_in, double *fits, int *sweeps,
                                  int *kernel_launches, void *stream) {
    return batched_impl(ntensors, dims, ranks, X, x_offsets, U, u_offsets, opt_in, nullptr, fits, sweeps,
                        kernel_launches, stream);
}

extern "C" int cud_cp_als_batched_target(int ntensors, const long *dims, const long *ranks, const float *X,
                                         const long *x_offsets, float *U, const long *u_offsets,
                                         const cud_cp_options *opt_in, const double *target_fits, double *fits,
                                         int *sweeps, int *kernel_launches, void *stream) {
    return batched_impl(ntensors, dims, ranks, X, x_offsets, U, u_offsets, opt_in, target_fits, fits, sweeps,
                        kernel_launches, stream);
}

extern "C" int cud_cp_batched_tune(int ntensors, const long *dims, const long *ranks, const float *X,
                                   const long *x_offsets, float *U_scratch, const long *u_offsets,
                                   int *threads, int *ctas_per_sm, void *stream) {
    if (ntensors <= 0 || !dims || !ranks) return set_status(CUD_ERR_INVALID_ARGUMENT);
    std::vector<int> hd(3 * ntensors), hr(ntensors);
    for (int t = 0; t < ntensors; t++) {
        for (int k = 0; k < 3; k++) hd[3 * t + k] = (int)dims[3 * t + k];
        hr[t] = (int)ranks[t];
    }
    long key = shape_class(ntensors, hd.data(), hr.data());
    const int shapes[][2] = {{128, 2}, {128, 3}, {128, 4}, {256, 1}, {256, 2}, {256, 3}};
    std::vector<BatchCfg> cand;
    for (int rt : {2, 4})
        for (auto &sh : shapes) cand.push_back({sh[0], sh[1], rt});
    float best = 1e30f;
    BatchCfg bestc{256, 2, 4};
    cudaStream_t s = as_stream(stream);
    cudaEvent_t e0, e1;
    CUD_CHECK(cudaEventCreate(&e0));
    CUD_CHECK(cudaEventCreate(&e1));
    for (auto &c : cand) {
        {
            std::lock_guard<std::mutex> lk(g_tune_mu);
            g_tune[key] = c;
        }
        cud_cp_options opt;
        cud_cp_default_options(&opt);
        opt.max_sweeps = 2;
        opt.tol = 0.0;
        opt.use_graph = 0;
        opt.check_every = 2;
        cudaEventRecord(e0, s);
        int st = cud_cp_als_batched(ntensors, dims, ranks, X, x_offsets, U_scratch, u_offsets, &opt,
                                    nullptr, nullptr, nullptr, stream);
        cudaEventRecord(e1, s);
        cudaEventSynchronize(e1);
        if (st) { cudaEventDestroy(e0); cudaEventDestroy(e1); return set_status(st); }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) { best = ms; bestc = c; }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tune[key] = bestc;
    }
    if (threads) *threads = bestc.threads;
    if (ctas_per_sm) *ctas_per_sm = bestc.ctas;
    return set_status(CUD_OK);
}
