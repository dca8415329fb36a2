// Strided GEMM on CUDA cores: the workhorse for the Tucker side (mode
// products, unfolding Grams, reconstructions).  64x64 output tile per CTA,
// 16-deep contraction slices staged through shared memory, 4x4 register tile
// per thread; optional split of the contraction with an FP64 reduction.
// The same kernels run on FP32 and FP64 operands (the FP64 Tucker path).
#include "kernels.cuh"

namespace cud {

namespace {

constexpr int BM = 64, BN = 64, BK = 16, NT = 256;

struct Kidx {
    long kin, kout;
};

__device__ __forceinline__ Kidx split_k(long kappa, long Kin, bool two_level) {
    if (!two_level) return {kappa, 0};
    return {kappa % Kin, kappa / Kin};
}

__device__ __forceinline__ float fma_t(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double fma_t(double a, double b, double c) { return fma(a, b, c); }
__device__ __forceinline__ void load4(const float *p, float *x) {
    const float4 v = *reinterpret_cast<const float4 *>(p);
    x[0] = v.x; x[1] = v.y; x[2] = v.z; x[3] = v.w;
}
__device__ __forceinline__ void load4(const double *p, double *x) {
    const double2 a = *reinterpret_cast<const double2 *>(p), b = *reinterpret_cast<const double2 *>(p + 2);
    x[0] = a.x; x[1] = a.y; x[2] = b.x; x[3] = b.y;
}

template <bool kTwoLevel, typename T>
__global__ void __launch_bounds__(NT) k_gemm(GemmDescT<T> d, long kchunk, T *part) {
    __shared__ __align__(16) T As[BK][BM];
    __shared__ __align__(16) T Bs[BK][BN];
    const int t = threadIdx.x;
    const long m_tiles = (d.M + BM - 1) / BM;
    const long m0 = (blockIdx.x % m_tiles) * BM;
    const long n0 = (blockIdx.x / m_tiles) * BN;
    const long b = blockIdx.y;
    const int z = blockIdx.z;
    const long K = d.Kin * d.Kout;
    const long kbeg = (long)z * kchunk;
    const long kend = min(K, kbeg + kchunk);

    const T *A = d.A + b * d.a_b;
    const T *B = d.B + b * d.b_b;
    const bool a_mfast = (d.a_m == 1);
    const bool b_nfast = (d.b_n == 1) && (d.b_kin != 1);

    const int tx = t & 15, ty = t >> 4;
    T acc[4][4];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j] = 0;

    for (long k0 = kbeg; k0 < kend; k0 += BK) {
#pragma unroll
        for (int i = 0; i < 4; i++) {
            int e = t + NT * i;
            int mm, kk;
            if (a_mfast) { mm = e % BM; kk = e / BM; }
            else { kk = e % BK; mm = e / BK; }
            long m = m0 + mm, kap = k0 + kk;
            T v = 0;
            if (m < d.M && kap < kend) {
                Kidx ki = split_k(kap, d.Kin, kTwoLevel);
                v = A[m * d.a_m + ki.kin * d.a_kin + ki.kout * d.a_kout];
            }
            As[kk][mm] = v;
        }
#pragma unroll
        for (int i = 0; i < 4; i++) {
            int e = t + NT * i;
            int nn, kk;
            if (b_nfast) { nn = e % BN; kk = e / BN; }
            else { kk = e % BK; nn = e / BK; }
            long n = n0 + nn, kap = k0 + kk;
            T v = 0;
            if (n < d.N && kap < kend) {
                Kidx ki = split_k(kap, d.Kin, kTwoLevel);
                v = B[ki.kin * d.b_kin + ki.kout * d.b_kout + n * d.b_n];
            }
            Bs[kk][nn] = v;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < BK; kk++) {
            T av[4], bv[4];
            load4(&As[kk][tx * 4], av);
            load4(&Bs[kk][ty * 4], bv);
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) acc[i][j] = fma_t(av[i], bv[j], acc[i][j]);
        }
        __syncthreads();
    }

    if (part) {
        // partial[z][b][n][m] dense M x N
        T *P = part + ((long)z * d.batch + b) * d.M * d.N;
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
            for (int j = 0; j < 4; j++) {
                long m = m0 + tx * 4 + i, n = n0 + ty * 4 + j;
                if (m < d.M && n < d.N) P[m + d.M * n] = acc[i][j];
            }
    } else {
        T *C = static_cast<T *>(d.C) + b * d.c_b;
#pragma unroll
        for (int i = 0; i < 4; i++)
#pragma unroll
            for (int j = 0; j < 4; j++) {
                long m = m0 + tx * 4 + i, n = n0 + ty * 4 + j;
                if (m < d.M && n < d.N) {
                    T *c = C + m * d.c_m + n * d.c_n;
                    T v = d.alpha * acc[i][j];
                    if (d.beta != T(0)) v = fma_t(d.beta, *c, v);
                    *c = v;
                }
            }
    }
}

template <typename T>
__global__ void k_gemm_reduce(GemmDescT<T> d, int splits, const T *__restrict__ part) {
    long MN = d.M * d.N;
    long total = MN * d.batch;
    long tid = blockIdx.x * (long)blockDim.x + threadIdx.x;
    long stride = (long)gridDim.x * blockDim.x;
    for (long e = tid; e < total; e += stride) {
        long b = e / MN, mn = e % MN;
        long m = mn % d.M, n = mn / d.M;
        double s = 0.0;
        for (int z = 0; z < splits; z++) s += (double)part[((long)z * d.batch + b) * MN + mn];
        s *= (double)d.alpha;
        long off = b * d.c_b + m * d.c_m + n * d.c_n;
        if (d.out_f64) {
            double *C = static_cast<double *>(d.C);
            C[off] = (d.beta != T(0)) ? s + (double)d.beta * C[off] : s;
        } else {
            T *C = static_cast<T *>(d.C);
            C[off] = (T)((d.beta != T(0)) ? s + (double)d.beta * C[off] : s);
        }
    }
}

}  // namespace

template <typename T>
int gemm_simt_impl(const GemmDescT<T> &d0, cudaStream_t s) {
    GemmDescT<T> d = d0;
    if (d.M <= 0 || d.N <= 0 || d.batch <= 0) return CUD_OK;
    long K = d.Kin * d.Kout;
    long tiles = ((d.M + BM - 1) / BM) * ((d.N + BN - 1) / BN);
    if (tiles * d.batch > 0x7fffffffL || d.batch > 65535) return CUD_ERR_UNSUPPORTED;
    int splits = d.splits;
    if (splits <= 0) {
        long want = (2L * kNumSMs + tiles * d.batch - 1) / (tiles * d.batch);
        long maxs = (K + 8 * BK - 1) / (8 * BK);
        splits = (int)std::max(1L, std::min(std::min(want, maxs), 64L));
    }
    if (d.out_f64 && splits < 1) splits = 1;
    long kchunk = (K + splits - 1) / splits;
    kchunk = (kchunk + BK - 1) / BK * BK;
    if (kchunk == 0) kchunk = BK;
    splits = (int)((K + kchunk - 1) / kchunk);
    if (splits < 1) splits = 1;
    bool need_part = d.out_f64 || splits > 1;
    T *part = nullptr;
    if (need_part) {
        int st;
        part = (T *)scratch(kSlotTmp2, sizeof(T) * (size_t)splits * d.batch * d.M * d.N, &st);
        if (!part) return st;
    }
    if (K == 0) {
        // alpha * 0 + beta * C
        splits = 1;
        if (!need_part) {
            int st;
            part = (T *)scratch(kSlotTmp2, sizeof(T) * (size_t)d.batch * d.M * d.N, &st);
            if (!part) return st;
        }
        CUD_CHECK(cudaMemsetAsync(part, 0, sizeof(T) * (size_t)d.batch * d.M * d.N, s));
        k_gemm_reduce<T><<<blocks_for(d.M * d.N * d.batch, 256), 256, 0, s>>>(d, 1, part);
        CUD_CHECK_LAUNCH("gemm_simt(K=0)");
        return CUD_OK;
    }
    dim3 grid((unsigned)tiles, (unsigned)d.batch, (unsigned)splits);
    if (d.Kout > 1)
        k_gemm<true, T><<<grid, NT, 0, s>>>(d, kchunk, need_part ? part : nullptr);
    else
        k_gemm<false, T><<<grid, NT, 0, s>>>(d, kchunk, need_part ? part : nullptr);
    CUD_CHECK_LAUNCH("gemm_simt");
    if (need_part) {
        k_gemm_reduce<T><<<blocks_for(d.M * d.N * d.batch, 256), 256, 0, s>>>(d, splits, part);
        CUD_CHECK_LAUNCH("gemm_simt reduce");
    }
    return CUD_OK;
}

int gemm_simt(const GemmDesc &d, cudaStream_t s) { return gemm_simt_impl<float>(d, s); }

int gemm_simt_f64(const GemmDesc64 &d, cudaStream_t s) {
    if (d.out_f64) return CUD_ERR_INVALID_ARGUMENT;  // FP64 output is the plain path here
    return gemm_simt_impl<double>(d, s);
}

}  // namespace cud
