// Bandwidth-bound primitives: Hadamard products, Khatri-Rao, Kronecker,
// unfoldings (batched smem-tiled transposes), FP32->FP16/BF16 packing,
// subtraction/identity helpers and the fused residual norm.  Every result is
// bit-exact with the reference's one-rounding definitions.
#include "common.cuh"

namespace cud {

// ---------------------------------------------------------------------------
// Element-wise products.  128-bit vector path when every pointer is 16-byte
// aligned; grid-stride loops sized to a few waves of the 148 SMs.
// ---------------------------------------------------------------------------

__global__ void k_mul2(const float *__restrict__ A, const float *__restrict__ B,
                       float *__restrict__ C, long n, int vec) {
    long tid = blockIdx.x * (long)blockDim.x + threadIdx.x;
    long stride = (long)gridDim.x * blockDim.x;
    if (vec) {
        long n4 = n >> 2;
        const float4 *a4 = reinterpret_cast<const float4 *>(A);
        const float4 *b4 = reinterpret_cast<const float4 *>(B);
        float4 *c4 = reinterpret_cast<float4 *>(C);
        for (long i = tid; i < n4; i += stride) {
            float4 x = __ldcs(a4 + i), y = __ldcs(b4 + i);
            float4 z;
            z.x = __fmul_rn(x.x, y.x); z.y = __fmul_rn(x.y, y.y);
            z.z = __fmul_rn(x.z, y.z); z.w = __fmul_rn(x.w, y.w);
            __stcs(c4 + i, z);
        }
        for (long i = (n4 << 2) + tid; i < n; i += stride) C[i] = __fmul_rn(A[i], B[i]);
    } else {
        for (long i = tid; i < n; i += stride) C[i] = __fmul_rn(A[i], B[i]);
    }
}

__global__ void k_mul3(const float *__restrict__ A, const float *__restrict__ B,
                       const float *__restrict__ K, float *__restrict__ D, long n, int vec) {
    long tid = blockIdx.x * (long)blockDim.x + threadIdx.x;
    long stride = (long)gridDim.x * blockDim.x;
    if (vec) {
        long n4 = n >> 2;
        const float4 *a4 = reinterpret_cast<const float4 *>(A);
        const float4 *b4 = reinterpret_cast<const float4 *>(B);
        const float4 *k4 = reinterpret_cast<const float4 *>(K);
        float4 *d4 = reinterpret_cast<float4 *>(D);
        for (long i = tid; i < n4; i += stride) {
            float4 x = __ldcs(a4 + i), y = __ldcs(b4 + i), z = __ldcs(k4 + i), o;
            o.x = __fmul_rn(__fmul_rn(x.x, y.x), z.x);
            o.y = __fmul_rn(__fmul_rn(x.y, y.y), z.y);
            o.z = __fmul_rn(__fmul_rn(x.z, y.z), z.z);
            o.w = __fmul_rn(__fmul_rn(x.w, y.w), z.w);
            __stcs(d4 + i, o);
        }
        for (long i = (n4 << 2) + tid; i < n; i += stride)
            D[i] = __fmul_rn(__fmul_rn(A[i], B[i]), K[i]);
    } else {
        for (long i = tid; i < n; i += stride) D[i] = __fmul_rn(__fmul_rn(A[i], B[i]), K[i]);
    }
}

__global__ void k_sub_into(const float *__restrict__ M, float *__restrict__ N, long n) {
    long tid = blockIdx.x * (long)blockDim.x + threadIdx.x;
    long stride = (long)gridDim.x * blockDim.x;
    for (long i = tid; i < n; i += stride) N[i] = __fsub_rn(M[i], N[i]);
}

__global__ void k_identity(float *A, long m) {
    long tid = blockIdx.x * (long)blockDim.x + threadIdx.x;
    long stride = (long)gridDim.x * blockDim.x;
    for (long i = tid; i < m * m; i += stride) A[i] = (i % m == i / m) ? 1.0f : 0.0f;
}

static inline bool aligned16(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

// ---------------------------------------------------------------------------
// Khatri-Rao and Kronecker: each output column is the Kronecker product of two
// input columns, second operand fastest.  One thread per output element; the
// write stream is coalesced, the (tiny) inputs come from L1/L2.
// ---------------------------------------------------------------------------

// out[x + y*b + t*a*b] = B[x + t*ldb] * A[y + t*lda]  (src/kr.cu:9)
__global__ void k_khatri_rao(const float *__restrict__ A, const float *__restrict__ B,
                             float *__restrict__ out, long a, long b, long r) {
    long n = a * b * r;
    long tid = blockIdx.x * (long)blockDim.x + threadIdx.x;
    long stride = (long)gridDim.x * blockDim.x;
    for (long e = tid; e < n; e += stride) {
        long x = e % b;
        long rest = e / b;
        long y = rest % a;
        long t = rest / a;
        out[e] = __fmul_rn(B[x + t * b], A[y + t * a]);
    }
}

// C[(x + c*y) + a*c*(t + d*i)] = A[y + a*i] * B[x + c*t]  (src/tensorproduct.cu:9-11)
__global__ void k_kron(const float *__restrict__ A, const float *__restrict__ B,
                       float *__restrict__ C, long a, long b, long c, long d) {
    long rows = a * c;
    long n = rows * b * d;
    long tid = blockIdx.x * (long)blockDim.x + threadIdx.x;
    long stride = (long)gridDim.x * blockDim.x;
    for (long e = tid; e < n; e += stride) {
        long row = e % rows, col = e / rows;
        long x = row % c, y = row / c;
        long t = col % d, i = col / d;
        C[e] = __fmul_rn(A[y + a * i], B[x + c * t]);
    }
}

// ---------------------------------------------------------------------------
// Batched transpose: in is `batch` column-major rows x cols matrices (stride
// rows*cols), out the cols x rows transposes.  32x32 tiles through padded
// shared memory so both the read and the write are coalesced.
// ---------------------------------------------------------------------------

__global__ void __launch_bounds__(256) k_transpose(const float *__restrict__ in,
                                                   float *__restrict__ out, long rows,
                                                   long cols, long batch) {
    __shared__ float tile[32][33];
    long tr = (rows + 31) / 32, tc = (cols + 31) / 32;
    long ntiles = tr * tc * batch;
    int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;  // 32 x 8
    for (long t = blockIdx.x; t < ntiles; t += gridDim.x) {
        long bidx = t / (tr * tc);
        long rem = t % (tr * tc);
        long r0 = (rem % tr) * 32, c0 = (rem / tr) * 32;
        const float *src = in + bidx * rows * cols;
        float *dst = out + bidx * rows * cols;
        for (int j = ty; j < 32; j += 8) {
            long r = r0 + tx, c = c0 + j;
            if (r < rows && c < cols) tile[j][tx] = src[r + rows * c];
        }
        __syncthreads();
        for (int j = ty; j < 32; j += 8) {
            long c = c0 + tx, r = r0 + j;  // out[c + cols*r]
            if (r < rows && c < cols) dst[c + cols * r] = tile[tx][j];
        }
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// Packing to 16-bit formats (round to nearest even).
// ---------------------------------------------------------------------------

__global__ void k_to_half(const float *__restrict__ A, __half *__restrict__ B, long n) {
    long tid = blockIdx.x * (long)blockDim.x + threadIdx.x;
    long stride = (long)gridDim.x * blockDim.x;
    for (long i = tid; i < n; i += stride) B[i] = __float2half_rn(A[i]);
}

__global__ void k_to_bf16(const float *__restrict__ A, __nv_bfloat16 *__restrict__ B, long n) {
    long tid = blockIdx.x * (long)blockDim.x + threadIdx.x;
    long stride = (long)gridDim.x * blockDim.x;
    for (long i = tid; i < n; i += stride) B[i] = __float2bfloat16_rn(A[i]);
}

// ---------------------------------------------------------------------------
// Fused residual: X1 <- X - X1 and the two sums of squares in FP64, written
// as per-block partials, then reduced in fixed order (deterministic).
// ---------------------------------------------------------------------------

template <int NT>
__device__ __forceinline__ double block_sum(double v, double *sh) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    __syncthreads();
    if (l == 0) sh[w] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (int i = 0; i < NT / 32; i++) s += sh[i];
    return s;
}

__global__ void __launch_bounds__(256) k_residual_partials(const float *__restrict__ X,
                                                           float *__restrict__ X1, long n,
                                                           int subtract,
                                                           double *__restrict__ part) {
    __shared__ double sh[8];
    long tid = blockIdx.x * (long)blockDim.x + threadIdx.x;
    long stride = (long)gridDim.x * blockDim.x;
    double s1 = 0.0, s2 = 0.0;
    for (long i = tid; i < n; i += stride) {
        float x = X[i];
        s2 += (double)x * x;
        if (subtract) {
            float d = __fsub_rn(x, X1[i]);
            X1[i] = d;
            s1 += (double)d * d;
        }
    }
    double t1 = block_sum<256>(s1, sh);
    double t2 = block_sum<256>(s2, sh);
    if (threadIdx.x == 0) {
        part[2 * blockIdx.x] = t1;
        part[2 * blockIdx.x + 1] = t2;
    }
}

__global__ void k_reduce_partials(const double *__restrict__ part, int nparts,
                                  double *__restrict__ out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int i = 0; i < nparts; i++) {
            a += part[2 * i];
            b += part[2 * i + 1];
        }
        out[0] = a;
        out[1] = b;
    }
}

// Sums of squares of X (and of X - X1 after writing it into X1 when subtract
// is set) into host out[0..1].  Synchronises the stream.
int residual_norms(const float *X, float *X1, long n, int subtract, double *out, cudaStream_t s) {
    const int nparts = 148 * 4;
    int st;
    double *part = (double *)scratch(kSlotReduce, sizeof(double) * (2 * nparts + 2), &st);
    if (!part) return st;
    k_residual_partials<<<nparts, 256, 0, s>>>(X, X1, n, subtract, part);
    k_reduce_partials<<<1, 32, 0, s>>>(part, nparts, part + 2 * nparts);
    CUD_CHECK_LAUNCH("residual_norms");
    CUD_CHECK(cudaMemcpyAsync(out, part + 2 * nparts, 2 * sizeof(double), cudaMemcpyDeviceToHost, s));
    CUD_CHECK(cudaStreamSynchronize(s));
    return CUD_OK;
}

}  // namespace cud

using namespace cud;

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------

extern "C" int cud_hadmard(const float *A, const float *B, float *C, long a, long b, void *stream) {
    if (a < 0 || b < 0 || (a * b > 0 && (!A || !B || !C))) return set_status(CUD_ERR_INVALID_ARGUMENT);
    long n = a * b;
    if (n == 0) return set_status(CUD_OK);
    int vec = aligned16(A) && aligned16(B) && aligned16(C);
    k_mul2<<<blocks_for(vec ? n / 4 : n, 256), 256, 0, as_stream(stream)>>>(A, B, C, n, vec);
    CUD_CHECK_LAUNCH("cud_hadmard");
    return set_status(CUD_OK);
}

extern "C" int cud_hadmard3(const float *A, const float *B, const float *C, float *D, long a,
                            long b, void *stream) {
    if (a < 0 || b < 0 || (a * b > 0 && (!A || !B || !C || !D))) return set_status(CUD_ERR_INVALID_ARGUMENT);
    long n = a * b;
    if (n == 0) return set_status(CUD_OK);
    int vec = aligned16(A) && aligned16(B) && aligned16(C) && aligned16(D);
    k_mul3<<<blocks_for(vec ? n / 4 : n, 256), 256, 0, as_stream(stream)>>>(A, B, C, D, n, vec);
    CUD_CHECK_LAUNCH("cud_hadmard3");
    return set_status(CUD_OK);
}

extern "C" int cud_elepro3(const float *A, const float *B, const float *C, float *D, long n,
                           void *stream) {
    return cud_hadmard3(A, B, C, D, n, 1, stream);
}

extern "C" int cud_tminust(const float *M, float *N, long m, void *stream) {
    if (m < 0 || (m > 0 && (!M || !N))) return set_status(CUD_ERR_INVALID_ARGUMENT);
    if (m == 0) return set_status(CUD_OK);
    k_sub_into<<<blocks_for(m, 256), 256, 0, as_stream(stream)>>>(M, N, m);
    CUD_CHECK_LAUNCH("cud_tminust");
    return set_status(CUD_OK);
}

extern "C" int cud_init_identity(float *A, long m, void *stream) {
    if (m < 0 || (m > 0 && !A)) return set_status(CUD_ERR_INVALID_ARGUMENT);
    if (m == 0) return set_status(CUD_OK);
    k_identity<<<blocks_for(m * m, 256), 256, 0, as_stream(stream)>>>(A, m);
    CUD_CHECK_LAUNCH("cud_init_identity");
    return set_status(CUD_OK);
}

extern "C" int cud_kr(const float *A, const float *B, float *AkrB, long a, long b, long r,
                      void *stream) {
    if (a < 0 || b < 0 || r < 0) return set_status(CUD_ERR_INVALID_ARGUMENT);
    long n = a * b * r;
    if (n == 0) return set_status(CUD_OK);
    if (!A || !B || !AkrB) return set_status(CUD_ERR_INVALID_ARGUMENT);
    k_khatri_rao<<<blocks_for(n, 256), 256, 0, as_stream(stream)>>>(A, B, AkrB, a, b, r);
    CUD_CHECK_LAUNCH("cud_kr");
    return set_status(CUD_OK);
}

extern "C" int cud_tensor_product(const float *A, const float *B, float *C, long a, long b,
                                  long c, long d, void *stream) {
    if (a < 0 || b < 0 || c < 0 || d < 0) return set_status(CUD_ERR_INVALID_ARGUMENT);
    long n = a * b * c * d;
    if (n == 0) return set_status(CUD_OK);
    if (!A || !B || !C) return set_status(CUD_ERR_INVALID_ARGUMENT);
    k_kron<<<blocks_for(n, 256), 256, 0, as_stream(stream)>>>(A, B, C, a, b, c, d);
    CUD_CHECK_LAUNCH("cud_tensor_product");
    return set_status(CUD_OK);
}

extern "C" int cud_f2h(const float *A, void *B, long n, void *stream) {
    if (n < 0 || (n > 0 && (!A || !B))) return set_status(CUD_ERR_INVALID_ARGUMENT);
    if (n == 0) return set_status(CUD_OK);
    k_to_half<<<blocks_for(n, 256), 256, 0, as_stream(stream)>>>(A, (__half *)B, n);
    CUD_CHECK_LAUNCH("cud_f2h");
    return set_status(CUD_OK);
}

extern "C" int cud_f2bf(const float *A, void *B, long n, void *stream) {
    if (n < 0 || (n > 0 && (!A || !B))) return set_status(CUD_ERR_INVALID_ARGUMENT);
    if (n == 0) return set_status(CUD_OK);
    k_to_bf16<<<blocks_for(n, 256), 256, 0, as_stream(stream)>>>(A, (__nv_bfloat16 *)B, n);
    CUD_CHECK_LAUNCH("cud_f2bf");
    return set_status(CUD_OK);
}

extern "C" int cud_t2m(const float *T1, float *T2, long flag, long m, long n, long k,
                       void *stream) {
    if (flag < 1 || flag > 3 || m < 0 || n < 0 || k < 0) return set_status(CUD_ERR_INVALID_ARGUMENT);
    long total = m * n * k;
    if (total == 0) return set_status(CUD_OK);
    if (!T1 || !T2) return set_status(CUD_ERR_INVALID_ARGUMENT);
    cudaStream_t s = as_stream(stream);
    if (flag == 1) {
        CUD_CHECK(cudaMemcpyAsync(T2, T1, sizeof(float) * total, cudaMemcpyDeviceToDevice, s));
    } else {
        long rows = flag == 2 ? m : m * n, cols = flag == 2 ? n : k, batch = flag == 2 ? k : 1;
        long tiles = ((rows + 31) / 32) * ((cols + 31) / 32) * batch;
        unsigned grid = (unsigned)(tiles < 148L * 32 ? tiles : 148L * 32);
        k_transpose<<<grid, 256, 0, s>>>(T1, T2, rows, cols, batch);
        CUD_CHECK_LAUNCH("cud_t2m");
    }
    return set_status(CUD_OK);
}

extern "C" int cud_rse(const float *X, float *X1, long n, float *err, void *stream) {
    if (n < 0 || !err || (n > 0 && (!X || !X1))) return set_status(CUD_ERR_INVALID_ARGUMENT);
    if (n == 0) { *err = 0.0f; return set_status(CUD_OK); }
    double out[2];
    int st = residual_norms(X, X1, n, 1, out, as_stream(stream));
    if (st != CUD_OK) return set_status(st);
    *err = (float)(sqrt(out[0]) / sqrt(out[1]));
    return set_status(CUD_OK);
}

extern "C" int cud_norm2(const float *x, long n, double *out, void *stream) {
    if (n < 0 || !out || (n > 0 && !x)) return set_status(CUD_ERR_INVALID_ARGUMENT);
    if (n == 0) { *out = 0.0; return set_status(CUD_OK); }
    double o[2];
    int st = residual_norms(x, nullptr, n, 0, o, as_stream(stream));
    if (st != CUD_OK) return set_status(st);
    *out = o[1];
    return set_status(CUD_OK);
}

// ---------------------------------------------------------------------------
// The reference's exported kernels (inc/cudecompose.h), one thread per element.
// ---------------------------------------------------------------------------

__global__ void hardm(float *M, float *N, float *res, long m, long n) {
    long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i < m * n) res[i] = __fmul_rn(M[i], N[i]);
}

__global__ void hardm3(float *M, float *N, float *K, float *res, long m, long n) {
    long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i < m * n) res[i] = __fmul_rn(__fmul_rn(M[i], N[i]), K[i]);
}

__global__ void floattohalf(float *AA, half *BB, long m) {
    long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i < m) BB[i] = __float2half_rn(AA[i]);
}

__global__ void tensorTomat1(float *T1, float *T2, long m, long n, long k) {
    long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i < m * n * k) T2[i] = T1[i];
}

__global__ void tensorTomat2(float *T1, float *T2, long m, long n, long k) {
    long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i < m * n * k) {
        long tube = i / (m * n), rem = i - tube * m * n;
        long row = rem % m, col = rem / m;
        T2[tube * m * n + row * n + col] = T1[i];
    }
}

__global__ void tensorTomat3(float *T1, float *T2, long m, long n, long k) {
    long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i < m * n * k) {
        long tube = i / (m * n), rem = i - tube * m * n;
        T2[k * rem + tube] = T1[i];
    }
}

__global__ void t_t(float *M, float *N, long m) {
    long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i < m) N[i] = __fsub_rn(M[i], N[i]);
}

__global__ void elemin(float *A, float *B, long n) {
    long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i < n) B[i] = __fsub_rn(A[i], B[i]);
}

__global__ void initIdeMat(float *AA, long m) {
    long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i < m * m) AA[i] = (i % m == i / m) ? 1.0f : 0.0f;
}

__global__ void initIdeMat(float *AA, int m) {
    long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i < (long)m * m) AA[i] = (i % m == i / m) ? 1.0f : 0.0f;
}

__global__ void elepro3(float *AA, float *BB, float *CC, float *DD, int m) {
    long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (i < m) DD[i] = __fmul_rn(__fmul_rn(AA[i], BB[i]), CC[i]);
}
