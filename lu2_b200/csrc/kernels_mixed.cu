// kernels_mixed.cu -- support kernels of the precision form: the FP32 updates
// inside the panel recursion, the per-panel power-of-two scales of the BF16
// operands, FP64 <-> FP32 conversions, the FP64 residual of the iterative
// refinement and the per-panel update of the FP32 forward solve.
#include <cuda_bf16.h>

#include "lu2gpu_internal.cuh"

namespace lu2gpu {

// ---------------------------------------------------------------------------
// C -= A Bt^T in FP32 on the CUDA cores (exact FP32 arithmetic for the panel,
// which the precision form keeps in FP32).  64 x 64 tiles, 256 threads of 4 x 4.
constexpr int SG_T = 64, SG_K = 32;

__global__ void __launch_bounds__(256) sgemm_update_kernel(const float *__restrict__ a, long lda,
                                                           const float *__restrict__ bt, float *c, long ldc, int M,
                                                           int N, int K)
{
    __shared__ float As[SG_K][SG_T + 4];
    __shared__ float Bs[SG_K][SG_T + 4];
    const int m0 = blockIdx.x * SG_T, n0 = blockIdx.y * SG_T;
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    float acc[4][4] = {};
    for (int k0 = 0; k0 < K; k0 += SG_K) {
        for (int idx = threadIdx.x; idx < SG_T * SG_K; idx += 256) {
            const int r = idx / SG_K, k = idx - r * SG_K;
            const int gk = k0 + k;
            As[k][r] = (m0 + r < M && gk < K) ? a[(size_t)(m0 + r) * lda + gk] : 0.f;
            Bs[k][r] = (n0 + r < N && gk < K) ? bt[(size_t)(n0 + r) * K + gk] : 0.f;
        }
        __syncthreads();
#pragma unroll 8
        for (int k = 0; k < SG_K; k++) {
            float av[4], bv[4];
#pragma unroll
            for (int i = 0; i < 4; i++) {
                av[i] = As[k][ty * 4 + i];
                bv[i] = Bs[k][tx * 4 + i];
            }
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) acc[i][j] = fmaf(av[i], bv[j], acc[i][j]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; i++) {
        const int m = m0 + ty * 4 + i;
        if (m >= M) continue;
#pragma unroll
        for (int j = 0; j < 4; j++) {
            const int n = n0 + tx * 4 + j;
            if (n < N) c[(size_t)m * ldc + n] -= acc[i][j];
        }
    }
}

cudaError_t launch_sgemm_update(const float *a, long lda, const float *bt, float *c, long ldc, int M, int N, int K,
                                cudaStream_t st)
{
    if (M <= 0 || N <= 0 || K <= 0) return cudaSuccess;
    dim3 grid((M + SG_T - 1) / SG_T, (N + SG_T - 1) / SG_T);
    if (grid.y > 65535) return cudaErrorInvalidConfiguration;
    count_launch();
    sgemm_update_kernel<<<grid, 256, 0, st>>>(a, lda, bt, c, ldc, M, N, K);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// per-panel power-of-two scales

// amax_bits = max(amax_bits, max |x|) (non-negative floats order as their bits)
__global__ void absmax_kernel(const float *__restrict__ x, long ld, int rows, int cols, unsigned *amax_bits)
{
    float m = 0.f;
    const long total = (long)rows * cols;
    for (long idx = (long)blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += (long)gridDim.x * blockDim.x) {
        const long r = idx / cols, c = idx - r * cols;
        m = fmaxf(m, fabsf(x[r * ld + c]));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(amax_bits, __float_as_uint(m));
}

cudaError_t launch_absmax(const float *x, long ld, int rows, int cols, unsigned *amax_bits, cudaStream_t st)
{
    if (rows <= 0 || cols <= 0) return cudaSuccess;
    long blocks = ((long)rows * cols + 255) / 256;
    if (blocks > 148 * 8) blocks = 148 * 8;
    count_launch();
    absmax_kernel<<<(unsigned)blocks, 256, 0, st>>>(x, ld, rows, cols, amax_bits);
    return cudaGetLastError();
}

// scales[0] = 1/sL, scales[1] = 1/sU, scales[2] = sL*sU for the two maxima in
// amax_bits[0..1]; sX = 2^e with max|X| <= 2^e (1 for an all-zero block).
__global__ void panel_scales_kernel(const unsigned *amax_bits, float *scales)
{
    float s[2];
    for (int i = 0; i < 2; i++) {
        const float m = __uint_as_float(amax_bits[i]);
        int e = 0;
        if (m > 0.f && isfinite(m)) frexpf(m, &e);
        s[i] = ldexpf(1.f, e);
    }
    scales[0] = 1.f / s[0];
    scales[1] = 1.f / s[1];
    scales[2] = s[0] * s[1];
}

cudaError_t launch_panel_scales(const unsigned *amax_bits, float *scales, cudaStream_t st)
{
    count_launch();
    panel_scales_kernel<<<1, 1, 0, st>>>(amax_bits, scales);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// conversions

__global__ void f64_to_f32_kernel(const double *__restrict__ x, long ldx, float *__restrict__ y, long ldy, int rows,
                                  int cols)
{
    const long total = (long)rows * cols;
    for (long idx = (long)blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += (long)gridDim.x * blockDim.x) {
        const long r = idx / cols, c = idx - r * cols;
        y[r * ldy + c] = (float)x[r * ldx + c];
    }
}

__global__ void f32_to_f64_kernel(const float *__restrict__ x, long ldx, double *__restrict__ y, long ldy, int rows,
                                  int cols)
{
    const long total = (long)rows * cols;
    for (long idx = (long)blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += (long)gridDim.x * blockDim.x) {
        const long r = idx / cols, c = idx - r * cols;
        y[r * ldy + c] = (double)x[r * ldx + c];
    }
}

static unsigned grid_for(long total)
{
    long b = (total + 255) / 256;
    if (b > 148 * 32) b = 148 * 32;
    return (unsigned)(b > 0 ? b : 1);
}

cudaError_t launch_f64_to_f32(const double *x, long ldx, float *y, long ldy, int rows, int cols, cudaStream_t st)
{
    if (rows <= 0 || cols <= 0) return cudaSuccess;
    count_launch();
    f64_to_f32_kernel<<<grid_for((long)rows * cols), 256, 0, st>>>(x, ldx, y, ldy, rows, cols);
    return cudaGetLastError();
}

cudaError_t launch_f32_to_f64(const float *x, long ldx, double *y, long ldy, int rows, int cols, cudaStream_t st)
{
    if (rows <= 0 || cols <= 0) return cudaSuccess;
    count_launch();
    f32_to_f64_kernel<<<grid_for((long)rows * cols), 256, 0, st>>>(x, ldx, y, ldy, rows, cols);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// r = b - A x in FP64, one warp per row (the refinement's residual; reads A once)
__global__ void __launch_bounds__(256) residual_kernel(const double *__restrict__ a, long lda, int n,
                                                       const double *__restrict__ b, const double *__restrict__ x,
                                                       double *__restrict__ r, double *__restrict__ rowabs)
{
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int i = blockIdx.x * 8 + warp; i < n; i += gridDim.x * 8) {
        const double *row = a + (size_t)i * lda;
        double s = 0.0, sa = 0.0;
        for (int j = lane * 2; j < n; j += 64) {
            if (j + 1 < n) {
                const double2 v = __ldcs(reinterpret_cast<const double2 *>(row + j));
                s = fma(v.x, x[j], s);
                s = fma(v.y, x[j + 1], s);
                sa += fabs(v.x) + fabs(v.y);
            } else {
                const double v = __ldcs(row + j);
                s = fma(v, x[j], s);
                sa += fabs(v);
            }
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            s += __shfl_xor_sync(0xffffffffu, s, o);
            sa += __shfl_xor_sync(0xffffffffu, sa, o);
        }
        if (lane == 0) {
            r[i] = b ? b[i] - s : s;  // without b: the product A x
            if (rowabs) rowabs[i] = sa;
        }
    }
}

cudaError_t launch_residual(const double *a, long lda, int n, const double *b, const double *x, double *r,
                            double *rowabs, cudaStream_t st)
{
    if (n <= 0) return cudaSuccess;
    if ((lda & 1) || (reinterpret_cast<uintptr_t>(a) & 15)) return cudaErrorInvalidValue;
    int blocks = (n + 7) / 8;
    if (blocks > 148 * 16) blocks = 148 * 16;
    count_launch();
    residual_kernel<<<blocks, 256, 0, st>>>(a, lda, n, b, x, r, rowabs);
    return cudaGetLastError();
}

// y[i] -= sum_k l[i][k] v[k] for i < rows, K <= 512 (one warp per row)
__global__ void __launch_bounds__(256) gemv_sub_kernel(const float *__restrict__ l, long ld, int rows, int K,
                                                       const float *__restrict__ v, float *__restrict__ y)
{
    __shared__ float vs[512];
    for (int k = threadIdx.x; k < K; k += blockDim.x) vs[k] = v[k];
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int i = blockIdx.x * 8 + warp; i < rows; i += gridDim.x * 8) {
        const float *row = l + (size_t)i * ld;
        float s = 0.f;
        for (int k = lane; k < K; k += 32) s = fmaf(__ldcs(row + k), vs[k], s);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) y[i] -= s;
    }
}

cudaError_t launch_gemv_sub(const float *l, long ld, int rows, int K, const float *v, float *y, cudaStream_t st)
{
    if (rows <= 0 || K <= 0) return cudaSuccess;
    if (K > 512) return cudaErrorInvalidValue;
    int blocks = (rows + 7) / 8;
    if (blocks > 148 * 16) blocks = 148 * 16;
    count_launch();
    gemv_sub_kernel<<<blocks, 256, 0, st>>>(l, ld, rows, K, v, y);
    return cudaGetLastError();
}

// bt[j][k] = BF16(u[k][j] * *scale): the U block row (K x N FP32, stride ld)
// transposed into the K-contiguous B operand of the BF16 update
__global__ void f32_transpose_bf16_kernel(const float *__restrict__ u, long ld, int K, int N,
                                          __nv_bfloat16 *__restrict__ bt, const float *__restrict__ scalep)
{
    __shared__ float tile[32][33];
    const float scale = *scalep;
    const int j0 = blockIdx.x * 32, k0 = blockIdx.y * 32;
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int k = k0 + r, j = j0 + threadIdx.x;
        tile[r][threadIdx.x] = (k < K && j < N) ? u[(size_t)k * ld + j] : 0.f;
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += blockDim.y) {
        const int j = j0 + r, k = k0 + threadIdx.x;
        if (j < N && k < K) bt[(size_t)j * K + k] = __float2bfloat16_rn(tile[threadIdx.x][r] * scale);
    }
}

cudaError_t launch_f32_transpose_bf16(const float *u, long ld, int K, int N, void *bt, const float *scale,
                                      cudaStream_t st)
{
    if (K <= 0 || N <= 0) return cudaSuccess;
    dim3 grid((N + 31) / 32, (K + 31) / 32);
    count_launch();
    f32_transpose_bf16_kernel<<<grid, dim3(32, 8), 0, st>>>(u, ld, K, N, (__nv_bfloat16 *)bt, scale);
    return cudaGetLastError();
}

// x[i] += (double)d[i]
__global__ void add_f32_to_f64_kernel(const float *__restrict__ d, double *__restrict__ x, int n)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[i] += (double)d[i];
}

cudaError_t launch_add_f32_to_f64(const float *d, double *x, int n, cudaStream_t st)
{
    if (n <= 0) return cudaSuccess;
    count_launch();
    add_f32_to_f64_kernel<<<grid_for(n), 256, 0, st>>>(d, x, n);
    return cudaGetLastError();
}

// out[slot] = max_i |v[i]| for a double vector (out zeroed by the caller;
// non-negative doubles order as their bits)
__global__ void vec_absmax_kernel(const double *__restrict__ v, int n, unsigned long long *out)
{
    double m = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) m = fmax(m, fabs(v[i]));
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

cudaError_t launch_vec_absmax(const double *v, int n, unsigned long long *out, cudaStream_t st)
{
    if (n <= 0) return cudaSuccess;
    count_launch();
    vec_absmax_kernel<<<grid_for(n) < 296 ? grid_for(n) : 296, 256, 0, st>>>(v, n, out);
    return cudaGetLastError();
}

}  // namespace lu2gpu
