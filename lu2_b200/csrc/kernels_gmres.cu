// kernels_gmres.cu -- FP64 vector kernels of GMRES-IR: the Krylov basis V
// (k vectors of length n, row j at V + j*ldv) is orthogonalised against with
// classical Gram-Schmidt applied twice, which needs k dot products at once
// and the matching combined update.  Dot products are summed in a fixed order
// (per-block partials, then one warp per product), so results do not depend
// on scheduling.
#include "lu2gpu_internal.cuh"

namespace lu2gpu {

constexpr int MD_BLOCKS = MULTI_DOT_BLOCKS;  // partial sums per dot product

// partial[j * MD_BLOCKS + b] = sum over block b's share of i of V[j][i] * z[i]
__global__ void __launch_bounds__(256) multi_dot_partial_kernel(const double *__restrict__ V, long ldv,
                                                                 const double *__restrict__ z, int n,
                                                                 double *__restrict__ partial)
{
    __shared__ double s[8];
    const int j = blockIdx.y;
    const double *v = V + (size_t)j * ldv;
    double acc = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) acc = fma(v[i], z[i], acc);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) s[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < 8; w++) t += s[w];
        partial[(size_t)j * MD_BLOCKS + blockIdx.x] = t;
    }
}

__global__ void multi_dot_final_kernel(const double *__restrict__ partial, int k, double *__restrict__ out)
{
    const int j = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    if (j >= k) return;
    double t = 0.0;
    for (int b = lane; b < MD_BLOCKS; b += 32) t += partial[(size_t)j * MD_BLOCKS + b];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    if (lane == 0) out[j] = t;
}

// out[j] = <V[j], z> for j < k; partial holds k * 148 doubles
cudaError_t launch_multi_dot(const double *V, long ldv, int k, const double *z, int n, double *partial, double *out,
                             cudaStream_t st)
{
    if (k <= 0 || n <= 0) return cudaSuccess;
    if (k > 65535) return cudaErrorInvalidValue;
    count_launch();
    multi_dot_partial_kernel<<<dim3(MD_BLOCKS, k), 256, 0, st>>>(V, ldv, z, n, partial);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    count_launch();
    multi_dot_final_kernel<<<(k + 7) / 8, 256, 0, st>>>(partial, k, out);
    return cudaGetLastError();
}

// z[i] += sign * sum_{j<k} c[j] V[j][i]   (k <= 64)
__global__ void __launch_bounds__(256) multi_axpy_kernel(const double *__restrict__ V, long ldv, int k,
                                                          const double *__restrict__ c, double sign,
                                                          double *__restrict__ z, int n)
{
    __shared__ double cs[64];
    for (int j = threadIdx.x; j < k; j += blockDim.x) cs[j] = sign * c[j];
    __syncthreads();
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double t = z[i];
        for (int j = 0; j < k; j++) t = fma(cs[j], V[(size_t)j * ldv + i], t);
        z[i] = t;
    }
}

cudaError_t launch_multi_axpy(const double *V, long ldv, int k, const double *c, double sign, double *z, int n,
                              cudaStream_t st)
{
    if (k <= 0 || n <= 0) return cudaSuccess;
    if (k > 64) return cudaErrorInvalidValue;
    int blocks = (n + 255) / 256;
    if (blocks > 148 * 8) blocks = 148 * 8;
    count_launch();
    multi_axpy_kernel<<<blocks, 256, 0, st>>>(V, ldv, k, c, sign, z, n);
    return cudaGetLastError();
}

// y = alpha * x
__global__ void vec_scale_kernel(const double *__restrict__ x, double alpha, double *__restrict__ y, int n)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] = alpha * x[i];
}

cudaError_t launch_vec_scale(const double *x, double alpha, double *y, int n, cudaStream_t st)
{
    if (n <= 0) return cudaSuccess;
    int blocks = (n + 255) / 256;
    if (blocks > 148 * 8) blocks = 148 * 8;
    count_launch();
    vec_scale_kernel<<<blocks, 256, 0, st>>>(x, alpha, y, n);
    return cudaGetLastError();
}

}  // namespace lu2gpu
