// kernels_fp8.cu -- the FP8 form's operand quantization: FP32 panels to
// E4M3 with one power-of-two scale per 128 x 128 tile, for the tcgen05
// trailing update in kernels_lowp.cu (kind::f8f6f4, per-k-block accumulators
// so that each tile's scales are applied in the epilogue).
#include <cuda_fp16.h>
#include <cuda_fp8.h>

#include "lu2gpu_internal.cuh"

namespace lu2gpu {

// ---------------------------------------------------------------------------
// Per-tile quantization: q (rows x cols E4M3, row stride ldq bytes) and
// dq[tile_r * (cols/128) + tile_c] = 2^-k, where 2^k is the largest power of
// two with max|x over the tile| * 2^k <= 448 (the largest finite E4M3 value).

__device__ __forceinline__ int fp8_tile_exponent(float amax)
{
    if (!(amax > 0.f)) return 0;
    int e;
    const float mant = frexpf(amax, &e);  // amax = mant * 2^e, mant in [0.5, 1)
    // amax = (2 mant) 2^(e-1); 448 = 1.75 * 2^8
    int k = (2.f * mant <= 1.75f) ? 8 - (e - 1) : 7 - (e - 1);
    return k > 126 ? 126 : (k < -126 ? -126 : k);
}

__global__ void __launch_bounds__(256) quant_fp8_tiles_kernel(const float *__restrict__ x, long ldx, int rows,
                                                              int cols, uint8_t *__restrict__ q, long ldq,
                                                              float *__restrict__ dq)
{
    __shared__ float s_red[8];
    const int tr = blockIdx.x, tc = blockIdx.y, tid = threadIdx.x;
    const int r0 = tr * 128, c0 = tc * 128;
    const int nr = min(128, rows - r0);
    // 128 x 128 tile = 4096 float4; 16 per thread (cols is a multiple of 128)
    float amax = 0.f;
    for (int idx = tid; idx < nr * 32; idx += 256) {
        const int r = idx >> 5, c4 = idx & 31;
        const float4 v = *reinterpret_cast<const float4 *>(x + (size_t)(r0 + r) * ldx + c0 + 4 * c4);
        amax = fmaxf(amax, fmaxf(fmaxf(fabsf(v.x), fabsf(v.y)), fmaxf(fabsf(v.z), fabsf(v.w))));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) amax = fmaxf(amax, __shfl_xor_sync(0xffffffffu, amax, o));
    if ((tid & 31) == 0) s_red[tid >> 5] = amax;
    __syncthreads();
    amax = s_red[0];
#pragma unroll
    for (int w = 1; w < 8; w++) amax = fmaxf(amax, s_red[w]);
    const int k = fp8_tile_exponent(amax);
    const float scale = ldexpf(1.f, k);
    if (tid == 0) dq[(size_t)tr * (cols / 128) + tc] = ldexpf(1.f, -k);
    for (int idx = tid; idx < nr * 32; idx += 256) {
        const int r = idx >> 5, c4 = idx & 31;
        const float4 v = *reinterpret_cast<const float4 *>(x + (size_t)(r0 + r) * ldx + c0 + 4 * c4);
        const __nv_fp8x2_storage_t lo =
            __nv_cvt_float2_to_fp8x2(make_float2(v.x * scale, v.y * scale), __NV_SATFINITE, __NV_E4M3);
        const __nv_fp8x2_storage_t hi =
            __nv_cvt_float2_to_fp8x2(make_float2(v.z * scale, v.w * scale), __NV_SATFINITE, __NV_E4M3);
        *reinterpret_cast<uint32_t *>(q + (size_t)(r0 + r) * ldq + c0 + 4 * c4) =
            (uint32_t)lo | ((uint32_t)hi << 16);
    }
}

cudaError_t launch_quant_fp8_tiles(const float *x, long ldx, int rows, int cols, uint8_t *q, long ldq, float *dq,
                                   cudaStream_t st)
{
    if (rows <= 0 || cols <= 0) return cudaSuccess;
    if ((cols % 128) || (ldx & 3) || (reinterpret_cast<uintptr_t>(x) & 15) || (ldq & 3) ||
        (reinterpret_cast<uintptr_t>(q) & 3))
        return cudaErrorInvalidValue;
    count_launch();
    dim3 grid((rows + 127) / 128, cols / 128);
    quant_fp8_tiles_kernel<<<grid, 256, 0, st>>>(x, ldx, rows, cols, q, ldq, dq);
    return cudaGetLastError();
}

// E4M3 bytes back to FP32 (dequantized with the tile factors): for tests and
// for the error analysis of the quantization
__global__ void dequant_fp8_tiles_kernel(const uint8_t *__restrict__ q, long ldq, const float *__restrict__ dq,
                                         int rows, int cols, float *__restrict__ y, long ldy)
{
    const long total = (long)rows * cols;
    for (long idx = (long)blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += (long)gridDim.x * blockDim.x) {
        const long r = idx / cols, c = idx - r * cols;
        const __half_raw h = __nv_cvt_fp8_to_halfraw(q[r * ldq + c], __NV_E4M3);
        y[r * ldy + c] = __half2float(__half(h)) * dq[(r / 128) * (cols / 128) + c / 128];
    }
}

cudaError_t launch_dequant_fp8_tiles(const uint8_t *q, long ldq, const float *dq, int rows, int cols, float *y,
                                     long ldy, cudaStream_t st)
{
    if (rows <= 0 || cols <= 0) return cudaSuccess;
    if (cols % 128) return cudaErrorInvalidValue;
    long blocks = ((long)rows * cols + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    count_launch();
    dequant_fp8_tiles_kernel<<<(unsigned)blocks, 256, 0, st>>>(q, ldq, dq, rows, cols, y, ldy);
    return cudaGetLastError();
}

}  // namespace lu2gpu
