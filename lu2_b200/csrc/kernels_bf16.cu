// kernels_bf16.cu -- FP32 -> BF16 conversion of the precision form's L21
// panel (with its per-panel power-of-two scale) for the tcgen05 trailing
// update in kernels_lowp.cu.
#include <cuda_bf16.h>

#include "lu2gpu_internal.cuh"

namespace lu2gpu {

// ---------------------------------------------------------------------------
// FP32 <-> BF16 helpers for the precision form

// out (rows x cols, stride ldo, BF16) = in (FP32, stride ldi) * *scale
__global__ void f32_to_bf16_kernel(const float *__restrict__ in, long ldi, __nv_bfloat16 *__restrict__ out, long ldo,
                                   int rows, int cols, const float *scalep)
{
    const float scale = *scalep;
    const long total = (long)rows * cols;
    for (long idx = (long)blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += (long)gridDim.x * blockDim.x) {
        const long r = idx / cols, c = idx - r * cols;
        out[r * ldo + c] = __float2bfloat16_rn(in[r * ldi + c] * scale);
    }
}

cudaError_t launch_f32_to_bf16(const float *in, long ldi, void *out, long ldo, int rows, int cols,
                               const float *scale, cudaStream_t st)
{
    if (rows <= 0 || cols <= 0) return cudaSuccess;
    long total = (long)rows * cols;
    long blocks = (total + 255) / 256;
    if (blocks > 148 * 16) blocks = 148 * 16;
    count_launch();
    f32_to_bf16_kernel<<<(unsigned)blocks, 256, 0, st>>>(in, ldi, (__nv_bfloat16 *)out, ldo, rows, cols, scale);
    return cudaGetLastError();
}

}  // namespace lu2gpu
