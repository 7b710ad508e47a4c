// kernels_fp8.cu -- the FP8 form of the precision path's trailing update:
// C (FP32, row-major) -= sum over 128-wide k blocks kb of
//     dA(tile_m, kb) * dB(tile_n, kb) * (Aq_kb Bq_kb^T)
// where Aq (M x K) and Bq (N x K, the transposed U block row) hold E4M3 values
// quantized per 128 x 128 tile with power-of-two scales, and dA, dB are the
// tiles' dequantization factors.
//
// Per CTA one 128 x 128 tile of C.  TMA brings each k block of both operands
// (128 rows x 128 bytes, 128-byte swizzle) into its own shared-memory stage;
// one thread issues tcgen05.mma kind::f8f6f4 (E4M3 x E4M3, FP32 accumulate,
// 128 x 128 x 32 per instruction) into a separate tensor-memory accumulator
// per k block, since the tile scales differ between k blocks.  While that
// runs every thread loads its row of C; the epilogue reads both accumulators
// with tcgen05.ld and applies C -= sum_kb s_kb * acc_kb.  K <= 256 keeps the
// footprint at 65 KB of shared memory and 256 TMEM columns, so two CTAs share
// an SM.
//
// The update this replaces is lu2's mmmulandsub -> mydgemm (lu2.c:312-343,
// lu2lib.c:2079); the FP8 form keeps lu2's algorithm and storage in FP32.
#include <cuda_fp16.h>
#include <cuda_fp8.h>

#include "lu2gpu_internal.cuh"

namespace lu2gpu {

constexpr int F8_BM = 128, F8_BN = 128;
constexpr int F8_BK = 128;  // E4M3 elements per 128-byte swizzle row = one TMA box = one scale block
constexpr int F8_KMAX = 256;
constexpr int F8_THREADS = 128;

__device__ __forceinline__ uint32_t f8_smem_addr(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ bool f8_mbar_wait(uint64_t *bar, uint32_t parity, int *status, int where)
{
    const unsigned long long t0 = globaltimer_ns();
    while (true) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred P1;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}"
            : "=r"(ok)
            : "r"(f8_smem_addr(bar)), "r"(parity)
            : "memory");
        if (ok) return true;
        if (globaltimer_ns() - t0 > WAIT_LIMIT_NS) {
            record_error(status, ERR_MBAR_TIMEOUT, where);
            return false;
        }
    }
}

// K-major, 128-byte-swizzled operand tile (8-row groups 1024 bytes apart)
__device__ __forceinline__ uint64_t f8_desc_sw128(uint32_t saddr)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)1 << 16;
    d |= (uint64_t)(1024 >> 4) << 32;
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)2 << 61;
    return d;
}

// kind::f8f6f4 instruction descriptor: FP32 accumulate, A and B E4M3 (format
// 0), both K-major
__host__ __device__ constexpr uint32_t umma_idesc_e4m3(int M, int N)
{
    return (1u << 4) | (0u << 7) | (0u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

struct Fp8Params {
    int M, N, K;
    float *C;
    long ldc;
    const float *da;  // [tiles_m][K/128] dequantization factors of A's tiles
    const float *db;  // [tiles_n][K/128] of Bt's tiles
    int tiles_m, tiles_n, group_m;
    int *status;
};

__global__ void __launch_bounds__(F8_THREADS, 2)
    fp8_update_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, Fp8Params p)
{
    constexpr int A_BYTES = F8_BM * F8_BK, B_BYTES = F8_BN * F8_BK, STAGE = A_BYTES + B_BYTES;
    constexpr int KBMAX = F8_KMAX / F8_BK;
    extern __shared__ uint8_t smem_raw[];
    __shared__ __align__(8) uint64_t full_bar[KBMAX];
    __shared__ __align__(8) uint64_t mma_bar;
    __shared__ uint32_t s_tmem;
    uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int KB = p.K / F8_BK;  // 1 or 2: every k block has its own stage and accumulator

    const int bid = blockIdx.x;
    const int per_group = p.group_m * p.tiles_n;
    const int first_m = (bid / per_group) * p.group_m;
    const int gsize = min(p.tiles_m - first_m, p.group_m);
    const int tm = first_m + (bid % per_group) % gsize;
    const int tn = (bid % per_group) / gsize;
    const int m0 = tm * F8_BM, n0 = tn * F8_BN;
    const uint32_t tcols = KB == 1 ? 128u : 256u;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(f8_smem_addr(&s_tmem)),
                     "r"(tcols)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int s = 0; s < KBMAX; s++)
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(f8_smem_addr(&full_bar[s])) : "memory");
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(f8_smem_addr(&mma_bar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;

    if (tid == 0) {
        for (int kb = 0; kb < KB; kb++) {
            uint8_t *sa = smem + kb * STAGE;
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(f8_smem_addr(&full_bar[kb])),
                         "r"(STAGE)
                         : "memory");
            asm volatile(
                "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
                "[%4];" ::"r"(f8_smem_addr(sa)),
                "l"(&tmA), "r"(kb * F8_BK), "r"(m0), "r"(f8_smem_addr(&full_bar[kb]))
                : "memory");
            asm volatile(
                "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
                "[%4];" ::"r"(f8_smem_addr(sa + A_BYTES)),
                "l"(&tmB), "r"(kb * F8_BK), "r"(n0), "r"(f8_smem_addr(&full_bar[kb]))
                : "memory");
        }
    }

    // each thread's tile row of C (TMEM lane = row), loaded while the operands
    // stream in and the MMAs run
    const int row = warp * 32 + lane;
    const int m = m0 + row;
    const bool rowok = m < p.M;
    float *crow = p.C + (size_t)(rowok ? m : 0) * p.ldc + n0;
    const bool vec = rowok && n0 + F8_BN <= p.N && ((reinterpret_cast<uintptr_t>(crow) & 15) == 0);
    float4 cv[F8_BN / 4];
#pragma unroll
    for (int q = 0; q < F8_BN / 4; q++) {
        if (vec) {
            cv[q] = *reinterpret_cast<const float4 *>(crow + 4 * q);
        } else {
            float e[4] = {0.f, 0.f, 0.f, 0.f};
            for (int j = 0; j < 4; j++)
                if (rowok && n0 + 4 * q + j < p.N) e[j] = crow[4 * q + j];
            cv[q] = make_float4(e[0], e[1], e[2], e[3]);
        }
    }

    if (tid == 0) {
        constexpr uint32_t idesc = umma_idesc_e4m3(F8_BM, F8_BN);
        for (int kb = 0; kb < KB; kb++) {
            if (!f8_mbar_wait(&full_bar[kb], 0u, p.status, 8)) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t sa = f8_smem_addr(smem + kb * STAGE), sb = sa + A_BYTES;
            const uint32_t dacc = tmem + (uint32_t)(kb * F8_BN);
#pragma unroll
            for (int kk = 0; kk < F8_BK / 32; kk++) {
                const uint64_t da = f8_desc_sw128(sa + kk * 32), db = f8_desc_sw128(sb + kk * 32);
                const uint32_t acc = kk ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f8f6f4 [%0], %1, %2, %3, p;\n\t}" ::"r"(dacc),
                    "l"(da), "l"(db), "r"(idesc), "r"(acc)
                    : "memory");
            }
        }
        // arrives once every MMA issued above has completed
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         f8_smem_addr(&mma_bar))
                     : "memory");
    }
    __syncwarp();
    const bool done = f8_mbar_wait(&mma_bar, 0, p.status, 9);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const bool good = done && *(volatile const int *)&p.status[1] == 0;
    float skb[KBMAX];
#pragma unroll
    for (int kb = 0; kb < KBMAX; kb++)
        skb[kb] = kb < KB ? p.da[(size_t)tm * KB + kb] * p.db[(size_t)tn * KB + kb] : 0.f;

    // epilogue: warp w owns TMEM lanes 32w..32w+31 (its tile rows); 32 columns per load
#pragma unroll
    for (int cb = 0; cb < F8_BN / 32; cb++) {
#pragma unroll
        for (int kb = 0; kb < KBMAX; kb++) {
            if (kb >= KB) break;
            uint32_t r[32];
            const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(kb * F8_BN + cb * 32);
            asm volatile(
                "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                  "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),
                  "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]),
                  "=r"(r[22]), "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]),
                  "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                : "r"(taddr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            const float s = skb[kb];
#pragma unroll
            for (int q = 0; q < 8; q++) {
                float4 &c = cv[cb * 8 + q];
                c.x -= s * __uint_as_float(r[4 * q]);
                c.y -= s * __uint_as_float(r[4 * q + 1]);
                c.z -= s * __uint_as_float(r[4 * q + 2]);
                c.w -= s * __uint_as_float(r[4 * q + 3]);
            }
        }
    }
    if (good && rowok) {
#pragma unroll
        for (int q = 0; q < F8_BN / 4; q++) {
            if (vec) {
                *reinterpret_cast<float4 *>(crow + 4 * q) = cv[q];
            } else {
                const float e[4] = {cv[q].x, cv[q].y, cv[q].z, cv[q].w};
                for (int j = 0; j < 4; j++)
                    if (n0 + 4 * q + j < p.N) crow[4 * q + j] = e[j];
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(tcols) : "memory");
    }
}

typedef CUresult (*PFN_encodeTiled_fp8)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                        const cuuint64_t *, const cuuint32_t *, const cuuint32_t *,
                                        CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion,
                                        CUtensorMapFloatOOBfill);

// 2-D map over an E4M3 matrix (rows x cols bytes, row stride ld bytes), boxes
// of 128 bytes x box_rows
static cudaError_t make_map_fp8(CUtensorMap *m, const void *base, long ld, long rows, long cols, int box_rows)
{
    static PFN_encodeTiled_fp8 fn = nullptr;
    if (!fn) {
        void *ptr = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return cudaErrorNotSupported;
        fn = reinterpret_cast<PFN_encodeTiled_fp8>(ptr);
    }
    if ((reinterpret_cast<uintptr_t>(base) & 15) || (ld & 15) || rows <= 0 || cols <= 0 || (cols % F8_BK))
        return cudaErrorInvalidValue;
    cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)ld};
    cuuint32_t box[2] = {F8_BK, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<void *>(base), dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

cudaError_t launch_fp8_update(const uint8_t *a8, long lda, const float *da, const uint8_t *bt8, long ldb,
                              const float *db, float *c, long ldc, int M, int N, int K, int *status, cudaStream_t st)
{
    if (M <= 0 || N <= 0) return cudaSuccess;
    if (K != 128 && K != 256) return cudaErrorInvalidValue;
    CUtensorMap ta, tb;
    cudaError_t e = make_map_fp8(&ta, a8, lda, M, K, F8_BM);
    if (e != cudaSuccess) return e;
    e = make_map_fp8(&tb, bt8, ldb, N, K, F8_BN);
    if (e != cudaSuccess) return e;
    Fp8Params p;
    p.M = M;
    p.N = N;
    p.K = K;
    p.C = c;
    p.ldc = ldc;
    p.da = da;
    p.db = db;
    p.tiles_m = (M + F8_BM - 1) / F8_BM;
    p.tiles_n = (N + F8_BN - 1) / F8_BN;
    p.group_m = 16;
    p.status = status;
    const int smem = (F8_KMAX / F8_BK) * (F8_BM + F8_BN) * F8_BK + 1024;
    e = cudaFuncSetAttribute(fp8_update_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    const long tiles = (long)p.tiles_m * p.tiles_n;
    if (tiles > 0x7fffffffL) return cudaErrorInvalidConfiguration;
    count_launch();
    fp8_update_kernel<<<(unsigned)tiles, F8_THREADS, smem, st>>>(ta, tb, p);
    return cudaGetLastError();
}

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
