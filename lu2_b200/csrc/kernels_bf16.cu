// kernels_bf16.cu -- the trailing update of the precision form on the 5th
// generation tensor cores: C (FP32, row-major) -= scale * A * Bt^T with A
// (M x K) and Bt (N x K) in BF16, both K-contiguous.
//
// Per CTA one 128 x BN tile: TMA streams both operands through two shared
// memory stages (128-byte swizzled boxes of 64 BF16 along K, full/empty
// mbarriers per stage), one thread issues tcgen05.mma (kind::f16, BF16
// inputs, FP32 accumulator in tensor memory, 128 x BN x 16 per instruction)
// as each k block lands and releases the stage with tcgen05.commit.  Every
// thread loads its tile row of C (TMEM lane = row) into registers while that
// runs, then reads the accumulator with tcgen05.ld and writes C - scale*acc.
// The small footprint (65 KB of shared memory, 128 TMEM columns) lets two
// CTAs share an SM, so one CTA's C traffic overlaps the other's MMAs.
//
// The update this replaces is lu2's mmmulandsub -> mydgemm (lu2.c:312-343,
// lu2lib.c:2079); the precision form keeps lu2's algorithm and storage, in
// FP32 with BF16 trailing products.
#include <cuda_bf16.h>

#include "lu2gpu_internal.cuh"

namespace lu2gpu {

constexpr int UB_BM = 128;      // UMMA M (one CTA, cta_group::1)
constexpr int UB_BK = 64;       // BF16 elements per 128-byte swizzle row = one TMA box along K
constexpr int UB_KMAX = 256;    // all of K resident in shared memory
constexpr int UB_THREADS = 128; // 4 warps = the 128 TMEM lanes

__device__ __forceinline__ uint32_t smem_addr(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ bool mbar_wait_limit(uint64_t *bar, uint32_t parity, int *status, int where)
{
    const unsigned long long t0 = globaltimer_ns();
    while (true) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred P1;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}"
            : "=r"(ok)
            : "r"(smem_addr(bar)), "r"(parity)
            : "memory");
        if (ok) return true;
        if (globaltimer_ns() - t0 > WAIT_LIMIT_NS) {
            record_error(status, ERR_MBAR_TIMEOUT, where);
            return false;
        }
    }
}

// K-major, 128-byte-swizzled operand tile: 8-row groups 1024 bytes apart
// (SBO), leading offset unused for this layout (1), descriptor version 1.
__device__ __forceinline__ uint64_t umma_desc_sw128(uint32_t saddr)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)1 << 16;            // LBO (16 B units)
    d |= (uint64_t)(1024 >> 4) << 32;  // SBO
    d |= (uint64_t)1 << 46;            // version
    d |= (uint64_t)2 << 61;            // SWIZZLE_128B
    return d;
}

// kind::f16 instruction descriptor: FP32 accumulate, BF16 A and B, both K-major
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int M, int N)
{
    return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

struct Bf16Params {
    int M, N, K;
    float *C;
    long ldc;
    const float *scale;  // device scalar: C -= *scale * A Bt^T
    int tiles_m, tiles_n, group_m;
    int *status;
};

constexpr int UB_STAGES = 2;  // 64-wide k blocks in flight per CTA

template <int BN>
__global__ void __launch_bounds__(UB_THREADS, 2)
    bf16_update_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, Bf16Params p)
{
    constexpr int A_BYTES = UB_BM * 128, B_BYTES = BN * 128, STAGE = A_BYTES + B_BYTES;
    extern __shared__ uint8_t smem_raw[];
    __shared__ __align__(8) uint64_t full_bar[UB_STAGES];
    __shared__ __align__(8) uint64_t empty_bar[UB_STAGES];
    __shared__ __align__(8) uint64_t mma_bar;
    __shared__ uint32_t s_tmem;
    uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int KB = p.K / UB_BK;

    const int bid = blockIdx.x;
    const int per_group = p.group_m * p.tiles_n;
    const int first_m = (bid / per_group) * p.group_m;
    const int gsize = min(p.tiles_m - first_m, p.group_m);
    const int m0 = (first_m + (bid % per_group) % gsize) * UB_BM;
    const int n0 = ((bid % per_group) / gsize) * BN;

    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(&s_tmem)),
                     "r"(BN)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        for (int s = 0; s < UB_STAGES; s++) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&full_bar[s])) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&empty_bar[s])) : "memory");
        }
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&mma_bar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;

    auto issue = [&](int kb, int s) {
        uint8_t *sa = smem + s * STAGE;
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(&full_bar[s])),
                     "r"(STAGE)
                     : "memory");
        asm volatile(
            "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
            "[%4];" ::"r"(smem_addr(sa)),
            "l"(&tmA), "r"(kb * UB_BK), "r"(m0), "r"(smem_addr(&full_bar[s]))
            : "memory");
        asm volatile(
            "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], "
            "[%4];" ::"r"(smem_addr(sa + A_BYTES)),
            "l"(&tmB), "r"(kb * UB_BK), "r"(n0), "r"(smem_addr(&full_bar[s]))
            : "memory");
    };
    if (tid == 0)
        for (int kb = 0; kb < UB_STAGES && kb < KB; kb++) issue(kb, kb);

    // each thread's tile row of C (TMEM lane = row), loaded while the operands
    // stream in and the MMAs run
    const int row = warp * 32 + lane;
    const int m = m0 + row;
    const bool rowok = m < p.M;
    float *crow = p.C + (size_t)(rowok ? m : 0) * p.ldc + n0;
    const bool vec = rowok && n0 + BN <= p.N && ((reinterpret_cast<uintptr_t>(crow) & 15) == 0);
    float4 cv[BN / 4];
#pragma unroll
    for (int q = 0; q < BN / 4; q++) {
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
        constexpr uint32_t idesc = umma_idesc_bf16(UB_BM, BN);
        bool ok = true;
        for (int kb = 0; kb < KB && ok; kb++) {
            // refill the stage the previous k block used, once its MMAs are done
            if (kb >= 1 && kb - 1 + UB_STAGES < KB) {
                const int ps = (kb - 1) % UB_STAGES;
                if (!mbar_wait_limit(&empty_bar[ps], (uint32_t)((kb - 1) / UB_STAGES) & 1u, p.status, 7)) {
                    ok = false;
                    break;
                }
                issue(kb - 1 + UB_STAGES, ps);
            }
            const int s = kb % UB_STAGES;
            if (!mbar_wait_limit(&full_bar[s], (uint32_t)(kb / UB_STAGES) & 1u, p.status, 5)) {
                ok = false;
                break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            const uint32_t sa = smem_addr(smem + s * STAGE), sb = sa + A_BYTES;
#pragma unroll
            for (int kk = 0; kk < UB_BK / 16; kk++) {
                const uint64_t da = umma_desc_sw128(sa + kk * 32), db = umma_desc_sw128(sb + kk * 32);
                const uint32_t acc = (kb | kk) ? 1u : 0u;
                asm volatile(
                    "{\n\t.reg .pred p;\n\t"
                    "setp.ne.b32 p, %4, 0;\n\t"
                    "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem),
                    "l"(da), "l"(db), "r"(idesc), "r"(acc)
                    : "memory");
            }
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                             smem_addr(&empty_bar[s]))
                         : "memory");
        }
        // arrives once every MMA issued above has completed
        asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                         smem_addr(&mma_bar))
                     : "memory");
    }
    __syncwarp();
    const bool done = mbar_wait_limit(&mma_bar, 0, p.status, 6);
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const bool good = done && *(volatile const int *)&p.status[1] == 0;
    const float scale = *p.scale;

    // epilogue: warp w owns TMEM lanes 32w..32w+31 (its tile rows); 32 columns per load
#pragma unroll
    for (int cb = 0; cb < BN / 32; cb++) {
        uint32_t r[32];
        const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(cb * 32);
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
            "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
              "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
              "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]),
              "=r"(r[23]), "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]),
              "=r"(r[30]), "=r"(r[31])
            : "r"(taddr));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
        for (int q = 0; q < 8; q++) {
            float4 &c = cv[cb * 8 + q];
            c.x -= scale * __uint_as_float(r[4 * q]);
            c.y -= scale * __uint_as_float(r[4 * q + 1]);
            c.z -= scale * __uint_as_float(r[4 * q + 2]);
            c.w -= scale * __uint_as_float(r[4 * q + 3]);
        }
    }
    if (good && rowok) {
#pragma unroll
        for (int q = 0; q < BN / 4; q++) {
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
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(BN) : "memory");
    }
}

typedef CUresult (*PFN_encodeTiled_bf16)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                         const cuuint64_t *, const cuuint32_t *, const cuuint32_t *,
                                         CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion,
                                         CUtensorMapFloatOOBfill);

static cudaError_t make_map_bf16(CUtensorMap *m, const void *base, long ld, long rows, long cols, int box_rows)
{
    static PFN_encodeTiled_bf16 fn = nullptr;
    if (!fn) {
        void *ptr = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return cudaErrorNotSupported;
        fn = reinterpret_cast<PFN_encodeTiled_bf16>(ptr);
    }
    // 16-byte aligned base and row stride (ld multiple of 8 elements)
    if ((reinterpret_cast<uintptr_t>(base) & 15) || (ld & 7) || rows <= 0 || cols <= 0) return cudaErrorInvalidValue;
    cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)ld * 2};
    cuuint32_t box[2] = {UB_BK, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(base), dims, strides, box, estr,
                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

cudaError_t launch_bf16_update(const void *a_bf16, long lda, const void *bt_bf16, long ldb, float *c, long ldc, int M,
                               int N, int K, const float *scale, int *status, cudaStream_t st)
{
    if (M <= 0 || N <= 0) return cudaSuccess;
    if (K <= 0 || K > UB_KMAX || (K % UB_BK)) return cudaErrorInvalidValue;
    constexpr int BN = 128;
    CUtensorMap ta, tb;
    cudaError_t e = make_map_bf16(&ta, a_bf16, lda, M, K, UB_BM);
    if (e != cudaSuccess) return e;
    e = make_map_bf16(&tb, bt_bf16, ldb, N, K, BN);
    if (e != cudaSuccess) return e;
    Bf16Params p;
    p.M = M;
    p.N = N;
    p.K = K;
    p.C = c;
    p.ldc = ldc;
    p.scale = scale;
    p.tiles_m = (M + UB_BM - 1) / UB_BM;
    p.tiles_n = (N + BN - 1) / BN;
    p.group_m = 16;
    p.status = status;
    const int smem = UB_STAGES * (UB_BM * 128 + BN * 128) + 1024;
    e = cudaFuncSetAttribute(bf16_update_kernel<BN>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    if (e != cudaSuccess) return e;
    const long tiles = (long)p.tiles_m * p.tiles_n;
    if (tiles > 0x7fffffffL) return cudaErrorInvalidConfiguration;
    count_launch();
    bf16_update_kernel<BN><<<(unsigned)tiles, UB_THREADS, smem, st>>>(ta, tb, p);
    return cudaGetLastError();
}

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
