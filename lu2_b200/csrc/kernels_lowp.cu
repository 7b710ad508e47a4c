// kernels_lowp.cu -- the precision forms' trailing update as a persistent,
// warp-specialized tcgen05 kernel:
//   C (FP32, row-major) -= scale * A Bt^T
// with A (M x K) and Bt (N x K) K-contiguous, either BF16 (one scale per
// panel) or FP8 E4M3 (one power-of-two scale per 128 x 128 tile of each
// operand, applied per 128-wide k block), K <= 256.
//
// The update is HBM-bound (K = 256 gives 64 FLOP per byte of C for BF16), so
// the design is about streaming C: one CTA per SM walks its share of the
// 128 x 128 output tiles.
//   warp 4 (producer): TMA loads of the operand k-chunks (128 rows x 128
//     bytes each, 128-byte swizzle) through a 2-stage ring, and of the C tile
//     (four 128 x 32 FP32 boxes, 128-byte swizzle) into one of two C buffers;
//   warp 5 (MMA): tcgen05.mma into one of two tensor-memory accumulators
//     (per k block for FP8, since the tile scales differ between k blocks);
//   warps 0-3 (epilogue, TMEM lane = tile row): tcgen05.ld of the
//     accumulator, C -= scale * acc on the swizzled shared-memory tile
//     (conflict-free: the 16-byte chunk index is XORed with the row), then one
//     TMA store of the tile.
// C is read and written once, in bulk, with the next tile's C load and MMAs
// overlapping this tile's epilogue and store.  Every wait is bounded; a
// timeout in any role sets an error bit and a shared abort flag that ends all
// roles.
//
// The update this replaces is lu2's mmmulandsub -> mydgemm (lu2.c:312-343,
// lu2lib.c:2079); the precision forms keep lu2's algorithm in FP32.
#include <cuda_bf16.h>

#include "lu2gpu_internal.cuh"

namespace lu2gpu {

constexpr int LP_BM = 128, LP_BN = 128;
constexpr int LP_CHUNK = 128 * 128;      // bytes of one operand k-chunk (128 rows x 128 bytes)
constexpr int LP_STAGE = 2 * LP_CHUNK;   // A chunk + B chunk
constexpr int LP_STAGES = 2;
constexpr int LP_CBUF = LP_BM * LP_BN * 4;  // one FP32 C tile
constexpr int LP_SMEM = LP_STAGES * LP_STAGE + 2 * LP_CBUF + 1024;
constexpr int LP_THREADS = 192;
constexpr int LP_GROUP_M = 16;

struct LowpParams {
    int M, N, K;
    float *C;  // for the ragged last column tile (N not a multiple of 4)
    long ldc;
    const float *scale;  // BF16: device scalar
    const float *da;     // FP8: [tiles_m][K/128]
    const float *db;     // FP8: [tiles_n][K/128]
    int tiles_m, tiles_n;
    int *status;
};

__device__ __forceinline__ uint32_t lp_smem(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// bounded wait; gives up at once when another role has aborted
__device__ __forceinline__ bool lp_wait(uint64_t *bar, uint32_t parity, int *status, int where, volatile int *abort)
{
    const unsigned long long t0 = globaltimer_ns();
    while (true) {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred P1;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
            "selp.b32 %0, 1, 0, P1;\n\t}"
            : "=r"(ok)
            : "r"(lp_smem(bar)), "r"(parity)
            : "memory");
        if (ok) return true;
        if (*abort) return false;
        if (globaltimer_ns() - t0 > WAIT_LIMIT_NS) {
            record_error(status, ERR_MBAR_TIMEOUT, where);
            *abort = 1;
            return false;
        }
    }
}

__device__ __forceinline__ uint64_t lp_desc_sw128(uint32_t saddr)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);
    d |= (uint64_t)1 << 16;
    d |= (uint64_t)(1024 >> 4) << 32;
    d |= (uint64_t)1 << 46;
    d |= (uint64_t)2 << 61;
    return d;
}

__device__ __forceinline__ void lp_tma_load(uint32_t dst, const CUtensorMap *map, int x, int y, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            dst),
        "l"(map), "r"(x), "r"(y), "r"(lp_smem(bar))
        : "memory");
}

__device__ __forceinline__ void lp_tile(int t, int tiles_m, int tiles_n, int &tm, int &tn)
{
    const int per_group = LP_GROUP_M * tiles_n;
    const int first_m = (t / per_group) * LP_GROUP_M;
    const int gsize = min(tiles_m - first_m, LP_GROUP_M);
    tm = first_m + (t % per_group) % gsize;
    tn = (t % per_group) / gsize;
}

// FP8 = false: kind::f16 with BF16 operands (64 elements per chunk);
// FP8 = true: kind::f8f6f4 with E4M3 operands (128 elements per chunk = one scale block)
template <bool FP8>
__global__ void __launch_bounds__(LP_THREADS, 1)
    lowp_update_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB,
                       const __grid_constant__ CUtensorMap tmC, LowpParams p)
{
    constexpr int CHUNK_ELEMS = FP8 ? 128 : 64;
    constexpr int KSTEP_BYTES = 32;  // one MMA: K = 16 BF16 or 32 E4M3 = 32 bytes
    constexpr int ACC_COLS = FP8 ? 2 * LP_BN : LP_BN;  // per buffer: one accumulator per k block for FP8
    constexpr uint32_t TMEM_COLS = 2 * ACC_COLS;        // 256 (BF16) or 512 (FP8)
    constexpr uint32_t IDESC = FP8 ? ((1u << 4) | ((uint32_t)(LP_BN >> 3) << 17) | ((uint32_t)(LP_BM >> 4) << 24))
                                   : ((1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(LP_BN >> 3) << 17) |
                                      ((uint32_t)(LP_BM >> 4) << 24));

    extern __shared__ uint8_t smem_raw[];
    __shared__ __align__(8) uint64_t op_full[LP_STAGES], op_empty[LP_STAGES];
    __shared__ __align__(8) uint64_t acc_full[2], acc_empty[2], c_full[2], c_empty[2];
    __shared__ uint32_t s_tmem;
    __shared__ volatile int s_abort;
    uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    uint8_t *cbuf = smem + LP_STAGES * LP_STAGE;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int KC = p.K / CHUNK_ELEMS;
    const int tiles = p.tiles_m * p.tiles_n;

    if (warp == 5) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(lp_smem(&s_tmem)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    if (tid == 0) {
        s_abort = 0;
        for (int s = 0; s < LP_STAGES; s++) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(lp_smem(&op_full[s])) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(lp_smem(&op_empty[s])) : "memory");
        }
        for (int b = 0; b < 2; b++) {
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(lp_smem(&acc_full[b])) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 128;" ::"r"(lp_smem(&acc_empty[b])) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(lp_smem(&c_full[b])) : "memory");
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(lp_smem(&c_empty[b])) : "memory");
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = s_tmem;

    if (warp == 4) {
        // ---------------- producer ----------------
        if (lane == 0) {
            int it = 0;
            for (int t = blockIdx.x; t < tiles && !s_abort; t += gridDim.x, it++) {
                int tm, tn;
                lp_tile(t, p.tiles_m, p.tiles_n, tm, tn);
                const int m0 = tm * LP_BM, n0 = tn * LP_BN;
                for (int kc = 0; kc < KC; kc++) {
                    const int q = it * KC + kc, s = q % LP_STAGES, k = q / LP_STAGES;
                    if (!lp_wait(&op_empty[s], (uint32_t)(k & 1) ^ 1u, p.status, 20, &s_abort)) break;
                    uint8_t *st = smem + s * LP_STAGE;
                    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(lp_smem(&op_full[s])),
                                 "r"(LP_STAGE)
                                 : "memory");
                    lp_tma_load(lp_smem(st), &tmA, kc * CHUNK_ELEMS, m0, &op_full[s]);
                    lp_tma_load(lp_smem(st + LP_CHUNK), &tmB, kc * CHUNK_ELEMS, n0, &op_full[s]);
                }
                const int b = it & 1, u = it >> 1;
                if (!lp_wait(&c_empty[b], (uint32_t)(u & 1) ^ 1u, p.status, 21, &s_abort)) break;
                uint8_t *cb = cbuf + b * LP_CBUF;
                asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(lp_smem(&c_full[b])),
                             "r"(LP_CBUF)
                             : "memory");
#pragma unroll
                for (int j = 0; j < 4; j++) lp_tma_load(lp_smem(cb + j * (LP_CBUF / 4)), &tmC, n0 + 32 * j, m0, &c_full[b]);
            }
        }
        __syncwarp();
    } else if (warp == 5) {
        // ---------------- MMA issuer ----------------
        if (lane == 0) {
            int it = 0;
            for (int t = blockIdx.x; t < tiles && !s_abort; t += gridDim.x, it++) {
                const int b = it & 1, u = it >> 1;
                if (!lp_wait(&acc_empty[b], (uint32_t)(u & 1) ^ 1u, p.status, 22, &s_abort)) break;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                bool ok = true;
                for (int kc = 0; kc < KC; kc++) {
                    const int q = it * KC + kc, s = q % LP_STAGES, k = q / LP_STAGES;
                    if (!lp_wait(&op_full[s], (uint32_t)(k & 1), p.status, 23, &s_abort)) {
                        ok = false;
                        break;
                    }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const uint32_t sa = lp_smem(smem + s * LP_STAGE), sb = sa + LP_CHUNK;
                    const uint32_t dacc = tmem + (uint32_t)(b * ACC_COLS + (FP8 ? kc * LP_BN : 0));
#pragma unroll
                    for (int kk = 0; kk < 128 / KSTEP_BYTES; kk++) {
                        const uint64_t da = lp_desc_sw128(sa + kk * KSTEP_BYTES);
                        const uint64_t db = lp_desc_sw128(sb + kk * KSTEP_BYTES);
                        const uint32_t accum = FP8 ? (kk ? 1u : 0u) : ((kc | kk) ? 1u : 0u);
                        if (FP8)
                            asm volatile(
                                "{\n\t.reg .pred pp;\n\t"
                                "setp.ne.b32 pp, %4, 0;\n\t"
                                "tcgen05.mma.cta_group::1.kind::f8f6f4 [%0], %1, %2, %3, pp;\n\t}" ::"r"(dacc),
                                "l"(da), "l"(db), "r"(IDESC), "r"(accum)
                                : "memory");
                        else
                            asm volatile(
                                "{\n\t.reg .pred pp;\n\t"
                                "setp.ne.b32 pp, %4, 0;\n\t"
                                "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, pp;\n\t}" ::"r"(dacc),
                                "l"(da), "l"(db), "r"(IDESC), "r"(accum)
                                : "memory");
                    }
                    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                     lp_smem(&op_empty[s]))
                                 : "memory");
                }
                if (!ok) break;
                asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                 lp_smem(&acc_full[b]))
                             : "memory");
            }
        }
        __syncwarp();
    } else {
        // ---------------- epilogue: warps 0-3, TMEM lane = tile row ----------------
        const int row = warp * 32 + lane;
        const int sw = row & 7;
        int it = 0;
        for (int t = blockIdx.x; t < tiles; t += gridDim.x, it++) {
            int tm, tn;
            lp_tile(t, p.tiles_m, p.tiles_n, tm, tn);
            const int b = it & 1, u = it >> 1;
            bool ok = lp_wait(&acc_full[b], (uint32_t)(u & 1), p.status, 24, &s_abort);
            ok = ok && lp_wait(&c_full[b], (uint32_t)(u & 1), p.status, 25, &s_abort);
            // one decision for all 128 epilogue threads (they share named
            // barriers and warp-collective TMEM loads below)
            uint32_t fail = (ok && !s_abort) ? 0u : 1u, any_fail;
            asm volatile(
                "{\n\t.reg .pred q, r;\n\t"
                "setp.ne.u32 q, %1, 0;\n\t"
                "bar.red.or.pred r, 1, 128, q;\n\t"
                "selp.u32 %0, 1, 0, r;\n\t}"
                : "=r"(any_fail)
                : "r"(fail)
                : "memory");
            if (any_fail) break;
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            float s0, s1 = 0.f;
            const bool two = FP8 && p.K > 128;  // FP8: the second k block's accumulator holds data
            if (FP8) {
                const int KB = p.K / 128;
                s0 = p.da[(size_t)tm * KB] * p.db[(size_t)tn * KB];
                if (two) s1 = p.da[(size_t)tm * KB + 1] * p.db[(size_t)tn * KB + 1];
            } else {
                s0 = *p.scale;
            }
            uint8_t *cb = cbuf + b * LP_CBUF;
#pragma unroll 1
            for (int c32 = 0; c32 < 4; c32++) {
                uint32_t r0[32], r1[32];
                const uint32_t ta = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(b * ACC_COLS + c32 * 32);
                asm volatile(
                    "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
                    "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                    : "=r"(r0[0]), "=r"(r0[1]), "=r"(r0[2]), "=r"(r0[3]), "=r"(r0[4]), "=r"(r0[5]), "=r"(r0[6]),
                      "=r"(r0[7]), "=r"(r0[8]), "=r"(r0[9]), "=r"(r0[10]), "=r"(r0[11]), "=r"(r0[12]), "=r"(r0[13]),
                      "=r"(r0[14]), "=r"(r0[15]), "=r"(r0[16]), "=r"(r0[17]), "=r"(r0[18]), "=r"(r0[19]),
                      "=r"(r0[20]), "=r"(r0[21]), "=r"(r0[22]), "=r"(r0[23]), "=r"(r0[24]), "=r"(r0[25]),
                      "=r"(r0[26]), "=r"(r0[27]), "=r"(r0[28]), "=r"(r0[29]), "=r"(r0[30]), "=r"(r0[31])
                    : "r"(ta));
                if (two) {
                    const uint32_t tb = ta + LP_BN;
                    asm volatile(
                        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,"
                        "%15,%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
                        : "=r"(r1[0]), "=r"(r1[1]), "=r"(r1[2]), "=r"(r1[3]), "=r"(r1[4]), "=r"(r1[5]), "=r"(r1[6]),
                          "=r"(r1[7]), "=r"(r1[8]), "=r"(r1[9]), "=r"(r1[10]), "=r"(r1[11]), "=r"(r1[12]),
                          "=r"(r1[13]), "=r"(r1[14]), "=r"(r1[15]), "=r"(r1[16]), "=r"(r1[17]), "=r"(r1[18]),
                          "=r"(r1[19]), "=r"(r1[20]), "=r"(r1[21]), "=r"(r1[22]), "=r"(r1[23]), "=r"(r1[24]),
                          "=r"(r1[25]), "=r"(r1[26]), "=r"(r1[27]), "=r"(r1[28]), "=r"(r1[29]), "=r"(r1[30]),
                          "=r"(r1[31])
                        : "r"(tb));
                }
                asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
                // box c32 holds tile columns 32*c32 .. +31: 128 rows x 128 bytes, chunk j of row r at (j ^ (r & 7))
                uint8_t *rowp = cb + c32 * (LP_CBUF / 4) + row * 128;
#pragma unroll
                for (int j = 0; j < 8; j++) {
                    float4 *cp = reinterpret_cast<float4 *>(rowp + ((j ^ sw) << 4));
                    float4 c = *cp;
                    float a0 = __uint_as_float(r0[4 * j]), a1 = __uint_as_float(r0[4 * j + 1]);
                    float a2 = __uint_as_float(r0[4 * j + 2]), a3 = __uint_as_float(r0[4 * j + 3]);
                    c.x -= s0 * a0;
                    c.y -= s0 * a1;
                    c.z -= s0 * a2;
                    c.w -= s0 * a3;
                    if (two) {
                        c.x -= s1 * __uint_as_float(r1[4 * j]);
                        c.y -= s1 * __uint_as_float(r1[4 * j + 1]);
                        c.z -= s1 * __uint_as_float(r1[4 * j + 2]);
                        c.w -= s1 * __uint_as_float(r1[4 * j + 3]);
                    }
                    *cp = c;
                }
            }
            // accumulator buffer b is free for tile it + 2
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(lp_smem(&acc_empty[b])) : "memory");
            // the shared-memory tile is complete: one thread stores it with TMA,
            // except a last column tile that ends inside a 16-byte chunk (the
            // bulk store writes whole chunks), which every thread stores by row
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            asm volatile("bar.sync 1, 128;" ::: "memory");
            const int m0 = tm * LP_BM, n0 = tn * LP_BN;
            if (n0 + LP_BN > p.N && (p.N & 3)) {
                const int m = m0 + row, ncols = p.N - n0;
                if (m < p.M) {
                    float *dst = p.C + (size_t)m * p.ldc + n0;
                    for (int col = 0; col < ncols; col++) {
                        const int j = (col & 31) >> 2;
                        const float *src = reinterpret_cast<const float *>(cb + (col >> 5) * (LP_CBUF / 4) + row * 128 +
                                                                           ((j ^ sw) << 4)) +
                                           (col & 3);
                        dst[col] = *src;
                    }
                }
                asm volatile("bar.sync 1, 128;" ::: "memory");
                if (row == 0)
                    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(lp_smem(&c_empty[b])) : "memory");
            } else if (row == 0) {
#pragma unroll
                for (int j = 0; j < 4; j++)
                    asm volatile(
                        "cp.async.bulk.tensor.2d.global.shared::cta.bulk_group [%0, {%1, %2}], [%3];" ::"l"(&tmC),
                        "r"(n0 + 32 * j), "r"(m0), "r"(lp_smem(cb + j * (LP_CBUF / 4)))
                        : "memory");
                asm volatile("cp.async.bulk.commit_group;" ::: "memory");
                asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
                asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(lp_smem(&c_empty[b])) : "memory");
            }
            __syncwarp();
        }
        if (row == 0) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 5) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
    }
}

typedef CUresult (*PFN_encodeTiled_lp)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                       const cuuint64_t *, const cuuint32_t *, const cuuint32_t *,
                                       CUtensorMapInterleave, CUtensorMapSwizzle, CUtensorMapL2promotion,
                                       CUtensorMapFloatOOBfill);

// 2-D map, 128-byte swizzle: rows x cols elements of `esize` bytes, row stride
// ld elements, boxes of (128 / esize) elements x box_rows
static cudaError_t lp_map(CUtensorMap *m, CUtensorMapDataType dt, int esize, const void *base, long ld, long rows,
                          long cols, int box_rows)
{
    static PFN_encodeTiled_lp fn = nullptr;
    if (!fn) {
        void *ptr = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            return cudaErrorNotSupported;
        fn = reinterpret_cast<PFN_encodeTiled_lp>(ptr);
    }
    if ((reinterpret_cast<uintptr_t>(base) & 15) || ((ld * esize) & 15) || rows <= 0 || cols <= 0)
        return cudaErrorInvalidValue;
    cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)(ld * esize)};
    cuuint32_t box[2] = {(cuuint32_t)(128 / esize), (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = fn(m, dt, 2, const_cast<void *>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                    CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

template <bool FP8>
static cudaError_t lp_launch(const void *a, long lda, const void *bt, long ldb, float *c, long ldc, int M, int N,
                             int K, const float *scale, const float *da, const float *db, int *status, int max_ctas,
                             cudaStream_t st)
{
    if (M <= 0 || N <= 0) return cudaSuccess;
    const int chunk = FP8 ? 128 : 64;
    if (K <= 0 || K > 256 || (K % chunk)) return cudaErrorInvalidValue;
    if (reinterpret_cast<uintptr_t>(c) & 15) return cudaErrorInvalidValue;
    const CUtensorMapDataType dt = FP8 ? CU_TENSOR_MAP_DATA_TYPE_UINT8 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16;
    const int es = FP8 ? 1 : 2;
    CUtensorMap ta, tb, tc;
    cudaError_t e = lp_map(&ta, dt, es, a, lda, M, K, LP_BM);
    if (e != cudaSuccess) return e;
    if ((e = lp_map(&tb, dt, es, bt, ldb, N, K, LP_BN)) != cudaSuccess) return e;
    if ((e = lp_map(&tc, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, c, ldc, M, N, LP_BM)) != cudaSuccess) return e;
    LowpParams p;
    p.M = M;
    p.N = N;
    p.K = K;
    p.C = c;
    p.ldc = ldc;
    p.scale = scale;
    p.da = da;
    p.db = db;
    p.tiles_m = (M + LP_BM - 1) / LP_BM;
    p.tiles_n = (N + LP_BN - 1) / LP_BN;
    p.status = status;
    e = cudaFuncSetAttribute(lowp_update_kernel<FP8>, cudaFuncAttributeMaxDynamicSharedMemorySize, LP_SMEM);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 148;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    const long tiles = (long)p.tiles_m * p.tiles_n;
    if (tiles > 0x7fffffffL) return cudaErrorInvalidConfiguration;
    if (max_ctas > 0 && max_ctas < sms) sms = max_ctas;  // leave SMs to a concurrent panel
    const int grid = tiles < sms ? (int)tiles : sms;
    count_launch();
    lowp_update_kernel<FP8><<<grid, LP_THREADS, LP_SMEM, st>>>(ta, tb, tc, p);
    return cudaGetLastError();
}

cudaError_t launch_lowp_update_bf16(const void *a16, long lda, const void *bt16, long ldb, float *c, long ldc, int M,
                                    int N, int K, const float *scale, int *status, int max_ctas, cudaStream_t st)
{
    return lp_launch<false>(a16, lda, bt16, ldb, c, ldc, M, N, K, scale, nullptr, nullptr, status, max_ctas, st);
}

cudaError_t launch_lowp_update_fp8(const uint8_t *a8, long lda, const float *da, const uint8_t *bt8, long ldb,
                                   const float *db, float *c, long ldc, int M, int N, int K, int *status,
                                   int max_ctas, cudaStream_t st)
{
    return lp_launch<true>(a8, lda, bt8, ldb, c, ldc, M, N, K, nullptr, da, db, status, max_ctas, st);
}

}  // namespace lu2gpu
