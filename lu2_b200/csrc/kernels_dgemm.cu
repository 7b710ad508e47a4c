// kernels_dgemm.cu -- FP64 tensor-core GEMM for the trailing update and the
// DGEMM offload entry points.
//
// The trailing update of lu2 (mmmulandsub, lu2.c:312-343 -> mydgemm,
// lu2lib.c:2079-2136) is C -= L21 * U12 with K = nb.  Here both operands
// reach shared memory by TMA (cp.async.bulk.tensor, 128-byte swizzle, an
// mbarrier per stage) and are multiplied with the FP64 tensor-core MMA
// (mma.sync m16n8k8 f64; sm_100a has no tcgen05 kind for f64).  Both operands
// are K-contiguous: A is the matrix itself (row-major, K = its columns) and B
// is the transposed U block row written by the TRSM kernel.
//
// k-permutation: the reduction index inside each 8-wide MMA step is permuted
// consistently for A and B so that every thread's two k values are adjacent
// in memory (one 16-byte shared load per fragment row).
#include <cstdlib>

#include "lu2gpu_internal.cuh"

namespace lu2gpu {

// ---------------------------------------------------------------------------
// PTX helpers

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_barrier_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait on an mbarrier phase; false after WAIT_LIMIT_NS.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t *bar, uint32_t parity, int *status, int where)
{
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = globaltimer_ns();
    while (true) {
        if (mbar_try_wait(bar, parity)) return true;
        if (globaltimer_ns() - t0 > WAIT_LIMIT_NS) {
            record_error(status, ERR_MBAR_TIMEOUT, where);
            return false;
        }
    }
}

__device__ __forceinline__ void tma_load_2d(void *dst, const CUtensorMap *map, int x, int y, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            smem_u32(dst)),
        "l"(map), "r"(x), "r"(y), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void dmma_16x8x8(double (&c)[4], double a0, double a1, double a2, double a3, double b0,
                                            double b1)
{
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
        : "d"(a0), "d"(a1), "d"(a2), "d"(a3), "d"(b0), "d"(b1));
}

// 16-byte chunk `chunk` (0..7) of row `row` in a 128-byte-swizzled tile
__device__ __forceinline__ double2 lds_sw128(const uint8_t *tile, int row, int chunk)
{
    return *reinterpret_cast<const double2 *>(tile + row * 128 + ((chunk ^ (row & 7)) << 4));
}

// ---------------------------------------------------------------------------

struct GemmParams {
    int M, N, K;
    int a_x0, a_y0;  // TMA coordinates of A(0,0): x = column, y = row
    int b_x0, b_y0;  // TMA coordinates of Bt(0,0)
    double *C;
    long ldc;
    double alpha, beta;
    int tiles_m, tiles_n, group_m;
    int *status;
};

template <int BM, int BN, int WM, int WN, int STAGES>
struct GemmCfg {
    static constexpr int WARPS_M = BM / WM;
    static constexpr int WARPS_N = BN / WN;
    static constexpr int THREADS = WARPS_M * WARPS_N * 32;
    static constexpr int MT = WM / 16;
    static constexpr int NT = WN / 8;
    static constexpr int A_BYTES = BM * 128;
    static constexpr int B_BYTES = BN * 128;
    static constexpr int STAGE_BYTES = A_BYTES + B_BYTES;
    static constexpr int SMEM = STAGES * STAGE_BYTES + 1024;
    // 4-warp tiles are sized so that two CTAs share an SM
    static constexpr int MINB = (THREADS <= 128) ? 2 : 1;
};

// MODE 0: C = C + A * Bt^T with Bt = -U12^T as the block solve writes it
// (accumulator starts from C): the trailing update C - L21 U12.
// MODE 1: C = alpha * A * Bt^T + beta * C (C not read when beta == 0).
template <int BM, int BN, int WM, int WN, int STAGES, int MODE>
__global__ void __launch_bounds__(GemmCfg<BM, BN, WM, WN, STAGES>::THREADS, GemmCfg<BM, BN, WM, WN, STAGES>::MINB)
    dgemm_tn_kernel(const __grid_constant__ CUtensorMap tmA, const __grid_constant__ CUtensorMap tmB, GemmParams p)
{
    using Cfg = GemmCfg<BM, BN, WM, WN, STAGES>;
    constexpr int MT = Cfg::MT, NT = Cfg::NT;
    extern __shared__ uint8_t smem_raw[];
    __shared__ __align__(8) uint64_t full_bar[STAGES];
    uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int g = lane >> 2, t = lane & 3;
    const int warp_m = warp % Cfg::WARPS_M, warp_n = warp / Cfg::WARPS_M;

    // grouped rasterization: GROUP_M tile-rows share their A tiles in L2
    const int bid = blockIdx.x;
    const int per_group = p.group_m * p.tiles_n;
    const int first_m = (bid / per_group) * p.group_m;
    const int gsize = min(p.tiles_m - first_m, p.group_m);
    const int tm = first_m + (bid % per_group) % gsize;
    const int tn = (bid % per_group) / gsize;
    const int m0 = tm * BM, n0 = tn * BN;
    const int KT = p.K >> 4;

    if (tid == 0) {
        for (int s = 0; s < STAGES; s++) mbar_init(&full_bar[s], 1);
        fence_barrier_init();
    }
    __syncthreads();

    auto issue = [&](int kt, int s) {
        uint8_t *sa = smem + s * Cfg::STAGE_BYTES;
        mbar_expect_tx(&full_bar[s], Cfg::STAGE_BYTES);
        tma_load_2d(sa, &tmA, p.a_x0 + kt * 16, p.a_y0 + m0, &full_bar[s]);
        tma_load_2d(sa + Cfg::A_BYTES, &tmB, p.b_x0 + kt * 16, p.b_y0 + n0, &full_bar[s]);
    };
    if (tid == 0) {
        for (int s = 0; s < STAGES && s < KT; s++) issue(s, s);
    }

    // Fragment row g of every 8-row group is tile row pg = (g>>1) + 4(g&1), for
    // A (M) and B (N) alike: the two rows a quarter-warp reads together are then
    // r and r+4, which the 128-byte swizzle puts in opposite bank halves (rows g
    // and g+1 would share the same 16 banks).  So accumulator c0 (MMA column 2t)
    // is tile column t and c1 (2t+1) is tile column t+4.
    const int pg = (g >> 1) + ((g & 1) << 2);
    double acc[MT][NT][4];
    const int row_base = m0 + warp_m * WM + pg;
    const int col_base = n0 + warp_n * WN + t;
#pragma unroll
    for (int mt = 0; mt < MT; mt++)
#pragma unroll
        for (int nt = 0; nt < NT; nt++)
#pragma unroll
            for (int h = 0; h < 2; h++) {
                double v0 = 0.0, v1 = 0.0;
                if (MODE == 0) {
                    const int m = row_base + mt * 16 + h * 8, n = col_base + nt * 8;
                    if (m < p.M) {
                        const double *cp = p.C + (size_t)m * p.ldc + n;
                        if (n < p.N) v0 = cp[0];
                        if (n + 4 < p.N) v1 = cp[4];
                    }
                }
                acc[mt][nt][2 * h] = v0;
                acc[mt][nt][2 * h + 1] = v1;
            }

    bool ok = true;
    for (int kt = 0; kt < KT; kt++) {
        const int s = kt % STAGES;
        const uint32_t par = (uint32_t)(kt / STAGES) & 1u;
        if (!mbar_wait_bounded(&full_bar[s], par, p.status, 3)) {
            ok = false;
            break;
        }
        const uint8_t *sa = smem + s * Cfg::STAGE_BYTES;
        const uint8_t *sb = sa + Cfg::A_BYTES;
#pragma unroll
        for (int kk = 0; kk < 2; kk++) {
            const int chunk = kk * 4 + t;
            double bf[NT][2];
#pragma unroll
            for (int nt = 0; nt < NT; nt++) {
                const double2 v = lds_sw128(sb, warp_n * WN + nt * 8 + pg, chunk);
                bf[nt][0] = v.x;
                bf[nt][1] = v.y;
            }
#pragma unroll
            for (int mt = 0; mt < MT; mt++) {
                const int r = warp_m * WM + mt * 16 + pg;
                const double2 lo = lds_sw128(sa, r, chunk);
                const double2 hi = lds_sw128(sa, r + 8, chunk);
#pragma unroll
                for (int nt = 0; nt < NT; nt++) dmma_16x8x8(acc[mt][nt], lo.x, hi.x, lo.y, hi.y, bf[nt][0], bf[nt][1]);
            }
        }
        __syncthreads();
        if (tid == 0 && kt + STAGES < KT) issue(kt + STAGES, s);
    }
    if (!ok) return;

#pragma unroll
    for (int mt = 0; mt < MT; mt++)
#pragma unroll
        for (int nt = 0; nt < NT; nt++)
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int m = row_base + mt * 16 + h * 8, n = col_base + nt * 8;
                if (m >= p.M || n >= p.N) continue;
                double *cp = p.C + (size_t)m * p.ldc + n;
                double v0 = acc[mt][nt][2 * h], v1 = acc[mt][nt][2 * h + 1];
                const bool two = n + 4 < p.N;
                if (MODE == 1) {
                    v0 *= p.alpha;
                    v1 *= p.alpha;
                    if (p.beta != 0.0) {
                        v0 += p.beta * cp[0];
                        if (two) v1 += p.beta * cp[4];
                    }
                }
                cp[0] = v0;
                if (two) cp[4] = v1;
            }
}

// ---------------------------------------------------------------------------
// tensor maps (driver entry point fetched through the runtime: the library
// has no link-time dependency on libcuda)

typedef CUresult (*PFN_encodeTiled_t)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                      const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                      CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static PFN_encodeTiled_t encode_fn()
{
    static PFN_encodeTiled_t fn = nullptr;
    if (!fn) {
        void *ptr = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &ptr, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_encodeTiled_t>(ptr);
    }
    return fn;
}

// 2-D FP64 map over `rows` x `cols` (row stride ld doubles), box 16 x box_rows,
// 128-byte swizzle.  Requirements checked here: 16-byte aligned base, ld even.
static cudaError_t make_map(CUtensorMap *m, const double *base, long ld, long rows, long cols, int box_rows)
{
    PFN_encodeTiled_t enc = encode_fn();
    if (!enc) return cudaErrorNotSupported;
    if ((reinterpret_cast<uintptr_t>(base) & 15) || (ld & 1) || rows <= 0 || cols <= 0) return cudaErrorInvalidValue;
    cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)ld * sizeof(double)};
    cuuint32_t box[2] = {16, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 2, const_cast<double *>(base), dims, strides, box, estr,
                     CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

template <int BM, int BN, int WM, int WN, int STAGES, int MODE>
static cudaError_t run_gemm(const CUtensorMap &ta, const CUtensorMap &tb, GemmParams p, cudaStream_t st)
{
    using Cfg = GemmCfg<BM, BN, WM, WN, STAGES>;
    auto kern = dgemm_tn_kernel<BM, BN, WM, WN, STAGES, MODE>;
    // per-device attribute; cheap to repeat
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, Cfg::SMEM);
    if (e != cudaSuccess) return e;
    p.tiles_m = (p.M + BM - 1) / BM;
    p.tiles_n = (p.N + BN - 1) / BN;
    p.group_m = 16;
    const long tiles = (long)p.tiles_m * p.tiles_n;
    if (tiles <= 0) return cudaSuccess;
    if (tiles > 0x7fffffffL) return cudaErrorInvalidConfiguration;
    count_launch();
    kern<<<(unsigned)tiles, Cfg::THREADS, Cfg::SMEM, st>>>(ta, tb, p);
    return cudaGetLastError();
}

// Tile shapes: wide trailing updates use 128x128 (8 warps of 64x32); narrow
// right parts inside the panel recursion use 128x32.
#define LU2_GEMM_WIDE 128, 128, 64, 32, 4
#define LU2_GEMM_WIDE2 128, 64, 64, 32, 4
#define LU2_GEMM_NARROW 128, 32, 32, 32, 4

// wide tile shape: 1 = 128x64 with two CTAs per SM (default: one CTA's
// prologue/epilogue overlaps the other's main loop; 89% of cuBLAS DGEMM at
// N=32768 against 73% for 128x128), 0 = 128x128 with one CTA per SM.
// LU2GPU_GEMM_WIDE=0 selects the latter (read once).
static int wide_config()
{
    static int cfg = -1;
    if (cfg < 0) {
        const char *e = getenv("LU2GPU_GEMM_WIDE");
        cfg = (e && e[0] == '0') ? 0 : 1;
    }
    return cfg;
}

// p.K is the loop extent (a multiple of 16); the maps' own extents
// (a_cols, b_cols) bound what is read, the rest of a box reads as zero.
template <int MODE>
static cudaError_t gemm_dispatch(const double *a, long lda, long a_rows, long a_cols, int a_row0, int a_col0,
                                 const double *bt, long ldb, long b_rows, long b_cols, GemmParams p, cudaStream_t st)
{
    if (p.M <= 0 || p.N <= 0) return cudaSuccess;
    if (p.K <= 0 || (p.K & 15)) return cudaErrorInvalidValue;
    const bool narrow = p.N <= 64;
    const int wide = wide_config();
    const int bm = 128, bn = narrow ? 32 : (wide == 1 ? 64 : 128);
    CUtensorMap ta, tb;
    cudaError_t e = make_map(&ta, a, lda, a_rows, a_cols, bm);
    if (e != cudaSuccess) return e;
    e = make_map(&tb, bt, ldb, b_rows, b_cols, bn);
    if (e != cudaSuccess) return e;
    p.a_x0 = a_col0;
    p.a_y0 = a_row0;
    p.b_x0 = 0;
    p.b_y0 = 0;
    if (narrow) return run_gemm<LU2_GEMM_NARROW, MODE>(ta, tb, p, st);
    if (wide == 1) return run_gemm<LU2_GEMM_WIDE2, MODE>(ta, tb, p, st);
    return run_gemm<LU2_GEMM_WIDE, MODE>(ta, tb, p, st);
}

cudaError_t launch_dgemm_update(const double *a, long ld, int a_rows, int a_row0, int a_col0, const double *bt,
                                double *c, long ldc, int M, int N, int K, int *status, cudaStream_t st)
{
    GemmParams p{};
    p.M = M;
    p.N = N;
    p.K = K;
    p.C = c;
    p.ldc = ldc;
    p.alpha = -1.0;
    p.beta = 1.0;
    p.status = status;
    // A covers the whole matrix: columns [0, ld) and rows [0, a_rows); rows of
    // a tile past a_rows read as zero.
    return gemm_dispatch<0>(a, ld, a_rows, ld, a_row0, a_col0, bt, K, N, K, p, st);
}

cudaError_t launch_dgemm_general(const double *x, long ldx, const double *y, long ldy, double *c, long ldc, int M,
                                 int N, int K, double alpha, double beta, int *status, cudaStream_t st)
{
    GemmParams p{};
    p.M = M;
    p.N = N;
    p.K = (K + 15) & ~15;
    p.C = c;
    p.ldc = ldc;
    p.alpha = alpha;
    p.beta = beta;
    p.status = status;
    return gemm_dispatch<1>(x, ldx, M, K, 0, 0, y, ldy, N, K, p, st);
}

// ---------------------------------------------------------------------------
__global__ void transpose_kernel(const double *__restrict__ in, long ldi, double *__restrict__ out, long ldo, int rows,
                                 int cols)
{
    __shared__ double tile[32][33];
    const int bx = blockIdx.x * 32, by = blockIdx.y * 32;
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int r = by + k, c = bx + threadIdx.x;
        if (r < rows && c < cols) tile[k][threadIdx.x] = in[(size_t)r * ldi + c];
    }
    __syncthreads();
    for (int k = threadIdx.y; k < 32; k += blockDim.y) {
        const int c = bx + k, r = by + threadIdx.x;
        if (r < rows && c < cols) out[(size_t)c * ldo + r] = tile[threadIdx.x][k];
    }
}

cudaError_t launch_transpose(const double *in, long ldi, double *out, long ldo, int rows, int cols, cudaStream_t st)
{
    if (rows <= 0 || cols <= 0) return cudaSuccess;
    dim3 grid((cols + 31) / 32, (rows + 31) / 32);
    if (grid.y > 65535) return cudaErrorInvalidConfiguration;
    count_launch();
    transpose_kernel<<<grid, dim3(32, 8), 0, st>>>(in, ldi, out, ldo, rows, cols);
    return cudaGetLastError();
}

}  // namespace lu2gpu
