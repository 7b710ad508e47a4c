// kernels_panel.cu -- panel kernels: the shared-memory leaf factorization
// with warp-shuffle pivot search, the pivot-apply (swap + 1/pivot scale) and
// the unit-lower triangular solve of the U block row.
//
// Reference behaviour followed (telmin/lu2):
//   leaf        lu2tlib.c:1041-1066 (column_decomposition) inside the slab
//               recursion lu2tlib.c:1095-1128; pivot search lu2tlib.c:42-52
//   swap+scale  lu2.c:251-291 (swaprows_simple_with_scale), lu2.c:541-554,
//               lu2.c:1107-1118
//   trsm        lu2.c:485-521 (solve_triangle: U12 = L11^{-1} A12)
#include <climits>

#include "lu2gpu_internal.cuh"

namespace lu2gpu {

constexpr int LEAF_W = 16;          // widest leaf (lu2.c:1097: m <= 16)
constexpr int LEAF_THREADS = 256;
constexpr int LEAF_LDS = LEAF_W + 1;  // padded smem row: conflict-free column walks
constexpr int LEAF_MIN_ROWS = 128;    // rows per CTA below which fewer CTAs are used
constexpr int LEAF_SMEM_MAX = 200 * 1024;

struct LeafParams {
    double *a;
    long ld;
    int n, c0, w, rows_per_cta, mode, goff;
    int *ipiv;
    double *dinv;
    LeafBuffers buf;
    int *status;
};

// Grid-wide barrier for a cooperative launch.  Monotonic counter (zeroed before
// the launch); waits at most WAIT_LIMIT_NS, then records an error and lets
// every CTA leave.  Returns false on timeout or when another CTA failed.
__device__ __forceinline__ bool grid_barrier(unsigned *bar, unsigned target, int *status, int where)
{
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        __threadfence();
        atomicAdd(bar, 1u);
        unsigned long long t0 = globaltimer_ns();
        unsigned spins = 0;
        while (true) {
            unsigned v;
            asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(bar) : "memory");
            if (v >= target) break;
            if ((++spins & 63u) == 0) {
                if (*(volatile int *)&status[1] != 0) {
                    ok = 0;
                    break;
                }
                if (globaltimer_ns() - t0 > WAIT_LIMIT_NS) {
                    record_error(status, ERR_BARRIER_TIMEOUT, where);
                    ok = 0;
                    break;
                }
            }
        }
        __threadfence();
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

// Block-wide argmax; every thread returns the block result.
__device__ __forceinline__ void block_argmax(double &v, int &i)
{
    __shared__ double s_v[LEAF_THREADS / 32];
    __shared__ int s_i[LEAF_THREADS / 32];
    warp_argmax(v, i);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
        s_v[warp] = v;
        s_i[warp] = i;
    }
    __syncthreads();
    if (warp == 0) {
        v = lane < (int)(blockDim.x >> 5) ? s_v[lane] : -1.0;
        i = lane < (int)(blockDim.x >> 5) ? s_i[lane] : INT_MAX;
        warp_argmax(v, i);
        if (lane == 0) {
            s_v[0] = v;
            s_i[0] = i;
        }
    }
    __syncthreads();
    v = s_v[0];
    i = s_i[0];
    __syncthreads();
}

// One CTA per slice of rows; the whole leaf slab (rows c0..n-1, w <= 16
// columns) lives in shared memory across the grid.  Per column: local argmax
// -> publish candidate (|a|, row, row values) -> grid barrier -> every CTA
// picks the same winner -> swap/scale -> rank-1 update of its own rows.
__global__ void __launch_bounds__(LEAF_THREADS) leaf_kernel(LeafParams P)
{
    extern __shared__ double slab[];
    __shared__ double s_prow[LEAF_W], s_rowc[LEAF_W];
    const int G = gridDim.x, bid = blockIdx.x, tid = threadIdx.x;
    const int w = P.w, c0 = P.c0;
    const int rb = c0 + bid * P.rows_per_cta;
    const int re = min(P.n, rb + P.rows_per_cta);
    const int nr = max(0, re - rb);

    for (int idx = tid; idx < nr * LEAF_W; idx += LEAF_THREADS) {
        const int lr = idx / LEAF_W, j = idx - lr * LEAF_W;
        slab[lr * LEAF_LDS + j] = (j < w) ? P.a[(size_t)(rb + lr) * P.ld + c0 + j] : 0.0;
    }
    __syncthreads();

    bool ok = true;
    for (int ip = 0; ip < w && ok; ip++) {
        const int c = c0 + ip, par = ip & 1;
        // REF mode: the second column of each aligned 2-column leaf is pivoted
        // on the first column's values (lu2tlib.c:1052 with findpivot scanning a[0]).
        int sc = ip;
        if (P.mode == PIVOT_REF && ((c + P.goff) & 1) && ip > 0) sc = ip - 1;
        if (P.mode == PIVOT_REF_FIRST) sc = 0;

        double bv = -1.0;
        int bi = INT_MAX;
        for (int lr = max(0, c - rb) + tid; lr < nr; lr += LEAF_THREADS) {
            const double v = fabs(slab[lr * LEAF_LDS + sc]);
            if (v > bv) {  // rows visited in increasing order: keeps the first max
                bv = v;
                bi = rb + lr;
            }
        }
        block_argmax(bv, bi);

        double *xrow = P.buf.xrow + ((size_t)par * G + bid) * LEAF_W;
        if (tid < LEAF_W) {
            const double v = (bi != INT_MAX) ? slab[(bi - rb) * LEAF_LDS + tid] : 0.0;
            __stcg(xrow + tid, v);
            if (c >= rb && c < re) __stcg(P.buf.rowc + par * LEAF_W + tid, slab[(c - rb) * LEAF_LDS + tid]);
        }
        if (tid == 0) {
            __stcg(P.buf.xval + par * G + bid, bv);
            __stcg(P.buf.xidx + par * G + bid, bi);
        }
        ok = grid_barrier(P.buf.bar, (unsigned)G * (unsigned)(ip + 1), P.status, 1);
        if (!ok) break;

        double gv = -1.0;
        int gi = INT_MAX;
        for (int s = tid; s < G; s += LEAF_THREADS) {
            const double v = __ldcg(P.buf.xval + par * G + s);
            const int i = __ldcg(P.buf.xidx + par * G + s);
            if (argmax_better(v, i, gv, gi)) {
                gv = v;
                gi = i;
            }
        }
        block_argmax(gv, gi);
        // no finite candidate at all (a NaN column): keep row c in place
        const int p = (gi == INT_MAX) ? c : gi;
        const int owner = (p - c0) / P.rows_per_cta;
        if (tid < LEAF_W) {
            s_rowc[tid] = __ldcg(P.buf.rowc + par * LEAF_W + tid);
            s_prow[tid] = (p == c) ? s_rowc[tid] : __ldcg(P.buf.xrow + ((size_t)par * G + owner) * LEAF_W + tid);
        }
        __syncthreads();
        const double d = s_prow[ip];
        const bool zero = (d == 0.0);
        const double inv = zero ? 1.0 : 1.0 / d;
        if (bid == 0 && tid == 0) {
            P.ipiv[c] = p + P.goff;
            P.dinv[c] = inv;
            if (zero) atomicMin(&P.status[0], c + 1);
        }
        if (tid < w) {
            if (p != c && p >= rb && p < re) slab[(p - rb) * LEAF_LDS + tid] = s_rowc[tid];
            if (c >= rb && c < re)
                slab[(c - rb) * LEAF_LDS + tid] = (tid == ip || zero) ? s_prow[tid] : s_prow[tid] * inv;
        }
        __syncthreads();
        if (!zero) {
            for (int lr = max(0, c + 1 - rb) + tid; lr < nr; lr += LEAF_THREADS) {
                double *row = slab + lr * LEAF_LDS;
                const double l = row[ip];
                for (int j = ip + 1; j < w; j++) row[j] -= l * (s_prow[j] * inv);
            }
        }
        __syncthreads();
    }

    for (int idx = tid; idx < nr * LEAF_W; idx += LEAF_THREADS) {
        const int lr = idx / LEAF_W, j = idx - lr * LEAF_W;
        if (j < w) P.a[(size_t)(rb + lr) * P.ld + c0 + j] = slab[lr * LEAF_LDS + j];
    }
}

int leaf_max_ctas(int device)
{
    int sms = 0, per_sm = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    cudaFuncSetAttribute(leaf_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, LEAF_SMEM_MAX);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, leaf_kernel, LEAF_THREADS, LEAF_SMEM_MAX);
    if (per_sm < 1) per_sm = 1;
    return sms * per_sm;
}

cudaError_t launch_leaf(double *a, long ld, int n, int c0, int w, int mode, int goff, int *ipiv, double *dinv,
                        const LeafBuffers &buf, int *status, int max_ctas, cudaStream_t st)
{
    if (w <= 0) return cudaSuccess;
    if (w > LEAF_W) return cudaErrorInvalidValue;
    const int rows = n - c0;
    int G = (rows + LEAF_MIN_ROWS - 1) / LEAF_MIN_ROWS;
    if (G > max_ctas) G = max_ctas;
    if (G < 1) G = 1;
    const int rpc = (rows + G - 1) / G;
    G = (rows + rpc - 1) / rpc;
    const size_t smem = (size_t)rpc * LEAF_LDS * sizeof(double);
    if (smem > (size_t)LEAF_SMEM_MAX) return cudaErrorInvalidConfiguration;
    cudaError_t e = cudaMemsetAsync(buf.bar, 0, sizeof(unsigned), st);
    if (e != cudaSuccess) return e;
    LeafParams P{a, ld, n, c0, w, rpc, mode, goff, ipiv, dinv, buf, status};
    void *args[] = {&P};
    count_launch();
    return cudaLaunchCooperativeKernel((const void *)leaf_kernel, dim3(G), dim3(LEAF_THREADS), args, smem, st);
}

// ---------------------------------------------------------------------------
// Pivot apply: every thread owns one column and replays the swaps in order,
// scaling row k right after its swap (row k is final once swapped, since
// later pivots only exchange rows > k).
__global__ void laswp_scale_kernel(double *a, long ld, int k0, int k1, const int *__restrict__ ipiv, int goff,
                                   const double *__restrict__ dinv, int cs, int ce, int scale)
{
    const int j = cs + blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= ce) return;
    for (int k = k0; k < k1; k++) {
        const int p = __ldg(ipiv + k) - goff;
        double *rk = a + (size_t)k * ld + j;
        double v;
        if (p != k) {
            double *rp = a + (size_t)p * ld + j;
            v = *rp;
            *rp = *rk;
        } else {
            v = *rk;
        }
        *rk = scale ? v * __ldg(dinv + k) : v;
    }
}

cudaError_t launch_laswp_scale(double *a, long ld, int k0, int k1, const int *ipiv, int goff, const double *dinv,
                               int cs, int ce, bool scale, cudaStream_t st)
{
    if (ce <= cs || k1 <= k0) return cudaSuccess;
    const int threads = 128;
    const int blocks = (ce - cs + threads - 1) / threads;
    count_launch();
    laswp_scale_kernel<<<blocks, threads, 0, st>>>(a, ld, k0, k1, ipiv, goff, dinv, cs, ce, scale ? 1 : 0);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Unit-lower triangular solve of a 32-column strip of the block row, staged
// in shared memory; 16-row diagonal blocks solved by one warp, the rows below
// updated by all warps with the 16-wide row segments of T.
constexpr int TRSM_TW = 32;
constexpr int TRSM_LDS = TRSM_TW + 1;
constexpr int TRSM_BK = 16;

__global__ void __launch_bounds__(256) trsm_unit_lower_kernel(double *a, long ld, int r0, int K, int cs, int ce,
                                                              double *bt)
{
    extern __shared__ double X[];  // K x TRSM_LDS
    __shared__ double Td[TRSM_BK][TRSM_BK + 1];
    const int col = threadIdx.x & 31, rg = threadIdx.x >> 5;
    const int j = cs + blockIdx.x * TRSM_TW + col;
    const bool jok = j < ce;
    for (int r = rg; r < K; r += 8) X[r * TRSM_LDS + col] = jok ? a[(size_t)(r0 + r) * ld + j] : 0.0;
    const double *T = a + (size_t)r0 * ld + r0;
    for (int lb = 0; lb < K; lb += TRSM_BK) {
        const int bk = min(TRSM_BK, K - lb);
        {
            const int rr = threadIdx.x >> 4, cc = threadIdx.x & 15;
            Td[rr][cc] = (rr < bk && cc < rr) ? T[(size_t)(lb + rr) * ld + lb + cc] : 0.0;
        }
        __syncthreads();
        if (rg == 0) {
            for (int r = 1; r < bk; r++) {
                double s = X[(lb + r) * TRSM_LDS + col];
                for (int l = 0; l < r; l++) s -= Td[r][l] * X[(lb + l) * TRSM_LDS + col];
                X[(lb + r) * TRSM_LDS + col] = s;
            }
        }
        __syncthreads();
        double xb[TRSM_BK];
#pragma unroll
        for (int l = 0; l < TRSM_BK; l++) xb[l] = (l < bk) ? X[(lb + l) * TRSM_LDS + col] : 0.0;
        for (int r = lb + bk + rg; r < K; r += 8) {
            const double *Tr = T + (size_t)r * ld + lb;
            double s = 0.0;
            if (bk == TRSM_BK) {
#pragma unroll
                for (int l = 0; l < TRSM_BK; l++) s += __ldg(Tr + l) * xb[l];
            } else {
                for (int l = 0; l < bk; l++) s += __ldg(Tr + l) * xb[l];
            }
            X[r * TRSM_LDS + col] -= s;
        }
        __syncthreads();
    }
    for (int r = rg; r < K; r += 8)
        if (jok) a[(size_t)(r0 + r) * ld + j] = X[r * TRSM_LDS + col];
    const int jbase = blockIdx.x * TRSM_TW;
    for (int idx = threadIdx.x; idx < TRSM_TW * K; idx += 256) {
        const int cc = idx / K, r = idx - cc * K;
        if (cs + jbase + cc < ce) bt[(size_t)(jbase + cc) * K + r] = X[r * TRSM_LDS + cc];
    }
}

cudaError_t launch_trsm_unit_lower(double *a, long ld, int r0, int K, int cs, int ce, double *bt, cudaStream_t st)
{
    if (ce <= cs || K <= 0) return cudaSuccess;
    const size_t smem = (size_t)K * TRSM_LDS * sizeof(double);
    if (smem > 200 * 1024) return cudaErrorInvalidValue;
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(trsm_unit_lower_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             200 * 1024);
        if (e != cudaSuccess) return e;
    }
    const int blocks = (ce - cs + TRSM_TW - 1) / TRSM_TW;
    count_launch();
    trsm_unit_lower_kernel<<<blocks, 256, smem, st>>>(a, ld, r0, K, cs, ce, bt);
    return cudaGetLastError();
}

}  // namespace lu2gpu
