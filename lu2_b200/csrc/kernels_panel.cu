// kernels_panel.cu -- panel kernels: the pivot-apply (swap + 1/pivot scale)
// and the unit-lower triangular solve of the U block row (the leaf is in
// kernels_leaf.cu).
//
// Reference behaviour followed (telmin/lu2):
//   swap+scale  lu2.c:251-291 (swaprows_simple_with_scale), lu2.c:541-554,
//               lu2.c:1107-1118
//   trsm        lu2.c:485-521 (solve_triangle: U12 = L11^{-1} A12)
#include <climits>
#include <cstdlib>

#include <cuda_bf16.h>

#include "lu2gpu_internal.cuh"

namespace lu2gpu {

// ---------------------------------------------------------------------------
// Pivot apply (lu2's sequence of row exchanges, each pivot row scaled by
// 1/pivot right after its exchange; row k is final once exchanged, since
// later pivots only exchange rows > k).
//
// The npiv exchanges (row k <-> row p_k, k = k0..k1-1 in order, p_k >= k)
// compose to one permutation of at most 2 npiv rows, which every CTA derives
// in parallel in shared memory:
//   A(k)  = the original row sitting at position k just before step k: the
//           row A(i) moved there by the latest step i < k with p_i = k, else k
//           itself -- a chain i -> k resolved by pointer jumping
//           (ceil(log2 npiv) rounds);
//   row k (k0 <= k < k1) finally holds what position p_k held before step k:
//           A(k) if p_k = k, else A(j) for the latest j < k with p_j = p_k,
//           else the original row p_k;
//   row q >= k1 (some p_j = q) finally holds A(j) for the last such j.
// Then each CTA gathers the source rows of its column chunks (one 128-byte
// line per row, 16-byte loads, eight in flight per thread) into shared
// memory and scatters them to their destinations, scaling the pivot rows.
// Pivots outside [k, nrows) are refused (ERR_BAD_ARG, nothing written), and
// nothing is done once an earlier wait of the same call has given up (its
// pivots were never written).
constexpr int SWAP_THREADS = 256;
constexpr int SWAP_MAX_PIV = 512;

template <typename T, int V>
struct SwapVec;
template <>
struct SwapVec<double, 2> {
    using type = double2;
};
template <>
struct SwapVec<float, 4> {
    using type = float4;
};
template <typename T>
struct SwapVec<T, 1> {
    using type = T;
};

template <typename T, int V>
__device__ __forceinline__ void swap_ld(const T *p, int avail, T *out)
{
    if (avail >= V) {
        const typename SwapVec<T, V>::type x = *reinterpret_cast<const typename SwapVec<T, V>::type *>(p);
        const T *e = reinterpret_cast<const T *>(&x);
#pragma unroll
        for (int q = 0; q < V; q++) out[q] = e[q];
    } else {
#pragma unroll
        for (int q = 0; q < V; q++) out[q] = (q < avail) ? p[q] : T(0);
    }
}

template <typename T, int V>
__device__ __forceinline__ void swap_st(T *p, int avail, const T *in)
{
    if (avail >= V) {
        typename SwapVec<T, V>::type x;
        T *e = reinterpret_cast<T *>(&x);
#pragma unroll
        for (int q = 0; q < V; q++) e[q] = in[q];
        *reinterpret_cast<typename SwapVec<T, V>::type *>(p) = x;
    } else {
#pragma unroll
        for (int q = 0; q < V; q++)
            if (q < avail) p[q] = in[q];
    }
}

// The composed permutation of the exchanges k <-> ipiv[k] - goff, k = k0..k1-1
// (see above), built by the whole CTA: slot i moves row src[i] to row dst[i];
// slots 0..npiv-1 are the rows k0..k1-1 (in order), the others the rows >= k1
// the exchanges name.  P and A: npiv ints each, src and dst: 2 npiv each.
// Returns false (every thread) when the call must do nothing: an earlier wait
// gave up, or a pivot lies outside [k, nrows) (then ERR_BAD_ARG is recorded).
__device__ bool swap_plan(const int *__restrict__ ipiv, int goff, int k0, int k1, int nrows, int *P, int *A, int *src,
                          int *dst, int *p_nslot, int *p_bad, int *status)
{
    const int npiv = k1 - k0, tid = threadIdx.x, nth = blockDim.x;
    int &s_nslot = *p_nslot, &s_bad = *p_bad;
    if (status && *(volatile int *)&status[1] != 0) return false;
    if (tid == 0) {
        s_bad = 0;
        s_nslot = npiv;
    }
    __syncthreads();
    for (int t = tid; t < npiv; t += nth) {
        const int p = __ldg(ipiv + k0 + t) - goff;
        P[t] = p;
        A[t] = -1;
        if (p < k0 + t || p >= nrows) s_bad = 1;
    }
    __syncthreads();
    if (s_bad) {
        if (blockIdx.x == 0 && tid == 0 && status) record_error(status, ERR_BAD_ARG, 3);
        return false;
    }
    for (int i = tid; i < npiv; i += nth) {
        const int q = P[i];
        if (q != k0 + i && q < k1) atomicMax(&A[q - k0], i);
    }
    __syncthreads();
    for (int t = tid; t < npiv; t += nth)
        if (A[t] < 0) A[t] = -(k0 + t) - 1;
    __syncthreads();
    {
        // pointer jumping, double-buffered through src (free until the slots
        // are written): after r rounds every pointer has advanced 2^r links or
        // reached its root, and a chain has fewer than npiv links
        int *cur = A, *nxt = src;
        for (int span = 1; span < npiv; span <<= 1) {
            for (int t = tid; t < npiv; t += nth) {
                const int v = cur[t];
                nxt[t] = (v >= 0) ? cur[v] : v;
            }
            __syncthreads();
            int *tmp = cur;
            cur = nxt;
            nxt = tmp;
        }
        if (cur != A) {
            for (int t = tid; t < npiv; t += nth) A[t] = cur[t];
            __syncthreads();
        }
    }
    for (int t = tid; t < npiv; t += nth) {
        const int p = P[t], k = k0 + t;
        int s;
        if (p == k) {
            s = -A[t] - 1;
        } else {
            int j = t - 1;
            while (j >= 0 && P[j] != p) j--;
            s = (j >= 0) ? -A[j] - 1 : p;
            if (p >= k1) {
                int q = t + 1;
                while (q < npiv && P[q] != p) q++;
                if (q == npiv) {  // the last exchange that names row p
                    const int e = atomicAdd(&s_nslot, 1);
                    src[e] = -A[t] - 1;
                    dst[e] = p;
                }
            }
        }
        src[t] = s;
        dst[t] = k;
    }
    __syncthreads();
    return true;
}

// NS > 0: every thread keeps its NS row segments of a chunk in registers
// (all NS loads in flight at once, one barrier per chunk, no staging in
// shared memory; used while the slots fit, nslot <= NS * rows per pass);
// NS = 0: the chunk is staged in shared memory.
template <typename T, int V, int NS>
__global__ void __launch_bounds__(SWAP_THREADS, NS > 0 ? 2 : 1)
    laswp_scale_kernel(T *a, long ld, int nrows, int k0, int k1, const int *__restrict__ ipiv, int goff,
                       const T *__restrict__ dinv, int cs, int ce, int scale, int *status)
{
    constexpr int COLS = 128 / (int)sizeof(T);  // one 128-byte line of a row per chunk
    constexpr int TPR = COLS / V;               // threads per row segment
    constexpr int RPP = SWAP_THREADS / TPR;     // rows per pass
    constexpr int U = 8;                        // loads in flight per thread
    extern __shared__ __align__(16) unsigned char swap_smem[];
    const int npiv = k1 - k0;
    T *S = reinterpret_cast<T *>(swap_smem);     // [2 npiv][COLS] staged row segments (NS = 0)
    int *P = reinterpret_cast<int *>(S + (NS > 0 ? 0 : (size_t)2 * npiv * COLS));
    int *A = P + npiv;        // chain pointer (>= 0) or root code -(row)-1
    int *src = A + npiv;      // [2 npiv] source row of each slot
    int *dst = src + 2 * npiv; // [2 npiv] destination row of each slot
    __shared__ int s_nslot, s_bad;
    const int tid = threadIdx.x;

    if (!swap_plan(ipiv, goff, k0, k1, nrows, P, A, src, dst, &s_nslot, &s_bad, status)) return;
    const int nslot = s_nslot;
    const int cq = (tid % TPR) * V, r0 = tid / TPR;
    const int nchunk = (ce - cs + COLS - 1) / COLS;
    if constexpr (NS > 0) {
        for (int chunk = blockIdx.x; chunk < nchunk; chunk += gridDim.x) {
            const int j = cs + chunk * COLS + cq;
            const int avail = ce - j;
            T v[NS][V];
#pragma unroll
            for (int u = 0; u < NS; u++) {
                const int s = r0 + u * RPP;
                if (s < nslot && avail > 0) swap_ld<T, V>(a + (size_t)src[s] * ld + j, avail, v[u]);
            }
            __syncthreads();  // every gather of this chunk's columns precedes every scatter to them
#pragma unroll
            for (int u = 0; u < NS; u++) {
                const int s = r0 + u * RPP;
                if (s < nslot && avail > 0) {
                    if (scale && s < npiv) {
                        const T d = __ldg(dinv + k0 + s);
#pragma unroll
                        for (int q = 0; q < V; q++) v[u][q] *= d;
                    }
                    swap_st<T, V>(a + (size_t)dst[s] * ld + j, avail, v[u]);
                }
            }
        }
    } else {
    for (int chunk = blockIdx.x; chunk < nchunk; chunk += gridDim.x) {
        const int j = cs + chunk * COLS + cq;
        const int avail = ce - j;
        for (int s0 = r0; s0 < nslot; s0 += U * RPP) {
            T v[U][V];
#pragma unroll
            for (int u = 0; u < U; u++) {
                const int s = s0 + u * RPP;
                if (s < nslot && avail > 0) {
                    swap_ld<T, V>(a + (size_t)src[s] * ld + j, avail, v[u]);
                } else {
#pragma unroll
                    for (int q = 0; q < V; q++) v[u][q] = T(0);
                }
            }
#pragma unroll
            for (int u = 0; u < U; u++) {
                const int s = s0 + u * RPP;
                if (s < nslot) swap_st<T, V>(S + (size_t)s * COLS + cq, V, v[u]);
            }
        }
        __syncthreads();
        if (avail > 0) {
            for (int s = r0; s < nslot; s += RPP) {
                T v[V];
                swap_ld<T, V>(S + (size_t)s * COLS + cq, V, v);
                if (scale && s < npiv) {
                    const T d = __ldg(dinv + k0 + s);
#pragma unroll
                    for (int q = 0; q < V; q++) v[q] *= d;
                }
                swap_st<T, V>(a + (size_t)dst[s] * ld + j, avail, v);
            }
        }
        __syncthreads();
    }
    }
}

template <typename T, int V, int NS>
static cudaError_t launch_laswp_v(T *a, long ld, int nrows, int k0, int k1, const int *ipiv, int goff, const T *dinv,
                                  int cs, int ce, bool scale, int *status, cudaStream_t st)
{
    constexpr int COLS = 128 / (int)sizeof(T);
    const int npiv = k1 - k0;
    const size_t smem = (NS > 0 ? 0 : (size_t)2 * npiv * COLS * sizeof(T)) + (size_t)6 * npiv * sizeof(int);
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(laswp_scale_kernel<T, V, NS>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        if (e != cudaSuccess) return e;
    }
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int per_sm = NS > 0 ? 2 : (int)((220 * 1024) / (smem + 1024));
    per_sm = per_sm < 1 ? 1 : (per_sm > 4 ? 4 : per_sm);
    int blocks = (ce - cs + COLS - 1) / COLS;
    if (blocks > per_sm * sms) blocks = per_sm * sms;
    count_launch();
    laswp_scale_kernel<T, V, NS><<<blocks, SWAP_THREADS, smem, st>>>(a, ld, nrows, k0, k1, ipiv, goff, dinv, cs,
                                                                      ce, scale ? 1 : 0, status);
    return cudaGetLastError();
}

// registers while 2 npiv slots fit NS passes of SWAP_THREADS / (COLS / V) rows
template <typename T, int V>
static cudaError_t launch_laswp_pick(T *a, long ld, int nrows, int k0, int k1, const int *ipiv, int goff,
                                     const T *dinv, int cs, int ce, bool scale, int *status, cudaStream_t st)
{
    constexpr int RPP = SWAP_THREADS / ((128 / (int)sizeof(T)) / V);
    constexpr int NSR = (V > 1) ? 16 : 0;  // 16 passes: 512 slots (npiv <= 256) at 16-byte accesses
    if (NSR > 0 && 2 * (k1 - k0) <= NSR * RPP)
        return launch_laswp_v<T, V, NSR>(a, ld, nrows, k0, k1, ipiv, goff, dinv, cs, ce, scale, status, st);
    return launch_laswp_v<T, V, 0>(a, ld, nrows, k0, k1, ipiv, goff, dinv, cs, ce, scale, status, st);
}

template <typename T>
static cudaError_t launch_laswp_scale_t(T *a, long ld, int nrows, int k0, int k1, const int *ipiv, int goff,
                                        const T *dinv, int cs, int ce, bool scale, int *status, cudaStream_t st)
{
    if (ce <= cs || k1 <= k0) return cudaSuccess;
    if (k1 - k0 > SWAP_MAX_PIV || k0 < 0 || k1 > nrows) return cudaErrorInvalidValue;
    constexpr int VW = 16 / (int)sizeof(T);
    // 16-byte accesses when every row segment starts on a 16-byte boundary
    if ((reinterpret_cast<uintptr_t>(a) & 15) == 0 && ld % VW == 0 && cs % VW == 0)
        return launch_laswp_pick<T, VW>(a, ld, nrows, k0, k1, ipiv, goff, dinv, cs, ce, scale, status, st);
    return launch_laswp_pick<T, 1>(a, ld, nrows, k0, k1, ipiv, goff, dinv, cs, ce, scale, status, st);
}

cudaError_t launch_laswp_scale(double *a, long ld, int nrows, int k0, int k1, const int *ipiv, int goff,
                               const double *dinv, int cs, int ce, bool scale, int *status, cudaStream_t st)
{
    return launch_laswp_scale_t(a, ld, nrows, k0, k1, ipiv, goff, dinv, cs, ce, scale, status, st);
}

cudaError_t launch_laswp_scale(float *a, long ld, int nrows, int k0, int k1, const int *ipiv, int goff,
                               const float *dinv, int cs, int ce, bool scale, int *status, cudaStream_t st)
{
    return launch_laswp_scale_t(a, ld, nrows, k0, k1, ipiv, goff, dinv, cs, ce, scale, status, st);
}

// ---------------------------------------------------------------------------
// Unit-lower triangular solve of a 32-column strip of the block row, staged
// in shared memory.  T is consumed in 16-column blocks: each block of T
// (rows lb..K-1) is first copied to shared memory with coalesced 128-byte row
// loads, the 16x16 diagonal block is solved by one lane per column in
// registers, and the rows below are updated from the staged copy.
constexpr int TRSM_TW = 32;
constexpr int TRSM_LDS = TRSM_TW + 1;
constexpr int TRSM_BK = 16;
constexpr int TRSM_TLD = TRSM_BK + 1;

// T: the unit lower triangle (strict lower part used), row stride ldt; X: the
// K x ncols block (row stride ldx) solved in place; bt (optional) receives
// X^T * bt_scale converted to BT (double, float or bf16), negated when bt_neg
// (the FP64 trailing update reads -U12^T and adds).
template <typename E, typename BT>
__global__ void __launch_bounds__(256) trsm_unit_lower_kernel(const E *T, long ldt, E *Xg, long ldx, int K, int ncols,
                                                              BT *bt, const float *bt_scale, int bt_neg)
{
    extern __shared__ __align__(16) unsigned char trsm_smem[];
    E *X = reinterpret_cast<E *>(trsm_smem);  // K x TRSM_LDS, then Ts: K x TRSM_TLD
    E *Ts = X + (size_t)K * TRSM_LDS;
    const int col = threadIdx.x & 31, rg = threadIdx.x >> 5;
    const int j = blockIdx.x * TRSM_TW + col;
    const bool jok = j < ncols;
    for (int r = rg; r < K; r += 8) X[r * TRSM_LDS + col] = jok ? Xg[(size_t)r * ldx + j] : 0.0;
    for (int lb = 0; lb < K; lb += TRSM_BK) {
        const int bk = min(TRSM_BK, K - lb);
        __syncthreads();  // previous block's readers of Ts are done
        {
            const int cc = threadIdx.x & 15;
            for (int r = lb + (threadIdx.x >> 4); r < K; r += 16)
                Ts[(r - lb) * TRSM_TLD + cc] = (cc < bk) ? T[(size_t)r * ldt + lb + cc] : 0.0;
        }
        __syncthreads();
        // the bk x bk unit triangle: one lane of warp 0 per column, in
        // registers, without barriers (same operations in the same order as
        // the row-by-row elimination)
        if (rg == 0) {
            E xd[TRSM_BK];
#pragma unroll
            for (int l = 0; l < TRSM_BK; l++) xd[l] = (l < bk) ? X[(lb + l) * TRSM_LDS + col] : E(0);
#pragma unroll
            for (int l = 0; l < TRSM_BK - 1; l++)
#pragma unroll
                for (int r = l + 1; r < TRSM_BK; r++)
                    if (r < bk) xd[r] -= Ts[r * TRSM_TLD + l] * xd[l];
#pragma unroll
            for (int l = 0; l < TRSM_BK; l++)
                if (l < bk) X[(lb + l) * TRSM_LDS + col] = xd[l];
        }
        __syncthreads();
        E xb[TRSM_BK];
#pragma unroll
        for (int l = 0; l < TRSM_BK; l++) xb[l] = (l < bk) ? X[(lb + l) * TRSM_LDS + col] : 0.0;
        // four rows at a time: independent dot-product chains overlap
        int r = lb + bk + rg;
        for (; r + 24 < K; r += 32) {
            const E *Tr = Ts + (r - lb) * TRSM_TLD;
            E s0 = 0, s1 = 0, s2 = 0, s3 = 0;
#pragma unroll
            for (int l = 0; l < TRSM_BK; l++) {
                s0 += Tr[l] * xb[l];
                s1 += Tr[8 * TRSM_TLD + l] * xb[l];
                s2 += Tr[16 * TRSM_TLD + l] * xb[l];
                s3 += Tr[24 * TRSM_TLD + l] * xb[l];
            }
            X[r * TRSM_LDS + col] -= s0;
            X[(r + 8) * TRSM_LDS + col] -= s1;
            X[(r + 16) * TRSM_LDS + col] -= s2;
            X[(r + 24) * TRSM_LDS + col] -= s3;
        }
        for (; r < K; r += 8) {
            const E *Tr = Ts + (r - lb) * TRSM_TLD;
            E s = 0;
#pragma unroll
            for (int l = 0; l < TRSM_BK; l++) s += Tr[l] * xb[l];
            X[r * TRSM_LDS + col] -= s;
        }
    }
    __syncthreads();
    for (int r = rg; r < K; r += 8)
        if (jok) Xg[(size_t)r * ldx + j] = X[r * TRSM_LDS + col];
    if (!bt) return;
    const float sc = bt_scale ? *bt_scale : 1.0f;
    const int jbase = blockIdx.x * TRSM_TW;
    for (int idx = threadIdx.x; idx < TRSM_TW * K; idx += 256) {
        const int cc = idx / K, r = idx - cc * K;
        if (jbase + cc < ncols) {
            const E v = X[r * TRSM_LDS + cc];
            bt[(size_t)(jbase + cc) * K + r] = bt_scale ? (BT)(float)(v * (E)sc) : (BT)(bt_neg ? -v : v);
        }
    }
}

// ---------------------------------------------------------------------------
// FP64 block-row solve on the FP64 tensor pipe (mma.sync m16n8k8 f64), for
// K a multiple of 16 up to 256.  X := T^{-1} X is done in 16-row blocks b:
// block b is finished by forward substitution with T's 16x16 unit-lower
// diagonal block (the CUDA-core solve's order of operations: for l, for r > l,
// x_r -= t_rl x_l), then X_i -= T_ib X_b for every block i below on the
// tensor pipe -- the blocked substitution of lu2's solve_triangle
// (lu2.c:485-521).  Each warp owns 8 columns of X and keeps all K rows of them
// in registers as MMA accumulators, so no step waits for another warp; T's
// 16-column block b (rows 16b..K-1: the diagonal block, then the rows below
// it) is staged in shared memory per step, double-buffered with cp.async, and
// shared by the CTA's warps.  Two 4-warp CTAs share an SM, so one CTA's substitutions overlap the
// other's products.  Outputs: X in place (16-byte stores) and
// bt[j*K + r] = -X[r][j] written in 128-byte column segments through a
// per-warp scratch tile.
constexpr int TD_WARPS = 4;
constexpr int TD_COLS = 8 * TD_WARPS;  // columns of X per CTA
constexpr int TD_MAXB = 16;            // K <= 256
// padded pitch (doubles) of a staged T block: a half-warp's A-fragment loads
// (rows g = 0..3, columns t = 0..3) fall on 16 distinct bank pairs (4g + t)
constexpr int TD_TP = 20;
constexpr int TD_SP = 9;                // pitch of the per-warp 16 x 8 scratch tile
constexpr int TD_TROWS = 16 * TD_MAXB;  // rows of a staged T block (its diagonal block first)
constexpr size_t TD_SMEM = (size_t)(2 * TD_TROWS * TD_TP + TD_WARPS * 16 * TD_SP) * sizeof(double);

__device__ __forceinline__ void td_mma(double (&c)[4], double a0, double a1, double a2, double a3, double b0, double b1)
{
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f64.f64.f64.f64 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
        "{%0,%1,%2,%3};\n"
        : "+d"(c[0]), "+d"(c[1]), "+d"(c[2]), "+d"(c[3])
        : "d"(a0), "d"(a1), "d"(a2), "d"(a3), "d"(b0), "d"(b1));
}

__device__ __forceinline__ void td_cp16(void *dst, const void *src)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((unsigned)__cvta_generic_to_shared(dst)),
                 "l"(src)
                 : "memory");
}

__global__ void __launch_bounds__(TD_WARPS * 32, 2)
    trsm_dmma_kernel(const double *__restrict__ T, long ldt, double *X, long ldx, int K, int ncols, double *bt)
{
    extern __shared__ __align__(16) double td_smem[];
    double *Tb = td_smem;  // [2][TD_TROWS][TD_TP]
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int g = lane >> 2, t = lane & 3;
    double *S = Tb + 2 * TD_TROWS * TD_TP + warp * 16 * TD_SP;  // this warp's 16 x 8 tile
    const int nbk = K >> 4;
    const int c0 = blockIdx.x * TD_COLS + warp * 8;

    // T's column block b, rows 16b..K-1, into Tb[b & 1] (row r of the block
    // at row r - 16b: the diagonal block, of which the substitution reads the
    // strict lower part, then the blocks below); 16-byte copies, 8 per row
    auto stage = [&](int b) {
        double *dst = Tb + (b & 1) * TD_TROWS * TD_TP;
        const int rows = K - 16 * b;
        for (int q = tid; q < rows * 8; q += TD_WARPS * 32) {
            const int r = q >> 3, ch = q & 7;
            td_cp16(dst + r * TD_TP + 2 * ch, T + (size_t)(16 * b + r) * ldt + 16 * b + 2 * ch);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };
    stage(0);

    // this warp's columns of X as accumulators: block i, rows 16i+g and
    // 16i+g+8, columns c0+2t and c0+2t+1
    const int col = c0 + 2 * t;
    const bool c_ok0 = col < ncols, c_ok1 = col + 1 < ncols;
    // 16-byte accesses to X where its rows allow them
    const bool xvec = ((reinterpret_cast<uintptr_t>(X) & 15) == 0) && ((ldx & 1) == 0);
    double acc[TD_MAXB][4];
#pragma unroll
    for (int i = 0; i < TD_MAXB; i++) {
#pragma unroll
        for (int h = 0; h < 2; h++) {
            double v0 = 0.0, v1 = 0.0;
            if (i < nbk) {
                const double *p = X + (size_t)(16 * i + g + 8 * h) * ldx + col;
                if (c_ok1 && xvec) {
                    const double2 w = *reinterpret_cast<const double2 *>(p);
                    v0 = w.x;
                    v1 = w.y;
                } else {
                    if (c_ok0) v0 = p[0];
                    if (c_ok1) v1 = p[1];
                }
            }
            acc[i][2 * h] = v0;
            acc[i][2 * h + 1] = v1;
        }
    }

#pragma unroll
    for (int b = 0; b < TD_MAXB; b++) {
        if (b >= nbk) break;
        asm volatile("cp.async.wait_group 0;" ::: "memory");
        __syncthreads();  // Tb[b & 1] visible; step b-1's readers of Tb[(b+1) & 1] done
        if (b + 1 < nbk) stage(b + 1);
        // block b by forward substitution, one lane per column, through the scratch tile
        S[g * TD_SP + 2 * t] = acc[b][0];
        S[g * TD_SP + 2 * t + 1] = acc[b][1];
        S[(g + 8) * TD_SP + 2 * t] = acc[b][2];
        S[(g + 8) * TD_SP + 2 * t + 1] = acc[b][3];
        __syncwarp();
        const double *Tc = Tb + (b & 1) * TD_TROWS * TD_TP;
        if (lane < 8) {
            const double *Lb = Tc;
            double xd[16];
#pragma unroll
            for (int r = 0; r < 16; r++) xd[r] = S[r * TD_SP + lane];
#pragma unroll
            for (int l = 0; l < 15; l++)
#pragma unroll
                for (int r = l + 1; r < 16; r++) xd[r] -= Lb[r * TD_TP + l] * xd[l];
#pragma unroll
            for (int r = 0; r < 16; r++) S[r * TD_SP + lane] = xd[r];
        }
        __syncwarp();
        // final rows 16b.. of X, and -X^T into bt (column j = lane / 4, rows 4(lane % 4)..+3)
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const double x0 = S[(g + 8 * h) * TD_SP + 2 * t], x1 = S[(g + 8 * h) * TD_SP + 2 * t + 1];
            double *p = X + (size_t)(16 * b + g + 8 * h) * ldx + col;
            if (c_ok1 && xvec) {
                *reinterpret_cast<double2 *>(p) = make_double2(x0, x1);
            } else {
                if (c_ok0) p[0] = x0;
                if (c_ok1) p[1] = x1;
            }
        }
        if (bt) {
            const int j = lane >> 2, q = lane & 3;
            if (c0 + j < ncols) {
                double *p = bt + (size_t)(c0 + j) * K + 16 * b + 4 * q;
                *reinterpret_cast<double2 *>(p) = make_double2(-S[(4 * q) * TD_SP + j], -S[(4 * q + 1) * TD_SP + j]);
                *reinterpret_cast<double2 *>(p + 2) =
                    make_double2(-S[(4 * q + 2) * TD_SP + j], -S[(4 * q + 3) * TD_SP + j]);
            }
        }
        // X_b as the operand of the updates below
        double bb[2][2];
#pragma unroll
        for (int kk = 0; kk < 2; kk++) {
            bb[kk][0] = S[(8 * kk + t) * TD_SP + g];
            bb[kk][1] = S[(8 * kk + t + 4) * TD_SP + g];
        }
        __syncwarp();  // the scratch is rewritten at the next step
#pragma unroll
        for (int i = 0; i < TD_MAXB; i++) {
            if (i <= b || i >= nbk) continue;
            // s = T_ib X_b from zero, then X_i -= s: the CUDA-core solve's rounding structure
            const double *A = Tc + (16 * (i - b)) * TD_TP;
            double sum[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
            for (int kk = 0; kk < 2; kk++)
                td_mma(sum, A[g * TD_TP + 8 * kk + t], A[(g + 8) * TD_TP + 8 * kk + t], A[g * TD_TP + 8 * kk + t + 4],
                       A[(g + 8) * TD_TP + 8 * kk + t + 4], bb[kk][0], bb[kk][1]);
#pragma unroll
            for (int q = 0; q < 4; q++) acc[i][q] -= sum[q];
        }
    }
}

// the tensor-pipe solve when its layout conditions hold (K a multiple of 16
// up to 256; T and bt 16-byte aligned, T's stride even), else the CUDA-core
// one.  The choice never depends on the number of columns: each column's
// result depends only on T and that column, so a schedule that solves a
// column group on its own gets the same bits as one that solves it as part of
// a wider block.
static bool trsm_dmma_ok(const double *t, long ldt, const double *x, long ldx, int K, int ncols, const double *bt)
{
    if (K <= 0 || K > 16 * TD_MAXB || (K & 15) || ncols <= 0) return false;
    if ((reinterpret_cast<uintptr_t>(t) & 15) || (ldt & 1)) return false;  // cp.async of T's rows
    if (reinterpret_cast<uintptr_t>(x) & 7) return false;
    if (bt && (reinterpret_cast<uintptr_t>(bt) & 15)) return false;
    return true;
}

static cudaError_t launch_trsm_dmma(const double *t, long ldt, double *x, long ldx, int K, int ncols, double *bt,
                                    cudaStream_t st)
{
    cudaError_t e = cudaFuncSetAttribute(trsm_dmma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)TD_SMEM);
    if (e != cudaSuccess) return e;
    const int blocks = (ncols + TD_COLS - 1) / TD_COLS;
    count_launch();
    trsm_dmma_kernel<<<blocks, TD_WARPS * 32, TD_SMEM, st>>>(t, ldt, x, ldx, K, ncols, bt);
    return cudaGetLastError();
}

template <typename E, typename BT>
static cudaError_t launch_trsm_t(const E *t, long ldt, E *x, long ldx, int K, int ncols, BT *bt, const float *bt_scale, int bt_neg,
                                 cudaStream_t st)
{
    if (ncols <= 0 || K <= 0) return cudaSuccess;
    const size_t smem = (size_t)K * (TRSM_LDS + TRSM_TLD) * sizeof(E);
    if (smem > 210 * 1024) return cudaErrorInvalidValue;
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(trsm_unit_lower_kernel<E, BT>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, 210 * 1024);
        if (e != cudaSuccess) return e;
    }
    const int blocks = (ncols + TRSM_TW - 1) / TRSM_TW;
    count_launch();
    trsm_unit_lower_kernel<E, BT><<<blocks, 256, smem, st>>>(t, ldt, x, ldx, K, ncols, bt, bt_scale, bt_neg);
    return cudaGetLastError();
}

cudaError_t launch_trsm_unit_lower_tx(const double *t, long ldt, double *x, long ldx, int K, int ncols, double *bt,
                                      cudaStream_t st)
{
    if (ncols <= 0 || K <= 0) return cudaSuccess;
    static int use_dmma = -1;  // LU2GPU_TRSM_DMMA=0 selects the CUDA-core solve everywhere (A/B checks)
    if (use_dmma < 0) {
        const char *e = getenv("LU2GPU_TRSM_DMMA");
        use_dmma = (e && e[0] == '0') ? 0 : 1;
    }
    if (use_dmma && trsm_dmma_ok(t, ldt, x, ldx, K, ncols, bt)) return launch_trsm_dmma(t, ldt, x, ldx, K, ncols, bt, st);
    return launch_trsm_t<double, double>(t, ldt, x, ldx, K, ncols, bt, nullptr, 1, st);
}

cudaError_t launch_trsm_unit_lower(double *a, long ld, int r0, int K, int cs, int ce, double *bt, cudaStream_t st)
{
    return launch_trsm_unit_lower_tx(a + (size_t)r0 * ld + r0, ld, a + (size_t)r0 * ld + cs, ld, K, ce - cs, bt, st);
}

cudaError_t launch_trsm_unit_lower_f32(const float *t, long ldt, float *x, long ldx, int K, int ncols, float *bt,
                                       cudaStream_t st)
{
    return launch_trsm_t<float, float>(t, ldt, x, ldx, K, ncols, bt, nullptr, 0, st);
}

cudaError_t launch_trsm_unit_lower_f32_bf16(const float *t, long ldt, float *x, long ldx, int K, int ncols, void *bt,
                                            const float *bt_scale, cudaStream_t st)
{
    return launch_trsm_t<float, __nv_bfloat16>(t, ldt, x, ldx, K, ncols, (__nv_bfloat16 *)bt, bt_scale, 0, st);
}

}  // namespace lu2gpu
