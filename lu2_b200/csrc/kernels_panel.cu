// kernels_panel.cu -- panel kernels: the pivot-apply (swap + 1/pivot scale)
// and the unit-lower triangular solve of the U block row (the leaf is in
// kernels_leaf.cu).
//
// Reference behaviour followed (telmin/lu2):
//   swap+scale  lu2.c:251-291 (swaprows_simple_with_scale), lu2.c:541-554,
//               lu2.c:1107-1118
//   trsm        lu2.c:485-521 (solve_triangle: U12 = L11^{-1} A12)
#include <climits>

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

    if (status && *(volatile int *)&status[1] != 0) return;
    if (tid == 0) {
        s_bad = 0;
        s_nslot = npiv;
    }
    __syncthreads();
    for (int t = tid; t < npiv; t += SWAP_THREADS) {
        const int p = __ldg(ipiv + k0 + t) - goff;
        P[t] = p;
        A[t] = -1;
        if (p < k0 + t || p >= nrows) s_bad = 1;
    }
    __syncthreads();
    if (s_bad) {
        if (blockIdx.x == 0 && tid == 0 && status) record_error(status, ERR_BAD_ARG, 3);
        return;
    }
    for (int i = tid; i < npiv; i += SWAP_THREADS) {
        const int q = P[i];
        if (q != k0 + i && q < k1) atomicMax(&A[q - k0], i);
    }
    __syncthreads();
    for (int t = tid; t < npiv; t += SWAP_THREADS)
        if (A[t] < 0) A[t] = -(k0 + t) - 1;
    __syncthreads();
    {
        // pointer jumping, double-buffered through src (free until the slots
        // are written): after r rounds every pointer has advanced 2^r links or
        // reached its root, and a chain has fewer than npiv links
        int *cur = A, *nxt = src;
        for (int span = 1; span < npiv; span <<= 1) {
            for (int t = tid; t < npiv; t += SWAP_THREADS) {
                const int v = cur[t];
                nxt[t] = (v >= 0) ? cur[v] : v;
            }
            __syncthreads();
            int *tmp = cur;
            cur = nxt;
            nxt = tmp;
        }
        if (cur != A) {
            for (int t = tid; t < npiv; t += SWAP_THREADS) A[t] = cur[t];
            __syncthreads();
        }
    }
    for (int t = tid; t < npiv; t += SWAP_THREADS) {
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
        return;
    }
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
