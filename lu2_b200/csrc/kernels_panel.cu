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
// Instead of replaying the npiv exchanges element by element (npiv dependent
// memory round trips), every CTA first builds the composite permutation of the
// touched rows in shared memory: slots 0..npiv-1 are the rows k0..k1-1, further
// slots the distinct rows ipiv[k] >= k1 in order of first appearance; the
// exchanges are replayed on slot indices only.  Then the CTA gathers the
// source rows of its 16 columns (128-byte row segments) into shared memory and
// scatters them to their destinations.
constexpr int SWAP_COLS = 16;
constexpr int SWAP_THREADS = 256;

template <typename T>
__global__ void __launch_bounds__(SWAP_THREADS) laswp_scale_kernel(T *a, long ld, int k0, int k1,
                                                                   const int *__restrict__ ipiv, int goff,
                                                                   const T *__restrict__ dinv, int cs, int ce,
                                                                   int scale)
{
    extern __shared__ int sw[];
    const int npiv = k1 - k0;
    int *prow = sw;               // [npiv] view row of each pivot
    int *first = prow + npiv;     // [npiv] index of the first pivot naming the same row (rows >= k1)
    int *slot = first + npiv;     // [npiv] extra slot of a first occurrence
    int *cur = slot + npiv;       // [2 npiv] slot content
    int *rowof = cur + 2 * npiv;  // [2 npiv] row of each slot
    __shared__ int s_nslot;
    T *V = reinterpret_cast<T *>(sw + ((7 * npiv + 1) & ~1));  // [2 npiv][SWAP_COLS], 8-byte aligned
    const int tid = threadIdx.x;

    for (int t = tid; t < npiv; t += SWAP_THREADS) {
        prow[t] = __ldg(ipiv + k0 + t) - goff;
        rowof[t] = k0 + t;
    }
    for (int s = tid; s < 2 * npiv; s += SWAP_THREADS) cur[s] = s;
    __syncthreads();
    for (int t = tid; t < npiv; t += SWAP_THREADS) {
        const int p = prow[t];
        int f = -1;
        if (p >= k1) {
            f = t;
            for (int q = 0; q < t; q++)
                if (prow[q] == p) {
                    f = q;
                    break;
                }
        }
        first[t] = f;
    }
    __syncthreads();
    if (tid == 0) {
        int nex = 0;
        for (int t = 0; t < npiv; t++) {
            const int p = prow[t];
            int b;
            if (p < k1) {
                b = p - k0;
            } else {
                const int f = first[t];
                if (f == t) {
                    slot[t] = npiv + nex;
                    rowof[npiv + nex] = p;
                    nex++;
                }
                b = slot[f];
            }
            const int tmp = cur[t];
            cur[t] = cur[b];
            cur[b] = tmp;
        }
        s_nslot = npiv + nex;
    }
    __syncthreads();
    const int nslot = s_nslot;
    const int c = tid & (SWAP_COLS - 1);
    const int nchunk = (ce - cs + SWAP_COLS - 1) / SWAP_COLS;
    for (int chunk = blockIdx.x; chunk < nchunk; chunk += gridDim.x) {
        const int j = cs + chunk * SWAP_COLS + c;
        const bool jok = j < ce;
        // gather with GATHER_U loads in flight per thread
        constexpr int STEP = SWAP_THREADS / SWAP_COLS, GATHER_U = 8;
        for (int s0 = tid / SWAP_COLS; s0 < nslot; s0 += GATHER_U * STEP) {
            T v[GATHER_U];
#pragma unroll
            for (int u = 0; u < GATHER_U; u++) {
                const int s = s0 + u * STEP;
                v[u] = (jok && s < nslot) ? a[(size_t)rowof[cur[s]] * ld + j] : T(0);
            }
#pragma unroll
            for (int u = 0; u < GATHER_U; u++) {
                const int s = s0 + u * STEP;
                if (s < nslot) V[s * SWAP_COLS + c] = v[u];
            }
        }
        __syncthreads();
        if (jok) {
            for (int s = tid / SWAP_COLS; s < nslot; s += SWAP_THREADS / SWAP_COLS) {
                T v = V[s * SWAP_COLS + c];
                if (scale && s < npiv) v *= __ldg(dinv + k0 + s);
                a[(size_t)rowof[s] * ld + j] = v;
            }
        }
        __syncthreads();
    }
}

template <typename T>
static cudaError_t launch_laswp_scale_t(T *a, long ld, int k0, int k1, const int *ipiv, int goff, const T *dinv,
                                        int cs, int ce, bool scale, cudaStream_t st)
{
    if (ce <= cs || k1 <= k0) return cudaSuccess;
    const int npiv = k1 - k0;
    const size_t smem = (size_t)7 * npiv * sizeof(int) + 8 + (size_t)2 * npiv * SWAP_COLS * sizeof(T);
    if (smem > 200 * 1024) return cudaErrorInvalidValue;
    if (smem > 48 * 1024) {
        cudaError_t e =
            cudaFuncSetAttribute(laswp_scale_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
        if (e != cudaSuccess) return e;
    }
    // the permutation is built once per CTA; CTAs then stride over 16-column chunks
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    int blocks = (ce - cs + SWAP_COLS - 1) / SWAP_COLS;
    if (blocks > 3 * sms) blocks = 3 * sms;
    count_launch();
    laswp_scale_kernel<T><<<blocks, SWAP_THREADS, smem, st>>>(a, ld, k0, k1, ipiv, goff, dinv, cs, ce, scale ? 1 : 0);
    return cudaGetLastError();
}

cudaError_t launch_laswp_scale(double *a, long ld, int k0, int k1, const int *ipiv, int goff, const double *dinv,
                               int cs, int ce, bool scale, cudaStream_t st)
{
    return launch_laswp_scale_t(a, ld, k0, k1, ipiv, goff, dinv, cs, ce, scale, st);
}

cudaError_t launch_laswp_scale(float *a, long ld, int k0, int k1, const int *ipiv, int goff, const float *dinv,
                               int cs, int ce, bool scale, cudaStream_t st)
{
    return launch_laswp_scale_t(a, ld, k0, k1, ipiv, goff, dinv, cs, ce, scale, st);
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
