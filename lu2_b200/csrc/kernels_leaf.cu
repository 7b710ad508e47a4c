// kernels_leaf.cu -- the panel leaf: LU with partial pivoting of a slab of at
// most 16 columns (rows c0..n-1), held in shared memory across one
// cooperative grid.
//
// Reference behaviour (telmin/lu2): column_decomposition, lu2tlib.c:1041-1066,
// inside the slab recursion lu2tlib.c:1095-1128 (16 -> 8 -> 4 -> 2); pivot
// search cblas_idamax (first max of |a|), lu2tlib.c:42-52; the pivot row is
// scaled by 1/pivot in every column but the diagonal, lu2tlib.c:1057-1059.
// The leaf here runs the columns right-looking one by one, which is the same
// elimination in a different order of operations.
//
// Per column the critical path is one exchange between CTAs: every CTA
// publishes its candidate (largest |a| among its rows, its row values, and --
// from the CTA owning row c -- row c itself) in a slot whose every 64-bit word
// carries the column's 32-bit stamp beside 32 bits of payload (relaxed
// stores, no fence).  Warp 0 of every CTA polls the slots' heads (each lane
// re-loads the heads it still waits for back to back; a head whose words all
// carry the stamp is complete and already holds the candidate), reduces them
// to the same winner, loads the winner's row and row c (stamp-checked, re-read
// until complete) into shared memory, and after a CTA barrier every warp
// updates its own rows.  (Copying every candidate row into every CTA instead
// measured slower: 148 CTAs reading the same 148 slot lines each column.)
// Each thread owns fixed slab rows, so the exchange, the swap, the rank-1
// update and the next column's local argmax need two CTA barriers per column.
// Slots are double-buffered by column parity: a CTA can be at most one column
// ahead of any other, because it needs every CTA's previous publication to
// advance, and it reads a column's slots before its own next publication.
#include <climits>

#include "lu2gpu_internal.cuh"

namespace lu2gpu {

constexpr int LEAF_W = 16;            // widest leaf (lu2.c:1097: m <= 16)
constexpr int LEAF_THREADS = 256;
constexpr int LEAF_WARPS = LEAF_THREADS / 32;
constexpr int LEAF_LDS = LEAF_W + 1;  // padded smem row
constexpr int LEAF_MIN_ROWS = 128;    // rows per CTA below which fewer CTAs are used
constexpr int LEAF_SMEM_MAX = 200 * 1024;

template <typename T>
struct LeafParams {
    T *a;
    long ld;
    int n, c0, w, rows_per_cta, mode, goff;
    int *ipiv;
    T *dinv;
    LeafSlot *slots;  // [2][gridDim.x]
    unsigned long long seq0;
    int *status;
    unsigned long long wait_ns;  // every wait gives up after this long
    int withhold;                // test hook: this CTA never publishes (-1: none)
};

// The 32-bit stamp of publication `seq` (never 0, the value of unwritten slots)
__device__ __forceinline__ unsigned stamp_of(unsigned long long seq)
{
    return (unsigned)(seq % 4294967295ull) + 1u;
}

// T = double (plain form) or float (the precision form's FP32 panel); the
// exchanged candidate rows are carried as double, which holds either exactly.
template <typename T>
__global__ void __launch_bounds__(LEAF_THREADS) leaf_kernel(LeafParams<T> P)
{
    extern __shared__ __align__(16) unsigned char leaf_smem[];
    T *slab = reinterpret_cast<T *>(leaf_smem);
    const int G = gridDim.x, bid = blockIdx.x, tid = threadIdx.x;
    const int warp = tid >> 5, lane = tid & 31;
    const int w = P.w, c0 = P.c0, rpc = P.rows_per_cta;
    // per-warp partial argmax of the CTA's own candidate; the column's winner
    __shared__ double s_wv[LEAF_WARPS];
    __shared__ int s_wi[LEAF_WARPS];
    __shared__ int s_fail, s_win;
    __shared__ double s_prow[2 * LEAF_W];  // the column's pivot row, then row c
    const int rb = c0 + bid * rpc;
    const int re = min(P.n, rb + rpc);
    const int nr = max(0, re - rb);

    // the slab, with SLAB_U loads in flight per thread
    constexpr int SLAB_U = 8;
    for (int idx0 = tid; idx0 < nr * LEAF_W; idx0 += SLAB_U * LEAF_THREADS) {
        T v[SLAB_U];
#pragma unroll
        for (int u = 0; u < SLAB_U; u++) {
            const int idx = idx0 + u * LEAF_THREADS;
            const int lr = idx / LEAF_W, j = idx - lr * LEAF_W;
            v[u] = (idx < nr * LEAF_W && j < w) ? P.a[(size_t)(rb + lr) * P.ld + c0 + j] : T(0);
        }
#pragma unroll
        for (int u = 0; u < SLAB_U; u++) {
            const int idx = idx0 + u * LEAF_THREADS;
            const int lr = idx / LEAF_W, j = idx - lr * LEAF_W;
            if (idx < nr * LEAF_W) slab[lr * LEAF_LDS + j] = v[u];
        }
    }
    if (tid == 0) s_fail = 0;
    __syncthreads();

    // search column of global column c (view column c0+ip)
    auto search_col = [&](int ip) -> int {
        const int c = c0 + ip;
        if (P.mode == PIVOT_REF && ((c + P.goff) & 1) && ip > 0) return ip - 1;  // lu2tlib.c:1052
        if (P.mode == PIVOT_REF_FIRST) return 0;
        return ip;
    };
    // this thread's argmax over its own rows >= c in slab column sc
    auto local_argmax = [&](int c, int sc, double &bv, int &bi) {
        bv = -1.0;
        bi = INT_MAX;
        for (int lr = tid; lr < nr; lr += LEAF_THREADS) {
            if (rb + lr < c) continue;
            const double v = fabs(slab[lr * LEAF_LDS + sc]);
            if (v > bv) {  // own rows visited in increasing order: keeps the first max
                bv = v;
                bi = rb + lr;
            }
        }
    };

    double bv;
    int bi;
    local_argmax(c0, search_col(0), bv, bi);

    for (int ip = 0; ip < w; ip++) {
        const int c = c0 + ip, par = ip & 1;
        const unsigned tag = stamp_of(P.seq0 + (unsigned long long)ip + 1ull);
        LeafSlot *myslot = P.slots + (size_t)par * G + bid;
        const int owner_c = (c - c0) / rpc;

        // CTA candidate -> warp 0 publishes it (and row c, from its owner)
        warp_argmax(bv, bi);
        if (lane == 0) {
            s_wv[warp] = bv;
            s_wi[warp] = bi;
        }
        __syncthreads();  // S1
        if (warp == 0 && bid != P.withhold) {
            double v = lane < LEAF_WARPS ? s_wv[lane] : -1.0;
            int i = lane < LEAF_WARPS ? s_wi[lane] : INT_MAX;
            warp_argmax(v, i);
            if (lane < LEAF_W) {
                st_stamped(&myslot->row[2 * lane], tag, (i != INT_MAX) ? (double)slab[(i - rb) * LEAF_LDS + lane] : 0.0);
            } else if (c >= rb && c < re) {
                st_stamped(&myslot->rowc[2 * (lane - LEAF_W)], tag, (double)slab[(c - rb) * LEAF_LDS + lane - LEAF_W]);
            }
            if (lane == 0) {
                st_stamped(&myslot->head[0], tag, v);
                const unsigned long long t = (unsigned long long)tag << 32;
                asm volatile("st.relaxed.gpu.global.v2.u64 [%0], {%1, %2};" ::"l"(&myslot->head[2]),
                             "l"(t | (unsigned)i), "l"(t)
                             : "memory");
            }
        }

        // warp 0 waits for every CTA's candidate of this column, reduces them
        // to the winner and fetches the winner's row and row c into shared
        // memory.  Each lane watches up to LEAF_THREADS/32 slots: it loads the
        // heads of all those it still waits for back to back, so the polls
        // overlap instead of costing one L2 round trip each; a head whose
        // three words carry this column's stamp is complete.
        if (warp == 0) {
            constexpr int QMAX = LEAF_THREADS / 32;
            const LeafSlot *sl = P.slots + (size_t)par * G;
            unsigned pending = 0;
#pragma unroll
            for (int k = 0; k < QMAX; k++)
                if (lane + 32 * k < G) pending |= 1u << k;
            const unsigned long long t0 = globaltimer_ns();
            unsigned spins = 0;
            bool failed = false;
            double gv = -1.0;
            int gi = INT_MAX;
            while (pending) {
                unsigned long long h0[QMAX], h1[QMAX], h2[QMAX], h3[QMAX];
#pragma unroll
                for (int k = 0; k < QMAX; k++) {
                    h0[k] = h1[k] = h2[k] = h3[k] = 0ull;
                    if ((pending >> k) & 1u) {
                        ld_pair(&sl[lane + 32 * k].head[0], h0[k], h1[k]);
                        ld_pair(&sl[lane + 32 * k].head[2], h2[k], h3[k]);
                    }
                }
#pragma unroll
                for (int k = 0; k < QMAX; k++)
                    if (((pending >> k) & 1u) && stamped(h0[k], tag) && stamped(h1[k], tag) && stamped(h2[k], tag)) {
                        pending &= ~(1u << k);
                        const double v = unstamp(h0[k], h1[k]);
                        const int i = (int)(unsigned)(h2[k] & 0xffffffffull);
                        if (argmax_better(v, i, gv, gi)) {
                            gv = v;
                            gi = i;
                        }
                    }
                if (pending && (++spins & 63u) == 0 &&
                    (*(volatile int *)&P.status[1] != 0 || globaltimer_ns() - t0 > P.wait_ns)) {
                    failed = true;
                    break;
                }
            }
            if (!__any_sync(0xffffffffu, failed)) {
                warp_argmax(gv, gi);
                // lanes 0..15: the pivot row (row c itself when there is no
                // finite candidate: a NaN column keeps row c); lanes 16..31: row c
                const int p = (gi == INT_MAX) ? c : gi;
                const int owner_p = (p - c0) / rpc;
                const unsigned long long *src =
                    (lane < LEAF_W) ? ((gi == INT_MAX) ? &sl[owner_c].rowc[2 * lane] : &sl[owner_p].row[2 * lane])
                                    : &sl[owner_c].rowc[2 * (lane - LEAF_W)];
                unsigned long long hi = 0ull, lo = 0ull;
                bool ok = false;
                for (unsigned tries = 1;; tries++) {  // the loop's exits are warp-uniform
                    ld_pair(src, hi, lo);
                    ok = stamped(hi, tag) && stamped(lo, tag);
                    if (__all_sync(0xffffffffu, ok)) break;
                    const bool late = (tries & 63u) == 0 && (*(volatile int *)&P.status[1] != 0 ||
                                                             globaltimer_ns() - t0 > P.wait_ns);
                    if (__any_sync(0xffffffffu, late)) {
                        failed = true;
                        break;
                    }
                }
                const int j = (lane < LEAF_W) ? lane : lane - LEAF_W;
                s_prow[lane] = (j < w && ok) ? unstamp(hi, lo) : 0.0;
                if (lane == 0) s_win = gi;
            }
            if (__any_sync(0xffffffffu, failed) && lane == 0) {
                if (*(volatile int *)&P.status[1] == 0) record_error(P.status, ERR_BARRIER_TIMEOUT, 1);
                s_fail = 1;
            }
        }
        __syncthreads();  // S2
        if (s_fail) break;
        const int gi = s_win;

        const int p = (gi == INT_MAX) ? c : gi;  // no finite candidate (a NaN column): keep row c
        const T d = (T)s_prow[ip];
        const bool zero = (d == T(0));
        const T inv = zero ? T(1) : T(1) / d;
        T u[LEAF_W];   // scaled pivot row
        T rc[LEAF_W];  // old row c (goes to row p)
#pragma unroll
        for (int j = 0; j < LEAF_W; j++) {
            const T x = (T)s_prow[j];
            u[j] = (j == ip || zero) ? x : x * inv;
            rc[j] = (T)s_prow[LEAF_W + j];
        }
        if (bid == 0 && tid == 0) {
            P.ipiv[c] = p + P.goff;
            P.dinv[c] = inv;
            if (zero) atomicMin(&P.status[0], c + 1);
        }
        // swap (by the threads owning rows c and p), then the rank-1 update of
        // the own rows below c, then the own argmax for the next column
        const int sc_next = (ip + 1 < w) ? search_col(ip + 1) : 0;
        bv = -1.0;
        bi = INT_MAX;
        for (int lr = tid; lr < nr; lr += LEAF_THREADS) {
            const int r = rb + lr;
            if (r < c) continue;
            T *row = slab + lr * LEAF_LDS;
            if (r == c) {
#pragma unroll
                for (int j = 0; j < LEAF_W; j++) row[j] = u[j];
                continue;
            }
            if (r == p) {
#pragma unroll
                for (int j = 0; j < LEAF_W; j++) row[j] = rc[j];
            }
            if (!zero) {
                const T l = row[ip];
#pragma unroll
                for (int j = 0; j < LEAF_W; j++)
                    if (j > ip && j < w) row[j] -= l * u[j];
            }
            if (ip + 1 < w) {
                const double v = fabs(row[sc_next]);
                if (v > bv) {
                    bv = v;
                    bi = r;
                }
            }
        }
    }
    __syncthreads();
    for (int idx = tid; idx < nr * LEAF_W; idx += LEAF_THREADS) {
        const int lr = idx / LEAF_W, j = idx - lr * LEAF_W;
        if (j < w) P.a[(size_t)(rb + lr) * P.ld + c0 + j] = slab[lr * LEAF_LDS + j];
    }
}

int leaf_min_ctas(int rows, size_t tsize)
{
    return (int)(((size_t)rows * LEAF_LDS * tsize + LEAF_SMEM_MAX - 1) / LEAF_SMEM_MAX);
}

int leaf_max_ctas(int device)
{
    int sms = 0, per_sm = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    cudaFuncSetAttribute(leaf_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize, LEAF_SMEM_MAX);
    cudaFuncSetAttribute(leaf_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize, LEAF_SMEM_MAX);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, leaf_kernel<double>, LEAF_THREADS, LEAF_SMEM_MAX);
    if (per_sm < 1) per_sm = 1;
    return sms * per_sm;
}

template <typename T>
static cudaError_t launch_leaf_t(T *a, long ld, int n, int c0, int w, int mode, int goff, int *ipiv, T *dinv,
                                 const LeafBuffers &buf, int *status, int max_ctas, cudaStream_t st)
{
    if (w <= 0) return cudaSuccess;
    if (w > LEAF_W) return cudaErrorInvalidValue;
    const int rows = n - c0;
    int G = (rows + LEAF_MIN_ROWS - 1) / LEAF_MIN_ROWS;
    if (G > max_ctas) G = max_ctas;
    if (G > LEAF_THREADS) G = LEAF_THREADS;  // one polling thread per slot
    if (G < 1) G = 1;
    const int rpc = (rows + G - 1) / G;
    G = (rows + rpc - 1) / rpc;
    const size_t smem = (size_t)rpc * LEAF_LDS * sizeof(T);
    if (smem > (size_t)LEAF_SMEM_MAX) return cudaErrorInvalidConfiguration;
    LeafParams<T> P{a, ld, n, c0, w, rpc, mode, goff, ipiv, dinv, buf.slots, *buf.seq, status, buf.wait_ns,
                    buf.withhold};
    *buf.seq += (unsigned long long)w;
    void *args[] = {&P};
    count_launch();
    return cudaLaunchCooperativeKernel((const void *)leaf_kernel<T>, dim3(G), dim3(LEAF_THREADS), args, smem, st);
}

cudaError_t launch_leaf(double *a, long ld, int n, int c0, int w, int mode, int goff, int *ipiv, double *dinv,
                        const LeafBuffers &buf, int *status, int max_ctas, cudaStream_t st)
{
    return launch_leaf_t(a, ld, n, c0, w, mode, goff, ipiv, dinv, buf, status, max_ctas, st);
}

cudaError_t launch_leaf(float *a, long ld, int n, int c0, int w, int mode, int goff, int *ipiv, float *dinv,
                        const LeafBuffers &buf, int *status, int max_ctas, cudaStream_t st)
{
    return launch_leaf_t(a, ld, n, c0, w, mode, goff, ipiv, dinv, buf, status, max_ctas, st);
}

}  // namespace lu2gpu
