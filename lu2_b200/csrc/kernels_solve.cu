// kernels_solve.cu -- back substitution with the unit upper factor, and the
// on-device matrix generator.
//
// backward_sub (lu2.c:110-116) is x_j = y_j - sum_{k>j} U'_jk x_k with U' unit
// upper and y the transformed right-hand side column.  Here it is blocked
// from the bottom: a 128x128 diagonal block is solved in shared memory, then
// every row above is updated by one warp reading its 1 KB row segment.
//
// randomsetmat (lu2.c:70-85) draws glibc drand48 values row by row.  The
// device generator reproduces that stream exactly: the 48-bit LCG
// X' = 0x5DEECE66D X + 0xB (mod 2^48) is jumped ahead with the affine-map
// doubling (A, C) o (A, C) = (A^2, A C + C), and drand48() = X 2^-48.
#include "lu2gpu_internal.cuh"

namespace lu2gpu {

constexpr int BS_BLOCK = 128;
constexpr int BS_MAXR = 8;  // right-hand sides handled per pass

// Solve the unit upper diagonal block rows r0..r0+bs-1 for columns
// n+c0..n+c0+nr-1 (nr <= BS_MAXR).  One CTA.
template <typename T>
__global__ void __launch_bounds__(256) backsolve_diag_kernel(const T *a, long ld, int r0, int bs, T *x, long ldx,
                                                             int c0, int nr)
{
    extern __shared__ __align__(16) unsigned char bs_smem[];
    T *U = reinterpret_cast<T *>(bs_smem);  // bs x (bs+1): an odd row pitch, conflict-free column reads
    __shared__ T X[BS_BLOCK][BS_MAXR];
    const int lds = bs + 1;
    // the block, PER loads in flight per thread before they are stored
    constexpr int PER = 16;
    for (int base = 0; base < bs * bs; base += PER * 256) {
        T v[PER];
#pragma unroll
        for (int q = 0; q < PER; q++) {
            const int idx = base + q * 256 + (int)threadIdx.x;
            const int r = idx / bs, c = idx - r * bs;
            v[q] = (idx < bs * bs) ? a[(size_t)(r0 + r) * ld + r0 + c] : T(0);
        }
#pragma unroll
        for (int q = 0; q < PER; q++) {
            const int idx = base + q * 256 + (int)threadIdx.x;
            const int r = idx / bs, c = idx - r * bs;
            if (idx < bs * bs) U[r * lds + c] = v[q];
        }
    }
    for (int idx = threadIdx.x; idx < bs * nr; idx += blockDim.x) {
        const int r = idx / nr, c = idx - r * nr;
        X[r][c] = x[(size_t)(r0 + r) * ldx + c0 + c];
    }
    __syncthreads();
    // one warp per right-hand side, column-oriented: lane l holds rows l,
    // l+32, l+64, l+96; once x_j is final (its owner lane's value) every row
    // i < j subtracts U'[i][j] x_j
    constexpr int QB = BS_BLOCK / 32;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int c = warp; c < nr; c += blockDim.x >> 5) {
        T y[QB];
#pragma unroll
        for (int q = 0; q < QB; q++) y[q] = (q * 32 + lane < bs) ? X[q * 32 + lane][c] : T(0);
#pragma unroll
        for (int qo = QB - 1; qo >= 0; qo--) {
            for (int l = 31; l >= 0; l--) {
                const int j = qo * 32 + l;
                if (j >= bs) continue;  // warp-uniform
                const T xj = __shfl_sync(0xffffffffu, y[qo], l);
#pragma unroll
                for (int q = 0; q <= qo; q++) {
                    const int i = q * 32 + lane;
                    if (i < j) y[q] -= U[i * lds + j] * xj;
                }
            }
        }
#pragma unroll
        for (int q = 0; q < QB; q++)
            if (q * 32 + lane < bs) X[q * 32 + lane][c] = y[q];
    }
    __syncthreads();
    for (int idx = threadIdx.x; idx < bs * nr; idx += blockDim.x) {
        const int r = idx / nr, c = idx - r * nr;
        x[(size_t)(r0 + r) * ldx + c0 + c] = X[r][c];
    }
}

// y[i][c] -= sum_{k in block} U'[i][k] x[k][c] for rows i < r0; one warp per row.
template <typename T>
__global__ void __launch_bounds__(256) backsolve_update_kernel(const T *a, long ld, int r0, int bs, T *x, long ldx,
                                                               int c0, int nr)
{
    __shared__ T X[BS_BLOCK][BS_MAXR];
    for (int idx = threadIdx.x; idx < bs * nr; idx += blockDim.x) {
        const int r = idx / nr, c = idx - r * nr;
        X[r][c] = x[(size_t)(r0 + r) * ldx + c0 + c];
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wpb = blockDim.x >> 5;
    for (int i = blockIdx.x * wpb + warp; i < r0; i += gridDim.x * wpb) {
        const T *row = a + (size_t)i * ld + r0;
        T s[BS_MAXR];
#pragma unroll
        for (int c = 0; c < BS_MAXR; c++) s[c] = 0;
        for (int k = lane; k < bs; k += 32) {
            const T u = __ldcs(row + k);
#pragma unroll
            for (int c = 0; c < BS_MAXR; c++)
                if (c < nr) s[c] += u * X[k][c];
        }
#pragma unroll
        for (int c = 0; c < BS_MAXR; c++) {
            if (c >= nr) break;
            T v = s[c];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (lane == 0) x[(size_t)i * ldx + c0 + c] -= v;
        }
    }
}

template <typename T>
static cudaError_t launch_backsolve_t(const T *a, long ld, int n, int nrhs, T *x, long ldx, cudaStream_t st)
{
    cudaError_t e = cudaFuncSetAttribute(backsolve_diag_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         BS_BLOCK * (BS_BLOCK + 1) * (int)sizeof(T));
    if (e != cudaSuccess) return e;
    int sms = 148, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    for (int c0 = 0; c0 < nrhs; c0 += BS_MAXR) {
        const int nr = nrhs - c0 < BS_MAXR ? nrhs - c0 : BS_MAXR;
        const int nblk = (n + BS_BLOCK - 1) / BS_BLOCK;
        for (int b = nblk - 1; b >= 0; b--) {
            const int r0 = b * BS_BLOCK;
            const int bs = (n - r0) < BS_BLOCK ? (n - r0) : BS_BLOCK;
            const size_t smem = (size_t)bs * (bs + 1) * sizeof(T);
            count_launch();
            backsolve_diag_kernel<T><<<1, 256, smem, st>>>(a, ld, r0, bs, x, ldx, c0, nr);
            if (r0 > 0) {
                int blocks = (r0 + 7) / 8;
                if (blocks > sms * 8) blocks = sms * 8;
                count_launch();
                backsolve_update_kernel<T><<<blocks, 256, 0, st>>>(a, ld, r0, bs, x, ldx, c0, nr);
            }
        }
    }
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Persistent back substitution for large n.  Rows are cut into 64-row blocks,
// counted from the bottom (p = 0 is the last block); block p belongs to CTA
// p mod G of a cooperative grid of G co-resident CTAs, which keeps the
// right-hand sides of all its blocks in shared memory.  The blocks' solutions
// x_p are published in the order p = 0, 1, 2, ...: when x_p is out, every CTA
// subtracts U(block q, block p) x_p from each of its blocks q > p, in that
// order, so every element receives its updates in a fixed order; the CTA
// owning block p+1 does that block first and solves it at once (column
// oriented, one warp per right-hand side), so the critical path per block is
// one 64x64 product and one 64x64 solve.  Each block of U is read once: a
// CTA issues the loads of the U tiles its next BSP_AHEAD pending blocks take
// from a source before it waits for that source's x, so that their DRAM
// latency overlaps the wait (the tiles do not depend on x).
// Publication: the solving warps store the block's x straight from their
// registers into the block's slot as stamped words (the call's epoch beside
// each 32-bit half, no fence); a reader re-loads the slot's words until all
// carry the epoch (bounded wait), which gives it x in the same round trip.
constexpr int BSP = 64;          // rows per block
constexpr int BSP_THREADS = 256;
constexpr int BSP_AHEAD = 2;     // U tiles per CTA loaded before a source's x is awaited
static_assert(BS_SLOT_WORDS == BSP * BS_MAXR * 2, "an x slot holds a block's rows x right-hand sides as stamped pairs");

template <typename T>
struct BsParams {
    const T *a;
    long ld;
    int n, nblk;
    T *x;
    long ldx;
    int c0, nr;
    unsigned long long *xslots;  // [nblk][BS_SLOT_WORDS]: element (r, q) of a block at 2 (r BS_MAXR + q)
    unsigned epoch;
    int *status;
};

template <typename T>
__global__ void __launch_bounds__(BSP_THREADS, 2) backsolve_persistent_kernel(BsParams<T> P)
{
    extern __shared__ __align__(16) unsigned char bsp_smem[];
    const int G = gridDim.x, cta = blockIdx.x, tid = threadIdx.x;
    const int nblk = P.nblk, nr = P.nr;
    const int n_own = cta < nblk ? (nblk - cta + G - 1) / G : 0;
    T *acc = reinterpret_cast<T *>(bsp_smem);      // [n_own][BSP][BS_MAXR]
    T *Ud = acc + (size_t)n_own * BSP * BS_MAXR;    // [BSP][BSP + 1]
    T *xs = Ud + BSP * (BSP + 1);                   // [2][BSP][BS_MAXR]
    // block p covers rows r0(p) .. r0(p) + rows(p) - 1
    auto r0_of = [&](int p) { return (nblk - 1 - p) * BSP; };
    auto rows_of = [&](int p) { return min(BSP, P.n - r0_of(p)); };

    for (int k = 0; k < n_own; k++) {
        const int p = cta + k * G, r0 = r0_of(p), rows = rows_of(p);
        for (int e = tid; e < BSP * BS_MAXR; e += BSP_THREADS) {
            const int r = e / BS_MAXR, q = e % BS_MAXR;
            acc[((size_t)k * BSP + r) * BS_MAXR + q] = (r < rows && q < nr) ? P.x[(size_t)(r0 + r) * P.ldx + P.c0 + q] : T(0);
        }
    }
    __syncthreads();

    // owned block k's diagonal tile into Ud, asynchronously (issued right after
    // the previous solve, so the copy is off the critical path); only the
    // strict upper part of the first `rows` rows and columns is read later
    auto prefetch_diag = [&](int k) {
        const int p = cta + k * G, r0 = r0_of(p), rows = rows_of(p);
        for (int e = tid; e < BSP * BSP; e += BSP_THREADS) {
            const int r = e / BSP, c = e % BSP;
            if (r < rows && c < rows && c > r) {
                const unsigned dst = (unsigned)__cvta_generic_to_shared(&Ud[r * (BSP + 1) + c]);
                if constexpr (sizeof(T) == 8)
                    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(dst),
                                 "l"(P.a + (size_t)(r0 + r) * P.ld + r0 + c)
                                 : "memory");
                else
                    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(dst),
                                 "l"(P.a + (size_t)(r0 + r) * P.ld + r0 + c)
                                 : "memory");
            }
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    };

    // solve owned block k (all updates from the blocks below applied) into
    // xs[buf] and x; the solving warps publish it first
    auto solve = [&](int k, int buf) {
        const int p = cta + k * G, r0 = r0_of(p), rows = rows_of(p);
        asm volatile("cp.async.wait_group 0;" ::: "memory");
        __syncthreads();
        const int warp = tid >> 5, lane = tid & 31;
        T *A = acc + (size_t)k * BSP * BS_MAXR;
        if (warp < nr) {
            T y0 = A[lane * BS_MAXR + warp], y1 = A[(lane + 32) * BS_MAXR + warp];
            for (int c = rows - 1; c >= 0; c--) {  // x_c final: rows above subtract U'[r][c] x_c
                const T xc = __shfl_sync(0xffffffffu, c >= 32 ? y1 : y0, c & 31);
                if (lane < c) y0 -= Ud[lane * (BSP + 1) + c] * xc;
                if (lane + 32 < c) y1 -= Ud[(lane + 32) * (BSP + 1) + c] * xc;
            }
            unsigned long long *slot = P.xslots + (size_t)(nblk - 1 - p) * BS_SLOT_WORDS;
            if (lane < rows) st_stamped(slot + 2 * (lane * BS_MAXR + warp), P.epoch, (double)y0);
            if (lane + 32 < rows) st_stamped(slot + 2 * ((lane + 32) * BS_MAXR + warp), P.epoch, (double)y1);
            A[lane * BS_MAXR + warp] = y0;
            A[(lane + 32) * BS_MAXR + warp] = y1;
        }
        __syncthreads();
        T *X = xs + buf * BSP * BS_MAXR;
        for (int e = tid; e < BSP * BS_MAXR; e += BSP_THREADS) {
            const int r = e / BS_MAXR, q = e % BS_MAXR;
            const T v = (r < rows && q < nr) ? A[e] : T(0);
            X[e] = v;
            if (r < rows && q < nr) P.x[(size_t)(r0 + r) * P.ldx + P.c0 + q] = v;
        }
        __syncthreads();
        if (k + 1 < n_own) prefetch_diag(k + 1);
    };

    // thread (r, part) of owned block k's U tile for source p_src: row r,
    // the column pairs 8 j + 2 part, 8 j + 2 part + 1 (j = 0..7) as v[2j],
    // v[2j+1] (zero outside the tile): the four threads of a row read 64
    // contiguous bytes per load, with one 2-element vector load each where
    // the matrix's alignment and row stride allow
    const bool uvec = ((reinterpret_cast<uintptr_t>(P.a) & (2 * sizeof(T) - 1)) == 0) && ((P.ld & 1) == 0);
    auto load_u = [&](int k, int p_src, T (&v)[16]) {
        const int p = cta + k * G, r0 = r0_of(p), rows = rows_of(p);
        const int c0 = r0_of(p_src), cols = rows_of(p_src);
        const int r = tid >> 2, part = tid & 3;
        if (r < rows) {
            const T *u = P.a + (size_t)(r0 + r) * P.ld + c0 + 2 * part;
            if (uvec && cols == BSP) {
#pragma unroll
                for (int j = 0; j < 8; j++) {
                    if constexpr (sizeof(T) == 8) {
                        const double2 w = __ldg(reinterpret_cast<const double2 *>(u + 8 * j));
                        v[2 * j] = w.x;
                        v[2 * j + 1] = w.y;
                    } else {
                        const float2 w = __ldg(reinterpret_cast<const float2 *>(u + 8 * j));
                        v[2 * j] = w.x;
                        v[2 * j + 1] = w.y;
                    }
                }
            } else {
#pragma unroll
                for (int j = 0; j < 8; j++) {
                    const int col = 8 * j + 2 * part;
                    v[2 * j] = col < cols ? __ldg(u + 8 * j) : T(0);
                    v[2 * j + 1] = col + 1 < cols ? __ldg(u + 8 * j + 1) : T(0);
                }
            }
        } else {
#pragma unroll
            for (int e = 0; e < 16; e++) v[e] = T(0);
        }
    };

    // acc[k] -= U(block of k, block p_src) * X, X the source's solution (BSP x nr)
    auto apply_u = [&](int k, const T (&v)[16], const T *X) {
        const int p = cta + k * G, rows = rows_of(p);
        const int r = tid >> 2, part = tid & 3;  // 16 columns per thread
        T s[BS_MAXR];
#pragma unroll
        for (int q = 0; q < BS_MAXR; q++) s[q] = T(0);
        if (r < rows) {
#pragma unroll
            for (int e = 0; e < 16; e++)
#pragma unroll
                for (int q = 0; q < BS_MAXR; q++)
                    if (q < nr) s[q] += v[e] * X[(8 * (e >> 1) + 2 * part + (e & 1)) * BS_MAXR + q];
        }
#pragma unroll
        for (int q = 0; q < BS_MAXR; q++) {
            s[q] += __shfl_xor_sync(0xffffffffu, s[q], 1);
            s[q] += __shfl_xor_sync(0xffffffffu, s[q], 2);
        }
        if (part == 0 && r < rows)
#pragma unroll
            for (int q = 0; q < BS_MAXR; q++)
                if (q < nr) acc[((size_t)k * BSP + r) * BS_MAXR + q] -= s[q];
    };

    int next = 0;
    if (n_own > 0) prefetch_diag(0);
    if (n_own > 0 && cta == 0) {  // the bottom block needs no update
        solve(0, 0);
        next = 1;
    }
    const unsigned long long t0 = globaltimer_ns();
    for (int p_src = 0; p_src < nblk; p_src++) {
        const int buf = p_src & 1;
        T *X = xs + buf * BSP * BS_MAXR;
        // the U tiles of the first pending owned blocks, before the wait
        const int k_first = next;
        T v[BSP_AHEAD][16];
#pragma unroll
        for (int j = 0; j < BSP_AHEAD; j++)
            if (k_first + j < n_own) load_u(k_first + j, p_src, v[j]);
        if (p_src % G != cta) {
            // the source block's x from its slot: each thread re-loads its
            // elements until they carry this call's epoch; the CTA agrees on
            // completion, or on giving up, at one barrier per round
            const unsigned long long *slot = P.xslots + (size_t)(nblk - 1 - p_src) * BS_SLOT_WORDS;
            const int rows = rows_of(p_src);
            constexpr int EPT = BSP * BS_MAXR / BSP_THREADS;  // elements per thread
            unsigned todo = 0;
#pragma unroll
            for (int u = 0; u < EPT; u++) {
                const int e = tid + u * BSP_THREADS, r = e / BS_MAXR, q = e % BS_MAXR;
                if (r < rows && q < nr)
                    todo |= 1u << u;
                else
                    X[e] = T(0);
            }
            for (unsigned round = 1;; round++) {
#pragma unroll
                for (int u = 0; u < EPT; u++) {
                    if (!((todo >> u) & 1u)) continue;
                    const int e = tid + u * BSP_THREADS;
                    unsigned long long hi, lo;
                    ld_pair(slot + 2 * e, hi, lo);
                    if (stamped(hi, P.epoch) && stamped(lo, P.epoch)) {
                        X[e] = (T)unstamp(hi, lo);
                        todo &= ~(1u << u);
                    }
                }
                if (__syncthreads_and(todo == 0)) break;
                const bool late = (round & 63u) == 0 && tid == 0 &&
                                  (*(volatile int *)&P.status[1] != 0 || globaltimer_ns() - t0 > WAIT_LIMIT_NS);
                if (__syncthreads_or(late)) {
                    if (tid == 0 && *(volatile int *)&P.status[1] == 0) record_error(P.status, ERR_BARRIER_TIMEOUT, 6);
                    return;
                }
            }
        }
        if (k_first < n_own) {
            apply_u(k_first, v[0], X);
            if (cta + k_first * G == p_src + 1) {
                __syncthreads();
                solve(k_first, buf ^ 1);
                next = k_first + 1;
            }
        }
#pragma unroll
        for (int j = 1; j < BSP_AHEAD; j++)
            if (k_first + j < n_own) apply_u(k_first + j, v[j], X);
        for (int k0 = k_first + BSP_AHEAD; k0 < n_own; k0 += BSP_AHEAD) {
#pragma unroll
            for (int j = 0; j < BSP_AHEAD; j++)
                if (k0 + j < n_own) load_u(k0 + j, p_src, v[j]);
#pragma unroll
            for (int j = 0; j < BSP_AHEAD; j++)
                if (k0 + j < n_own) apply_u(k0 + j, v[j], X);
        }
        __syncthreads();  // X (this buffer) is overwritten two sources later
    }
}

template <typename T>
static cudaError_t launch_backsolve_persistent(const T *a, long ld, int n, int nrhs, T *x, long ldx,
                                               const BsBuffers &bs, cudaStream_t st, bool *used)
{
    *used = false;
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int nblk = (n + BSP - 1) / BSP;
    if (nblk > bs.cap) return cudaSuccess;
    cudaError_t e = cudaFuncSetAttribute(backsolve_persistent_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         200 * 1024);
    if (e != cudaSuccess) return e;
    // two CTAs per SM where they fit: each then owns half as many blocks, so
    // less of its work sits between a publication and the next block's solve
    int G = 0, n_own = 0;
    size_t smem = 0;
    for (int want = 2; want >= 1 && G == 0; want--) {
        const int g = nblk < want * sms ? nblk : want * sms;
        const int own = (nblk + g - 1) / g;
        const size_t sm = ((size_t)own * BSP * BS_MAXR + BSP * (BSP + 1) + 2 * BSP * BS_MAXR) * sizeof(T);
        if (sm > 200 * 1024) continue;
        int per_sm = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, backsolve_persistent_kernel<T>, BSP_THREADS, sm);
        if (e != cudaSuccess) return e;
        if (per_sm >= want || g == nblk) {
            if ((long)per_sm * sms < g) continue;
            G = g;
            n_own = own;
            smem = sm;
        }
    }
    if (G == 0) return cudaSuccess;  // the blocked launches take it
    (void)n_own;
    for (int c0 = 0; c0 < nrhs; c0 += BS_MAXR) {
        BsParams<T> P{a, ld, n, nblk, x, ldx, c0, nrhs - c0 < BS_MAXR ? nrhs - c0 : BS_MAXR, bs.xslots, 0u, bs.status};
        P.epoch = ++*bs.epoch;
        if (P.epoch == 0) P.epoch = ++*bs.epoch;
        void *args[] = {&P};
        count_launch();
        e = cudaLaunchCooperativeKernel((const void *)backsolve_persistent_kernel<T>, dim3(G), dim3(BSP_THREADS), args,
                                        smem, st);
        if (e != cudaSuccess) return e;
    }
    *used = true;
    return cudaSuccess;
}

template <typename T>
static cudaError_t launch_backsolve_any(const T *a, long ld, int n, int nrhs, T *x, long ldx, const BsBuffers *bs,
                                       cudaStream_t st)
{
    if (bs && bs->xslots && n >= BSP_PERSISTENT_MIN_N) {
        bool used = false;
        cudaError_t e = launch_backsolve_persistent(a, ld, n, nrhs, x, ldx, *bs, st, &used);
        if (e != cudaSuccess || used) return e;
    }
    return launch_backsolve_t(a, ld, n, nrhs, x, ldx, st);
}

cudaError_t launch_backsolve(const double *a, long ld, int n, int nrhs, double *x, long ldx, const BsBuffers *bs,
                             cudaStream_t st)
{
    return launch_backsolve_any(a, ld, n, nrhs, x, ldx, bs, st);
}

cudaError_t launch_backsolve(const float *a, long ld, int n, int nrhs, float *x, long ldx, const BsBuffers *bs,
                             cudaStream_t st)
{
    return launch_backsolve_any(a, ld, n, nrhs, x, ldx, bs, st);
}

// out[k] = 1 / a[k][k] (1 where the pivot is exactly zero), the same value the
// leaf stored for the factorization's own 1/pivot scaling.
template <typename T>
__global__ void diag_inv_kernel(const T *a, long ld, int n, T *out)
{
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    const T d = a[(size_t)k * ld + k];
    out[k] = (d == T(0)) ? T(1) : T(1) / d;
}

cudaError_t launch_diag_inv(const double *a, long ld, int n, double *out, cudaStream_t st)
{
    if (n <= 0) return cudaSuccess;
    count_launch();
    diag_inv_kernel<double><<<(n + 255) / 256, 256, 0, st>>>(a, ld, n, out);
    return cudaGetLastError();
}

cudaError_t launch_diag_inv(const float *a, long ld, int n, float *out, cudaStream_t st)
{
    if (n <= 0) return cudaSuccess;
    count_launch();
    diag_inv_kernel<float><<<(n + 255) / 256, 256, 0, st>>>(a, ld, n, out);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// drand48 stream

constexpr unsigned long long LCG_A = 0x5DEECE66Dull, LCG_C = 0xBull, LCG_MASK = (1ull << 48) - 1;

struct Affine {
    unsigned long long a, c;
};

// k applications of the drand48 step
__host__ __device__ inline Affine lcg_jump(unsigned long long k)
{
    Affine r{1, 0}, b{LCG_A, LCG_C};
    while (k) {
        if (k & 1) r = Affine{(b.a * r.a) & LCG_MASK, (b.a * r.c + b.c) & LCG_MASK};
        b = Affine{(b.a * b.a) & LCG_MASK, (b.a * b.c + b.c) & LCG_MASK};
        k >>= 1;
    }
    return r;
}

// One CTA per matrix row: row i holds draws i*(n+1)+1 .. i*(n+1)+n+1 (the
// last is b_i).  kind 1 replaces a_ii by sum_j |a_ij| over the generated row.
__global__ void __launch_bounds__(256) gen_rows_kernel(double *a, long ld, int n, unsigned long long x_seed, int kind,
                                                       Affine step)
{
    const long i = blockIdx.x;
    const unsigned long long first = (unsigned long long)i * (unsigned long long)(n + 1) + threadIdx.x + 1;
    const Affine j = lcg_jump(first);
    unsigned long long x = (j.a * x_seed + j.c) & LCG_MASK;
    double *row = a + (size_t)i * ld;
    double asum = 0.0;
    for (int c = threadIdx.x; c <= n; c += blockDim.x) {
        const double v = (double)x * (1.0 / 281474976710656.0) - 0.5;
        row[c] = v;
        if (c < n) asum += fabs(v);
        x = (step.a * x + step.c) & LCG_MASK;
    }
    if (kind == 1) {
        __shared__ double red[8];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) asum += __shfl_xor_sync(0xffffffffu, asum, o);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = asum;
        __syncthreads();
        if (threadIdx.x == 0) {
            double s = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); w++) s += red[w];
            row[i] = s;
        }
    }
}

// extra right-hand sides r = 1..nrhs-1: draw n*(n+1) + (r-1)*n + i + 1
__global__ void gen_rhs_kernel(double *a, long ld, int n, int nrhs, unsigned long long x_seed)
{
    const long q = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const long total = (long)n * (nrhs - 1);
    if (q >= total) return;
    const long r = 1 + q / n, i = q % n;
    const Affine j = lcg_jump((unsigned long long)n * (unsigned long long)(n + 1) + (unsigned long long)q + 1);
    const unsigned long long x = (j.a * x_seed + j.c) & LCG_MASK;
    a[(size_t)i * ld + n + r] = (double)x * (1.0 / 281474976710656.0) - 0.5;
}

cudaError_t launch_generate(double *a, long ld, int n, int nrhs, long seed, int kind, cudaStream_t st)
{
    if (n <= 0) return cudaSuccess;
    const unsigned long long x_seed = ((((unsigned long long)seed) & 0xffffffffull) << 16) | 0x330Eull;
    const Affine step = lcg_jump(256);
    count_launch();
    gen_rows_kernel<<<n, 256, 0, st>>>(a, ld, n, x_seed, kind, step);
    if (nrhs > 1) {
        const long total = (long)n * (nrhs - 1);
        count_launch();
        gen_rhs_kernel<<<(unsigned)((total + 255) / 256), 256, 0, st>>>(a, ld, n, nrhs, x_seed);
    }
    return cudaGetLastError();
}

}  // namespace lu2gpu
