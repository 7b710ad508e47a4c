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

cudaError_t launch_backsolve(const double *a, long ld, int n, int nrhs, double *x, long ldx, cudaStream_t st)
{
    return launch_backsolve_t(a, ld, n, nrhs, x, ldx, st);
}

cudaError_t launch_backsolve(const float *a, long ld, int n, int nrhs, float *x, long ldx, cudaStream_t st)
{
    return launch_backsolve_t(a, ld, n, nrhs, x, ldx, st);
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
