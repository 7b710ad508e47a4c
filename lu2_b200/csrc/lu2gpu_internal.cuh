// lu2gpu_internal.cuh -- shared declarations of the sm_100a LU library.
//
// Storage convention (same as lu2, lu2.c:28 and lu2.c:1122-1144): the matrix
// is row-major, `ld` doubles per row, with the right-hand sides riding along
// as the augmented columns n..n+nrhs-1.  Pivot rows are scaled by 1/pivot in
// every column except the diagonal (unit upper U, lu2.c:551-552,
// lu2tlib.c:1057-1059); L columns of earlier panels are not swapped by later
// panels (lu2.c:543-553).  The full pivot sequence ipiv[0..n) (0-based, LAPACK
// order) and dinv[c] = 1/pivot are kept on the device.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace lu2gpu {

// device status words (int[4]) written by kernels
//   [0] first zero pivot: column + 1 (atomicMin; INFO_NONE when none)
//   [1] error bits below
//   [2] where the first error happened (kernel id)
enum : int {
    ERR_BARRIER_TIMEOUT = 1,
    ERR_MBAR_TIMEOUT = 2,
    ERR_BAD_ARG = 4,
};
constexpr int INFO_NONE = 0x7f7f7f7f;  // memset byte 0x7f
constexpr unsigned long long WAIT_LIMIT_NS = 2000000000ull;  // every device wait gives up after 2 s

constexpr int PIVOT_REF = 0;       // lu2 as shipped: 2nd column of each 2-column leaf pivots on the 1st
constexpr int PIVOT_PARTIAL = 1;   // partial pivoting
constexpr int PIVOT_REF_FIRST = 2; // lu2tlib.c column_decomposition called directly on a wider slab:
                                   // every column searches the slab's first column

__device__ __forceinline__ unsigned long long globaltimer_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void record_error(int *status, int bit, int where)
{
    if (atomicOr(&status[1], bit) == 0) atomicExch(&status[2], where);
}

// Stamped publication between CTAs without fences: a double travels as two
// 64-bit words, each a 32-bit stamp (the publication's tag, never 0) beside
// 32 bits of the value; a reader re-loads until both words carry the tag it
// waits for (aligned 64-bit accesses are single-copy atomic).
__device__ __forceinline__ void st_stamped(unsigned long long *p, unsigned tag, double x)
{
    const unsigned long long b = (unsigned long long)__double_as_longlong(x), t = (unsigned long long)tag << 32;
    const unsigned long long hi = t | (b >> 32), lo = t | (b & 0xffffffffull);
    asm volatile("st.relaxed.gpu.global.v2.u64 [%0], {%1, %2};" ::"l"(p), "l"(hi), "l"(lo) : "memory");
}

__device__ __forceinline__ void ld_pair(const unsigned long long *p, unsigned long long &a, unsigned long long &b)
{
    asm volatile("ld.relaxed.gpu.global.v2.u64 {%0, %1}, [%2];" : "=l"(a), "=l"(b) : "l"(p) : "memory");
}

__device__ __forceinline__ bool stamped(unsigned long long w, unsigned tag) { return (unsigned)(w >> 32) == tag; }

__device__ __forceinline__ double unstamp(unsigned long long hi, unsigned long long lo)
{
    return __longlong_as_double((long long)((hi << 32) | (lo & 0xffffffffull)));
}

// (value, row) ordering for the pivot search: larger |a| wins, ties go to the
// lower row index (cblas_idamax semantics, lu2tlib.c:47).
__device__ __forceinline__ bool argmax_better(double v1, int i1, double v2, int i2)
{
    return v1 > v2 || (v1 == v2 && i1 < i2);
}

__device__ __forceinline__ void warp_argmax(double &v, int &i)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        double ov = __shfl_xor_sync(0xffffffffu, v, o);
        int oi = __shfl_xor_sync(0xffffffffu, i, o);
        if (argmax_better(ov, oi, v, i)) {
            v = ov;
            i = oi;
        }
    }
}

// ---------------------------------------------------------------------------
// host-side launchers (all asynchronous on `st`)

// process-wide count of this library's kernel launches (lu2gpu_kernel_launches)
void count_launch(long k = 1);

// One CTA's publication for one leaf column.  Every 64-bit word carries the
// column's 32-bit stamp in its high half and 32 bits of payload in its low
// half, so a reader validates each word it loads by its stamp (each aligned
// 64-bit access is single-copy atomic) without release/acquire ordering.
struct __align__(64) LeafSlot {
    unsigned long long head[4];   // |a| of the candidate (high, low halves), its row (INT_MAX if none), unused
    unsigned long long row[32];   // the candidate row's 16 leaf columns, two words per double
    unsigned long long rowc[32];  // row c, written by the CTA owning row c only
};

struct LeafBuffers {
    LeafSlot *slots = nullptr;          // [2][max CTAs], zeroed once
    unsigned long long *seq = nullptr;  // host-side stamp counter, advanced by every leaf launch
    // fault-path test hook (lu2gpu_test_leaf_withhold): the wait limit of the
    // exchange, and a CTA that skips its publications (-1: none) so that every
    // other CTA's wait runs out
    unsigned long long wait_ns = WAIT_LIMIT_NS;
    int withhold = -1;
};

// Factor the leaf panel: rows c0..n-1, columns c0..c0+w-1 (w <= 16) of the
// view `a` whose element (0,0) is global (goff, goff).  ipiv/dinv are indexed
// by view column; ipiv receives global row numbers (view row + goff).
cudaError_t launch_leaf(double *a, long ld, int n, int c0, int w, int mode, int goff, int *ipiv, double *dinv,
                        const LeafBuffers &buf, int *status, int max_ctas, cudaStream_t st);
cudaError_t launch_leaf(float *a, long ld, int n, int c0, int w, int mode, int goff, int *ipiv, float *dinv,
                        const LeafBuffers &buf, int *status, int max_ctas, cudaStream_t st);
int leaf_max_ctas(int device);
// fewest leaf CTAs whose slabs of `rows` rows (elements of tsize bytes) fit shared memory
int leaf_min_ctas(int rows, size_t tsize);

// Apply the pivots k0..k1-1 (row k <-> row ipiv[k], in order; k1 - k0 <= 512)
// to columns cs..ce-1 of the nrows-row matrix and, when `scale`, multiply row
// k by dinv[k] after its swap.  ipiv holds global rows; the view's row is
// ipiv[k] - goff.  A pivot outside [k, nrows) sets ERR_BAD_ARG in status[1]
// and nothing is written; with status[1] already nonzero nothing is done.
cudaError_t launch_laswp_scale(double *a, long ld, int nrows, int k0, int k1, const int *ipiv, int goff,
                               const double *dinv, int cs, int ce, bool scale, int *status, cudaStream_t st);
cudaError_t launch_laswp_scale(float *a, long ld, int nrows, int k0, int k1, const int *ipiv, int goff,
                               const float *dinv, int cs, int ce, bool scale, int *status, cudaStream_t st);

// In place X := T^{-1} X for the unit lower triangle T = strict lower part of
// a[r0..r0+K)[r0..r0+K) and X = a[r0..r0+K)[cs..ce); also writes
// bt[(j-cs)*K + l] = -X[l][j] (the negated transposed block row the update GEMM adds).
cudaError_t launch_trsm_unit_lower(double *a, long ld, int r0, int K, int cs, int ce, double *bt, cudaStream_t st);
// The same with the triangle T (row stride ldt) and the K x ncols block X
// (row stride ldx) given separately; bt may be null.
cudaError_t launch_trsm_unit_lower_tx(const double *t, long ldt, double *x, long ldx, int K, int ncols, double *bt,
                                      cudaStream_t st);
// FP32 versions for the precision form; the _bf16 one writes the transposed
// block row as BF16 multiplied by *bt_scale (a device scalar).
cudaError_t launch_trsm_unit_lower_f32(const float *t, long ldt, float *x, long ldx, int K, int ncols, float *bt,
                                       cudaStream_t st);
cudaError_t launch_trsm_unit_lower_f32_bf16(const float *t, long ldt, float *x, long ldx, int K, int ncols, void *bt,
                                            const float *bt_scale, cudaStream_t st);

// C[m][n] += sum_k A[m][k] * Bt[n][k] with Bt = -U12^T (as the block solve
// writes it), i.e. the trailing update C - L21 U12.  A is the
// row-major matrix starting at (a_row0, a_col0) of `a` (stride ld, rows < a_rows
// exist); Bt is (N x K) row-major with stride K.  K % 16 == 0.
cudaError_t launch_dgemm_update(const double *a, long ld, int a_rows, int a_row0, int a_col0, const double *bt,
                                double *c, long ldc, int M, int N, int K, int *status, cudaStream_t st);

// General C = alpha * X * Y^T + beta * C (row-major C, M x N), X (M x K) and Y
// (N x K) both K-contiguous with strides ldx, ldy (device pointers).
cudaError_t launch_dgemm_general(const double *x, long ldx, const double *y, long ldy, double *c, long ldc, int M,
                                 int N, int K, double alpha, double beta, int *status, cudaStream_t st);

// out[j][i] = in[i][j] for an (rows x cols) block; strides in doubles.
cudaError_t launch_transpose(const double *in, long ldi, double *out, long ldo, int rows, int cols, cudaStream_t st);

// x = U'^{-1} y for the unit upper triangle of a[0..n)[0..n) (lu2's backward_sub,
// lu2.c:110-116); y (n x nrhs, row stride ldx) is overwritten by x.  For lu2's
// own layout x = a + n, ldx = ld.  With bs (a stamped x slot for each of the
// n / 64 blocks, zeroed once; a host epoch counter; the status words) and
// n >= BSP_PERSISTENT_MIN_N one persistent cooperative launch per 8
// right-hand sides does it; otherwise blocked launches (one per 128-row block
// and one per update).
constexpr int BS_SLOT_WORDS = 64 * 8 * 2;  // 64 rows x 8 right-hand sides, two stamped words each
struct BsBuffers {
    unsigned long long *xslots = nullptr;  // [cap][BS_SLOT_WORDS], zeroed at allocation
    int cap = 0;
    unsigned *epoch = nullptr;  // host-side counter, advanced per launch
    int *status = nullptr;
};
constexpr int BSP_PERSISTENT_MIN_N = 4096;
cudaError_t launch_backsolve(const double *a, long ld, int n, int nrhs, double *x, long ldx, const BsBuffers *bs,
                             cudaStream_t st);
cudaError_t launch_backsolve(const float *a, long ld, int n, int nrhs, float *x, long ldx, const BsBuffers *bs,
                             cudaStream_t st);

// out[k] = 1 / a[k][k] (1 for an exactly zero pivot)
cudaError_t launch_diag_inv(const double *a, long ld, int n, double *out, cudaStream_t st);
cudaError_t launch_diag_inv(const float *a, long ld, int n, float *out, cudaStream_t st);

// ---------------------------------------------------------------------------
// precision form (kernels_bf16.cu, kernels_mixed.cu; the trailing update in kernels_lowp.cu)

// out = BF16(in * *scale) for a rows x cols FP32 block
cudaError_t launch_f32_to_bf16(const float *in, long ldi, void *out, long ldo, int rows, int cols,
                               const float *scale, cudaStream_t st);
// C (FP32) -= A Bt^T, A (M x K, stride lda), Bt (N x K, stride K): the
// updates inside the FP32 panel recursion (CUDA cores, exact FP32)
cudaError_t launch_sgemm_update(const float *a, long lda, const float *bt, float *c, long ldc, int M, int N, int K,
                                cudaStream_t st);
// per-panel power-of-two scales for the BF16 operands: scales[0] = 1/sL,
// scales[1] = 1/sU, scales[2] = sL*sU with sX = 2^ceil(log2(max|X|)) of the
// rows x cols block X (called once per block; amax[] accumulates maxima)
cudaError_t launch_absmax(const float *x, long ld, int rows, int cols, unsigned *amax_bits, cudaStream_t st);
cudaError_t launch_panel_scales(const unsigned *amax_bits, float *scales, cudaStream_t st);
// y = FP32(x) for an n x cols FP64 block and back
cudaError_t launch_f64_to_f32(const double *x, long ldx, float *y, long ldy, int rows, int cols, cudaStream_t st);
cudaError_t launch_f32_to_f64(const float *x, long ldx, double *y, long ldy, int rows, int cols, cudaStream_t st);
// r = b - A x (FP64, A n x n stride lda, b and x n-vectors), or r = A x when b
// is null; rowabs (optional) receives sum_j |a_ij| for the HPL norm
cudaError_t launch_residual(const double *a, long lda, int n, const double *b, const double *x, double *r,
                            double *rowabs, cudaStream_t st);
// per-panel update of the forward solve: y[rows] -= L (rows x K, stride ld) * v (K)
cudaError_t launch_gemv_sub(const float *l, long ld, int rows, int K, const float *v, float *y, cudaStream_t st);
// bt (N x K BF16) = transpose of u (K x N FP32, stride ld) * *scale
cudaError_t launch_f32_transpose_bf16(const float *u, long ld, int K, int N, void *bt, const float *scale,
                                      cudaStream_t st);
// x += (double) d
cudaError_t launch_add_f32_to_f64(const float *d, double *x, int n, cudaStream_t st);

// ---------------------------------------------------------------------------
// batching form (kernels_batch.cu)

// one system of a batch: its augmented matrix (n x (n+nrhs), row stride ld)
// starts at data + off; pw = the panel width of its blocked path (0: the
// launch's), set per size bucket by the autotuner
struct BatchSys {
    long long off;
    int n, nrhs, ld, pw;
};
// The row exchanges of one panel composed into a plan: U row q takes the
// content of panel row blk[q], and the rows ext_row[e] >= w take the old
// content of U row ext_src[e] (every displaced row receives a U row, since
// each exchange moves row c < w).
struct BatchPlan {
    int blk[64];
    int ext_row[64];
    int ext_src[64];
    int next;
};

// warp 0, once the pivot p of column c is known: compose c <-> p into the
// plan (the rows >= w already displaced are searched by the whole warp)
__device__ __forceinline__ void batch_plan_step(BatchPlan &s, int c, int p, int w, int lane)
{
    const int ne = s.next;
    unsigned hit = 0;
    for (int e0 = 0; e0 < ne; e0 += 32) {
        const unsigned b = __ballot_sync(0xffffffffu, e0 + lane < ne && s.ext_row[e0 + lane] == p);
        if (b && !hit) hit = (unsigned)(e0 + __ffs(b));  // index + 1
    }
    if (lane == 0) {
        const int xc = s.blk[c];
        if (p < w) {
            s.blk[c] = s.blk[p];
            s.blk[p] = xc;
        } else if (p != c) {
            int e = (int)hit - 1;
            if (!hit) {
                e = ne;
                s.ext_row[e] = p;
                s.ext_src[e] = p;
                s.next = e + 1;
            }
            s.blk[c] = s.ext_src[e];
            s.ext_src[e] = xc;
        }
    }
    __syncwarp();
}

// dynamic shared memory a CTA of the batched launch may use
constexpr size_t BATCH_SMEM_MAX = 220 * 1024;
// blocked path: panel row stride pw + BATCH_PANEL_PAD (odd, so that lanes on
// consecutive rows hit different banks); the U chunk of the update
constexpr int BATCH_PANEL_PAD = 1;
constexpr int BATCH_UNIT_COLS = 32;  // columns of a warp's update tile, 16 rows x this (16 measured slower: 41.3 vs 40.9 ms)
constexpr int BATCH_U_CHUNK = 64;  // columns of U12 staged per update step (128 measured slower: 42.3 vs 40.9 ms)
constexpr int BATCH_U_STRIDE = BATCH_U_CHUNK + 4;  // B-fragment reads of a half-warp on distinct banks
// shared-memory doubles a CTA needs for the systems sys[0..count) with panel width pw
long batch_smem_doubles(const BatchSys *sys, int count, int pw);
// persistent grid for a launch shape (sets the kernel's shared-memory limit;
// call outside stream capture)
cudaError_t batch_lu_grid(int threads, long smem_doubles, int ctas_per_sm, int count, int *grid);
// factor + solve every system, CTAs pulling systems in `order` from `counter`
cudaError_t launch_batch_lu(double *data, const BatchSys *sys, const int *order, int count, int *counter, int *info,
                            long smem_doubles, int pw, int threads, int grid, cudaStream_t st);
cudaError_t launch_batch_residual(const double *orig, const double *solved, const BatchSys *sys, int count,
                                  double *out, cudaStream_t st);

// FP32-LU + FP64 refinement variant (kernels_batch_ir.cu).  Work arena slot
// of a system: FP32 factors (n x n), pivots (n), x and r (n x nrhs doubles).
constexpr int IR_MAX_RHS = 8;
__host__ __device__ inline size_t ir_align16(size_t b) { return (b + 15) & ~(size_t)15; }
__host__ __device__ inline size_t ir_slot_bytes(int n, int nrhs)
{
    return ir_align16((size_t)n * n * 4) + ir_align16((size_t)n * 4) + (size_t)16 * n * nrhs;
}
// shared-memory floats a CTA needs: the blocked path of every system, at least floor_floats
long batch_ir_smem_floats(const BatchSys *sys, int count, int pw, long floor_floats);
cudaError_t batch_ir_grid(int threads, long smem_floats, int ctas_per_sm, int count, int *grid);
cudaError_t launch_batch_ir(double *data, const BatchSys *sys, const long long *woff, uint8_t *arena,
                            const int *order, int count, int *counter, int *info, int *iters, long smem_floats, int pw,
                            int threads, int grid, int max_iter, cudaStream_t st);
// system i := lu2's randomsetmat stream with seed seeds[i] (device list) or seed_base + i
cudaError_t launch_batch_generate(double *data, const BatchSys *sys, int count, unsigned long long seed_base,
                                  const long long *seeds, cudaStream_t st);
// *out = max(*out, max |v|) as double bits
cudaError_t launch_vec_absmax(const double *v, int n, unsigned long long *out, cudaStream_t st);

// persistent warp-specialized trailing update of the precision forms
// (kernels_lowp.cu): C (FP32, 16-byte aligned, ldc a multiple of 4) -=
// *scale * A Bt^T with BF16 operands (K a multiple of 64, <= 256), or
// -= sum_kb da db Aq_kb Bq_kb^T with E4M3 operands and per-tile scales (K = 128 or 256)
// (max_ctas > 0 caps the persistent grid, leaving SMs free for a concurrent panel)
cudaError_t launch_lowp_update_bf16(const void *a16, long lda, const void *bt16, long ldb, float *c, long ldc, int M,
                                    int N, int K, const float *scale, int *status, int max_ctas, cudaStream_t st);
cudaError_t launch_lowp_update_fp8(const uint8_t *a8, long lda, const float *da, const uint8_t *bt8, long ldb,
                                   const float *db, float *c, long ldc, int M, int N, int K, int *status,
                                   int max_ctas, cudaStream_t st);

// FP8 form operands (kernels_fp8.cu): per-128x128-tile E4M3 quantization with power-of-two scales; dq = [ceil(rows/128)][cols/128]
cudaError_t launch_quant_fp8_tiles(const float *x, long ldx, int rows, int cols, uint8_t *q, long ldq, float *dq,
                                   cudaStream_t st);
cudaError_t launch_dequant_fp8_tiles(const uint8_t *q, long ldq, const float *dq, int rows, int cols, float *y,
                                     long ldy, cudaStream_t st);

// GMRES vector kernels (kernels_gmres.cu)
constexpr int MULTI_DOT_BLOCKS = 148;
// out[j] = <V[j], z>, j < k; partial: k * MULTI_DOT_BLOCKS doubles
cudaError_t launch_multi_dot(const double *V, long ldv, int k, const double *z, int n, double *partial, double *out,
                             cudaStream_t st);
// z += sign * sum_{j<k} c[j] V[j] (k <= 64, c on the device)
cudaError_t launch_multi_axpy(const double *V, long ldv, int k, const double *c, double sign, double *z, int n,
                              cudaStream_t st);
cudaError_t launch_vec_scale(const double *x, double alpha, double *y, int n, cudaStream_t st);

// lu2's matrix generator (randomsetmat, lu2.c:70-85) on the device, bit-identical to
// glibc drand48: row i holds draws i*(n+1) .. i*(n+1)+n (b_i last); extra
// right-hand sides continue the stream.  kind 1 then sets a_ii = sum_j |a_ij|.
cudaError_t launch_generate(double *a, long ld, int n, int nrhs, long seed, int kind, cudaStream_t st);

}  // namespace lu2gpu
