/*
 * lu2gpu.h -- C ABI of liblu2gpu.so, the B200 (sm_100a) implementation of
 * telmin/lu2's single-node blocked recursive LU with partial pivoting and its
 * solve.
 *
 * Two groups of entry points:
 *
 *  1. lu2's own signatures, drop-in replacements for the functions a caller of
 *     lu2 links against (paths within telmin/lu2).  All pointers are HOST
 *     pointers, as in the reference; the library stages them through the GPU.
 *     C99 VLA parameters of the reference (double a[n][n+16]) are ABI-identical
 *     to the plain pointers declared here.
 *
 *  2. a handle-based API on DEVICE pointers (the performance path: the matrix
 *     stays resident in HBM), returning int status codes.
 *
 * Status codes (group 2, and lu2gpu_lumcolumn): 0 ok; > 0 the factorization
 * met an exact zero pivot at column (status - 1) and completed without
 * scaling that column (LAPACK getrf's info convention); < 0 an error below.
 * lu2gpu_last_error() describes the last failure of the calling thread.
 *
 * The reference's own entry points return void.  On failure they print the
 * error and end the process (the reference's MP_error convention,
 * lu2_mp_nompi.c:55-58) unless lu2gpu_set_abort_on_error(0) was called;
 * gdr_dgemm_ instead reports through *doneflag = 0 (gdrdgemm.c:113-116).
 * There is no CPU fallback.
 *
 * Storage (same as lu2, lu2.c:28): row-major, leading dimension in doubles,
 * right-hand sides as augmented columns n..n+nrhs-1 that ride through every
 * swap and update (lu2.c:1138).  Factors: unit upper U' (pivot rows scaled by
 * 1/pivot, diagonal keeps the pivot) and L' below; earlier panels' L columns
 * are not swapped by later panels (lu2.c:543-553).  The full pivot sequence is
 * kept (0-based LAPACK ipiv order: row c was exchanged with row ipiv[c]).
 */
#ifndef LU2GPU_H
#define LU2GPU_H

#ifdef __cplusplus
extern "C" {
#endif

#define LU2GPU_OK 0
#define LU2GPU_ERR_ARG (-1)
#define LU2GPU_ERR_CUDA (-2)
#define LU2GPU_ERR_NOMEM (-3)
#define LU2GPU_ERR_TIMEOUT (-4) /* a bounded device wait gave up */
#define LU2GPU_ERR_NODEV (-5)
#define LU2GPU_ERR_NOCONV (-6) /* iterative refinement did not reach its residual bound */

/* pivot search */
#define LU2GPU_PIVOT_REF 0     /* bug-compatible with lu2tlib.c:1052 (see below) */
#define LU2GPU_PIVOT_PARTIAL 1 /* true partial pivoting (default) */

/* trailing-update precision of the precision form's factorization */
#define LU2GPU_UPDATE_BF16 0 /* BF16 operands, per-panel power-of-two scales */
#define LU2GPU_UPDATE_FP8 1  /* FP8 E4M3 operands, per-128x128-tile power-of-two scales */

/* CBLAS enum values (CBLAS_ORDER / CBLAS_TRANSPOSE) accepted by gdrblas_dgemm */
#define LU2GPU_CBLAS_ROWMAJOR 101
#define LU2GPU_CBLAS_COLMAJOR 102
#define LU2GPU_CBLAS_NOTRANS 111
#define LU2GPU_CBLAS_TRANS 112

/* ======================================================================
 * 1. Reference signatures (host pointers)
 * ====================================================================== */

/* lu2.c:1122-1144.  In-place LU of a[n][n+16] (row-major, b in column n) with
 * block size m (a multiple of 16), then backward substitution: x -> b[n].
 * a receives the factors (y in column n); pv[0..m) the last panel's pivot
 * rows, as the reference leaves them.  awork and recursive are accepted and
 * unused.  Pivot mode: LU2GPU_PIVOT_PARTIAL unless lu2gpu_set_pivot_mode()
 * or the environment variable LU2GPU_PIVOT=ref selects the reference's.
 * With a in pinned (or registered) host memory the copies overlap the
 * factorization: a goes to the GPU in column chunks while the first panels
 * are factored left-looking, and finished factor blocks come back while the
 * rest is factored; the result is bit-identical to the pageable path's. */
void lumcolumn(int n, double *a, double *b, int m, double *awork, int *pv, int recursive);

/* lu2.c's per-panel steps on the host matrix a[n][n+16] (each stages the
 * region it touches through the GPU; pivot mode as for lumcolumn):
 *  column_decomposition_recursive (lu2.c:1088-1120): factor the panel of
 *    columns i..i+m-1, rows i..n-1; pv[0..m) receives the pivot rows.
 *  process_right_part (lu2.c:524-581): apply pv[0..m) with the 1/pivot row
 *    scaling to columns i+m..iend-1, solve the U block row, update rows
 *    i+m..n-1 (m a multiple of 16 or not).
 *  backward_sub (lu2.c:110-116): b = x from the unit upper factor and column n.
 * awork is accepted and unused. */
void column_decomposition_recursive(int n, double *a, int m, double *awork, int *pv, int i);
void process_right_part(int n, double *a, int m, double *awork, int *pv, int i, int iend);
void backward_sub(int n, double *a, double *b);

/* lu2tlib.h:1-18, the column-major slab API (a[j][r] at a + j*n + r, i.e.
 * double a[n+1][n]): cm_column_decomposition_recursive (lu2tlib.c:1095-1128)
 * and cm_column_decomposition (lu2tlib.c:1041-1066, at most 16 columns; in
 * reference pivot mode every column searches the slab's first column, as
 * there) factor slab columns 0..m-1, rows i..n-1; cm_process_right_part
 * (lu2tlib.c:1068-1093) updates slab columns m..iend-i-1. */
void cm_column_decomposition_recursive(int n, double *a, int m, int *pv, int i);
void cm_column_decomposition(int n, double *a, int m, int *pv, int i);
void cm_process_right_part(int n, double *a, int m, int *pv, int i, int iend);

/* lu2lib.h:9-19, lu2lib.c:2079-2136: row-major C = alpha*A*B + beta*C.
 * This and the board-library DGEMMs below take host pointers; with C in
 * pinned host memory (and at least two ~16 MB column blocks of it) the copies
 * in, the products and the copies out of C's column blocks overlap on three
 * streams, bit-identical to the one-pass path (LU2GPU_DGEMM_OVERLAP=0 forces
 * that path). */
void mydgemm(int m, int n, int k, double alpha, double *a, int na, double *b, int nb, double beta, double *c,
             int nc);

/* lu2lib.h:2-7, lu2lib.c:1984-2077: C -= A*B, A (m x kk, stride n1),
 * B (kk x n, stride n2), C (m x n, stride n3), row-major. */
void matmul_for_small_nk(int n1, double *a, int n2, double *b, int n3, double *c, int m, int kk, int n);

/* lu2lib.c:2138-2168: initialise the offload device and run its self-test.
 * The GPU has no nb >= 2048 restriction; caller buffers are not touched. */
void reset_gdr(int m, double *a, int nb, double *awork, int n);

/* lu2lib.h:21-23: select the GPU (board id = CUDA device ordinal). */
void gdrsetboardid(int boardid);
/* lu2lib.c:2170-2178 board controls; accepted, no effect on a GPU. */
void gdrsetnboards(int nboards);
void gdrsetforceswapab(void);
void gdrresetforceswapab(void);
void gdrsetskipsendjmat(void);
void gdrresetskipsendjmat(void);
void set_matmul_msg_level(int level);
void gdrdgemm_set_stress_factor(int x);

/* The GRAPE-DR board library's symbols as gdrdgemm.c calls them
 * (gdrdgemm.c:55-56, 105-110, 171, 185-186; no header in the reference).
 * gdr_dgemm_: Fortran-style column-major C = alpha*op(A)*op(B) + beta*C,
 * *nota / *notb = 1 for no transpose, *doneflag = 1 on success, 0 on failure. */
void gdr_dgemm_(int *nota, int *notb, int *m, int *n, int *k, double *alpha, double *beta, int *lda, int *ldb,
                int *ldc, const double *a, const double *b, double *c, int *doneflag);
void gdr_init(void);
void gdr_free(void);
void gdrdgemm_set_procname(int procid);

/* gdrdgemm.h:15-37: CBLAS-style DGEMM (order/trans take the CBLAS enum values). */
void gdrblas_dgemm(int order, int transa, int transb, int M, int N, int K, double alpha, const double *A, int lda,
                   const double *B, int ldb, double beta, double *C, int ldc);

/* gdrdgemm.h:39-49: row-major C = alpha*A*B + beta*C. */
void mygdrdgemm(int m, int n, int k, double alpha, double *a, int na, double *b, int nb, double beta, double *c,
                int nc);

/* gdrdgemm.h:11-13, gdrdgemm.c:17-58: identity x B == B self-test on three
 * 2048x2048 host buffers, bounded to three attempts. */
void gdr_check_and_restart(double *a, double *b, double *c);

/* ======================================================================
 * 2. Device-resident API
 * ====================================================================== */

typedef struct lu2gpu_ctx lu2gpu_ctx;

/* One context per device; holds its stream, workspaces and pivot arrays. */
int lu2gpu_create(lu2gpu_ctx **ctx, int device);
int lu2gpu_destroy(lu2gpu_ctx *ctx);
/* Run on the caller's CUDA stream (a cudaStream_t) instead of the context's own. */
int lu2gpu_set_stream(lu2gpu_ctx *ctx, void *stream);

/* Factor the n x (n+nrhs) augmented row-major device matrix a (leading
 * dimension lda, even; a 16-byte aligned) in place with block size nb (a
 * multiple of 16): recursive panels down to 16 columns, lu2's storage.  The
 * right-hand-side columns come out forward-transformed (y).  ipiv (device,
 * n ints, may be NULL) receives the pivot sequence.  Synchronous.
 * From four panels up, the next panel is factored on a second stream of the
 * context (highest priority) while the rest of the trailing update runs
 * (the lookahead of lu2_mpi.c:3643-3847); every element sees the same
 * operations in the same order as in the serial schedule, so the result is
 * bit-identical.  LU2GPU_LOOKAHEAD=0 in the environment, or phase timing,
 * selects the serial schedule. */
int lu2gpu_factor(lu2gpu_ctx *ctx, int n, int nrhs, double *a, long lda, int nb, int pivot_mode, int *ipiv);

/* x = U'^{-1} y with the unit upper factor of a (lu2.c:110-116); y is the
 * n x nrhs device block x (row stride ldx), overwritten by x. */
int lu2gpu_backsolve(lu2gpu_ctx *ctx, int n, int nrhs, const double *a, long lda, double *x, long ldx);

/* Solve A x = b again from the factors an earlier lu2gpu_factor left in a,
 * with its pivot sequence ipiv (device) and its block size nb: the forward
 * solve applies, panel by panel, exactly what the factorization applied to its
 * augmented columns (pivots with 1/pivot scaling, unit-lower solve, update of
 * the rows below; lu2.c:524-581), then the back substitution.  lu2 itself
 * keeps only the last panel's pivots and cannot do this.  b (device, n x nrhs,
 * row stride ldb) is overwritten by x.  a is not modified. */
int lu2gpu_solve(lu2gpu_ctx *ctx, int n, const double *a, long lda, int nb, const int *ipiv, double *b, long ldb,
                 int nrhs);

/* lumcolumn on device memory: factor, then solve; x overwrites columns n..n+nrhs-1. */
int lu2gpu_lusolve(lu2gpu_ctx *ctx, int n, int nrhs, double *a, long lda, int nb, int pivot_mode, int *ipiv);

/* randomsetmat (lu2.c:70-85) on the device, bit-identical to glibc
 * srand48(seed)/drand48(): row i is n draws then b_i, each drand48()-0.5;
 * further right-hand sides continue the stream after the matrix.
 * kind 0: as lu2; kind 1: then a_ii = sum_j |a_ij| over the row (diagonally
 * dominant).  nrhs >= 1. */
int lu2gpu_generate(lu2gpu_ctx *ctx, int n, int nrhs, long seed, int kind, double *a, long lda);

/* Precision form (no counterpart in the reference, whose solver is FP64
 * only): solve A x = b for the FP64 n x n device matrix a (lda even, a
 * 16-byte aligned, not modified) by lu2's factorization of an FP32 copy --
 * the panel in FP32, the trailing updates as BF16 tensor-core products with
 * FP32 accumulation and per-panel power-of-two operand scales, block size nb
 * in {64, 128, 192, 256} -- followed by classical iterative refinement with
 * the residual r = b - A x and the update of x in FP64, until the HPL scaled
 * residual ||r||/(eps (||A|| ||x|| + ||b||) n) (inf-norms, eps = 2^-53) is
 * below 16 or max_iter corrections were applied.  b, x: device n-vectors.
 * out (host, may be NULL) receives {iterations, final scaled residual,
 * factorization seconds, refinement seconds}.  Returns 0 when the bound was
 * met, LU2GPU_ERR_NOCONV when not, > 0 on a zero pivot, < 0 on errors. */
int lu2gpu_mixed_solve(lu2gpu_ctx *ctx, int n, const double *a, long lda, const double *b, double *x, int nb,
                       int pivot_mode, int max_iter, double *out);

/* The precision form's trailing update on its own (the BF16 counterpart of
 * mmmulandsub, lu2.c:312-343): c (FP32, M x N, row stride ldc) -= scale *
 * a * bt^T with a (M x K) and bt (N x K) BF16 device matrices, K-contiguous
 * (row strides lda, ldb multiples of 8, 16-byte aligned), K in {64, 128,
 * 192, 256}; tcgen05 tensor cores with FP32 accumulation. */
int lu2gpu_bf16_update_dev(lu2gpu_ctx *ctx, int M, int N, int K, const void *a, long lda, const void *bt, long ldb,
                           float *c, long ldc, float scale);

/* GMRES-IR: A x = b (A FP64 n x n, row stride lda, 16-byte aligned, not
 * modified) with lu2's factorization of an FP32 copy -- the panel in FP32,
 * the trailing updates on the tensor cores with FP32 accumulation and `update`
 * operands: LU2GPU_UPDATE_BF16 (per-panel scales, nb in {64, 128, 192, 256})
 * or LU2GPU_UPDATE_FP8 (E4M3, per-128x128-tile scales, nb in {128, 256}) --
 * then iterative refinement whose residual r = b - A x and update of x are in
 * FP64 and whose correction equations A d = r are solved by GMRES(restart)
 * (restart <= 32) left-preconditioned by the low-precision factors, with FP64
 * Arnoldi vectors orthogonalised by classical Gram-Schmidt applied twice.  Each
 * correction is solved to a preconditioned relative residual of inner_tol.
 * Stops when the HPL scaled residual is below 16 or after max_iter GMRES
 * iterations in all.  out (host, may be NULL) receives {refinement steps,
 * GMRES iterations, final scaled residual, factorization seconds, refinement
 * seconds, 1 if the preconditioner stayed finite else 0}.  Returns 0 when the bound was met, LU2GPU_ERR_NOCONV when not,
 * > 0 on a zero pivot, < 0 on errors.  No counterpart in the reference. */
int lu2gpu_gmres_solve(lu2gpu_ctx *ctx, int n, const double *a, long lda, const double *b, double *x, int nb,
                       int update, int restart, double inner_tol, int max_iter, double *out);

/* The precision forms' factorization on its own (the preconditioner of
 * lu2gpu_mixed_solve and lu2gpu_gmres_solve; no counterpart in the
 * reference): lu2's LU (lu2.c:1122-1144 storage: row-scaled unit U', L'
 * below, earlier panels' L columns not swapped by later panels) of an FP32
 * copy of the FP64 device matrix a, the panels in FP32, the top-level trailing
 * updates with `update` operands (LU2GPU_UPDATE_BF16, nb in {64, 128, 192,
 * 256}; LU2GPU_UPDATE_FP8, nb in {128, 256}).  f (device, n x n FP32, row
 * stride ldf >= n) receives the factors, ipiv (device, n ints, may be NULL)
 * the pivot sequence.  a is not modified.  Synchronous; > 0 on a zero pivot. */
int lu2gpu_lowp_factor(lu2gpu_ctx *ctx, int n, const double *a, long lda, int nb, int update, float *f, long ldf,
                       int *ipiv);

/* The FP8 form's trailing update on its own: a (M x K) and bt (N x K) FP32
 * device matrices (row strides lda, ldb multiples of 4, 16-byte aligned) are
 * quantized to E4M3 with one power-of-two scale per 128 x 128 tile, then c
 * (FP32, M x N, row stride ldc) -= a_q * bt_q^T on the tcgen05 tensor cores
 * (kind::f8f6f4, FP32 accumulation), K in {128, 256}.  a_deq / bt_deq (device,
 * may be NULL) receive the dequantized operands (M x K, N x K, contiguous). */
int lu2gpu_fp8_update_dev(lu2gpu_ctx *ctx, int M, int N, int K, const float *a, long lda, const float *bt, long ldb,
                          float *c, long ldc, float *a_deq, float *bt_deq);

/* Batching form (no counterpart in the reference, which solves one system
 * per run): many independent systems of uneven order, each lu2's augmented
 * problem (row-major, b in columns n..n+nrhs-1, x replaces b) solved with
 * lu2's algorithm, all in one persistent launch replayed from a CUDA graph. */
typedef struct lu2gpu_batch lu2gpu_batch;
/* Describe count systems (orders n[i] <= 4096, nrhs[i] <= 64 right-hand
 * sides; nrhs may be NULL for one each) and allocate their packed storage. */
int lu2gpu_batch_create(lu2gpu_ctx *ctx, int count, const int *n, const int *nrhs, lu2gpu_batch **out);
/* Frees the batch; call it before lu2gpu_destroy of the batch's context (the
 * batch's memory and streams belong to that context). */
int lu2gpu_batch_destroy(lu2gpu_batch *b);
/* Device pointer to system i's augmented matrix and its row stride. */
int lu2gpu_batch_system(lu2gpu_batch *b, int i, double **a, long *ld);
/* System i := lu2's randomsetmat stream with seed (seed + i). */
int lu2gpu_batch_generate(lu2gpu_batch *b, long seed);
/* System i := lu2's randomsetmat stream with seed seeds[i] (host, count
 * seeds), so that a shard of a batch holds the same systems as the whole. */
int lu2gpu_batch_generate_seeds(lu2gpu_batch *b, const long long *seeds);
/* Keep a copy of the current systems (for residuals and for re-running). */
int lu2gpu_batch_snapshot(lu2gpu_batch *b);
int lu2gpu_batch_restore(lu2gpu_batch *b);
/* Arithmetic of lu2gpu_batch_solve: LU2GPU_BATCH_FP64 (default) factors and
 * solves in FP64; LU2GPU_BATCH_FP32_IR factors an FP32 copy of each system
 * (full-width row exchanges, lu2's 1/pivot row scaling) and refines x in
 * FP64 -- r = b - A x from the unchanged FP64 system, corrections from the
 * FP32 factors -- until every right-hand side's HPL scaled residual is below
 * 16 or max_iter corrections were applied (systems with at most 8 right-hand
 * sides).  Resets the launch shape to the mode's default. */
#define LU2GPU_BATCH_FP64 0
#define LU2GPU_BATCH_FP32_IR 1
int lu2gpu_batch_set_mode(lu2gpu_batch *b, int mode, int max_iter);
/* Corrections each system took in the last FP32_IR solve (count ints). */
int lu2gpu_batch_iterations(lu2gpu_batch *b, int *iters_host);
/* Launch shape: threads per CTA (64..512, a multiple of 32), panel width of
 * the blocked path (16..64), CTAs per SM. */
int lu2gpu_batch_set_config(lu2gpu_batch *b, int threads, int pw, int ctas_per_sm);
/* Time the launch shapes on this batch (the median of three launches per
 * candidate) and keep the fastest; in the FP64 mode then the panel width of
 * each size bucket (n in [1,64), [64,128), [128,256), [256,...)) the same way.
 * params_out (4 ints, may be NULL) = {threads, panel width, CTAs per SM,
 * microseconds}.  lu2gpu_batch_set_config and lu2gpu_batch_set_mode reset the
 * bucket widths.  No counterpart in lu2, whose block size is a fixed
 * command-line value (lu2.c:1220-1240). */
int lu2gpu_batch_autotune(lu2gpu_batch *b, int *params_out);
/* The autotuned panel width per size bucket: out[2k] = the smallest n of
 * bucket k, out[2k+1] = its width (0: the launch's); 8 ints. */
int lu2gpu_batch_bucket_pw(lu2gpu_batch *b, int *out);
/* Factor and solve all systems in place; info_host (count ints, may be NULL)
 * receives each system's zero-pivot status (0 or column + 1). */
int lu2gpu_batch_solve(lu2gpu_batch *b, int *info_host);
/* HPL scaled residual of every system against the snapshot (host out[count]). */
int lu2gpu_batch_residuals(lu2gpu_batch *b, double *out_host);
/* Orders log-uniform in [nmin, nmax] and, for a fraction frac_multi of the
 * systems, nrhs_multi right-hand sides, from a seeded drand48 stream. */
int lu2gpu_batch_sizes(int count, long seed, int nmin, int nmax, double frac_multi, int nrhs_multi, int *n_out,
                       int *nrhs_out);

/* Row-major device DGEMM, C = alpha*A*B + beta*C (mydgemm's contract). */
int lu2gpu_dgemm_dev(lu2gpu_ctx *ctx, int m, int n, int k, double alpha, const double *a, long lda, const double *b,
                     long ldb, double beta, double *c, long ldc);

/* Copy the context's last pivot sequence (n ints) to host memory. */
int lu2gpu_copy_pivots(lu2gpu_ctx *ctx, int *ipiv_host, int n);

/* lumcolumn with an explicit pivot mode and a status code instead of exit. */
int lu2gpu_lumcolumn(int n, double *a, double *b, int m, int *pv, int pivot_mode);

/* The context behind the reference-signature entry points (device set by
 * gdrsetboardid, default 0); lu2gpu_release() frees it. */
lu2gpu_ctx *lu2gpu_default_context(void);
int lu2gpu_release(void);

/* Pivot mode of lumcolumn (returns the previous mode). */
int lu2gpu_set_pivot_mode(int mode);
/* 1 (default): the reference's void entry points exit(-1) on failure; 0: they
 * return after printing.  Returns the previous setting. */
int lu2gpu_set_abort_on_error(int on);
const char *lu2gpu_last_error(void);

/* Per-phase CUDA-event timers (the GPU counterpart of lu2's timerlib):
 * 0 "col dec t" panel leaves, 1 "swaprows", 2 "solve tri", 3 "DGEMMrest"
 * trailing update, 4 "backward_sub", 5 "panel update" (the swaps, solves and
 * updates inside the panel recursion).  get_timers fills ms[] and counts[] (launches)
 * for up to nmax phases, returns the number of phases. */
int lu2gpu_set_timing(lu2gpu_ctx *ctx, int enable);
int lu2gpu_get_timers(lu2gpu_ctx *ctx, double *ms, long *counts, int nmax, int reset);
const char *lu2gpu_timer_name(int phase);

/* Number of CUDA kernels this library has launched in the process so far. */
long lu2gpu_kernel_launches(void);

/* Fault-path test hook (no counterpart in the reference): the panel leaf of
 * ctx's later factorizations gives up its cross-CTA waits after wait_ms
 * milliseconds (0 restores the default, 2000), and, when cta >= 0, CTA `cta`
 * of every leaf skips its publications, so that every wait of that leaf runs
 * out.  The call then returns LU2GPU_ERR_TIMEOUT; kernels after the failed
 * one do nothing that depends on the pivots it never wrote, and the context
 * stays usable.  lu2gpu_test_leaf_withhold(ctx, -1, 0) switches it off. */
int lu2gpu_test_leaf_withhold(lu2gpu_ctx *ctx, int cta, double wait_ms);

/* lu2.c:485-521 (solve_triangle: U12 = L11^{-1} A12) on the device: x (K x
 * ncols, row stride ldx) := T^{-1} x, T the unit lower triangle whose strict
 * lower part is that of the K x K block t (row stride ldt), K <= 512; bt
 * (device, may be NULL) receives -x^T (ncols x K, K-contiguous), the operand
 * the trailing update reads.  With K a multiple of 16 up to 256 and 16-byte
 * aligned operands with even strides it runs on the FP64 tensor pipe.
 * Synchronous. */
int lu2gpu_solve_triangle_dev(lu2gpu_ctx *ctx, int K, const double *t, long ldt, double *x, long ldx, int ncols,
                              double *bt);

/* lu2.c:251-291 (swaprows_simple_with_scale, as lu2.c:541-554 applies a
 * panel's pivots) on the device: for k = k0..k1-1 in order, exchange rows k and
 * ipiv[k] of columns cs..ce-1 of the n-row row-major device matrix a (leading
 * dimension lda), then multiply row k by dinv[k] (dinv NULL: no scaling).
 * k1 - k0 <= 512; every ipiv[k] must lie in [k, n), else LU2GPU_ERR_ARG and
 * a is left unchanged.  Synchronous. */
int lu2gpu_swaprows_dev(lu2gpu_ctx *ctx, int n, double *a, long lda, int k0, int k1, const int *ipiv,
                        const double *dinv, int cs, int ce);

/* lu2gpu_lusolve without any device allocation.  No counterpart in the
 * reference: it exists for callers that cannot allocate device memory at the
 * time they solve -- because another allocator already owns the device memory
 * (a framework's caching allocator, a fixed memory budget), or because
 * cudaMalloc/cudaFree would synchronize the whole device.  All scratch (pivot
 * workspace, the transposed U block row, panel-exchange buffers, status words)
 * comes from one fixed file-scope device array of about 2.1 MB that every GPU
 * loading this library keeps until the process exits.  Limits: n <= 2048,
 * 1 <= nrhs <= 16, 16 <= nb <= 128 (multiple of 16); larger sizes are
 * rejected with LU2GPU_ERR_ARG.  a (device, lda even, 16-byte aligned) is
 * factored and solved in place like lu2gpu_lusolve; ipiv (device, n ints) may
 * be NULL.  Runs on `stream` (a cudaStream_t, NULL = the legacy default
 * stream) on the current device and waits for it.  The first call on a device
 * looks up the array's device address and the leaf kernel's launch limits for
 * that device.  All calls share the one array, whose contents persist between
 * calls: calls that overlap on the GPU (other streams, other host threads)
 * race on it and must be serialized by the caller. */
int lu2gpu_lusolve_noalloc(int n, int nrhs, double *a, long lda, int nb, int pivot_mode, int *ipiv, void *stream);

#ifdef __cplusplus
}
#endif
#endif /* LU2GPU_H */
