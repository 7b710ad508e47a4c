/*
 * lu2_oracle.c -- CPU restatement of lu2's single-node factor + solve path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA path in
 * lu2_b200/: it is compiled into oracle/liblu2oracle.so and loaded by tests/,
 * by __graft_entry__.smoke() and by bench.py's cpu_baseline leg.  Nothing in
 * the product library links, loads or calls it.
 *
 * What it restates (reference file:line, paths within telmin/lu2):
 *   - randomsetmat               lu2.c:70-85      glibc srand48/drand48 stream
 *   - lumcolumn                  lu2.c:1122-1144  panel loop + backward_sub
 *   - column_decomposition_recursive (row-major)    lu2.c:1088-1120
 *   - column_decomposition_with_transpose           lu2.c:1072-1085
 *     (the transpose to a column-major slab is a storage detail; the
 *      arithmetic below works on the row-major matrix directly)
 *   - column_decomposition_recursive (slab)         lu2tlib.c:1095-1128
 *   - column_decomposition (2-column leaf)          lu2tlib.c:1041-1066
 *   - findpivot (cblas_idamax, first max wins)      lu2tlib.c:42-52
 *   - process_right_part (slab)                     lu2tlib.c:1068-1093
 *   - process_right_part (row-major, swap+scale, solve_triangle, update)
 *                                                   lu2.c:524-581
 *   - solve_triangle / solve_triangle_for_unit_mat{,_recursive,_internal}
 *                                                   lu2.c:370-521
 *   - mmmulandsub                                   lu2.c:312-343
 *   - backward_sub                                  lu2.c:110-116
 *
 * Pivot modes:
 *   ORC_PIVOT_REF     -- what the shipped reference computes: inside every
 *                        2-column leaf the pivot of the second column is
 *                        searched in the first column (lu2tlib.c:1052 passes
 *                        the leaf pointer `a`, and findpivot scans a[0],
 *                        lu2tlib.c:47).
 *   ORC_PIVOT_PARTIAL -- true partial pivoting (each column searches itself).
 *
 * The stored factors follow lu2 (row-scaled unit-U, L not swapped by later
 * panels, b riding along as the augmented columns n..n+nrhs-1).  The full
 * pivot sequence (LAPACK ipiv, 0-based) is returned, which lu2 itself keeps
 * only per panel.
 *
 * The reference needs nb to be a power of two and n a multiple of nb
 * (lu2.c:1088-1120 halves m with integer division); the oracle checks this.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>

#define ORC_PIVOT_REF 0
#define ORC_PIVOT_PARTIAL 1

#define A_(r, c) (o->a[(size_t)(r) * (size_t)o->lda + (size_t)(c)])

typedef struct {
    int n;       /* matrix order */
    int ncols;   /* n + nrhs: last column (exclusive) of every right-part update */
    long lda;    /* row stride in doubles */
    double *a;   /* row-major augmented matrix */
    int *ipiv;   /* global pivot sequence, length n */
    int mode;
} orc_t;

/* ---------------------------------------------------------------------- */
/* drand48 stream (glibc): X' = 0x5DEECE66D * X + 0xB mod 2^48,
 * srand48(s) sets X = (s & 0xffffffff) << 16 | 0x330E, drand48() = X * 2^-48. */

#define LCG_A 0x5DEECE66DULL
#define LCG_C 0xBULL
#define LCG_MASK ((1ULL << 48) - 1)

uint64_t orc_lcg_seed(long seed)
{
    return ((((uint64_t)seed) & 0xffffffffULL) << 16) | 0x330EULL;
}

double orc_lcg_next(uint64_t *x)
{
    *x = (LCG_A * (*x) + LCG_C) & LCG_MASK;
    return (double)(*x) * (1.0 / 281474976710656.0);
}

/* randomsetmat (lu2.c:70-85): row i gets n draws for A[i][0..n-1], then one
 * draw for b_i = A[i][n]; every draw is drand48() - 0.5.  Extra right-hand
 * sides (nrhs > 1) continue the same stream after the whole matrix. */
void orc_randomsetmat(int n, int nrhs, long seed, double *a, long lda)
{
    uint64_t x = orc_lcg_seed(seed);
    for (long i = 0; i < n; i++) {
        double *ap = a + (size_t)i * (size_t)lda;
        for (long j = 0; j < n; j++) ap[j] = orc_lcg_next(&x) - 0.5;
        ap[n] = orc_lcg_next(&x) - 0.5;
    }
    for (int r = 1; r < nrhs; r++)
        for (long i = 0; i < n; i++)
            a[(size_t)i * (size_t)lda + n + r] = orc_lcg_next(&x) - 0.5;
}

/* ---------------------------------------------------------------------- */
/* findpivot (lu2tlib.c:42-52): cblas_idamax over rows `from`..n-1 of column
 * `col`; returns the first row of maximal |a|. */
static int orc_idamax(const orc_t *o, int col, int from)
{
    int p = from;
    double amax = fabs(A_(from, col));
    for (int r = from + 1; r < o->n; r++) {
        double v = fabs(A_(r, col));
        if (v > amax) { amax = v; p = r; }
    }
    return p;
}

static void orc_swap_cols(orc_t *o, int r1, int r2, int c0, int c1)
{
    if (r1 == r2) return;
    for (int c = c0; c < c1; c++) {
        double t = A_(r1, c);
        A_(r1, c) = A_(r2, c);
        A_(r2, c) = t;
    }
}

static void orc_scale_cols(orc_t *o, int r, double s, int c0, int c1)
{
    for (int c = c0; c < c1; c++) A_(r, c) *= s;
}

/* column_decomposition, the slab leaf (lu2tlib.c:1041-1066).  Columns
 * c0..c0+m-1, rows c0..n-1.  In REF mode every column searches column c0,
 * the leaf's first column (lu2tlib.c:1052 -> findpivot scans a[0]). */
static void orc_leaf(orc_t *o, int c0, int m)
{
    for (int ip = 0; ip < m; ip++) {
        int ii = c0 + ip;
        int scol = (o->mode == ORC_PIVOT_REF) ? c0 : ii;
        int p = orc_idamax(o, scol, ii);
        o->ipiv[ii] = p;
        orc_swap_cols(o, p, ii, c0, c0 + m);
        double ainv = 1.0 / A_(ii, ii);
        orc_scale_cols(o, ii, ainv, c0, ii);
        orc_scale_cols(o, ii, ainv, ii + 1, c0 + m);
        /* vvmulandsub (lu2tlib.c:159-180): column by column */
        for (int k = ii + 1; k < c0 + m; k++) {
            double s = A_(ii, k);
            for (int r = ii + 1; r < o->n; r++) A_(r, k) -= A_(r, ii) * s;
        }
    }
}

/* process_right_part of the slab (lu2tlib.c:1068-1093): block rows
 * i..i+m-1, right columns i+m..iend-1. */
static void orc_slab_right(orc_t *o, int i, int m, int iend)
{
    for (int ii = i; ii < i + m; ii++) orc_swap_cols(o, o->ipiv[ii], ii, i + m, iend);
    for (int ii = i; ii < i + m; ii++) orc_scale_cols(o, ii, 1.0 / A_(ii, ii), i + m, iend);
    /* in-block forward substitution, vvmulandsub(n,a,ii-i,ii,m,iend-i,ii+1,i+m) */
    for (int ii = i; ii < i + m; ii++)
        for (int k = i + m; k < iend; k++) {
            double s = A_(ii, k);
            for (int r = ii + 1; r < i + m; r++) A_(r, k) -= A_(r, ii) * s;
        }
    /* mmmulandsub (lu2tlib.c:1003-1039): rank-m update of rows i+m..n-1 */
    for (int r = i + m; r < o->n; r++)
        for (int k = i + m; k < iend; k++) {
            double c = A_(r, k);
            for (int l = i; l < i + m; l++) c -= A_(r, l) * A_(l, k);
            A_(r, k) = c;
        }
}

/* column_decomposition_recursive of the slab (lu2tlib.c:1095-1128). */
static void orc_slab_recursive(orc_t *o, int i, int m)
{
    if (m <= 2) {
        orc_leaf(o, i, m);
        return;
    }
    int h = m / 2;
    orc_slab_recursive(o, i, h);
    orc_slab_right(o, i, h, i + m);
    orc_slab_recursive(o, i + h, h);
    for (int ii = i + h; ii < i + m; ii++) orc_swap_cols(o, o->ipiv[ii], ii, i, i + h);
    for (int ii = i + h; ii < i + m; ii++) orc_scale_cols(o, ii, 1.0 / A_(ii, ii), i, i + h);
}

/* ---------------------------------------------------------------------- */
/* solve_triangle_for_unit_mat_internal (lu2.c:370-381) */
static void orc_uli_internal(const double *t, long ldt, double *b, long ldb, int m)
{
    for (int ii = 0; ii < m; ii++)
        for (int j = ii + 1; j < m; j++) {
            double tj = t[(size_t)j * ldt + ii];
            for (int k = 0; k < m; k++) b[(size_t)j * ldb + k] -= tj * b[(size_t)ii * ldb + k];
        }
}

/* C = beta*C + alpha*A*B on small row-major blocks (the mydgemm calls inside
 * the triangle inversion, lu2.c:441-457). */
static void orc_small_gemm(int m, int n, int k, double alpha, const double *a, long lda,
                           const double *b, long ldb, double beta, double *c, long ldc)
{
    for (int r = 0; r < m; r++)
        for (int j = 0; j < n; j++) {
            double s = 0.0;
            for (int l = 0; l < k; l++) s += a[(size_t)r * lda + l] * b[(size_t)l * ldb + j];
            c[(size_t)r * ldc + j] = beta * c[(size_t)r * ldc + j] + alpha * s;
        }
}

/* solve_triangle_for_unit_mat_recursive (lu2.c:430-465): b (identity on
 * entry) becomes the inverse of the unit lower triangle whose strict lower
 * part is t. */
static void orc_uli_recursive(const double *t, long ldt, double *b, long ldb, int m)
{
    if (m < 16) {
        orc_uli_internal(t, ldt, b, ldb, m);
        return;
    }
    int h = m / 2;
    orc_uli_recursive(t, ldt, b, ldb, h);
    orc_small_gemm(h, h, h, -1.0, t + (size_t)h * ldt, ldt, b, ldb, 1.0, b + (size_t)h * ldb, ldb);
    double *w = calloc((size_t)h * h, sizeof(double));
    double *w2 = malloc((size_t)h * h * sizeof(double));
    for (int j = 0; j < h; j++) w[(size_t)j * h + j] = 1.0;
    orc_uli_recursive(t + (size_t)h * ldt + h, ldt, w, h, h);
    for (int r = 0; r < h; r++)
        for (int j = 0; j < h; j++) w2[(size_t)r * h + j] = b[(size_t)(r + h) * ldb + j];
    orc_small_gemm(h, h, h, 1.0, w, h, w2, h, 0.0, b + (size_t)h * ldb, ldb);
    for (int j = 0; j < h; j++)
        for (int k = 0; k <= j; k++) b[(size_t)(h + j) * ldb + h + k] = w[(size_t)j * h + k];
    free(w);
    free(w2);
}

/* solve_triangle (lu2.c:485-521): U12 = inv(T11) * A12 with T11 the unit
 * lower triangle of the block rows i..i+m-1. */
static void orc_solve_triangle(orc_t *o, int i, int m, int iend)
{
    int w = iend - i - m;
    if (w <= 0) return;
    double *b = calloc((size_t)m * m, sizeof(double));
    double *x = malloc((size_t)m * w * sizeof(double));
    for (int j = 0; j < m; j++) b[(size_t)j * m + j] = 1.0;
    orc_uli_recursive(&A_(i, i), o->lda, b, m, m);
    for (int r = 0; r < m; r++)
        for (int k = 0; k < w; k++) x[(size_t)r * w + k] = A_(i + r, i + m + k);
    for (int r = 0; r < m; r++) {
        double *dst = &A_(i + r, i + m);
        for (int k = 0; k < w; k++) dst[k] = 0.0;
        for (int l = 0; l < m; l++) {
            double blr = b[(size_t)r * m + l];
            const double *xl = x + (size_t)l * w;
            for (int k = 0; k < w; k++) dst[k] += blr * xl[k];
        }
    }
    free(b);
    free(x);
}

/* process_right_part (lu2.c:524-581): swap + 1/pivot scale of the block
 * rows over columns i+m..iend-1, solve_triangle, then mmmulandsub. */
static void orc_rm_right(orc_t *o, int i, int m, int iend)
{
    for (int ii = i; ii < i + m; ii++) {
        orc_swap_cols(o, o->ipiv[ii], ii, i + m, iend);
        orc_scale_cols(o, ii, 1.0 / A_(ii, ii), i + m, iend);
    }
    orc_solve_triangle(o, i, m, iend);
    /* mmmulandsub (lu2.c:312-343) -> mydgemm(n-i-m, iend-i-m, m, -1, L21, U12, 1, A22) */
    int r0 = i + m, n = o->n;
#pragma omp parallel for schedule(static)
    for (int r = r0; r < n; r++) {
        double *crow = &A_(r, i + m);
        for (int l = i; l < i + m; l++) {
            double arl = A_(r, l);
            const double *urow = &A_(l, i + m);
            for (int k = 0; k < iend - i - m; k++) crow[k] -= arl * urow[k];
        }
    }
}

/* column_decomposition_recursive, row-major (lu2.c:1088-1120). */
static void orc_rm_recursive(orc_t *o, int i, int m)
{
    if (m <= 16) {
        orc_slab_recursive(o, i, m);
        return;
    }
    int h = m / 2;
    orc_rm_recursive(o, i, h);
    orc_rm_right(o, i, h, i + m);
    orc_rm_recursive(o, i + h, h);
    for (int ii = i + h; ii < i + m; ii++) orc_swap_cols(o, o->ipiv[ii], ii, i, i + h);
    for (int ii = i + h; ii < i + m; ii++) orc_scale_cols(o, ii, 1.0 / A_(ii, ii), i, i + h);
}

/* ---------------------------------------------------------------------- */
/* lumcolumn (lu2.c:1122-1144) over an augmented row-major matrix with nrhs
 * right-hand sides in columns n..n+nrhs-1, then backward_sub (lu2.c:110-116)
 * into x (n x nrhs, row-major).  Returns 0, or -1 on an argument error. */
int orc_lumcolumn(int n, int nrhs, double *a, long lda, int nb, int mode, int *ipiv, double *x)
{
    if (n <= 0 || nb <= 0 || nrhs < 1 || lda < n + nrhs) return -1;
    if ((nb & (nb - 1)) != 0 || n % nb != 0) return -1;
    orc_t o_ = {n, n + nrhs, lda, a, ipiv, mode};
    orc_t *o = &o_;
    for (int i = 0; i < n; i += nb) {
        orc_rm_recursive(o, i, nb);
        orc_rm_right(o, i, nb, n + nrhs);
    }
    if (x) {
        for (int r = 0; r < nrhs; r++) {
            for (int i = 0; i < n; i++) x[(size_t)i * nrhs + r] = A_(i, n + r);
            for (int j = n - 2; j >= 0; j--) {
                double s = x[(size_t)j * nrhs + r];
                for (int k = j + 1; k < n; k++) s -= x[(size_t)k * nrhs + r] * A_(j, k);
                x[(size_t)j * nrhs + r] = s;
            }
        }
    }
    return 0;
}

/* ---------------------------------------------------------------------- */
/* Residual checks (untimed in the reference: lu2.c:45-60 showresult and
 * lu2_mpi.c:2170-2230 HPLerrorprint).  Given the ORIGINAL A (n x n, lda)
 * with b in column n, and x:
 *   out[0] = ||Ax-b||_inf   out[1] = ||A||_inf   out[2] = ||x||_inf
 *   out[3] = ||b||_inf      out[4] = ||A||_1     out[5] = ||x||_1
 *   out[6] = ||Ax-b||_inf / (eps (||A||_inf ||x||_inf + ||b||_inf) n), eps = 2^-53
 *   out[7..9] = the reference's three HPL residuals with eps = 2e-16
 *               (lu2_mpi.c:2170-2230): e/(eps |A|_1 n), e/(eps |A|_1 |x|_1),
 *               e/(eps |A|_inf |x|_inf n). */
void orc_residual(int n, const double *a, long lda, const double *x, double *out)
{
    double rinf = 0, ainf = 0, xinf = 0, binf = 0, x1 = 0;
    double *colsum = calloc((size_t)n, sizeof(double));
#pragma omp parallel for reduction(max : rinf, ainf) schedule(static)
    for (int i = 0; i < n; i++) {
        const double *ai = a + (size_t)i * lda;
        double s = 0, r = 0;
        for (int j = 0; j < n; j++) {
            s += fabs(ai[j]);
            r += ai[j] * x[j];
        }
        r -= ai[n];
        if (s > ainf) ainf = s;
        if (fabs(r) > rinf) rinf = fabs(r);
    }
    for (int i = 0; i < n; i++) {
        const double *ai = a + (size_t)i * lda;
        if (fabs(ai[n]) > binf) binf = fabs(ai[n]);
        if (fabs(x[i]) > xinf) xinf = fabs(x[i]);
        x1 += fabs(x[i]);
        for (int j = 0; j < n; j++) colsum[j] += fabs(ai[j]);
    }
    double a1 = 0;
    for (int j = 0; j < n; j++) if (colsum[j] > a1) a1 = colsum[j];
    free(colsum);
    const double eps53 = DBL_EPSILON / 2, eps_ref = 2e-16;
    out[0] = rinf; out[1] = ainf; out[2] = xinf; out[3] = binf; out[4] = a1; out[5] = x1;
    out[6] = rinf / (eps53 * (ainf * xinf + binf) * n);
    out[7] = rinf / (eps_ref * a1 * n);
    out[8] = rinf / (eps_ref * a1 * x1);
    out[9] = rinf / (eps_ref * ainf * xinf * n);
}
