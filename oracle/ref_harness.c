/*
 * ref_harness.c -- drives the UNMODIFIED reference sources (compiled from
 * telmin/lu2 into oracle/_ref/ by oracle/build_oracle.py) so that tests can pin the
 * oracle restatement against the reference itself, and bench.py can time the
 * reference's own CPU path.
 *
 * TEST AND CPU-BASELINE INFRASTRUCTURE ONLY: never linked into the product.
 *
 * Entry points used from the reference (file:line in telmin/lu2):
 *   randomsetmat                     lu2.c:70-85
 *   column_decomposition_recursive   lu2.c:1088-1120
 *   process_right_part               lu2.c:524-581
 *   backward_sub                     lu2.c:110-116
 *   lumcolumn                        lu2.c:1122-1144
 * The reference keeps only the current panel's pivots (pv is overwritten per
 * panel); ref_lu2_factor_solve drives the same per-panel calls as lumcolumn
 * and copies pv out after each panel to record the whole pivot sequence.
 *
 * The reference uses stack VLAs sized by nb (lu2.c:493, lu2.c:448-449), so
 * every call runs on a worker thread with a 512 MiB stack.
 */
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

/* The reference's prototypes take C99 VLA parameters, which decay to plain
 * pointers; these declarations are ABI-identical. */
void randomsetmat(int n, int seed, double *a);
void column_decomposition_recursive(int n, double *a, int m, double *awork, int pv[], int i);
void process_right_part(int n, double *a, int m, double *awork, int pv[], int i, int iend);
void backward_sub(int n, double *a, double b[]);
void lumcolumn(int n, double *a, double b[], int m, double *awork, int pv[], int recursive);

void openblas_set_num_threads(int);
void omp_set_num_threads(int);

typedef struct {
    int n, nb, seed, which;
    const double *diag; /* optional: a[i][i] := diag[i] after randomsetmat */
    double *x;
    int *piv;
    double seconds;
    int rc;
} job_t;

static double now_s(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

/* thread settings, applied by the worker thread itself: OpenMP's thread
 * count is a per-thread setting that a new pthread does not inherit */
static int g_blas_threads = 0, g_omp_threads = 0;

static void *run_job(void *arg)
{
    job_t *j = (job_t *)arg;
    if (g_blas_threads > 0) openblas_set_num_threads(g_blas_threads);
    if (g_omp_threads > 0) omp_set_num_threads(g_omp_threads);
    int n = j->n, nb = j->nb;
    size_t rdim = (size_t)n + 16;
    double *a = malloc(sizeof(double) * (size_t)n * rdim);
    double *awork = malloc(sizeof(double) * (size_t)nb * (size_t)n);
    int *pv = malloc(sizeof(int) * (size_t)n);
    double *b = malloc(sizeof(double) * (size_t)n);
    if (!a || !awork || !pv || !b) {
        j->rc = -2;
        goto out;
    }
    memset(a, 0, sizeof(double) * (size_t)n * rdim);
    randomsetmat(n, j->seed, a);
    if (j->diag)
        for (int i = 0; i < n; i++) a[(size_t)i * rdim + i] = j->diag[i];
    double t0 = now_s();
    if (j->which == 0) {
        for (int i = 0; i < n; i += nb) {
            column_decomposition_recursive(n, a, nb, awork, pv, i);
            process_right_part(n, a, nb, awork, pv, i, n + 1);
            if (j->piv)
                for (int k = 0; k < nb; k++) j->piv[i + k] = pv[k];
        }
        backward_sub(n, a, b);
    } else {
        lumcolumn(n, a, b, nb, awork, pv, 1);
    }
    j->seconds = now_s() - t0;
    if (j->x) memcpy(j->x, b, sizeof(double) * (size_t)n);
    j->rc = 0;
out:
    free(a);
    free(awork);
    free(pv);
    free(b);
    return NULL;
}

static int run_on_big_stack(job_t *j)
{
    pthread_attr_t attr;
    pthread_t th;
    pthread_attr_init(&attr);
    pthread_attr_setstacksize(&attr, (size_t)512 << 20);
    if (pthread_create(&th, &attr, run_job, j) != 0) return -3;
    pthread_join(th, NULL);
    pthread_attr_destroy(&attr);
    return j->rc;
}

/* Threads for OpenBLAS and for the reference's own OpenMP regions (0: leave
 * the library default, i.e. all cores unless OMP_NUM_THREADS /
 * OPENBLAS_NUM_THREADS say otherwise). */
void ref_set_threads(int blas_threads, int omp_threads)
{
    g_blas_threads = blas_threads;
    g_omp_threads = omp_threads;
    if (blas_threads > 0) openblas_set_num_threads(blas_threads);
}

/* Per-panel drive of the reference (records the full pivot sequence). */
int ref_lu2_factor_solve(int n, int nb, int seed, double *x_out, int *piv_out, double *seconds)
{
    if (n <= 0 || nb <= 0 || n % nb) return -1;
    job_t j = {n, nb, seed, 0, NULL, x_out, piv_out, 0.0, -1};
    int rc = run_on_big_stack(&j);
    if (seconds) *seconds = j.seconds;
    return rc;
}

/* The reference's own lumcolumn, timed like its main (lu2.c:1287-1296). */
int ref_lu2_lumcolumn(int n, int nb, int seed, double *x_out, double *seconds)
{
    if (n <= 0 || nb <= 0 || n % nb) return -1;
    job_t j = {n, nb, seed, 1, NULL, x_out, NULL, 0.0, -1};
    int rc = run_on_big_stack(&j);
    if (seconds) *seconds = j.seconds;
    return rc;
}

/* As ref_lu2_factor_solve, on randomsetmat's matrix with its diagonal replaced
 * by diag[0..n) (the diagonally dominant, well-conditioned parity cases). */
int ref_lu2_factor_solve_diag(int n, int nb, int seed, const double *diag, double *x_out, int *piv_out,
                              double *seconds)
{
    if (n <= 0 || nb <= 0 || n % nb || !diag) return -1;
    job_t j = {n, nb, seed, 0, diag, x_out, piv_out, 0.0, -1};
    int rc = run_on_big_stack(&j);
    if (seconds) *seconds = j.seconds;
    return rc;
}
