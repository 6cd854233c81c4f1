/*
 * Timed CPU restatement of the reference's host sweep -- TEST / BENCH INFRASTRUCTURE ONLY
 * (the reference arm of bench.py and the CPU-baseline leg; never the product path).
 *
 * Mirrors srcPerformanceTest/main.cpp:359-404 ("Multiple Dense Matrices" mode): a parallel
 * loop over frequencies (OpenMP in the reference, POSIX threads here), each thread owning one A buffer, per frequency the
 * assembly of src/analysis/KrylovROMSubstructure.cpp:1411-1420 followed by
 * LAPACKE_zgetrf + LAPACKE_zgetrs (main.cpp:393-395).  The reference links Intel MKL, which
 * is absent here; LAPACKE comes from an OpenBLAS shared object opened at run time
 * (1 BLAS thread per OpenMP thread, like the reference's parallel dense mode), and when no
 * OpenBLAS is given the oracle's own unblocked zgetrf/zgetrs restatement is used.
 */
#include <dlfcn.h>
#include <pthread.h>
#include <unistd.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

void oracle_assemble(int n, const double *K, const double *M, const double *D,
                     double eta, double omega, double *A);
int oracle_zgetrf(int n, double *A, int lda, int *ipiv);
void oracle_zgetrs(int n, int nrhs, const double *A, int lda, const int *ipiv, double *B, int ldb);

typedef int (*lapacke_zgetrf_t)(int, int, int, void *, int, int *);
typedef int (*lapacke_zgetrs_t)(int, char, int, int, const void *, int, const int *, void *, int);
typedef void (*set_threads_t)(int);

static lapacke_zgetrf_t p_zgetrf = 0;
static lapacke_zgetrs_t p_zgetrs = 0;

/* Returns 1 when the OpenBLAS LAPACKE entry points were found, 0 otherwise. */
int cpu_baseline_load_lapacke(const char *path, const char *prefix) {
    void *h = dlopen(path, RTLD_NOW | RTLD_LOCAL);
    if (!h) return 0;
    char name[128];
    strcpy(name, prefix); strcat(name, "LAPACKE_zgetrf");
    p_zgetrf = (lapacke_zgetrf_t)dlsym(h, name);
    strcpy(name, prefix); strcat(name, "LAPACKE_zgetrs");
    p_zgetrs = (lapacke_zgetrs_t)dlsym(h, name);
    strcpy(name, prefix); strcat(name, "openblas_set_num_threads");
    set_threads_t st = (set_threads_t)dlsym(h, name);
    if (st) st(1);
    if (!p_zgetrf || !p_zgetrs) { p_zgetrf = 0; p_zgetrs = 0; return 0; }
    return 1;
}

int cpu_baseline_using_lapacke(void) { return p_zgetrf != 0; }

typedef struct {
    int n, nrhs, ldb, f1;
    const double *K, *M, *D, *rhs, *omega;
    double eta;
    int f0;
    double *X;
    volatile int next; /* shared frequency counter (dynamic schedule, chunk 1) */
    pthread_mutex_t lock;
} sweep_job;

static void *sweep_worker(void *arg) {
    sweep_job *j = (sweep_job *)arg;
    int n = j->n;
    double *A = (double *)malloc(sizeof(double) * 2 * (size_t)n * n);
    int *ipiv = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    for (;;) {
        pthread_mutex_lock(&j->lock);
        int f = j->next++;
        pthread_mutex_unlock(&j->lock);
        if (f >= j->f1) break;
        oracle_assemble(n, j->K, j->M, j->D, j->eta, j->omega[f], A);
        double *x = j->X + (int64_t)(f - j->f0) * 2 * n * j->nrhs;
        for (int c = 0; c < j->nrhs; ++c)
            memcpy(x + (int64_t)c * 2 * n, j->rhs + (int64_t)c * 2 * j->ldb, sizeof(double) * 2 * n);
        if (p_zgetrf) {
            p_zgetrf(102 /* LAPACK_COL_MAJOR */, n, n, A, n, ipiv);
            p_zgetrs(102, 'N', n, j->nrhs, A, n, ipiv, x, n);
        } else {
            oracle_zgetrf(n, A, n, ipiv);
            oracle_zgetrs(n, j->nrhs, A, n, ipiv, x, n);
        }
    }
    free(A);
    free(ipiv);
    return 0;
}

int cpu_baseline_default_threads(void) {
    long c = sysconf(_SC_NPROCESSORS_ONLN);
    return c > 0 ? (int)c : 1;
}

/* Sweep frequencies [f0, f1) of one ROM with `threads` worker threads (<= 0: all cores),
 * each pulling the next frequency from a shared counter like an OpenMP dynamic loop.
 * X: (f1-f0) blocks of n x nrhs.  Returns the number of frequencies solved. */
int cpu_baseline_sweep(int n, int nrhs, const double *K, const double *M, const double *D,
                       double eta, const double *rhs, int ldb, const double *omega,
                       int f0, int f1, double *X, int threads) {
    if (threads <= 0) threads = cpu_baseline_default_threads();
    sweep_job job = {n, nrhs, ldb, f1, K, M, D, rhs, omega, eta, f0, X, f0,
                     PTHREAD_MUTEX_INITIALIZER};
    pthread_t *tid = (pthread_t *)malloc(sizeof(pthread_t) * (size_t)threads);
    for (int t = 0; t < threads; ++t) pthread_create(&tid[t], 0, sweep_worker, &job);
    for (int t = 0; t < threads; ++t) pthread_join(tid[t], 0);
    free(tid);
    return f1 - f0;
}
