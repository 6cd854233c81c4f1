/*
 * CPU oracle for the reduced-order frequency sweep -- TEST INFRASTRUCTURE ONLY.
 *
 * Only tests/, the smoke check and bench.py's CPU-baseline leg may load this library, and
 * only as the checker (or as the timed CPU restatement of the reference); the product path
 * never calls it.
 *
 * It restates, in plain C99 with IEEE double arithmetic and no FMA contraction
 * (-ffp-contract=off), the algorithm the reference runs for this path:
 *
 *   assembly   A(w) = K_r + (-w^2) M_r + (i w) D_r, three zaxpy passes in that order
 *              (src/analysis/KrylovROMSubstructure.cpp:1411-1420; K_r already carries the
 *              hysteretic factor, :330-333).
 *   factor     LAPACKE_zgetrf, column-major, partial pivoting
 *              (src/analysis/KrylovROMSubstructure.cpp:1428; srcPerformanceTest/main.cpp:393).
 *              The LAPACK routine lives in Intel MKL, which the reference does not vendor and
 *              pins to no version (cmake/modules/FindMKL.cmake).  Restated here from the
 *              published LAPACK zgetf2/zgetrf2 algorithm: the pivot is IZAMAX of the column
 *              (largest |re|+|im|, first index on ties), the whole row is swapped, the column
 *              below the pivot is scaled by 1/pivot, and the trailing matrix receives the
 *              rank-1 update column after column.  A zero pivot sets info = j+1 (1-based)
 *              and skips the scaling, as LAPACK does.
 *   solve      LAPACKE_zgetrs 'N' (KrylovROMSubstructure.cpp:1430; srcPerformanceTest/main.cpp:395):
 *              row interchanges applied to B in order, unit-lower forward substitution,
 *              then upper back substitution (ZTRSM column-oriented order).
 *   adjoint    the conjugate-transposed solve A^H lambda = g through the same factors
 *              (LAPACK zgetrs 'C'; the reference has no adjoint, this is the restated
 *              maths for the backward call).
 *
 * Rounding convention shared bit-for-bit with the CUDA FP64 kernels:
 *   - complex update c - a*b uses two fused multiply-adds per component (csubmul),
 *   - reciprocal / division use Smith's algorithm (crecip / cdiv),
 *   - every element of A receives its updates in increasing pivot-column order, which is
 *     what any right-looking blocking does, so a blocked GPU factorisation reproduces these
 *     factors exactly.
 * The "true" solution used for accuracy gates (x_ref) comes from oracle_refine_ld, which
 * refines the FP64 LU solution with residuals accumulated in x87 long double.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct { double re, im; } cplx;

static inline cplx csubmul(cplx c, cplx a, cplx b) {
    /* c - a*b with the FMA order used by the GPU kernels */
    cplx o;
    o.re = fma(-a.re, b.re, fma(a.im, b.im, c.re));
    o.im = fma(-a.re, b.im, fma(-a.im, b.re, c.im));
    return o;
}

static inline cplx cmul(cplx a, cplx b) {
    cplx o;
    double t0 = a.re * b.re, t1 = a.im * b.im, t2 = a.re * b.im, t3 = a.im * b.re;
    o.re = t0 - t1;
    o.im = t2 + t3;
    return o;
}

static inline cplx crecip(cplx z) {
    /* Smith's algorithm for 1/z */
    cplx o;
    if (fabs(z.re) >= fabs(z.im)) {
        double t = z.im / z.re;
        double d = z.re + z.im * t;
        o.re = 1.0 / d;
        o.im = -t / d;
    } else {
        double t = z.re / z.im;
        double d = z.re * t + z.im;
        o.re = t / d;
        o.im = -1.0 / d;
    }
    return o;
}

static inline cplx cdiv(cplx a, cplx b) {
    /* Smith's algorithm for a/b */
    cplx o;
    if (fabs(b.re) >= fabs(b.im)) {
        double t = b.im / b.re;
        double d = b.re + b.im * t;
        o.re = (a.re + a.im * t) / d;
        o.im = (a.im - a.re * t) / d;
    } else {
        double t = b.re / b.im;
        double d = b.re * t + b.im;
        o.re = (a.re * t + a.im) / d;
        o.im = (a.im * t - a.re) / d;
    }
    return o;
}

static inline double cabs1(cplx z) { return fabs(z.re) + fabs(z.im); }

/* A(w) = (1 + i eta) K + (-w^2) M + (i w) D ; D may be NULL.  K, M, D, A: n x n, ld = n. */
void oracle_assemble(int n, const double *K, const double *M, const double *D,
                     double eta, double omega, double *A) {
    const cplx *k = (const cplx *)K, *m = (const cplx *)M, *d = (const cplx *)D;
    cplx *a = (cplx *)A;
    double s = -(omega * omega);
    int64_t nn = (int64_t)n * n;
    for (int64_t e = 0; e < nn; ++e) {
        cplx kk = k[e];
        if (eta != 0.0) {
            double t1 = eta * kk.im, t2 = eta * kk.re;
            cplx kh;
            kh.re = kk.re - t1;
            kh.im = kk.im + t2;
            kk = kh;
        }
        cplx v = kk;  /* no mass term when M is NULL (explicit matrices, damped statics) */
        if (m) {
            double mr = s * m[e].re, mi = s * m[e].im;
            v.re = kk.re + mr;
            v.im = kk.im + mi;
        }
        if (d) {
            double dr = omega * d[e].im, di = omega * d[e].re;
            v.re = v.re - dr;
            v.im = v.im + di;
        }
        a[e] = v;
    }
}

/* zgetrf restatement: unblocked right-looking, partial pivoting.  ipiv is 1-based like
 * LAPACK.  Returns info (0 or first zero pivot, 1-based). */
int oracle_zgetrf(int n, double *Ad, int lda, int *ipiv) {
    cplx *A = (cplx *)Ad;
    int info = 0;
    for (int j = 0; j < n; ++j) {
        int p = j;
        double best = cabs1(A[j + (int64_t)j * lda]);
        for (int i = j + 1; i < n; ++i) {
            double v = cabs1(A[i + (int64_t)j * lda]);
            if (v > best) { best = v; p = i; }
        }
        ipiv[j] = p + 1;
        cplx piv = A[p + (int64_t)j * lda];
        if (piv.re != 0.0 || piv.im != 0.0) {
            if (p != j) {
                for (int c = 0; c < n; ++c) {
                    cplx t = A[j + (int64_t)c * lda];
                    A[j + (int64_t)c * lda] = A[p + (int64_t)c * lda];
                    A[p + (int64_t)c * lda] = t;
                }
            }
            cplx inv = crecip(A[j + (int64_t)j * lda]);
            for (int i = j + 1; i < n; ++i)
                A[i + (int64_t)j * lda] = cmul(A[i + (int64_t)j * lda], inv);
        } else if (info == 0) {
            info = j + 1;
        }
        for (int c = j + 1; c < n; ++c) {
            cplx u = A[j + (int64_t)c * lda];
            for (int i = j + 1; i < n; ++i)
                A[i + (int64_t)c * lda] = csubmul(A[i + (int64_t)c * lda], A[i + (int64_t)j * lda], u);
        }
    }
    return info;
}

/* zgetrs 'N': B (n x nrhs, ldb) <- A^-1 B using factors from oracle_zgetrf. */
void oracle_zgetrs(int n, int nrhs, const double *Ad, int lda, const int *ipiv,
                   double *Bd, int ldb) {
    const cplx *A = (const cplx *)Ad;
    cplx *B = (cplx *)Bd;
    for (int c = 0; c < nrhs; ++c) {
        cplx *b = B + (int64_t)c * ldb;
        for (int j = 0; j < n; ++j) {
            int p = ipiv[j] - 1;
            if (p != j) { cplx t = b[j]; b[j] = b[p]; b[p] = t; }
        }
        for (int j = 0; j < n; ++j) {
            cplx bj = b[j];
            for (int i = j + 1; i < n; ++i)
                b[i] = csubmul(b[i], A[i + (int64_t)j * lda], bj);
        }
        for (int j = n - 1; j >= 0; --j) {
            b[j] = cdiv(b[j], A[j + (int64_t)j * lda]);
            cplx bj = b[j];
            for (int i = 0; i < j; ++i)
                b[i] = csubmul(b[i], A[i + (int64_t)j * lda], bj);
        }
    }
}

/* zgetrs 'C': B <- A^-H B (A = P L U  =>  A^H = U^H L^H P^T).
 * Solve U^H y = b (forward, conj(U)), L^H z = y (backward, unit, conj(L)), then undo the
 * interchanges in reverse order. */
void oracle_zgetrs_conj(int n, int nrhs, const double *Ad, int lda, const int *ipiv,
                        double *Bd, int ldb) {
    const cplx *A = (const cplx *)Ad;
    cplx *B = (cplx *)Bd;
    for (int c = 0; c < nrhs; ++c) {
        cplx *b = B + (int64_t)c * ldb;
        for (int j = 0; j < n; ++j) {
            /* y_j = (b_j - sum_{i<j} conj(U_ij) y_i) / conj(U_jj) */
            cplx acc = b[j];
            for (int i = 0; i < j; ++i) {
                cplx u = A[i + (int64_t)j * lda];
                u.im = -u.im;
                acc = csubmul(acc, u, b[i]);
            }
            cplx d = A[j + (int64_t)j * lda];
            d.im = -d.im;
            b[j] = cdiv(acc, d);
        }
        for (int j = n - 1; j >= 0; --j) {
            cplx acc = b[j];
            for (int i = j + 1; i < n; ++i) {
                cplx l = A[i + (int64_t)j * lda];
                l.im = -l.im;
                acc = csubmul(acc, l, b[i]);
            }
            b[j] = acc;
        }
        for (int j = n - 1; j >= 0; --j) {
            int p = ipiv[j] - 1;
            if (p != j) { cplx t = b[j]; b[j] = b[p]; b[p] = t; }
        }
    }
}

/* Full reference sequence for one ROM: per frequency assemble, zgetrf, zgetrs.
 * X: F blocks of n x nrhs (ld n).  info: F ints (may be NULL).
 * Ws: caller scratch of n*n complex + n ints (pass NULL to allocate). */
void oracle_sweep(int n, int nrhs, const double *K, const double *M, const double *D,
                  double eta, const double *rhs, int ldb, int F, const double *omega,
                  double *X, int *info) {
    cplx *A = (cplx *)malloc(sizeof(cplx) * (size_t)n * n);
    int *ipiv = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    for (int f = 0; f < F; ++f) {
        oracle_assemble(n, K, M, D, eta, omega[f], (double *)A);
        int inf = oracle_zgetrf(n, (double *)A, n, ipiv);
        cplx *x = (cplx *)X + (int64_t)f * n * nrhs;
        for (int c = 0; c < nrhs; ++c)
            memcpy(x + (int64_t)c * n, (const cplx *)rhs + (int64_t)c * ldb, sizeof(cplx) * n);
        oracle_zgetrs(n, nrhs, (double *)A, n, ipiv, (double *)x, n);
        if (info) info[f] = inf;
    }
    free(A);
    free(ipiv);
}

/* ---------------------------------------------------------------------------------------
 * Back-projection y = C_R x per frequency: z_freq = C_R * z_krylov_freq, cblas_zgemm in
 * backTransformKMOR (src/analysis/KrylovROMSubstructure.cpp:1446-1449); with B_R as the
 * right-hand sides the same product gives H_R = C_R A^-1 B_R (:1433-1441).  MKL does not
 * specify zgemm's summation order; the restatement fixes it: y_ic is the sum over
 * j = 0 .. n-1 in increasing order of C_ij x_jc, each term added with two FMAs per component
 * (the order the GPU kernel uses).  C: n_out x n (ld ldc); X: F blocks of n x r (ld n);
 * Y: F blocks of n_out x r (ld n_out).
 * --------------------------------------------------------------------------------------- */
void oracle_backproject(int n, int r, int F, int n_out, int ldc, const double *Cd, const double *Xd,
                        double *Yd) {
    const cplx *C = (const cplx *)Cd, *X = (const cplx *)Xd;
    cplx *Y = (cplx *)Yd;
    for (int f = 0; f < F; ++f)
        for (int c = 0; c < r; ++c)
            for (int i = 0; i < n_out; ++i) {
                cplx acc = {0.0, 0.0};
                const cplx *x = X + ((int64_t)f * r + c) * n;
                for (int j = 0; j < n; ++j) {
                    const cplx a = C[i + (int64_t)j * ldc], b = x[j];
                    cplx o;
                    o.re = fma(a.re, b.re, fma(-a.im, b.im, acc.re));
                    o.im = fma(a.re, b.im, fma(a.im, b.re, acc.im));
                    acc = o;
                }
                Y[((int64_t)f * r + c) * n_out + i] = acc;
            }
}

/* x_ref for one frequency: FP64 LU solution refined with long-double residuals.
 * A: assembled n x n (ld n), B: n x nrhs (ld ldb), X out n x nrhs (ld n).
 * Returns the LAPACK info of the factorisation. */
int oracle_refine_ld(int n, int nrhs, const double *Ad, const double *Bd, int ldb,
                     int iters, double *Xd) {
    const cplx *A = (const cplx *)Ad;
    const cplx *B = (const cplx *)Bd;
    cplx *X = (cplx *)Xd;
    cplx *LU = (cplx *)malloc(sizeof(cplx) * (size_t)n * n);
    int *ipiv = (int *)malloc(sizeof(int) * (size_t)(n > 0 ? n : 1));
    cplx *r = (cplx *)malloc(sizeof(cplx) * (size_t)(n > 0 ? n : 1));
    memcpy(LU, A, sizeof(cplx) * (size_t)n * n);
    int info = oracle_zgetrf(n, (double *)LU, n, ipiv);
    for (int c = 0; c < nrhs; ++c) {
        cplx *x = X + (int64_t)c * n;
        const cplx *b = B + (int64_t)c * ldb;
        memcpy(x, b, sizeof(cplx) * n);
        oracle_zgetrs(n, 1, (double *)LU, n, ipiv, (double *)x, n);
        for (int it = 0; it < iters; ++it) {
            for (int i = 0; i < n; ++i) {
                long double sr = (long double)b[i].re, si = (long double)b[i].im;
                for (int j = 0; j < n; ++j) {
                    cplx a = A[i + (int64_t)j * n];
                    sr -= (long double)a.re * x[j].re - (long double)a.im * x[j].im;
                    si -= (long double)a.re * x[j].im + (long double)a.im * x[j].re;
                }
                r[i].re = (double)sr;
                r[i].im = (double)si;
            }
            oracle_zgetrs(n, 1, (double *)LU, n, ipiv, (double *)r, n);
            for (int i = 0; i < n; ++i) {
                x[i].re += r[i].re;
                x[i].im += r[i].im;
            }
        }
    }
    free(LU);
    free(ipiv);
    free(r);
    return info;
}

/* ---------------------------------------------------------------------------------------
 * Projection (generateROM, src/analysis/KrylovROMSubstructure.cpp:709-765).
 *   Y = S * V     mkl_sparse_z_mm with a symmetric-upper descriptor (src/tools/MathLibrary.cpp:491-532)
 *   R = V^T * Y   cblas_zgemm ConjTrans, column-major (src/tools/MathLibrary.cpp:177-234)
 * The real-valued form is used (the FE matrices and V of the projection workload are real).
 * CSR: n_rows, rowptr[n_rows+1], colind[nnz], values[nnz]; base 0 or 1; upper != 0 means
 * only the upper triangle (col >= row) is stored and the lower one is implied by symmetry.
 * V, Y: n_rows x k column-major with leading dimension ldv.
 * --------------------------------------------------------------------------------------- */
void oracle_csr_spmm(int n_rows, const int64_t *rowptr, const int *colind, const double *val,
                     int base, int upper, const double *V, int k, int64_t ldv, double *Y) {
    for (int c = 0; c < k; ++c)
        for (int i = 0; i < n_rows; ++i) Y[i + (int64_t)c * ldv] = 0.0;
    for (int i = 0; i < n_rows; ++i) {
        for (int64_t e = rowptr[i] - base; e < rowptr[i + 1] - base; ++e) {
            int j = colind[e] - base;
            double a = val[e];
            for (int c = 0; c < k; ++c) {
                Y[i + (int64_t)c * ldv] += a * V[j + (int64_t)c * ldv];
                if (upper && j != i) Y[j + (int64_t)c * ldv] += a * V[i + (int64_t)c * ldv];
            }
        }
    }
}

/* R (k x k, col-major) = V^T Y, summation over rows in increasing order. */
void oracle_gemm_tn(int n_rows, int k, const double *V, int64_t ldv, const double *Y, double *R) {
    for (int b = 0; b < k; ++b)
        for (int a = 0; a < k; ++a) {
            double s = 0.0;
            const double *va = V + (int64_t)a * ldv, *yb = Y + (int64_t)b * ldv;
            for (int i = 0; i < n_rows; ++i) s += va[i] * yb[i];
            R[a + (int64_t)b * k] = s;
        }
}

/* Modified Gram-Schmidt with one re-orthogonalisation pass, in place on V (N x k, ld ldv);
 * restates the block MGS loop with re-orthogonalisation of
 * src/analysis/KrylovROMSubstructure.cpp:433-454 for one column at a time. */
void oracle_mgs(int N, int k, double *V, int64_t ldv, int passes) {
    for (int j = 0; j < k; ++j) {
        double *vj = V + (int64_t)j * ldv;
        for (int pass = 0; pass < passes; ++pass) {
            for (int i = 0; i < j; ++i) {
                const double *vi = V + (int64_t)i * ldv;
                double h = 0.0;
                for (int t = 0; t < N; ++t) h += vi[t] * vj[t];
                for (int t = 0; t < N; ++t) vj[t] -= h * vi[t];
            }
        }
        double nrm = 0.0;
        for (int t = 0; t < N; ++t) nrm += vj[t] * vj[t];
        nrm = sqrt(nrm);
        for (int t = 0; t < N; ++t) vj[t] /= nrm;
    }
}
