/*
 * staccato_rom.h -- C ABI of the B200 reduced-order frequency sweep.
 *
 * The library replaces the ROM-projection and frequency-sweep bodies of STACCATO's
 * Krylov-substructure class (src/analysis/KrylovROMSubstructure.{h,cpp}) and the batched
 * sweeps of its GPU/CPU test programs.  Conventions follow the reference:
 *   - complex numbers are interleaved {re, im} doubles, the layout of MKL_Complex16 /
 *     STACCATOComplexDouble (src/tools/AuxiliaryParameters.h:52) and cuDoubleComplex;
 *   - dense matrices are column-major (LAPACK_COL_MAJOR, KrylovROMSubstructure.cpp:1428);
 *   - the caller owns every buffer; all pointers are device pointers unless named h_*;
 *   - every call returns an int status (SROM_OK = 0) instead of exit(EXIT_FAILURE)
 *     (the reference's error path, KrylovROMSubstructure.cpp:654-700);
 *   - a handle binds one device and one stream and is not thread-safe; distinct handles are.
 * No torch or CUDA types appear in the signatures; a CUDA stream is passed as void*.
 */
#ifndef STACCATO_ROM_H
#define STACCATO_ROM_H

#include <stdint.h>

#if defined(__GNUC__)
#define SROM_API __attribute__((visibility("default")))
#else
#define SROM_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef struct srom_handle srom_handle;

/* Layout-compatible with MKL_Complex16 / STACCATOComplexDouble / cuDoubleComplex. */
typedef struct {
    double re, im;
} srom_complex;

/* ---- status codes ---------------------------------------------------------------- */
#define SROM_OK 0
#define SROM_ERR_INVALID 1     /* bad argument (null pointer, size out of range, ...) */
#define SROM_ERR_CUDA 2        /* a CUDA runtime call failed; see srom_last_error */
#define SROM_ERR_ALLOC 3       /* device memory could not be obtained */
#define SROM_ERR_TIMEOUT 4     /* a bounded device-side wait ran out */
#define SROM_ERR_UNSUPPORTED 5 /* shape or option this build does not handle */

/* ---- per-frequency info values (int per frequency) ------------------------------- */
/*  0   solved;
 *  k>0 U(k,k) is exactly zero (1-based column), as LAPACK zgetrf reports it
 *      (the reference ignores this value, KrylovROMSubstructure.cpp:1428);
 * -1   mixed-precision refinement did not reach the tolerance within max_refine steps
 *      and SROM_FLAG_FALLBACK_FP64 was not set (the last iterate is returned);
 * -2   SROM_MIXED_TC only: a bounded device-side wait of the kernel ran out and the system
 *      was not solved (srom_sweep_host then returns SROM_ERR_TIMEOUT).                    */
#define SROM_INFO_NOT_CONVERGED (-1)
#define SROM_INFO_TIMEOUT (-2)

/* ---- precision of the factorisation ---------------------------------------------- */
#define SROM_FP64 0        /* all-FP64 complex LU, bit-identical to the restated zgetrf */
#define SROM_MIXED_FP32 1  /* complex FP32 LU + FP64 residual refinement               */
#define SROM_MIXED_TC 2    /* tensor-core form: the same LU and FP64 refinement as SROM_MIXED_FP32,
                              with every Schur update run on the tensor cores (tcgen05 MMAs on
                              three-piece bf16 splits of the FP32 operands, FP32 accumulation);
                              systems up to n = 512 (larger ones use the SROM_MIXED_FP32 kernel) */
#define SROM_MIXED_AUTO 3  /* each system on the faster of the two mixed kernels for its order and
                              right-hand sides: as srom_tune measured, else the tensor-core kernel
                              from n = 320 to 512 and the CUDA-core kernel elsewhere            */

/* ---- sweep flags ---------------------------------------------------------------------- */
#define SROM_FLAG_FALLBACK_FP64 1 /* re-solve non-converged frequencies in FP64 (steps = -1);
                                     with it, refinement stops early once the measured
                                     contraction shows tol cannot be reached in max_refine */
#define SROM_FLAG_KEEP_FACTORS 2  /* write LU factors + pivots into desc.LU / desc.ipiv (FP64) */
#define SROM_FLAG_MIXED_EVERY 4   /* mixed forms: factor every system in FP32.  Without it, systems
                                     small enough for two FP64 shared-memory factorisations per SM
                                     (n <= ~84) are solved by the FP64 kernel outright (steps = 0),
                                     which is faster than FP32 factors plus refinement there   */

/*
 * One reduced-order model and its frequency request.  Mirrors the members the reference's
 * sweep reads (myKComplexReduced, myMComplexReduced, myDComplexReduced, KrylovROMSubstructure.h:210-221)
 * and the arguments of backTransformKMOR (frequency list, load matrix, number of load cases;
 * KrylovROMSubstructure.h:156).
 *   A(w) = (1 + i*eta) * K + (-w^2) * M + (i*w) * D          (D may be NULL)
 * assembled per entry in the reference's zaxpy order (KrylovROMSubstructure.cpp:1411-1420).
 */
typedef struct {
    int n;                  /* ROM order (rows of K)                                 */
    int r;                  /* number of right-hand sides (load cases)               */
    int F;                  /* number of frequencies                                 */
    int ldk;                /* leading dimension of K, M, D (>= n)                   */
    const srom_complex *K;  /* n x n                                                 */
    const srom_complex *M;  /* n x n or NULL (no mass term: A = (1+i eta) K + i w D)   */
    const srom_complex *D;  /* n x n or NULL                                         */
    double eta;             /* hysteretic loss factor applied to K; 0 keeps K as is  */
    const srom_complex *rhs;/* n x r, leading dimension ldb (= B_r * F)              */
    int ldb;
    const double *omega;    /* F angular frequencies (rad/s)                         */
    srom_complex *X;        /* F blocks of n x r (ld n): x(w_f) = A(w_f)^-1 rhs      */
    int *info;              /* F ints or NULL                                        */
    int *steps;             /* F ints or NULL: refinement steps taken (0: solved in FP64
                               outright, -1: FP64 fallback)                          */
    double *berr;           /* F doubles or NULL: estimated relative error left (mixed) */
    srom_complex *LU;       /* F blocks of n x n or NULL (SROM_FLAG_KEEP_FACTORS)    */
    int *ipiv;              /* F blocks of n ints (1-based) or NULL                  */
    /* Back-projection (optional): y(w_f) = C x(w_f), the output of backTransformKMOR
     * (z_freq = C_R * z_krylov_freq, KrylovROMSubstructure.cpp:1446-1449).  With rhs = B_R
     * the same call yields the transfer functions H_R(w) = C_R A(w)^-1 B_R (:1433-1441). */
    int n_out;              /* rows of C (output DOFs); 0 = no back-projection       */
    int ldc;                /* leading dimension of C (>= n_out)                     */
    const srom_complex *C;  /* n_out x n or NULL                                     */
    srom_complex *Y;        /* F blocks of n_out x r (ld n_out) or NULL              */
} srom_rom_desc;

typedef struct {
    int precision;   /* SROM_FP64 / SROM_MIXED_FP32 / SROM_MIXED_TC / SROM_MIXED_AUTO */
    int max_refine;  /* refinement steps for the mixed forms (default 5 when <= 0)   */
    double tol;      /* a right-hand side stops refining when its error estimate
                        c (||d_s||/||d_s-1||) ||d_s||/||x|| <= tol (2-norms; c = 2, after the first
                        correction c = 4 with d_0 = x); 0 = 2^-34 */
    int flags;       /* SROM_FLAG_*                                                  */
} srom_sweep_opts;

/* ---- handle -------------------------------------------------------------------------- */
SROM_API int srom_create(srom_handle **h, int device);
SROM_API int srom_destroy(srom_handle *h);
SROM_API int srom_set_stream(srom_handle *h, void *cuda_stream);
SROM_API const char *srom_status_string(int status);
SROM_API const char *srom_last_error(const srom_handle *h);
SROM_API int srom_version(void);

/*
 * Frequency sweep over one or many ROMs in one call: for every (ROM, frequency) pair
 * assemble A(w), factor it with partial pivoting and solve for all r right-hand sides.
 * Replaces the hot loop of backTransformKMOR (KrylovROMSubstructure.cpp:1403-1453), the
 * dense CPU sweep of srcPerformanceTest/main.cpp:359-404 and the cuBLAS/cuSOLVER sweeps of
 * test/krylovTestGPU/matrixInSingleLoop/gpu/src/main.cu:236-387 and
 * test/krylovMidsizeTest/gpu/concurrent/batchedLU/src/main.cu:209-268 (which do not pivot).
 * All descriptor pointers are device pointers.  Asynchronous on the handle's stream.
 *
 * Sizes (B200, 227 KB of shared memory per block): the right-hand sides of a system live in
 * shared memory.  Orders whose 16-column panel also fits there (n <= 673 at r = 1, 548 at
 * r = 4, 314 at r = 16) run on the global kernel in every precision; larger ones, up to
 * n = 2560, on the large-order FP64 kernel, which needs n * r * 16 bytes + 64 KB (r <= 4 up to
 * n = 2559, r <= 8 up to n = 1388, r <= 16 up to n = 724); the mixed precisions solve those in
 * FP64 (steps = 0).  Requests beyond these limits return SROM_ERR_UNSUPPORTED.
 */
SROM_API int srom_sweep(srom_handle *h, const srom_rom_desc *roms, int n_roms, const srom_sweep_opts *opts);

/*
 * Same sweep with HOST buffers in every pointer of the descriptors (K, M, D, rhs, omega
 * in; X, info, steps, berr out).  Copies in, sweeps and copies out on the handle's stream,
 * then synchronises.  This is the drop-in form of backTransformKMOR, whose data live in
 * host std::vectors (KrylovROMSubstructure.h:210-221).
 */
SROM_API int srom_sweep_host(srom_handle *h, const srom_rom_desc *roms, int n_roms, const srom_sweep_opts *opts);

/* ---- captured sweeps and tuning ------------------------------------------------------- */
typedef struct srom_graph srom_graph;

/*
 * Plan a sweep over the given ROMs once (classification, cost-ordered work lists, scratch)
 * and capture its launches into a CUDA graph owned by the returned object; every
 * srom_graph_launch replays the whole batched sweep (all ROMs, all frequencies) on the
 * given stream with no host work.  The descriptors' device pointers must stay valid while
 * the graph exists; their contents may change between launches.
 */
SROM_API int srom_graph_create(srom_handle *h, const srom_rom_desc *roms, int n_roms, const srom_sweep_opts *opts,
                               srom_graph **graph);
SROM_API int srom_graph_launch(srom_graph *graph, void *cuda_stream);
SROM_API int srom_graph_destroy(srom_graph *graph);

/*
 * Autotune the kernel choices for each order in n_values with r right-hand sides, timed on a
 * synthetic system (2 x SMs frequencies) and used by later sweeps on this handle:
 *   - FP64: the whole system in shared memory vs. the blocked LU in global scratch;
 *   - mixed forms, where the FP64 choice is the shared-memory kernel: solving such systems in
 *     FP64 outright (steps = 0) vs. complex-FP32 factors in the mixed global kernel plus
 *     refinement (without a measurement the rule is: FP64 when two systems fit an SM).
 * Panel width, tile shapes and threads per system are fixed per kernel by its register and
 * shared-memory budget (compile-time).  cache_path (or NULL) is a JSON file of earlier choices
 * for this device, read first and rewritten with new entries.
 */
SROM_API int srom_tune(srom_handle *h, const int *n_values, int count, int r, const char *cache_path);

/* ---- adjoint (backward) sweep ---------------------------------------------------------- */
#define SROM_DPARAM_LOWRANK 0
#define SROM_DPARAM_DENSE 1

/* Derivative of A(w) with respect to one parameter:
 *   dA/dp(w) = (c0 + c1 (i w) + c2 (-w^2)) * G,   G = U diag(s) W^T (LOWRANK) or G (DENSE).
 * A stiffness-scaling parameter of a modal ROM is LOWRANK with U = W = its mode block and
 * s = the block's eigenvalues, c0 = 1 + i eta; the hysteretic loss factor is DENSE with
 * G = K and c0 = i; a damping scale is c1 = 1 with G = D; a mass scale is c2 = 1 with G = M. */
typedef struct {
    int kind;                /* SROM_DPARAM_LOWRANK or SROM_DPARAM_DENSE        */
    int rank;                /* LOWRANK: number of columns of U (and W)          */
    const srom_complex *U;   /* LOWRANK: n x rank (ld n)                         */
    const srom_complex *W;   /* LOWRANK: n x rank (ld n) or NULL for W = U       */
    const double *s;         /* LOWRANK: rank scales or NULL (ones)              */
    const srom_complex *G;   /* DENSE: n x n (ld n)                              */
    srom_complex c0, c1, c2; /* frequency polynomial of the derivative           */
} srom_dparam;

/*
 * Backward call of the FP64 sweep (no counterpart in the reference, which has no adjoint).
 * rom must come from srom_sweep with SROM_FLAG_KEEP_FACTORS (rom->LU, rom->ipiv, rom->X).
 * gbar: F blocks of n x r cotangents (leading dimension ldg, block stride ldg * r),
 * gbar_f = 2 dJ/d conj(x_f) for a real objective J.  For each frequency the kernel solves
 * A^H lambda = gbar_f with the kept factors and accumulates
 *     dJdp[j] = sum_f -Re( sum_c lambda_c^H dA_j(w_f) x_c ).
 * params: host array of n_params descriptors whose U/W/s/G are device pointers.
 * dJdp: n_params doubles (device).  lambda: F blocks of n x r (device) or NULL.
 */
SROM_API int srom_sweep_backward(srom_handle *h, const srom_rom_desc *rom, const srom_complex *gbar, int ldg,
                                 const srom_dparam *params, int n_params, double *dJdp, srom_complex *lambda);

/* ---- dense complex GEMM ------------------------------------------------------------ */
#define SROM_OP_N 0 /* op(X) = X   */
#define SROM_OP_T 1 /* op(X) = X^T */
#define SROM_OP_C 2 /* op(X) = X^H */

/*
 * Strided-batched complex FP64 GEMM on the FP64 tensor cores: C_b = alpha op(A_b) op(B_b) +
 * beta C_b for b < batch, with A_b = A + b * stride_a (likewise B, C; strides in elements, 0
 * broadcasts one matrix), column-major, op(A) m x k, op(B) k x n.  beta = 0 does not read C.
 * The batched products of the substructure coupling (the reference's cublasGemmBatchedEx calls,
 * test/IJCSA/src/IJSA.cu:875-979).  Summation order is fixed: results are deterministic.
 * batch <= 65535.  Asynchronous on the handle's stream.
 */
SROM_API int srom_zgemm_batched(srom_handle *h, int opa, int opb, int m, int n, int k, srom_complex alpha,
                                const srom_complex *A, int64_t lda, int64_t stride_a, const srom_complex *B,
                                int64_t ldb, int64_t stride_b, srom_complex beta, srom_complex *C, int64_t ldc,
                                int64_t stride_c, int batch);

/*
 * ROM projection R_m = V^T A_m V for up to three sparse FE matrices A_m (K, M, D) that share
 * one CSR pattern -- the real-valued form of generateROM (KrylovROMSubstructure.cpp:709-765:
 * mkl_sparse_z_mm for Y = A V, MathLibrary.cpp:491-532, then cblas_zgemm ConjTrans for
 * V^H Y, MathLibrary.cpp:177-234).  CSR: n_rows rows, rowptr[n_rows+1] (int64), colind
 * (int32), base 0 or 1 (the reference uses 1); upper != 0 means only the upper triangle of a
 * symmetric matrix is stored (the reference's SPARSE_FILL_MODE_UPPER, MathLibrary.cpp:502-507).
 * vals: host array of n_mats device pointers to the value arrays.  V: n_rows x k
 * column-major (ldv), k <= 4096: bases wider than 128 columns are projected in windows of 128
 * columns (one SpMM pass per window, one V^T Y pass per 128 x 128 block of R).  Device
 * workspace: (n_mats + 1) n_rows k doubles.  R: host array of n_mats device pointers, each k x k
 * column-major.  Summation order is fixed (deterministic results).
 */
SROM_API int srom_project_real(srom_handle *h, int64_t n_rows, const int64_t *rowptr, const int *colind, int base,
                               int upper, const double *const *vals, int n_mats, const double *V, int k, int64_t ldv,
                               double *const *R);

/*
 * Complex projection R_m = Z^H A_m V (Z = V when Z is NULL), the complex form of generateROM
 * (KrylovROMSubstructure.cpp:709-765: mkl_sparse_z_mm for y = A V, cblas_zgemm ConjTrans for
 * Z^H y, with Z the left basis of non-symmetric MIMO systems).  A_m: complex values (nnz each,
 * host array of n_mats device pointers) on one CSR pattern as in srom_project_real; upper != 0
 * stores the upper triangle of a complex-symmetric matrix (A_ji = A_ij, the reference's
 * SPARSE_MATRIX_TYPE_SYMMETRIC).  V, Z: n_rows x k complex column-major (ldv, ldz), k <= 2048.
 * R: host array of n_mats device pointers, each k x k complex column-major.  Runs on the real
 * kernels: the basis is split into [Re V | Im V] rows, A's real and imaginary parts are applied
 * as two value arrays of the same pattern, and the four real blocks of [Re Z | Im Z]^T
 * [Re Y | Im Y] combine into Z^H Y.  Summation order is fixed (deterministic results).
 */
SROM_API int srom_project_complex(srom_handle *h, int64_t n_rows, int64_t nnz, const int64_t *rowptr,
                                  const int *colind, int base, int upper, const srom_complex *const *vals, int n_mats,
                                  const srom_complex *V, int k, int64_t ldv, const srom_complex *Z, int64_t ldz,
                                  srom_complex *const *R);

/*
 * FP64 block Gram-Schmidt orthonormalisation of V (n_rows x k, column-major, ldv) in place,
 * the reference's block scheme with re-orthogonalisation (KrylovROMSubstructure.cpp:433-475,
 * :513-534): the columns are taken in panels of 32; each pass projects the panel out of the
 * orthonormal columns before it and orthonormalises it through the Cholesky factor of its
 * projected Gram matrix.  `passes` passes are made per panel (0 is taken as 1; two keep the
 * basis orthonormal to rounding level for condition numbers up to about 1e7).  The result is
 * the Q of V = Q R with a positive diagonal R.  Columns that are linearly dependent on the
 * ones before them come out non-finite (no rank revealing).
 */
SROM_API int srom_orthonormalize(srom_handle *h, double *V, int64_t n_rows, int k, int64_t ldv, int passes);

/*
 * Krylov basis of a substructure, KrylovROMSubstructure::addKrylovModesForExpansionPoint
 * (src/analysis/KrylovROMSubstructure.cpp:367-569).  For every expansion point f0 (Hz,
 * w0 = 2 pi f0): K~ = -(K - w0^2 M + i w0 D) is factored on the GPU (band LDL^T after a
 * reverse Cuthill-McKee ordering, no pivoting: K~ must be complex symmetric and its leading
 * blocks nonsingular), Q = K~^-1 B (then, from the second point on, re-orthogonalised against
 * the basis so far), and krylov_order - 1 times Q = K~^-1 (M Q) re-orthogonalised; each block
 * is reduced by a column-pivoted QR to its leading columns with |R_ii| > tol (absolute, as in
 * the reference; tol <= 0 means its 1e-8) and appended to V.
 *   rowptr/colind: CSR pattern shared by K, M, D (device; base 0 or 1; upper = 1 for the
 *   upper triangle of the symmetric matrix, 0 for the full symmetric pattern).  K, M, D
 *   (nullable): device values.  B: device n_rows x n_in, ldb.  exp_points_hz: HOST array.
 *   V: device n_rows x max_cols (ldv); *n_cols (host) receives the number of columns written.
 * Device memory: the band, (n_rows + 128) x (bandwidth + 129) x 16 bytes (srom_band_order
 * reports it), plus a few n_rows x n_in blocks.  Synchronises the handle's stream.
 */
SROM_API int srom_krylov_basis(srom_handle *h, int64_t n_rows, int64_t nnz, const int64_t *rowptr, const int *colind,
                               int base, int upper, const srom_complex *K, const srom_complex *M, const srom_complex *D,
                               const srom_complex *B, int n_in, int64_t ldb, const double *exp_points_hz, int n_points,
                               int krylov_order, double tol, srom_complex *V, int64_t ldv, int max_cols, int *n_cols);

/*
 * Full-order frequency sweep, KrylovROMSubstructure::performSolveFOM
 * (src/analysis/KrylovROMSubstructure.cpp:1355-1391): for every frequency f (Hz, w = 2 pi f)
 * solve (K - w^2 M + i w D) X_f = F directly on the GPU, with the band LDL^T of
 * srom_krylov_basis (same pattern arguments and memory; the matrix must be complex symmetric).
 *   F: device n_rows x r loads (ldf).  freq_hz: HOST array.  X: device, n_freq blocks of
 *   n_rows x r (leading dimension ldx, block f at X + f * ldx * r), stacked per frequency like
 *   the reference's results vector.  Synchronises the handle's stream.
 */
SROM_API int srom_fom_sweep(srom_handle *h, int64_t n_rows, int64_t nnz, const int64_t *rowptr, const int *colind,
                            int base, int upper, const srom_complex *K, const srom_complex *M, const srom_complex *D,
                            const srom_complex *F, int r, int64_t ldf, const double *freq_hz, int n_freq,
                            srom_complex *X, int64_t ldx);

/*
 * Pivots of the band L D L^T factorisations made by the last srom_krylov_basis or
 * srom_fom_sweep call on this handle.  The factorisation does not pivot; like PARDISO with the
 * reference's iparm[9] = 13 (KrylovROMSubstructure.cpp:621) it replaces a pivot d with
 * |d| < 1e-13 ||A||_inf by the value of the same phase and modulus 1e-13 ||A||_inf and goes on
 * (an exactly zero pivot still fails the call).  factorisations, perturbed: counts;
 * min_pivot_ratio: the smallest |d| / ||A||_inf before perturbation (a small value warns of a
 * shift close to an eigenvalue).  Any output pointer may be NULL.
 */
SROM_API int srom_band_pivot_report(const srom_handle *h, int64_t *factorisations, int64_t *perturbed,
                                    double *min_pivot_ratio);

/*
 * The handle keeps the full symmetric pattern and reverse Cuthill-McKee order of its last
 * srom_krylov_basis / srom_fom_sweep call on the device (about 12 bytes per stored entry and
 * 12 per row), and a later call whose pattern is the same (sizes, base, storage and a 64-bit hash
 * of rowptr and colind) reuses them instead of symmetrising, ordering and uploading again; a
 * different pattern replaces them.  The reference instead repeats PARDISO's analysis (phase 11)
 * before every factorisation (src/analysis/KrylovROMSubstructure.cpp:647, per expansion point
 * at :408 and per frequency of the full-order sweep at :1380).
 * srom_band_cache_report: reused = 1 if the last such call found its pattern in the cache;
 * cached_rows / bandwidth describe the cached pattern (0 when none).  Any pointer may be NULL.
 * srom_band_cache_release: frees the cached pattern's device memory (synchronises the stream).
 */
SROM_API int srom_band_cache_report(const srom_handle *h, int *reused, int64_t *cached_rows, int64_t *bandwidth);
SROM_API int srom_band_cache_release(srom_handle *h);

/*
 * Host-only: the reverse Cuthill-McKee ordering srom_krylov_basis uses for a pattern (HOST
 * rowptr/colind, as above).  perm (n_rows ints, may be NULL): perm[k] = original row of row k;
 * *bandwidth = max |new i - new j| over the entries; *band_bytes = device bytes of the band
 * factor.  err (may be NULL) receives a message on failure.
 */
SROM_API int srom_band_order(int64_t n_rows, int64_t nnz, const int64_t *rowptr, const int *colind, int base, int upper,
                             int *perm, int64_t *bandwidth, int64_t *band_bytes, char *err, int err_len);

/*
 * FP64 sweep of one ROM that allocates no device memory.  No counterpart in the reference.
 * For callers that cannot let a library allocate: programs that own all device memory
 * through their own pool, or real-time loops in which cudaMalloc's implicit synchronisation
 * and possible failure are not acceptable.  It needs no handle; it runs on the current
 * device and the given stream (NULL = legacy default stream) and returns after enqueueing.
 * Scratch is a 33 MB array inside the library (descriptor, work list and 32 MiB of matrix
 * slots), held on every device that loads the library until the process exits.
 * Limits: n <= 512, F <= 65536, and the blocked kernel's shared memory, about
 * 24 n r + 288 (n + 1) + 21 KB bytes, within the device's per-block limit (r <= 5 at n = 512,
 * r <= 16 at n <= 314 on a B200); larger requests return SROM_ERR_UNSUPPORTED with the reason
 * in err (err_len bytes).
 * The first call on each device looks up the array's device address; make that first call
 * before any stream capture.  After cudaDeviceReset the next call looks the address up again.  Every call reuses the array (the work counter is cleared on
 * each call): calls whose work overlaps on the GPU race and must be serialised by the caller.
 * Results (x and, when n_out > 0, y = C x) are bit-identical to srom_sweep with SROM_FP64.
 */
SROM_API int srom_sweep_fp64_noalloc(const srom_rom_desc *rom, void *cuda_stream, char *err, int err_len);

/* ---- dense ROM files (host only; no handle, no GPU work) ------------------------------- */
/*
 * Read a dense Matrix Market file, the format of the reference's ROM test inputs
 * (io::readMtxDense, test/krylovTestGPU/matrixInSingleLoop/gpu/src/io/io.cu:20-80): '%' lines,
 * "rows cols", then rows*cols entries column after column, each "re im" (complex, the default
 * and the reference's files) or one value ("%%MatrixMarket ... real" banner).  A banner with
 * "row major" (AuxiliaryFunctions.cpp:91) means entries row after row.  A is filled column-major
 * (ld rows); with A == NULL only *rows and *cols are set.  Short or over-long files and a
 * capacity below rows*cols return SROM_ERR_INVALID with the reason in err.
 */
SROM_API int srom_mtx_read_dense(const char *path, int64_t *rows, int64_t *cols, srom_complex *A, int64_t capacity,
                                 char *err, int err_len);
/* Write A (rows x cols, column-major, lda) in the reference's dense complex format
 * (AuxiliaryFunctions::writeMKLComplexDenseMatrixMtxFormat, src/tools/AuxiliaryFunctions.cpp:80-110),
 * 17 significant digits so that srom_mtx_read_dense returns the same bits. */
SROM_API int srom_mtx_write_dense(const char *path, int64_t rows, int64_t cols, const srom_complex *A, int64_t lda,
                                  char *err, int err_len);
/* Write a solution vector as the reference's "Real Imag" table (io::writeSolVecComplex,
 * io.cu:83-106: width-25 columns, CRLF lines), with 17 significant digits instead of 16. */
SROM_API int srom_write_solution(const char *path, const srom_complex *x, int64_t count, char *err, int err_len);

/* ---- per-launch timing -------------------------------------------------------------- */
/* One record per kernel launch issued while profiling is enabled: CUDA events recorded on
 * the handle's stream around the launch, plus the algorithmic work the launch performs
 * (complex LU + solve: 8/3 n^3 + 8 n^2 r real flops per system; projection: bytes). */
typedef struct {
    char name[32];
    float ms;         /* device time between the launch's start and end events */
    long long items;  /* systems (or rows) the launch processed                */
    double flops;     /* algorithmic real floating-point operations            */
    double bytes;     /* algorithmic DRAM bytes                                */
} srom_kernel_time;

SROM_API int srom_profile_enable(srom_handle *h, int enable);
/* Waits for the recorded launches, copies up to max records into out (may be NULL),
 * stores the number of records in *count and clears the list. */
SROM_API int srom_profile_read(srom_handle *h, srom_kernel_time *out, int max, int *count);

#ifdef __cplusplus
}
#endif

#endif /* STACCATO_ROM_H */
