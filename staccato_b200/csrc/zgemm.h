// Complex FP64 GEMM on the FP64 tensor cores (zgemm.cu): host-side entry points.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace srom {

enum { ZG_N = 0, ZG_T = 1, ZG_C = 2 };

// C[b] = alpha op(A[b]) op(B[b]) + beta C[b] for b < batch (column-major; A[b] = A + b sa,
// likewise B, C).  op(A) is m x k, op(B) k x n.  beta = 0 does not read C.  When the tiles of
// C cannot fill the GPU (sms SMs) and k is long, k is split over CTAs into partials held in
// work (work_elems double2; zgemm_work_elems gives the size that allows the full split) and
// reduced in split order; with work = null the product runs unsplit.
struct Zgemm {
    int opa = ZG_N, opb = ZG_N;
    int m = 0, n = 0, k = 0;
    double2 alpha{1.0, 0.0}, beta{0.0, 0.0};
    const double2 *A = nullptr;
    int64_t lda = 0, sa = 0;
    const double2 *B = nullptr;
    int64_t ldb = 0, sb = 0;
    double2 *C = nullptr;
    int64_t ldc = 0, sc = 0;
    int batch = 1;
    double2 *work = nullptr;
    int64_t work_elems = 0;
    int sms = 148;
};

cudaError_t zgemm(const Zgemm &z, cudaStream_t st);
int64_t zgemm_work_elems(int m, int n, int k, int batch, int sms);

// out (device) = ||x||_2 over count complex entries, deterministic; work: znorm2_work_doubles()
size_t znorm2_work_doubles();
cudaError_t znorm2(const double2 *x, int64_t count, double *work, double *out, cudaStream_t st);

}  // namespace srom
