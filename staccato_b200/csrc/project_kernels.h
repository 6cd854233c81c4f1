// Host-side entry points of the projection kernels (used by the C ABI in capi.cu).
#pragma once

#include <algorithm>
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace srom {

struct ProjVals {
    const double *v[3];
};
struct ProjOut {
    double *r[3];
};

// widest basis of the projection (real form; the complex form projects 2k real columns)
constexpr int PRJ_MAX_K = 4096;

cudaError_t launch_transpose(const double *V, int64_t N, int k, int64_t ldv, double *Vt, cudaStream_t st);
cudaError_t launch_spmm(int64_t N, const int64_t *rowptr, const int *colind, int base, int upper, ProjVals vals,
                        int n_mats, const double *Vt, int k, double *Y, int64_t y_stride, int sms, cudaStream_t st);
// doubles of the V^T Y partials buffer (one window of at most 128 x 128 per matrix and CTA)
size_t vty_partial_doubles(int k, int n_mats, int nblk);
cudaError_t launch_vty(int64_t N, int k, const double *Vt, const double *Y, int64_t y_stride, int n_mats, int nblk,
                       double *partial, ProjOut out, cudaStream_t st);
cudaError_t launch_transpose_split(const double2 *V, int64_t N, int k, int64_t ldv, double *Wt, cudaStream_t st);
cudaError_t launch_split_values(const double2 *a, int64_t nnz, double *re, double *im, int sms, cudaStream_t st);
cudaError_t launch_combine_y(double *Pr, const double *Pi, int64_t N, int k, int sms, cudaStream_t st);
cudaError_t launch_combine_r(const double *G, int k, double2 *R, cudaStream_t st);
size_t gs_workspace_doubles(int k, int nblk);
cudaError_t launch_gram_schmidt(double *V, int64_t N, int k, int64_t ldv, int passes, double *work, int nblk,
                                cudaStream_t st);

}  // namespace srom
