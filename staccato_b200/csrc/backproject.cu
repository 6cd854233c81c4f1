// Back-projection of the swept solutions onto the output DOFs: Y_f = C X_f for every
// frequency f of one ROM (C: n_out x n, ld ldc; X_f: n x r, ld n; Y_f: n_out x r, ld n_out).
//
// Reference: backTransformKMOR forms z_freq = C_R * z_krylov_freq with cblas_zgemm per
// frequency (KrylovROMSubstructure.cpp:1446-1449) and, with B_R as right-hand sides, the
// transfer functions H_R = C_R (A^-1 B_R) (:1433-1441).  Here one launch covers all F
// frequencies after the sweep; each output entry is the sequential complex FMA chain
// y_ic = sum_j C_ij x_jc over increasing j (the order the oracle restates), so FP64 results
// are reproducible bit for bit.  Threads of a CTA take consecutive rows i (coalesced reads
// of C's columns); the CTA's X_f block is staged in shared memory when it fits.
#include <cuda_runtime.h>
#include <stdint.h>

#include "srom_device.cuh"
#include "sweep_kernels.h"

namespace srom {

constexpr int BP_NT = 256;
constexpr int BP_SMEM_MAX = 48 * 1024;

__device__ __forceinline__ double2 bp_cfma(double2 a, double2 b, double2 c) {  // c + a*b
    return make_double2(__fma_rn(a.x, b.x, __fma_rn(-a.y, b.y, c.x)), __fma_rn(a.x, b.y, __fma_rn(a.y, b.x, c.y)));
}

__global__ void __launch_bounds__(BP_NT) backproject_kernel(BackProj p, int stage_x) {
    extern __shared__ double2 xs[];
    const int64_t nr = (int64_t)p.n * p.r;
    const int64_t outs = (int64_t)p.n_out * p.r;
    for (int f = blockIdx.x; f < p.F; f += gridDim.x) {
        const double2 *Xf = p.X + (int64_t)f * nr;
        const double2 *xsrc = Xf;
        if (stage_x) {
            __syncthreads();
            for (int64_t e = threadIdx.x; e < nr; e += BP_NT) xs[e] = Xf[e];
            __syncthreads();
            xsrc = xs;
        }
        double2 *Yf = p.Y + (int64_t)f * outs;
        for (int64_t e = threadIdx.x; e < outs; e += BP_NT) {
            const int i = (int)(e % p.n_out), c = (int)(e / p.n_out);
            const double2 *xc = xsrc + (int64_t)c * p.n;
            double2 acc = make_double2(0.0, 0.0);
            for (int j = 0; j < p.n; ++j) acc = bp_cfma(p.C[i + (int64_t)j * p.ldc], xc[j], acc);
            Yf[e] = acc;
        }
    }
}

cudaError_t launch_backproject(const BackProj &p, int sms, cudaStream_t st) {
    if (p.F <= 0 || p.n_out <= 0 || p.r <= 0) return cudaSuccess;
    const size_t xb = sizeof(double2) * (size_t)p.n * p.r;
    const int stage = xb <= (size_t)BP_SMEM_MAX ? 1 : 0;
    const int grid = (int)(p.F < sms * 8 ? p.F : sms * 8);
    backproject_kernel<<<grid, BP_NT, stage ? xb : 0, st>>>(p, stage);
    return cudaGetLastError();
}

}  // namespace srom
