// Host-side entry points of the adjoint (backward) sweep kernels.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include "srom_device.cuh"

namespace srom {

// dA/dp(w) = (c0 + c1 (i w) + c2 (-w^2)) G, G = U diag(s) W^T (kind 0) or dense (kind 1)
struct DParamDev {
    int kind, rank, term0, nterm;
    const double2 *U, *W;
    const double *s;
    const double2 *G;
    double2 c0, c1, c2;
};
struct DParamTerm {
    int param, k;
};
struct AdjointArgs {
    const RomDev *rom;
    const double2 *gbar;
    int64_t ldg, ldg_f;
    const DParamDev *params;
    int n_params;
    const DParamTerm *terms;
    int n_terms;
    double *partial;  // F x n_params
    double2 *lambda;  // optional F x n x r
    int *counter;
};

size_t adjoint_smem_bytes(int n, int r, int n_terms);
cudaError_t launch_adjoint(const AdjointArgs &a, int n, int r, int F, int grid, double *dJdp, cudaStream_t st);

}  // namespace srom
