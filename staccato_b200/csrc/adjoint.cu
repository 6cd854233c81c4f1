// Adjoint (backward) sweep: parameter gradients of a real objective J(x(w_1..w_F)).
//
// For every frequency, with the FP64 factors P A = L U kept by the forward sweep
// (SROM_FLAG_KEEP_FACTORS) and the cotangent gbar_f = 2 dJ/d conj(x_f):
//     A^H lambda = gbar      (U^H y = gbar, L^H z = y, lambda = P z)
//     dJ/dp_j  += -Re( sum_c lambda_c^H dA_j(w) x_c ),
// where dA_j(w) = (c0 + c1 (i w) + c2 (-w^2)) G_j and G_j is either dense or U diag(s) W^T
// (low rank; the stiffness-scaling parameters of a modal ROM are rank-8 blocks).
// One CTA per frequency (persistent, work counter); per-frequency contributions are written
// to a partial array and summed over frequencies in a fixed order, so the gradient is
// deterministic.  The reference has no adjoint; this is the backward call of the sweep.
#include <cuda_runtime.h>
#include <stdint.h>

#include "adjoint_kernels.h"
#include "srom_device.cuh"

namespace srom {

constexpr int ADJ_NT = 256;
constexpr int ADJ_NW = ADJ_NT / 32;

__device__ __forceinline__ double2 conj2(double2 a) { return make_double2(a.x, -a.y); }
__device__ __forceinline__ double2 cfma(double2 a, double2 b, double2 c) {  // c + a*b
    return make_double2(fma(a.x, b.x, fma(-a.y, b.y, c.x)), fma(a.x, b.y, fma(a.y, b.x, c.y)));
}

__device__ __forceinline__ double2 warp_sum2(double2 v) {
#pragma unroll
    for (int off = 16; off; off >>= 1) {
        v.x += __shfl_xor_sync(FULL_MASK, v.x, off);
        v.y += __shfl_xor_sync(FULL_MASK, v.y, off);
    }
    return v;
}

// A^H lambda = g in place on Y (n x r, ld n, shared memory) using LU (n x n, ld n) and ipiv.
__device__ void conj_solve(const double2 *LU, const int *ipiv, int n, double2 *Y, int r) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    // U^H y = g: y_j = (g_j - sum_{i<j} conj(U_ij) y_i) / conj(U_jj)
    for (int jb = 0; jb < n; jb += 32) {
        const int je = min(jb + 32, n);
        // contributions of the solved rows [0, jb) to the rows of this block
        for (int t = warp; t < (je - jb) * r; t += ADJ_NW) {
            const int j = jb + t % (je - jb), c = t / (je - jb);
            double2 s = make_double2(0.0, 0.0);
            for (int i = lane; i < jb; i += 32) s = cfma(conj2(LU[i + (int64_t)j * n]), Y[i + (int64_t)c * n], s);
            s = warp_sum2(s);
            if (lane == 0) {
                double2 &y = Y[j + (int64_t)c * n];
                y.x -= s.x;
                y.y -= s.y;
            }
        }
        __syncthreads();
        for (int c = warp; c < r; c += ADJ_NW) {
            double2 *y = Y + (int64_t)c * n;
            for (int j = jb; j < je; ++j) {
                double2 s = make_double2(0.0, 0.0);
                for (int i = jb + lane; i < j; i += 32) s = cfma(conj2(LU[i + (int64_t)j * n]), y[i], s);
                s = warp_sum2(s);
                if (lane == 0) {
                    const double2 v = make_double2(y[j].x - s.x, y[j].y - s.y);
                    y[j] = cdiv(v, conj2(LU[j + (int64_t)j * n]));
                }
                __syncwarp();
            }
        }
        __syncthreads();
    }
    // L^H z = y: z_j = y_j - sum_{i>j} conj(L_ij) z_i   (unit diagonal)
    for (int jend = n; jend > 0; jend -= 32) {
        const int jb = max(jend - 32, 0);
        for (int t = warp; t < (jend - jb) * r; t += ADJ_NW) {
            const int j = jb + t % (jend - jb), c = t / (jend - jb);
            double2 s = make_double2(0.0, 0.0);
            for (int i = jend + lane; i < n; i += 32) s = cfma(conj2(LU[i + (int64_t)j * n]), Y[i + (int64_t)c * n], s);
            s = warp_sum2(s);
            if (lane == 0) {
                double2 &y = Y[j + (int64_t)c * n];
                y.x -= s.x;
                y.y -= s.y;
            }
        }
        __syncthreads();
        for (int c = warp; c < r; c += ADJ_NW) {
            double2 *y = Y + (int64_t)c * n;
            for (int j = jend - 1; j >= jb; --j) {
                double2 s = make_double2(0.0, 0.0);
                for (int i = j + 1 + lane; i < jend; i += 32) s = cfma(conj2(LU[i + (int64_t)j * n]), y[i], s);
                s = warp_sum2(s);
                if (lane == 0) {
                    y[j].x -= s.x;
                    y[j].y -= s.y;
                }
                __syncwarp();
            }
        }
        __syncthreads();
    }
    // lambda = P z: undo the interchanges in reverse order
    if (threadIdx.x < r) {
        double2 *y = Y + (int64_t)threadIdx.x * n;
        for (int j = n - 1; j >= 0; --j) {
            const int p = ipiv[j] - 1;
            if (p != j) swap2(y[j], y[p]);
        }
    }
    __syncthreads();
}

__global__ void __launch_bounds__(ADJ_NT) adjoint_kernel(AdjointArgs a) {
    extern __shared__ double2 sh[];
    __shared__ int s_item;
    const RomDev R = *a.rom;
    const int n = R.n, r = R.r;
    double2 *Y = sh;                       // lambda (n x r)
    double2 *Xs = Y + (int64_t)n * r;      // x (n x r)
    double2 *pairs = Xs + (int64_t)n * r;  // one complex per (parameter, rank term)
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (;;) {
        if (tid == 0) s_item = atomicAdd(a.counter, 1);
        __syncthreads();
        const int f = s_item;
        __syncthreads();
        if (f >= R.F) break;
        const double w = R.omega[f];
        const double2 *LU = R.LU + (int64_t)f * n * n;
        const int *ipiv = R.ipiv + (int64_t)f * n;
        for (int e = tid; e < n * r; e += ADJ_NT) {
            const int i = e % n, c = e / n;
            Y[i + (int64_t)c * n] = a.gbar[(int64_t)f * a.ldg_f + i + (int64_t)c * a.ldg];
            Xs[i + (int64_t)c * n] = R.X[(int64_t)f * n * r + i + (int64_t)c * n];
        }
        __syncthreads();
        conj_solve(LU, ipiv, n, Y, r);
        if (a.lambda)
            for (int e = tid; e < n * r; e += ADJ_NT) a.lambda[(int64_t)f * n * r + e] = Y[e];
        // one warp per (parameter, term): S = sum_c (lambda_c^H U_k)(W_k^T x_c) s_k, or lambda_c^H G x_c
        for (int t = warp; t < a.n_terms; t += ADJ_NW) {
            const DParamTerm T = a.terms[t];
            const DParamDev &P = a.params[T.param];
            double2 S = make_double2(0.0, 0.0);
            for (int c = 0; c < r; ++c) {
                const double2 *lam = Y + (int64_t)c * n;
                const double2 *x = Xs + (int64_t)c * n;
                if (P.kind == 0) {
                    const int k = T.k;
                    const double2 *u = P.U + (int64_t)k * n;
                    const double2 *wv = (P.W ? P.W : P.U) + (int64_t)k * n;
                    double2 av = make_double2(0.0, 0.0), bv = make_double2(0.0, 0.0);
                    for (int i = lane; i < n; i += 32) {
                        av = cfma(conj2(lam[i]), u[i], av);
                        bv = cfma(wv[i], x[i], bv);
                    }
                    av = warp_sum2(av);
                    bv = warp_sum2(bv);
                    const double sk = P.s ? P.s[k] : 1.0;
                    S = cfma(make_double2(sk * av.x, sk * av.y), bv, S);
                } else {
                    // dense: sum_i conj(lam_i) (G x)_i, rows split over lanes
                    double2 acc = make_double2(0.0, 0.0);
                    for (int i = lane; i < n; i += 32) {
                        double2 gx = make_double2(0.0, 0.0);
                        for (int l = 0; l < n; ++l) gx = cfma(P.G[i + (int64_t)l * n], x[l], gx);
                        acc = cfma(conj2(lam[i]), gx, acc);
                    }
                    acc = warp_sum2(acc);
                    S.x += acc.x;
                    S.y += acc.y;
                }
            }
            if (lane == 0) pairs[t] = S;
        }
        __syncthreads();
        for (int j = tid; j < a.n_params; j += ADJ_NT) {
            const DParamDev &P = a.params[j];
            double2 S = make_double2(0.0, 0.0);
            for (int t = P.term0; t < P.term0 + P.nterm; ++t) {
                S.x += pairs[t].x;
                S.y += pairs[t].y;
            }
            // coef(w) = c0 + c1 (i w) + c2 (-w^2)
            const double2 coef = make_double2(P.c0.x - w * P.c1.y - w * w * P.c2.x, P.c0.y + w * P.c1.x - w * w * P.c2.y);
            const double re = coef.x * S.x - coef.y * S.y;
            a.partial[(int64_t)f * a.n_params + j] = -re;
        }
        __syncthreads();
    }
}

__global__ void adjoint_reduce_kernel(const double *__restrict__ partial, int F, int P, double *__restrict__ out) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < P; j += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int f = 0; f < F; ++f) s += partial[(int64_t)f * P + j];
        out[j] = s;
    }
}

size_t adjoint_smem_bytes(int n, int r, int n_terms) {
    return sizeof(double2) * ((size_t)2 * n * r + (size_t)n_terms);
}

cudaError_t launch_adjoint(const AdjointArgs &a, int n, int r, int F, int grid, double *dJdp, cudaStream_t st) {
    const size_t smem = adjoint_smem_bytes(n, r, a.n_terms);
    cudaError_t e = cudaFuncSetAttribute(adjoint_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    adjoint_kernel<<<grid, ADJ_NT, smem, st>>>(a);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    adjoint_reduce_kernel<<<(a.n_params + 127) / 128, 128, 0, st>>>(a.partial, F, a.n_params, dJdp);
    return cudaGetLastError();
}

}  // namespace srom
