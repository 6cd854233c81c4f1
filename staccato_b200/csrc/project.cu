// ROM projection kernels: R_m = V^T A_m V for sparse FE matrices A_m sharing one CSR pattern,
// and the FP64 Gram-Schmidt orthonormalisation of the basis V.
//
// Reference: generateROM (src/analysis/KrylovROMSubstructure.cpp:709-765) computes
// Y = A V with mkl_sparse_z_mm (src/tools/MathLibrary.cpp:491-532) and R = V^H Y with
// cblas_zgemm ConjTrans (src/tools/MathLibrary.cpp:177-234), one matrix after another; the
// basis comes from block Gram-Schmidt with re-orthogonalisation (KrylovROMSubstructure.cpp:433-454).
//
// B200 layout: V is transposed once into row-major Vt (N x k) so that the k entries of a
// basis row are contiguous; the SpMM gives each warp one row and each lane k/32 basis
// columns, and every gathered Vt row feeds all matrices of the pattern (K and M share it);
// Y_m is written row-major.  R_m = Vt^T Y_m runs on the FP64 tensor cores
// (mma.sync m8n8k4 f64): each CTA reduces a contiguous row range into a private k x k
// partial, and a second kernel sums the partials in CTA order (deterministic).
#include <cuda_runtime.h>
#include <stdint.h>

#include "project_kernels.h"

namespace srom {

constexpr int PRJ_MAX_MATS = 3;

// ---- V (column-major, ldv) -> Vt (row-major N x k) --------------------------------------
__global__ void transpose_kernel(const double *__restrict__ V, int64_t N, int k, int64_t ldv,
                                 double *__restrict__ Vt) {
    __shared__ double t[32][33];
    const int64_t r0 = (int64_t)blockIdx.x * 32;
    const int c0 = blockIdx.y * 32;
    for (int y = threadIdx.y; y < 32; y += blockDim.y) {
        const int64_t r = r0 + threadIdx.x;
        const int c = c0 + y;
        if (r < N && c < k) t[y][threadIdx.x] = V[r + (int64_t)c * ldv];
    }
    __syncthreads();
    for (int y = threadIdx.y; y < 32; y += blockDim.y) {
        const int64_t r = r0 + y;
        const int c = c0 + threadIdx.x;
        if (r < N && c < k) Vt[r * k + c] = t[threadIdx.x][y];
    }
}

// ---- Y_m = A_m V  (full CSR pattern, shared by the n_mats value arrays) -----------------
template <int CPL>
__global__ void spmm_full_kernel(int64_t N, const int64_t *__restrict__ rowptr, const int *__restrict__ colind,
                                 int base, ProjVals vals, int n_mats, const double *__restrict__ Vt, int k,
                                 double *__restrict__ Y, int64_t y_stride) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarp = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t row = warp; row < N; row += nwarp) {
        double acc[PRJ_MAX_MATS][CPL];
#pragma unroll
        for (int m = 0; m < PRJ_MAX_MATS; ++m)
#pragma unroll
            for (int q = 0; q < CPL; ++q) acc[m][q] = 0.0;
        const int64_t e0 = rowptr[row] - base, e1 = rowptr[row + 1] - base;
        for (int64_t e = e0; e < e1; ++e) {
            const int64_t col = colind[e] - base;
            double a[PRJ_MAX_MATS];
#pragma unroll
            for (int m = 0; m < PRJ_MAX_MATS; ++m) a[m] = m < n_mats ? vals.v[m][e] : 0.0;
            const double *vr = Vt + col * k;
#pragma unroll
            for (int q = 0; q < CPL; ++q) {
                const int c = lane + 32 * q;
                const double v = c < k ? vr[c] : 0.0;
#pragma unroll
                for (int m = 0; m < PRJ_MAX_MATS; ++m) acc[m][q] = fma(a[m], v, acc[m][q]);
            }
        }
#pragma unroll
        for (int m = 0; m < PRJ_MAX_MATS; ++m) {
            if (m >= n_mats) break;
#pragma unroll
            for (int q = 0; q < CPL; ++q) {
                const int c = lane + 32 * q;
                if (c < k) Y[m * y_stride + row * k + c] = acc[m][q];
            }
        }
    }
}

// Upper-triangle storage of a symmetric matrix (the reference's CSR,
// src/tools/MathLibrary.cpp:502-507): the mirrored entries (j, i), j != i, are added with
// FP64 atomics after the row pass above has written the stored half.
__global__ void spmm_upper_mirror_kernel(int64_t N, const int64_t *__restrict__ rowptr,
                                         const int *__restrict__ colind, int base, ProjVals vals, int n_mats,
                                         const double *__restrict__ Vt, int k, double *__restrict__ Y,
                                         int64_t y_stride) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarp = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t row = warp; row < N; row += nwarp) {
        const int64_t e0 = rowptr[row] - base, e1 = rowptr[row + 1] - base;
        for (int64_t e = e0; e < e1; ++e) {
            const int64_t col = colind[e] - base;
            if (col == row) continue;
            for (int c = lane; c < k; c += 32) {
                const double v = Vt[row * k + c];
                for (int m = 0; m < n_mats; ++m) atomicAdd(&Y[m * y_stride + col * k + c], vals.v[m][e] * v);
            }
        }
    }
}

// ---- R_m partial = Vt[rows]^T Y_m[rows] on FP64 tensor cores ------------------------------
// One warp per 8-row band of R (kp/8 warps), 8x8 tiles across the band; rows of Vt / Y are
// staged 32 at a time in shared memory (leading dimension kp + 4 keeps the fragment loads
// free of bank conflicts).
template <int NMAT>
__global__ void __launch_bounds__(512) vty_partial_kernel(int64_t N, int k, const double *__restrict__ Vt, const double *__restrict__ Y,
                                   int64_t y_stride, int64_t rows_per_cta, double *__restrict__ partial) {
    extern __shared__ double sh[];
    const int kp = (k + 7) & ~7;
    const int ld = kp + 4;
    double *sV = sh;
    double *sY = sh + 32 * ld;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int ntile = kp / 8;
    const int64_t r_begin = (int64_t)blockIdx.x * rows_per_cta;
    const int64_t r_end = min(N, r_begin + rows_per_cta);
    double acc[NMAT][16][2];
#pragma unroll
    for (int m = 0; m < NMAT; ++m)
#pragma unroll
        for (int t = 0; t < 16; ++t) acc[m][t][0] = acc[m][t][1] = 0.0;
    for (int64_t r0 = r_begin; r0 < r_end; r0 += 32) {
        const int nr = (int)min((int64_t)32, r_end - r0);
        for (int e = threadIdx.x; e < 32 * kp; e += blockDim.x) {
            const int rr = e / kp, c = e % kp;
            const bool ok = rr < nr && c < k;
            sV[rr * ld + c] = ok ? Vt[(r0 + rr) * k + c] : 0.0;
#pragma unroll
            for (int m = 0; m < NMAT; ++m) sY[m * 32 * ld + rr * ld + c] = ok ? Y[m * y_stride + (r0 + rr) * k + c] : 0.0;
        }
        __syncthreads();
        if (warp < ntile) {
#pragma unroll
            for (int kk = 0; kk < 8; ++kk) {
                const int rr = 4 * kk + (lane & 3);
                const double a = sV[rr * ld + 8 * warp + (lane >> 2)];
#pragma unroll
                for (int t = 0; t < 16; ++t) {
                    if (t < ntile) {
#pragma unroll
                        for (int m = 0; m < NMAT; ++m) {
                            const double b = sY[m * 32 * ld + rr * ld + 8 * t + (lane >> 2)];
                            asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                                         : "+d"(acc[m][t][0]), "+d"(acc[m][t][1])
                                         : "d"(a), "d"(b));
                        }
                    }
                }
            }
        }
        __syncthreads();
    }
    if (warp < ntile) {
        // lane holds D[row = lane/4][col = 2*(lane%4) + {0,1}] of tile (warp, t)
        const int ra = 8 * warp + (lane >> 2);
#pragma unroll
        for (int m = 0; m < NMAT; ++m)
#pragma unroll
            for (int t = 0; t < 16; ++t) {
                if (t < ntile) {
                    const int cb = 8 * t + 2 * (lane & 3);
                    double *P = partial + ((int64_t)m * gridDim.x + blockIdx.x) * kp * kp;
                    P[ra + (int64_t)cb * kp] = acc[m][t][0];
                    P[ra + (int64_t)(cb + 1) * kp] = acc[m][t][1];
                }
            }
    }
}

__global__ void reduce_partials_kernel(const double *__restrict__ partial, int nblk, int nmat, int k, int kp,
                                       ProjOut out) {
    const int64_t tot = (int64_t)nmat * k * k;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
        const int m = (int)(e / ((int64_t)k * k));
        const int rem = (int)(e % ((int64_t)k * k));
        const int a = rem % k, b = rem / k;
        double s = 0.0;
        for (int blk = 0; blk < nblk; ++blk) s += partial[((int64_t)m * nblk + blk) * kp * kp + a + (int64_t)b * kp];
        out.r[m][a + (int64_t)b * k] = s;
    }
}

// ---- classical Gram-Schmidt with re-orthogonalisation, one column at a time ---------------
// h = V[:, :j]^T v_j (per-CTA partials + fixed-order reduction), v_j -= V[:, :j] h; twice;
// then v_j /= ||v_j||.  Column-major V (N x k, ldv).
__global__ void gs_dots_kernel(const double *__restrict__ V, int64_t N, int64_t ldv, int j,
                               double *__restrict__ part) {
    // part[blk * (j+1) + i] = sum over this CTA's rows of V[r, i] * V[r, j], i <= j
    extern __shared__ double red[];
    const int64_t rows_per = (N + gridDim.x - 1) / gridDim.x;
    const int64_t r0 = (int64_t)blockIdx.x * rows_per, r1 = min(N, r0 + rows_per);
    const int nw = blockDim.x >> 5, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int i = 0; i <= j; ++i) {
        double s = 0.0;
        for (int64_t r = r0 + threadIdx.x; r < r1; r += blockDim.x) s = fma(V[r + i * ldv], V[r + j * ldv], s);
#pragma unroll
        for (int off = 16; off; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
        if (lane == 0) red[warp] = s;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0.0;
            for (int w = 0; w < nw; ++w) t += red[w];
            part[(int64_t)blockIdx.x * (j + 1) + i] = t;
        }
        __syncthreads();
    }
}

__global__ void gs_reduce_kernel(const double *__restrict__ part, int nblk, int j, double *__restrict__ h) {
    for (int i = threadIdx.x; i <= j; i += blockDim.x) {
        double s = 0.0;
        for (int b = 0; b < nblk; ++b) s += part[(int64_t)b * (j + 1) + i];
        h[i] = s;
    }
}

__global__ void gs_update_kernel(double *__restrict__ V, int64_t N, int64_t ldv, int j, const double *__restrict__ h) {
    extern __shared__ double hs[];
    for (int i = threadIdx.x; i < j; i += blockDim.x) hs[i] = h[i];
    __syncthreads();
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < N; r += (int64_t)gridDim.x * blockDim.x) {
        double v = V[r + j * ldv];
        for (int i = 0; i < j; ++i) v = fma(-hs[i], V[r + i * ldv], v);
        V[r + j * ldv] = v;
    }
}

__global__ void gs_scale_kernel(double *__restrict__ V, int64_t N, int64_t ldv, int j, const double *__restrict__ h) {
    const double s = 1.0 / sqrt(h[j]);
    for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < N; r += (int64_t)gridDim.x * blockDim.x)
        V[r + j * ldv] *= s;
}

// ---- host launchers -------------------------------------------------------------------------
cudaError_t launch_transpose(const double *V, int64_t N, int k, int64_t ldv, double *Vt, cudaStream_t st) {
    dim3 grid((unsigned)((N + 31) / 32), (unsigned)((k + 31) / 32)), block(32, 8);
    transpose_kernel<<<grid, block, 0, st>>>(V, N, k, ldv, Vt);
    return cudaGetLastError();
}

cudaError_t launch_spmm(int64_t N, const int64_t *rowptr, const int *colind, int base, int upper, ProjVals vals,
                        int n_mats, const double *Vt, int k, double *Y, int64_t y_stride, int sms, cudaStream_t st) {
    const int threads = 256;
    const int64_t warps_needed = N;
    int grid = (int)std::min<int64_t>((warps_needed * 32 + threads - 1) / threads, (int64_t)sms * 8);
    if (k <= 32) spmm_full_kernel<1><<<grid, threads, 0, st>>>(N, rowptr, colind, base, vals, n_mats, Vt, k, Y, y_stride);
    else if (k <= 64) spmm_full_kernel<2><<<grid, threads, 0, st>>>(N, rowptr, colind, base, vals, n_mats, Vt, k, Y, y_stride);
    else if (k <= 96) spmm_full_kernel<3><<<grid, threads, 0, st>>>(N, rowptr, colind, base, vals, n_mats, Vt, k, Y, y_stride);
    else spmm_full_kernel<4><<<grid, threads, 0, st>>>(N, rowptr, colind, base, vals, n_mats, Vt, k, Y, y_stride);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess || !upper) return e;
    spmm_upper_mirror_kernel<<<grid, threads, 0, st>>>(N, rowptr, colind, base, vals, n_mats, Vt, k, Y, y_stride);
    return cudaGetLastError();
}

size_t vty_smem_bytes(int k, int n_mats) {
    (void)n_mats;
    const int kp = (k + 7) & ~7;
    return sizeof(double) * (size_t)32 * (kp + 4) * 2;
}

cudaError_t launch_vty(int64_t N, int k, const double *Vt, const double *Y, int64_t y_stride, int n_mats,
                       int nblk, double *partial, ProjOut out, cudaStream_t st) {
    const int kp = (k + 7) & ~7;
    const int threads = 32 * (kp / 8);
    const int64_t rows_per = (N + nblk - 1) / nblk;
    const size_t smem = vty_smem_bytes(k, n_mats);
    // one launch per matrix: the k x k accumulators of one matrix already take ~100 registers
    auto kf = vty_partial_kernel<1>;
    cudaError_t e = cudaFuncSetAttribute(kf, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    for (int m = 0; m < n_mats; ++m) {
        kf<<<nblk, threads, smem, st>>>(N, k, Vt, Y + m * y_stride, y_stride,
                                        rows_per, partial + (int64_t)m * nblk * kp * kp);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    reduce_partials_kernel<<<(n_mats * k * k + 255) / 256, 256, 0, st>>>(partial, nblk, n_mats, k, kp, out);
    return cudaGetLastError();
}

cudaError_t launch_gram_schmidt(double *V, int64_t N, int k, int64_t ldv, int passes, double *part, double *h,
                                int nblk, cudaStream_t st) {
    const int threads = 256;
    int ugrid = (int)std::min<int64_t>((N + threads - 1) / threads, (int64_t)nblk * 4);
    for (int j = 0; j < k; ++j) {
        for (int p = 0; p < passes && j > 0; ++p) {
            gs_dots_kernel<<<nblk, threads, sizeof(double) * (threads / 32), st>>>(V, N, ldv, j - 1 + 1, part);
            gs_reduce_kernel<<<1, 256, 0, st>>>(part, nblk, j, h);
            gs_update_kernel<<<ugrid, threads, sizeof(double) * (size_t)j, st>>>(V, N, ldv, j, h);
        }
        gs_dots_kernel<<<nblk, threads, sizeof(double) * (threads / 32), st>>>(V, N, ldv, j, part);
        gs_reduce_kernel<<<1, 256, 0, st>>>(part, nblk, j, h);
        gs_scale_kernel<<<ugrid, threads, 0, st>>>(V, N, ldv, j, h);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

}  // namespace srom
