// FP64 complex frequency-sweep kernels: fused assembly + partial-pivot LU + solve.
//
// One CTA owns one (ROM, frequency) system at a time and pulls the next one from a work
// counter (persistent launch, largest systems first).  Two storage classes:
//   * smem   : the whole n x n matrix and the right-hand sides live in shared memory
//              (n up to ~112); unblocked right-looking LU;
//   * global : the matrix lives in a per-CTA scratch slot in global memory (L2-resident);
//              blocked right-looking LU with an NB-column panel factorised in shared
//              memory, a TRSM of the U row block and a register-tiled Schur update.
// Both reproduce, bit for bit, LAPACK zgetrf/zgetrs as restated in the oracle: pivots are
// IZAMAX (largest |re|+|im|, first index), every entry receives its updates in increasing
// pivot-column order with the same fused multiply-adds, so blocking changes no rounding.
// Reference sequence: src/analysis/KrylovROMSubstructure.cpp:1403-1453 (host, MKL) and the
// unpivoted cuBLAS batched sweep test/krylovMidsizeTest/gpu/concurrent/batchedLU/src/main.cu:223-267.
#include <climits>

#include "srom_device.cuh"
#include "sweep_kernels.h"

namespace srom {

// ------------------------------------------------------------------------------------
// Panel factorisation in shared memory (LAPACK zgetf2 order).
// P: m rows x ncols columns, leading dimension ldp.  Local row i is global row row_off+i.
// Pivots are written 1-based and global into ipiv[col_off + jj].  Row interchanges are
// applied to every panel column and, when Bs != nullptr, to the right-hand-side block.
// ------------------------------------------------------------------------------------
template <int NT>
__device__ void panel_factor(double2 *P, int ldp, int m, int ncols, int row_off, int *ipiv,
                             int col_off, int *s_info, double2 *Bs, int ldbs, int nrhs,
                             int *s_bc) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int NW = NT / 32;
    for (int jj = 0; jj < ncols; ++jj) {
        if (warp == 0) {
            double best = -1.0;
            int bi = INT_MAX;
            for (int i = jj + lane; i < m; i += 32) {
                double v = cabs1(P[i + (int64_t)jj * ldp]);
                if (v > best) {
                    best = v;
                    bi = i;
                }
            }
#pragma unroll
            for (int off = 16; off; off >>= 1) {
                double ob = __shfl_xor_sync(FULL_MASK, best, off);
                int oi = __shfl_xor_sync(FULL_MASK, bi, off);
                if (ob > best || (ob == best && oi < bi)) {
                    best = ob;
                    bi = oi;
                }
            }
            // IZAMAX starts from the first entry: a NaN there is returned as the pivot.
            double first = cabs1(P[jj + (int64_t)jj * ldp]);
            if (bi == INT_MAX || first != first) bi = jj;
            double2 piv = P[bi + (int64_t)jj * ldp];
            bool nz = (piv.x != 0.0 || piv.y != 0.0);
            if (nz) {
                if (bi != jj) {
                    if (lane == 0) {
                        P[bi + (int64_t)jj * ldp] = P[jj + (int64_t)jj * ldp];
                        P[jj + (int64_t)jj * ldp] = piv;
                    }
                    if (Bs)
                        for (int c = lane; c < nrhs; c += 32)
                            swap2(Bs[jj + (int64_t)c * ldbs], Bs[bi + (int64_t)c * ldbs]);
                }
                __syncwarp();
                double2 inv = crecip(piv);
                for (int i = jj + 1 + lane; i < m; i += 32)
                    P[i + (int64_t)jj * ldp] = cmul(P[i + (int64_t)jj * ldp], inv);
            } else if (lane == 0 && *s_info == 0) {
                *s_info = row_off + jj + 1;
            }
            if (lane == 0) {
                s_bc[0] = bi;
                s_bc[1] = nz ? 1 : 0;
                ipiv[col_off + jj] = row_off + bi + 1;
            }
        }
        __syncthreads();
        const int p = s_bc[0];
        const bool doswap = s_bc[1] && p != jj;
        if (doswap)
            for (int c = tid; c < jj; c += NT) swap2(P[jj + (int64_t)c * ldp], P[p + (int64_t)c * ldp]);
        for (int c = jj + 1 + warp; c < ncols; c += NW) {
            double2 *col = P + (int64_t)c * ldp;
            if (doswap) {
                if (lane == 0) swap2(col[jj], col[p]);
                __syncwarp();
            }
            const double2 u = col[jj];
            const double2 *lcol = P + (int64_t)jj * ldp;
            for (int i = jj + 1 + lane; i < m; i += 32) col[i] = csubmul(col[i], lcol[i], u);
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------------------------------
// zgetrs 'N' on an in-place LU (A, lda) with B (n x nrhs, ldb) in shared memory; the row
// interchanges have already been applied to B.  Forward then backward substitution in
// 32-row blocks: one warp per right-hand side solves the diagonal triangle, then all
// threads apply the block to the remaining rows.  Each entry of B still receives its
// updates in the oracle's order.
// ------------------------------------------------------------------------------------
template <int NT>
__device__ void lu_solve(const double2 *A, int64_t lda, int n, double2 *B, int ldb, int nrhs) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int NW = NT / 32;
    for (int jb = 0; jb < n; jb += 32) {
        const int je = min(jb + 32, n);
        for (int c = warp; c < nrhs; c += NW) {
            double2 *b = B + (int64_t)c * ldb;
            for (int j = jb; j < je; ++j) {
                const double2 bj = b[j];
                const int i = j + 1 + lane;
                if (i < je) b[i] = csubmul(b[i], A[i + j * lda], bj);
                __syncwarp();
            }
        }
        __syncthreads();
        const int rows = n - je;
        for (int e = tid; e < rows * nrhs; e += NT) {
            const int i = je + e % rows, c = e / rows;
            double2 *b = B + (int64_t)c * ldb;
            double2 acc = b[i];
            for (int j = jb; j < je; ++j) acc = csubmul(acc, A[i + j * lda], b[j]);
            b[i] = acc;
        }
        __syncthreads();
    }
    for (int jend = n; jend > 0; jend -= 32) {
        const int jb = max(jend - 32, 0);
        for (int c = warp; c < nrhs; c += NW) {
            double2 *b = B + (int64_t)c * ldb;
            for (int j = jend - 1; j >= jb; --j) {
                if (lane == 0) b[j] = cdiv(b[j], A[j + j * lda]);
                __syncwarp();
                const double2 bj = b[j];
                const int i = jb + lane;
                if (i < j) b[i] = csubmul(b[i], A[i + j * lda], bj);
                __syncwarp();
            }
        }
        __syncthreads();
        for (int e = tid; e < jb * nrhs; e += NT) {
            const int i = e % jb, c = e / jb;
            double2 *b = B + (int64_t)c * ldb;
            double2 acc = b[i];
            for (int j = jend - 1; j >= jb; --j) acc = csubmul(acc, A[i + j * lda], b[j]);
            b[i] = acc;
        }
        __syncthreads();
    }
}

template <int NT>
__device__ __forceinline__ int next_item(int *counter, int *s_item) {
    if (threadIdx.x == 0) *s_item = atomicAdd(counter, 1);
    __syncthreads();
    int it = *s_item;
    __syncthreads();
    return it;
}

template <int NT>
__device__ void assemble_into(double2 *A, int64_t lda, const RomDev &R, double w) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int NW = NT / 32;
    const double s = -__dmul_rn(w, w);
    for (int j = warp; j < R.n; j += NW)
        for (int i = lane; i < R.n; i += 32) {
            const int64_t e = i + (int64_t)j * R.ldk;
            A[i + j * lda] = assemble_entry(R.K[e], R.M[e], R.D, e, R.eta, s, w);
        }
}

template <int NT>
__device__ void load_rhs(double2 *B, int ldbs, const RomDev &R) {
    for (int e = threadIdx.x; e < R.n * R.r; e += NT) {
        const int i = e % R.n, c = e / R.n;
        B[i + (int64_t)c * ldbs] = R.rhs[i + (int64_t)c * R.ldb];
    }
}

template <int NT>
__device__ void store_solution(const double2 *B, int ldbs, const RomDev &R, int f) {
    double2 *X = R.X + (int64_t)f * R.n * R.r;
    for (int e = threadIdx.x; e < R.n * R.r; e += NT) {
        const int i = e % R.n, c = e / R.n;
        X[i + (int64_t)c * R.n] = B[i + (int64_t)c * ldbs];
    }
}

// ------------------------------------------------------------------------------------
// smem class: whole system in shared memory.
// Dynamic shared memory: A n x (n|1), B n x r, ipiv n ints.
// ------------------------------------------------------------------------------------
template <int NT>
__global__ void __launch_bounds__(NT) sweep_fp64_smem_kernel(const RomDev *__restrict__ roms,
                                                              const Item *__restrict__ items,
                                                              int n_items, int *counter) {
    extern __shared__ double2 smem[];
    __shared__ int s_item, s_info, s_bc[2];
    for (;;) {
        const int it = next_item<NT>(counter, &s_item);
        if (it >= n_items) break;
        const Item w = items[it];
        const RomDev R = roms[w.rom];
        const int n = R.n;
        const int lda = n | 1;
        double2 *A = smem;
        double2 *B = A + (int64_t)n * lda;
        int *ipiv = reinterpret_cast<int *>(B + (int64_t)n * R.r);
        const double om = R.omega[w.f];
        assemble_into<NT>(A, lda, R, om);
        load_rhs<NT>(B, n, R);
        if (threadIdx.x == 0) s_info = 0;
        __syncthreads();
        panel_factor<NT>(A, lda, n, n, 0, ipiv, 0, &s_info, B, n, R.r, s_bc);
        lu_solve<NT>(A, lda, n, B, n, R.r);
        store_solution<NT>(B, n, R, w.f);
        if (R.LU) {
            double2 *LU = R.LU + (int64_t)w.f * n * n;
            for (int j = threadIdx.x >> 5; j < n; j += NT / 32)
                for (int i = threadIdx.x & 31; i < n; i += 32) LU[i + (int64_t)j * n] = A[i + j * lda];
            for (int j = threadIdx.x; j < n; j += NT) R.ipiv[(int64_t)w.f * n + j] = ipiv[j];
        }
        if (threadIdx.x == 0) {
            if (R.info) R.info[w.f] = s_info;
            if (R.steps) R.steps[w.f] = 0;
            if (R.berr) R.berr[w.f] = 0.0;
        }
        __syncthreads();
    }
}

// ------------------------------------------------------------------------------------
// global class: matrix in a scratch slot (or in the caller's LU buffer).
// Dynamic shared memory: panel ldp x NB, U tile NB x TN, B n x r, ipiv n ints.
// ------------------------------------------------------------------------------------
template <int NT, int NB, int TN>
__device__ void schur_update_tile(double2 *A, int64_t lda, const double2 *P, int ldp,
                                  const double2 *Ut, int row0, int mr, int nbc, int c0, int tn,
                                  int prow0) {
    // A[row0 + i, c0 + c] -= sum_l P[prow0 + i, l] * Ut[l, c]   (i < mr, c < tn)
    constexpr int NW = NT / 32;
    constexpr int CW = TN / NW;  // columns per warp
    constexpr int RQ = 4;        // rows per lane per pass
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int cbase = warp * CW;
    for (int rb = 0; rb < mr; rb += 32 * RQ) {
        double2 acc[RQ][CW];
#pragma unroll
        for (int q = 0; q < RQ; ++q) {
            const int i = rb + lane + 32 * q;
#pragma unroll
            for (int cc = 0; cc < CW; ++cc) {
                const int c = cbase + cc;
                acc[q][cc] = (i < mr && c < tn) ? A[(row0 + i) + (int64_t)(c0 + c) * lda]
                                                : make_double2(0.0, 0.0);
            }
        }
        for (int l = 0; l < nbc; ++l) {
            double2 lv[RQ], uv[CW];
#pragma unroll
            for (int q = 0; q < RQ; ++q) {
                const int i = rb + lane + 32 * q;
                lv[q] = (i < mr) ? P[(prow0 + i) + (int64_t)l * ldp] : make_double2(0.0, 0.0);
            }
#pragma unroll
            for (int cc = 0; cc < CW; ++cc) uv[cc] = Ut[l + (cbase + cc) * NB];
#pragma unroll
            for (int q = 0; q < RQ; ++q)
#pragma unroll
                for (int cc = 0; cc < CW; ++cc) acc[q][cc] = csubmul(acc[q][cc], lv[q], uv[cc]);
        }
#pragma unroll
        for (int q = 0; q < RQ; ++q) {
            const int i = rb + lane + 32 * q;
#pragma unroll
            for (int cc = 0; cc < CW; ++cc) {
                const int c = cbase + cc;
                if (i < mr && c < tn) A[(row0 + i) + (int64_t)(c0 + c) * lda] = acc[q][cc];
            }
        }
    }
}

template <int NT, int NB, int TN>
__global__ void __launch_bounds__(NT) sweep_fp64_global_kernel(const RomDev *__restrict__ roms,
                                                                const Item *__restrict__ items,
                                                                int n_items, int *counter,
                                                                double2 *scratch,
                                                                int64_t slot_elems, int ldp) {
    extern __shared__ double2 smem[];
    __shared__ int s_item, s_info, s_bc[2];
    double2 *P = smem;
    double2 *Ut = P + (int64_t)ldp * NB;
    double2 *B = Ut + NB * TN;
    for (;;) {
        const int it = next_item<NT>(counter, &s_item);
        if (it >= n_items) break;
        const Item w = items[it];
        const RomDev R = roms[w.rom];
        const int n = R.n;
        const int64_t lda = n;
        int *ipiv = reinterpret_cast<int *>(B + (int64_t)n * R.r);
        double2 *A = R.LU ? R.LU + (int64_t)w.f * n * n : scratch + (int64_t)blockIdx.x * slot_elems;
        const double om = R.omega[w.f];
        assemble_into<NT>(A, lda, R, om);
        load_rhs<NT>(B, n, R);
        if (threadIdx.x == 0) s_info = 0;
        __syncthreads();
        for (int j0 = 0; j0 < n; j0 += NB) {
            const int nbc = min(NB, n - j0);
            const int m = n - j0;
            for (int c = threadIdx.x >> 5; c < nbc; c += NT / 32)
                for (int i = threadIdx.x & 31; i < m; i += 32)
                    P[i + (int64_t)c * ldp] = A[(j0 + i) + (j0 + c) * lda];
            __syncthreads();
            panel_factor<NT>(P, ldp, m, nbc, j0, ipiv, j0, &s_info, nullptr, 0, 0, s_bc);
            for (int c = threadIdx.x >> 5; c < nbc; c += NT / 32)
                for (int i = threadIdx.x & 31; i < m; i += 32)
                    A[(j0 + i) + (j0 + c) * lda] = P[i + (int64_t)c * ldp];
            // Row interchanges of this panel on the columns outside it and on B.
            for (int c = threadIdx.x; c < n + R.r; c += NT) {
                if (c >= j0 && c < j0 + nbc) continue;
                for (int jj = 0; jj < nbc; ++jj) {
                    const int p = ipiv[j0 + jj] - 1;
                    if (p != j0 + jj) {
                        if (c < n) swap2(A[(j0 + jj) + c * lda], A[p + c * lda]);
                        else swap2(B[(j0 + jj) + (int64_t)(c - n) * n], B[p + (int64_t)(c - n) * n]);
                    }
                }
            }
            __syncthreads();
            for (int c0 = j0 + nbc; c0 < n; c0 += TN) {
                const int tn = min(TN, n - c0);
                for (int e = threadIdx.x; e < nbc * tn; e += NT) {
                    const int l = e % nbc, c = e / nbc;
                    Ut[l + c * NB] = A[(j0 + l) + (c0 + c) * lda];
                }
                __syncthreads();
                if (threadIdx.x < tn) {
                    const int c = threadIdx.x;
                    for (int jj = 1; jj < nbc; ++jj) {
                        double2 acc = Ut[jj + c * NB];
                        for (int l = 0; l < jj; ++l) acc = csubmul(acc, P[jj + (int64_t)l * ldp], Ut[l + c * NB]);
                        Ut[jj + c * NB] = acc;
                    }
                }
                __syncthreads();
                for (int e = threadIdx.x; e < nbc * tn; e += NT) {
                    const int l = e % nbc, c = e / nbc;
                    A[(j0 + l) + (c0 + c) * lda] = Ut[l + c * NB];
                }
                schur_update_tile<NT, NB, TN>(A, lda, P, ldp, Ut, j0 + nbc, n - j0 - nbc, nbc, c0, tn, nbc);
                __syncthreads();
            }
        }
        lu_solve<NT>(A, lda, n, B, n, R.r);
        store_solution<NT>(B, n, R, w.f);
        if (threadIdx.x == 0) {
            if (R.info) R.info[w.f] = s_info;
            if (R.steps) R.steps[w.f] = 0;
            if (R.berr) R.berr[w.f] = 0.0;
        }
        if (R.ipiv)
            for (int j = threadIdx.x; j < n; j += NT) R.ipiv[(int64_t)w.f * n + j] = ipiv[j];
        __syncthreads();
    }
}

// ------------------------------------------------------------------------------------
// Host-side launch helpers
// ------------------------------------------------------------------------------------
constexpr int FP64_NT = 256;
constexpr int FP64_NB = 16;
constexpr int FP64_TN = 32;

size_t fp64_smem_bytes(int n, int r) {
    const size_t lda = (size_t)(n | 1);
    return sizeof(double2) * (lda * n + (size_t)n * r) + sizeof(int) * (size_t)n;
}

size_t fp64_global_smem_bytes(int n_max, int r_max) {
    const size_t ldp = (size_t)(n_max | 1);
    return sizeof(double2) * (ldp * FP64_NB + FP64_NB * FP64_TN + (size_t)n_max * r_max) +
           sizeof(int) * (size_t)n_max;
}

cudaError_t launch_fp64_smem(const RomDev *roms, const Item *items, int n_items, int *counter,
                             size_t smem, int grid, cudaStream_t st) {
    auto k = sweep_fp64_smem_kernel<FP64_NT>;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k<<<grid, FP64_NT, smem, st>>>(roms, items, n_items, counter);
    return cudaGetLastError();
}

int fp64_smem_blocks_per_sm(size_t smem) {
    int b = 0;
    auto k = sweep_fp64_smem_kernel<FP64_NT>;
    if (cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess) return 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, k, FP64_NT, smem) != cudaSuccess) return 0;
    return b;
}

cudaError_t launch_fp64_global(const RomDev *roms, const Item *items, int n_items, int *counter,
                               double2 *scratch, int64_t slot_elems, int n_max, int r_max,
                               int grid, cudaStream_t st) {
    auto k = sweep_fp64_global_kernel<FP64_NT, FP64_NB, FP64_TN>;
    const size_t smem = fp64_global_smem_bytes(n_max, r_max);
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k<<<grid, FP64_NT, smem, st>>>(roms, items, n_items, counter, scratch, slot_elems, n_max | 1);
    return cudaGetLastError();
}

}  // namespace srom
