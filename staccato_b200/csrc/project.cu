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
constexpr int PRJ_WIN = 128;  // basis columns per SpMM pass and per side of a V^T Y window

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
// A warp takes three consecutive rows.  FE matrices numbered node by node give the three
// DOF rows of a node the same column pattern; when the warp finds that (equal lengths and
// equal column lists, checked with a warp vote), every gathered Vt row feeds all three rows
// and all matrices, cutting the Vt gathers -- the dominant L2 traffic -- by three.  Otherwise
// the rows are processed one after the other.  The column indices and values of a row are
// staged 32 entries at a time in the warp's shared-memory slot (coalesced loads), so that
// the Vt gathers of SPMM_DEPTH consecutive entries are independent loads in flight together.
// Every Y entry is the sequential FMA chain over the row's entries in storage order.
constexpr int SPMM_THREADS = 256;
constexpr int SPMM_WARPS = SPMM_THREADS / 32;
constexpr int SPMM_DEPTH = 4;

struct SpmmStage {
    int col[32];
    double val[3 * PRJ_MAX_MATS][32];
};

// Column window: the k (<= 32 CPL) basis columns starting at Vt (row stride ldv) into Y (row
// stride ldy); a basis wider than 128 columns is projected window by window.
template <int CPL, int NMAT, int NR>
__device__ __forceinline__ void spmm_rows(int64_t row, const int64_t *__restrict__ rowptr,
                                          const int *__restrict__ colind, int base, const ProjVals &vals,
                                          const double *__restrict__ Vt, int k, int ldv, double *__restrict__ Y,
                                          int ldy, int64_t y_stride, int lane, SpmmStage &st) {
    const int64_t e0 = rowptr[row] - base, e1 = rowptr[row + 1] - base;
    int64_t off[NR];
#pragma unroll
    for (int r = 0; r < NR; ++r) off[r] = (rowptr[row + r] - base) - e0;
    double acc[NR][NMAT][CPL];
#pragma unroll
    for (int r = 0; r < NR; ++r)
#pragma unroll
        for (int m = 0; m < NMAT; ++m)
#pragma unroll
            for (int q = 0; q < CPL; ++q) acc[r][m][q] = 0.0;
    for (int64_t c0 = e0; c0 < e1; c0 += 32) {
        const int cnt = (int)min((int64_t)32, e1 - c0);
        __syncwarp();
        if (lane < cnt) {
            st.col[lane] = colind[c0 + lane] - base;
#pragma unroll
            for (int r = 0; r < NR; ++r)
#pragma unroll
                for (int m = 0; m < NMAT; ++m) st.val[r * NMAT + m][lane] = vals.v[m][c0 + lane + off[r]];
        }
        __syncwarp();
        int j = 0;
        for (; j + SPMM_DEPTH <= cnt; j += SPMM_DEPTH) {
            double v[SPMM_DEPTH][CPL];
#pragma unroll
            for (int u = 0; u < SPMM_DEPTH; ++u) {
                const double *vr = Vt + (int64_t)st.col[j + u] * ldv;
#pragma unroll
                for (int q = 0; q < CPL; ++q) {
                    const int c = lane + 32 * q;
                    v[u][q] = c < k ? vr[c] : 0.0;
                }
            }
#pragma unroll
            for (int u = 0; u < SPMM_DEPTH; ++u)
#pragma unroll
                for (int r = 0; r < NR; ++r)
#pragma unroll
                    for (int m = 0; m < NMAT; ++m) {
                        const double a = st.val[r * NMAT + m][j + u];
#pragma unroll
                        for (int q = 0; q < CPL; ++q) acc[r][m][q] = fma(a, v[u][q], acc[r][m][q]);
                    }
        }
        for (; j < cnt; ++j) {
            const double *vr = Vt + (int64_t)st.col[j] * ldv;
#pragma unroll
            for (int q = 0; q < CPL; ++q) {
                const int c = lane + 32 * q;
                const double v = c < k ? vr[c] : 0.0;
#pragma unroll
                for (int r = 0; r < NR; ++r)
#pragma unroll
                    for (int m = 0; m < NMAT; ++m) acc[r][m][q] = fma(st.val[r * NMAT + m][j], v, acc[r][m][q]);
            }
        }
    }
#pragma unroll
    for (int r = 0; r < NR; ++r)
#pragma unroll
        for (int m = 0; m < NMAT; ++m)
#pragma unroll
            for (int q = 0; q < CPL; ++q) {
                const int c = lane + 32 * q;
                if (c < k) Y[m * y_stride + (row + r) * ldy + c] = acc[r][m][q];
            }
}

template <int CPL, int NMAT>
__global__ void __launch_bounds__(SPMM_THREADS) spmm_full_kernel(int64_t N, const int64_t *__restrict__ rowptr,
                                                                 const int *__restrict__ colind, int base,
                                                                 ProjVals vals, const double *__restrict__ Vt, int k,
                                                                 int ldv, double *__restrict__ Y, int ldy,
                                                                 int64_t y_stride) {
    __shared__ SpmmStage stage[SPMM_WARPS];
    const int lane = threadIdx.x & 31;
    SpmmStage &st = stage[threadIdx.x >> 5];
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarp = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t r0 = warp * 3; r0 < N; r0 += nwarp * 3) {
        const int nr = (int)min((int64_t)3, N - r0);
        bool same = nr == 3;
        if (same) {
            const int64_t a0 = rowptr[r0], a1 = rowptr[r0 + 1], a2 = rowptr[r0 + 2], a3 = rowptr[r0 + 3];
            const int64_t len = a1 - a0;
            same = (a2 - a1) == len && (a3 - a2) == len;
            // the trip count is warp-uniform, so every lane takes part in every vote
            for (int64_t t0 = 0; same && t0 < len; t0 += 32) {
                const int64_t t = t0 + lane;
                bool eq = true;
                if (t < len) {
                    const int c0 = colind[a0 - base + t];
                    eq = c0 == colind[a1 - base + t] && c0 == colind[a2 - base + t];
                }
                same = __all_sync(0xffffffffu, eq);
            }
        }
        if (same) {
            spmm_rows<CPL, NMAT, 3>(r0, rowptr, colind, base, vals, Vt, k, ldv, Y, ldy, y_stride, lane, st);
        } else {
            for (int r = 0; r < nr; ++r)
                spmm_rows<CPL, NMAT, 1>(r0 + r, rowptr, colind, base, vals, Vt, k, ldv, Y, ldy, y_stride, lane, st);
        }
    }
}

// grid = at most one wave of resident CTAs (the row loop is grid-strided)
template <int CPL, int NMAT>
static void spmm_full_launch(int grid, cudaStream_t st, int64_t N, const int64_t *rowptr, const int *colind,
                             int base, const ProjVals &vals, const double *Vt, int k, int ldv, double *Y, int ldy,
                             int64_t y_stride) {
    int per_sm = 0, dev = 0, sms = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, spmm_full_kernel<CPL, NMAT>, SPMM_THREADS, 0) ==
            cudaSuccess &&
        cudaGetDevice(&dev) == cudaSuccess &&
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess && per_sm > 0)
        grid = std::min(grid, per_sm * sms);
    spmm_full_kernel<CPL, NMAT><<<grid, SPMM_THREADS, 0, st>>>(N, rowptr, colind, base, vals, Vt, k, ldv, Y, ldy,
                                                               y_stride);
}

template <int CPL>
static void launch_spmm_full(int grid, cudaStream_t st, int64_t N, const int64_t *rowptr, const int *colind,
                             int base, const ProjVals &vals, int n_mats, const double *Vt, int k, int ldv, double *Y,
                             int ldy, int64_t y_stride) {
    if (n_mats == 1) spmm_full_launch<CPL, 1>(grid, st, N, rowptr, colind, base, vals, Vt, k, ldv, Y, ldy, y_stride);
    else if (n_mats == 2) spmm_full_launch<CPL, 2>(grid, st, N, rowptr, colind, base, vals, Vt, k, ldv, Y, ldy, y_stride);
    else spmm_full_launch<CPL, 3>(grid, st, N, rowptr, colind, base, vals, Vt, k, ldv, Y, ldy, y_stride);
}

// Upper-triangle storage of a symmetric matrix (the reference's CSR,
// src/tools/MathLibrary.cpp:502-507): the mirrored entries (j, i), j != i, are added with
// FP64 atomics after the row pass above has written the stored half.
__global__ void spmm_upper_mirror_kernel(int64_t N, const int64_t *__restrict__ rowptr,
                                         const int *__restrict__ colind, int base, ProjVals vals, int n_mats,
                                         const double *__restrict__ Vt, int k, int ldv, double *__restrict__ Y,
                                         int ldy, int64_t y_stride) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarp = ((int64_t)gridDim.x * blockDim.x) >> 5;
    for (int64_t row = warp; row < N; row += nwarp) {
        const int64_t e0 = rowptr[row] - base, e1 = rowptr[row + 1] - base;
        for (int64_t e = e0; e < e1; ++e) {
            const int64_t col = colind[e] - base;
            if (col == row) continue;
            for (int c = lane; c < k; c += 32) {
                const double v = Vt[row * ldv + c];
                for (int m = 0; m < n_mats; ++m) atomicAdd(&Y[m * y_stride + col * ldy + c], vals.v[m][e] * v);
            }
        }
    }
}

// ---- R_m partial = Vt[rows]^T Y_m[rows] on FP64 tensor cores ------------------------------
// One launch covers nm matrices and one window of R: ka rows (basis columns of Vt, row stride
// ldv) by kb columns (columns of Y_m, row stride ldy), both <= 128.  Warp w owns matrix
// w / nband and the 8-row band w % nband of the window (nband = kap / 8), 8x8 tiles across it.
// The rows of Vt and of the nm Y's are staged 32 at a time in shared memory (leading
// dimension padded by 4 keeps the fragment loads free of bank conflicts); the Vt chunk is
// staged once for all nm matrices, and the chunks are double-buffered with cp.async so the
// loads of chunk c + 1 overlap the MMAs of chunk c.  Each CTA takes a contiguous range of
// chunks and writes a private kap x kbp partial.
__device__ __forceinline__ void cp_async8(double *dst, const double *src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src));
}

struct VtyWindow {
    const double *Vt;  // first basis column of the window's rows
    int ka, ldv;
    const double *Y;   // first column of the window's columns (matrix 0)
    int kb, ldy;
    int64_t y_stride;  // between matrices
};

template <int TMAX, int MAXT>
__global__ void __launch_bounds__(MAXT) vty_partial_kernel(int64_t N, VtyWindow w, int nm, int64_t chunks_per_cta,
                                                           double *__restrict__ partial) {
    extern __shared__ double sh[];
    const int kap = (w.ka + 7) & ~7, kbp = (w.kb + 7) & ~7;
    const int lda = kap + 4, ldb = kbp + 4;
    const int nband = kap / 8, ntile = kbp / 8;
    const int a_sz = 32 * lda, b_sz = 32 * ldb;
    const int stage = a_sz + nm * b_sz;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int mloc = warp / nband, band = warp % nband;
    const bool active = mloc < nm;
    const int64_t n_chunks = (N + 31) / 32;
    const int64_t c_begin = (int64_t)blockIdx.x * chunks_per_cta;
    const int64_t c_end = min(n_chunks, c_begin + chunks_per_cta);
    const int a_tot = 32 * kap, total = a_tot + nm * 32 * kbp;

    auto issue = [&](int64_t ch, int buf) {
        double *dst0 = sh + buf * stage;
        const int64_t r0 = ch * 32;
        const int nr = (int)min((int64_t)32, N - r0);
        for (int e = threadIdx.x; e < total; e += blockDim.x) {
            double *dst;
            const double *src = nullptr;
            if (e < a_tot) {
                const int rr = e / kap, c = e - rr * kap;
                dst = dst0 + rr * lda + c;
                if (rr < nr && c < w.ka) src = w.Vt + (r0 + rr) * w.ldv + c;
            } else {
                const int eb = e - a_tot, mat = eb / (32 * kbp), rem = eb - mat * 32 * kbp;
                const int rr = rem / kbp, c = rem - rr * kbp;
                dst = dst0 + a_sz + mat * b_sz + rr * ldb + c;
                if (rr < nr && c < w.kb) src = w.Y + mat * w.y_stride + (r0 + rr) * w.ldy + c;
            }
            if (src) cp_async8(dst, src);
            else *dst = 0.0;
        }
        asm volatile("cp.async.commit_group;");
    };

    double acc[TMAX][2];
#pragma unroll
    for (int t = 0; t < TMAX; ++t) acc[t][0] = acc[t][1] = 0.0;
    if (c_begin < c_end) issue(c_begin, 0);
    for (int64_t ch = c_begin; ch < c_end; ++ch) {
        const int buf = (int)((ch - c_begin) & 1);
        if (ch + 1 < c_end) {
            issue(ch + 1, buf ^ 1);
            asm volatile("cp.async.wait_group 1;");
        } else {
            asm volatile("cp.async.wait_group 0;");
        }
        __syncthreads();
        if (active) {
            const double *sV = sh + buf * stage;
            const double *sY = sV + a_sz + mloc * b_sz;
#pragma unroll
            for (int kk = 0; kk < 8; ++kk) {
                const int rr = 4 * kk + (lane & 3);
                const double a = sV[rr * lda + 8 * band + (lane >> 2)];
#pragma unroll
                for (int t = 0; t < TMAX; ++t) {
                    if (t < ntile) {
                        const double b = sY[rr * ldb + 8 * t + (lane >> 2)];
                        asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                                     : "+d"(acc[t][0]), "+d"(acc[t][1])
                                     : "d"(a), "d"(b));
                    }
                }
            }
        }
        __syncthreads();
    }
    if (active) {
        // lane holds D[row = lane/4][col = 2*(lane%4) + {0,1}] of tile (band, t)
        const int ra = 8 * band + (lane >> 2);
        double *P = partial + ((int64_t)mloc * gridDim.x + blockIdx.x) * kap * kbp;
#pragma unroll
        for (int t = 0; t < TMAX; ++t) {
            if (t < ntile) {
                const int cb = 8 * t + 2 * (lane & 3);
                P[ra + (int64_t)cb * kap] = acc[t][0];
                P[ra + (int64_t)(cb + 1) * kap] = acc[t][1];
            }
        }
    }
}

// out.r[m][a + b * ldr] = sum over the CTA partials, in CTA order (deterministic)
__global__ void reduce_partials_kernel(const double *__restrict__ partial, int nblk, int nmat, int ka, int kb,
                                       int kap, int kbp, ProjOut out, int ldr) {
    const int64_t tot = (int64_t)nmat * ka * kb;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
        const int m = (int)(e / ((int64_t)ka * kb));
        const int rem = (int)(e % ((int64_t)ka * kb));
        const int a = rem % ka, b = rem / ka;
        double s = 0.0;
        for (int blk = 0; blk < nblk; ++blk) s += partial[((int64_t)m * nblk + blk) * kap * kbp + a + (int64_t)b * kap];
        out.r[m][a + (int64_t)b * ldr] = s;
    }
}

// ---- block Gram-Schmidt with re-orthogonalisation --------------------------------------
// The columns of V (column-major, N x k, ldv) are taken in panels P of GS_B columns.  One pass
// over a panel with the orthonormal columns Q = V[:, :j0] before it:
//     C = [Q P]^T P                 (one reduction: H = Q^T P on top, G = P^T P below)
//     R^T R = G - H^T H             (Cholesky; the Gram matrix of P - Q H by Pythagoras)
//     P <- (P - Q H) R^-1
// and `passes` passes are made (two keep the basis orthonormal to rounding level).  This is
// the reference's block scheme -- block projection against V repeated, then an orthonormal
// basis of the block (KrylovROMSubstructure.cpp:433-475, :513-534) -- with the QR of the block
// taken through its Gram matrix so that every pass is one reduction and one row update.
constexpr int GS_B = 32;        // panel width
constexpr int GS_WIN = 128;     // columns of [Q P] per reduction launch (16 bands of 8)
constexpr int GS_LDR = 36;      // staged column stride (32 rows + 4: conflict-free fragments)
constexpr int GS_THREADS = 512;
constexpr int GS_HCHUNK = 128;  // rows of H staged per round of the row update

// part[blk][x0 + i][c] = sum over this CTA's rows of V[r, x0 + i] * V[r, j0 + c]
// (i < w, c < b), on the FP64 tensor cores; chunks of 32 rows double-buffered with cp.async.
__global__ void __launch_bounds__(GS_THREADS) gs_gram_kernel(const double *__restrict__ V, int64_t N, int64_t ldv,
                                                             int x0, int w, int j0, int b, int rows_c,
                                                             int64_t chunks_per_cta, double *__restrict__ part) {
    extern __shared__ double sh[];
    const int wp = (w + 7) & ~7, bp = (b + 7) & ~7;
    const int stage = (wp + bp) * GS_LDR;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nband = wp / 8, ntile = bp / 8;
    const int64_t n_chunks = (N + 31) / 32;
    const int64_t c_begin = (int64_t)blockIdx.x * chunks_per_cta;
    const int64_t c_end = min(n_chunks, c_begin + chunks_per_cta);
    const int total = (wp + bp) * 32;

    auto issue = [&](int64_t ch, int buf) {
        double *dst0 = sh + buf * stage;
        const int64_t r0 = ch * 32;
        const int nr = (int)min((int64_t)32, N - r0);
        for (int e = threadIdx.x; e < total; e += blockDim.x) {
            const int col = e >> 5, rr = e & 31;  // staged column col: X for col < wp, P after
            const bool isx = col < wp;
            const int cc = isx ? col : col - wp;
            const bool ok = rr < nr && (isx ? cc < w : cc < b);
            double *dst = dst0 + col * GS_LDR + rr;
            if (ok) {
                const int64_t vc = isx ? x0 + cc : j0 + cc;
                const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
                asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(V + r0 + rr + vc * ldv));
            } else {
                *dst = 0.0;
            }
        }
        asm volatile("cp.async.commit_group;");
    };

    double acc[4][2];
#pragma unroll
    for (int t = 0; t < 4; ++t) acc[t][0] = acc[t][1] = 0.0;
    if (c_begin < c_end) issue(c_begin, 0);
    for (int64_t ch = c_begin; ch < c_end; ++ch) {
        const int buf = (int)((ch - c_begin) & 1);
        if (ch + 1 < c_end) {
            issue(ch + 1, buf ^ 1);
            asm volatile("cp.async.wait_group 1;");
        } else {
            asm volatile("cp.async.wait_group 0;");
        }
        __syncthreads();
        if (warp < nband) {
            const double *sX = sh + buf * stage;
            const double *sP = sX + wp * GS_LDR;
#pragma unroll
            for (int kk = 0; kk < 8; ++kk) {
                const int rr = 4 * kk + (lane & 3);
                const double a = sX[(8 * warp + (lane >> 2)) * GS_LDR + rr];
#pragma unroll
                for (int t = 0; t < 4; ++t) {
                    if (t < ntile) {
                        const double bv = sP[(8 * t + (lane >> 2)) * GS_LDR + rr];
                        asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
                                     : "+d"(acc[t][0]), "+d"(acc[t][1])
                                     : "d"(a), "d"(bv));
                    }
                }
            }
        }
        __syncthreads();
    }
    if (warp < nband) {
        const int i = x0 + 8 * warp + (lane >> 2);
        double *P = part + (int64_t)blockIdx.x * rows_c * GS_B;
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            const int c = 8 * t + 2 * (lane & 3);
            if (i < rows_c) {  // tiles past b hold zeros
                P[(int64_t)i * GS_B + c] = acc[t][0];
                P[(int64_t)i * GS_B + c + 1] = acc[t][1];
            }
        }
    }
}

// C[i][c] = sum_blk part[blk][i][c] in CTA order (deterministic)
__global__ void gs_reduce_kernel(const double *__restrict__ part, int nblk, int rows_c, double *__restrict__ Cm) {
    const int64_t tot = (int64_t)rows_c * GS_B;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int blk = 0; blk < nblk; ++blk) s += part[(int64_t)blk * tot + e];
        Cm[e] = s;
    }
}

// One CTA: G' = G - H^T H, Cholesky R^T R = G', Rinv = R^-1 (upper), written to rinv[a][c].
__global__ void gs_chol_kernel(const double *__restrict__ Cm, int j0, int b, double *__restrict__ rinv) {
    __shared__ double G[GS_B][GS_B + 1];
    __shared__ double R[GS_B][GS_B + 1];
    for (int e = threadIdx.x; e < GS_B * GS_B; e += blockDim.x) {
        const int a = e / GS_B, c = e % GS_B;
        double g = 0.0;
        if (a < b && c < b) {
            g = Cm[(int64_t)(j0 + a) * GS_B + c];
            double s = 0.0;
            for (int i = 0; i < j0; ++i) s = fma(Cm[(int64_t)i * GS_B + a], Cm[(int64_t)i * GS_B + c], s);
            g -= s;
        }
        G[a][c] = g;
        R[a][c] = 0.0;
    }
    __syncthreads();
    // right-looking Cholesky of the symmetric G' (upper factor R, row by row)
    for (int j = 0; j < b; ++j) {
        const double d = sqrt(G[j][j]);
        __syncthreads();
        for (int c = j + threadIdx.x; c < b; c += blockDim.x) R[j][c] = c == j ? d : G[j][c] / d;
        __syncthreads();
        for (int e = threadIdx.x; e < (b - j - 1) * (b - j - 1); e += blockDim.x) {
            const int a = j + 1 + e / (b - j - 1), c = j + 1 + e % (b - j - 1);
            G[a][c] = fma(-R[j][a], R[j][c], G[a][c]);
        }
        __syncthreads();
    }
    // Rinv column c by back substitution: R x = e_c, one thread per column
    for (int c = threadIdx.x; c < GS_B; c += blockDim.x) {
        double x[GS_B];
#pragma unroll
        for (int i = 0; i < GS_B; ++i) x[i] = 0.0;
        if (c < b) {
            for (int i = c; i >= 0; --i) {
                double s = i == c ? 1.0 : 0.0;
                for (int l = i + 1; l <= c; ++l) s = fma(-R[i][l], x[l], s);
                x[i] = s / R[i][i];
            }
        }
        for (int i = 0; i < GS_B; ++i) rinv[i * GS_B + c] = x[i];
    }
}

// Two threads per row, 16 panel columns each: p <- (p - q H) Rinv with q = V[r, :j0] and
// p = V[r, j0:j0+b].  Lane l of a warp takes row (l & 15) and columns 16 (l >> 4) ...; the
// upper half reads the lower half's p through shuffles for the triangular product.
constexpr int GS_HALF = GS_B / 2;
__global__ void __launch_bounds__(256, 2) gs_update_kernel(double *__restrict__ V, int64_t N, int64_t ldv, int j0, int b,
                                                        const double *__restrict__ Cm, const double *__restrict__ rinv) {
    __shared__ __align__(16) double Hs[GS_HCHUNK * GS_B];
    __shared__ __align__(16) double Rs[GS_B * GS_B];
    for (int e = threadIdx.x; e < GS_B * GS_B; e += blockDim.x) Rs[e] = rinv[e];
    const int lane = threadIdx.x & 31, half = lane >> 4;
    const int64_t r = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x - lane) / 2 + (lane & 15);
    const bool live = r < N;
    const int cb = half * GS_HALF;
    double p[GS_HALF];
#pragma unroll
    for (int c = 0; c < GS_HALF; ++c) p[c] = (live && cb + c < b) ? V[r + (int64_t)(j0 + cb + c) * ldv] : 0.0;
    for (int i0 = 0; i0 < j0; i0 += GS_HCHUNK) {
        const int ni = min(GS_HCHUNK, j0 - i0);
        __syncthreads();
        for (int e = threadIdx.x; e < ni * GS_B; e += blockDim.x) Hs[e] = Cm[(int64_t)i0 * GS_B + e];
        __syncthreads();
        if (live) {
#pragma unroll 4
            for (int i = 0; i < ni; ++i) {
                const double q = V[r + (int64_t)(i0 + i) * ldv];
                const double2 *h2 = reinterpret_cast<const double2 *>(Hs + i * GS_B + cb);
#pragma unroll
                for (int c2 = 0; c2 < GS_HALF / 2; ++c2) {
                    const double2 hv = h2[c2];
                    p[2 * c2] = fma(-q, hv.x, p[2 * c2]);
                    p[2 * c2 + 1] = fma(-q, hv.y, p[2 * c2 + 1]);
                }
            }
        }
    }
    __syncthreads();
    // p <- p Rinv (upper): column c takes the row's p[0..c]
    double o[GS_HALF];
#pragma unroll
    for (int u = 0; u < GS_HALF; ++u) o[u] = 0.0;
#pragma unroll
    for (int i = 0; i < GS_HALF; ++i) {
        const double lo = __shfl_sync(0xffffffffu, p[i], lane & 15);  // the row's p[i], i < 16
#pragma unroll
        for (int u = 0; u < GS_HALF; ++u) {
            if (half == 0) {
                if (i <= u) o[u] = fma(lo, Rs[i * GS_B + u], o[u]);
            } else {
                o[u] = fma(lo, Rs[i * GS_B + GS_HALF + u], o[u]);
            }
        }
    }
    if (half == 1) {
#pragma unroll
        for (int i = 0; i < GS_HALF; ++i)
#pragma unroll
            for (int u = 0; u < GS_HALF; ++u)
                if (i <= u) o[u] = fma(p[i], Rs[(GS_HALF + i) * GS_B + GS_HALF + u], o[u]);
    }
    if (!live) return;
#pragma unroll
    for (int c = 0; c < GS_HALF; ++c)
        if (cb + c < b) V[r + (int64_t)(j0 + cb + c) * ldv] = o[c];
}

// ---- complex projection R = Z^H A V through the real kernels ------------------------------
// With A = Ar + i Ai and the basis stored as the real N x 2k rows [Re V | Im V], the real SpMM
// over the two value arrays (Ar, Ai) gives P_r = Ar [Vr | Vi] and P_i = Ai [Vr | Vi]; then
// Y = A V has Re Y = Ar Vr - Ai Vi and Im Y = Ar Vi + Ai Vr (combined in place into P_r's rows
// as [Re Y | Im Y]), and the real V^T Y kernel on W = [Re Z | Im Z] gives G = W^T [Re Y | Im Y],
// whose four k x k blocks combine into Z^H Y = (Zr^T Yr + Zi^T Yi) + i (Zr^T Yi - Zi^T Yr).

// V (complex, column-major, ldv) -> Wt (real, row-major N x 2k: [Re V(row) | Im V(row)])
__global__ void transpose_split_kernel(const double2 *__restrict__ V, int64_t N, int k, int64_t ldv,
                                       double *__restrict__ Wt) {
    __shared__ double2 t[32][33];
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
        if (r < N && c < k) {
            const double2 v = t[threadIdx.x][y];
            Wt[r * 2 * k + c] = v.x;
            Wt[r * 2 * k + k + c] = v.y;
        }
    }
}

// complex values -> separate real and imaginary arrays
__global__ void split_values_kernel(const double2 *__restrict__ a, int64_t nnz, double *__restrict__ re,
                                    double *__restrict__ im) {
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < nnz; e += (int64_t)gridDim.x * blockDim.x) {
        const double2 v = a[e];
        re[e] = v.x;
        im[e] = v.y;
    }
}

// rows of P_r = [Ar Vr | Ar Vi] and P_i = [Ai Vr | Ai Vi] -> rows of P_r = [Re Y | Im Y]
__global__ void combine_y_kernel(double *__restrict__ Pr, const double *__restrict__ Pi, int64_t N, int k) {
    const int64_t tot = N * k;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t r = e / k;
        const int c = (int)(e % k);
        double *pr = Pr + r * 2 * k;
        const double *pi = Pi + r * 2 * k;
        const double yr = pr[c] - pi[k + c];
        const double yi = pr[k + c] + pi[c];
        pr[c] = yr;
        pr[k + c] = yi;
    }
}

// G (2k x 2k, column-major) -> R (k x k complex, column-major)
__global__ void combine_r_kernel(const double *__restrict__ G, int k, double2 *__restrict__ R) {
    const int k2 = 2 * k;
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < k * k; e += gridDim.x * blockDim.x) {
        const int a = e % k, b = e / k;
        const double re = G[a + (int64_t)b * k2] + G[(k + a) + (int64_t)(k + b) * k2];
        const double im = G[a + (int64_t)(k + b) * k2] - G[(k + a) + (int64_t)b * k2];
        R[a + (int64_t)b * k] = make_double2(re, im);
    }
}

cudaError_t launch_transpose_split(const double2 *V, int64_t N, int k, int64_t ldv, double *Wt, cudaStream_t st) {
    dim3 grid((unsigned)((N + 31) / 32), (unsigned)((k + 31) / 32)), block(32, 8);
    transpose_split_kernel<<<grid, block, 0, st>>>(V, N, k, ldv, Wt);
    return cudaGetLastError();
}

cudaError_t launch_split_values(const double2 *a, int64_t nnz, double *re, double *im, int sms, cudaStream_t st) {
    const int grid = (int)std::min<int64_t>((nnz + 255) / 256, (int64_t)sms * 8);
    if (grid > 0) split_values_kernel<<<grid, 256, 0, st>>>(a, nnz, re, im);
    return cudaGetLastError();
}

cudaError_t launch_combine_y(double *Pr, const double *Pi, int64_t N, int k, int sms, cudaStream_t st) {
    const int grid = (int)std::min<int64_t>((N * k + 255) / 256, (int64_t)sms * 8);
    if (grid > 0) combine_y_kernel<<<grid, 256, 0, st>>>(Pr, Pi, N, k);
    return cudaGetLastError();
}

cudaError_t launch_combine_r(const double *G, int k, double2 *R, cudaStream_t st) {
    combine_r_kernel<<<(k * k + 255) / 256, 256, 0, st>>>(G, k, R);
    return cudaGetLastError();
}

// ---- host launchers -------------------------------------------------------------------------
cudaError_t launch_transpose(const double *V, int64_t N, int k, int64_t ldv, double *Vt, cudaStream_t st) {
    dim3 grid((unsigned)((N + 31) / 32), (unsigned)((k + 31) / 32)), block(32, 8);
    transpose_kernel<<<grid, block, 0, st>>>(V, N, k, ldv, Vt);
    return cudaGetLastError();
}

cudaError_t launch_spmm(int64_t N, const int64_t *rowptr, const int *colind, int base, int upper, ProjVals vals,
                        int n_mats, const double *Vt, int k, double *Y, int64_t y_stride, int sms, cudaStream_t st) {
    const int threads = SPMM_THREADS;
    const int64_t warps_needed = (N + 2) / 3;
    int grid = (int)std::min<int64_t>((warps_needed * 32 + threads - 1) / threads, (int64_t)sms * 8);
    // window by window (PRJ_WIN columns of the basis at a time), each into its columns of Y
    for (int j0 = 0; j0 < k; j0 += PRJ_WIN) {
        const int kw = std::min(PRJ_WIN, k - j0);
        const double *Vw = Vt + j0;
        double *Yw = Y + j0;
        if (kw <= 32) launch_spmm_full<1>(grid, st, N, rowptr, colind, base, vals, n_mats, Vw, kw, k, Yw, k, y_stride);
        else if (kw <= 64) launch_spmm_full<2>(grid, st, N, rowptr, colind, base, vals, n_mats, Vw, kw, k, Yw, k, y_stride);
        else if (kw <= 96) launch_spmm_full<3>(grid, st, N, rowptr, colind, base, vals, n_mats, Vw, kw, k, Yw, k, y_stride);
        else launch_spmm_full<4>(grid, st, N, rowptr, colind, base, vals, n_mats, Vw, kw, k, Yw, k, y_stride);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
        if (upper) {
            spmm_upper_mirror_kernel<<<grid, threads, 0, st>>>(N, rowptr, colind, base, vals, n_mats, Vw, kw, k, Yw, k,
                                                               y_stride);
            if ((e = cudaGetLastError()) != cudaSuccess) return e;
        }
    }
    return cudaSuccess;
}

// matrices per launch: 24 warps at most (768 threads, <= 85 registers a thread) for windows
// up to 12 tiles wide, 16 warps (512 threads) for wider ones
static int vty_group(int ka, int kb, int n_mats) {
    const int nband = ((ka + 7) & ~7) / 8, ntile = ((kb + 7) & ~7) / 8;
    return std::max(1, std::min(n_mats, (ntile > 12 ? 16 : 24) / nband));
}

size_t vty_partial_doubles(int k, int n_mats, int nblk) {
    const int kp = (std::min(k, PRJ_WIN) + 7) & ~7;
    return (size_t)nblk * n_mats * kp * kp;
}

template <int TMAX, int MAXT>
static cudaError_t vty_launch(int64_t N, const VtyWindow &w, int nm, int nblk, double *partial, cudaStream_t st) {
    const int kap = (w.ka + 7) & ~7, kbp = (w.kb + 7) & ~7;
    const int threads = 32 * nm * (kap / 8);
    const size_t smem = sizeof(double) * (size_t)2 * 32 * ((kap + 4) + (size_t)nm * (kbp + 4));
    auto kf = vty_partial_kernel<TMAX, MAXT>;
    cudaError_t e = cudaFuncSetAttribute(kf, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const int64_t n_chunks = (N + 31) / 32;
    const int64_t per = (n_chunks + nblk - 1) / nblk;
    kf<<<nblk, threads, smem, st>>>(N, w, nm, per, partial);
    return cudaGetLastError();
}

// R_m = Vt^T Y_m (k x k, leading dimension k) window by window: PRJ_WIN x PRJ_WIN blocks of R,
// each one DMMA pass over the rows plus a deterministic reduction into its block.
cudaError_t launch_vty(int64_t N, int k, const double *Vt, const double *Y, int64_t y_stride, int n_mats,
                       int nblk, double *partial, ProjOut out, cudaStream_t st) {
    for (int i0 = 0; i0 < k; i0 += PRJ_WIN) {
        const int ka = std::min(PRJ_WIN, k - i0);
        const int kap = (ka + 7) & ~7;
        for (int j0 = 0; j0 < k; j0 += PRJ_WIN) {
            const int kb = std::min(PRJ_WIN, k - j0);
            const int kbp = (kb + 7) & ~7, ntile = kbp / 8;
            const int group = vty_group(ka, kb, n_mats);
            for (int m0 = 0; m0 < n_mats; m0 += group) {
                const int nm = std::min(group, n_mats - m0);
                const VtyWindow w{Vt + i0, ka, k, Y + m0 * y_stride + j0, kb, k, y_stride};
                double *Pm = partial + (int64_t)m0 * nblk * kap * kbp;
                cudaError_t e;
                if (ntile <= 4) e = vty_launch<4, 768>(N, w, nm, nblk, Pm, st);
                else if (ntile <= 8) e = vty_launch<8, 768>(N, w, nm, nblk, Pm, st);
                else if (ntile <= 12) e = vty_launch<12, 768>(N, w, nm, nblk, Pm, st);
                else e = vty_launch<16, 512>(N, w, nm, nblk, Pm, st);
                if (e != cudaSuccess) return e;
            }
            ProjOut o{};
            for (int m = 0; m < n_mats; ++m) o.r[m] = out.r[m] + i0 + (int64_t)j0 * k;
            const int64_t tot = (int64_t)n_mats * ka * kb;
            reduce_partials_kernel<<<(int)((tot + 255) / 256), 256, 0, st>>>(partial, nblk, n_mats, ka, kb, kap, kbp,
                                                                               o, k);
            cudaError_t e = cudaGetLastError();
            if (e != cudaSuccess) return e;
        }
    }
    return cudaSuccess;
}

size_t gs_workspace_doubles(int k, int nblk) {
    const size_t rows_c = (size_t)((k + 7) & ~7) + GS_B;
    return (size_t)nblk * rows_c * GS_B + rows_c * GS_B + (size_t)GS_B * GS_B;
}

cudaError_t launch_gram_schmidt(double *V, int64_t N, int k, int64_t ldv, int passes, double *work, int nblk,
                                cudaStream_t st) {
    const int rows_max = ((k + 7) & ~7) + GS_B;
    double *part = work;
    double *Cm = part + (size_t)nblk * rows_max * GS_B;
    double *rinv = Cm + (size_t)rows_max * GS_B;
    const size_t smem = sizeof(double) * (size_t)2 * (GS_WIN + GS_B) * GS_LDR;
    cudaError_t e = cudaFuncSetAttribute(gs_gram_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const int64_t n_chunks = (N + 31) / 32;
    const int64_t per = (n_chunks + nblk - 1) / nblk;
    const int ugrid = (int)((N + 127) / 128);  // 128 rows per 256-thread CTA
    passes = std::max(passes, 1);
    for (int j0 = 0; j0 < k; j0 += GS_B) {
        const int b = std::min(GS_B, k - j0);
        const int rows_c = j0 + ((b + 7) & ~7);  // rows of C: Q's j0 columns, then P's (padded)
        for (int pass = 0; pass < passes; ++pass) {
            for (int x0 = 0; x0 < j0 + b; x0 += GS_WIN) {
                const int w = std::min(GS_WIN, j0 + b - x0);
                gs_gram_kernel<<<nblk, GS_THREADS, smem, st>>>(V, N, ldv, x0, w, j0, b, rows_c, per, part);
            }
            const int64_t tot = (int64_t)rows_c * GS_B;
            gs_reduce_kernel<<<(int)std::min<int64_t>((tot + 255) / 256, 1024), 256, 0, st>>>(part, nblk, rows_c, Cm);
            gs_chol_kernel<<<1, 256, 0, st>>>(Cm, j0, b, rinv);
            gs_update_kernel<<<ugrid, 256, 0, st>>>(V, N, ldv, j0, b, Cm, rinv);
            if ((e = cudaGetLastError()) != cudaSuccess) return e;
        }
    }
    return cudaSuccess;
}

}  // namespace srom
