// Krylov basis generation on the GPU: the block Arnoldi process with block Gram-Schmidt
// re-orthogonalisation and rank-revealing deflation of
// KrylovROMSubstructure::addKrylovModesForExpansionPoint (src/analysis/KrylovROMSubstructure.cpp:367-569).
//
// Per expansion point f0 (w0 = 2 pi f0) the reference factors K~ = -(K - w0^2 M + i w0 D) with
// PARDISO (:387-406, :571-707).  Here K~ is factored directly on the GPU as a band matrix:
//
//  * ordering  -- reverse Cuthill-McKee on the host (once per pattern) to shrink the bandwidth bw;
//  * storage   -- the lower band, column j holding rows j-NB .. j+bw+NB at band[j*ldab + i-j+NB]
//                 (NB rows of headroom above the diagonal), so that every dense sub-block of the
//                 band is a column-major matrix with leading dimension ldab-1;
//  * factor    -- blocked LDL^T without pivoting (K~ is complex symmetric), NB columns a step:
//                 the NB x NB diagonal block in one CTA, the panel L21 = A21 L11^-T D^-1 by one
//                 warp a row, and the trailing update A22 -= (L21 D) L21^T as one strided-batched
//                 complex GEMM over the column blocks of the window (zgemm.cu, FP64 tensor cores);
//  * solves    -- blocked forward / diagonal / backward substitution for all right-hand sides,
//                 the off-diagonal block updates as complex GEMMs (split over k when short and wide).
//
// The rest of the process runs on the GPU as in the reference: M Q by a complex CSR SpMM, the
// re-orthogonalisation Q <- Q - V (V^H Q) with complex GEMMs (V^H Q split over the rows, reduced
// in a fixed order) until the norm ratio exceeds 1/sqrt(2),
// and the column-pivoted Householder QR (the steps of zgeqp3 with exact partial column norms)
// whose leading |R_ii| > tol decide the rank, Q formed from the reflectors (zungqr).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/staccato_rom.h"
#include "krylov_kernels.h"
#include "zgemm.h"

namespace srom {
namespace kry {

constexpr int NB = 64;   // columns per elimination step (and rows of band headroom)
constexpr int KT = 256;  // threads per CTA
constexpr int SLD = NB + 1;
constexpr double PIVOT_EPS = 1e-13;  // small-pivot threshold relative to ||A||_inf (PARDISO iparm[9] = 13)

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// c - a b
__device__ __forceinline__ double2 cfms(double2 c, double2 a, double2 b) {
    return make_double2(fma(-a.x, b.x, fma(a.y, b.y, c.x)), fma(-a.x, b.y, fma(-a.y, b.x, c.y)));
}
// a / b by Smith's method
__device__ __forceinline__ double2 cdiv(double2 a, double2 b) {
    if (fabs(b.x) >= fabs(b.y)) {
        const double r = b.y / b.x, den = b.x + b.y * r;
        return make_double2((a.x + a.y * r) / den, (a.y - a.x * r) / den);
    }
    const double r = b.x / b.y, den = b.y + b.x * r;
    return make_double2((a.x * r + a.y) / den, (a.y * r - a.x) / den);
}
// 1 / b = conj(b) / |b|^2 (one division; this solver carries no bit-exactness contract)
__device__ __forceinline__ double2 crecip(double2 b) {
    const double s = 1.0 / fma(b.x, b.x, b.y * b.y);
    return make_double2(b.x * s, -b.y * s);
}
__device__ __forceinline__ double2 shfl2(double2 v, int src) {
    return make_double2(__shfl_sync(0xffffffffu, v.x, src), __shfl_sync(0xffffffffu, v.y, src));
}

// ---- K~ into band storage -----------------------------------------------------------------
// Full symmetric pattern (0-based, rows of the original numbering); vmap[e] indexes the caller's
// value arrays.  Entry (i, j) lands at (pi, pj) = (iperm[i], iperm[j]) when pi >= pj, so every
// unordered pair is written once.  Value sign * (K - w^2 M + i w D): sign = -1 gives the Krylov
// process's K~, +1 the full-order dynamic stiffness.  One warp per row.
// Also the infinity norm of the matrix (largest row sum of |a_ij| over the full pattern) into
// anorm_bits, as the bits of a non-negative double (their unsigned order is the numeric order).
__global__ void scatter_band_kernel(int64_t n, const int64_t *__restrict__ rp, const int *__restrict__ ci,
                                    const int64_t *__restrict__ vmap, const double2 *__restrict__ K,
                                    const double2 *__restrict__ M, const double2 *__restrict__ D, double w,
                                    double sign, const int *__restrict__ iperm, double2 *__restrict__ band,
                                    int64_t ldab, unsigned long long *__restrict__ anorm_bits) {
    const int lane = threadIdx.x & 31;
    const double w2 = w * w;
    for (int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; i < n;
         i += ((int64_t)gridDim.x * blockDim.x) >> 5) {
        const int pi = iperm[i];
        double rs = 0.0;
        for (int64_t e = rp[i] + lane; e < rp[i + 1]; e += 32) {
            const int pj = iperm[ci[e]];
            const int64_t v = vmap[e];
            const double2 k = K[v], m = M[v];
            double re = k.x - w2 * m.x, im = k.y - w2 * m.y;
            if (D) {
                const double2 d = D[v];
                re -= w * d.y;
                im += w * d.x;
            }
            rs += hypot(re, im);
            if (pi < pj) continue;
            band[(int64_t)pj * ldab + (pi - pj + NB)] = make_double2(sign * re, sign * im);
        }
#pragma unroll
        for (int off = 16; off; off >>= 1) rs += __shfl_xor_sync(0xffffffffu, rs, off);
        if (lane == 0) atomicMax(anorm_bits, (unsigned long long)__double_as_longlong(rs));
    }
}

// ---- blocked LDL^T ------------------------------------------------------------------------
// The nb x nb diagonal block at column j0: A11 = L11 D L11^T (unit L11, no pivoting), in place
// (D on the diagonal).  The block is held whole (both triangles) in shared memory; step k
// updates a_ij -= a_ik (a_kj / d_k) for i, j > k, each thread owning one column j (its row
// entries are contiguous across the warp) and every fourth row, so a step needs one barrier.
// The columns are scaled by 1/d_k once at the end.  The first exactly-zero pivot is recorded
// 1-based in *info.
// Small pivots are perturbed as PARDISO does with the reference's setting iparm[9] = 13
// (KrylovROMSubstructure.cpp:621): a pivot d with |d| < 1e-13 ||A||_inf is replaced by the value
// of the same phase and modulus 1e-13 ||A||_inf, and counted in *perturbed; *min_ratio_bits
// keeps the smallest |d| / ||A||_inf (bits of a non-negative double).  An exactly zero pivot
// is still reported in *info (the matrix is singular, not merely ill-conditioned).
__device__ __forceinline__ double2 perturb_pivot(double2 d, double tau) {
    const double a = hypot(d.x, d.y);
    if (a >= tau) return d;
    if (a == 0.0) return make_double2(tau, 0.0);
    const double s = tau / a;
    return make_double2(d.x * s, d.y * s);
}

__global__ void __launch_bounds__(KT) ldlt_diag_kernel(double2 *__restrict__ band, int64_t ldab, int64_t j0, int nb,
                                                       int *__restrict__ info,
                                                       const unsigned long long *__restrict__ anorm_bits,
                                                       int *__restrict__ perturbed,
                                                       unsigned long long *__restrict__ min_ratio_bits) {
    extern __shared__ double2 S[];  // S[i * SLD + j], full symmetric block
    constexpr int RS = KT / NB;     // row stride of a thread
    const int t = threadIdx.x;
    const double anorm = __longlong_as_double((long long)*anorm_bits);
    const double tau = PIVOT_EPS * anorm;
    for (int e = t; e < nb * nb; e += KT) {
        const int i = e / nb, j = e % nb;
        const int r = max(i, j), c = min(i, j);
        S[i * SLD + j] = band[(j0 + c) * ldab + (r - c + NB)];
    }
    __syncthreads();
    const int j = t % NB, ir = t / NB;
    for (int k = 0; k < nb; ++k) {
        const double2 d0 = S[k * SLD + k];
        const double2 d = perturb_pivot(d0, tau);  // the same value in every thread
        if (t == 0) {
            if (d0.x == 0.0 && d0.y == 0.0) atomicCAS(info, 0, (int)(j0 + k + 1));
            const double a = hypot(d0.x, d0.y);
            if (a < tau) atomicAdd(perturbed, 1);
            if (anorm > 0.0) atomicMin(min_ratio_bits, (unsigned long long)__double_as_longlong(a / anorm));
        }
        if (j > k && j < nb) {
            const double2 cj = cmul(S[k * SLD + j], crecip(d));
            for (int i = k + 1 + ((ir - (k + 1)) % RS + RS) % RS; i < nb; i += RS)
                S[i * SLD + j] = cfms(S[i * SLD + j], S[i * SLD + k], cj);
        }
        __syncthreads();
    }
    for (int e = t; e < nb * nb; e += KT) {
        const int i = e % nb, c = e / nb;
        const double2 dc = perturb_pivot(S[c * SLD + c], tau);  // step c never changes S[c][c]
        if (i > c)
            band[(j0 + c) * ldab + (i - c + NB)] = cmul(S[i * SLD + c], crecip(dc));
        else if (i == c)
            band[(j0 + c) * ldab + NB] = dc;
    }
}

// Loads the factored diagonal block (L11 below, D on the diagonal) into shared memory.
__device__ __forceinline__ void load_l11(const double2 *band, int64_t ldab, int64_t j0, int nb, double2 *S) {
    for (int e = threadIdx.x; e < nb * nb; e += blockDim.x) {
        const int i = e % nb, j = e / nb;
        if (i >= j) S[i * SLD + j] = band[(j0 + j) * ldab + (i - j + NB)];
    }
    __syncthreads();
}

// Panel rows t in [0, rows) (matrix rows j0+nb+t): x L11^T = a, L21 = x D^-1; x goes to W
// (= L21 D) and L21 to Lp and to the band.  Rows [rows, zero_to) of W and Lp are zeroed (the
// strided-batched update reads up to NB * (batches - 1) + rows rows).  One warp a row, lane l
// holding columns l and l + 32.
__global__ void __launch_bounds__(KT) ldlt_panel_kernel(double2 *__restrict__ band, int64_t ldab, int64_t j0, int nb,
                                                        int rows, int zero_to, double2 *__restrict__ W,
                                                        double2 *__restrict__ Lp, int ldw) {
    extern __shared__ double2 S[];  // L11 (NB x SLD) then 1/d (NB)
    double2 *Dinv = S + NB * SLD;
    load_l11(band, ldab, j0, nb, S);
    for (int k = threadIdx.x; k < nb; k += blockDim.x) Dinv[k] = crecip(S[k * SLD + k]);
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int t = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5);
    if (t >= zero_to) return;
    if (t >= rows) {
        for (int k = lane; k < NB; k += 32) {
            W[t + (int64_t)k * ldw] = make_double2(0.0, 0.0);
            Lp[t + (int64_t)k * ldw] = make_double2(0.0, 0.0);
        }
        return;
    }
    const int64_t r = j0 + nb + t;
    double2 x[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const int k = lane + 32 * h;
        x[h] = k < nb ? band[(j0 + k) * ldab + (r - (j0 + k) + NB)] : make_double2(0.0, 0.0);
    }
    for (int m = 0; m < nb; ++m) {
        const double2 xm = m < 32 ? shfl2(x[0], m) : shfl2(x[1], m - 32);
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int k = lane + 32 * h;
            if (k > m && k < nb) x[h] = cfms(x[h], S[k * SLD + m], xm);
        }
    }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const int k = lane + 32 * h;
        if (k < NB) {
            double2 l = make_double2(0.0, 0.0), wv = make_double2(0.0, 0.0);
            if (k < nb) {
                wv = x[h];
                l = cmul(x[h], Dinv[k]);
                band[(j0 + k) * ldab + (r - (j0 + k) + NB)] = l;
            }
            W[t + (int64_t)k * ldw] = wv;
            Lp[t + (int64_t)k * ldw] = l;
        }
    }
}

// Triangular solves with the unit L11 of block j0 for all right-hand sides (X rows j0..j0+nb):
// forward (trans = 0) L11 y = x, backward (trans = 1) L11^T y = x.  One warp a right-hand side.
__global__ void __launch_bounds__(KT) trsv_block_kernel(const double2 *__restrict__ band, int64_t ldab, int64_t j0,
                                                        int nb, double2 *__restrict__ X, int64_t ldx, int nrhs,
                                                        int trans) {
    extern __shared__ double2 S[];
    load_l11(band, ldab, j0, nb, S);
    const int lane = threadIdx.x & 31;
    for (int c = (int)((blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5); c < nrhs;
         c += (int)(((int64_t)gridDim.x * blockDim.x) >> 5)) {
        double2 *x = X + (int64_t)c * ldx + j0;
        double2 v[2];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int k = lane + 32 * h;
            v[h] = k < nb ? x[k] : make_double2(0.0, 0.0);
        }
        if (!trans) {
            for (int m = 0; m < nb; ++m) {
                const double2 vm = m < 32 ? shfl2(v[0], m) : shfl2(v[1], m - 32);
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int k = lane + 32 * h;
                    if (k > m && k < nb) v[h] = cfms(v[h], S[k * SLD + m], vm);
                }
            }
        } else {
            for (int m = nb - 1; m >= 0; --m) {
                const double2 vm = m < 32 ? shfl2(v[0], m) : shfl2(v[1], m - 32);
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int k = lane + 32 * h;
                    if (k < m) v[h] = cfms(v[h], S[m * SLD + k], vm);
                }
            }
        }
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int k = lane + 32 * h;
            if (k < nb) x[k] = v[h];
        }
    }
}

// X[i, c] /= D_i (the diagonal of the factored band).
__global__ void diag_scale_kernel(const double2 *__restrict__ band, int64_t ldab, int64_t n, double2 *__restrict__ X,
                                  int64_t ldx, int nrhs) {
    const int64_t total = n * nrhs;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = e % n, c = e / n;
        X[i + c * ldx] = cdiv(X[i + c * ldx], band[i * ldab + NB]);
    }
}

// dst[iperm[i], c] = src[i, c] (to = 1) or dst[i, c] = src[iperm[i], c] (to = 0).
__global__ void permute_kernel(int64_t n, int nrhs, const int *__restrict__ iperm, const double2 *__restrict__ src,
                               int64_t lds, double2 *__restrict__ dst, int64_t ldd, int to) {
    const int64_t total = n * nrhs;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = e % n, c = e / n;
        if (to)
            dst[iperm[i] + c * ldd] = src[i + c * lds];
        else
            dst[i + c * ldd] = src[iperm[i] + c * lds];
    }
}

// Y = A Q for the full pattern with values A[vmap[e]]; one warp a row, lanes over its entries.
__global__ void csr_spmm_complex_kernel(int64_t n, const int64_t *__restrict__ rp, const int *__restrict__ ci,
                                        const int64_t *__restrict__ vmap, const double2 *__restrict__ A,
                                        const double2 *__restrict__ Q, int64_t ldq, int k, double2 *__restrict__ Y,
                                        int64_t ldy) {
    const int lane = threadIdx.x & 31;
    for (int64_t i = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 5; i < n;
         i += ((int64_t)gridDim.x * blockDim.x) >> 5) {
        for (int c = 0; c < k; ++c) {
            double2 acc = make_double2(0.0, 0.0);
            for (int64_t e = rp[i] + lane; e < rp[i + 1]; e += 32) {
                const double2 a = A[vmap[e]], q = Q[ci[e] + (int64_t)c * ldq];
                acc.x = fma(a.x, q.x, fma(-a.y, q.y, acc.x));
                acc.y = fma(a.x, q.y, fma(a.y, q.x, acc.y));
            }
#pragma unroll
            for (int off = 16; off; off >>= 1) {
                acc.x += __shfl_xor_sync(0xffffffffu, acc.x, off);
                acc.y += __shfl_xor_sync(0xffffffffu, acc.y, off);
            }
            if (lane == 0) Y[i + (int64_t)c * ldy] = acc;
        }
    }
}

// ---- column-pivoted Householder QR pieces (one CTA a column) -------------------------------
__device__ __forceinline__ double block_sum(double v, double *red) {
    for (int off = 16; off; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    __syncthreads();
    if (lane == 0) red[w] = v;
    __syncthreads();
    v = threadIdx.x < (KT >> 5) ? red[threadIdx.x] : 0.0;
    if (w == 0)
        for (int off = 16; off; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
    return v;
}

// out[j - j0] = sum_{i >= r0} |A[i, j]|^2 for j in [j0, j0 + count)
__global__ void __launch_bounds__(KT) col_norm2_kernel(const double2 *__restrict__ A, int64_t lda, int64_t n, int64_t r0,
                                                       int j0, double *__restrict__ out) {
    __shared__ double red[KT / 32];
    const int j = j0 + blockIdx.x;
    double s = 0.0;
    for (int64_t i = r0 + threadIdx.x; i < n; i += KT) {
        const double2 a = A[i + (int64_t)j * lda];
        s = fma(a.x, a.x, fma(a.y, a.y, s));
    }
    s = block_sum(s, red);
    if (threadIdx.x == 0) out[blockIdx.x] = s;
}

__global__ void swap_cols_kernel(double2 *__restrict__ A, int64_t lda, int64_t n, int a, int b) {
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const double2 t = A[i + (int64_t)a * lda];
        A[i + (int64_t)a * lda] = A[i + (int64_t)b * lda];
        A[i + (int64_t)b * lda] = t;
    }
}

// Column k of A becomes the Householder vector (v_k = 1 implicit, A[k, k] = beta): rows > k
// scaled by s.
__global__ void householder_scale_kernel(double2 *__restrict__ A, int64_t lda, int64_t n, int k, double2 s,
                                         double beta) {
    double2 *a = A + (int64_t)k * lda;
    for (int64_t i = k + 1 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
        a[i] = cmul(a[i], s);
    if (blockIdx.x == 0 && threadIdx.x == 0) a[k] = make_double2(beta, 0.0);
}

// w[j - j0] = v^H T[k:, j] with v = (1, V[k+1:, vk]) for j in [j0, j0 + count)
__global__ void __launch_bounds__(KT) reflector_dots_kernel(const double2 *__restrict__ Vr, int64_t ldv, int vk,
                                                            const double2 *__restrict__ T, int64_t ldt, int64_t n,
                                                            int64_t k, int j0, double2 *__restrict__ w) {
    __shared__ double red[KT / 32];
    const int j = j0 + blockIdx.x;
    const double2 *v = Vr + (int64_t)vk * ldv;
    const double2 *t = T + (int64_t)j * ldt;
    double sr = 0.0, si = 0.0;
    for (int64_t i = k + threadIdx.x; i < n; i += KT) {
        const double2 vi = i == k ? make_double2(1.0, 0.0) : v[i];
        const double2 ti = t[i];
        sr = fma(vi.x, ti.x, fma(vi.y, ti.y, sr));  // conj(v) t
        si = fma(vi.x, ti.y, fma(-vi.y, ti.x, si));
    }
    sr = block_sum(sr, red);
    si = block_sum(si, red);
    if (threadIdx.x == 0) w[blockIdx.x] = make_double2(sr, si);
}

// T[i, j] -= tau v_i w_j for i >= k, j in [j0, j0 + count)
__global__ void reflector_apply_kernel(const double2 *__restrict__ Vr, int64_t ldv, int vk, double2 *__restrict__ T,
                                       int64_t ldt, int64_t n, int64_t k, int j0, int count,
                                       const double2 *__restrict__ w, double2 tau) {
    const double2 *v = Vr + (int64_t)vk * ldv;
    const int64_t rows = n - k, total = rows * count;
    for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < total; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = k + e % rows;
        const int j = j0 + (int)(e / rows);
        const double2 vi = i == k ? make_double2(1.0, 0.0) : v[i];
        T[i + (int64_t)j * ldt] = cfms(T[i + (int64_t)j * ldt], cmul(tau, vi), w[j - j0]);
    }
}

// Column i of Q from reflector i (zung2r): Q[r, i] = -tau v_r (r > i), 1 - tau (r = i), 0 (r < i).
__global__ void reflector_column_kernel(const double2 *__restrict__ Vr, int64_t ldv, int vi, double2 *__restrict__ Q,
                                        int64_t ldq, int64_t n, int i, double2 tau) {
    const double2 *v = Vr + (int64_t)vi * ldv;
    for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
        double2 q;
        if (r < i)
            q = make_double2(0.0, 0.0);
        else if (r == i)
            q = make_double2(1.0 - tau.x, -tau.y);
        else
            q = make_double2(-(tau.x * v[r].x - tau.y * v[r].y), -(tau.x * v[r].y + tau.y * v[r].x));
        Q[r + (int64_t)i * ldq] = q;
    }
}

// ==================================================================================================
// host side
// ==================================================================================================
namespace {

struct Err {
    int code = SROM_OK;
    std::string msg;
    int set(int c, const std::string &m) {
        if (code == SROM_OK) {
            code = c;
            msg = m;
        }
        return c;
    }
};

#define KCU(call)                                                                           \
    do {                                                                                    \
        cudaError_t _e = (call);                                                            \
        if (_e != cudaSuccess) return E.set(SROM_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(_e)); \
    } while (0)

// Device buffers freed at scope exit (after the stream has drained).
struct Bufs {
    cudaStream_t st = nullptr;
    std::vector<void *> ptrs;
    ~Bufs() {
        if (st) cudaStreamSynchronize(st);
        for (void *p : ptrs) cudaFree(p);
    }
    template <typename T>
    cudaError_t alloc(T **p, size_t count) {
        void *q = nullptr;
        cudaError_t e = cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T));
        if (e == cudaSuccess) ptrs.push_back(q);
        *p = static_cast<T *>(q);
        return e;
    }
};

int grid_for(int64_t work, int threads) {
    const int64_t b = (work + threads - 1) / threads;
    return (int)std::max<int64_t>(1, std::min<int64_t>(b, 148 * 16));
}

}  // namespace

// Full symmetric pattern of a CSR matrix given in full or upper storage (base 0 or 1), with the
// index of each entry's value in the caller's arrays.
int full_pattern(int64_t n, int64_t nnz, const int64_t *rp, const int *ci, int base, int upper, std::vector<int64_t> &frp,
                 std::vector<int> &fci, std::vector<int64_t> &fmap, std::string *err) {
    frp.assign(n + 1, 0);
    for (int64_t i = 0; i < n; ++i)
        if (rp[i + 1] < rp[i] || rp[i + 1] - base > nnz) {
            if (err) *err = "rowptr decreases or passes nnz at row " + std::to_string(i);
            return SROM_ERR_INVALID;
        }
    for (int64_t i = 0; i < n; ++i) {
        for (int64_t e = rp[i] - base; e < rp[i + 1] - base; ++e) {
            const int64_t j = (int64_t)ci[e] - base;
            if (j < 0 || j >= n) {
                if (err) *err = "column index out of range in row " + std::to_string(i);
                return SROM_ERR_INVALID;
            }
            if (upper && j < i) {
                if (err) *err = "upper storage holds an entry below the diagonal in row " + std::to_string(i);
                return SROM_ERR_INVALID;
            }
            frp[i + 1]++;
            if (upper && j != i) frp[j + 1]++;
        }
    }
    for (int64_t i = 0; i < n; ++i) frp[i + 1] += frp[i];
    fci.assign(frp[n], 0);
    fmap.assign(frp[n], 0);
    std::vector<int64_t> pos(frp.begin(), frp.end() - 1);
    for (int64_t i = 0; i < n; ++i)
        for (int64_t e = rp[i] - base; e < rp[i + 1] - base; ++e) {
            const int64_t j = (int64_t)ci[e] - base;
            fci[pos[i]] = (int)j;
            fmap[pos[i]++] = e;
            if (upper && j != i) {
                fci[pos[j]] = (int)i;
                fmap[pos[j]++] = e;
            }
        }
    return SROM_OK;
}

// Reverse Cuthill-McKee on the full pattern: perm[k] = old index of new row k; each connected
// component starts from a pseudo-peripheral node (George & Liu), neighbours visited by increasing
// degree.  Returns the bandwidth max |iperm[i] - iperm[j]| over the entries.
int64_t rcm_order(int64_t n, const std::vector<int64_t> &frp, const std::vector<int> &fci, std::vector<int> &perm) {
    std::vector<int> deg(n), level(n, -1), order;
    order.reserve(n);
    for (int64_t i = 0; i < n; ++i) deg[i] = (int)(frp[i + 1] - frp[i]);
    std::vector<char> done(n, 0);
    std::vector<int> queue(n), nbr;
    auto bfs_levels = [&](int s, int &last_level, std::vector<int> &touched) {
        // breadth-first levels from s among nodes not yet ordered; returns nodes visited
        touched.clear();
        int head = 0, tail = 0;
        queue[tail++] = s;
        level[s] = 0;
        touched.push_back(s);
        last_level = 0;
        while (head < tail) {
            const int u = queue[head++];
            last_level = std::max(last_level, level[u]);
            for (int64_t e = frp[u]; e < frp[u + 1]; ++e) {
                const int v = fci[e];
                if (!done[v] && level[v] < 0) {
                    level[v] = level[u] + 1;
                    queue[tail++] = v;
                    touched.push_back(v);
                }
            }
        }
    };
    std::vector<int> touched;
    std::vector<int64_t> by_degree(n);
    for (int64_t i = 0; i < n; ++i) by_degree[i] = i;
    std::stable_sort(by_degree.begin(), by_degree.end(), [&](int64_t a, int64_t b) { return deg[a] < deg[b]; });
    for (int64_t idx = 0; idx < n; ++idx) {
        int s = (int)by_degree[idx];
        if (done[s]) continue;
        // pseudo-peripheral start node
        int ecc = -1;
        for (int it = 0; it < 16; ++it) {
            int last = 0;
            bfs_levels(s, last, touched);
            int best = -1;
            for (int v : touched)
                if (level[v] == last && (best < 0 || deg[v] < deg[best])) best = v;
            for (int v : touched) level[v] = -1;
            if (last <= ecc || best < 0) break;
            ecc = last;
            s = best;
        }
        // Cuthill-McKee from s
        int head = (int)order.size();
        order.push_back(s);
        done[s] = 1;
        while (head < (int)order.size()) {
            const int u = order[head++];
            nbr.clear();
            for (int64_t e = frp[u]; e < frp[u + 1]; ++e) {
                const int v = fci[e];
                if (!done[v]) {
                    done[v] = 1;
                    nbr.push_back(v);
                }
            }
            std::stable_sort(nbr.begin(), nbr.end(), [&](int a, int b) { return deg[a] < deg[b]; });
            order.insert(order.end(), nbr.begin(), nbr.end());
        }
    }
    std::reverse(order.begin(), order.end());
    perm = order;
    std::vector<int> iperm(n);
    for (int64_t k = 0; k < n; ++k) iperm[perm[k]] = (int)k;
    int64_t bw = 0;
    for (int64_t i = 0; i < n; ++i)
        for (int64_t e = frp[i]; e < frp[i + 1]; ++e) bw = std::max<int64_t>(bw, std::llabs((int64_t)iperm[i] - iperm[fci[e]]));
    return bw;
}

int64_t band_bytes(int64_t n, int64_t bw) { return (n + 2 * NB) * (bw + 2 * NB + 1) * (int64_t)sizeof(double2); }

namespace {

// One factorisation K~ = L D L^T in band storage and its solves.
struct BandLDLT {
    int64_t n = 0, bw = 0, ldab = 0;
    int ldw = 0;
    double2 *band = nullptr, *W = nullptr, *Lp = nullptr;
    int *d_info = nullptr;
    cudaStream_t st = nullptr;
    double2 *zwork = nullptr;  // split-k partials of the complex GEMMs
    int64_t zwork_elems = 0;
    int sms = 148;
    // ||A||_inf of the assembled matrix, perturbed-pivot count, smallest |d| / ||A||_inf (device)
    unsigned long long *d_anorm = nullptr, *d_minr = nullptr;
    int *d_pert = nullptr;
    PivotStats *stats = nullptr;  // accumulated over the factorisations of a call (may be null)

    // complex GEMM C -= op(A) op(B) (beta = 1) on this factor's stream and workspace
    Zgemm gemm(int opa, int opb, int m, int nn, int k, const double2 *A, int64_t lda, const double2 *Bm, int64_t ldb,
               double2 *C, int64_t ldc) const {
        Zgemm z;
        z.opa = opa;
        z.opb = opb;
        z.m = m;
        z.n = nn;
        z.k = k;
        z.alpha = make_double2(-1.0, 0.0);
        z.beta = make_double2(1.0, 0.0);
        z.A = A;
        z.lda = lda;
        z.B = Bm;
        z.ldb = ldb;
        z.C = C;
        z.ldc = ldc;
        z.work = zwork;
        z.work_elems = zwork_elems;
        z.sms = sms;
        return z;
    }

    int factor(Err &E) {
        const size_t smem = sizeof(double2) * NB * SLD;
        const unsigned long long inf_bits = 0x7FF0000000000000ull;
        KCU(cudaMemsetAsync(d_info, 0, sizeof(int), st));
        KCU(cudaMemsetAsync(d_pert, 0, sizeof(int), st));
        KCU(cudaMemcpyAsync(d_minr, &inf_bits, sizeof inf_bits, cudaMemcpyHostToDevice, st));
        int prev_rows = ldw;
        for (int64_t j0 = 0; j0 < n; j0 += NB) {
            const int nb = (int)std::min<int64_t>(NB, n - j0);
            ldlt_diag_kernel<<<1, KT, smem, st>>>(band, ldab, j0, nb, d_info, d_anorm, d_pert, d_minr);
            const int rows = (int)std::min<int64_t>(bw, n - j0 - nb);
            if (rows <= 0) continue;
            const int zero_to = std::max(rows, prev_rows);
            prev_rows = rows;
            ldlt_panel_kernel<<<(zero_to + KT / 32 - 1) / (KT / 32), KT, smem + sizeof(double2) * NB, st>>>(
                band, ldab, j0, nb, rows, zero_to, W, Lp, ldw);
            // trailing update of the window: column block b (NB columns) -= W_b Lp_b^T, with
            // W_b, Lp_b the panel rows from b NB on
            const int batches = (rows + NB - 1) / NB;
            double2 *C0 = band + (j0 + nb) * ldab + NB;
            Zgemm z = gemm(ZG_N, ZG_T, rows, NB, nb, W, ldw, Lp, ldw, C0, ldab - 1);
            z.sa = NB;
            z.sb = NB;
            z.sc = (int64_t)NB * ldab;
            z.batch = batches;
            KCU(zgemm(z, st));
        }
        KCU(cudaGetLastError());
        int info = 0, pert = 0;
        unsigned long long minr = inf_bits;
        KCU(cudaMemcpyAsync(&info, d_info, sizeof(int), cudaMemcpyDeviceToHost, st));
        KCU(cudaMemcpyAsync(&pert, d_pert, sizeof(int), cudaMemcpyDeviceToHost, st));
        KCU(cudaMemcpyAsync(&minr, d_minr, sizeof minr, cudaMemcpyDeviceToHost, st));
        KCU(cudaStreamSynchronize(st));
        if (stats) {
            double r;
            std::memcpy(&r, &minr, sizeof r);
            stats->factorisations += 1;
            stats->perturbed += pert;
            stats->min_pivot_ratio = std::min(stats->min_pivot_ratio, r);
        }
        if (info != 0)
            return E.set(SROM_ERR_INVALID, "K~ has an exactly zero pivot at (permuted) row " + std::to_string(info) +
                                               ": the shifted matrix is singular");
        return SROM_OK;
    }

    // X (n x nrhs, ldx, permuted order) <- K~^-1 X
    int solve(double2 *X, int64_t ldx, int nrhs, Err &E) {
        const size_t smem = sizeof(double2) * NB * SLD;
        const int tgrid = (nrhs + KT / 32 - 1) / (KT / 32);
        for (int64_t j0 = 0; j0 < n; j0 += NB) {
            const int nb = (int)std::min<int64_t>(NB, n - j0);
            trsv_block_kernel<<<tgrid, KT, smem, st>>>(band, ldab, j0, nb, X, ldx, nrhs, 0);
            const int rows = (int)std::min<int64_t>(bw, n - j0 - nb);
            if (rows <= 0) continue;
            KCU(zgemm(gemm(ZG_N, ZG_N, rows, nrhs, nb, band + j0 * ldab + NB + nb, ldab - 1, X + j0, ldx,
                           X + j0 + nb, ldx), st));
        }
        diag_scale_kernel<<<grid_for(n * nrhs, KT), KT, 0, st>>>(band, ldab, n, X, ldx, nrhs);
        const int64_t last = ((n - 1) / NB) * NB;
        for (int64_t j0 = last; j0 >= 0; j0 -= NB) {
            const int nb = (int)std::min<int64_t>(NB, n - j0);
            const int rows = (int)std::min<int64_t>(bw, n - j0 - nb);
            if (rows > 0)
                KCU(zgemm(gemm(ZG_T, ZG_N, nb, nrhs, rows, band + j0 * ldab + NB + nb, ldab - 1, X + j0 + nb, ldx,
                               X + j0, ldx), st));
            trsv_block_kernel<<<tgrid, KT, smem, st>>>(band, ldab, j0, nb, X, ldx, nrhs, 1);
        }
        KCU(cudaGetLastError());
        return SROM_OK;
    }
};

// Q (n x m, ld n) <- Q - V (V^H Q) repeated until ||Q_new||_F / ||Q_old||_F > 1/sqrt(2).
// S: kv x m; nrm: znorm2_work_doubles() + 2 doubles (the two norms end in its last two).
int reorthogonalize(const BandLDLT &F, cudaStream_t st, const double2 *V, int64_t ldv, int kv, double2 *&Q,
                    double2 *&U, int64_t n, int m, double2 *S, double *nrm, Err &E) {
    if (kv == 0 || m == 0) return SROM_OK;
    const double eta = 1.0 / std::sqrt(2.0);
    double *nrm_out = nrm + znorm2_work_doubles();
    for (int it = 0; it < 64; ++it) {
        Zgemm h = F.gemm(ZG_C, ZG_N, kv, m, (int)n, V, ldv, Q, n, S, kv);  // S = V^H Q
        h.alpha = make_double2(1.0, 0.0);
        h.beta = make_double2(0.0, 0.0);
        KCU(zgemm(h, st));
        KCU(cudaMemcpyAsync(U, Q, sizeof(double2) * n * m, cudaMemcpyDeviceToDevice, st));
        KCU(zgemm(F.gemm(ZG_N, ZG_N, (int)n, m, kv, V, ldv, S, kv, U, n), st));  // U = Q - V S
        KCU(znorm2(U, n * m, nrm, nrm_out, st));
        KCU(znorm2(Q, n * m, nrm, nrm_out + 1, st));
        double nh[2] = {0.0, 0.0};
        KCU(cudaMemcpyAsync(nh, nrm_out, sizeof nh, cudaMemcpyDeviceToHost, st));
        KCU(cudaStreamSynchronize(st));
        const double nu = nh[0], nq = nh[1];
        std::swap(Q, U);
        if (!(nu / nq <= eta)) return SROM_OK;  // also leaves on NaN
    }
    return SROM_OK;
}

// Column-pivoted Householder QR of A (n x m, ld n) in place (zgeqp3's steps, partial norms
// recomputed exactly each step); |R_ii| in order go to rdiag; then Qo (n x rr, ld n) = the first
// rr columns of the orthonormal factor (zungqr), rr = leading |R_ii| > tol.
int pivoted_qr(cudaStream_t st, double2 *A, int64_t n, int m, double tol, double2 *Qo, double *d_norms, double2 *d_w,
               std::vector<double> &rdiag, int &rr, Err &E) {
    std::vector<double2> taus(m);
    std::vector<double> norms(m);
    const int kmax = (int)std::min<int64_t>(n, m);
    rdiag.assign(kmax, 0.0);
    for (int k = 0; k < kmax; ++k) {
        const int cnt = m - k;
        col_norm2_kernel<<<cnt, KT, 0, st>>>(A, n, n, k, k, d_norms);
        KCU(cudaMemcpyAsync(norms.data(), d_norms, sizeof(double) * cnt, cudaMemcpyDeviceToHost, st));
        KCU(cudaStreamSynchronize(st));
        int p = 0;
        for (int j = 1; j < cnt; ++j)
            if (norms[j] > norms[p]) p = j;
        if (p != 0) swap_cols_kernel<<<grid_for(n, KT), KT, 0, st>>>(A, n, n, k, k + p);
        double2 alpha;
        KCU(cudaMemcpyAsync(&alpha, A + k + (int64_t)k * n, sizeof(double2), cudaMemcpyDeviceToHost, st));
        KCU(cudaStreamSynchronize(st));
        const double xnorm2 = std::max(0.0, norms[p] - (alpha.x * alpha.x + alpha.y * alpha.y));
        double2 tau = make_double2(0.0, 0.0);
        double beta = alpha.x;
        if (!(xnorm2 == 0.0 && alpha.y == 0.0)) {
            const double nrm = std::sqrt(norms[p]);
            beta = alpha.x >= 0.0 ? -nrm : nrm;
            tau = make_double2((beta - alpha.x) / beta, -alpha.y / beta);
            // s = 1 / (alpha - beta)
            const double ar = alpha.x - beta, ai = alpha.y, den = ar * ar + ai * ai;
            householder_scale_kernel<<<grid_for(n, KT), KT, 0, st>>>(A, n, n, k, make_double2(ar / den, -ai / den), beta);
        }
        taus[k] = tau;
        rdiag[k] = std::fabs(beta) > 0.0 ? std::fabs(beta) : std::hypot(alpha.x, alpha.y);
        if (k + 1 < m && (tau.x != 0.0 || tau.y != 0.0)) {
            reflector_dots_kernel<<<m - k - 1, KT, 0, st>>>(A, n, k, A, n, n, k, k + 1, d_w);
            reflector_apply_kernel<<<grid_for((n - k) * (m - k - 1), KT), KT, 0, st>>>(
                A, n, k, A, n, n, k, k + 1, m - k - 1, d_w, make_double2(tau.x, -tau.y));
        }
    }
    KCU(cudaGetLastError());
    rr = 0;
    while (rr < kmax && rdiag[rr] > tol) ++rr;
    // Q = H_0 H_1 ... H_{rr-1} applied to the first rr unit columns, last reflector first
    for (int i = rr - 1; i >= 0; --i) {
        const double2 tau = taus[i];
        if (i + 1 < rr) {
            reflector_dots_kernel<<<rr - i - 1, KT, 0, st>>>(A, n, i, Qo, n, n, i, i + 1, d_w);
            reflector_apply_kernel<<<grid_for((n - i) * (rr - i - 1), KT), KT, 0, st>>>(A, n, i, Qo, n, n, i, i + 1,
                                                                                      rr - i - 1, d_w, tau);
        }
        reflector_column_kernel<<<grid_for(n, KT), KT, 0, st>>>(A, n, i, Qo, n, n, i, tau);
    }
    KCU(cudaGetLastError());
    return SROM_OK;
}

}  // namespace

void PatternCache::release() {
    if (d_frp) cudaFree(d_frp);
    if (d_fci) cudaFree(d_fci);
    if (d_fmap) cudaFree(d_fmap);
    if (d_iperm) cudaFree(d_iperm);
    d_frp = d_fmap = nullptr;
    d_fci = d_iperm = nullptr;
    n = nnz = -1;
    base = upper = -1;
    hash = 0;
    bw = nfull = 0;
    last_reused = false;
}

namespace {

// 64-bit hash of a CSR pattern (rowptr words, then colind in pairs): a multiply-xorshift step per
// 64-bit word.  Equal patterns give equal hashes; the cache also compares the sizes, base and
// storage.
uint64_t pattern_hash(const std::vector<int64_t> &rp, const std::vector<int> &ci) {
    uint64_t h = 0x243F6A8885A308D3ull;
    auto step = [&](uint64_t w) {
        h = (h ^ w) * 0xBF58476D1CE4E5B9ull;
        h ^= h >> 29;
    };
    for (int64_t v : rp) step((uint64_t)v);
    size_t i = 0;
    for (; i + 1 < ci.size(); i += 2) step((uint64_t)(uint32_t)ci[i] | ((uint64_t)(uint32_t)ci[i + 1] << 32));
    if (i < ci.size()) step((uint64_t)(uint32_t)ci[i] | (1ull << 63));
    step((uint64_t)ci.size());
    return h;
}

// The factorisation context shared by the Krylov basis and the full-order sweep: the pattern
// (full symmetric, on host and device), its RCM order, the band factor and its panels, and the
// split-k workspace of the complex GEMMs.  The device buffers are released after the stream
// drains.
struct BandContext {
    Bufs B;
    cudaStream_t st = nullptr;
    int64_t n = 0;
    std::vector<int64_t> frp, fmap;
    std::vector<int> fci, perm, iperm;
    int64_t *d_frp = nullptr, *d_fmap = nullptr;
    int *d_fci = nullptr, *d_iperm = nullptr;
    double *d_nrm = nullptr;
    BandLDLT F;

    // The pattern's full symmetric form and RCM order: from the handle's cache when it holds
    // this pattern, else computed on the host and uploaded (into the cache when there is one).
    int init(cudaStream_t stream, int64_t n_rows, int64_t nnz, const int64_t *rowptr, const int *colind, int base,
             int upper, PatternCache *cache, Err &E) {
        st = stream;
        n = n_rows;
        B.st = st;
        std::vector<int64_t> rp(n + 1);
        std::vector<int> ci(nnz);
        KCU(cudaMemcpyAsync(rp.data(), rowptr, sizeof(int64_t) * (n + 1), cudaMemcpyDeviceToHost, st));
        if (nnz > 0) KCU(cudaMemcpyAsync(ci.data(), colind, sizeof(int) * nnz, cudaMemcpyDeviceToHost, st));
        KCU(cudaStreamSynchronize(st));
        if (rp[0] != base || rp[n] - base != nnz)
            return E.set(SROM_ERR_INVALID, "rowptr does not start at base or does not end at base + nnz");
        const uint64_t hsh = pattern_hash(rp, ci);
        const bool reuse = cache && cache->matches(n, nnz, base, upper, hsh);
        int64_t bw = 0, nfull = 0;
        if (reuse) {
            bw = cache->bw;
            nfull = cache->nfull;
        } else {
            std::string err;
            int s = full_pattern(n, nnz, rp.data(), ci.data(), base, upper, frp, fci, fmap, &err);
            if (s) return E.set(s, err);
            bw = rcm_order(n, frp, fci, perm);
            iperm.assign(n, 0);
            for (int64_t k = 0; k < n; ++k) iperm[perm[k]] = (int)k;
            nfull = frp[n];
        }
        if (cache) cache->last_reused = reuse;
        F.n = n;
        F.bw = bw;
        F.ldab = bw + 2 * NB + 1;
        F.ldw = (int)(2 * bw + NB);
        F.st = st;
        auto need = [&](cudaError_t e, const char *what) {
            if (e != cudaSuccess)
                E.set(e == cudaErrorMemoryAllocation ? SROM_ERR_ALLOC : SROM_ERR_CUDA,
                      std::string("allocating ") + what + " (" + std::to_string(band_bytes(n, bw)) +
                          " bytes for the band): " + cudaGetErrorString(e));
            return e == cudaSuccess;
        };
        if (!need(B.alloc(&F.band, (size_t)(n + 2 * NB) * F.ldab), "the band factor") ||
            !need(B.alloc(&F.W, (size_t)F.ldw * NB), "the panel") ||
            !need(B.alloc(&F.Lp, (size_t)F.ldw * NB), "the panel") || !need(B.alloc(&F.d_info, 1), "info"))
            return E.code;
        if (reuse) {
            d_frp = cache->d_frp;
            d_fci = cache->d_fci;
            d_fmap = cache->d_fmap;
            d_iperm = cache->d_iperm;
        } else if (cache) {
            // a different pattern replaces the cached one (the previous call has drained the stream)
            cache->release();
            auto dev = [&](void **p, size_t bytes, const char *what) {
                const cudaError_t e = cudaMalloc(p, std::max<size_t>(bytes, 1));
                if (e != cudaSuccess) {
                    *p = nullptr;
                    E.set(e == cudaErrorMemoryAllocation ? SROM_ERR_ALLOC : SROM_ERR_CUDA,
                          std::string("allocating ") + what + ": " + cudaGetErrorString(e));
                }
                return e == cudaSuccess;
            };
            if (!dev(reinterpret_cast<void **>(&cache->d_frp), sizeof(int64_t) * (n + 1), "the pattern") ||
                !dev(reinterpret_cast<void **>(&cache->d_fci), sizeof(int) * nfull, "the pattern") ||
                !dev(reinterpret_cast<void **>(&cache->d_fmap), sizeof(int64_t) * nfull, "the pattern") ||
                !dev(reinterpret_cast<void **>(&cache->d_iperm), sizeof(int) * n, "the ordering")) {
                cache->release();
                return E.code;
            }
            d_frp = cache->d_frp;
            d_fci = cache->d_fci;
            d_fmap = cache->d_fmap;
            d_iperm = cache->d_iperm;
        } else if (!need(B.alloc(&d_frp, n + 1), "the pattern") || !need(B.alloc(&d_fci, nfull), "the pattern") ||
                   !need(B.alloc(&d_fmap, nfull), "the pattern") || !need(B.alloc(&d_iperm, n), "the ordering")) {
            return E.code;
        }
        {
            int dev = 0;
            KCU(cudaGetDevice(&dev));
            KCU(cudaDeviceGetAttribute(&F.sms, cudaDevAttrMultiProcessorCount, dev));
        }
        // split-k partials: at most (2 SMs' worth + the tiles) 64 x 64 blocks
        F.zwork_elems = (int64_t)(4 * F.sms + 64) * 64 * 64;
        if (!need(B.alloc(&F.zwork, (size_t)F.zwork_elems), "the GEMM workspace") ||
            !need(B.alloc(&d_nrm, znorm2_work_doubles() + 2), "the norm workspace") ||
            !need(B.alloc(&F.d_anorm, 1), "the pivot statistics") || !need(B.alloc(&F.d_minr, 1), "the pivot statistics") ||
            !need(B.alloc(&F.d_pert, 1), "the pivot statistics"))
            return E.code;
        const size_t smem = sizeof(double2) * NB * SLD;
        KCU(cudaFuncSetAttribute(ldlt_diag_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        KCU(cudaFuncSetAttribute(ldlt_panel_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)(smem + sizeof(double2) * NB)));
        KCU(cudaFuncSetAttribute(trsv_block_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        if (!reuse) {
            KCU(cudaMemcpyAsync(d_frp, frp.data(), sizeof(int64_t) * (n + 1), cudaMemcpyHostToDevice, st));
            KCU(cudaMemcpyAsync(d_fci, fci.data(), sizeof(int) * nfull, cudaMemcpyHostToDevice, st));
            KCU(cudaMemcpyAsync(d_fmap, fmap.data(), sizeof(int64_t) * nfull, cudaMemcpyHostToDevice, st));
            KCU(cudaMemcpyAsync(d_iperm, iperm.data(), sizeof(int) * n, cudaMemcpyHostToDevice, st));
            if (cache) {
                cache->n = n;
                cache->nnz = nnz;
                cache->base = base;
                cache->upper = upper;
                cache->hash = hsh;
                cache->bw = bw;
                cache->nfull = nfull;
            }
        }
        KCU(cudaMemsetAsync(F.W, 0, sizeof(double2) * F.ldw * NB, st));
        KCU(cudaMemsetAsync(F.Lp, 0, sizeof(double2) * F.ldw * NB, st));
        return SROM_OK;
    }

    // sign * (K - w^2 M + i w D) into the band, then L D L^T
    int assemble_factor(const void *K, const void *M, const void *D, double w, double sign, Err &E) {
        KCU(cudaMemsetAsync(F.band, 0, sizeof(double2) * (size_t)(n + 2 * NB) * F.ldab, st));
        KCU(cudaMemsetAsync(F.d_anorm, 0, sizeof(unsigned long long), st));
        scatter_band_kernel<<<grid_for(n * 32, KT), KT, 0, st>>>(
            n, d_frp, d_fci, d_fmap, reinterpret_cast<const double2 *>(K), reinterpret_cast<const double2 *>(M),
            reinterpret_cast<const double2 *>(D), w, sign, d_iperm, F.band, F.ldab, F.d_anorm);
        KCU(cudaGetLastError());
        return F.factor(E);
    }

    // Y (n x m, ldy) = A^-1 X (n x m, ldx) with the current factor; work: n x m scratch
    int solve(const double2 *X, int64_t ldx, double2 *Y, int64_t ldy, int m, double2 *work, Err &E) {
        permute_kernel<<<grid_for(n * m, KT), KT, 0, st>>>(n, m, d_iperm, X, ldx, work, n, 1);
        int s = F.solve(work, n, m, E);
        if (s) return s;
        permute_kernel<<<grid_for(n * m, KT), KT, 0, st>>>(n, m, d_iperm, work, n, Y, ldy, 0);
        KCU(cudaGetLastError());
        return SROM_OK;
    }
};

}  // namespace

int krylov_basis(const KrylovArgs &a, std::string *msg, int *n_cols, KrylovLog *log) {
    Err E;
    *n_cols = 0;
    if (log) log->blocks.clear();
    if (a.n_rows == 0 || a.n_in == 0 || a.n_points == 0) return SROM_OK;
    BandContext X;
    if (X.init(a.stream, a.n_rows, a.nnz, a.rowptr, a.colind, a.base, a.upper, a.cache, E)) {
        *msg = E.msg;
        return E.code;
    }
    if (log) log->bandwidth = X.F.bw;
    X.F.stats = a.stats;
    cudaStream_t st = a.stream;
    const int64_t n = a.n_rows;
    const int mmax = std::max(a.n_in, 1);
    double2 *Q = nullptr, *U = nullptr, *Qo = nullptr, *S = nullptr, *d_w = nullptr, *work = nullptr;
    double *d_norms = nullptr;
    for (auto e : {X.B.alloc(&Q, (size_t)n * mmax), X.B.alloc(&U, (size_t)n * mmax), X.B.alloc(&Qo, (size_t)n * mmax),
                   X.B.alloc(&work, (size_t)n * mmax), X.B.alloc(&S, (size_t)std::max(a.max_cols, 1) * mmax),
                   X.B.alloc(&d_w, mmax), X.B.alloc(&d_norms, mmax)})
        if (e != cudaSuccess) {
            *msg = std::string("allocating the Krylov blocks: ") + cudaGetErrorString(e);
            return e == cudaErrorMemoryAllocation ? SROM_ERR_ALLOC : SROM_ERR_CUDA;
        }
    auto run = [&]() -> int {
        int kv = 0;  // columns of V so far
        std::vector<double> rdiag;
        for (int ip = 0; ip < a.n_points; ++ip) {
            const double w = 2.0 * 3.141592653589793 * a.exp_points_hz[ip];
            // K~ = -(K - w^2 M + i w D)
            int s = X.assemble_factor(a.K, a.M, a.D, w, -1.0, E);
            if (s) return s;
            int m = a.n_in;
            s = X.solve(reinterpret_cast<const double2 *>(a.B), a.ldb, Q, n, m, work, E);  // Q = K~^-1 B
            if (s) return s;
            for (int order = 1; order <= a.order; ++order) {
                if (order > 1) {
                    // Q = K~^-1 (M Q)
                    csr_spmm_complex_kernel<<<grid_for(n * 32, KT), KT, 0, st>>>(
                        n, X.d_frp, X.d_fci, X.d_fmap, reinterpret_cast<const double2 *>(a.M), Qo, n, m, U, n);
                    s = X.solve(U, n, Q, n, m, work, E);
                    if (s) return s;
                }
                if (ip > 0 || order > 1) {
                    s = reorthogonalize(X.F, st, reinterpret_cast<const double2 *>(a.V), a.ldv, kv, Q, U, n, m, S,
                                        X.d_nrm, E);
                    if (s) return s;
                }
                int rr = 0;
                s = pivoted_qr(st, Q, n, m, a.tol, Qo, d_norms, d_w, rdiag, rr, E);
                if (s) return s;
                if (log) log->blocks.push_back({a.exp_points_hz[ip], order, rr, rdiag});
                if (rr == 0) break;
                if (kv + rr > a.max_cols)
                    return E.set(SROM_ERR_INVALID, "the basis needs more than max_cols = " + std::to_string(a.max_cols) +
                                                       " columns");
                KCU(cudaMemcpy2DAsync(reinterpret_cast<double2 *>(a.V) + (int64_t)kv * a.ldv, sizeof(double2) * a.ldv, Qo,
                                      sizeof(double2) * n, sizeof(double2) * n, rr, cudaMemcpyDeviceToDevice, st));
                kv += rr;
                *n_cols = kv;
                m = rr;
            }
        }
        KCU(cudaStreamSynchronize(st));
        return SROM_OK;
    };
    const int s = run();
    if (s) *msg = E.msg;
    return s;
}

int fom_sweep(const FomArgs &a, std::string *msg) {
    Err E;
    if (a.n_rows == 0 || a.r == 0 || a.n_freq == 0) return SROM_OK;
    BandContext X;
    if (X.init(a.stream, a.n_rows, a.nnz, a.rowptr, a.colind, a.base, a.upper, a.cache, E)) {
        *msg = E.msg;
        return E.code;
    }
    X.F.stats = a.stats;
    double2 *work = nullptr;
    cudaError_t e = X.B.alloc(&work, (size_t)a.n_rows * a.r);
    if (e != cudaSuccess) {
        *msg = std::string("allocating the solve block: ") + cudaGetErrorString(e);
        return e == cudaErrorMemoryAllocation ? SROM_ERR_ALLOC : SROM_ERR_CUDA;
    }
    auto run = [&]() -> int {
        for (int f = 0; f < a.n_freq; ++f) {
            const double w = 2.0 * 3.141592653589793 * a.freq_hz[f];
            int s = X.assemble_factor(a.K, a.M, a.D, w, 1.0, E);  // K - w^2 M + i w D
            if (s) return E.set(s, "frequency " + std::to_string(f) + ": " + E.msg);
            double2 *Xf = reinterpret_cast<double2 *>(a.X) + (int64_t)f * a.ldx * a.r;
            s = X.solve(reinterpret_cast<const double2 *>(a.F), a.ldf, Xf, a.ldx, a.r, work, E);
            if (s) return s;
        }
        KCU(cudaStreamSynchronize(a.stream));
        return SROM_OK;
    };
    const int s = run();
    if (s) *msg = E.msg;
    return s;
}

}  // namespace kry
}  // namespace srom
