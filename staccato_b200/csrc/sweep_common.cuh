// Device code shared by the sweep kernels (sweep.cu: CUDA-core LU; sweep_tc.cu: tensor-core
// Schur updates): persistent work distribution, assembly, the partial-pivot panel
// factorisation and the mixed form's FP64 refinement (residual, correction solve, update).
#pragma once

#include <climits>
#include <type_traits>

#include "srom_device.cuh"
#include "sweep_kernels.h"

namespace srom {

constexpr int NT = 256;
constexpr int NW = NT / 32;
constexpr int CWG = 8;     // trailing columns per warp group
constexpr int NB64 = 16;   // FP64 panel width
constexpr int NB32 = 32;   // FP32 panel width
constexpr int RMAX_SOLVE = 16;  // right-hand sides per solve (register accumulators)

// Asynchronous global -> shared copies (each thread stages only the values it will use).
template <typename T>
__device__ __forceinline__ void cp_async_elem(T *dst, const T *src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    if constexpr (sizeof(T) == 16)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src));
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N)); }
// wait_group takes an immediate: a runtime pending count (clamped to 0..15) picks the case.
__device__ __forceinline__ void cp_async_wait_dyn(int n) {
    switch (n <= 0 ? 0 : (n > 15 ? 15 : n)) {
        case 0: cp_async_wait<0>(); break;
        case 1: cp_async_wait<1>(); break;
        case 2: cp_async_wait<2>(); break;
        case 3: cp_async_wait<3>(); break;
        case 4: cp_async_wait<4>(); break;
        case 5: cp_async_wait<5>(); break;
        case 6: cp_async_wait<6>(); break;
        case 7: cp_async_wait<7>(); break;
        case 8: cp_async_wait<8>(); break;
        case 9: cp_async_wait<9>(); break;
        case 10: cp_async_wait<10>(); break;
        case 11: cp_async_wait<11>(); break;
        case 12: cp_async_wait<12>(); break;
        case 13: cp_async_wait<13>(); break;
        case 14: cp_async_wait<14>(); break;
        default: cp_async_wait<15>(); break;
    }
}

__device__ __forceinline__ int next_item(int *counter, int *s_item) {
    if (threadIdx.x == 0) *s_item = atomicAdd(counter, 1);
    __syncthreads();
    int it = *s_item;
    __syncthreads();
    return it;
}

// Start of a CTA's sweep over the columns of a ROM's K, M, D (in units of `units` column
// batches): the frequency index spreads it, so that the CTAs sweeping the same ROM at the same
// time read different columns (different L2 slices) instead of all the same ones.
__device__ __forceinline__ int sweep_start(int f, int units) { return units > 0 ? (int)(((unsigned)f * 97u) % (unsigned)units) : 0; }

template <typename T>
__device__ __forceinline__ T to_store(double2 v);
template <>
__device__ __forceinline__ double2 to_store<double2>(double2 v) { return v; }
template <>
__device__ __forceinline__ float2 to_store<float2>(double2 v) {
    return make_float2(__double2float_rn(v.x), __double2float_rn(v.y));
}

// A(w) into A (ld lda), element by element; column j0 = sweep_start(f) first (see there).
template <typename T>
__device__ void assemble_into(T *A, int64_t lda, const RomDev &R, double w, int f) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const double s = -__dmul_rn(w, w);
    const uint64_t pol = l2_keep_policy();
    const int j0 = sweep_start(f, R.n);
    for (int jj = warp; jj < R.n; jj += NW)
        for (int i = lane; i < R.n; i += 32) {
            const int j = jj + j0 < R.n ? jj + j0 : jj + j0 - R.n;
            const int64_t e = i + (int64_t)j * R.ldk;
            A[i + j * lda] = to_store<T>(assemble_entry(ld_keep(R.K + e, pol), ld_keep(R.M + e, pol), R.D, e, R.eta, s, w));
        }
}

static __device__ void load_rhs(double2 *B, int ldbs, const RomDev &R) {
    for (int e = threadIdx.x; e < R.n * R.r; e += NT) {
        const int i = e % R.n, c = e / R.n;
        B[i + (int64_t)c * ldbs] = R.rhs[i + (int64_t)c * R.ldb];
    }
}

static __device__ void store_solution(const double2 *B, int ldbs, const RomDev &R, int f) {
    double2 *X = R.X + (int64_t)f * R.n * R.r;
    for (int e = threadIdx.x; e < R.n * R.r; e += NT) {
        const int i = e % R.n, c = e / R.n;
        X[i + (int64_t)c * R.n] = B[i + (int64_t)c * ldbs];
    }
}

template <typename Rl>
struct PivotXchg {
    Rl val[2][NW];
    int lg[2][NW];
    int ph[2][NW];
    int physjj[2];
    int firstnan[2];
};

struct PanelLists {
    int nmoved;
    int info;
    int grp;  // next trailing column group of the current panel
};

// Factor the m x ncols panel P (physical row order, leading dimension ldp) with partial
// pivoting.  Thread t owns physical rows t + k*NT.  On return s_perm[l] is the physical row
// at logical position l, s_pivlg[jj] the logical row chosen at step jj (LAPACK ipiv - 1,
// relative to the panel), and (s_mdst, s_msrc) list every row whose position changed.
template <typename T, int RPT>
__device__ void panel_factor_par(T *P, int ldp, int m, int ncols, int *s_perm, int *s_pivlg,
                                 int *s_mdst, int *s_msrc, PanelLists &PL, int info_off,
                                 PivotXchg<typename CT<T>::R> &X) {
    using C = CT<T>;
    using Rl = typename C::R;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    int lg[RPT];
    bool done[RPT];
#pragma unroll
    for (int k = 0; k < RPT; ++k) {
        const int ph = tid + k * NT;
        lg[k] = ph;
        done[k] = ph >= m;
    }
    for (int jj = 0; jj < ncols; ++jj) {
        const int buf = jj & 1;
        Rl best = Rl(-1);
        int bl = INT_MAX, bp = -1;
#pragma unroll
        for (int k = 0; k < RPT; ++k) {
            if (done[k]) continue;
            const int ph = tid + k * NT;
            const Rl v = C::abs1(P[ph + (int64_t)jj * ldp]);
            if (v > best || (v == best && lg[k] < bl)) {
                best = v;
                bl = lg[k];
                bp = ph;
            }
            if (lg[k] == jj) {
                X.physjj[buf] = ph;
                X.firstnan[buf] = (v != v);
            }
        }
#pragma unroll
        for (int off = 16; off; off >>= 1) {
            const Rl ob = __shfl_xor_sync(FULL_MASK, best, off);
            const int ol = __shfl_xor_sync(FULL_MASK, bl, off);
            const int op = __shfl_xor_sync(FULL_MASK, bp, off);
            if (ob > best || (ob == best && ol < bl)) {
                best = ob;
                bl = ol;
                bp = op;
            }
        }
        if (lane == 0) {
            X.val[buf][warp] = best;
            X.lg[buf][warp] = bl;
            X.ph[buf][warp] = bp;
        }
        __syncthreads();
        best = X.val[buf][0];
        bl = X.lg[buf][0];
        bp = X.ph[buf][0];
#pragma unroll
        for (int w = 1; w < NW; ++w) {
            const Rl ob = X.val[buf][w];
            const int ol = X.lg[buf][w];
            if (ob > best || (ob == best && ol < bl)) {
                best = ob;
                bl = ol;
                bp = X.ph[buf][w];
            }
        }
        const int physjj = X.physjj[buf];
        // IZAMAX starts from the first entry: a NaN there is the pivot; all-NaN likewise.
        if (X.firstnan[buf] || bp < 0) {
            bp = physjj;
            bl = jj;
        }
        const T piv = P[bp + (int64_t)jj * ldp];
        const bool nz = (piv.x != 0 || piv.y != 0);
        if (!nz) {  // LAPACK interchanges nothing for a zero pivot
            bp = physjj;
            bl = jj;
        }
        if (tid == 0) {
            s_pivlg[jj] = bl;
            if (!nz && PL.info == 0) PL.info = info_off + jj + 1;
        }
        const T inv = nz ? C::recip(piv) : C::zero();
#pragma unroll
        for (int k = 0; k < RPT; ++k) {
            if (done[k]) continue;
            const int ph = tid + k * NT;
            if (ph == bp) {
                done[k] = true;
                lg[k] = jj;
                continue;
            }
            if (ph == physjj) lg[k] = bl;
            T l = P[ph + (int64_t)jj * ldp];
            if (nz) {
                l = C::mul(l, inv);
                P[ph + (int64_t)jj * ldp] = l;
            }
            // rank-1 update of this row, four columns per batch so the shared-memory loads
            // overlap (each entry still receives exactly this column's update)
            int c = jj + 1;
            for (; c + 4 <= ncols; c += 4) {
                T v[4], u[4];
#pragma unroll
                for (int t = 0; t < 4; ++t) {
                    v[t] = P[ph + (int64_t)(c + t) * ldp];
                    u[t] = P[bp + (int64_t)(c + t) * ldp];
                }
#pragma unroll
                for (int t = 0; t < 4; ++t) P[ph + (int64_t)(c + t) * ldp] = C::subm(v[t], l, u[t]);
            }
            for (; c < ncols; ++c)
                P[ph + (int64_t)c * ldp] = C::subm(P[ph + (int64_t)c * ldp], l, P[bp + (int64_t)c * ldp]);
        }
    }
#pragma unroll
    for (int k = 0; k < RPT; ++k) {
        const int ph = tid + k * NT;
        if (ph < m) {
            s_perm[lg[k]] = ph;
            if (lg[k] != ph) {
                const int e = atomicAdd(&PL.nmoved, 1);
                s_mdst[e] = lg[k];
                s_msrc[e] = ph;
            }
        }
    }
    __syncthreads();
}

// r = b - A(w) x in FP64 with A(w) re-assembled from K, M, D (the FP64 assembly arithmetic),
// written permuted and rounded to FP32 into B32 (B32[pos[i]] = r[i]) for the next correction.
// Thread t owns rows t + k*NT; right-hand sides are processed four at a time; the column
// batches are taken cyclically from batch sweep_start(f).
// Only the right-hand sides still refined: column act[c] of x and b gives column c of B32
// (c < ra).
template <int RPT>
__device__ void residual64(const RomDev &R, double w, const double2 *X64, float2 *B32, const int *s_pos, int f,
                           const int *act, int ra) {
    constexpr int JB = RPT >= 3 ? 1 : 4 / RPT;  // columns of K, M, D loaded per batch
    const int tid = threadIdx.x;
    const int n = R.n;
    const int nbat = (n + JB - 1) / JB, b0 = sweep_start(f, nbat);
    const double s = -__dmul_rn(w, w);
    const uint64_t pol = l2_keep_policy();
    for (int c0 = 0; c0 < ra; c0 += 4) {
        const int nc = min(4, ra - c0);
        int col[4];
#pragma unroll
        for (int cc = 0; cc < 4; ++cc) col[cc] = cc < nc ? act[c0 + cc] : 0;
        double2 acc[RPT][4];
#pragma unroll
        for (int k = 0; k < RPT; ++k) {
            const int i = tid + k * NT;
#pragma unroll
            for (int cc = 0; cc < 4; ++cc)
                acc[k][cc] = (i < n && cc < nc) ? R.rhs[i + (int64_t)col[cc] * R.ldb] : make_double2(0.0, 0.0);
        }
        for (int bt = 0; bt < nbat; ++bt) {
            const int bb = b0 + bt, j0 = (bb < nbat ? bb : bb - nbat) * JB;
            double2 kv[RPT][JB], mv[RPT][JB], dv[RPT][JB];
#pragma unroll
            for (int k = 0; k < RPT; ++k) {
                const int i = tid + k * NT;
#pragma unroll
                for (int jj = 0; jj < JB; ++jj) {
                    if (i < n && j0 + jj < n) {
                        const int64_t e = i + (int64_t)(j0 + jj) * R.ldk;
                        kv[k][jj] = ld_keep(R.K + e, pol);
                        mv[k][jj] = ld_keep(R.M + e, pol);
                        dv[k][jj] = R.D ? ld_keep(R.D + e, pol) : make_double2(0.0, 0.0);
                    }
                }
            }
#pragma unroll
            for (int jj = 0; jj < JB; ++jj) {
                const int j = j0 + jj;
                if (j >= n) break;
                double2 xj[4];
#pragma unroll
                for (int cc = 0; cc < 4; ++cc)
                    xj[cc] = cc < nc ? X64[j + (int64_t)col[cc] * n] : make_double2(0.0, 0.0);
#pragma unroll
                for (int k = 0; k < RPT; ++k) {
                    const int i = tid + k * NT;
                    if (i < n) {
                        double2 kk = kv[k][jj];
                        if (R.eta != 0.0) {
                            const double t1 = __dmul_rn(R.eta, kk.y), t2 = __dmul_rn(R.eta, kk.x);
                            kk.x = __dsub_rn(kk.x, t1);
                            kk.y = __dadd_rn(kk.y, t2);
                        }
                        double2 a;
                        a.x = __dadd_rn(kk.x, __dmul_rn(s, mv[k][jj].x));
                        a.y = __dadd_rn(kk.y, __dmul_rn(s, mv[k][jj].y));
                        if (R.D) {
                            a.x = __dsub_rn(a.x, __dmul_rn(w, dv[k][jj].y));
                            a.y = __dadd_rn(a.y, __dmul_rn(w, dv[k][jj].x));
                        }
#pragma unroll
                        for (int cc = 0; cc < 4; ++cc) acc[k][cc] = csubmul(acc[k][cc], a, xj[cc]);
                    }
                }
            }
        }
#pragma unroll
        for (int k = 0; k < RPT; ++k) {
            const int i = tid + k * NT;
            if (i < n) {
#pragma unroll
                for (int cc = 0; cc < 4; ++cc)
                    if (cc < nc)
                        B32[s_pos[i] + (int64_t)(c0 + cc) * n] =
                            make_float2(__double2float_rn(acc[k][cc].x), __double2float_rn(acc[k][cc].y));
            }
        }
    }
    __syncthreads();
}

// x += d (FP32 correction) and, per right-hand side, the relative correction size
// ||d||_2 / ||x||_2 into s_dx; one warp per right-hand side.  The 2-norm is the norm of the
// accuracy criterion (relative 2-norm error per system): with max norms the estimate missed
// errors spread over many entries of a solution dominated by a few (near resonance).
// Column c of B32 (c < ra) corrects column act[c] of X.
static __device__ void apply_correction(double2 *X, const float2 *B32, int n, const int *act, int ra, double *s_dx) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int c = warp; c < ra; c += NW) {
        double dm = 0.0, xm = 0.0;
        const int col = act[c];
        for (int i = lane; i < n; i += 32) {
            const float2 d = B32[i + (int64_t)c * n];
            double2 &x = X[i + (int64_t)col * n];
            x.x += (double)d.x;
            x.y += (double)d.y;
            dm = fma((double)d.x, (double)d.x, fma((double)d.y, (double)d.y, dm));
            xm = fma(x.x, x.x, fma(x.y, x.y, xm));
        }
#pragma unroll
        for (int off = 16; off; off >>= 1) {
            dm += __shfl_xor_sync(FULL_MASK, dm, off);
            xm += __shfl_xor_sync(FULL_MASK, xm, off);
        }
        if (lane == 0) s_dx[c] = xm > 0.0 ? sqrt(dm / xm) : (dm > 0.0 ? INFINITY : 0.0);
    }
    __syncthreads();
}

// Correction solve of the mixed form: LU x = b with the complex-FP32 factor in global memory
// (ld lda) and b (n x nrhs, ld n, interchanges applied) in shared memory.  The factor is read
// strip by strip (SW columns; the forward strips from the first, then the backward ones from
// the last), each strip through one slot of a ring of ns shared-memory slots, so that up to
// ns - 1 strips' loads are in flight while one is processed.  Each thread copies the rows it
// will update itself; the strip's diagonal block, copied by its rows' owners, is read by the
// triangle after a barrier.  One warp per right-hand side solves the triangle (the backward
// one multiplies by the reciprocals of U's diagonal), then every thread updates its rows.
template <int SW, int RPT>
__device__ void lu_solve_ring(const float2 *A, int n, int64_t lda, float2 *B, int nrhs, unsigned char *ring, int ring_bytes,
                              const float2 *dinv) {
    using C = CT<float2>;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int nblk = (n + SW - 1) / SW;
    const int slot = SW * n;  // S[j * n + r] = A[r, jb + j]
    const int ns = min(8, ring_bytes / (slot * 8));
    float2 *S0 = reinterpret_cast<float2 *>(ring);
    const int total = 2 * nblk;
    auto range = [&](int s, int &jb, int &bs) {
        if (s < nblk) {
            jb = s * SW;
            bs = min(SW, n - jb);
        } else {
            const int jend = n - (s - nblk) * SW;
            jb = max(jend - SW, 0);
            bs = jend - jb;
        }
    };
    auto issue = [&](int s) {
        if (s < total) {
            int jb, bs;
            range(s, jb, bs);
            const int lo = s < nblk ? jb : 0, hi = s < nblk ? n : jb + bs;
            float2 *d = S0 + (s % ns) * slot;
#pragma unroll
            for (int k = 0; k < RPT; ++k) {
                const int r = tid + k * NT;
                if (r >= lo && r < hi)
                    for (int j = 0; j < bs; ++j) cp_async_elem(d + j * n + r, A + r + (int64_t)(jb + j) * lda);
            }
        }
        cp_async_commit();
    };
    for (int s = 0; s < ns - 1; ++s) issue(s);
    for (int s = 0; s < total; ++s) {
        asm volatile("" ::: "memory");
        issue(s + ns - 1);
        cp_async_wait_dyn(ns - 1);
        __syncthreads();
        int jb, bs;
        range(s, jb, bs);
        const bool fwd = s < nblk;
        const float2 *S = S0 + (s % ns) * slot;
        for (int c = warp; c < nrhs; c += NW) {
            float2 *b = B + (int64_t)c * n + jb;
            float2 v = lane < bs ? b[lane] : C::zero();
            if (fwd) {
                for (int j = 0; j < bs; ++j) {
                    const float2 bj = C::shfl(v, j, 32);
                    if (lane > j && lane < bs) v = C::subm(v, S[j * n + jb + lane], bj);
                }
            } else {
                for (int j = bs - 1; j >= 0; --j) {
                    if (lane == j) v = C::mul(v, dinv[jb + j]);
                    const float2 bj = C::shfl(v, j, 32);
                    if (lane < j) v = C::subm(v, S[j * n + jb + lane], bj);
                }
            }
            if (lane < bs) b[lane] = v;
        }
        __syncthreads();
        const int lo = fwd ? jb + bs : 0, hi = fwd ? n : jb;
#pragma unroll
        for (int k = 0; k < RPT; ++k) {
            const int r = tid + k * NT;
            if (r >= lo && r < hi) {
                for (int c0 = 0; c0 < nrhs; c0 += 4) {
                    const int nc = min(4, nrhs - c0);
                    float2 acc[4];
#pragma unroll
                    for (int cc = 0; cc < 4; ++cc) acc[cc] = cc < nc ? B[r + (int64_t)(c0 + cc) * n] : C::zero();
#pragma unroll
                    for (int j = 0; j < SW; ++j) {
                        if (j < bs) {
                            const float2 a = S[j * n + r];
#pragma unroll
                            for (int cc = 0; cc < 4; ++cc)
                                if (cc < nc) acc[cc] = C::subm(acc[cc], a, B[jb + j + (int64_t)(c0 + cc) * n]);
                        }
                    }
#pragma unroll
                    for (int cc = 0; cc < 4; ++cc)
                        if (cc < nc) B[r + (int64_t)(c0 + cc) * n] = acc[cc];
                }
            }
        }
    }
    cp_async_wait<0>();
    __syncthreads();
}

// Strips of 16 columns: the ring (at least the u and panel regions, 16 KB + 256 ldp bytes)
// always holds two of them; with fewer, wider strips the triangles and barriers cost less than
// narrower strips gain in depth (measured at n = 128..512).
template <int RPT>
__device__ void solve_ring(const float2 *A, int n, int64_t lda, float2 *B, int nrhs, unsigned char *ring, int ring_bytes,
                           const float2 *dinv) {
    lu_solve_ring<16, RPT>(A, n, lda, B, nrhs, ring, ring_bytes, dinv);
}

constexpr int RMAX_MIXED = 16;
constexpr int SROM_INFO_NOT_CONVERGED_DEV = -1;

// Columns per cp.async batch in the solves: two batches of NT rows fit the panel region.
template <typename T>
__host__ __device__ constexpr int stage_cb(int ldp) {
    const int cb = (int)(((size_t)ldp * 256) / (2 * NT * sizeof(T)));
    return cb < 1 ? 1 : (cb > 32 ? 32 : cb);
}

// Work areas of the mixed forms' refinement (shared memory unless noted).
struct MixedWork {
    double2 *X;            // n x r FP64 iterate (ld n)
    float2 *B32;           // n x r FP32 right-hand side / correction, rows in the factor's order
    int *s_pos;            // s_pos[original row] = row of the factor
    const int *s_ptot;     // s_ptot[row of the factor] = original row
    float2 *s_dinv;        // reciprocals of diag(U)
    unsigned char *ring;   // staging ring of the correction solves
    int ring_bytes;
    double *s_dx;          // per right-hand side relative correction size
    int lda;               // leading dimension of the factor
};

// Correction solve of the CUDA-core mixed kernel: the factor streamed through the strip ring.
template <int RPT>
struct RingSolve {
    const float2 *A;
    int n, lda;
    unsigned char *ring;
    int ring_bytes;
    const float2 *dinv;
    __device__ void operator()(float2 *B, int nrhs) const { solve_ring<RPT>(A, n, lda, B, nrhs, ring, ring_bytes, dinv); }
};

// Refinement of one system after its complex-FP32 factorisation (A32, ld n, LAPACK layout with
// rows in the factor's order; info = the factorisation's zero-pivot report): x_0 from the FP32
// factors, then r = b - A(w) x in FP64 and x += LU \ r (solve(B32, k) replaces the k right-hand
// sides in B32 by their corrections).  Each right-hand side stops on its own once its predicted
// error c rho ||d_s|| / ||x||, rho = ||d_s|| / ||d_s-1|| (c = 2; after the first correction,
// where d_0 = x, c = 4), is at most tol (default 2^-34): later residuals and solves carry only
// the columns still refined.  At most max_refine corrections.  Non-converged systems are
// appended to the FP64 fallback list when one is given (write_status = false: that launch
// writes the results).
template <int RPT, class Solve>
__device__ void mixed_refine(const GlobalArgs &a, const RomDev &R, const Item &wi, double w, const float2 *A32,
                             const MixedWork &W, const Solve &solve, int &info, int &steps, double &berr,
                             bool &write_status) {
    __shared__ int s_act[RMAX_MIXED];       // right-hand sides still refined
    __shared__ double s_prev[RMAX_MIXED];   // their previous relative correction size
    __shared__ double s_be[RMAX_MIXED];     // latest error estimate of every right-hand side
    __shared__ int s_ra, s_state;           // active count; 1 converged, 2 hopeless
    const int tid = threadIdx.x;
    const int n = R.n;
    for (int l = tid; l < n; l += NT) {
        W.s_pos[W.s_ptot[l]] = l;
        W.s_dinv[l] = CT<float2>::recip(A32[l + (int64_t)l * W.lda]);
    }
    if (tid < R.r) {
        s_act[tid] = tid;
        s_prev[tid] = 1.0;  // the first correction is x itself
        s_be[tid] = 0.0;
    }
    if (tid == 0) {
        s_ra = R.r;
        s_state = 0;
    }
    __syncthreads();
    for (int e = tid; e < n * R.r; e += NT) {
        const int i = e % n, c = e / n;
        W.X[i + (int64_t)c * n] = make_double2(0.0, 0.0);
        const double2 b = R.rhs[i + (int64_t)c * R.ldb];
        W.B32[W.s_pos[i] + (int64_t)c * n] = make_float2(__double2float_rn(b.x), __double2float_rn(b.y));
    }
    __syncthreads();
    const double tol_x = a.tol > 0.0 ? a.tol : 5.820766091346741e-11;  // 2^-34
    for (int s = 0;; ++s) {
        const int ra = s_ra;
        if (s > 0) residual64<RPT>(R, w, W.X, W.B32, W.s_pos, wi.f, s_act, ra);
        solve(W.B32, ra);
        apply_correction(W.X, W.B32, n, s_act, ra, W.s_dx);
        if (s > 0 && tid == 0) {
            // error left after this correction ~ rho ||d||, rho ~ ||d_s|| / ||d_s-1|| (the
            // contraction), taken twice for safety; after the first correction the ratio is
            // ||d_1|| / ||x||, the relative error of the first solve, a weaker stand-in for
            // the contraction: taken four times.  With the FP64 fallback on, a column whose
            // measured contraction (no safety factor) cannot reach tol in the steps left makes
            // the system hopeless: its corrections would be discarded by the re-solve anyway.
            int keep = 0;
            bool hopeless = false;
            for (int c = 0; c < ra; ++c) {
                const int col = s_act[c];
                const double dx = W.s_dx[c], ratio = dx / s_prev[col];
                const double be = dx * fmin(1.0, (s == 1 ? 4.0 : 2.0) * ratio);
                s_be[col] = be;
                s_prev[col] = dx;
                if (be <= tol_x) continue;
                if (a.fb_items && s >= 2 && s < a.max_refine) {
                    double pred = dx * ratio;
                    for (int k = s; k < a.max_refine && pred > tol_x; ++k) pred *= ratio;
                    hopeless = hopeless || ratio >= 1.0 || pred > tol_x;
                }
                s_act[keep++] = col;  // keep < = c: compaction in place
            }
            s_ra = keep;
            s_state = keep == 0 ? 1 : (hopeless ? 2 : 0);
        }
        __syncthreads();
        steps = s;
        if (s_state != 0 || s >= a.max_refine) break;
    }
    const bool conv = s_state == 1;
    berr = 0.0;
    for (int c = 0; c < R.r; ++c) berr = fmax(berr, s_be[c]);
    if (!conv && a.fb_items) {
        // re-solved by the FP64 kernel that runs after this one; it writes X and status
        if (tid == 0) a.fb_items[atomicAdd(a.fb_count, 1)] = wi;
        write_status = false;
    } else {
        store_solution(W.X, n, R, wi.f);
        if (!conv) info = info == 0 ? SROM_INFO_NOT_CONVERGED_DEV : info;
    }
}


}  // namespace srom
