// Complex FP64 GEMM on the FP64 tensor cores (mma.sync m8n8k4 f64), strided batched, with an
// optional deterministic split over k.  It serves the band LDL^T solver behind the Krylov basis
// and the full-order sweep (trailing updates, solve updates, block re-orthogonalisation) and
// the batched products of the substructure coupling, in place of cuBLAS ZGEMM.
//
// C[b] = alpha op(A[b]) op(B[b]) + beta C[b], column-major, op in {N, T, C}.  A CTA computes a
// 64 x 64 complex tile of C with four warps (2 x 2, each 32 x 32 = 4 x 4 tiles of 8 x 8).  The
// complex product is four real MMAs per 8 x 8 x 4 block (4M: Cr += Ar Br - Ai Bi, Ci += Ar Bi +
// Ai Br).  Operands move by 16-byte cp.async (one complex entry each, transposed in the copy
// where the operand is stored along k) into a four-deep ring of shared-memory stages of 8 k
// (A as [k][64 rows], B as [k][64 columns], complex interleaved); conjugation is applied when
// the fragments are read.  A fragment load (eight consecutive entries on each of four k-rows)
// takes the minimum four shared-memory wavefronts.
//
// Summation order: every C entry accumulates its k terms in a fixed order (chunks of four k in
// increasing k, the real-by-real products of a chunk before the imaginary-by-imaginary ones);
// with a split over k the partial sums are added in split order by the reduction kernel, so
// results are deterministic.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "zgemm.h"

namespace srom {

namespace {

constexpr int ZG_BM = 64, ZG_BN = 64, ZG_BK = 8;
constexpr int ZG_STAGES = 4;                          // cp.async pipeline depth
constexpr int ZG_TILE = ZG_BK * 64;                   // complex entries of one staged A or B tile
constexpr size_t ZG_SMEM = sizeof(double2) * 2 * ZG_TILE * ZG_STAGES;
constexpr int64_t ZG_SHORT_K = 128;                   // k per CTA up to which eight warps are used

struct ZgArgs {
    int m, n, k, opa, opb, beta_zero, splits;
    int64_t kchunk;
    double2 alpha, beta;
    const double2 *A;
    int64_t lda, sa;
    const double2 *B;
    int64_t ldb, sb;
    double2 *C;
    int64_t ldc, sc;
    double2 *work;  // splits > 1: partials [split][batch][m x n]
    int batch;
};

// not volatile: the compiler may interleave independent MMAs (the accumulator operands order
// the dependent ones)
__device__ __forceinline__ void dmma(double &c0, double &c1, double a, double b) {
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};"
        : "+d"(c0), "+d"(c1)
        : "d"(a), "d"(b));
}

// 16-byte cp.async; src_bytes = 0 fills the destination with zeros (rows / k past the end)
__device__ __forceinline__ void cp16(void *dst, const void *src, int src_bytes) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(d), "l"(src), "r"(src_bytes));
}

// Stage element q of this thread (NTH threads, 512 / NTH elements each): A tile (64 rows x 8 k)
// and B tile (8 k x 64 columns).  N-operands of A and T-operands of B are read along the
// 64-long dimension (coalesced), the others along k.
template <int NTH>
__device__ __forceinline__ void a_coords(int opa, int t, int q, int &i, int &kk) {
    if (opa == ZG_N) { i = t & 63; kk = (t >> 6) + (NTH / 64) * q; }
    else { kk = t & 7; i = (t >> 3) + (NTH / 8) * q; }
}
template <int NTH>
__device__ __forceinline__ void b_coords(int opb, int t, int q, int &kk, int &j) {
    if (opb == ZG_N) { kk = t & 7; j = (t >> 3) + (NTH / 8) * q; }
    else { j = t & 63; kk = (t >> 6) + (NTH / 64) * q; }
}

// WN: 8 x 8 tiles per warp along n.  WN = 4: four warps of 32 x 32; WN = 2: eight warps of
// 32 x 16 (half the accumulators a thread, twice the warps an SM: better for short k).
template <int WN>
__global__ void __launch_bounds__(128 * (4 / WN), 2) zgemm_kernel(ZgArgs g) {
    constexpr int NTH = 128 * (4 / WN), PER = 512 / NTH;
    extern __shared__ double2 zs[];  // per stage: A[k][64] then B[k][64], complex interleaved
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int wm = warp & 1, wn = warp >> 1;  // 2 warps along m, NTH / 64 along n
    const int b = blockIdx.z / g.splits, split = blockIdx.z - b * g.splits;
    const int i0 = blockIdx.x * ZG_BM, j0 = blockIdx.y * ZG_BN;
    const int64_t kbeg = (int64_t)split * g.kchunk;
    const int64_t kend = min((int64_t)g.k, kbeg + g.kchunk);
    const double2 *A = g.A + (int64_t)b * g.sa;
    const double2 *B = g.B + (int64_t)b * g.sb;
    const double sga = g.opa == ZG_C ? -1.0 : 1.0, sgb = g.opb == ZG_C ? -1.0 : 1.0;

    // stage s of the k range into buffer s % ZG_STAGES (one commit group per stage, empty ones
    // past the end keep the group count uniform)
    const int nst = kend > kbeg ? (int)((kend - kbeg + ZG_BK - 1) / ZG_BK) : 0;
    auto issue = [&](int s) {
        if (s < nst) {
            double2 *SA = zs + (s % ZG_STAGES) * 2 * ZG_TILE, *SB = SA + ZG_TILE;
            const int64_t k0 = kbeg + (int64_t)s * ZG_BK;
#pragma unroll
            for (int q = 0; q < PER; ++q) {
                int i, kk, j, kb;
                a_coords<NTH>(g.opa, t, q, i, kk);
                const int64_t gi = i0 + i, gk = k0 + kk;
                const bool oka = gi < g.m && gk < kend;
                cp16(SA + kk * 64 + i, oka ? (g.opa == ZG_N ? A + gi + gk * g.lda : A + gk + gi * g.lda) : A, oka ? 16 : 0);
                b_coords<NTH>(g.opb, t, q, kb, j);
                const int64_t gj = j0 + j, gk2 = k0 + kb;
                const bool okb = gj < g.n && gk2 < kend;
                cp16(SB + kb * 64 + j, okb ? (g.opb == ZG_N ? B + gk2 + gj * g.ldb : B + gj + gk2 * g.ldb) : B, okb ? 16 : 0);
            }
        }
        asm volatile("cp.async.commit_group;");
    };

    double cr[4][WN][2], ci[4][WN][2];
#pragma unroll
    for (int x = 0; x < 4; ++x)
#pragma unroll
        for (int y = 0; y < WN; ++y) cr[x][y][0] = cr[x][y][1] = ci[x][y][0] = ci[x][y][1] = 0.0;

#pragma unroll
    for (int s = 0; s < ZG_STAGES - 1; ++s) issue(s);
    for (int s = 0; s < nst; ++s) {
        asm volatile("cp.async.wait_group %0;" ::"n"(ZG_STAGES - 2));
        __syncthreads();  // stage s visible to all; everyone is done with stage s - 1's buffer
        issue(s + ZG_STAGES - 1);
        const double2 *SA = zs + (s % ZG_STAGES) * 2 * ZG_TILE, *SB = SA + ZG_TILE;
#pragma unroll
        for (int k4 = 0; k4 < ZG_BK; k4 += 4) {
            const int kr = (k4 + (lane & 3)) * 64 + (lane >> 2);
            double ar[4], ai[4], nai[4], br[WN], bi[WN];
#pragma unroll
            for (int x = 0; x < 4; ++x) {
                const double2 v = SA[kr + wm * 32 + 8 * x];
                ar[x] = v.x;
                ai[x] = sga * v.y;
                nai[x] = -ai[x];
            }
#pragma unroll
            for (int y = 0; y < WN; ++y) {
                const double2 v = SB[kr + wn * 8 * WN + 8 * y];
                br[y] = v.x;
                bi[y] = sgb * v.y;
            }
            // two passes over the accumulators, so that consecutive MMAs are independent
#pragma unroll
            for (int x = 0; x < 4; ++x)
#pragma unroll
                for (int y = 0; y < WN; ++y) {
                    dmma(cr[x][y][0], cr[x][y][1], ar[x], br[y]);
                    dmma(ci[x][y][0], ci[x][y][1], ar[x], bi[y]);
                }
#pragma unroll
            for (int x = 0; x < 4; ++x)
#pragma unroll
                for (int y = 0; y < WN; ++y) {
                    dmma(cr[x][y][0], cr[x][y][1], nai[x], bi[y]);
                    dmma(ci[x][y][0], ci[x][y][1], ai[x], br[y]);
                }
        }
    }
    asm volatile("cp.async.wait_group 0;");

    // lane holds C[row = lane / 4][col = 2 (lane % 4) + {0, 1}] of each 8 x 8 tile
#pragma unroll
    for (int x = 0; x < 4; ++x)
#pragma unroll
        for (int y = 0; y < WN; ++y)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int gi = i0 + wm * 32 + 8 * x + (lane >> 2);
                const int gj = j0 + wn * 8 * WN + 8 * y + 2 * (lane & 3) + h;
                if (gi >= g.m || gj >= g.n) continue;
                const double vr = cr[x][y][h], vi = ci[x][y][h];
                if (g.splits > 1) {
                    g.work[((int64_t)split * g.batch + b) * g.m * g.n + gi + (int64_t)gj * g.m] = make_double2(vr, vi);
                } else {
                    double2 *c = g.C + (int64_t)b * g.sc + gi + (int64_t)gj * g.ldc;
                    double2 o = make_double2(g.alpha.x * vr - g.alpha.y * vi, g.alpha.x * vi + g.alpha.y * vr);
                    if (!g.beta_zero) {
                        const double2 old = *c;
                        o.x += g.beta.x * old.x - g.beta.y * old.y;
                        o.y += g.beta.x * old.y + g.beta.y * old.x;
                    }
                    *c = o;
                }
            }
}

// C = alpha * (sum of the split partials, in split order) + beta * C
__global__ void zgemm_reduce_kernel(ZgArgs g) {
    const int64_t per = (int64_t)g.m * g.n, tot = per * g.batch;
    for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < tot; e += (int64_t)gridDim.x * blockDim.x) {
        const int64_t b = e / per, r = e - b * per;
        const int64_t i = r % g.m, j = r / g.m;
        double sr = 0.0, si = 0.0;
        for (int s = 0; s < g.splits; ++s) {
            const double2 p = g.work[((int64_t)s * g.batch + b) * per + r];
            sr += p.x;
            si += p.y;
        }
        double2 *c = g.C + b * g.sc + i + j * g.ldc;
        double2 o = make_double2(g.alpha.x * sr - g.alpha.y * si, g.alpha.x * si + g.alpha.y * sr);
        if (!g.beta_zero) {
            const double2 old = *c;
            o.x += g.beta.x * old.x - g.beta.y * old.y;
            o.y += g.beta.x * old.y + g.beta.y * old.x;
        }
        *c = o;
    }
}

constexpr int NRM_THREADS = 256, NRM_BLOCKS = 296;

// per-CTA partial sums of |x_e|^2 over a fixed grid-stride partition, then one CTA adds the
// partials in CTA order (deterministic)
__global__ void __launch_bounds__(NRM_THREADS) znorm2_partial_kernel(const double2 *x, int64_t count, double *part) {
    __shared__ double red[NRM_THREADS / 32];
    double s = 0.0;
    for (int64_t e = (int64_t)blockIdx.x * NRM_THREADS + threadIdx.x; e < count; e += (int64_t)gridDim.x * NRM_THREADS) {
        const double2 v = x[e];
        s = fma(v.x, v.x, fma(v.y, v.y, s));
    }
#pragma unroll
    for (int off = 16; off; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < NRM_THREADS / 32; ++w) t += red[w];
        part[blockIdx.x] = t;
    }
}

__global__ void znorm2_final_kernel(const double *part, int n, double *out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        double t = 0.0;
        for (int i = 0; i < n; ++i) t += part[i];
        *out = sqrt(t);
    }
}

}  // namespace

int64_t zgemm_work_elems(int m, int n, int k, int batch, int sms) {
    const int64_t tiles = (int64_t)((m + ZG_BM - 1) / ZG_BM) * ((n + ZG_BN - 1) / ZG_BN) * batch;
    const int64_t want = 2LL * sms;
    if (tiles >= want || k < 4 * 64) return 0;
    const int64_t splits = std::min<int64_t>((want + tiles - 1) / tiles, k / 64);
    return splits > 1 ? splits * batch * (int64_t)m * n : 0;
}

cudaError_t zgemm(const Zgemm &z, cudaStream_t st) {
    if (z.m <= 0 || z.n <= 0 || z.batch <= 0) return cudaSuccess;
    if (z.opa < ZG_N || z.opa > ZG_C || z.opb < ZG_N || z.opb > ZG_C) return cudaErrorInvalidValue;
    ZgArgs g{};
    g.m = z.m;
    g.n = z.n;
    g.k = std::max(z.k, 0);
    g.opa = z.opa;
    g.opb = z.opb;
    g.alpha = z.alpha;
    g.beta = z.beta;
    g.beta_zero = z.beta.x == 0.0 && z.beta.y == 0.0;
    g.A = z.A;
    g.lda = z.lda;
    g.sa = z.sa;
    g.B = z.B;
    g.ldb = z.ldb;
    g.sb = z.sb;
    g.C = z.C;
    g.ldc = z.ldc;
    g.sc = z.sc;
    g.batch = z.batch;
    g.work = z.work;
    // split over k when the tiles alone cannot fill the GPU and the workspace allows it
    const int64_t tiles = (int64_t)((g.m + ZG_BM - 1) / ZG_BM) * ((g.n + ZG_BN - 1) / ZG_BN) * g.batch;
    int splits = 1;
    if (z.work && z.work_elems > 0 && tiles < 2LL * z.sms && g.k >= 4 * 64) {
        int64_t s = std::min<int64_t>((2LL * z.sms + tiles - 1) / tiles, g.k / 64);
        s = std::min<int64_t>(s, z.work_elems / std::max<int64_t>(1, (int64_t)g.batch * g.m * g.n));
        splits = (int)std::max<int64_t>(1, std::min<int64_t>(s, 1024));
    }
    g.splits = splits;
    g.kchunk = ((int64_t)g.k + splits - 1) / splits;
    g.kchunk = (g.kchunk + ZG_BK - 1) / ZG_BK * ZG_BK;
    if ((int64_t)g.batch * splits > 65535) return cudaErrorInvalidValue;
    dim3 grid((unsigned)((g.m + ZG_BM - 1) / ZG_BM), (unsigned)((g.n + ZG_BN - 1) / ZG_BN), (unsigned)(g.batch * splits));
    // eight warps of 32 x 16 when each CTA has few k stages (their prologue and epilogue then
    // weigh most, and more resident warps overlap them), four of 32 x 32 otherwise
    const bool short_k = g.kchunk <= ZG_SHORT_K;
    auto kf = short_k ? zgemm_kernel<2> : zgemm_kernel<4>;
    cudaError_t ea = cudaFuncSetAttribute(kf, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ZG_SMEM);
    if (ea != cudaSuccess) return ea;
    kf<<<grid, short_k ? 256 : 128, ZG_SMEM, st>>>(g);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess || splits == 1) return e;
    const int64_t tot = (int64_t)g.batch * g.m * g.n;
    zgemm_reduce_kernel<<<(int)std::min<int64_t>((tot + 255) / 256, 4LL * z.sms), 256, 0, st>>>(g);
    return cudaGetLastError();
}

size_t znorm2_work_doubles() { return NRM_BLOCKS + 1; }

cudaError_t znorm2(const double2 *x, int64_t count, double *work, double *out, cudaStream_t st) {
    znorm2_partial_kernel<<<NRM_BLOCKS, NRM_THREADS, 0, st>>>(x, count, work);
    znorm2_final_kernel<<<1, 32, 0, st>>>(work, NRM_BLOCKS, out);
    return cudaGetLastError();
}

}  // namespace srom
