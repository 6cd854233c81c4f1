// Tensor-core form of the mixed-precision sweep (SROM_MIXED_TC).
//
// Same contract as the complex-FP32 global kernel (sweep.cu): one CTA owns one (ROM, frequency)
// system at a time, assembles A(w) in FP64 and rounds it to complex FP32, factors it with
// partial pivoting (LAPACK zgetrf's row order and layout, NB = 32 panels), then refines the
// solution with FP64 residuals (mixed_refine).  What changes is the trailing (Schur) update
// A22 -= L21 U12 of every panel step: it runs on the 5th-generation tensor cores.
//
// Schur update as real GEMMs.  With L21 = Lr + i Li (m x 32) and U12 = Ur + i Ui (32 x c):
//     [Re | Im](L21 U12) = [Lr | Li] * [[Ur, Ui], [-Ui, Ur]]
// i.e. one real GEMM with depth K = 64 whose B operand carries the 4M arrangement, so a tile of
// 128 rows x 32 complex columns is one M = 128, N = 64, K = 64 product whose accumulator
// columns 0..31 hold the real parts and 32..63 the imaginary parts.
//
// FP32 accuracy from bf16 tensor cores.  Every FP32 operand value x is split into three bf16
// pieces x = x0 + x1 + x2, each the round-to-nearest of what the previous ones left; for a
// normal FP32 value the split is exact (8 + 8 + 8 significant bits).  The product is
// accumulated from the six piece products a_i b_j with i + j <= 2, smallest first, into FP32
// accumulators in tensor memory (tcgen05.mma kind::f16, 24 MMAs of 128 x 64 x 16 per tile); the
// dropped terms a_1 b_2, a_2 b_1, a_2 b_2 are at most 2^-24 relative each, the size of one
// FP32 rounding, so the factor is about as accurate as a CUDA-core FP32 factorisation (measured:
// the refinement needs the same number of steps; the two further products changed nothing).
// (The split-operand scheme for emulating a higher precision on lower-precision tensor cores
// is the published one of Henry, Tang and Heinecke, "Leveraging the bfloat16 Artificial
// Intelligence Datatype For Higher-Precision Computations", 2019.)
//
// Data flow of one panel step j0 (matrix in the CTA's global scratch slot, L2-resident):
//   A  panel: columns j0..j0+31 staged in shared memory and factored (panel_factor_par); the
//      factored panel is written back in logical row order; L11^-1 (unit lower, 32 x 32) is
//      formed in shared memory; L21 is written to the CTA's A-operand buffer in global memory
//      as ready-made tcgen05 operand tiles (three bf16 pieces, K-major core-matrix layout);
//   B  every trailing column: the panel's row interchanges, U12 = L11^-1 (pivot rows), and the
//      column's four 4M entries written to the B-operand buffer (same tile format);
//   C  Schur tiles (row tiles of 128 outer, column tiles of 32 inner): operand tiles are
//      brought into shared memory by bulk asynchronous copies (cp.async.bulk with mbarrier
//      completion; the A tile once per row tile, the B tiles through a 3-deep ring), one thread
//      issues a tile's 24 MMAs into one of two TMEM accumulators, and while the tensor cores
//      work on tile t four epilogue warps take tile t-1's accumulator (tcgen05.ld), subtract it
//      from the tile's old values (copied into shared memory two tiles ahead, each lane its own
//      row, by cp.async) and store the result; producer and epilogue hand over through mbarriers
//      only (schur_tc).
// The row interchanges of a panel are applied to the columns left of it once, after the last
// panel (unswap_left), and the correction solves use inverse diagonal blocks built per panel.
// No thread-block clusters: every copy reads this GPU's own memory into this CTA alone.
//
// Every mbarrier wait is bounded (about 2 s of device time); a wait that runs out marks the
// system (info = -2), sets the launch's error word, drains the copies and MMAs this CTA has in
// flight (bounded as well), frees its tensor memory and ends the CTA.
//
// Reference sequence: src/analysis/KrylovROMSubstructure.cpp:1411-1430 (assembly, zgetrf,
// zgetrs per frequency) and the batched cuBLAS sweep of
// test/krylovMidsizeTest/gpu/concurrent/batchedLU/src/main.cu:223-267.
#include <cuda_bf16.h>

#include "sweep_common.cuh"

namespace srom {
namespace tcm {

constexpr int NB = 32;                 // panel width (complex columns)
constexpr int KP = 2 * NB;             // depth of the real Schur GEMM: [Re L | Im L]
constexpr int TM = 128;                // rows of a tile (TMEM lanes)
constexpr int TNC = 32;                // complex columns of a tile
constexpr int TN = 2 * TNC;            // real accumulator columns of a tile: [Re | Im]
constexpr int PIECES = 3;              // bf16 pieces per FP32 value
constexpr int MMA_K = 16;              // depth of one kind::f16 MMA
constexpr int KSTEPS = KP / MMA_K;     // MMAs per piece product
constexpr int STAGES = 3;              // B-operand ring depth
constexpr int A_PIECE = TM * KP * 2;                // one bf16 piece of an A tile (128 rows)
constexpr int B_PIECE = TN * KP * 2;                // one bf16 piece of a B tile (64 rows)
constexpr int A_TILE = PIECES * A_PIECE;            // 48 KB
constexpr int B_TILE = PIECES * B_PIECE;            // 24 KB
constexpr int C_TILE = TM * TNC * 8;                // 32 KB: a tile of the trailing matrix
constexpr int OP_B = A_TILE;                        // B ring offset in the operand region
constexpr int OP_C = OP_B + STAGES * B_TILE;        // C tiles (two) offset
constexpr int OP_BYTES = OP_C + 2 * C_TILE;         // A tile + B ring + two C tiles
constexpr int TMEM_COLS = 2 * TN;                   // two accumulator buffers
constexpr int NBARS = 6 + STAGES;                   // mbarriers of the pipeline (see Bars)
constexpr int EPI_WARP0 = 4;                        // warps 4..7 run the Schur epilogue
constexpr int LDL = 33;                             // leading dimension of L11^-1 in smem
constexpr int CPW = 4;                              // trailing columns per warp pass (phase B)
constexpr int INFO_TIMEOUT = -2;

// Instruction descriptor: D f32, A and B bf16, both K-major, M = 128, N = 64.
constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(TN >> 3) << 17) |
                           ((uint32_t)(TM >> 4) << 24);

static_assert(TN % 16 == 0 && TN >= 16 && TN <= 256, "N of an M = 128 MMA");
static_assert(TMEM_COLS >= 32 && (TMEM_COLS & (TMEM_COLS - 1)) == 0, "TMEM allocations are powers of two >= 32");
static_assert(OP_BYTES >= (512 | 1) * NB * 8, "the panel of an n = 512 system fits the operand region");

// Byte offset of element (row, k) in one operand piece: K-major with the 128-byte swizzle.  A
// row's 64 bf16 fill one 128-byte line, 8-row groups are 1024 bytes apart (SBO), and the 16-byte
// chunk c of row r sits at chunk c ^ (r & 7) of its line, so that the tensor cores' reads of
// eight rows at one K position fall in different shared-memory banks.  A pieces have 128 rows,
// B pieces 64; every piece starts on a 1024-byte boundary (the swizzle uses address bits 4-9).
__host__ __device__ constexpr int op_off(int row, int k) {
    return (row >> 3) * 1024 + (row & 7) * 128 + ((((k >> 3) ^ row) & 7) << 4) + (k & 7) * 2;
}

// Shared-memory layout (offsets from a 1024-byte aligned base).  The operand region holds the
// panel during phase A, the A tile, the B ring and two C tiles during phase C, and the
// refinement's iterate, right-hand sides and staging ring after the factorisation.
struct TcSmem {
    size_t op, perm, ptot, pos, ipiv, moved, dinv, linv, bars, tmem, flags, total;
    size_t work64, work32, ring;
    static __host__ __device__ size_t up(size_t b) { return (b + 255) / 256 * 256; }
    __host__ __device__ TcSmem(int ldp, int n_max, int r_max) {
        op = 0;
        perm = op + OP_BYTES;
        ptot = perm + up((size_t)ldp * 4);
        pos = ptot + up((size_t)ldp * 4);
        ipiv = pos + up((size_t)ldp * 4);
        moved = ipiv + up((size_t)ldp * 4);
        dinv = moved + up((size_t)2 * 2 * NB * 4);
        linv = dinv + up((size_t)ldp * 8);
        bars = linv + up((size_t)NB * LDL * 8);
        tmem = bars + up((size_t)NBARS * 8);
        flags = tmem + 256;
        total = flags + up((size_t)((ldp + NB - 1) / NB) * 4);
        work64 = op;
        work32 = work64 + up((size_t)n_max * r_max * 16);
        ring = work32 + up((size_t)n_max * r_max * 8);
    }
};

// Leading dimension of the scratch matrix: even, so that every column starts on a 16-byte
// boundary (the C tiles are moved by bulk copies, one per column).
__host__ __device__ constexpr int tc_lda(int n) { return n + (n & 1); }

// Global scratch of one CTA: the complex-FP32 matrix (ld tc_lda(n)), the A- and B-operand tile
// buffers, the inverse diagonal blocks of the factor (L_bb^-1, U_bb^-1 of every 32-row block b,
// each 32 x 32 column-major, zero outside the block) used by the correction solves, and every
// panel's row-interchange record (applied to the columns left of it once, at the end).
constexpr int MV_INTS = 4 + 4 * NB;  // a panel's interchange record: count, pad, dst[2 NB], src[2 NB]

struct TcSlot {
    size_t a32, abuf, bbuf, inv, moves, total;
    __host__ __device__ TcSlot(int n_max) {
        const int mt = n_max > NB ? n_max - NB : 1;
        const int nbk = (n_max + NB - 1) / NB;
        a32 = 0;
        abuf = ((size_t)tc_lda(n_max) * n_max * 8 + 1023) / 1024 * 1024;
        bbuf = abuf + (size_t)((mt + TM - 1) / TM) * A_TILE;
        inv = bbuf + (size_t)((mt + TNC - 1) / TNC) * B_TILE;
        moves = inv + (size_t)nbk * 2 * NB * NB * 8;
        total = moves + (size_t)nbk * MV_INTS * 4;
    }
};

// ---------------------------------------------------------------------------- PTX wrappers
__device__ __forceinline__ uint32_t su32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t globaltimer() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ bool mbar_test(uint32_t bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// Wait for the completion of the barrier phase with the given parity, at most about 2 s of
// device time (and a bounded number of polls).  Returns false when the wait ran out.
__device__ __noinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    if (mbar_test(bar, parity)) return true;
    const uint64_t t0 = globaltimer();
    for (uint32_t it = 0; it < (1u << 28); ++it) {
        if (mbar_test(bar, parity)) return true;
        if ((it & 255u) == 255u && globaltimer() - t0 > 2000000000ull) return false;
    }
    return false;
}

// Bulk copy global -> this CTA's shared memory, completion counted on an mbarrier.
__device__ __forceinline__ void bulk_load(uint32_t dst, const void *src, uint32_t bytes, uint32_t bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
                 "l"(src), "r"(bytes), "r"(bar)
                 : "memory");
}

__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Shared-memory matrix descriptor: K-major, 128-byte swizzle (layout type 2), SBO 1024 B (LBO
// unused: a K step of 16 bf16 stays inside the 128-byte line), descriptor version 1 (sm_100),
// base offset 0 (1024-byte aligned pieces).  The K steps of a piece start 32 bytes apart.
__device__ __forceinline__ uint64_t sdesc(uint32_t saddr) {
    return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)1 << 16) | ((uint64_t)(1024 >> 4) << 32) | (1ull << 46) |
           (2ull << 61);
}

__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(d_tmem),
        "l"(adesc), "l"(bdesc), "r"(IDESC), "r"(accumulate), "r"(0), "r"(0), "r"(0), "r"(0));
}

__device__ __forceinline__ void mma_commit(uint32_t bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}

// 16 consecutive 32-bit accumulator columns of this thread's TMEM lane, waited for in the same
// statement (so no use of the registers can be scheduled before the load completes).
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15}, [%16];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// x = p0 + p1 + p2 (+ below 2^-24 |x|): each piece the bf16 rounding of what is left.
__device__ __forceinline__ void split3(float x, __nv_bfloat16 (&p)[3]) {
    p[0] = __float2bfloat16_rn(x);
    const float r1 = x - __bfloat162float(p[0]);
    p[1] = __float2bfloat16_rn(r1);
    const float r2 = r1 - __bfloat162float(p[1]);
    p[2] = __float2bfloat16_rn(r2);
}

__device__ __forceinline__ unsigned short bfbits(__nv_bfloat16 v) { return __bfloat16_as_ushort(v); }

// u += a * b (complex FP32)
__device__ __forceinline__ float2 cfma(float2 u, float2 a, float2 b) {
    return make_float2(__fmaf_rn(a.x, b.x, __fmaf_rn(-a.y, b.y, u.x)), __fmaf_rn(a.x, b.y, __fmaf_rn(a.y, b.x, u.y)));
}

// ---------------------------------------------------------------------------- pipeline state
// Barrier words: bar_a (A tile), bar_full[s] (ring slot s), bar_mma[b] (accumulator b holds a
// finished tile), bar_free[b] (the four epilogue warps are done with accumulator b and C buffer
// b), bar_panel (the panel's columns have landed in shared memory).
struct Bars {
    uint32_t base;
    __device__ uint32_t a() const { return base; }
    __device__ uint32_t full(int s) const { return base + 8u * (uint32_t)(1 + s); }
    __device__ uint32_t mma(int b) const { return base + 8u * (uint32_t)(1 + STAGES + b); }
    __device__ uint32_t free(int b) const { return base + 8u * (uint32_t)(3 + STAGES + b); }
    __device__ uint32_t panel() const { return base + 8u * (uint32_t)(5 + STAGES); }
};

// Counters that give every barrier wait its parity.  Tiles are numbered over the CTA's life
// (g): tile g uses ring slot g % STAGES (its (g / STAGES)-th fill), accumulator g & 1 and C
// buffer g & 1 (their (g >> 1)-th commit / fill).  All threads keep g; thread 0 (the issuer)
// also keeps the fill counts for the drain after a timeout.
struct TcState {
    int g;         // tiles issued so far
    int loaded;    // B tiles whose copies were issued (global tile numbers [0, loaded))
    int a_loads;   // A tiles issued
    int panels;    // panel copies issued
};

__device__ __forceinline__ void set_abort(int *s_abort, int *err_flag) {
    *reinterpret_cast<volatile int *>(s_abort) = 1;
    if (err_flag) atomicExch(err_flag, 1);
}

__device__ __forceinline__ bool aborted(const int *s_abort) { return *reinterpret_cast<const volatile int *>(s_abort) != 0; }

// Thread 0 after a timeout: wait (bounded) for every copy and MMA this CTA may still have in
// flight, so that no asynchronous write lands after the CTA has freed its resources.
__device__ void drain(const Bars &B, const TcState &S) {
    for (int k = 1; k <= 2 && S.g - k >= 0; ++k) {
        const int g = S.g - k;
        mbar_wait(B.mma(g & 1), (uint32_t)(g >> 1) & 1u);
    }
    for (int k = 1; k <= STAGES && S.loaded - k >= 0; ++k) {
        const int g = S.loaded - k;
        mbar_wait(B.full(g % STAGES), (uint32_t)(g / STAGES) & 1u);
    }
    if (S.a_loads > 0) mbar_wait(B.a(), (uint32_t)(S.a_loads - 1) & 1u);
}

// ---------------------------------------------------------------------------- assembly
// A(w) = (1 + i eta) K + (-w^2) M + (i w) D rounded to complex FP32 into A (ld lda), with the
// FP64 arithmetic of assemble_entry: the mixed kernel's column sweep (a warp a column, column
// sweep_start(f) first), in a function of its own so that its registers do not weigh on the
// factorisation's.  (A batched form, eight entries of NT-strided column-major positions per
// thread with their loads issued together, measured 1.8x slower at n = 512: two integer
// divisions an entry and spills.)
__device__ __noinline__ void assemble_fp32(float2 *A, int lda, const RomDev &R, double w, int f) {
    assemble_into<float2>(A, lda, R, w, f);
}

// ---------------------------------------------------------------------------- phase A helpers
// Inverse diagonal blocks of the factored panel (logical rows and columns 0..bs-1).  Warp w
// forms columns j = w, w + 8, w + 16, w + 24 of both inverses together (lane i holds row i):
// L11^-1 e_j by forward elimination (y_i -= L[i][k] y_k for k = j..bs-2, i > k) and U11^-1 e_j
// by back substitution (y_k = (e_j - sum_{m>k} U[k][m] y_m) / U[k][k], k = j..0), the entry of
// L or U and the pivot's reciprocal of each step shared by the four columns.  L11^-1 goes to
// shared memory (phase B) and both to the CTA's global inverse buffer (the correction solves),
// 32 x 32 column-major with zeros outside bs x bs.
__device__ __forceinline__ void build_inverses(const float2 *P, int ldp, const int *s_perm, int bs, float2 *s_linv,
                               float2 *ginv) {
    using C = CT<float2>;
    constexpr int Q = NB / NW;  // columns per warp
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const bool act = lane < bs;
    const int pr = act ? s_perm[lane] : 0;
    float2 y[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) y[q] = (act && lane == warp + NW * q) ? make_float2(1.f, 0.f) : C::zero();
    for (int k = warp; k < bs - 1; ++k) {
        const float2 l = (act && lane > k) ? P[pr + (int64_t)k * ldp] : C::zero();
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const float2 yk = C::shfl(y[q], k, 32);
            if (act && lane > k && k >= warp + NW * q) y[q] = C::subm(y[q], l, yk);
        }
    }
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const int j = warp + NW * q;
        const float2 v = (act && j < bs && lane >= j) ? y[q] : C::zero();
        s_linv[lane + j * LDL] = v;
        ginv[lane + j * NB] = v;
    }
    float2 acc[Q];
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        y[q] = C::zero();
        acc[q] = (act && lane == warp + NW * q) ? make_float2(1.f, 0.f) : C::zero();
    }
    for (int k = min(warp + NW * (Q - 1), bs - 1); k >= 0; --k) {
        const float2 u = act ? P[pr + (int64_t)k * ldp] : C::zero();  // U[lane][k]
        const float2 rk = C::shfl(lane == k ? C::recip(u) : C::zero(), k, 32);
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            if (k > warp + NW * q) continue;  // column j = warp + NW q starts at k = j
            if (lane == k) y[q] = C::mul(acc[q], rk);
            const float2 yk = C::shfl(y[q], k, 32);
            if (act && lane < k) acc[q] = C::subm(acc[q], u, yk);
        }
    }
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const int j = warp + NW * q;
        const float2 v = (act && j < bs && lane <= j) ? y[q] : C::zero();
        ginv[NB * NB + lane + j * NB] = v;
    }
}

// L21 (logical rows 32..m-1 of the factored panel) as A-operand tiles: row r of tile r / 128,
// k < 32 the real parts of panel column k, k >= 32 the imaginary parts of column k - 32; three
// bf16 pieces per tile.  Rows past the last (to the tile's 128) are zero.  One thread per
// (8-row group, 8-deep chunk pair): two 16-byte stores per piece, consecutive threads on
// consecutive 16-byte rows of a core matrix.
__device__ __forceinline__ void build_abuf(const float2 *P, int ldp, const int *s_perm, int mt, unsigned char *abuf) {
    const int nrt = (mt + TM - 1) / TM;
    const int total = nrt * (TM / 8) * 32;
    for (int e = threadIdx.x; e < total; e += NT) {
        const int r8 = e & 7, kc = (e >> 3) & 3, g8 = e >> 5;
        const int r = g8 * 8 + r8;  // row of L21
        const int rt = r / TM, rr = r % TM;
        float re[8], im[8];
        if (r < mt) {
            const int pr = s_perm[NB + r];
#pragma unroll
            for (int t = 0; t < 8; ++t) {
                const float2 v = P[pr + (int64_t)(8 * kc + t) * ldp];
                re[t] = v.x;
                im[t] = v.y;
            }
        } else {
#pragma unroll
            for (int t = 0; t < 8; ++t) re[t] = im[t] = 0.f;
        }
        unsigned short pr_[3][8], pi_[3][8];
#pragma unroll
        for (int t = 0; t < 8; ++t) {
            __nv_bfloat16 a[3], b[3];
            split3(re[t], a);
            split3(im[t], b);
#pragma unroll
            for (int p = 0; p < 3; ++p) {
                pr_[p][t] = bfbits(a[p]);
                pi_[p][t] = bfbits(b[p]);
            }
        }
        unsigned char *tile = abuf + (size_t)rt * A_TILE;
#pragma unroll
        for (int p = 0; p < 3; ++p) {
            uint4 vr, vi;
            vr.x = pr_[p][0] | ((uint32_t)pr_[p][1] << 16);
            vr.y = pr_[p][2] | ((uint32_t)pr_[p][3] << 16);
            vr.z = pr_[p][4] | ((uint32_t)pr_[p][5] << 16);
            vr.w = pr_[p][6] | ((uint32_t)pr_[p][7] << 16);
            vi.x = pi_[p][0] | ((uint32_t)pi_[p][1] << 16);
            vi.y = pi_[p][2] | ((uint32_t)pi_[p][3] << 16);
            vi.z = pi_[p][4] | ((uint32_t)pi_[p][5] << 16);
            vi.w = pi_[p][6] | ((uint32_t)pi_[p][7] << 16);
            unsigned char *piece = tile + (size_t)p * A_PIECE;
            *reinterpret_cast<uint4 *>(piece + op_off(rr, 8 * kc)) = vr;
            *reinterpret_cast<uint4 *>(piece + op_off(rr, 32 + 8 * kc)) = vi;
        }
    }
}

// The row interchanges of every panel applied to the columns left of it (LAPACK's laswp on
// A(:, 0:j0)), done once after the factorisation instead of after every panel: block column p
// was written in the row order of step p, and panels p+1.. moved rows below it since.  idx[f]
// (shared memory) = stored row holding final row f: starting from the identity, going from the
// last panel down, idx <- map_k(idx) with map_k(q) = the source of q if panel k moved a row to
// q, else q; after panel k = p+1 is folded in, block column p's rows f >= 32 (p + 1) are
// gathered from rows idx[f], eight columns at a time (all reads, a barrier, all writes).
// moves: the panels' records (count, dst[], src[] relative to the panel's first row).
__device__ __forceinline__ void unswap_left(float2 *A, int n, int lda, const int *moves, int *idx, int *map) {
    constexpr int CG = 8;
    constexpr int MAXR = (512 + NT - 1) / NT;  // rows per thread (TC_MAX_N)
    const int tid = threadIdx.x;
    const int nbk = (n + NB - 1) / NB;
    for (int f = tid; f < n; f += NT) {
        idx[f] = f;
        map[f] = f;
    }
    __syncthreads();
    for (int p = nbk - 2; p >= 0; --p) {
        const int k = p + 1, jk = NB * k;
        const int *rec = moves + (size_t)k * MV_INTS;
        const int nm = rec[0];
        const int e = tid < nm ? tid : -1;
        const int dst = e >= 0 ? jk + rec[4 + e] : 0, src = e >= 0 ? jk + rec[4 + 2 * NB + e] : 0;
        if (e >= 0) map[dst] = src;
        __syncthreads();
        for (int f = jk + tid; f < n; f += NT) idx[f] = map[idx[f]];
        __syncthreads();
        if (e >= 0) map[dst] = dst;
        // gather block column p (columns NB p .. NB p + 31, all inside the matrix) below row jk
        for (int c0 = NB * p; c0 < NB * p + NB; c0 += CG) {
            float2 v[MAXR][CG];
#pragma unroll
            for (int q = 0; q < MAXR; ++q) {
                const int f = jk + tid + q * NT;
                if (f < n) {
                    const int sr = idx[f];
#pragma unroll
                    for (int c = 0; c < CG; ++c) v[q][c] = A[sr + (int64_t)(c0 + c) * lda];
                }
            }
            __syncthreads();
#pragma unroll
            for (int q = 0; q < MAXR; ++q) {
                const int f = jk + tid + q * NT;
                if (f < n) {
#pragma unroll
                    for (int c = 0; c < CG; ++c) A[f + (int64_t)(c0 + c) * lda] = v[q][c];
                }
            }
            __syncthreads();
        }
    }
}

// ---------------------------------------------------------------------------- phase B
// Trailing columns c >= j0 + 32, a warp per column, CPW columns per pass: the panel's
// interchanges (pivot rows read into x, displaced rows moved down to the pivot rows' places),
// U12 = L11^-1 x written to the matrix, and the column's 4M entries (Ur, Ui; -Ui, Ur) as three
// bf16 pieces into the B-operand tiles.  After this phase rows j0+32.. of the trailing matrix
// are in the factor's (logical) order.
__device__ __forceinline__ void trailing_rows(float2 *A, int n, int lda, int j0, const int *s_perm, const int *s_mdst,
                              const int *s_msrc, int nmoved, const float2 *s_linv, unsigned char *bbuf) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int c0 = j0 + NB;
    const int ncols = n - c0;
    const int prow = j0 + s_perm[lane];
    int md[2], ms[2];
    bool mvok[2];
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const int e = lane + 32 * q;
        mvok[q] = e < nmoved && s_mdst[e] >= NB;
        md[q] = mvok[q] ? j0 + s_mdst[e] : 0;
        ms[q] = mvok[q] ? j0 + s_msrc[e] : 0;
    }
    // the next pass's loads are issued before this pass's arithmetic (two register sets)
    float2 nx[CPW], nmv[CPW][2];
    auto load = [&](int cb) {
#pragma unroll
        for (int t = 0; t < CPW; ++t) {
            if (cb + t < ncols) {
                const float2 *col = A + (int64_t)(c0 + cb + t) * lda;
                nx[t] = col[prow];
#pragma unroll
                for (int q = 0; q < 2; ++q)
                    if (mvok[q]) nmv[t][q] = col[ms[q]];
            } else {
                nx[t] = make_float2(0.f, 0.f);
            }
        }
    };
    if (warp * CPW < ncols) load(warp * CPW);
    for (int cb = warp * CPW; cb < ncols; cb += NW * CPW) {
        float2 x[CPW], mv[CPW][2];
#pragma unroll
        for (int t = 0; t < CPW; ++t) {
            x[t] = nx[t];
#pragma unroll
            for (int q = 0; q < 2; ++q) mv[t][q] = nmv[t][q];
        }
        if (cb + NW * CPW < ncols) load(cb + NW * CPW);
        __syncwarp();
#pragma unroll
        for (int t = 0; t < CPW; ++t) {
            if (cb + t < ncols) {
                float2 *col = A + (int64_t)(c0 + cb + t) * lda;
#pragma unroll
                for (int q = 0; q < 2; ++q)
                    if (mvok[q]) col[md[q]] = mv[t][q];
            }
        }
        // u_l = x_l + sum_{j<l} Linv[l][j] x_j
        float2 u[CPW];
#pragma unroll
        for (int t = 0; t < CPW; ++t) u[t] = x[t];
        for (int j = 0; j < NB - 1; ++j) {
            const float2 lv = s_linv[lane + j * LDL];
#pragma unroll
            for (int t = 0; t < CPW; ++t) {
                const float2 xj = CT<float2>::shfl(x[t], j, 32);
                if (lane > j) u[t] = cfma(u[t], lv, xj);
            }
        }
#pragma unroll
        for (int t = 0; t < CPW; ++t) {
            if (cb + t >= ncols) continue;
            A[(int64_t)(c0 + cb + t) * lda + j0 + lane] = u[t];
            const int cc = cb + t, ct = cc / TNC, q = cc % TNC;
            __nv_bfloat16 pr[3], pi[3];
            split3(u[t].x, pr);
            split3(u[t].y, pi);
            unsigned char *tile = bbuf + (size_t)ct * B_TILE;
#pragma unroll
            for (int p = 0; p < 3; ++p) {
                unsigned char *piece = tile + (size_t)p * B_PIECE;
                const unsigned short rb = bfbits(pr[p]), ib = bfbits(pi[p]);
                *reinterpret_cast<unsigned short *>(piece + op_off(q, lane)) = rb;
                *reinterpret_cast<unsigned short *>(piece + op_off(TNC + q, lane)) = ib;
                *reinterpret_cast<unsigned short *>(piece + op_off(q, NB + lane)) = (unsigned short)(ib ^ 0x8000u);
                *reinterpret_cast<unsigned short *>(piece + op_off(TNC + q, NB + lane)) = rb;
            }
        }
    }
}

// ---------------------------------------------------------------------------- phase C
// Row r0q + lane (this lane's row of one epilogue warp's quarter of a tile) of complex columns
// c0 .. c0 + 31 into the warp's quarter of a C buffer (column-major, 128 rows) with cp.async, one
// group per tile.  For a column the warp's 32 copies are 256 contiguous bytes; a lane reads back
// only the row it copied, so its own wait_group is the whole handoff (no barrier, no proxy fence).
__device__ __forceinline__ void load_c_row(const float2 *A, int n, int lda, int r0q, int c0, float2 *dst) {
    const int lane = threadIdx.x & 31, gr = r0q + lane;
    const int cols = min(TNC, n - c0);
    if (gr < n)
        for (int c = 0; c < cols; ++c) cp_async_elem(dst + lane + c * TM, A + gr + (int64_t)(c0 + c) * lda);
    cp_async_commit();
}

// Schur update of rows and columns [j0 + 32, n) from the operand buffers (see the file header),
// warp-specialised with mbarrier handoffs only:
//   thread 0      loads the A tile (per row tile) and the B ring, waits for accumulator g & 1 to
//                 be free (bar_free of tile g - 2), issues tile g's MMAs into it and commits to
//                 bar_mma; once tile g - 1's MMAs are done its ring slot takes tile g - 1 + STAGES;
//   warps 4..7    (warp 4 + q owns TMEM lanes and tile rows 32 q .. +31) wait for bar_mma and their
//                 C rows (cp.async, two tiles ahead), subtract the accumulator from the old values
//                 and store the results to the matrix, arrive on bar_free, and then load their rows
//                 of tile g + 2 into the buffer;
//   warps 1..3    wait at the closing barrier.
__device__ __forceinline__ void schur_tc(float2 *A, int n, int lda, int j0, unsigned char *op, const unsigned char *abuf,
                         const unsigned char *bbuf, uint32_t tmem, const Bars &B, TcState &S, int *s_abort,
                         int *err_flag) {
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int mt = n - j0 - NB;
    const int nrt = (mt + TM - 1) / TM, nct = (mt + TNC - 1) / TNC, T = nrt * nct;
    const uint32_t opa = su32(op);
    auto slot = [&](int s) { return opa + (uint32_t)(OP_B + s * B_TILE); };
    auto tile_r0 = [&](int t) { return j0 + NB + (t / nct) * TM; };
    auto tile_c0 = [&](int t) { return j0 + NB + (t % nct) * TNC; };
    const int g0 = S.g;
    if (tid == 0) {
        // piece products (A piece, B piece), smallest first: all i + j <= 2
        constexpr int NPROD = 6;
        constexpr int PA[NPROD] = {2, 1, 0, 1, 0, 0};
        constexpr int PB[NPROD] = {0, 1, 2, 0, 1, 0};
        bool ok = !aborted(s_abort);
        if (ok) {
            mbar_expect_tx(B.a(), A_TILE);
            bulk_load(opa, abuf, A_TILE, B.a());
            S.a_loads++;
            for (int i = 0; i < STAGES && i < T; ++i) {
                const int g = g0 + i;
                mbar_expect_tx(B.full(g % STAGES), B_TILE);
                bulk_load(slot(g % STAGES), bbuf + (size_t)(i % nct) * B_TILE, B_TILE, B.full(g % STAGES));
                S.loaded = g + 1;
            }
        }
        for (int t = 0; t < T && ok; ++t) {
            const int g = g0 + t;
            const int rt = t / nct;
            const bool new_rt = t == 0 || rt != (t - 1) / nct;
            if (t > 0 && new_rt) {
                // the A tile is free once every MMA reading it has completed, i.e. tile t-1's
                ok = mbar_wait(B.mma((g - 1) & 1), (uint32_t)((g - 1) >> 1) & 1u);
                if (!ok) break;
                mbar_expect_tx(B.a(), A_TILE);
                bulk_load(opa, abuf + (size_t)rt * A_TILE, A_TILE, B.a());
                S.a_loads++;
            }
            if (new_rt) ok = mbar_wait(B.a(), (uint32_t)(S.a_loads - 1) & 1u);
            if (ok) ok = mbar_wait(B.full(g % STAGES), (uint32_t)(g / STAGES) & 1u);
            if (ok && t >= 2) ok = mbar_wait(B.free(g & 1), (uint32_t)((g - 2) >> 1) & 1u);
            if (!ok) break;
            tc_fence_after();
            const uint32_t d = tmem + (uint32_t)((g & 1) * TN);
            const uint32_t bsl = slot(g % STAGES);
#pragma unroll
            for (int p = 0; p < NPROD; ++p)
#pragma unroll
                for (int ks = 0; ks < KSTEPS; ++ks) {
                    const uint64_t ad = sdesc(opa + (uint32_t)(PA[p] * A_PIECE + ks * 32));
                    const uint64_t bd = sdesc(bsl + (uint32_t)(PB[p] * B_PIECE + ks * 32));
                    mma_bf16(d, ad, bd, (uint32_t)(p | ks));
                }
            mma_commit(B.mma(g & 1));
            S.g = g + 1;
            const int tn = t - 1 + STAGES;
            if (t > 0 && tn < T) {
                // tile t-1's MMAs are done (they precede tile t's): its slot takes tile t-1+STAGES
                ok = mbar_wait(B.mma((g - 1) & 1), (uint32_t)((g - 1) >> 1) & 1u);
                if (!ok) break;
                const int gn = g0 + tn;
                mbar_expect_tx(B.full(gn % STAGES), B_TILE);
                bulk_load(slot(gn % STAGES), bbuf + (size_t)(tn % nct) * B_TILE, B_TILE, B.full(gn % STAGES));
                S.loaded = gn + 1;
            }
        }
        if (!ok) {
            set_abort(s_abort, err_flag);
            drain(B, S);
        }
    } else if (warp >= EPI_WARP0) {
        const int q = warp - EPI_WARP0;
        float2 *cs = reinterpret_cast<float2 *>(op + OP_C);
        auto cq = [&](int g) { return cs + (size_t)(g & 1) * (C_TILE / 8) + 32 * q; };
        bool ok = !aborted(s_abort);
        // one cp.async group per tile, committed even when empty: before tile t's use exactly the
        // group of tile t + 1 may still be pending
        for (int i = 0; i < 2; ++i) {
            if (i < T) load_c_row(A, n, lda, tile_r0(i) + 32 * q, tile_c0(i), cq(g0 + i));
            else cp_async_commit();
        }
        for (int t = 0; t < T && ok; ++t) {
            const int g = g0 + t, b = g & 1;
            const uint32_t par = (uint32_t)(g >> 1) & 1u;
            ok = !aborted(s_abort) && mbar_wait(B.mma(b), par);
            ok = __all_sync(FULL_MASK, ok);
            if (!ok) break;
            tc_fence_after();
            cp_async_wait<1>();
            const int row = 32 * q + lane, gr = tile_r0(t) + row, c0 = tile_c0(t);
            const uint32_t tb = tmem + ((uint32_t)(32 * q) << 16) + (uint32_t)(b * TN);
            const float2 *cbuf = cs + (size_t)b * (C_TILE / 8);
#pragma unroll
            for (int r = 0; r < 2; ++r) {
                float re[16], im[16];
                tmem_ld16(tb + (uint32_t)(16 * r), re);
                tmem_ld16(tb + (uint32_t)(TNC + 16 * r), im);
                if (gr < n) {
#pragma unroll
                    for (int i = 0; i < 16; ++i) {
                        const int c = 16 * r + i;
                        if (c0 + c < n) {
                            const float2 v = cbuf[row + c * TM];
                            A[gr + (int64_t)(c0 + c) * lda] = make_float2(v.x - re[i], v.y - im[i]);
                        }
                    }
                }
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(B.free(b));
            if (t + 2 < T) load_c_row(A, n, lda, tile_r0(t + 2) + 32 * q, tile_c0(t + 2), cq(g + 2));
            else cp_async_commit();
        }
        cp_async_wait<0>();  // also after a timeout: no copy lands after the CTA moves on
        if (!ok) set_abort(s_abort, err_flag);
    }
    __syncthreads();
    if (!aborted(s_abort)) S.g = g0 + T;  // after a timeout thread 0 keeps its count of issued tiles
}

// ---------------------------------------------------------------------------- correction solves
// LU x = b for the complex-FP32 factor in A (ld lda, LAPACK layout, rows in the factor's order) and
// b (n x nrhs, ld n) in shared memory; x replaces b.  Blocked by the 32-row blocks of the
// factorisation, with the inverse diagonal blocks formed there (ginv), and run as a warp-level
// dataflow instead of CTA-wide steps:
//   forward  y_b = L_bb^-1 (b_b - sum_{c<b} L_bc y_c),    blocks b = w, w + 8, ... on warp w;
//   backward x_b = U_bb^-1 (y_b - sum_{c>b} U_bc x_c),    blocks b = nb-1-w, nb-1-w-8, ...
// A warp streams the 32 x 32 tiles its blocks need (L_bc / U_bc from the factor, then the
// block's inverse) through its own ring of ns shared-memory tiles with cp.async, so its copies
// run ahead of the dependencies; before using y_c (x_c) it waits for block c's flag, which the
// owner sets after writing the block's rows of b.  Flags carry a phase that grows with every
// solve (forward phase, backward phase + 1), so they are never reset.  Every wait is bounded.
constexpr int DF_TILE = NB * NB;  // float2 per tile
constexpr uint32_t DF_SPIN_LIMIT = 1u << 24;

__device__ __forceinline__ bool df_wait(const int *flag, int target) {
    for (uint32_t it = 0; it < DF_SPIN_LIMIT; ++it) {
        if (*reinterpret_cast<const volatile int *>(flag) >= target) {
            __threadfence_block();
            return true;
        }
        __nanosleep(32);
    }
    return false;
}

template <int RC>
__device__ __forceinline__ void solve_df(const float2 *A, int n, int lda, float2 *B, int nrhs, const float2 *ginv,
                                      float2 *stage, int ns, int *s_flag, int phase, int *s_abort, int *err_flag) {
    using C = CT<float2>;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nb = (n + NB - 1) / NB;
    float2 *ring = stage + (size_t)warp * ns * DF_TILE;
    bool ok = true;
    for (int dir = 0; dir < 2; ++dir) {
        const int target = phase + dir;
        auto block_of = [&](int k) { return dir == 0 ? warp + NW * k : nb - 1 - warp - NW * k; };
        auto valid = [&](int k) {
            const int b = block_of(k);
            return b >= 0 && b < nb;
        };
        auto ntiles = [&](int b) { return (dir == 0 ? b : nb - 1 - b) + 1; };
        auto col_of = [&](int t) { return dir == 0 ? t : nb - 1 - t; };
        int ik = 0, it = 0, qi = 0;  // issue position: owned block ik, its tile it; tiles issued
        auto issue = [&]() {
            if (valid(ik)) {
                const int b = block_of(ik);
                float2 *dst = ring + (qi % ns) * DF_TILE;
                if (it < ntiles(b) - 1) {
                    const int row = NB * b + lane, c0 = NB * col_of(it);
                    const int kmax = min(NB, n - c0);
                    if (row < n)
                        for (int kk = 0; kk < kmax; ++kk)
                            cp_async_elem(dst + kk * NB + lane, A + row + (int64_t)(c0 + kk) * lda);
                } else {
                    const float2 *src = ginv + (size_t)(2 * b + dir) * DF_TILE;
                    for (int kk = 0; kk < NB; ++kk) cp_async_elem(dst + kk * NB + lane, src + kk * NB + lane);
                }
                if (++it == ntiles(b)) {
                    ++ik;
                    it = 0;
                }
            }
            cp_async_commit();
            ++qi;
        };
        // backward: no block's rows of b may be overwritten before every forward reader is done,
        // which the last block's forward flag implies
        if (dir == 1 && !df_wait(s_flag + nb - 1, phase)) ok = false;
        for (int q = 0; q < ns - 1; ++q) issue();
        int q = 0;
        float2 acc[RC];
        for (int k = 0; valid(k); ++k) {
            const int b = block_of(k), nt = ntiles(b);
            const int r0 = NB * b, bs = min(NB, n - r0);
#pragma unroll
            for (int c = 0; c < RC; ++c)
                if (c < nrhs) acc[c] = lane < bs ? B[r0 + lane + (int64_t)c * n] : C::zero();
            for (int t = 0; t < nt; ++t, ++q) {
                issue();
                cp_async_wait_dyn(ns - 1);
                __syncwarp();
                const float2 *S = ring + (q % ns) * DF_TILE;
                if (t < nt - 1) {
                    const int cb = col_of(t), c0 = NB * cb, kmax = min(NB, n - c0);
                    if (!df_wait(s_flag + cb, target)) ok = false;
                    for (int kk = 0; kk < kmax; ++kk) {
                        const float2 a = S[kk * NB + lane];
#pragma unroll
                        for (int c = 0; c < RC; ++c)
                            if (c < nrhs) acc[c] = C::subm(acc[c], a, B[c0 + kk + (int64_t)c * n]);
                    }
                } else {
                    if (lane < bs) {
#pragma unroll
                        for (int c = 0; c < RC; ++c)
                            if (c < nrhs) B[r0 + lane + (int64_t)c * n] = acc[c];
                    }
                    __syncwarp();
#pragma unroll
                    for (int c = 0; c < RC; ++c) acc[c] = C::zero();
                    for (int kk = 0; kk < bs; ++kk) {
                        const float2 a = S[kk * NB + lane];
#pragma unroll
                        for (int c = 0; c < RC; ++c)
                            if (c < nrhs) acc[c] = cfma(acc[c], a, B[r0 + kk + (int64_t)c * n]);
                    }
                    __syncwarp();
                    if (lane < bs) {
#pragma unroll
                        for (int c = 0; c < RC; ++c)
                            if (c < nrhs) B[r0 + lane + (int64_t)c * n] = acc[c];
                    }
                    __threadfence_block();
                    __syncwarp();
                    if (lane == 0) *reinterpret_cast<volatile int *>(s_flag + b) = target;
                }
                __syncwarp();
            }
        }
        cp_async_wait<0>();
        __syncwarp();
    }
    if (!__all_sync(FULL_MASK, ok)) set_abort(s_abort, err_flag);
    __syncthreads();
}

// Correction solve of the tensor-core kernel.  One right-hand side: the dataflow solve (its
// critical path is short when a tile step is one complex multiply-add per entry).  More: the
// strip-ring solve of the CUDA-core kernel, whose CTA-wide strips amortise the per-block
// latency over all right-hand sides.  The launch guarantees the ring DF_MIN_RING bytes (two
// tiles per warp, which is also two 16-column strips of the largest system).
constexpr int DF_MIN_RING = 2 * NW * DF_TILE * (int)sizeof(float2);

template <int RPT>
struct TcSolve {
    const float2 *A;
    int n, lda;
    const float2 *ginv;
    unsigned char *ring;
    int ring_bytes;
    const float2 *dinv;
    int *s_flag;
    int *s_phase;
    int *s_abort;
    int *err_flag;
    __device__ void operator()(float2 *B, int nrhs) const {
        if (nrhs > 1) {
            solve_ring<RPT>(A, n, lda, B, nrhs, ring, ring_bytes, dinv);
            return;
        }
        const int ns = min(4, ring_bytes / (NW * DF_TILE * (int)sizeof(float2)));
        const int phase = *s_phase;
        solve_df<1>(A, n, lda, B, nrhs, ginv, reinterpret_cast<float2 *>(ring), ns, s_flag, phase, s_abort, err_flag);
        if (threadIdx.x == 0) *s_phase = phase + 2;  // read again only after the next CTA barrier
    }
};

// ---------------------------------------------------------------------------- factorisation
// Blocked LU of the complex-FP32 system in A (n x n, ld lda): the same output as factor_global
// (LAPACK layout, rows in final order, s_ptot the composite permutation, s_ipiv the pivots,
// PL.info the first zero pivot), with the Schur updates on the tensor cores.
template <int RPT>
__device__ __forceinline__ void factor_tc(float2 *A, int n, int lda, int ldp, unsigned char *sm, const TcSmem &L,
                                       unsigned char *abuf, unsigned char *bbuf, float2 *ginv, int *moves, PanelLists &PL,
                                       PivotXchg<float> &X, int *s_pivlg, uint32_t tmem, const Bars &B, TcState &S,
                                       int *s_abort, int *err_flag) {
    float2 *P = reinterpret_cast<float2 *>(sm + L.op);
    int *s_perm = reinterpret_cast<int *>(sm + L.perm);
    int *s_ptot = reinterpret_cast<int *>(sm + L.ptot);
    int *s_ipiv = reinterpret_cast<int *>(sm + L.ipiv);
    int *s_mdst = reinterpret_cast<int *>(sm + L.moved);
    int *s_msrc = s_mdst + 2 * NB;
    float2 *s_linv = reinterpret_cast<float2 *>(sm + L.linv);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int i = tid; i < n; i += NT) s_ptot[i] = i;
    if (tid == 0) PL.info = 0;
    fence_proxy_async();  // the assembly's stores and earlier generic use of the panel region
    __syncthreads();
    for (int j0 = 0; j0 < n; j0 += NB) {
        const int nbc = min(NB, n - j0);
        const int m = n - j0;
        const int mt = m - NB;  // trailing rows and columns (> 0 only for full panels)
        // the panel's columns into shared memory, one bulk copy per column (rows rounded up to
        // an even count: the row past n of an odd order is the scratch matrix's padding row)
        if (warp == 0) {
            const int rows_copy = (m + 1) & ~1;
            if (lane == 0) mbar_expect_tx(B.panel(), (uint32_t)(nbc * rows_copy * 8));
            __syncwarp();
            if (lane < nbc)
                bulk_load(su32(P + (int64_t)lane * ldp), A + j0 + (int64_t)(j0 + lane) * lda, (uint32_t)(rows_copy * 8),
                          B.panel());
        }
        if (tid == 0) {
            PL.nmoved = 0;
            PL.grp = 0;
        }
        if (!mbar_wait(B.panel(), (uint32_t)S.panels & 1u)) set_abort(s_abort, err_flag);
        ++S.panels;
        __syncthreads();
        if (aborted(s_abort)) return;
        panel_factor_par<float2, RPT>(P, ldp, m, nbc, s_perm, s_pivlg, s_mdst, s_msrc, PL, j0, X);
        const int nmoved = PL.nmoved;
        for (int c = warp; c < nbc; c += NW)
            for (int i = lane; i < m; i += 32) A[(j0 + i) + (int64_t)(j0 + c) * lda] = P[s_perm[i] + (int64_t)c * ldp];
        if (tid < nbc) s_ipiv[j0 + tid] = j0 + s_pivlg[tid] + 1;
        if (warp == NW - 1) {
            int v[2];
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const int e = lane + 32 * q;
                if (e < nmoved) v[q] = s_ptot[j0 + s_msrc[e]];
            }
            __syncwarp();
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const int e = lane + 32 * q;
                if (e < nmoved) s_ptot[j0 + s_mdst[e]] = v[q];
            }
            __syncwarp();
        }
        build_inverses(P, ldp, s_perm, nbc, s_linv, ginv + (size_t)(j0 / NB) * 2 * NB * NB);
        if (mt > 0) build_abuf(P, ldp, s_perm, mt, abuf);
        {
            int *rec = moves + (size_t)(j0 / NB) * MV_INTS;
            if (tid == 0) rec[0] = nmoved;
            if (tid < nmoved) {
                rec[4 + tid] = s_mdst[tid];
                rec[4 + 2 * NB + tid] = s_msrc[tid];
            }
        }
        __syncthreads();
        if (mt > 0) {
            trailing_rows(A, n, lda, j0, s_perm, s_mdst, s_msrc, nmoved, s_linv, bbuf);
            fence_proxy_async();  // generic writes (operand buffers, panel smem) before async-proxy use
            __syncthreads();
            schur_tc(A, n, lda, j0, sm + L.op, abuf, bbuf, tmem, B, S, s_abort, err_flag);
            fence_proxy_async();  // async-proxy writes of the operand region before generic reuse
            if (aborted(s_abort)) return;
        }
        fence_proxy_async();  // this step's generic use of the panel region before the next copy
        __syncthreads();
    }
    // the operand region is free again: index maps of the deferred interchanges
    int *idx = reinterpret_cast<int *>(sm + L.op);
    unswap_left(A, n, lda, moves, idx, idx + ldp);
    __syncthreads();
}

template <int RPT>
__global__ void __launch_bounds__(NT, 1) sweep_tc_kernel(GlobalArgs a) {
    extern __shared__ unsigned char sm_raw[];
    __shared__ int s_item;
    __shared__ int s_pivlg[NB];
    __shared__ PanelLists PL;
    __shared__ PivotXchg<float> Xx;
    __shared__ double s_dx[RMAX_MIXED];
    __shared__ int s_abort, s_phase;
    unsigned char *sm = sm_raw + ((1024u - (su32(sm_raw) & 1023u)) & 1023u);
    const TcSmem L(a.ldp, a.n_max, a.r_max);
    const TcSlot SL(a.n_max);
    const int tid = threadIdx.x, warp = tid >> 5;
    uint32_t *s_tmem = reinterpret_cast<uint32_t *>(sm + L.tmem);
    const Bars B{su32(sm + L.bars)};
    if (tid == 0) {
        mbar_init(B.a(), 1);
        for (int s = 0; s < STAGES; ++s) mbar_init(B.full(s), 1);
        for (int b = 0; b < 2; ++b) {
            mbar_init(B.mma(b), 1);
            mbar_init(B.free(b), NW - EPI_WARP0);
        }
        mbar_init(B.panel(), 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        s_abort = 0;
        s_phase = 1;
    }
    int *s_flag = reinterpret_cast<int *>(sm + L.flags);
    for (int i = tid; i < (a.ldp + NB - 1) / NB; i += NT) s_flag[i] = 0;
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(su32(s_tmem)),
                     "r"(TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *s_tmem;
    TcState S{0, 0, 0, 0};
    unsigned char *slotp = a.scratch + (int64_t)blockIdx.x * a.slot_bytes;
    float2 *A32 = reinterpret_cast<float2 *>(slotp + SL.a32);
    unsigned char *abuf = slotp + SL.abuf;
    unsigned char *bbuf = slotp + SL.bbuf;
    float2 *ginv = reinterpret_cast<float2 *>(slotp + SL.inv);
    int *moves = reinterpret_cast<int *>(slotp + SL.moves);

    for (;;) {
        const int it = next_item(a.counter, &s_item);
        if (it >= a.n_items) break;
        const Item wi = a.items[it];
        const RomDev R = a.roms[wi.rom];
        const int n = R.n;
        const double w = R.omega[wi.f];
        int steps = 0, info = 0;
        double berr = 0.0;
        bool write_status = true;
        const int lda = tc_lda(n);
        assemble_fp32(A32, lda, R, w, wi.f);
        __syncthreads();
        factor_tc<RPT>(A32, n, lda, a.ldp, sm, L, abuf, bbuf, ginv, moves, PL, Xx, s_pivlg, tmem, B, S, &s_abort,
                       a.err_flag);
        __syncthreads();
        if (aborted(&s_abort)) {
            if (tid == 0 && R.info) R.info[wi.f] = INFO_TIMEOUT;
            break;
        }
        info = PL.info;
        MixedWork W{reinterpret_cast<double2 *>(sm + L.work64),
                    reinterpret_cast<float2 *>(sm + L.work32),
                    reinterpret_cast<int *>(sm + L.pos),
                    reinterpret_cast<int *>(sm + L.ptot),
                    reinterpret_cast<float2 *>(sm + L.dinv),
                    sm + L.ring,
                    (int)(OP_BYTES - L.ring),
                    s_dx,
                    lda};
        const TcSolve<RPT> solve{A32, n, lda, ginv, W.ring, W.ring_bytes, W.s_dinv, s_flag, &s_phase, &s_abort, a.err_flag};
        mixed_refine<RPT>(a, R, wi, w, A32, W, solve, info, steps, berr, write_status);
        __syncthreads();
        if (aborted(&s_abort)) {
            if (tid == 0 && R.info) R.info[wi.f] = INFO_TIMEOUT;
            break;
        }
        if (tid == 0 && write_status) {
            if (R.info) R.info[wi.f] = info;
            if (R.steps) R.steps[wi.f] = steps;
            if (R.berr) R.berr[wi.f] = berr;
        }
        __syncthreads();
    }
    if (tid == 0 && aborted(&s_abort)) drain(B, S);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS) : "memory");
}

}  // namespace tcm

// ---------------------------------------------------------------------------- host side
size_t tc_slot_bytes(int n_max) { return tcm::TcSlot(n_max).total; }

size_t tc_smem_bytes(int n_max, int r_max) { return tcm::TcSmem(tcm::tc_lda(n_max), n_max, r_max).total + 1024; }

bool tc_supported(int n_max, int r_max, int smem_optin, const char **why) {
    const char *w = nullptr;
    if (n_max > TC_MAX_N) w = "order above the tensor-core kernel's limit";
    else if (r_max > MIXED_MAX_R) w = "too many right-hand sides";
    else {
        const tcm::TcSmem L(tcm::tc_lda(n_max), n_max, r_max);
        if (tcm::OP_BYTES < (int64_t)L.ring || tcm::OP_BYTES - (int64_t)L.ring < tcm::DF_MIN_RING)
            w = "refinement work areas exceed shared memory";
        else if (tc_smem_bytes(n_max, r_max) + GLOBAL_STATIC_SMEM > (size_t)smem_optin)
            w = "shared memory";
    }
    if (why) *why = w;
    return w == nullptr;
}

template <int RPT>
static cudaError_t launch_tc_t(const GlobalArgs &a0, int grid, cudaStream_t st) {
    auto k = tcm::sweep_tc_kernel<RPT>;
    GlobalArgs a = a0;
    const size_t smem = tc_smem_bytes(a.n_max, a.r_max);
    a.smem_dyn = (int)smem;
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    k<<<grid, NT, smem, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_tc(const GlobalArgs &a0, int grid, cudaStream_t st) {
    GlobalArgs a = a0;
    a.ldp = tcm::tc_lda(a.n_max);  // even: the panel's columns are bulk-copy destinations
    if (a.n_max > TC_MAX_N || a.r_max > MIXED_MAX_R || a.slot_bytes < (int64_t)tc_slot_bytes(a.n_max))
        return cudaErrorInvalidValue;
    const int rpt = global_rpt(a.n_max);
    if (rpt <= 1) return launch_tc_t<1>(a, grid, st);
    if (rpt == 2) return launch_tc_t<2>(a, grid, st);
    return cudaErrorInvalidValue;
}

}  // namespace srom
