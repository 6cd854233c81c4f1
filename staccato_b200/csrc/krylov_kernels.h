// Host-side entry of the Krylov basis generation (krylov.cu), used by the C ABI in capi.cu.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

namespace srom {
namespace kry {

// Pivots of the band LDL^T factorisations of one call: how many were below 1e-13 ||A||_inf and
// were perturbed (PARDISO iparm[9] = 13), and the smallest |d| / ||A||_inf seen.
struct PivotStats {
    int64_t factorisations = 0;
    int64_t perturbed = 0;
    double min_pivot_ratio = 1.0 / 0.0;
};

// The full symmetric pattern of the last band factorisation on a handle and its RCM order, on
// the device, kept between calls: a call whose pattern matches (sizes, base, storage and a 64-bit
// hash of rowptr and colind) skips the symmetrisation, the ordering and their uploads.  (The
// reference redoes PARDISO's analysis, phase 11, before every factorisation:
// src/analysis/KrylovROMSubstructure.cpp:647, per expansion point at :408 and per frequency of
// the full-order sweep at :1380.)
struct PatternCache {
    int64_t n = -1, nnz = -1;
    int base = -1, upper = -1;
    uint64_t hash = 0;
    int64_t bw = 0;
    int64_t nfull = 0;  // entries of the full pattern
    int64_t *d_frp = nullptr, *d_fmap = nullptr;
    int *d_fci = nullptr, *d_iperm = nullptr;
    bool last_reused = false;  // the last call found its pattern here
    bool matches(int64_t n_, int64_t nnz_, int base_, int upper_, uint64_t hash_) const {
        return d_frp && n == n_ && nnz == nnz_ && base == base_ && upper == upper_ && hash == hash_;
    }
    // frees the device arrays (after the caller's stream has drained) and forgets the key
    void release();
};

struct KrylovArgs {
    cudaStream_t stream;
    int64_t n_rows, nnz;
    const int64_t *rowptr;  // device, CSR (base 0 or 1), full symmetric or upper storage
    const int *colind;
    int base, upper;
    const void *K, *M, *D;  // device srom_complex values on the pattern; D may be null
    const void *B;          // device n_rows x n_in inputs, leading dimension ldb
    int n_in;
    int64_t ldb;
    const double *exp_points_hz;  // host
    int n_points, order;
    double tol;
    void *V;  // device n_rows x max_cols output, leading dimension ldv
    int64_t ldv;
    int max_cols;
    PivotStats *stats;     // may be null
    PatternCache *cache;   // may be null (no reuse between calls)
};

struct KrylovBlock {
    double point_hz;
    int order, rank;
    std::vector<double> rdiag;  // |R_ii| of the block's pivoted QR
};

struct KrylovLog {
    int64_t bandwidth = 0;
    std::vector<KrylovBlock> blocks;
};

int krylov_basis(const KrylovArgs &a, std::string *msg, int *n_cols, KrylovLog *log);

struct FomArgs {
    cudaStream_t stream;
    int64_t n_rows, nnz;
    const int64_t *rowptr;  // device CSR as in KrylovArgs
    const int *colind;
    int base, upper;
    const void *K, *M, *D;  // device values; D may be null
    const void *F;          // device n_rows x r loads, leading dimension ldf
    int r;
    int64_t ldf;
    const double *freq_hz;  // host
    int n_freq;
    void *X;  // device: n_freq blocks of n_rows x r (leading dimension ldx, block stride ldx * r)
    int64_t ldx;
    PivotStats *stats;     // may be null
    PatternCache *cache;   // may be null (no reuse between calls)
};

// (K - w^2 M + i w D) X_f = F for every frequency: band LDL^T per frequency.
int fom_sweep(const FomArgs &a, std::string *msg);

// host helpers (also behind srom_band_order)
int full_pattern(int64_t n, int64_t nnz, const int64_t *rp, const int *ci, int base, int upper, std::vector<int64_t> &frp,
                 std::vector<int> &fci, std::vector<int64_t> &fmap, std::string *err);
int64_t rcm_order(int64_t n, const std::vector<int64_t> &frp, const std::vector<int> &fci, std::vector<int> &perm);
int64_t band_bytes(int64_t n, int64_t bw);

}  // namespace kry
}  // namespace srom
