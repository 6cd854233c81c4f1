// C++ caller of the Krylov basis and full-order sweep entry points, shaped like
// KrylovROMSubstructure::addKrylovModesForExpansionPoint (KrylovROMSubstructure.cpp:367-569) and
// performSolveFOM (:1355-1391): the FE matrices (here a fixed-free chain of n springs and
// masses, 1-based upper CSR as the reference stores them) are copied to the device, the basis
// is generated for two expansion points, and the full-order response is computed at one
// frequency.  Prints the basis size and the largest deviation of V^H V from the identity.
#include <cuda_runtime.h>

#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "staccato_rom.h"

#define CK(x)                                                                     \
    do {                                                                          \
        if ((x) != cudaSuccess) {                                                 \
            std::fprintf(stderr, "%s failed\n", #x);                              \
            return 2;                                                             \
        }                                                                         \
    } while (0)

int main(int argc, char **argv) {
    const int n = argc > 1 ? std::atoi(argv[1]) : 200;
    // upper CSR, base 1: K = tridiag(-1, 2, -1) (last diagonal 1: free end), M = I / n
    std::vector<int64_t> rowptr(n + 1);
    std::vector<int> colind;
    std::vector<srom_complex> K, M;
    rowptr[0] = 1;
    for (int i = 0; i < n; ++i) {
        colind.push_back(i + 1);
        K.push_back({i == n - 1 ? 1.0 : 2.0, 0.0});
        M.push_back({1.0 / n, 0.0});
        if (i + 1 < n) {
            colind.push_back(i + 2);
            K.push_back({-1.0, 0.0});
            M.push_back({0.0, 0.0});
        }
        rowptr[i + 1] = (int64_t)colind.size() + 1;
    }
    const int64_t nnz = (int64_t)colind.size();
    std::vector<srom_complex> B(n, {0.0, 0.0});
    B[n - 1] = {1.0, 0.0};  // unit force at the free end
    const int max_cols = 16;

    int64_t *d_rp;
    int *d_ci;
    srom_complex *d_K, *d_M, *d_B, *d_V, *d_X;
    CK(cudaMalloc(&d_rp, sizeof(int64_t) * (n + 1)));
    CK(cudaMalloc(&d_ci, sizeof(int) * nnz));
    CK(cudaMalloc(&d_K, sizeof(srom_complex) * nnz));
    CK(cudaMalloc(&d_M, sizeof(srom_complex) * nnz));
    CK(cudaMalloc(&d_B, sizeof(srom_complex) * n));
    CK(cudaMalloc(&d_V, sizeof(srom_complex) * n * max_cols));
    CK(cudaMalloc(&d_X, sizeof(srom_complex) * n));
    CK(cudaMemcpy(d_rp, rowptr.data(), sizeof(int64_t) * (n + 1), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d_ci, colind.data(), sizeof(int) * nnz, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d_K, K.data(), sizeof(srom_complex) * nnz, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d_M, M.data(), sizeof(srom_complex) * nnz, cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d_B, B.data(), sizeof(srom_complex) * n, cudaMemcpyHostToDevice));

    srom_handle *h = nullptr;
    if (srom_create(&h, 0) != SROM_OK) return 3;
    const double points[2] = {0.01, 0.05};  // Hz, below and between the first resonances
    int ncols = 0;
    int s = srom_krylov_basis(h, n, nnz, d_rp, d_ci, 1, 1, d_K, d_M, nullptr, d_B, 1, n, points, 2, 4, 1e-8, d_V, n,
                              max_cols, &ncols);
    if (s != SROM_OK) {
        std::fprintf(stderr, "srom_krylov_basis: %s\n", srom_last_error(h));
        return 4;
    }
    std::vector<std::complex<double>> V((size_t)n * ncols);
    CK(cudaMemcpy(V.data(), d_V, sizeof(srom_complex) * n * ncols, cudaMemcpyDeviceToHost));
    double dev = 0.0;
    for (int a = 0; a < ncols; ++a)
        for (int b = 0; b < ncols; ++b) {
            std::complex<double> g = 0.0;
            for (int i = 0; i < n; ++i) g += std::conj(V[(size_t)a * n + i]) * V[(size_t)b * n + i];
            dev = std::fmax(dev, std::abs(g - (a == b ? 1.0 : 0.0)));
        }
    const double freq = 0.03;
    s = srom_fom_sweep(h, n, nnz, d_rp, d_ci, 1, 1, d_K, d_M, nullptr, d_B, 1, n, &freq, 1, d_X, n);
    if (s != SROM_OK) {
        std::fprintf(stderr, "srom_fom_sweep: %s\n", srom_last_error(h));
        return 5;
    }
    srom_complex tip;
    CK(cudaMemcpy(&tip, d_X + (n - 1), sizeof(srom_complex), cudaMemcpyDeviceToHost));
    std::printf("columns %d orthonormality %.3e tip %.17g %.17g\n", ncols, dev, tip.re, tip.im);
    srom_destroy(h);
    return 0;
}
