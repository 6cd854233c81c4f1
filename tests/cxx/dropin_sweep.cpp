// C++ caller of the C ABI, shaped like the body of KrylovROMSubstructure::backTransformKMOR
// (src/analysis/KrylovROMSubstructure.cpp:1393-1460) with its frequency loop replaced by the C ABI:
// the reduced operators live in host std::vectors of an MKL_Complex16-like struct, the whole
// frequency loop is one srom_sweep_host call, and y = C_r x comes back stacked [w][n_out x r].
//
// usage: dropin_sweep <dir> <eta> <f0_hz> <f1_hz> <count>
//   reads <dir>/K.mtx, M.mtx, BF.mtx (n x r = B_r * F) and C.mtx (n_out x n), writes <dir>/Y.mtx
//   (n_out*r x F: column f holds y(w_f) column-major) and <dir>/info.txt.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "staccato_rom.h"

struct STACCATOComplexDouble {  // layout of MKL_Complex16 / srom_complex
    double real, imag;
};

static std::vector<STACCATOComplexDouble> read(const std::string &path, int64_t &rows, int64_t &cols) {
    char err[256];
    if (srom_mtx_read_dense(path.c_str(), &rows, &cols, nullptr, 0, err, sizeof err) != SROM_OK) {
        std::fprintf(stderr, "%s\n", err);
        std::exit(2);
    }
    std::vector<STACCATOComplexDouble> a((size_t)(rows * cols));
    if (srom_mtx_read_dense(path.c_str(), &rows, &cols, reinterpret_cast<srom_complex *>(a.data()),
                            (int64_t)a.size(), err, sizeof err) != SROM_OK) {
        std::fprintf(stderr, "%s\n", err);
        std::exit(2);
    }
    return a;
}

int main(int argc, char **argv) {
    if (argc != 6) return 1;
    const std::string dir = argv[1];
    const double eta = std::atof(argv[2]), f0 = std::atof(argv[3]), f1 = std::atof(argv[4]);
    const int count = std::atoi(argv[5]);
    int64_t n = 0, n2 = 0, r = 0, n_out = 0;
    std::vector<STACCATOComplexDouble> K = read(dir + "/K.mtx", n, n2);
    std::vector<STACCATOComplexDouble> M = read(dir + "/M.mtx", n, n2);
    std::vector<STACCATOComplexDouble> BF = read(dir + "/BF.mtx", n2, r);
    std::vector<STACCATOComplexDouble> Cr = read(dir + "/C.mtx", n_out, n2);

    std::vector<double> freq(count), omega(count);
    for (int i = 0; i < count; ++i) {
        freq[i] = count > 1 ? f0 + (f1 - f0) * i / (count - 1) : f0;
        omega[i] = 2 * M_PI * freq[i];  // as in backTransformKMOR (:1408)
    }
    std::vector<STACCATOComplexDouble> x((size_t)(count * n * r)), y((size_t)(count * n_out * r));
    std::vector<int> info(count);

    srom_handle *h = nullptr;
    if (srom_create(&h, 0) != SROM_OK) return 3;
    srom_rom_desc d = {};
    d.n = (int)n;
    d.r = (int)r;
    d.F = count;
    d.ldk = (int)n;
    d.K = reinterpret_cast<const srom_complex *>(K.data());
    d.M = reinterpret_cast<const srom_complex *>(M.data());
    d.D = nullptr;
    d.eta = eta;
    d.rhs = reinterpret_cast<const srom_complex *>(BF.data());
    d.ldb = (int)n;
    d.omega = omega.data();
    d.X = reinterpret_cast<srom_complex *>(x.data());
    d.info = info.data();
    d.n_out = (int)n_out;
    d.ldc = (int)n_out;
    d.C = reinterpret_cast<const srom_complex *>(Cr.data());
    d.Y = reinterpret_cast<srom_complex *>(y.data());
    srom_sweep_opts o = {SROM_FP64, 5, 0.0, 0};
    if (srom_sweep_host(h, &d, 1, &o) != SROM_OK) {
        std::fprintf(stderr, "%s\n", srom_last_error(h));
        return 4;
    }
    srom_destroy(h);

    char err[256];
    if (srom_mtx_write_dense((dir + "/Y.mtx").c_str(), n_out * r, count, reinterpret_cast<const srom_complex *>(y.data()),
                             n_out * r, err, sizeof err) != SROM_OK) {
        std::fprintf(stderr, "%s\n", err);
        return 5;
    }
    FILE *fp = std::fopen((dir + "/info.txt").c_str(), "w");
    for (int i = 0; i < count; ++i) std::fprintf(fp, "%d\n", info[i]);
    std::fclose(fp);
    return 0;
}
