// Host-side readers and writers for the dense ROM files of the reference's tests (no GPU work).
//
//   dense Matrix Market  read:  io::readMtxDense (test/krylovTestGPU/matrixInSingleLoop/gpu/
//                               src/io/io.cu:20-80): '%' lines skipped, "rows cols", then the
//                               entries column after column;
//                        write: AuxiliaryFunctions::writeMKLComplexDenseMatrixMtxFormat
//                               (src/tools/AuxiliaryFunctions.cpp:80-110): banner
//                               "%%MatrixMarket matrix coordinate complex dense column major",
//                               "rows<TAB>cols", one "re<TAB>im" line per entry;
//   solution table       write: io::writeSolVecComplex (io.cu:83-106): "Real" / "Imag" header,
//                               two left-aligned columns of width 25, CRLF line ends.
//
// The reader also takes a standard Matrix Market "array real" file (one value per entry; the
// reference's REAL branch reads two numbers per entry, which such files do not have) and the
// reference's "dense row major" banner (entries row after row).  Numbers are written with 17
// significant digits, so a write followed by a read returns the same bits.
#include <cctype>
#include <cerrno>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/staccato_rom.h"

namespace {

int io_fail(char *err, int err_len, int code, const std::string &msg) {
    if (err && err_len > 0) snprintf(err, (size_t)err_len, "%s", msg.c_str());
    return code;
}

bool read_file(const char *path, std::string &out) {
    FILE *fp = fopen(path, "rb");
    if (!fp) return false;
    char buf[1 << 16];
    size_t got;
    while ((got = fread(buf, 1, sizeof buf, fp)) > 0) out.append(buf, got);
    const bool ok = !ferror(fp);
    fclose(fp);
    return ok;
}

std::string lower(std::string s) {
    for (char &c : s) c = (char)tolower((unsigned char)c);
    return s;
}

// Cursor over the file text: skips blanks and '%' comment lines, parses numbers.
struct Cursor {
    const char *p, *end;
    void skip() {
        for (;;) {
            while (p < end && isspace((unsigned char)*p)) ++p;
            if (p < end && *p == '%') {
                while (p < end && *p != '\n') ++p;
                continue;
            }
            return;
        }
    }
    bool number(double &v) {
        skip();
        if (p >= end) return false;
        char *q = nullptr;
        errno = 0;
        v = strtod(p, &q);
        if (q == p) return false;
        p = q;
        return true;
    }
    bool integer(long long &v) {
        skip();
        if (p >= end) return false;
        char *q = nullptr;
        v = strtoll(p, &q, 10);
        if (q == p) return false;
        p = q;
        return true;
    }
};

}  // namespace

extern "C" {

int srom_mtx_read_dense(const char *path, int64_t *rows, int64_t *cols, srom_complex *A, int64_t capacity,
                        char *err, int err_len) {
    if (!path || !rows || !cols) return io_fail(err, err_len, SROM_ERR_INVALID, "path, rows and cols must be non-null");
    std::string text;
    if (!read_file(path, text)) return io_fail(err, err_len, SROM_ERR_INVALID, std::string("cannot read ") + path);
    bool complex_vals = true, row_major = false;
    if (text.compare(0, 14, "%%MatrixMarket") == 0) {
        const std::string banner = lower(text.substr(0, text.find('\n')));
        if (banner.find("complex") == std::string::npos && banner.find("real") != std::string::npos)
            complex_vals = false;
        if (banner.find("integer") != std::string::npos || banner.find("pattern") != std::string::npos)
            return io_fail(err, err_len, SROM_ERR_UNSUPPORTED, "only real or complex dense files are read");
        row_major = banner.find("row major") != std::string::npos;
    }
    Cursor cur{text.data(), text.data() + text.size()};
    long long nr = 0, nc = 0;
    if (!cur.integer(nr) || !cur.integer(nc) || nr < 0 || nc < 0)
        return io_fail(err, err_len, SROM_ERR_INVALID, std::string(path) + ": no \"rows cols\" line");
    *rows = nr;
    *cols = nc;
    if (!A) return SROM_OK;
    const int64_t count = (int64_t)nr * nc;
    if (capacity < count)
        return io_fail(err, err_len, SROM_ERR_INVALID,
                       std::string(path) + ": buffer holds fewer than rows*cols entries");
    for (int64_t e = 0; e < count; ++e) {
        double re = 0.0, im = 0.0;
        if (!cur.number(re) || (complex_vals && !cur.number(im))) {
            char b[160];
            snprintf(b, sizeof b, "%s: file ends after %lld of %lld entries", path, (long long)e, (long long)count);
            return io_fail(err, err_len, SROM_ERR_INVALID, b);
        }
        const int64_t i = row_major ? e / nc : e % nr, j = row_major ? e % nc : e / nr;
        A[i + j * nr] = srom_complex{re, im};
    }
    cur.skip();
    if (cur.p != cur.end)
        return io_fail(err, err_len, SROM_ERR_INVALID, std::string(path) + ": more numbers than rows*cols entries");
    return SROM_OK;
}

int srom_mtx_write_dense(const char *path, int64_t rows, int64_t cols, const srom_complex *A, int64_t lda,
                         char *err, int err_len) {
    if (!path || rows < 0 || cols < 0 || (rows * cols > 0 && !A) || lda < rows)
        return io_fail(err, err_len, SROM_ERR_INVALID, "bad arguments");
    FILE *fp = fopen(path, "wb");
    if (!fp) return io_fail(err, err_len, SROM_ERR_INVALID, std::string("cannot write ") + path);
    fprintf(fp, "%%%%MatrixMarket matrix coordinate complex dense column major\n%lld\t%lld\n", (long long)rows,
            (long long)cols);
    for (int64_t j = 0; j < cols; ++j)
        for (int64_t i = 0; i < rows; ++i) {
            const srom_complex z = A[i + j * lda];
            fprintf(fp, "%.16e\t%.16e\n", z.re, z.im);
        }
    fputc('\n', fp);
    const bool ok = !ferror(fp);
    if (fclose(fp) != 0 || !ok) return io_fail(err, err_len, SROM_ERR_INVALID, std::string("write failed: ") + path);
    return SROM_OK;
}

int srom_write_solution(const char *path, const srom_complex *x, int64_t count, char *err, int err_len) {
    if (!path || count < 0 || (count > 0 && !x)) return io_fail(err, err_len, SROM_ERR_INVALID, "bad arguments");
    FILE *fp = fopen(path, "wb");
    if (!fp) return io_fail(err, err_len, SROM_ERR_INVALID, std::string("cannot write ") + path);
    fprintf(fp, "%-25s    %-25s\r\n", "Real", "Imag");
    for (int64_t i = 0; i < count; ++i) fprintf(fp, "%-25.17g    %-25.17g\r\n", x[i].re, x[i].im);
    const bool ok = !ferror(fp);
    if (fclose(fp) != 0 || !ok) return io_fail(err, err_len, SROM_ERR_INVALID, std::string("write failed: ") + path);
    return SROM_OK;
}

}  // extern "C"
