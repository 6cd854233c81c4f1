// C ABI of the B200 frequency sweep (declarations in include/staccato_rom.h).
//
// Host responsibilities: argument validation, turning the ROM descriptors into one flat,
// cost-sorted list of (ROM, frequency) systems, staging that list to the device, sizing
// scratch memory and launching the persistent kernels on the handle's stream.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <vector>

#include "../../include/staccato_rom.h"
#include "srom_device.cuh"
#include "adjoint_kernels.h"
#include "krylov_kernels.h"
#include "project_kernels.h"
#include "zgemm.h"
#include "sweep_kernels.h"

using srom::Item;
using srom::RomDev;

struct srom_handle {
    int device = 0;
    cudaStream_t stream = nullptr;
    int sm_count = 0;
    int max_smem_optin = 0;
    // per-CTA scratch for the global-storage kernels
    void *scratch = nullptr;
    size_t scratch_bytes = 0;
    // descriptor + work-list staging
    void *d_meta = nullptr;
    size_t d_meta_bytes = 0;
    void *h_meta = nullptr;
    size_t h_meta_bytes = 0;
    cudaEvent_t meta_done = nullptr;
    bool meta_pending = false;
    // device buffers used by srom_sweep_host
    void *d_host_arena = nullptr;
    size_t d_host_arena_bytes = 0;
    // projection / Gram-Schmidt scratch
    void *d_proj = nullptr;
    size_t d_proj_bytes = 0;
    // adjoint descriptors + partials
    void *d_adj = nullptr;
    size_t d_adj_bytes = 0;
    // zeros standing in for M when a descriptor has none (see SweepPlan::null_m)
    void *d_zero = nullptr;
    size_t d_zero_bytes = 0;
    // split-k partials of srom_zgemm_batched
    void *d_zwork = nullptr;
    size_t d_zwork_bytes = 0;
    // pivots of the band factorisations of the last srom_krylov_basis / srom_fom_sweep call
    srom::kry::PivotStats band_stats;
    // full pattern and RCM order of the last band factorisation, reused by a call on the same pattern
    srom::kry::PatternCache band_cache;
    // per-launch profiling
    struct ProfRec {
        std::string name;
        cudaEvent_t a, b;
        long long items;
        double flops, bytes;
    };
    bool prof = false;
    std::vector<ProfRec> recs;
    // FP64 storage class chosen by srom_tune per (n << 16 | r): 0 smem kernel, 1 global kernel
    std::map<long long, int> tune_fp64;
    // mixed-form routing chosen by srom_tune per (n << 16 | r) where the FP64 smem kernel is
    // the FP64 choice: 0 solve in FP64 outright, 1 mixed global kernel
    std::map<long long, int> tune_mixed;
    // SROM_MIXED_AUTO's kernel chosen by srom_tune per (n << 16 | r): 0 CUDA-core, 1 tensor-core
    std::map<long long, int> tune_tc;
    std::vector<cudaEvent_t> event_pool;
    // error word of the last tensor-core sweep (device, inside d_meta) and its pinned host copy
    int *tc_flag_dev = nullptr;
    int *h_flag = nullptr;
    std::string err;
};

namespace {

int set_err(srom_handle *h, int code, const char *fmt, ...) {
    if (h) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof buf, fmt, ap);
        va_end(ap);
        h->err = buf;
    }
    return code;
}

#define SROM_CUDA(h, call)                                                                  \
    do {                                                                                    \
        cudaError_t _e = (call);                                                            \
        if (_e != cudaSuccess)                                                              \
            return set_err((h), SROM_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(_e)); \
    } while (0)

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

int ensure_device_buffer(srom_handle *h, void **ptr, size_t *have, size_t need) {
    if (*have >= need) return SROM_OK;
    if (*ptr) {
        // The previous buffer may still be read by queued work on the handle's stream.
        SROM_CUDA(h, cudaStreamSynchronize(h->stream));
        SROM_CUDA(h, cudaFree(*ptr));
        *ptr = nullptr;
        *have = 0;
    }
    size_t sz = std::max(need, (size_t)(*have * 5 / 4));
    cudaError_t e = cudaMalloc(ptr, sz);
    if (e != cudaSuccess) {
        *ptr = nullptr;
        cudaGetLastError();
        return set_err(h, SROM_ERR_ALLOC, "cudaMalloc(%zu) failed: %s", sz, cudaGetErrorString(e));
    }
    *have = sz;
    return SROM_OK;
}

int ensure_host_pinned(srom_handle *h, size_t need) {
    if (h->h_meta_bytes >= need) return SROM_OK;
    if (h->meta_pending) {
        SROM_CUDA(h, cudaEventSynchronize(h->meta_done));
        h->meta_pending = false;
    }
    if (h->h_meta) SROM_CUDA(h, cudaFreeHost(h->h_meta));
    h->h_meta = nullptr;
    size_t sz = std::max(need, h->h_meta_bytes * 2);
    SROM_CUDA(h, cudaMallocHost(&h->h_meta, sz));
    h->h_meta_bytes = sz;
    return SROM_OK;
}

size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

cudaEvent_t pooled_event(srom_handle *h) {
    if (!h->event_pool.empty()) {
        cudaEvent_t e = h->event_pool.back();
        h->event_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}

// Brackets one launch with events when profiling is on.
struct ProfScope {
    srom_handle *h;
    int idx = -1;
    ProfScope(srom_handle *h_, const char *name, long long items, double flops, double bytes) : h(h_) {
        if (!h->prof) return;
        srom_handle::ProfRec r{name, pooled_event(h), pooled_event(h), items, flops, bytes};
        cudaEventRecord(r.a, h->stream);
        h->recs.push_back(r);
        idx = (int)h->recs.size() - 1;
    }
    ~ProfScope() {
        if (idx >= 0) cudaEventRecord(h->recs[idx].b, h->stream);
    }
};

double lu_flops(int n, int r) { return 8.0 / 3.0 * (double)n * n * n + 8.0 * (double)n * n * r; }

int validate_desc(srom_handle *h, const srom_rom_desc &d, int idx) {
    if (d.n < 0 || d.r < 0 || d.F < 0) return set_err(h, SROM_ERR_INVALID, "rom %d: negative size", idx);
    if (d.n == 0 || d.F == 0 || d.r == 0) return SROM_OK;
    if (!d.K || !d.rhs || !d.omega || !d.X)
        return set_err(h, SROM_ERR_INVALID, "rom %d: K, rhs, omega and X must be non-null", idx);
    if (d.ldk < d.n) return set_err(h, SROM_ERR_INVALID, "rom %d: ldk (%d) < n (%d)", idx, d.ldk, d.n);
    if (d.ldb < d.n) return set_err(h, SROM_ERR_INVALID, "rom %d: ldb (%d) < n (%d)", idx, d.ldb, d.n);
    if ((d.LU == nullptr) != (d.ipiv == nullptr))
        return set_err(h, SROM_ERR_INVALID, "rom %d: LU and ipiv must be given together", idx);
    if (d.n_out < 0) return set_err(h, SROM_ERR_INVALID, "rom %d: negative n_out", idx);
    if (d.n_out > 0) {
        if (!d.C || !d.Y) return set_err(h, SROM_ERR_INVALID, "rom %d: n_out > 0 needs C and Y", idx);
        if (d.ldc < d.n_out) return set_err(h, SROM_ERR_INVALID, "rom %d: ldc (%d) < n_out (%d)", idx, d.ldc, d.n_out);
    }
    return SROM_OK;
}

// Device descriptors (srom_sweep, graphs, srom_sweep_backward): every array must be aligned to
// its element's vector width.  srom_sweep_host copies into its own aligned arena instead.
int validate_device_alignment(srom_handle *h, const srom_rom_desc &d, int idx) {
    if (d.n == 0 || d.F == 0 || d.r == 0) return SROM_OK;
    const void *cz[] = {d.K, d.M, d.D, d.rhs, d.X, d.LU, d.C, d.Y};
    for (const void *p : cz)
        if (srom::misaligned(p, 16))
            return set_err(h, SROM_ERR_INVALID, "rom %d: complex arrays on the device must be 16-byte aligned", idx);
    if (srom::misaligned(d.omega, 8) || srom::misaligned(d.berr, 8) || srom::misaligned(d.info, 4) ||
        srom::misaligned(d.steps, 4) || srom::misaligned(d.ipiv, 4))
        return set_err(h, SROM_ERR_INVALID, "rom %d: omega/berr must be 8-byte and info/steps/ipiv 4-byte aligned", idx);
    return SROM_OK;
}

// Back-projection launch parameters of a descriptor (n_out = 0: none).
srom::BackProj backproj_of(const srom_rom_desc &d) {
    srom::BackProj b{};
    if (d.n_out <= 0 || d.n == 0 || d.F == 0 || d.r == 0) return b;
    b.n = d.n;
    b.r = d.r;
    b.F = d.F;
    b.n_out = d.n_out;
    b.ldc = d.ldc;
    b.C = reinterpret_cast<const double2 *>(d.C);
    b.X = reinterpret_cast<const double2 *>(d.X);
    b.Y = reinterpret_cast<double2 *>(d.Y);
    return b;
}

RomDev to_dev(const srom_rom_desc &d) {
    RomDev r;
    r.n = d.n;
    r.r = d.r;
    r.F = d.F;
    r.ldk = d.ldk;
    r.K = reinterpret_cast<const double2 *>(d.K);
    r.M = reinterpret_cast<const double2 *>(d.M);
    r.D = reinterpret_cast<const double2 *>(d.D);
    r.eta = d.eta;
    r.rhs = reinterpret_cast<const double2 *>(d.rhs);
    r.ldb = d.ldb;
    r.omega = d.omega;
    r.X = reinterpret_cast<double2 *>(d.X);
    r.info = d.info;
    r.steps = d.steps;
    r.berr = d.berr;
    r.LU = reinterpret_cast<double2 *>(d.LU);
    r.ipiv = d.ipiv;
    return r;
}

}  // namespace

extern "C" {

int srom_version(void) { return 100; }

const char *srom_status_string(int s) {
    switch (s) {
        case SROM_OK: return "ok";
        case SROM_ERR_INVALID: return "invalid argument";
        case SROM_ERR_CUDA: return "CUDA error";
        case SROM_ERR_ALLOC: return "device allocation failed";
        case SROM_ERR_TIMEOUT: return "device wait timed out";
        case SROM_ERR_UNSUPPORTED: return "unsupported shape or option";
        default: return "unknown status";
    }
}

const char *srom_last_error(const srom_handle *h) { return h ? h->err.c_str() : "null handle"; }

int srom_create(srom_handle **out, int device) {
    if (!out) return SROM_ERR_INVALID;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return SROM_ERR_CUDA;
    }
    if (device < 0 || device >= ndev) return SROM_ERR_INVALID;
    srom_handle *h = new srom_handle();
    h->device = device;
    DeviceGuard g(device);
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device) != cudaSuccess) {
        delete h;
        return SROM_ERR_CUDA;
    }
    h->sm_count = prop.multiProcessorCount;
    h->max_smem_optin = (int)prop.sharedMemPerBlockOptin;
    if (cudaEventCreateWithFlags(&h->meta_done, cudaEventDisableTiming) != cudaSuccess) {
        delete h;
        return SROM_ERR_CUDA;
    }
    *out = h;
    return SROM_OK;
}

int srom_destroy(srom_handle *h) {
    if (!h) return SROM_OK;
    DeviceGuard g(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    else cudaDeviceSynchronize();
    if (h->scratch) cudaFree(h->scratch);
    if (h->d_meta) cudaFree(h->d_meta);
    if (h->d_host_arena) cudaFree(h->d_host_arena);
    if (h->d_proj) cudaFree(h->d_proj);
    if (h->d_adj) cudaFree(h->d_adj);
    if (h->d_zero) cudaFree(h->d_zero);
    if (h->d_zwork) cudaFree(h->d_zwork);
    h->band_cache.release();
    if (h->h_meta) cudaFreeHost(h->h_meta);
    if (h->h_flag) cudaFreeHost(h->h_flag);
    if (h->meta_done) cudaEventDestroy(h->meta_done);
    for (auto &r : h->recs) {
        cudaEventDestroy(r.a);
        cudaEventDestroy(r.b);
    }
    for (auto e : h->event_pool) cudaEventDestroy(e);
    delete h;
    return SROM_OK;
}

int srom_set_stream(srom_handle *h, void *stream) {
    if (!h) return SROM_ERR_INVALID;
    h->stream = reinterpret_cast<cudaStream_t>(stream);
    return SROM_OK;
}

int srom_profile_enable(srom_handle *h, int enable) {
    if (!h) return SROM_ERR_INVALID;
    h->prof = enable != 0;
    return SROM_OK;
}

int srom_profile_read(srom_handle *h, srom_kernel_time *out, int max, int *count) {
    if (!h) return SROM_ERR_INVALID;
    DeviceGuard g(h->device);
    int k = 0;
    for (auto &r : h->recs) {
        SROM_CUDA(h, cudaEventSynchronize(r.b));
        if (out && k < max) {
            srom_kernel_time &t = out[k];
            memset(&t, 0, sizeof t);
            strncpy(t.name, r.name.c_str(), sizeof(t.name) - 1);
            SROM_CUDA(h, cudaEventElapsedTime(&t.ms, r.a, r.b));
            t.items = r.items;
            t.flops = r.flops;
            t.bytes = r.bytes;
        }
        ++k;
        h->event_pool.push_back(r.a);
        h->event_pool.push_back(r.b);
    }
    h->recs.clear();
    if (count) *count = k;
    return SROM_OK;
}

}  // extern "C"

namespace {

// A validated, classified and ordered sweep: the host image of the device metadata
// (descriptors, cost-ordered work lists, fallback list, zeroed counters) plus launch shapes.
// Storage classes of a plan: 0 FP64 shared-memory kernel, 1 global kernel (FP64, or the
// CUDA-core mixed kernel), 2 large-order FP64 kernel, 3 tensor-core mixed kernel.
constexpr int NCLS = 4;

struct SweepPlan {
    bool mixed = false;
    srom_sweep_opts o{};
    std::vector<char> meta;
    size_t off_items[NCLS] = {0, 0, 0, 0};
    size_t off_fb = 0, off_ctr = 0;
    long long n_items[NCLS] = {0, 0, 0, 0};
    double flops[NCLS] = {0.0, 0.0, 0.0, 0.0};
    size_t smem_max = 0;
    int g_nmax = 0, g_rmax = 0;    // class 1: the global kernels' largest order and RHS count
    int b_nmax = 0, b_rmax = 0;    // class 2: the large-order FP64 kernel's
    int t_nmax = 0, t_rmax = 0;    // class 3: the tensor-core kernel's
    int f_nmax = 0, f_rmax = 0;    // the FP64 re-solve of non-converged mixed systems (classes 1, 3)
    long long grid0 = 0, grid1 = 0, grid2 = 0, grid3 = 0;
    int64_t slot_bytes = 0, slot2_bytes = 0, slot3_bytes = 0, slotf_bytes = 0;
    bool need_scratch = false;
    std::vector<srom::BackProj> backproj;  // ROMs whose solutions are projected onto outputs
    // ROMs without a mass matrix.  Their descriptors point M at a zero matrix instead: for any
    // finite w, K + (-w^2)*0 adds -0, which leaves every value (and the sign of zero) as it is,
    // so the kernels compute (1 + i eta) K + i w D bit for bit without a second code path.
    std::vector<int> null_m;
    size_t zero_bytes = 0;
};

// Point the mass matrix of every ROM in P.null_m at the zero buffer (host image of the metadata).
void patch_null_m(SweepPlan &P, const void *zero) {
    RomDev *rd = reinterpret_cast<RomDev *>(P.meta.data());
    for (int i : P.null_m) rd[i].M = static_cast<const double2 *>(zero);
}

// Systems whose panel does not fit the global kernel's shared memory (n above ~690 for r = 1,
// less for more right-hand sides; every n > 768) run on the large-order FP64 kernel (class 2).
bool large_order(const srom_handle *h, int n, int r) { return !srom::global_panel_fits(n, r, h->max_smem_optin); }

// FP64 storage class of an n x n system with r right-hand sides: 0 smem kernel, 1 global
// kernel, 2 large-order global kernel.  The tuning table (srom_tune) overrides the default
// "smem when it fits".
int fp64_class(const srom_handle *h, int n, int r) {
    if (large_order(h, n, r)) return 2;
    const bool fits = srom::fp64_smem_bytes(n, r) <= (size_t)h->max_smem_optin;
    if (!fits) return 1;
    auto it = h->tune_fp64.find(((long long)n << 16) | r);
    if (it != h->tune_fp64.end()) return it->second;
    return 0;
}

// Mixed-form class: a system the FP64 shared-memory kernel holds two or more at a time per SM
// is solved there outright.  At those orders (n <= ~84 for r <= 4) one FP64 factorisation in
// shared memory is faster than complex-FP32 factors in the global kernel plus refinement
// (measured 1.5-2.2x at n = 32..80), and its result is the FP64 form's, bit for bit (steps = 0).
// Larger systems, or any with SROM_FLAG_MIXED_EVERY, go to the mixed global kernel.  Orders
// whose panel does not fit the global kernel's shared memory have no mixed kernel: they run on
// the large-order FP64 kernel (steps = 0).
int mixed_class(const srom_handle *h, int n, int r, int flags) {
    if (large_order(h, n, r)) return 2;
    if (flags & SROM_FLAG_MIXED_EVERY) return 1;
    if (fp64_class(h, n, r) != 0) return 1;
    auto it = h->tune_mixed.find(((long long)n << 16) | r);  // srom_tune's measurement, if any
    if (it != h->tune_mixed.end()) return it->second;
    return srom::fp64_smem_blocks_per_sm(srom::fp64_smem_bytes(n, r)) >= 2 ? 0 : 1;
}

// SROM_MIXED_AUTO: the tensor-core kernel from this order up (without a measurement).  On the
// batching shapes it is 2-8 % faster than the CUDA-core kernel from n = 384 on and 8 % slower at
// n = 256 (r = 8); the factorisation's panel, inverse blocks and per-column work weigh more at
// smaller orders.
constexpr int TC_AUTO_MIN_N = 320;

// Whether a mixed system of the global class runs on the tensor-core kernel.
bool use_tc(const srom_handle *h, int n, int r, int precision) {
    if (n > srom::TC_MAX_N) return false;
    if (precision == SROM_MIXED_TC) return true;
    if (precision != SROM_MIXED_AUTO) return false;
    auto it = h->tune_tc.find(((long long)n << 16) | r);
    if (it != h->tune_tc.end()) return it->second != 0;
    return n >= TC_AUTO_MIN_N;
}

int make_plan(srom_handle *h, const srom_rom_desc *roms, int n_roms, const srom_sweep_opts *opts, SweepPlan &P) {
    if (n_roms < 0 || (n_roms > 0 && !roms)) return set_err(h, SROM_ERR_INVALID, "roms is null");
    srom_sweep_opts o = opts ? *opts : srom_sweep_opts{SROM_FP64, 5, 0.0, 0};
    if (o.precision != SROM_FP64 && o.precision != SROM_MIXED_FP32 && o.precision != SROM_MIXED_TC &&
        o.precision != SROM_MIXED_AUTO)
        return set_err(h, SROM_ERR_UNSUPPORTED, "precision %d not available in this build", o.precision);
    const bool mixed = o.precision != SROM_FP64;
    if (o.max_refine <= 0) o.max_refine = 5;
    if (o.tol < 0.0) return set_err(h, SROM_ERR_INVALID, "tol must be >= 0");
    for (int i = 0; i < n_roms; ++i) {
        int s = validate_desc(h, roms[i], i);
        if (!s) s = validate_device_alignment(h, roms[i], i);
        if (s) return s;
        if (mixed && roms[i].LU)
            return set_err(h, SROM_ERR_UNSUPPORTED, "rom %d: factors are kept only by the FP64 form", i);
        if (mixed && roms[i].r > srom::MIXED_MAX_R)
            return set_err(h, SROM_ERR_UNSUPPORTED, "rom %d: mixed form supports r <= %d", i, srom::MIXED_MAX_R);
    }
    P.mixed = mixed;
    P.o = o;
    // FP64: systems that fit shared memory use the smem kernel (unless tuned otherwise),
    // the rest the global kernel.  Mixed: the smallest systems use the FP64 smem kernel
    // (mixed_class), the rest the mixed global kernel.
    const size_t smem_cap = (size_t)h->max_smem_optin;
    std::vector<RomDev> dev(n_roms);
    std::vector<int> cls(n_roms, -1);
    for (int i = 0; i < n_roms; ++i) {
        dev[i] = to_dev(roms[i]);
        if (!roms[i].M && roms[i].n > 0 && roms[i].F > 0 && roms[i].r > 0) {
            P.null_m.push_back(i);
            P.zero_bytes = std::max(P.zero_bytes, sizeof(srom_complex) * (size_t)roms[i].ldk * roms[i].n);
        }
        if (roms[i].n_out > 0 && roms[i].n > 0 && roms[i].F > 0 && roms[i].r > 0)
            P.backproj.push_back(backproj_of(roms[i]));
        const srom_rom_desc &d = roms[i];
        if (d.n == 0 || d.F == 0 || d.r == 0) continue;
        cls[i] = mixed ? mixed_class(h, d.n, d.r, o.flags) : fp64_class(h, d.n, d.r);
    }
    // The global kernel runs with the largest n and the largest r of its systems: while that
    // pair does not fit, the largest system moves to the large-order FP64 kernel.
    for (;;) {
        int gn = 0, gr = 0, big = -1;
        for (int i = 0; i < n_roms; ++i)
            if (cls[i] == 1) {
                gn = std::max(gn, roms[i].n);
                gr = std::max(gr, roms[i].r);
                if (big < 0 || roms[i].n > roms[big].n) big = i;
            }
        if (big < 0 || srom::global_panel_fits(gn, gr, h->max_smem_optin)) break;
        cls[big] = 2;
    }
    // mixed systems of the global class that the tensor-core kernel takes (SROM_MIXED_TC: every
    // one it can; SROM_MIXED_AUTO: where it is the faster); if the kernel cannot run their
    // largest order and RHS count together, they stay on the CUDA-core kernel
    if (mixed) {
        int tn = 0, tr = 0;
        for (int i = 0; i < n_roms; ++i)
            if (cls[i] == 1 && use_tc(h, roms[i].n, roms[i].r, o.precision)) {
                cls[i] = 3;
                tn = std::max(tn, roms[i].n);
                tr = std::max(tr, roms[i].r);
            }
        if (tn > 0 && !srom::tc_supported(tn, tr, h->max_smem_optin, nullptr))
            for (int i = 0; i < n_roms; ++i)
                if (cls[i] == 3) cls[i] = 1;
    }
    for (int i = 0; i < n_roms; ++i) {
        const srom_rom_desc &d = roms[i];
        if (cls[i] < 0) continue;
        if (cls[i] == 0) {
            P.smem_max = std::max(P.smem_max, srom::fp64_smem_bytes(d.n, d.r));
        } else if (cls[i] == 1) {
            P.g_nmax = std::max(P.g_nmax, d.n);
            P.g_rmax = std::max(P.g_rmax, d.r);
        } else if (cls[i] == 2) {
            P.b_nmax = std::max(P.b_nmax, d.n);
            P.b_rmax = std::max(P.b_rmax, d.r);
        } else {
            P.t_nmax = std::max(P.t_nmax, d.n);
            P.t_rmax = std::max(P.t_rmax, d.r);
        }
        P.n_items[cls[i]] += d.F;
        P.flops[cls[i]] += lu_flops(d.n, d.r) * d.F;
    }
    if (P.b_nmax > srom::BIG_MAX_N)
        return set_err(h, SROM_ERR_UNSUPPORTED, "n=%d exceeds the largest supported order %d", P.b_nmax,
                       srom::BIG_MAX_N);
    if (P.b_nmax > 0 && srom::global_smem_bytes(P.b_nmax, P.b_rmax, true) + srom::GLOBAL_STATIC_SMEM > smem_cap)
        return set_err(h, SROM_ERR_UNSUPPORTED,
                       "n=%d with r=%d: the right-hand sides (n*r*16 bytes) exceed shared memory", P.b_nmax,
                       P.b_rmax);
    if (P.n_items[0] + P.n_items[1] + P.n_items[2] + P.n_items[3] > INT32_MAX)
        return set_err(h, SROM_ERR_UNSUPPORTED, "too many systems");
    if (P.n_items[0] > 0) {
        const int bps = srom::fp64_smem_blocks_per_sm(P.smem_max);
        if (bps <= 0) return set_err(h, SROM_ERR_UNSUPPORTED, "smem kernel cannot be resident (%zu B)", P.smem_max);
        P.grid0 = std::min<long long>(P.n_items[0], (long long)bps * h->sm_count);
    }
    if (P.n_items[1] > 0) {
        P.grid1 = std::min<long long>(P.n_items[1], h->sm_count);
        P.slot_bytes = (int64_t)P.g_nmax * P.g_nmax * (int64_t)sizeof(double2);
        P.need_scratch = mixed;
        for (int i = 0; i < n_roms; ++i)
            if (cls[i] == 1 && !roms[i].LU) P.need_scratch = true;
    }
    if (P.n_items[3] > 0) {
        P.grid3 = std::min<long long>(P.n_items[3], h->sm_count);
        P.slot3_bytes = (int64_t)srom::tc_slot_bytes(P.t_nmax);
        P.need_scratch = true;
    }
    if (mixed && (o.flags & SROM_FLAG_FALLBACK_FP64) && P.n_items[1] + P.n_items[3] > 0) {
        // the FP64 re-solve covers the systems of both mixed kernels, one CTA per SM
        P.f_nmax = std::max(P.g_nmax, P.t_nmax);
        P.f_rmax = std::max(P.g_rmax, P.t_rmax);
        P.slotf_bytes = srom::global_panel_fits(P.f_nmax, P.f_rmax, h->max_smem_optin)
                            ? (int64_t)P.f_nmax * P.f_nmax * (int64_t)sizeof(double2)
                            : srom::big_slot_bytes(P.f_nmax);
    }
    if (P.n_items[2] > 0) {
        // one system per CTA: matrix (or the caller's LU buffer) and the panel in the CTA's slot;
        // classes 1 and 2 run one after the other and share the scratch buffer
        P.grid2 = std::min<long long>(P.n_items[2], h->sm_count);
        P.slot2_bytes = srom::big_slot_bytes(P.b_nmax);
        P.need_scratch = true;
    }
    // Work lists: largest systems first (longest-processing-time order for the persistent CTAs).
    std::vector<int> order(n_roms);
    for (int i = 0; i < n_roms; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return roms[a].n > roms[b].n; });
    P.off_items[0] = align_up(sizeof(RomDev) * std::max(n_roms, 1), 256);
    for (int c = 1; c < NCLS; ++c)
        P.off_items[c] = P.off_items[c - 1] + align_up(sizeof(Item) * (size_t)P.n_items[c - 1] + 1, 256);
    P.off_fb = P.off_items[NCLS - 1] + align_up(sizeof(Item) * (size_t)P.n_items[NCLS - 1] + 1, 256);
    P.off_ctr = P.off_fb + (mixed ? align_up(sizeof(Item) * (size_t)(P.n_items[1] + P.n_items[3]) + 1, 256) : 0);
    P.meta.assign(P.off_ctr + 256, 0);
    char *hm = P.meta.data();
    if (n_roms) memcpy(hm, dev.data(), sizeof(RomDev) * n_roms);
    Item *its[NCLS];
    for (int c = 0; c < NCLS; ++c) its[c] = reinterpret_cast<Item *>(hm + P.off_items[c]);
    long long k[NCLS] = {0, 0, 0, 0};
    for (int oi = 0; oi < n_roms; ++oi) {
        const int i = order[oi];
        if (cls[i] < 0) continue;
        for (int f = 0; f < roms[i].F; ++f) its[cls[i]][k[cls[i]]++] = Item{i, f};
    }
    return SROM_OK;
}

// Scratch bytes of a plan: the global, tensor-core, FP64 re-solve and large-order launches run
// one after the other on one stream and share it.
size_t plan_scratch_bytes(const SweepPlan &P) {
    size_t b = std::max<size_t>((size_t)P.slot_bytes * P.grid1, (size_t)P.slot2_bytes * P.grid2);
    b = std::max<size_t>(b, (size_t)P.slot3_bytes * P.grid3);
    return std::max<size_t>(b, (size_t)P.slotf_bytes * std::max(P.grid1, P.grid3));
}

// Counters live at off_ctr and must be zero when the launches start (the metadata copy zeroes
// them, or zero_counters does): 0 smem kernel, 1 global kernel, 2 fallback count, 3 fallback
// work, 4 tensor-core error word, 5 large-order kernel, 6 tensor-core kernel.
int enqueue_plan(srom_handle *h, const SweepPlan &P, char *dm, void *scratch, cudaStream_t st, bool zero_counters,
                 bool profile) {
    const RomDev *d_roms = reinterpret_cast<const RomDev *>(dm);
    auto items = [&](int c) { return reinterpret_cast<const Item *>(dm + P.off_items[c]); };
    int *d_ctr = reinterpret_cast<int *>(dm + P.off_ctr);
    if (zero_counters) SROM_CUDA(h, cudaMemsetAsync(d_ctr, 0, 8 * sizeof(int), st));
    const bool prof_prev = h->prof;
    if (!profile) h->prof = false;
    int rc = SROM_OK;
    if (P.n_items[0] > 0) {
        ProfScope ps(h, "fp64_smem", P.n_items[0], P.flops[0], 0.0);
        cudaError_t e = srom::launch_fp64_smem(d_roms, items(0), (int)P.n_items[0], d_ctr, P.smem_max, (int)P.grid0, st);
        if (e != cudaSuccess) rc = set_err(h, SROM_ERR_CUDA, "fp64 smem launch: %s", cudaGetErrorString(e));
    }
    Item *fb_items = nullptr;
    int *fb_count = nullptr;
    if (P.mixed && (P.o.flags & SROM_FLAG_FALLBACK_FP64)) {
        fb_items = reinterpret_cast<Item *>(dm + P.off_fb);
        fb_count = d_ctr + 2;
    }
    auto mixed_args = [&](int c, int *counter, int64_t slot, int n_max, int r_max) {
        srom::GlobalArgs a{};
        a.roms = d_roms;
        a.items = items(c);
        a.n_items = (int)P.n_items[c];
        a.counter = counter;
        a.scratch = static_cast<unsigned char *>(scratch);
        a.slot_bytes = slot;
        a.n_max = n_max;
        a.r_max = r_max;
        a.max_refine = P.o.max_refine;
        a.tol = P.o.tol;
        a.fb_items = fb_items;
        a.fb_count = fb_count;
        return a;
    };
    if (rc == SROM_OK && P.n_items[1] > 0) {
        srom::GlobalArgs a = mixed_args(1, d_ctr + 1, P.slot_bytes, P.g_nmax, P.g_rmax);
        if (!P.mixed) a.fb_items = nullptr, a.fb_count = nullptr;
        ProfScope ps(h, P.mixed ? "mixed_global" : "fp64_global", P.n_items[1], P.flops[1], 0.0);
        cudaError_t e = srom::launch_global(P.mixed, a, (int)P.grid1, st);
        if (e != cudaSuccess) rc = set_err(h, SROM_ERR_CUDA, "global launch: %s", cudaGetErrorString(e));
    }
    if (rc == SROM_OK && P.n_items[3] > 0) {
        srom::GlobalArgs a = mixed_args(3, d_ctr + 6, P.slot3_bytes, P.t_nmax, P.t_rmax);
        a.err_flag = d_ctr + 4;
        ProfScope ps(h, "mixed_tc", P.n_items[3], P.flops[3], 0.0);
        cudaError_t e = srom::launch_tc(a, (int)P.grid3, st);
        if (e != cudaSuccess) rc = set_err(h, SROM_ERR_CUDA, "tensor-core launch: %s", cudaGetErrorString(e));
    }
    if (rc == SROM_OK && fb_items && P.n_items[1] + P.n_items[3] > 0) {
        // FP64 re-solve of the systems the mixed kernels could not refine; the item count stays
        // on the device, so the launch needs no host synchronisation
        srom::GlobalArgs b{};
        b.roms = d_roms;
        b.items = fb_items;
        b.n_items_dev = fb_count;
        b.counter = d_ctr + 3;
        b.scratch = static_cast<unsigned char *>(scratch);
        b.slot_bytes = P.slotf_bytes;
        b.n_max = P.f_nmax;
        b.r_max = P.f_rmax;
        b.steps_value = -1;
        const int grid = (int)std::max(P.grid1, P.grid3);
        ProfScope ps(h, "fp64_fallback", 0, 0.0, 0.0);
        cudaError_t e = srom::global_panel_fits(P.f_nmax, P.f_rmax, h->max_smem_optin)
                            ? srom::launch_global(false, b, grid, st)
                            : srom::launch_global_big(b, grid, st);
        if (e != cudaSuccess) rc = set_err(h, SROM_ERR_CUDA, "fallback launch: %s", cudaGetErrorString(e));
    }
    if (rc == SROM_OK && P.n_items[2] > 0) {
        srom::GlobalArgs a{};
        a.roms = d_roms;
        a.items = items(2);
        a.n_items = (int)P.n_items[2];
        a.counter = d_ctr + 5;
        a.scratch = static_cast<unsigned char *>(scratch);
        a.slot_bytes = P.slot2_bytes;
        a.n_max = P.b_nmax;
        a.r_max = P.b_rmax;
        ProfScope ps(h, "fp64_large", P.n_items[2], P.flops[2], 0.0);
        cudaError_t e = srom::launch_global_big(a, (int)P.grid2, st);
        if (e != cudaSuccess) rc = set_err(h, SROM_ERR_CUDA, "large-order launch: %s", cudaGetErrorString(e));
    }
    for (size_t i = 0; rc == SROM_OK && i < P.backproj.size(); ++i) {
        const srom::BackProj &b = P.backproj[i];
        ProfScope ps(h, "backproject", b.F, 8.0 * (double)b.n_out * b.n * b.r * b.F, 0.0);
        cudaError_t e = srom::launch_backproject(b, h->sm_count, st);
        if (e != cudaSuccess) rc = set_err(h, SROM_ERR_CUDA, "back-projection launch: %s", cudaGetErrorString(e));
    }
    h->prof = prof_prev;
    return rc;
}

}  // namespace

struct srom_graph {
    srom_handle *h = nullptr;
    void *d_meta = nullptr;
    void *scratch = nullptr;
    void *d_zero = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

extern "C" {

int srom_sweep(srom_handle *h, const srom_rom_desc *roms, int n_roms, const srom_sweep_opts *opts) {
    if (!h) return SROM_ERR_INVALID;
    h->err.clear();
    SweepPlan P;
    int s = make_plan(h, roms, n_roms, opts, P);
    if (s) return s;
    DeviceGuard g(h->device);
    s = ensure_host_pinned(h, P.meta.size());
    if (s) return s;
    if (h->meta_pending) {
        SROM_CUDA(h, cudaEventSynchronize(h->meta_done));
        h->meta_pending = false;
    }
    s = ensure_device_buffer(h, &h->d_meta, &h->d_meta_bytes, P.meta.size());
    if (s) return s;
    void *scr = nullptr;
    if (P.need_scratch) {
        s = ensure_device_buffer(h, &h->scratch, &h->scratch_bytes, plan_scratch_bytes(P));
        if (s) return s;
        scr = h->scratch;
    }
    if (P.zero_bytes > 0) {
        const size_t before = h->d_zero_bytes;
        s = ensure_device_buffer(h, &h->d_zero, &h->d_zero_bytes, P.zero_bytes);
        if (s) return s;
        if (h->d_zero_bytes != before) SROM_CUDA(h, cudaMemsetAsync(h->d_zero, 0, h->d_zero_bytes, h->stream));
        patch_null_m(P, h->d_zero);
    }
    memcpy(h->h_meta, P.meta.data(), P.meta.size());
    SROM_CUDA(h, cudaMemcpyAsync(h->d_meta, h->h_meta, P.meta.size(), cudaMemcpyHostToDevice, h->stream));
    SROM_CUDA(h, cudaEventRecord(h->meta_done, h->stream));
    h->meta_pending = true;
    h->tc_flag_dev = P.n_items[3] > 0 ? reinterpret_cast<int *>(static_cast<char *>(h->d_meta) + P.off_ctr) + 4 : nullptr;
    return enqueue_plan(h, P, static_cast<char *>(h->d_meta), scr, h->stream, false, true);
}

int srom_graph_create(srom_handle *h, const srom_rom_desc *roms, int n_roms, const srom_sweep_opts *opts,
                      srom_graph **out) {
    if (!h || !out) return SROM_ERR_INVALID;
    *out = nullptr;
    h->err.clear();
    SweepPlan P;
    int s = make_plan(h, roms, n_roms, opts, P);
    if (s) return s;
    DeviceGuard g(h->device);
    srom_graph *G = new srom_graph();
    G->h = h;
    auto fail = [&](int code) {
        if (G->d_meta) cudaFree(G->d_meta);
        if (G->scratch) cudaFree(G->scratch);
        if (G->d_zero) cudaFree(G->d_zero);
        if (G->exec) cudaGraphExecDestroy(G->exec);
        if (G->graph) cudaGraphDestroy(G->graph);
        delete G;
        return code;
    };
    cudaError_t e = cudaMalloc(&G->d_meta, P.meta.size());
    if (e != cudaSuccess) return fail(set_err(h, SROM_ERR_ALLOC, "graph metadata: %s", cudaGetErrorString(e)));
    if (P.need_scratch && (e = cudaMalloc(&G->scratch, plan_scratch_bytes(P))) != cudaSuccess)
        return fail(set_err(h, SROM_ERR_ALLOC, "graph scratch: %s", cudaGetErrorString(e)));
    if (P.zero_bytes > 0) {
        if ((e = cudaMalloc(&G->d_zero, P.zero_bytes)) != cudaSuccess)
            return fail(set_err(h, SROM_ERR_ALLOC, "graph zero matrix: %s", cudaGetErrorString(e)));
        if ((e = cudaMemset(G->d_zero, 0, P.zero_bytes)) != cudaSuccess)
            return fail(set_err(h, SROM_ERR_CUDA, "graph zero matrix: %s", cudaGetErrorString(e)));
        patch_null_m(P, G->d_zero);
    }
    if ((e = cudaMemcpy(G->d_meta, P.meta.data(), P.meta.size(), cudaMemcpyHostToDevice)) != cudaSuccess)
        return fail(set_err(h, SROM_ERR_CUDA, "graph metadata copy: %s", cudaGetErrorString(e)));
    cudaStream_t cs;
    if ((e = cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking)) != cudaSuccess)
        return fail(set_err(h, SROM_ERR_CUDA, "capture stream: %s", cudaGetErrorString(e)));
    // Kernel attributes are set before capture (the launchers set them on every call).
    if ((e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal)) != cudaSuccess) {
        cudaStreamDestroy(cs);
        return fail(set_err(h, SROM_ERR_CUDA, "begin capture: %s", cudaGetErrorString(e)));
    }
    s = enqueue_plan(h, P, static_cast<char *>(G->d_meta), G->scratch, cs, true, false);
    cudaGraph_t graph = nullptr;
    e = cudaStreamEndCapture(cs, &graph);
    cudaStreamDestroy(cs);
    if (s) {
        if (graph) cudaGraphDestroy(graph);
        return fail(s);
    }
    if (e != cudaSuccess) return fail(set_err(h, SROM_ERR_CUDA, "end capture: %s", cudaGetErrorString(e)));
    G->graph = graph;
    if ((e = cudaGraphInstantiate(&G->exec, graph, 0)) != cudaSuccess)
        return fail(set_err(h, SROM_ERR_CUDA, "instantiate: %s", cudaGetErrorString(e)));
    *out = G;
    return SROM_OK;
}

int srom_graph_launch(srom_graph *G, void *stream) {
    if (!G || !G->exec) return SROM_ERR_INVALID;
    DeviceGuard g(G->h->device);
    cudaError_t e = cudaGraphLaunch(G->exec, reinterpret_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) return set_err(G->h, SROM_ERR_CUDA, "graph launch: %s", cudaGetErrorString(e));
    return SROM_OK;
}

int srom_graph_destroy(srom_graph *G) {
    if (!G) return SROM_OK;
    DeviceGuard g(G->h->device);
    cudaDeviceSynchronize();
    if (G->exec) cudaGraphExecDestroy(G->exec);
    if (G->graph) cudaGraphDestroy(G->graph);
    if (G->d_meta) cudaFree(G->d_meta);
    if (G->scratch) cudaFree(G->scratch);
    if (G->d_zero) cudaFree(G->d_zero);
    delete G;
    return SROM_OK;
}

int srom_band_pivot_report(const srom_handle *h, int64_t *factorisations, int64_t *perturbed,
                           double *min_pivot_ratio) {
    if (!h) return SROM_ERR_INVALID;
    if (factorisations) *factorisations = h->band_stats.factorisations;
    if (perturbed) *perturbed = h->band_stats.perturbed;
    if (min_pivot_ratio) *min_pivot_ratio = h->band_stats.min_pivot_ratio;
    return SROM_OK;
}

int srom_band_cache_report(const srom_handle *h, int *reused, int64_t *cached_rows, int64_t *bandwidth) {
    if (!h) return SROM_ERR_INVALID;
    const srom::kry::PatternCache &c = h->band_cache;
    if (reused) *reused = c.last_reused ? 1 : 0;
    if (cached_rows) *cached_rows = c.d_frp ? c.n : 0;
    if (bandwidth) *bandwidth = c.d_frp ? c.bw : 0;
    return SROM_OK;
}

int srom_band_cache_release(srom_handle *h) {
    if (!h) return SROM_ERR_INVALID;
    DeviceGuard g(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    h->band_cache.release();
    return SROM_OK;
}

int srom_zgemm_batched(srom_handle *h, int opa, int opb, int m, int n, int k, srom_complex alpha, const srom_complex *A,
                       int64_t lda, int64_t stride_a, const srom_complex *B, int64_t ldb, int64_t stride_b,
                       srom_complex beta, srom_complex *C, int64_t ldc, int64_t stride_c, int batch) {
    if (!h) return SROM_ERR_INVALID;
    h->err.clear();
    if (m < 0 || n < 0 || k < 0 || batch < 0) return set_err(h, SROM_ERR_INVALID, "negative size");
    if (opa < SROM_OP_N || opa > SROM_OP_C || opb < SROM_OP_N || opb > SROM_OP_C)
        return set_err(h, SROM_ERR_INVALID, "op must be SROM_OP_N, SROM_OP_T or SROM_OP_C");
    if (m == 0 || n == 0 || batch == 0) return SROM_OK;
    const int64_t arows = opa == SROM_OP_N ? m : k, brows = opb == SROM_OP_N ? k : n;
    if (lda < std::max<int64_t>(1, arows) || ldb < std::max<int64_t>(1, brows) || ldc < std::max(1, m))
        return set_err(h, SROM_ERR_INVALID, "leading dimension too small (lda %lld, ldb %lld, ldc %lld)",
                       (long long)lda, (long long)ldb, (long long)ldc);
    if (stride_a < 0 || stride_b < 0 || stride_c < 0) return set_err(h, SROM_ERR_INVALID, "negative stride");
    if (!C || (k > 0 && (!A || !B))) return set_err(h, SROM_ERR_INVALID, "A, B and C must be non-null");
    if (srom::misaligned(A, 16) || srom::misaligned(B, 16) || srom::misaligned(C, 16))
        return set_err(h, SROM_ERR_INVALID, "A, B and C must be 16-byte aligned");
    if ((int64_t)batch > 65535) return set_err(h, SROM_ERR_UNSUPPORTED, "batch %d exceeds 65535", batch);
    DeviceGuard g(h->device);
    srom::Zgemm z;
    z.opa = opa;
    z.opb = opb;
    z.m = m;
    z.n = n;
    z.k = k;
    z.alpha = make_double2(alpha.re, alpha.im);
    z.beta = make_double2(beta.re, beta.im);
    z.A = reinterpret_cast<const double2 *>(A);
    z.lda = lda;
    z.sa = stride_a;
    z.B = reinterpret_cast<const double2 *>(B);
    z.ldb = ldb;
    z.sb = stride_b;
    z.C = reinterpret_cast<double2 *>(C);
    z.ldc = ldc;
    z.sc = stride_c;
    z.batch = batch;
    z.sms = h->sm_count;
    const int64_t we = srom::zgemm_work_elems(m, n, k, batch, h->sm_count);
    if (we > 0) {
        int s = ensure_device_buffer(h, &h->d_zwork, &h->d_zwork_bytes, sizeof(double2) * (size_t)we);
        if (s) return s;
        z.work = static_cast<double2 *>(h->d_zwork);
        z.work_elems = (int64_t)(h->d_zwork_bytes / sizeof(double2));
    }
    ProfScope ps(h, "zgemm", batch, 8.0 * m * n * (double)k * batch, 0.0);
    SROM_CUDA(h, srom::zgemm(z, h->stream));
    return SROM_OK;
}

int srom_project_real(srom_handle *h, int64_t n_rows, const int64_t *rowptr, const int *colind, int base, int upper,
                      const double *const *vals, int n_mats, const double *V, int k, int64_t ldv, double *const *R) {
    if (!h) return SROM_ERR_INVALID;
    h->err.clear();
    if (n_rows < 0 || k < 0) return set_err(h, SROM_ERR_INVALID, "negative size");
    if (n_mats < 1 || n_mats > 3) return set_err(h, SROM_ERR_INVALID, "n_mats must be 1..3");
    if (k > srom::PRJ_MAX_K) return set_err(h, SROM_ERR_UNSUPPORTED, "k = %d exceeds %d", k, srom::PRJ_MAX_K);
    if (base != 0 && base != 1) return set_err(h, SROM_ERR_INVALID, "base must be 0 or 1");
    if (!vals || !R) return set_err(h, SROM_ERR_INVALID, "vals and R must be non-null");
    for (int m = 0; m < n_mats; ++m)
        if (!vals[m] || !R[m]) return set_err(h, SROM_ERR_INVALID, "vals[%d] / R[%d] is null", m, m);
    if (n_rows == 0 || k == 0) return SROM_OK;
    if (!rowptr || !colind || !V) return set_err(h, SROM_ERR_INVALID, "rowptr, colind and V must be non-null");
    if (ldv < n_rows) return set_err(h, SROM_ERR_INVALID, "ldv < n_rows");
    DeviceGuard g(h->device);
    const int nblk = h->sm_count;  // one V^T Y CTA per SM
    const size_t vt_b = align_up(sizeof(double) * (size_t)n_rows * k, 256);
    const size_t y_b = align_up(sizeof(double) * (size_t)n_rows * k * n_mats, 256);
    const size_t p_b = align_up(sizeof(double) * srom::vty_partial_doubles(k, n_mats, nblk), 256);
    int s = ensure_device_buffer(h, &h->d_proj, &h->d_proj_bytes, vt_b + y_b + p_b);
    if (s) return s;
    char *base_p = static_cast<char *>(h->d_proj);
    double *Vt = reinterpret_cast<double *>(base_p);
    double *Y = reinterpret_cast<double *>(base_p + vt_b);
    double *part = reinterpret_cast<double *>(base_p + vt_b + y_b);
    srom::ProjVals pv{};
    srom::ProjOut po{};
    for (int m = 0; m < n_mats; ++m) {
        pv.v[m] = vals[m];
        po.r[m] = R[m];
    }
    SROM_CUDA(h, srom::launch_transpose(V, n_rows, k, ldv, Vt, h->stream));
    {
        ProfScope ps(h, "spmm", n_rows, 0.0, 0.0);
        SROM_CUDA(h, srom::launch_spmm(n_rows, rowptr, colind, base, upper, pv, n_mats, Vt, k, Y,
                                       (int64_t)n_rows * k, h->sm_count, h->stream));
    }
    {
        ProfScope ps(h, "vty_dmma", n_rows, 2.0 * (double)n_rows * k * k * n_mats, 0.0);
        SROM_CUDA(h, srom::launch_vty(n_rows, k, Vt, Y, (int64_t)n_rows * k, n_mats, nblk, part, po, h->stream));
    }
    return SROM_OK;
}

int srom_project_complex(srom_handle *h, int64_t n_rows, int64_t nnz, const int64_t *rowptr, const int *colind,
                         int base, int upper, const srom_complex *const *vals, int n_mats, const srom_complex *V, int k,
                         int64_t ldv, const srom_complex *Z, int64_t ldz, srom_complex *const *R) {
    if (!h) return SROM_ERR_INVALID;
    h->err.clear();
    if (n_rows < 0 || k < 0 || nnz < 0) return set_err(h, SROM_ERR_INVALID, "negative size");
    if (n_mats < 1 || n_mats > 3) return set_err(h, SROM_ERR_INVALID, "n_mats must be 1..3");
    if (k > srom::PRJ_MAX_K / 2)
        return set_err(h, SROM_ERR_UNSUPPORTED, "k = %d exceeds %d (complex form)", k, srom::PRJ_MAX_K / 2);
    if (base != 0 && base != 1) return set_err(h, SROM_ERR_INVALID, "base must be 0 or 1");
    if (!vals || !R) return set_err(h, SROM_ERR_INVALID, "vals and R must be non-null");
    for (int m = 0; m < n_mats; ++m)
        if (!vals[m] || !R[m]) return set_err(h, SROM_ERR_INVALID, "vals[%d] / R[%d] is null", m, m);
    if (n_rows == 0 || k == 0) return SROM_OK;
    if (!rowptr || !colind || !V) return set_err(h, SROM_ERR_INVALID, "rowptr, colind and V must be non-null");
    if (ldv < n_rows || (Z && ldz < n_rows)) return set_err(h, SROM_ERR_INVALID, "ldv / ldz < n_rows");
    bool bad = srom::misaligned(V, 16) || srom::misaligned(Z, 16) || srom::misaligned(rowptr, 8) ||
               srom::misaligned(colind, 4);
    for (int m = 0; m < n_mats; ++m) bad = bad || srom::misaligned(vals[m], 16) || srom::misaligned(R[m], 16);
    if (bad) return set_err(h, SROM_ERR_INVALID, "complex arrays must be 16-byte aligned (rowptr 8, colind 4)");
    DeviceGuard g(h->device);
    const int k2 = 2 * k;
    const int nblk = h->sm_count;
    const size_t w_b = align_up(sizeof(double) * (size_t)n_rows * k2, 256);
    const size_t v_b = align_up(sizeof(double) * (size_t)nnz, 256);
    const size_t p_b = align_up(sizeof(double) * srom::vty_partial_doubles(k2, 1, nblk), 256);
    const size_t g_b = align_up(sizeof(double) * (size_t)k2 * k2, 256);
    // Vt2 [Re V | Im V], Zt2 (when Z is given), Ar, Ai, P_r, P_i, partials, G
    const size_t need = w_b * (Z ? 4 : 3) + 2 * v_b + p_b + g_b;
    int s = ensure_device_buffer(h, &h->d_proj, &h->d_proj_bytes, need);
    if (s) return s;
    char *bp = static_cast<char *>(h->d_proj);
    double *Vt2 = reinterpret_cast<double *>(bp);
    bp += w_b;
    double *Zt2 = Vt2;
    if (Z) {
        Zt2 = reinterpret_cast<double *>(bp);
        bp += w_b;
    }
    double *Pr = reinterpret_cast<double *>(bp);
    bp += w_b;
    double *Pi = reinterpret_cast<double *>(bp);
    bp += w_b;
    double *Ar = reinterpret_cast<double *>(bp);
    bp += v_b;
    double *Ai = reinterpret_cast<double *>(bp);
    bp += v_b;
    double *part = reinterpret_cast<double *>(bp);
    bp += p_b;
    double *G = reinterpret_cast<double *>(bp);
    SROM_CUDA(h, srom::launch_transpose_split(reinterpret_cast<const double2 *>(V), n_rows, k, ldv, Vt2, h->stream));
    if (Z) SROM_CUDA(h, srom::launch_transpose_split(reinterpret_cast<const double2 *>(Z), n_rows, k, ldz, Zt2, h->stream));
    for (int m = 0; m < n_mats; ++m) {
        SROM_CUDA(h, srom::launch_split_values(reinterpret_cast<const double2 *>(vals[m]), nnz, Ar, Ai, h->sm_count,
                                               h->stream));
        srom::ProjVals pv{};
        pv.v[0] = Ar;
        pv.v[1] = Ai;
        {
            ProfScope ps(h, "spmm_complex", n_rows, 0.0, 0.0);
            // P_r and P_i are adjacent: the SpMM writes matrix m' of pv at Pr + m' * (n_rows * 2k)
            SROM_CUDA(h, srom::launch_spmm(n_rows, rowptr, colind, base, upper, pv, 2, Vt2, k2, Pr,
                                           (int64_t)(Pi - Pr), h->sm_count, h->stream));
        }
        SROM_CUDA(h, srom::launch_combine_y(Pr, Pi, n_rows, k, h->sm_count, h->stream));
        srom::ProjOut po{};
        po.r[0] = G;
        {
            ProfScope ps(h, "vty_dmma_complex", n_rows, 2.0 * (double)n_rows * k2 * k2, 0.0);
            SROM_CUDA(h, srom::launch_vty(n_rows, k2, Zt2, Pr, 0, 1, nblk, part, po, h->stream));
        }
        SROM_CUDA(h, srom::launch_combine_r(G, k, reinterpret_cast<double2 *>(R[m]), h->stream));
    }
    return SROM_OK;
}

int srom_sweep_backward(srom_handle *h, const srom_rom_desc *rom, const srom_complex *gbar, int ldg,
                        const srom_dparam *params, int n_params, double *dJdp, srom_complex *lambda) {
    if (!h) return SROM_ERR_INVALID;
    h->err.clear();
    if (!rom) return set_err(h, SROM_ERR_INVALID, "rom is null");
    int s = validate_desc(h, *rom, 0);
    if (!s) s = validate_device_alignment(h, *rom, 0);
    if (s) return s;
    if (srom::misaligned(gbar, 16) || srom::misaligned(lambda, 16) || srom::misaligned(dJdp, 8))
        return set_err(h, SROM_ERR_INVALID, "gbar/lambda must be 16-byte and dJdp 8-byte aligned");
    if (n_params < 0 || (n_params > 0 && (!params || !dJdp)))
        return set_err(h, SROM_ERR_INVALID, "params and dJdp must be non-null");
    if (rom->n == 0 || rom->F == 0 || rom->r == 0 || n_params == 0) {
        if (n_params > 0) SROM_CUDA(h, cudaMemsetAsync(dJdp, 0, sizeof(double) * n_params, h->stream));
        return SROM_OK;
    }
    if (!rom->LU || !rom->ipiv) return set_err(h, SROM_ERR_INVALID, "rom->LU / rom->ipiv missing: run srom_sweep with SROM_FLAG_KEEP_FACTORS");
    if (!gbar || ldg < rom->n) return set_err(h, SROM_ERR_INVALID, "gbar null or ldg < n");
    std::vector<srom::DParamDev> pd(n_params);
    std::vector<srom::DParamTerm> terms;
    for (int j = 0; j < n_params; ++j) {
        const srom_dparam &p = params[j];
        if (srom::misaligned(p.U, 16) || srom::misaligned(p.W, 16) || srom::misaligned(p.G, 16))
            return set_err(h, SROM_ERR_INVALID, "param %d: U, W and G must be 16-byte aligned", j);
        srom::DParamDev &d = pd[j];
        d.kind = p.kind;
        d.rank = p.rank;
        d.U = reinterpret_cast<const double2 *>(p.U);
        d.W = reinterpret_cast<const double2 *>(p.W);
        d.s = p.s;
        d.G = reinterpret_cast<const double2 *>(p.G);
        d.c0 = make_double2(p.c0.re, p.c0.im);
        d.c1 = make_double2(p.c1.re, p.c1.im);
        d.c2 = make_double2(p.c2.re, p.c2.im);
        d.term0 = (int)terms.size();
        if (p.kind == SROM_DPARAM_LOWRANK) {
            if (p.rank < 0 || (p.rank > 0 && !p.U)) return set_err(h, SROM_ERR_INVALID, "param %d: U missing", j);
            for (int k = 0; k < p.rank; ++k) terms.push_back({j, k});
        } else if (p.kind == SROM_DPARAM_DENSE) {
            if (!p.G) return set_err(h, SROM_ERR_INVALID, "param %d: G missing", j);
            terms.push_back({j, 0});
        } else {
            return set_err(h, SROM_ERR_INVALID, "param %d: unknown kind %d", j, p.kind);
        }
        d.nterm = (int)terms.size() - d.term0;
    }
    const size_t smem = srom::adjoint_smem_bytes(rom->n, rom->r, (int)terms.size());
    if (smem > (size_t)h->max_smem_optin) return set_err(h, SROM_ERR_UNSUPPORTED, "n*r or parameter terms too large");
    DeviceGuard g(h->device);
    const size_t o_rom = 0, o_par = align_up(sizeof(RomDev), 256);
    const size_t o_term = o_par + align_up(sizeof(srom::DParamDev) * n_params, 256);
    const size_t o_ctr = o_term + align_up(sizeof(srom::DParamTerm) * std::max<size_t>(terms.size(), 1), 256);
    const size_t o_part = o_ctr + 256;
    const size_t total = o_part + sizeof(double) * (size_t)rom->F * n_params;
    if (h->meta_pending) {
        SROM_CUDA(h, cudaEventSynchronize(h->meta_done));
        h->meta_pending = false;
    }
    s = ensure_host_pinned(h, o_part);
    if (s) return s;
    s = ensure_device_buffer(h, &h->d_adj, &h->d_adj_bytes, total);
    if (s) return s;
    char *hm = static_cast<char *>(h->h_meta);
    RomDev rd = to_dev(*rom);
    memcpy(hm + o_rom, &rd, sizeof rd);
    memcpy(hm + o_par, pd.data(), sizeof(srom::DParamDev) * n_params);
    if (!terms.empty()) memcpy(hm + o_term, terms.data(), sizeof(srom::DParamTerm) * terms.size());
    memset(hm + o_ctr, 0, 256);
    char *dm = static_cast<char *>(h->d_adj);
    SROM_CUDA(h, cudaMemcpyAsync(dm, hm, o_part, cudaMemcpyHostToDevice, h->stream));
    SROM_CUDA(h, cudaEventRecord(h->meta_done, h->stream));
    h->meta_pending = true;
    srom::AdjointArgs a{};
    a.rom = reinterpret_cast<const RomDev *>(dm + o_rom);
    a.gbar = reinterpret_cast<const double2 *>(gbar);
    a.ldg = ldg;
    a.ldg_f = (int64_t)ldg * rom->r;
    a.params = reinterpret_cast<const srom::DParamDev *>(dm + o_par);
    a.n_params = n_params;
    a.terms = reinterpret_cast<const srom::DParamTerm *>(dm + o_term);
    a.n_terms = (int)terms.size();
    a.partial = reinterpret_cast<double *>(dm + o_part);
    a.lambda = reinterpret_cast<double2 *>(lambda);
    a.counter = reinterpret_cast<int *>(dm + o_ctr);
    const int grid = std::min(rom->F, h->sm_count * 4);
    const double n3 = (double)rom->n * rom->n;
    ProfScope ps(h, "adjoint", rom->F, (8.0 * n3 * rom->r) * rom->F, 0.0);
    SROM_CUDA(h, srom::launch_adjoint(a, rom->n, rom->r, rom->F, grid, dJdp, h->stream));
    return SROM_OK;
}

int srom_krylov_basis(srom_handle *h, int64_t n_rows, int64_t nnz, const int64_t *rowptr, const int *colind, int base,
                      int upper, const srom_complex *K, const srom_complex *M, const srom_complex *D,
                      const srom_complex *B, int n_in, int64_t ldb, const double *exp_points_hz, int n_points,
                      int krylov_order, double tol, srom_complex *V, int64_t ldv, int max_cols, int *n_cols) {
    if (!h) return SROM_ERR_INVALID;
    h->err.clear();
    if (!n_cols) return set_err(h, SROM_ERR_INVALID, "n_cols is null");
    *n_cols = 0;
    if (n_rows < 0 || nnz < 0 || n_in < 0 || n_points < 0 || max_cols < 0)
        return set_err(h, SROM_ERR_INVALID, "negative size");
    if (n_rows > INT32_MAX - 1) return set_err(h, SROM_ERR_UNSUPPORTED, "n_rows above 2^31 - 2");
    if (base != 0 && base != 1) return set_err(h, SROM_ERR_INVALID, "base must be 0 or 1");
    if (krylov_order < 1) return set_err(h, SROM_ERR_INVALID, "krylov_order must be >= 1");
    if (n_rows == 0 || n_in == 0 || n_points == 0) return SROM_OK;
    if (!rowptr || !colind || !K || !M || !B || !V || !exp_points_hz)
        return set_err(h, SROM_ERR_INVALID, "rowptr, colind, K, M, B, V and exp_points_hz must be non-null");
    if (ldb < n_rows || ldv < n_rows) return set_err(h, SROM_ERR_INVALID, "ldb and ldv must be >= n_rows");
    if (n_rows * (int64_t)n_in > INT32_MAX) return set_err(h, SROM_ERR_UNSUPPORTED, "n_rows * n_in above 2^31 - 1");
    if (srom::misaligned(K, 16) || srom::misaligned(M, 16) || srom::misaligned(D, 16) || srom::misaligned(B, 16) ||
        srom::misaligned(V, 16) || srom::misaligned(rowptr, 8) || srom::misaligned(colind, 4))
        return set_err(h, SROM_ERR_INVALID, "complex arrays must be 16-byte aligned (rowptr 8, colind 4)");
    for (int i = 0; i < n_points; ++i)
        if (!std::isfinite(exp_points_hz[i])) return set_err(h, SROM_ERR_INVALID, "expansion point %d is not finite", i);
    DeviceGuard g(h->device);
    srom::kry::KrylovArgs a{};
    a.stream = h->stream;
    a.n_rows = n_rows;
    a.nnz = nnz;
    a.rowptr = rowptr;
    a.colind = colind;
    a.base = base;
    a.upper = upper ? 1 : 0;
    a.K = K;
    a.M = M;
    a.D = D;
    a.B = B;
    a.n_in = n_in;
    a.ldb = ldb;
    a.exp_points_hz = exp_points_hz;
    a.n_points = n_points;
    a.order = krylov_order;
    a.tol = tol > 0.0 ? tol : 1e-8;
    a.V = V;
    a.ldv = ldv;
    a.max_cols = max_cols;
    h->band_stats = srom::kry::PivotStats{};
    a.stats = &h->band_stats;
    a.cache = &h->band_cache;
    h->band_cache.last_reused = false;
    std::string msg;
    ProfScope ps(h, "krylov_basis", n_points, 0.0, 0.0);
    const int s = srom::kry::krylov_basis(a, &msg, n_cols, nullptr);
    if (s) return set_err(h, s, "%s", msg.c_str());
    return SROM_OK;
}

int srom_fom_sweep(srom_handle *h, int64_t n_rows, int64_t nnz, const int64_t *rowptr, const int *colind, int base,
                   int upper, const srom_complex *K, const srom_complex *M, const srom_complex *D, const srom_complex *F,
                   int r, int64_t ldf, const double *freq_hz, int n_freq, srom_complex *X, int64_t ldx) {
    if (!h) return SROM_ERR_INVALID;
    h->err.clear();
    if (n_rows < 0 || nnz < 0 || r < 0 || n_freq < 0) return set_err(h, SROM_ERR_INVALID, "negative size");
    if (n_rows > INT32_MAX - 1) return set_err(h, SROM_ERR_UNSUPPORTED, "n_rows above 2^31 - 2");
    if (base != 0 && base != 1) return set_err(h, SROM_ERR_INVALID, "base must be 0 or 1");
    if (n_rows == 0 || r == 0 || n_freq == 0) return SROM_OK;
    if (!rowptr || !colind || !K || !M || !F || !X || !freq_hz)
        return set_err(h, SROM_ERR_INVALID, "rowptr, colind, K, M, F, X and freq_hz must be non-null");
    if (ldf < n_rows || ldx < n_rows) return set_err(h, SROM_ERR_INVALID, "ldf and ldx must be >= n_rows");
    if (n_rows * (int64_t)r > INT32_MAX) return set_err(h, SROM_ERR_UNSUPPORTED, "n_rows * r above 2^31 - 1");
    if (srom::misaligned(K, 16) || srom::misaligned(M, 16) || srom::misaligned(D, 16) || srom::misaligned(F, 16) ||
        srom::misaligned(X, 16) || srom::misaligned(rowptr, 8) || srom::misaligned(colind, 4))
        return set_err(h, SROM_ERR_INVALID, "complex arrays must be 16-byte aligned (rowptr 8, colind 4)");
    for (int i = 0; i < n_freq; ++i)
        if (!std::isfinite(freq_hz[i])) return set_err(h, SROM_ERR_INVALID, "frequency %d is not finite", i);
    DeviceGuard g(h->device);
    srom::kry::FomArgs a{};
    a.stream = h->stream;
    a.n_rows = n_rows;
    a.nnz = nnz;
    a.rowptr = rowptr;
    a.colind = colind;
    a.base = base;
    a.upper = upper ? 1 : 0;
    a.K = K;
    a.M = M;
    a.D = D;
    a.F = F;
    a.r = r;
    a.ldf = ldf;
    a.freq_hz = freq_hz;
    a.n_freq = n_freq;
    a.X = X;
    a.ldx = ldx;
    h->band_stats = srom::kry::PivotStats{};
    a.stats = &h->band_stats;
    a.cache = &h->band_cache;
    h->band_cache.last_reused = false;
    std::string msg;
    ProfScope ps(h, "fom_sweep", n_freq, 0.0, 0.0);
    const int s = srom::kry::fom_sweep(a, &msg);
    if (s) return set_err(h, s, "%s", msg.c_str());
    return SROM_OK;
}

int srom_band_order(int64_t n_rows, int64_t nnz, const int64_t *rowptr, const int *colind, int base, int upper,
                    int *perm, int64_t *bandwidth, int64_t *band_bytes_out, char *err, int err_len) {
    auto fail = [&](int code, const std::string &m) {
        if (err && err_len > 0) snprintf(err, (size_t)err_len, "%s", m.c_str());
        return code;
    };
    if (err && err_len > 0) err[0] = 0;
    if (n_rows < 0 || nnz < 0) return fail(SROM_ERR_INVALID, "negative size");
    if (n_rows > INT32_MAX - 1) return fail(SROM_ERR_UNSUPPORTED, "n_rows above 2^31 - 2");
    if (base != 0 && base != 1) return fail(SROM_ERR_INVALID, "base must be 0 or 1");
    if (n_rows > 0 && (!rowptr || (nnz > 0 && !colind))) return fail(SROM_ERR_INVALID, "rowptr and colind must be non-null");
    if (n_rows > 0 && (rowptr[0] != base || rowptr[n_rows] - base != nnz))
        return fail(SROM_ERR_INVALID, "rowptr does not start at base or does not end at base + nnz");
    std::vector<int64_t> frp, fmap;
    std::vector<int> fci, p;
    std::string m;
    int s = srom::kry::full_pattern(n_rows, nnz, rowptr, colind, base, upper, frp, fci, fmap, &m);
    if (s) return fail(s, m);
    const int64_t bw = srom::kry::rcm_order(n_rows, frp, fci, p);
    if (perm) std::copy(p.begin(), p.end(), perm);
    if (bandwidth) *bandwidth = bw;
    if (band_bytes_out) *band_bytes_out = srom::kry::band_bytes(n_rows, bw);
    return SROM_OK;
}

int srom_orthonormalize(srom_handle *h, double *V, int64_t n_rows, int k, int64_t ldv, int passes) {
    if (!h) return SROM_ERR_INVALID;
    h->err.clear();
    if (n_rows < 0 || k < 0 || passes < 0) return set_err(h, SROM_ERR_INVALID, "negative size");
    if (n_rows == 0 || k == 0) return SROM_OK;
    if (!V) return set_err(h, SROM_ERR_INVALID, "V is null");
    if (ldv < n_rows) return set_err(h, SROM_ERR_INVALID, "ldv < n_rows");
    if (k > n_rows) return set_err(h, SROM_ERR_INVALID, "k > n_rows: columns cannot be orthonormal");
    DeviceGuard g(h->device);
    const int nblk = h->sm_count;
    const size_t need = sizeof(double) * srom::gs_workspace_doubles(k, nblk);
    int s = ensure_device_buffer(h, &h->d_proj, &h->d_proj_bytes, need);
    if (s) return s;
    ProfScope ps(h, "gram_schmidt", k, 4.0 * (double)n_rows * k * k * std::max(passes, 1), 0.0);
    SROM_CUDA(h, srom::launch_gram_schmidt(V, n_rows, k, ldv, passes, static_cast<double *>(h->d_proj), nblk,
                                           h->stream));
    return SROM_OK;
}

int srom_sweep_host(srom_handle *h, const srom_rom_desc *roms, int n_roms, const srom_sweep_opts *opts) {
    if (!h) return SROM_ERR_INVALID;
    h->err.clear();
    if (n_roms < 0 || (n_roms > 0 && !roms)) return set_err(h, SROM_ERR_INVALID, "roms is null");
    for (int i = 0; i < n_roms; ++i) {
        int s = validate_desc(h, roms[i], i);
        if (s) return s;
    }
    DeviceGuard g(h->device);
    // Lay out every input and output of every ROM in one device arena.
    std::vector<size_t> offs(n_roms * 11, 0);
    size_t total = 0;
    auto take = [&](size_t bytes) {
        size_t o = total;
        total = align_up(total + bytes, 256);
        return o;
    };
    for (int i = 0; i < n_roms; ++i) {
        const srom_rom_desc &d = roms[i];
        if (d.n == 0 || d.F == 0 || d.r == 0) continue;
        const size_t nn = (size_t)d.ldk * d.n, cz = sizeof(srom_complex);
        size_t *o = &offs[i * 11];
        o[0] = take(cz * nn);
        o[1] = d.M ? take(cz * nn) : 0;
        o[2] = d.D ? take(cz * nn) : 0;
        o[3] = take(cz * (size_t)d.ldb * d.r);
        o[4] = take(sizeof(double) * d.F);
        o[5] = take(cz * (size_t)d.F * d.n * d.r);
        o[6] = d.info ? take(sizeof(int) * d.F) : 0;
        o[7] = d.steps ? take(sizeof(int) * d.F) : 0;
        o[8] = d.berr ? take(sizeof(double) * d.F) : 0;
        if (d.n_out > 0) {
            o[9] = take(cz * (size_t)d.ldc * d.n);
            o[10] = take(cz * (size_t)d.F * d.n_out * d.r);
        }
    }
    int s = ensure_device_buffer(h, &h->d_host_arena, &h->d_host_arena_bytes, std::max<size_t>(total, 256));
    if (s) return s;
    char *base = static_cast<char *>(h->d_host_arena);
    std::vector<srom_rom_desc> dd(roms, roms + n_roms);
    const cudaMemcpyKind H2D = cudaMemcpyHostToDevice, D2H = cudaMemcpyDeviceToHost;
    for (int i = 0; i < n_roms; ++i) {
        const srom_rom_desc &d = roms[i];
        if (d.n == 0 || d.F == 0 || d.r == 0) continue;
        const size_t nn = (size_t)d.ldk * d.n, cz = sizeof(srom_complex);
        size_t *o = &offs[i * 11];
        srom_rom_desc &e = dd[i];
        e.K = reinterpret_cast<const srom_complex *>(base + o[0]);
        e.M = d.M ? reinterpret_cast<const srom_complex *>(base + o[1]) : nullptr;
        e.D = d.D ? reinterpret_cast<const srom_complex *>(base + o[2]) : nullptr;
        e.rhs = reinterpret_cast<const srom_complex *>(base + o[3]);
        e.omega = reinterpret_cast<const double *>(base + o[4]);
        e.X = reinterpret_cast<srom_complex *>(base + o[5]);
        e.info = d.info ? reinterpret_cast<int *>(base + o[6]) : nullptr;
        e.steps = d.steps ? reinterpret_cast<int *>(base + o[7]) : nullptr;
        e.berr = d.berr ? reinterpret_cast<double *>(base + o[8]) : nullptr;
        e.LU = nullptr;
        e.ipiv = nullptr;
        if (d.n_out > 0) {
            e.C = reinterpret_cast<const srom_complex *>(base + o[9]);
            e.Y = reinterpret_cast<srom_complex *>(base + o[10]);
            SROM_CUDA(h, cudaMemcpyAsync((void *)e.C, d.C, cz * (size_t)d.ldc * d.n, H2D, h->stream));
        }
        SROM_CUDA(h, cudaMemcpyAsync((void *)e.K, d.K, cz * nn, H2D, h->stream));
        if (d.M) SROM_CUDA(h, cudaMemcpyAsync((void *)e.M, d.M, cz * nn, H2D, h->stream));
        if (d.D) SROM_CUDA(h, cudaMemcpyAsync((void *)e.D, d.D, cz * nn, H2D, h->stream));
        SROM_CUDA(h, cudaMemcpyAsync((void *)e.rhs, d.rhs, cz * (size_t)d.ldb * d.r, H2D, h->stream));
        SROM_CUDA(h, cudaMemcpyAsync((void *)e.omega, d.omega, sizeof(double) * d.F, H2D, h->stream));
    }
    s = srom_sweep(h, dd.data(), n_roms, opts);
    if (s) return s;
    int *flag_dev = h->tc_flag_dev;
    if (flag_dev) {
        if (!h->h_flag) SROM_CUDA(h, cudaMallocHost(reinterpret_cast<void **>(&h->h_flag), sizeof(int)));
        SROM_CUDA(h, cudaMemcpyAsync(h->h_flag, flag_dev, sizeof(int), D2H, h->stream));
    }
    for (int i = 0; i < n_roms; ++i) {
        const srom_rom_desc &d = roms[i];
        const srom_rom_desc &e = dd[i];
        if (d.n == 0 || d.F == 0 || d.r == 0) continue;
        SROM_CUDA(h, cudaMemcpyAsync(d.X, e.X, sizeof(srom_complex) * (size_t)d.F * d.n * d.r, D2H, h->stream));
        if (d.info) SROM_CUDA(h, cudaMemcpyAsync(d.info, e.info, sizeof(int) * d.F, D2H, h->stream));
        if (d.steps) SROM_CUDA(h, cudaMemcpyAsync(d.steps, e.steps, sizeof(int) * d.F, D2H, h->stream));
        if (d.berr) SROM_CUDA(h, cudaMemcpyAsync(d.berr, e.berr, sizeof(double) * d.F, D2H, h->stream));
        if (d.n_out > 0)
            SROM_CUDA(h, cudaMemcpyAsync(d.Y, e.Y, sizeof(srom_complex) * (size_t)d.F * d.n_out * d.r, D2H,
                                         h->stream));
    }
    SROM_CUDA(h, cudaStreamSynchronize(h->stream));
    if (flag_dev && *h->h_flag)
        return set_err(h, SROM_ERR_TIMEOUT, "a bounded device-side wait of the tensor-core kernel ran out "
                                            "(systems with info = -2 were not solved)");
    return SROM_OK;
}

int srom_tune(srom_handle *h, const int *n_values, int count, int r, const char *cache_path) {
    if (!h) return SROM_ERR_INVALID;
    h->err.clear();
    if (count < 0 || (count > 0 && !n_values) || r < 1) return set_err(h, SROM_ERR_INVALID, "bad tuning request");
    DeviceGuard g(h->device);
    cudaDeviceProp prop;
    SROM_CUDA(h, cudaGetDeviceProperties(&prop, h->device));
    // 1) cached choices for this device
    if (cache_path) {
        if (FILE *fp = fopen(cache_path, "r")) {
            char line[512], dev[256] = {0};
            bool same_dev = false;
            while (fgets(line, sizeof line, fp)) {
                if (sscanf(line, " \"device\": \"%255[^\"]\"", dev) == 1) same_dev = strcmp(dev, prop.name) == 0;
                int n = 0, rr = 0;
                char kern[32] = {0};
                if (same_dev && sscanf(line, " {\"precision\": \"fp64\", \"n\": %d, \"r\": %d, \"kernel\": \"%31[^\"]\"",
                                       &n, &rr, kern) == 3)
                    h->tune_fp64[((long long)n << 16) | rr] = strcmp(kern, "smem") == 0 ? 0 : 1;
                if (same_dev && sscanf(line, " {\"precision\": \"mixed\", \"n\": %d, \"r\": %d, \"kernel\": \"%31[^\"]\"",
                                       &n, &rr, kern) == 3)
                    h->tune_mixed[((long long)n << 16) | rr] = strcmp(kern, "fp64_smem") == 0 ? 0 : 1;
                if (same_dev && sscanf(line, " {\"precision\": \"auto\", \"n\": %d, \"r\": %d, \"kernel\": \"%31[^\"]\"",
                                       &n, &rr, kern) == 3)
                    h->tune_tc[((long long)n << 16) | rr] = strcmp(kern, "tensor_core") == 0 ? 1 : 0;
            }
            fclose(fp);
        }
    }
    // 2) time both storage classes for every requested n that has no entry yet
    struct Entry {
        int n, r, cls;
        float ms[2];
        int mcls;      // mixed routing (-1: not measured)
        float mms[2];  // mixed sweep: FP64 outright, mixed global kernel
        int tcls;      // SROM_MIXED_AUTO's kernel (-1: not measured)
        float tms[2];  // mixed sweep on every system: CUDA-core kernel, tensor-core kernel
    };
    std::vector<Entry> measured;
    for (int q = 0; q < count; ++q) {
        const int n = n_values[q];
        if (n <= 0) continue;
        const long long key = ((long long)n << 16) | r;
        // FP64: only a choice where the shared-memory kernel fits; the mixed kernels: orders
        // from 96 up to the tensor-core kernel's limit
        const bool need_fp64 = !h->tune_fp64.count(key) && srom::fp64_smem_bytes(n, r) <= (size_t)h->max_smem_optin;
        const bool need_tc = !h->tune_tc.count(key) && n >= 96 && n <= srom::TC_MAX_N && r <= srom::MIXED_MAX_R &&
                             srom::tc_supported(n, r, h->max_smem_optin, nullptr) &&
                             srom::global_panel_fits(n, r, h->max_smem_optin);
        if (!need_fp64 && !need_tc) continue;
        const int F = 2 * h->sm_count;
        std::vector<srom_complex> K((size_t)n * n), M((size_t)n * n), B((size_t)n * r);
        std::vector<double> om(F);
        uint64_t state = 0x9E3779B97F4A7C15ull ^ (uint64_t)n;
        auto rnd = [&]() {
            state ^= state << 13;
            state ^= state >> 7;
            state ^= state << 17;
            return (double)(state >> 11) * (1.0 / 9007199254740992.0) - 0.5;
        };
        for (int j = 0; j < n; ++j)
            for (int i = 0; i < n; ++i) {
                K[i + (size_t)j * n] = {rnd() + (i == j ? 2.0 * n : 0.0), rnd()};
                M[i + (size_t)j * n] = {i == j ? 1.0 : 0.0, 0.0};
            }
        for (auto &b : B) b = {rnd(), rnd()};
        for (int f = 0; f < F; ++f) om[f] = 0.1 + 0.01 * f;
        const size_t nn = sizeof(srom_complex) * (size_t)n * n;
        char *buf = nullptr;
        const size_t tot = 2 * nn + sizeof(srom_complex) * (size_t)n * r + sizeof(double) * F +
                           sizeof(srom_complex) * (size_t)F * n * r;
        cudaError_t e = cudaMalloc(&buf, tot);
        if (e != cudaSuccess) return set_err(h, SROM_ERR_ALLOC, "tuning buffers: %s", cudaGetErrorString(e));
        srom_rom_desc d{};
        d.n = n;
        d.r = r;
        d.F = F;
        d.ldk = n;
        d.ldb = n;
        d.K = reinterpret_cast<srom_complex *>(buf);
        d.M = reinterpret_cast<srom_complex *>(buf + nn);
        d.rhs = reinterpret_cast<srom_complex *>(buf + 2 * nn);
        d.omega = reinterpret_cast<double *>(buf + 2 * nn + sizeof(srom_complex) * (size_t)n * r);
        d.X = reinterpret_cast<srom_complex *>(buf + 2 * nn + sizeof(srom_complex) * (size_t)n * r + sizeof(double) * F);
        int rc = SROM_OK;
        const void *src[4] = {K.data(), M.data(), B.data(), om.data()};
        void *dst[4] = {(void *)d.K, (void *)d.M, (void *)d.rhs, (void *)d.omega};
        const size_t bytes[4] = {nn, nn, sizeof(srom_complex) * (size_t)n * r, sizeof(double) * F};
        for (int k = 0; k < 4 && rc == SROM_OK; ++k)
            if ((e = cudaMemcpy(dst[k], src[k], bytes[k], cudaMemcpyHostToDevice)) != cudaSuccess)
                rc = set_err(h, SROM_ERR_CUDA, "tuning input copy: %s", cudaGetErrorString(e));
        Entry ent{n, r, -1, {0.f, 0.f}, -1, {0.f, 0.f}, -1, {0.f, 0.f}};
        cudaEvent_t a = nullptr, b = nullptr;
        if (rc == SROM_OK && ((e = cudaEventCreate(&a)) != cudaSuccess || (e = cudaEventCreate(&b)) != cudaSuccess))
            rc = set_err(h, SROM_ERR_CUDA, "tuning events: %s", cudaGetErrorString(e));
        // one warm-up sweep, then three timed ones
        auto time_sweep = [&](const srom_sweep_opts &o, float *ms) {
            int q = srom_sweep(h, &d, 1, &o);
            if (q == SROM_OK && (e = cudaEventRecord(a, h->stream)) != cudaSuccess)
                q = set_err(h, SROM_ERR_CUDA, "tuning timer: %s", cudaGetErrorString(e));
            for (int rep = 0; rep < 3 && q == SROM_OK; ++rep) q = srom_sweep(h, &d, 1, &o);
            if (q == SROM_OK && ((e = cudaEventRecord(b, h->stream)) != cudaSuccess ||
                                 (e = cudaEventSynchronize(b)) != cudaSuccess ||
                                 (e = cudaEventElapsedTime(ms, a, b)) != cudaSuccess))
                q = set_err(h, SROM_ERR_CUDA, "tuning timer: %s", cudaGetErrorString(e));
            return q;
        };
        const srom_sweep_opts o64{SROM_FP64, 5, 0.0, 0};
        for (int c = 0; c < 2 && rc == SROM_OK && need_fp64; ++c) {
            h->tune_fp64[key] = c;
            rc = time_sweep(o64, &ent.ms[c]);
        }
        if (rc == SROM_OK && need_fp64) {
            ent.cls = ent.ms[1] < ent.ms[0] ? 1 : 0;
            h->tune_fp64[key] = ent.cls;
        }
        // SROM_MIXED_AUTO's kernel: every system on the CUDA-core, then on the tensor-core kernel
        if (rc == SROM_OK && need_tc) {
            const int fl = SROM_FLAG_FALLBACK_FP64 | SROM_FLAG_MIXED_EVERY;
            const srom_sweep_opts occ{SROM_MIXED_FP32, 5, 0.0, fl}, otc{SROM_MIXED_TC, 5, 0.0, fl};
            rc = time_sweep(occ, &ent.tms[0]);
            if (rc == SROM_OK) rc = time_sweep(otc, &ent.tms[1]);
            if (rc == SROM_OK) {
                ent.tcls = ent.tms[1] < ent.tms[0] ? 1 : 0;
                h->tune_tc[key] = ent.tcls;
            }
        }
        // the mixed form's routing of such a system: the FP64 shared-memory kernel outright, or
        // complex-FP32 factors in the mixed global kernel plus refinement (only a choice when the
        // FP64 choice is the shared-memory kernel)
        if (rc == SROM_OK && need_fp64 && ent.cls == 0 && r <= srom::MIXED_MAX_R) {
            const srom_sweep_opts om{SROM_MIXED_FP32, 5, 0.0, SROM_FLAG_FALLBACK_FP64};
            for (int c = 0; c < 2 && rc == SROM_OK; ++c) {
                h->tune_mixed[key] = c;
                rc = time_sweep(om, &ent.mms[c]);
            }
            if (rc == SROM_OK) {
                ent.mcls = ent.mms[1] < ent.mms[0] ? 1 : 0;
                h->tune_mixed[key] = ent.mcls;
            }
        }
        if (a) cudaEventDestroy(a);
        if (b) cudaEventDestroy(b);
        cudaStreamSynchronize(h->stream);
        cudaFree(buf);
        if (rc != SROM_OK) {
            if (need_fp64) {
                h->tune_fp64.erase(key);
                h->tune_mixed.erase(key);
            }
            if (need_tc) h->tune_tc.erase(key);
            return rc;
        }
        measured.push_back(ent);
    }
    // 3) rewrite the cache with every entry the handle knows
    if (cache_path && !measured.empty()) {
        FILE *fp = fopen(cache_path, "w");
        if (!fp) return set_err(h, SROM_ERR_INVALID, "cannot write %s", cache_path);
        fprintf(fp, "{\n  \"device\": \"%s\",\n  \"entries\": [\n", prop.name);
        const size_t total = h->tune_fp64.size() + h->tune_mixed.size() + h->tune_tc.size();
        size_t k = 0;
        for (const auto &kv : h->tune_fp64) {
            const int n = (int)(kv.first >> 16), rr = (int)(kv.first & 0xffff);
            float ms0 = -1.f, ms1 = -1.f;
            for (const auto &m : measured)
                if (m.n == n && m.r == rr && m.cls >= 0) {
                    ms0 = m.ms[0];
                    ms1 = m.ms[1];
                }
            fprintf(fp, "    {\"precision\": \"fp64\", \"n\": %d, \"r\": %d, \"kernel\": \"%s\", \"ms_smem\": %.4f, \"ms_global\": %.4f}%s\n",
                    n, rr, kv.second == 0 ? "smem" : "global", ms0, ms1, ++k < total ? "," : "");
        }
        for (const auto &kv : h->tune_mixed) {
            const int n = (int)(kv.first >> 16), rr = (int)(kv.first & 0xffff);
            float ms0 = -1.f, ms1 = -1.f;
            for (const auto &m : measured)
                if (m.n == n && m.r == rr && m.mcls >= 0) {
                    ms0 = m.mms[0];
                    ms1 = m.mms[1];
                }
            fprintf(fp, "    {\"precision\": \"mixed\", \"n\": %d, \"r\": %d, \"kernel\": \"%s\", \"ms_fp64_smem\": %.4f, \"ms_mixed_global\": %.4f}%s\n",
                    n, rr, kv.second == 0 ? "fp64_smem" : "mixed_global", ms0, ms1, ++k < total ? "," : "");
        }
        for (const auto &kv : h->tune_tc) {
            const int n = (int)(kv.first >> 16), rr = (int)(kv.first & 0xffff);
            float ms0 = -1.f, ms1 = -1.f;
            for (const auto &m : measured)
                if (m.n == n && m.r == rr && m.tcls >= 0) {
                    ms0 = m.tms[0];
                    ms1 = m.tms[1];
                }
            fprintf(fp, "    {\"precision\": \"auto\", \"n\": %d, \"r\": %d, \"kernel\": \"%s\", \"ms_cuda_core\": %.4f, \"ms_tensor_core\": %.4f}%s\n",
                    n, rr, kv.second ? "tensor_core" : "cuda_core", ms0, ms1, ++k < total ? "," : "");
        }
        fprintf(fp, "  ]\n}\n");
        fclose(fp);
    }
    return SROM_OK;
}

}  // extern "C"
