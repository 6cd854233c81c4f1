// FP64 frequency sweep that allocates no device memory (srom_sweep_fp64_noalloc).
//
// Who needs it: a host program that owns all device memory through its own pool and does
// not let a library call cudaMalloc -- a solver framework that hands plugins fixed device
// buffers, or a real-time loop in which cudaMalloc's implicit device synchronisation and
// its possible failure at run time are not acceptable.  srom_sweep needs a handle, whose
// creation and first calls allocate descriptor staging and one scratch matrix per resident
// CTA; this entry point instead takes one ROM descriptor, uses the scratch array below, and
// runs the same global-storage FP64 kernel (bit-identical results).
//
// The scratch array lives for as long as the library is loaded, on every device that loads
// it.  Every call uses the same array: its contents are whatever the last call left, so the
// work counter is cleared on every call, and two calls whose work overlaps on the GPU (for
// example on two streams) race on it and must be serialised by the caller.
#include <algorithm>
#include <cstdio>
#include <mutex>

#include "../../include/staccato_rom.h"
#include "srom_device.cuh"
#include "sweep_kernels.h"

namespace {

constexpr int NOALLOC_MAX_N = 512;
constexpr int NOALLOC_MAX_F = 65536;
constexpr size_t NOALLOC_HDR_BYTES = 512;  // RomDev at 0, work counter at 256
constexpr size_t NOALLOC_ITEM_BYTES = sizeof(srom::Item) * (size_t)NOALLOC_MAX_F;
constexpr size_t NOALLOC_SLOT_BYTES = size_t(32) << 20;  // matrices of in-flight systems
constexpr size_t NOALLOC_BYTES = NOALLOC_HDR_BYTES + NOALLOC_ITEM_BYTES + NOALLOC_SLOT_BYTES;
constexpr int NOALLOC_MAX_DEVICES = 64;

static_assert(sizeof(srom::RomDev) <= 256, "descriptor must fit its header slot");
static_assert((NOALLOC_HDR_BYTES + NOALLOC_ITEM_BYTES) % 256 == 0, "slots must stay 256-byte aligned");

}  // namespace

// 33 MB: descriptor, work counter, work list (65536 frequencies) and 32 MiB of matrix slots.
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_BYTES];

namespace {

std::mutex g_noalloc_mu;
void *g_noalloc_ptr[NOALLOC_MAX_DEVICES] = {};

// Device address of g_noalloc_scratch on the current device, looked up on the first call per
// device and cached.  A cached address that the runtime no longer knows as device memory of this
// device (the context was reset with cudaDeviceReset and the module loaded again) is looked up
// anew.
cudaError_t noalloc_scratch(int dev, unsigned char **out) {
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (g_noalloc_ptr[dev]) {
        cudaPointerAttributes a{};
        const cudaError_t e = cudaPointerGetAttributes(&a, g_noalloc_ptr[dev]);
        if (e != cudaSuccess || a.type != cudaMemoryTypeDevice || a.device != dev) {
            cudaGetLastError();
            g_noalloc_ptr[dev] = nullptr;
        }
    }
    if (!g_noalloc_ptr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_noalloc_ptr[dev] = p;
    }
    *out = static_cast<unsigned char *>(g_noalloc_ptr[dev]);
    return cudaSuccess;
}

__global__ void noalloc_prepare(srom::RomDev R, unsigned char *base) {
    srom::RomDev *rd = reinterpret_cast<srom::RomDev *>(base);
    int *ctr = reinterpret_cast<int *>(base + 256);
    srom::Item *items = reinterpret_cast<srom::Item *>(base + NOALLOC_HDR_BYTES);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        *rd = R;
        *ctr = 0;
    }
    for (int f = blockIdx.x * blockDim.x + threadIdx.x; f < R.F; f += gridDim.x * blockDim.x)
        items[f] = srom::Item{0, f};
}

int fail(char *err, int len, int code, const char *msg, const char *detail = nullptr) {
    if (err && len > 0) snprintf(err, (size_t)len, "%s%s%s", msg, detail ? ": " : "", detail ? detail : "");
    return code;
}

}  // namespace

extern "C" int srom_sweep_fp64_noalloc(const srom_rom_desc *d, void *cuda_stream, char *err, int err_len) {
    if (err && err_len > 0) err[0] = 0;
    if (!d) return fail(err, err_len, SROM_ERR_INVALID, "descriptor is null");
    if (d->n < 0 || d->r < 0 || d->F < 0) return fail(err, err_len, SROM_ERR_INVALID, "negative size");
    if (d->n == 0 || d->r == 0 || d->F == 0) return SROM_OK;
    if (!d->K || !d->M || !d->rhs || !d->omega || !d->X)
        return fail(err, err_len, SROM_ERR_INVALID, "K, M, rhs, omega and X must be non-null (M = NULL needs srom_sweep)");
    if (d->ldk < d->n || d->ldb < d->n) return fail(err, err_len, SROM_ERR_INVALID, "ldk and ldb must be >= n");
    if ((d->LU == nullptr) != (d->ipiv == nullptr))
        return fail(err, err_len, SROM_ERR_INVALID, "LU and ipiv must be given together");
    if (d->n_out < 0 || (d->n_out > 0 && (!d->C || !d->Y || d->ldc < d->n_out)))
        return fail(err, err_len, SROM_ERR_INVALID, "n_out > 0 needs C, Y and ldc >= n_out");
    {
        const void *cz[] = {d->K, d->M, d->D, d->rhs, d->X, d->LU, d->C, d->Y};
        bool bad = srom::misaligned(d->omega, 8) || srom::misaligned(d->berr, 8) || srom::misaligned(d->info, 4) ||
                   srom::misaligned(d->steps, 4) || srom::misaligned(d->ipiv, 4);
        for (const void *p : cz) bad = bad || srom::misaligned(p, 16);
        if (bad)
            return fail(err, err_len, SROM_ERR_INVALID,
                        "complex arrays must be 16-byte aligned (omega/berr 8, info/steps/ipiv 4)");
    }
    if (d->n > NOALLOC_MAX_N) {
        char b[96];
        snprintf(b, sizeof b, "n = %d exceeds the limit of %d", d->n, NOALLOC_MAX_N);
        return fail(err, err_len, SROM_ERR_UNSUPPORTED, "srom_sweep_fp64_noalloc", b);
    }
    if (d->F > NOALLOC_MAX_F) {
        char b[96];
        snprintf(b, sizeof b, "F = %d exceeds the limit of %d frequencies", d->F, NOALLOC_MAX_F);
        return fail(err, err_len, SROM_ERR_UNSUPPORTED, "srom_sweep_fp64_noalloc", b);
    }
    int dev = 0, sms = 0, smem_optin = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(err, err_len, SROM_ERR_CUDA, "cudaGetDevice", cudaGetErrorString(e));
    if (dev >= NOALLOC_MAX_DEVICES) return fail(err, err_len, SROM_ERR_UNSUPPORTED, "device index above 63");
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess ||
        (e = cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev)) != cudaSuccess)
        return fail(err, err_len, SROM_ERR_CUDA, "cudaDeviceGetAttribute", cudaGetErrorString(e));
    // the launch's own test (make_plan): rows per thread, and dynamic plus static shared memory
    if (srom::global_rpt(d->n) > srom::GLOBAL_MAX_RPT ||
        srom::fp64_global_smem_bytes(d->n, d->r) + srom::GLOBAL_STATIC_SMEM > (size_t)smem_optin) {
        char b[96];
        snprintf(b, sizeof b, "n = %d with r = %d needs more shared memory than a CTA has", d->n, d->r);
        return fail(err, err_len, SROM_ERR_UNSUPPORTED, "srom_sweep_fp64_noalloc", b);
    }
    unsigned char *base = nullptr;
    if ((e = noalloc_scratch(dev, &base)) != cudaSuccess)
        return fail(err, err_len, SROM_ERR_CUDA, "cudaGetSymbolAddress", cudaGetErrorString(e));

    srom::RomDev R;
    R.n = d->n;
    R.r = d->r;
    R.F = d->F;
    R.ldk = d->ldk;
    R.K = reinterpret_cast<const double2 *>(d->K);
    R.M = reinterpret_cast<const double2 *>(d->M);
    R.D = reinterpret_cast<const double2 *>(d->D);
    R.eta = d->eta;
    R.rhs = reinterpret_cast<const double2 *>(d->rhs);
    R.ldb = d->ldb;
    R.omega = d->omega;
    R.X = reinterpret_cast<double2 *>(d->X);
    R.info = d->info;
    R.steps = d->steps;
    R.berr = d->berr;
    R.LU = reinterpret_cast<double2 *>(d->LU);
    R.ipiv = d->ipiv;

    cudaStream_t st = reinterpret_cast<cudaStream_t>(cuda_stream);
    noalloc_prepare<<<(d->F + 255) / 256, 256, 0, st>>>(R, base);
    if ((e = cudaGetLastError()) != cudaSuccess)
        return fail(err, err_len, SROM_ERR_CUDA, "prepare launch", cudaGetErrorString(e));
    const int64_t slot = (int64_t)d->n * d->n;
    const long long slots = (long long)(NOALLOC_SLOT_BYTES / (sizeof(double2) * (size_t)slot));
    long long grid = std::min<long long>(std::min<long long>(d->F, sms), slots);
    auto *roms = reinterpret_cast<const srom::RomDev *>(base);
    auto *items = reinterpret_cast<const srom::Item *>(base + NOALLOC_HDR_BYTES);
    int *ctr = reinterpret_cast<int *>(base + 256);
    auto *slot_base = reinterpret_cast<double2 *>(base + NOALLOC_HDR_BYTES + NOALLOC_ITEM_BYTES);
    e = srom::launch_fp64_global(roms, items, d->F, ctr, slot_base, slot, d->n, d->r, (int)grid, st);
    if (e != cudaSuccess) return fail(err, err_len, SROM_ERR_CUDA, "sweep launch", cudaGetErrorString(e));
    if (d->n_out > 0) {
        srom::BackProj b{d->n, d->r, d->F, d->n_out, d->ldc, reinterpret_cast<const double2 *>(d->C),
                         reinterpret_cast<const double2 *>(d->X), reinterpret_cast<double2 *>(d->Y)};
        e = srom::launch_backproject(b, sms, st);
        if (e != cudaSuccess) return fail(err, err_len, SROM_ERR_CUDA, "back-projection launch", cudaGetErrorString(e));
    }
    return SROM_OK;
}
