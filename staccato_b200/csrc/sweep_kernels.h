// Host-side entry points of the sweep kernels (used by the C ABI in capi.cu).
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace srom {

struct RomDev;
struct Item;

// The kernels read and write complex values as 16-byte vectors (double2), doubles as 8 bytes
// and ints as 4; srom_complex itself only promises 8-byte alignment, so device pointers are
// checked on the host before any launch (a misaligned vector access would fault the kernel).
inline bool misaligned(const void *p, size_t a) { return p && (reinterpret_cast<uintptr_t>(p) % a) != 0; }

// ---- FP64 (bit-identical to the restated zgetrf/zgetrs) ----
size_t fp64_smem_bytes(int n, int r);
size_t fp64_global_smem_bytes(int n_max, int r_max);
int fp64_smem_blocks_per_sm(size_t smem);
cudaError_t launch_fp64_smem(const RomDev *roms, const Item *items, int n_items, int *counter,
                             size_t smem, int grid, cudaStream_t st);
// dynamic shared memory of the global kernels; big: the large-order FP64 instances
size_t global_smem_bytes(int n_max, int r_max, bool big = false);
// the shared-memory-panel instances (launch_global) can run (n_max, r_max)
bool global_panel_fits(int n_max, int r_max, int smem_optin);
int global_rpt(int n_max);
constexpr int GLOBAL_MAX_RPT = 3;   // rows per thread of the shared-memory-panel instances
constexpr int BIG_RPT = 10;         // the largest large-order FP64 instance: n <= NT * BIG_RPT = 2560
constexpr int BIG_MAX_N = 256 * BIG_RPT;
// large-order FP64 instance: global scratch per CTA (the matrix, then the 16-column panel)
int64_t big_panel_offset(int n_max);
int64_t big_slot_bytes(int n_max);
constexpr int MIXED_MAX_R = 16;
constexpr size_t GLOBAL_STATIC_SMEM = 4096;
// Arguments of the global-storage kernels.
struct GlobalArgs {
    const RomDev *roms;
    const Item *items;
    int n_items;
    const int *n_items_dev;  // when non-null, the item count is read from device memory
    int *counter;            // work counter (zero before the launch)
    unsigned char *scratch;  // one slot of slot_bytes per CTA
    int64_t slot_bytes;
    int ldp, n_max, r_max;
    int max_refine;
    double tol;
    Item *fb_items;  // mixed: non-converged systems are appended here (null: keep the last iterate)
    int *fb_count;
    int steps_value;  // FP64: value stored in steps (0; -1 when re-solving mixed fallbacks)
    int smem_dyn;     // dynamic shared memory of the launch (set by launch_global)
    int *err_flag;    // tensor-core kernel: set to 1 when a bounded device-side wait ran out
    int64_t panel_off;  // large-order FP64 instances: offset of the panel in a slot (set by launch_global_big)
};
// Global-storage kernel, FP64 (mixed = false) or complex-FP32 factors + FP64 refinement.
cudaError_t launch_global(bool mixed, const GlobalArgs &a, int grid, cudaStream_t st);
// FP64 sweep of orders up to BIG_MAX_N with the panel in global scratch (slot_bytes >=
// big_slot_bytes(n_max)); 3, 6 or 10 rows per thread by n_max
cudaError_t launch_global_big(const GlobalArgs &a, int grid, cudaStream_t st);
cudaError_t launch_fp64_global(const RomDev *roms, const Item *items, int n_items, int *counter,
                               double2 *scratch, int64_t slot_elems, int n_max, int r_max,
                               int grid, cudaStream_t st);

// ---- tensor-core mixed form (sweep_tc.cu): complex-FP32 LU whose Schur updates run as
// tcgen05 MMAs on three-piece bf16 splits, FP64 refinement as in the global kernel ----
constexpr int TC_MAX_N = 512;
size_t tc_slot_bytes(int n_max);                 // global scratch per CTA
size_t tc_smem_bytes(int n_max, int r_max);      // dynamic shared memory of the launch
// Whether the kernel handles systems up to n_max with r_max right-hand sides; why (may be
// null) receives the reason when it does not.
bool tc_supported(int n_max, int r_max, int smem_optin, const char **why);
// a.slot_bytes must be at least tc_slot_bytes(a.n_max); a.fb_items / a.err_flag as for the
// mixed global kernel.
cudaError_t launch_tc(const GlobalArgs &a, int grid, cudaStream_t st);

// Back-projection Y_f = C X_f of one ROM's solutions (F blocks of n x r -> n_out x r).
struct BackProj {
    int n, r, F, n_out, ldc;
    const double2 *C;
    const double2 *X;
    double2 *Y;
};
cudaError_t launch_backproject(const BackProj &p, int sms, cudaStream_t st);

}  // namespace srom
