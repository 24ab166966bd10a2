// bldm_solve_device_noalloc: the device-buffer solve without any device
// allocation.
//
// Some callers cannot allocate device memory when they solve:
//  * cudaMalloc and cudaFree can synchronise the whole device, which a
//    latency-bound caller (a serving loop sharing the GPU with other streams)
//    cannot afford on its hot path;
//  * in processes whose device memory is owned by another allocator (a
//    framework's caching allocator, or a server that reserves HBM up front), a
//    raw cudaMalloc can fail with out-of-memory even though the caller's own
//    pool has room;
//  * callers that must not fail half-way through a run on out-of-memory.
// This entry point takes the solver's scratch (the partial axis sums and the
// digamma tables of the fused sweep) from a fixed array in the library's
// device data, so the only device memory it touches is the caller's X, alpha,
// beta and S and that array.
//
// The array is kNoAllocScratchBytes (32 MiB) per GPU and stays allocated on
// every GPU where the library's device code is loaded until the process exits.
// Shapes whose scratch does not fit are rejected with BLDM_ERR_TOO_LARGE (for
// example 1024x1024x64 in FP64 needs 22.5 MB and fits).  All calls on a device
// share the one array: calls that overlap on the GPU (different streams or
// host threads at the same time) race and corrupt each other's results.
#include <mutex>

#include "bldm_internal.h"

using namespace bldm;

namespace {

constexpr size_t kNoAllocScratchBytes = size_t(32) << 20;

// The solver scratch.  In host code this name is only a stand-in for the
// device symbol; its device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void* g_scratch_dev_ptr[kMaxDevices] = {};

// Device address of the scratch array on the current device, looked up on the
// first call on that device and kept for the later ones.  A device reset (or
// anything else that unloads this library's device code from the device)
// invalidates the kept address; the public header tells callers not to use the
// entry point on such a device again.
int scratch_on_current_device(void** out) {
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return cuda_status(e);
    if (device < 0 || device >= kMaxDevices) return BLDM_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_dev_ptr[device]) {
        void* ptr = nullptr;
        e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_status(e);
        g_scratch_dev_ptr[device] = ptr;
    }
    *out = g_scratch_dev_ptr[device];
    return BLDM_OK;
}

}  // namespace

extern "C" int bldm_solve_device_noalloc(const void* d_X, const double* d_alpha,
                                         const double* d_beta, void* d_S, size_t x, size_t y,
                                         size_t z, int dtype, size_t max_iter, int psi_mode,
                                         double eps, void* stream) {
    if (!d_X || !d_alpha || !d_beta || !d_S) return BLDM_ERR_BAD_ARG;
    if (x == 0 || y == 0 || z == 0) return BLDM_ERR_BAD_ARG;
    if (psi_mode < BLDM_PSI_EXACT || psi_mode > BLDM_PSI_LEGACY_CUDA) return BLDM_ERR_BAD_ARG;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    void* scratch = nullptr;
    int rc = scratch_on_current_device(&scratch);
    if (rc) return rc;
    PlanImpl p;  // views into the scratch array; owns nothing
    size_t needed = 0;
    rc = plan_setup_in(&p, x, y, z, dtype, scratch, kNoAllocScratchBytes, &needed, st);
    if (rc) return rc;
    rc = plan_run(&p, d_X, d_alpha, d_beta, d_S, max_iter, psi_mode, eps, st, nullptr, 0);
    if (rc) return rc;
    return plan_check(&p, st);
}
