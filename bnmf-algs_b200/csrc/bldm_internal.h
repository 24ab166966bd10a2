// Host-side internals shared by the translation units of libbldm.so.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/bldm.h"

namespace bldm {

// Launch configuration of the fused sweep for one shape.
//
// The (i, j) plane of S is cut into CTA regions: a band of `band_w`
// consecutive columns j (contiguous fibers of one row, so one bulk copy per
// row) times a range of rows.  Region (band, rr) writes one row of S_pjk
// partials [rr][j in band][k] and, per row, one row of S_ipk partials
// [band][i][k]; the finalize kernel sums them in a fixed order.
struct SweepCfg {
    int vec;        // elements per lane access (16 / sizeof(T) when aligned)
    int lpf;        // lanes per fiber
    int mch;        // chunks (of vec elements) per lane
    int cpw;        // fiber passes per warp per row
    int warps;      // warps per CTA
    int wpr;        // warps per row (8 / wpr rows share a stage)
    int band_w;     // columns per band
    int n_bands;
    int n_rr;       // row ranges
    int rr_base, rr_extra;
    int stages;     // bulk-copy pipeline depth
    int ctas_per_sm;  // resident sweep CTAs per SM (shared-memory bound)
    uint32_t stage_bytes;
    size_t smem_update, smem_sums;
    int n_ablk, rows_per_ablk;  // finalize: row blocks for alpha_eph
    int fin_threads;
    // Long fibers (z beyond the lane layout): the two-pass kernels of
    // bldm_long.cu over n_kc k-chunks x n_bands bands of kLongBand columns x
    // n_rr row ranges; vec/lpf/mch/stages are unused.
    bool long_mode = false;
    int n_kc = 0;
};

// Byte offsets of the pieces of a plan's workspace (one block of device
// memory, 256-byte aligned pieces).
struct WorkspaceLayout {
    size_t o_pjk = 0, o_ipk = 0, o_psiB = 0, o_psiA = 0, o_psiAS = 0, o_asum = 0;
    size_t o_words = 0;  // finalize counter (+0), error word (+16), conservation (+32)
    size_t o_nzr = 0, o_nzc = 0;
    size_t o_fsum = 0;   // long fibers: per-fiber sums [x*y] double4
    size_t bytes = 0;
};
constexpr size_t kWorkspaceWords = 64;

struct PlanImpl {
    int device = 0;
    int dtype = BLDM_F64;
    size_t x = 0, y = 0, z = 0;
    size_t esize = 8;
    SweepCfg cfg{};
    // Workspace: one allocation carved into the pieces below.
    void* ws = nullptr;
    size_t ws_bytes = 0;
    bool owns_ws = false;         // allocated by plan_setup (plan_free releases it)
    WorkspaceLayout layout{};
    double* part_pjk = nullptr;   // [n_rr][y][z]
    double* part_ipk = nullptr;   // [n_bands][x][z]
    void* psiB = nullptr;         // [y][z]  T
    void* psiA = nullptr;         // [x][z]  T
    void* psiAS = nullptr;        // [z]     T
    double* asum_part = nullptr;  // [n_ablk][z]
    unsigned* counter = nullptr;  // finalize last-block counter
    int* err = nullptr;           // device error word
    unsigned long long* cons = nullptr;  // conservation residual (bits of a double >= 0)
    bool skip_zero = false;       // bldm_tuning::skip_zero_rows
    int* nz_rows = nullptr;       // [n_bands][x] rows with X != 0 per band (skip_zero)
    int* nz_cnt = nullptr;        // [n_bands][x + 1] running counts (skip_zero)
    void* fsum = nullptr;         // [x*y] double4 fiber sums (long fibers)
    uint64_t launches = 0;
};

// Implemented in bldm_sweep.cu.
int plan_setup(PlanImpl* p, size_t x, size_t y, size_t z, int dtype,
               const bldm_tuning* tune = nullptr);
void plan_free(PlanImpl* p);
int plan_run(PlanImpl* p, const void* dX, const double* dalpha, const double* dbeta,
             void* dS, size_t max_iter, int psi_mode, double eps, cudaStream_t st,
             cudaEvent_t* kernel_events, size_t n_kernel_events);
int plan_init_S(PlanImpl* p, const void* dX, void* dS, uint64_t seed, cudaStream_t st);
int plan_sums(PlanImpl* p, const void* dS, cudaStream_t st);
int plan_shard_step(PlanImpl* p, const void* dX, void* dS, const double* dalpha, double* d_red,
                    bool update, int psi_mode, double eps, cudaStream_t st);
int plan_shard_finish(PlanImpl* p, const double* dbeta, const double* d_red, int psi_mode,
                      cudaStream_t st);
int plan_check(PlanImpl* p, cudaStream_t st);
int plan_conservation_launch(PlanImpl* p, const void* dX, const void* dS, cudaStream_t st);
int plan_setup_in(PlanImpl* p, size_t x, size_t y, size_t z, int dtype, void* ws,
                  size_t ws_cap, size_t* ws_needed, cudaStream_t st);

int cuda_status(cudaError_t e);
int lane_config(size_t z, size_t es, SweepCfg& c);
int ensure_smem_attr(void* fn, size_t bytes);

}  // namespace bldm
