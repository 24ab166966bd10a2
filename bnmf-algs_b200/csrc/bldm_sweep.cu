// Fused multiplicative-update sweep over the allocation tensor S.
//
// One iteration of the reference (src/bld/bld_mult/bld_mult.hpp:123-147;
// stage formulas in bld_mult_funcs.hpp:130-327) is two launches here:
//
//   sweep<UPDATE>  reads every fiber S(i,j,:) once from HBM (bulk copies of a
//                  row segment into a shared-memory ring), computes
//                  S_ijp = sum_k S, psi(S+1), grad_plus, nom and denom in
//                  registers with lane-group shuffles, applies update_S, writes
//                  the fiber once, and accumulates the NEW tensor's axis sums
//                  S_pjk (over the CTA's rows) and S_ipk (over the CTA's band
//                  of columns) as deterministic per-region partials;
//   finalize       sums the partials in a fixed order, forms beta_eph and
//                  alpha_eph, and tabulates psi(beta_eph) (y*z), psi(alpha_eph)
//                  (x*z) and psi(sum_i alpha_eph) (z) for the next sweep, which
//                  rebuilds grad_minus(i,k) = psi(sum) - psi(alpha_eph) per row.
//
// HBM traffic per iteration is one read and one write of S plus one read of X
// and the small partial/table arrays, against eleven S-sized passes in the
// reference GPU path (tensor_sums 3, grad_plus 2, denom 2, nom 1, update_S 3).
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>

#include "bldm_device.cuh"
#include "bldm_internal.h"
#include "bldm_finalize.cuh"
#include "bldm_kernels.h"

namespace bldm {

template <typename T>
__global__ void __launch_bounds__(kFinThreads) finalize_kernel(const FinParams<T> p) {
    grid_dep_wait();  // the sweep's partials
    grid_dep_launch();
    __shared__ double acc[kFinAccDoubles];
    finalize_block<T, 16>(p.f, int(blockIdx.x), p.plus_appr, p.minus_appr, acc);
}

// Row-sharded solves: the digamma tables of the shared sums once every shard's
// red has been summed over the shards (red = [S_+jk (y*z) | sum alpha_eph (z)]).
template <typename T>
__global__ void __launch_bounds__(kFinThreads)
    shard_finish_kernel(const double* red, const double* beta, long long y, long long z,
                        T* psiB, T* psiAS, int plus_appr, int minus_appr) {
    const long long idx = (long long)blockIdx.x * kFinThreads + threadIdx.x;
    if (idx < y * z) psiB[idx] = T(psi_mode_f64(red[idx] + beta[idx % z], plus_appr != 0));
    if (idx < z) psiAS[idx] = T(psi_mode_f64(red[y * z + idx], minus_appr != 0));
}

void* pick_persist_f32_v4(int lpf, int mch, bool mr);
void* pick_persist_f32_v1(int lpf, int mch, bool mr);
void* pick_persist_f64_v2_appr(int lpf, int mch, bool mr);
void* pick_persist_f64_v2_exact(int lpf, int mch, bool mr);
void* pick_persist_f64_v1_appr(int lpf, int mch, bool mr);
void* pick_persist_f64_v1_exact(int lpf, int mch, bool mr);

void* pick_persist_fn(int dtype, int vec, int lpf, int mch, bool multirow, bool appr) {
    if (dtype == BLDM_F32) {
        if (vec == 4) return pick_persist_f32_v4(lpf, mch, multirow);
        if (vec == 1) return pick_persist_f32_v1(lpf, mch, multirow);
        return nullptr;
    }
    if (vec == 2)
        return appr ? pick_persist_f64_v2_appr(lpf, mch, multirow)
                    : pick_persist_f64_v2_exact(lpf, mch, multirow);
    if (vec == 1)
        return appr ? pick_persist_f64_v1_appr(lpf, mch, multirow)
                    : pick_persist_f64_v1_exact(lpf, mch, multirow);
    return nullptr;
}

// Five resident blocks per SM (48 registers, no spills): a batch's finalize is
// tens of thousands of short, latency-bound blocks, so occupancy sets its pace.
template <typename T>
__global__ void __launch_bounds__(kFinThreads, 5) finalize_batch_kernel(const BatchFinParams<T> p) {
    // instance owning this block: last i with block_off[i] <= blockIdx.x
    int lo = 0, hi = p.n_inst - 1;
    const int b = int(blockIdx.x);
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (p.block_off[mid] <= b) lo = mid;
        else hi = mid - 1;
    }
    const FinInst<T> f = p.insts[lo];
    __shared__ double acc[kFinAccDoubles];
    finalize_block<T, 8>(f, b - p.block_off[lo], p.plus_appr, p.minus_appr, acc);
}

void* finalize_batch_fn(int dtype) {
    return dtype == BLDM_F64 ? reinterpret_cast<void*>(&finalize_batch_kernel<double>)
                             : reinterpret_cast<void*>(&finalize_batch_kernel<float>);
}

// Seeded initial S: S(i,j,:) = X(i,j) * Dirichlet(1_z), the Dirichlet draw
// being normalised Exp(1) variates of a SplitMix64 counter hash.
__device__ __forceinline__ uint64_t splitmix64(uint64_t v) {
    v += 0x9E3779B97F4A7C15ull;
    v = (v ^ (v >> 30)) * 0xBF58476D1CE4E5B9ull;
    v = (v ^ (v >> 27)) * 0x94D049BB133111EBull;
    return v ^ (v >> 31);
}
__device__ __forceinline__ double exp1_variate(uint64_t hseed, uint64_t fiber, uint64_t k) {
    const uint64_t h = splitmix64(hseed ^ splitmix64(fiber * 0x100000001B3ull + k));
    const double u = (double(h >> 11) + 0.5) * (1.0 / 9007199254740992.0);
    return -log(u);
}

// Lane groups of lpf = min(32, pow2ceil(z)) lanes per fiber, 32 / lpf fibers
// per warp: lane q draws k = q, q + lpf, ...; the first four draws per lane stay
// in registers (each variate computed once for z <= 4 lpf; beyond that the rest
// are drawn again for the stores); the group adds the fiber's total by
// shuffles and the stores of consecutive lanes are consecutive elements.
template <typename T>
__global__ void init_S_kernel(const T* X, T* S, long long nf, long long z, uint64_t seed,
                              int lpf) {
    constexpr int R = 4;
    const long long gw = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const long long f = gw * (32 / lpf) + lane / lpf;
    const int q = lane % lpf;
    const bool on = f < nf;
    const uint64_t hs = splitmix64(seed ^ 0x5DEECE66Dull);
    double v[R];
    double tot = 0.0;
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const long long k = q + (long long)r * lpf;
        v[r] = (on && k < z) ? exp1_variate(hs, (uint64_t)f, (uint64_t)k) : 0.0;
        tot += v[r];
    }
    for (long long k = q + (long long)R * lpf; k < z; k += lpf)
        tot += on ? exp1_variate(hs, (uint64_t)f, (uint64_t)k) : 0.0;
    // every lane takes part in the shuffles; groups are lpf-aligned
    for (int o = 1; o < lpf; o <<= 1) tot += __shfl_xor_sync(0xffffffffu, tot, o);
    if (!on) return;
    const double xv = double(X[f]);
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const long long k = q + (long long)r * lpf;
        if (k < z) S[f * z + k] = T(xv * (v[r] / tot));
    }
    for (long long k = q + (long long)R * lpf; k < z; k += lpf)
        S[f * z + k] = T(xv * (exp1_variate(hs, (uint64_t)f, (uint64_t)k) / tot));
}

// ---------------------------------------------------------------------------
// Host side.
// ---------------------------------------------------------------------------
int cuda_status(cudaError_t e) {
    if (e == cudaSuccess) return BLDM_OK;
    if (e == cudaErrorMemoryAllocation) return BLDM_ERR_OOM;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return BLDM_ERR_NO_DEVICE;
    return BLDM_ERR_CUDA;
}

// The max-dynamic-shared-memory attribute belongs to the kernel function, not
// to a launch: plans and batches of different shapes share kernels, so the
// attribute only ever grows (a smaller value would break an earlier plan).
int ensure_smem_attr(void* fn, size_t bytes) {
    static std::mutex mu;
    static std::map<std::pair<int, void*>, size_t> set;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(mu);
    size_t& cur = set[std::make_pair(dev, fn)];
    if (bytes <= cur) return BLDM_OK;
    const cudaError_t e =
        cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes));
    if (e != cudaSuccess) return cuda_status(e);
    cur = bytes;
    return BLDM_OK;
}

#define BLDM_CU(call)                                   \
    do {                                                \
        cudaError_t e_ = (call);                        \
        if (e_ != cudaSuccess) return cuda_status(e_);  \
    } while (0)

template <typename T> using SweepFn = void (*)(const SweepParams<T>);
template <typename T> using BatchSweepFn = void (*)(const BatchSweepParams<T>);

// The sweep kernel for a lane shape: plain (one instance) or batch, one row
// or several rows per stage.  The instantiations live in bldm_pick_*.cu.
void* pick_sweep_fn(int dtype, int vec, int lpf, int mch, int mode, bool appr, bool batch,
                    bool multirow) {
    if (mode < SWEEP_SUMS || mode > SWEEP_COMPACT) return nullptr;
    if (dtype == BLDM_F64)
        return batch ? pick_sweep_f64_batch(vec, lpf, mch, mode, appr, multirow)
                     : pick_sweep_f64_plain(vec, lpf, mch, mode, appr, multirow);
    return batch ? pick_sweep_f32_batch(vec, lpf, mch, mode, multirow)
                 : pick_sweep_f32_plain(vec, lpf, mch, mode, multirow);
}

template <typename T> SweepFn<T> pick_sweep(const SweepCfg& c, int mode, bool appr) {
    return reinterpret_cast<SweepFn<T>>(pick_sweep_fn(sizeof(T) == 8 ? BLDM_F64 : BLDM_F32, c.vec,
                                                      c.lpf, c.mch, mode, appr, false,
                                                      c.wpr < kSweepWarps));
}

static int pow2ceil(long v) {
    int p = 1;
    while (p < v) p <<= 1;
    return p;
}
static size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

static int num_sms_of(int dev) {
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0)
        n = 148;
    return n;
}

// Lane shape for depth z: VEC elements per 16-byte access when the fiber is
// 16-byte aligned, LPF lanes per fiber, MCH chunks per lane, CPW passes.
int lane_config(size_t z, size_t es, SweepCfg& c) {
    const bool aligned = (z * es) % 16 == 0;
    c.vec = aligned ? int(16 / es) : 1;
    const long nch = long((z + c.vec - 1) / c.vec);
    if (nch <= 32) {
        c.lpf = pow2ceil(nch);
        c.mch = 1;
    } else {
        c.lpf = 32;
        c.mch = pow2ceil((nch + 31) / 32);
        if (c.mch > 8) return BLDM_ERR_UNSUPPORTED;
    }
    c.cpw = cpw_for(int(c.mch * c.vec * es));
    return BLDM_OK;
}

// Finalize row blocks: one row per thread (R rows of KT columns per block) up
// to ~256 blocks, so that a thread's sums of the band partials are not
// serialised over several rows.
static void finalize_blocks(SweepCfg& c, size_t x, size_t z) {
    const int KT = int(std::min<size_t>(z, kFinThreads));
    const int R = kFinThreads / KT;
    long rows = std::max<long>(R, long((x + 255) / 256));
    c.rows_per_ablk = int(rows);
    c.n_ablk = int((x + rows - 1) / rows);
    c.fin_threads = kFinThreads;
}

// Long fibers: tiles of (k-chunk, band of kLongBand columns, row range) for the
// two-pass kernels.  At least 32 rows per tile where x allows (each tile writes
// one S_+jk partial row per column, 1/rows of the S it sweeps) and about four
// waves of eight resident tiles per SM.
static int choose_long_cfg(SweepCfg& c, size_t x, size_t y, size_t z, int num_sms,
                           const bldm_tuning* tune) {
    if (tune && (tune->stages > 0 || tune->ctas_per_sm > 0)) return BLDM_ERR_UNSUPPORTED;
    c = SweepCfg{};
    c.long_mode = true;
    c.vec = 1;
    c.lpf = 32;
    c.warps = kSweepWarps;
    c.wpr = kSweepWarps;
    c.band_w = kLongBand;
    c.n_bands = int((y + kLongBand - 1) / kLongBand);
    c.n_kc = int((z + kLongThreads - 1) / kLongThreads);
    const long per_rr = long(c.n_kc) * c.n_bands;
    const long target = long(num_sms) * 8 * 4;
    long nrr = (target + per_rr - 1) / per_rr;
    nrr = std::min(nrr, std::max(1L, long(x / 32)));
    if (tune && tune->row_ranges > 0) nrr = tune->row_ranges;
    nrr = std::max(1L, std::min(long(x), nrr));
    c.n_rr = int(nrr);
    c.rr_base = int(x / nrr);
    c.rr_extra = int(x % nrr);
    finalize_blocks(c, x, z);
    return BLDM_OK;
}

static int choose_cfg(SweepCfg& c, size_t x, size_t y, size_t z, size_t es, int num_sms,
                      const bldm_tuning* tune) {
    if (lane_config(z, es, c) != BLDM_OK) return choose_long_cfg(c, x, y, z, num_sms, tune);
    c.long_mode = false;
    c.warps = kSweepWarps;
    const int fpw = 32 / c.lpf;
    // warps per row: as few as cover y, so that narrow rows share a stage
    c.wpr = kSweepWarps;
    while (c.wpr > 1 && size_t(c.wpr / 2) * c.cpw * fpw >= y) c.wpr /= 2;
    c.band_w = c.wpr * c.cpw * fpw;
    c.n_bands = int((y + c.band_w - 1) / c.band_w);
    const SlotLayout lay(c.band_w, (long long)z, int(es));
    c.stage_bytes = uint32_t(kSweepWarps / c.wpr) * (lay.capS + lay.capX + lay.capA);
    // each stage also owns a [warps][z] slice of S_ipk partials (FP64)
    const size_t per_stage = c.stage_bytes + size_t(kSweepWarps) * z * 8;
    const size_t fixed = 64 + z * es + 128;
    // Shared memory per SM is 228 KB; each CTA also holds 1 KB reserved and
    // the 2 KB static log table.  Registers (<= 128 per thread) allow at most
    // two 256-thread CTAs per SM.
    int cps = (tune && tune->ctas_per_sm > 0) ? tune->ctas_per_sm : 2;
    if (cps > 2) return BLDM_ERR_UNSUPPORTED;
    const size_t budget = (cps == 2 ? 110 : 220) * 1024;
    long st_max = budget > fixed ? long((budget - fixed) / per_stage) : 0;
    st_max = std::min(8L, st_max);
    // Default ring depth: about kRingBytes of copies per CTA (two CTAs per SM)
    // cover the memory latency; deeper rings add DRAM contention without
    // hiding more (1024x1024x64 update: 4 stages of 17 KB beat 5 in FP64 and
    // FP32, and all-zero X streams fastest at 2-3).
    constexpr long kRingBytes = 64 * 1024;
    long st = std::min(st_max, std::max(2L, long((kRingBytes + c.stage_bytes - 1) / c.stage_bytes)));
    if (st_max < 2) st = st_max;
    if (tune && tune->stages > 0) {
        if (tune->stages > st_max || tune->stages < 2) return BLDM_ERR_UNSUPPORTED;
        st = tune->stages;
    }
    if (st < 2) {
        if (tune && tune->ctas_per_sm == 2) return BLDM_ERR_UNSUPPORTED;
        // large slabs: one CTA per SM
        cps = 1;
        st = std::min(8L, long((220 * 1024 - fixed) / per_stage));
        if (st < 2) return BLDM_ERR_UNSUPPORTED;
    }
    // the end-of-tile S_pjk combine reuses the drained ring: [rows/stage][band_w][z]
    const size_t combine = size_t(kSweepWarps / c.wpr) * c.band_w * z * 8;
    if (!(tune && tune->stages > 0))
        while (c.wpr < kSweepWarps && combine > size_t(st) * c.stage_bytes && st < st_max) ++st;
    c.stages = int(st);
    if (c.wpr < kSweepWarps &&
        size_t(kSweepWarps / c.wpr) * c.band_w * z * 8 > size_t(c.stages) * c.stage_bytes)
        return BLDM_ERR_UNSUPPORTED;
    c.smem_update = size_t(c.stages) * per_stage + fixed;
    c.smem_sums = c.smem_update;
    c.ctas_per_sm = cps;
    // Row ranges: fill the resident CTA slots in one wave (a partial second
    // wave of a bandwidth-bound sweep costs a whole tail).
    const long target = long(c.ctas_per_sm) * num_sms;
    long nrr = target / c.n_bands;
    if (tune && tune->row_ranges > 0) nrr = tune->row_ranges;
    nrr = std::max(1L, std::min(long(x), nrr));
    c.n_rr = int(nrr);
    c.rr_base = int(x / nrr);
    c.rr_extra = int(x % nrr);
    finalize_blocks(c, x, z);
    return BLDM_OK;
}

// Shape, launch configuration and workspace layout of a plan (no device
// memory yet): plan_setup allocates the workspace, plan_setup_in places it in
// memory the caller provides.  Both bind through plan_bind_workspace, so the
// layout exists once.
static int plan_configure(PlanImpl* p, size_t x, size_t y, size_t z, int dtype,
                          const bldm_tuning* tune) {
    if (x == 0 || y == 0 || z == 0) return BLDM_ERR_BAD_ARG;
    if (dtype != BLDM_F64 && dtype != BLDM_F32) return BLDM_ERR_BAD_ARG;
    BLDM_CU(cudaGetDevice(&p->device));
    p->dtype = dtype;
    p->x = x;
    p->y = y;
    p->z = z;
    p->esize = dtype == BLDM_F64 ? 8 : 4;
    p->skip_zero = tune && tune->skip_zero_rows != 0;
    int rc = choose_cfg(p->cfg, x, y, z, p->esize, num_sms_of(p->device), tune);
    if (rc) return rc;
    const SweepCfg& c = p->cfg;
    // the long-fiber kernels sweep every row (no row lists)
    if (c.long_mode) p->skip_zero = false;
    WorkspaceLayout& L = p->layout;
    const size_t a = 256;
    size_t off = 0;
    L.o_pjk = off;
    off = align_up(off + size_t(c.n_rr) * y * z * 8, a);
    L.o_ipk = off;
    off = align_up(off + size_t(c.n_bands) * x * z * 8, a);
    L.o_psiB = off;
    off = align_up(off + y * z * p->esize, a);
    L.o_psiA = off;
    off = align_up(off + x * z * p->esize, a);
    L.o_psiAS = off;
    off = align_up(off + z * p->esize, a);
    L.o_asum = off;
    off = align_up(off + size_t(c.n_ablk) * z * 8, a);
    L.o_words = off;  // finalize counter | error word | conservation residual
    off = align_up(off + kWorkspaceWords, a);
    L.o_nzr = off;
    if (p->skip_zero) off = align_up(off + size_t(c.n_bands) * x * 4, a);
    L.o_nzc = off;
    if (p->skip_zero) off = align_up(off + size_t(c.n_bands) * (x + 1) * 4, a);
    L.o_fsum = off;
    if (c.long_mode) off = align_up(off + x * y * sizeof(double4), a);
    L.bytes = off;
    return BLDM_OK;
}

// Points the plan's pieces into `ws` (at least p->layout.bytes bytes) and opts
// the plan's kernels into their dynamic shared memory.
static int plan_bind_workspace(PlanImpl* p, void* ws) {
    const WorkspaceLayout& L = p->layout;
    p->ws_bytes = L.bytes;
    char* base = static_cast<char*>(ws);
    p->part_pjk = reinterpret_cast<double*>(base + L.o_pjk);
    p->part_ipk = reinterpret_cast<double*>(base + L.o_ipk);
    p->psiB = base + L.o_psiB;
    p->psiA = base + L.o_psiA;
    p->psiAS = base + L.o_psiAS;
    p->asum_part = reinterpret_cast<double*>(base + L.o_asum);
    p->counter = reinterpret_cast<unsigned*>(base + L.o_words);
    p->err = reinterpret_cast<int*>(base + L.o_words + 16);
    p->cons = reinterpret_cast<unsigned long long*>(base + L.o_words + 32);
    p->nz_rows = p->skip_zero ? reinterpret_cast<int*>(base + L.o_nzr) : nullptr;
    p->nz_cnt = p->skip_zero ? reinterpret_cast<int*>(base + L.o_nzc) : nullptr;
    const SweepCfg& c = p->cfg;
    p->fsum = c.long_mode ? base + L.o_fsum : nullptr;
    if (c.long_mode) return BLDM_OK;  // no dynamic shared memory
    for (int mode = SWEEP_SUMS; mode <= SWEEP_COMPACT; ++mode)
        for (int ap = 0; ap < 2; ++ap) {
            void* fn = nullptr;
            if (p->dtype == BLDM_F64)
                fn = reinterpret_cast<void*>(pick_sweep<double>(c, mode, ap != 0));
            else
                fn = reinterpret_cast<void*>(pick_sweep<float>(c, mode, ap != 0));
            if (!fn) return BLDM_ERR_UNSUPPORTED;
            const int rc_attr = ensure_smem_attr(fn, c.smem_update);
            if (rc_attr) return rc_attr;
        }
    return BLDM_OK;
}

int plan_setup(PlanImpl* p, size_t x, size_t y, size_t z, int dtype, const bldm_tuning* tune) {
    int rc = plan_configure(p, x, y, z, dtype, tune);
    if (rc) return rc;
    cudaError_t e = cudaMalloc(&p->ws, p->layout.bytes);
    if (e != cudaSuccess) {
        p->ws = nullptr;
        return cuda_status(e);
    }
    p->owns_ws = true;
    rc = plan_bind_workspace(p, p->ws);
    if (rc) return rc;
    BLDM_CU(cudaMemset(static_cast<char*>(p->ws) + p->layout.o_words, 0, kWorkspaceWords));
    return BLDM_OK;
}

// Lays the plan's workspace out in caller-provided device memory `ws` of
// `ws_cap` bytes instead of allocating it.  Returns BLDM_ERR_TOO_LARGE (and the
// bytes needed in *ws_needed) when the workspace does not fit.  The counter and
// error word are cleared on `st`.
int plan_setup_in(PlanImpl* p, size_t x, size_t y, size_t z, int dtype, void* ws,
                  size_t ws_cap, size_t* ws_needed, cudaStream_t st) {
    if (!ws) return BLDM_ERR_BAD_ARG;
    int rc = plan_configure(p, x, y, z, dtype, nullptr);
    if (rc) return rc;
    if (ws_needed) *ws_needed = p->layout.bytes;
    if (p->layout.bytes > ws_cap) return BLDM_ERR_TOO_LARGE;
    p->ws = ws;  // not owned: plan_free leaves it alone
    p->owns_ws = false;
    rc = plan_bind_workspace(p, ws);
    if (rc) return rc;
    BLDM_CU(cudaMemsetAsync(static_cast<char*>(ws) + p->layout.o_words, 0, kWorkspaceWords, st));
    return BLDM_OK;
}

void plan_free(PlanImpl* p) {
    if (p->ws && p->owns_ws) cudaFree(p->ws);
    p->ws = nullptr;
}

template <typename T>
static SweepParams<T> sweep_params(PlanImpl* p, const void* dX, void* dS, double eps) {
    const SweepCfg& c = p->cfg;
    SweepParams<T> s;
    SweepInst<T>& in = s.in;
    in.S = static_cast<T*>(dS);
    in.X = static_cast<const T*>(dX);
    in.psiB = static_cast<const T*>(p->psiB);
    in.psiA = static_cast<const T*>(p->psiA);
    in.psiAS = static_cast<const T*>(p->psiAS);
    in.part_pjk = p->part_pjk;
    in.part_ipk = p->part_ipk;
    in.delta_part = nullptr;
    in.nz_rows = p->nz_rows;
    in.nz_cnt = p->nz_cnt;
    in.x = (long long)p->x;
    in.y = (long long)p->y;
    in.z = (long long)p->z;
    in.n_bands = c.n_bands;
    in.band_w = c.band_w;
    in.wpr = c.wpr;
    in.n_rr = c.n_rr;
    in.rr_base = c.rr_base;
    in.rr_extra = c.rr_extra;
    s.L.stages = c.stages;
    s.L.stage_bytes = c.stage_bytes;
    s.L.eps = eps;
    s.L.err = p->err;
    return s;
}

template <typename T>
static FinParams<T> fin_params(PlanImpl* p, const double* dalpha, const double* dbeta,
                               int plus_appr, int minus_appr) {
    const SweepCfg& c = p->cfg;
    FinParams<T> fp;
    FinInst<T>& f = fp.f;
    f.part_pjk = p->part_pjk;
    f.part_ipk = p->part_ipk;
    f.alpha = dalpha;
    f.beta = dbeta;
    f.psiB = static_cast<T*>(p->psiB);
    f.psiA = static_cast<T*>(p->psiA);
    f.psiAS = static_cast<T*>(p->psiAS);
    f.asum_part = p->asum_part;
    f.counter = p->counter;
    f.delta_part = nullptr;
    f.rel_change = nullptr;
    f.red = nullptr;
    f.x = (long long)p->x;
    f.y = (long long)p->y;
    f.z = (long long)p->z;
    f.n_rr = c.n_rr;
    f.n_bands = c.n_bands;
    f.nbB = int((p->y * p->z + kFinThreads - 1) / kFinThreads);
    f.n_ablk = c.n_ablk;
    f.rows_per_ablk = c.rows_per_ablk;
    f.n_tiles = c.n_rr * c.n_bands;
    fp.plus_appr = plus_appr;
    fp.minus_appr = minus_appr;
    return fp;
}

template <typename T>
static LongSweepParams<T> long_params(PlanImpl* p, const void* dX, void* dS, double eps) {
    const SweepCfg& c = p->cfg;
    LongSweepParams<T> l;
    l.S = static_cast<T*>(dS);
    l.X = static_cast<const T*>(dX);
    l.psiB = static_cast<const T*>(p->psiB);
    l.psiA = static_cast<const T*>(p->psiA);
    l.psiAS = static_cast<const T*>(p->psiAS);
    l.part_pjk = p->part_pjk;
    l.part_ipk = p->part_ipk;
    l.fsum = static_cast<double4*>(p->fsum);
    l.x = (long long)p->x;
    l.y = (long long)p->y;
    l.z = (long long)p->z;
    l.n_kc = c.n_kc;
    l.n_bands = c.n_bands;
    l.n_rr = c.n_rr;
    l.rr_base = c.rr_base;
    l.rr_extra = c.rr_extra;
    l.eps = eps;
    return l;
}

// The iterations of a long-fiber plan: sums of S0, finalize, then per iteration
// the fiber-sums pass, the update pass and the finalize.  Events (profiling)
// bracket the two passes of each update.
template <typename T>
static int run_long(PlanImpl* p, const void* dX, const double* dalpha, const double* dbeta,
                    void* dS, size_t max_iter, int psi_mode, double eps, cudaStream_t st,
                    cudaEvent_t* ev, size_t nev) {
    const int plus_appr = psi_mode != BLDM_PSI_EXACT;
    const int minus_appr = psi_mode == BLDM_PSI_APPR;
    const LongSweepParams<T> lp = long_params<T>(p, dX, dS, eps);
    const FinParams<T> fp = fin_params<T>(p, dalpha, dbeta, plus_appr, minus_appr);
    const dim3 grid_f(unsigned(fp.f.nbB + fp.f.n_ablk));
    const int dt = sizeof(T) == 8 ? BLDM_F64 : BLDM_F32;
    const bool pdl = ev == nullptr;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    auto finalize = [&]() {
        cudaLaunchConfig_t lc = {};
        lc.gridDim = grid_f;
        lc.blockDim = dim3(kFinThreads);
        lc.stream = st;
        lc.attrs = pdl ? attr : nullptr;
        lc.numAttrs = pdl ? 1 : 0;
        p->launches += 1;
        return cuda_status(cudaLaunchKernelEx(&lc, finalize_kernel<T>, fp));
    };
    int rc = launch_long_sweep(dt, &lp, false, true, pdl, st, &p->launches);
    if (rc == BLDM_OK) rc = finalize();
    for (size_t it = 0; it < max_iter && rc == BLDM_OK; ++it) {
        if (ev && 2 * it + 1 < nev) cudaEventRecord(ev[2 * it], st);
        rc = launch_long_sweep(dt, &lp, true, plus_appr != 0, pdl, st, &p->launches);
        if (ev && 2 * it + 1 < nev) cudaEventRecord(ev[2 * it + 1], st);
        if (rc == BLDM_OK && it + 1 < max_iter) rc = finalize();
    }
    if (rc) return rc;
    return cuda_status(cudaGetLastError());
}

template <typename T>
static int run_typed(PlanImpl* p, const void* dX, const double* dalpha, const double* dbeta,
                     void* dS, size_t max_iter, int psi_mode, double eps, cudaStream_t st,
                     cudaEvent_t* ev, size_t nev) {
    if (p->cfg.long_mode)
        return run_long<T>(p, dX, dalpha, dbeta, dS, max_iter, psi_mode, eps, st, ev, nev);
    const SweepCfg& c = p->cfg;
    const int plus_appr = psi_mode != BLDM_PSI_EXACT;
    const int minus_appr = psi_mode == BLDM_PSI_APPR;
    SweepFn<T> fsum = pick_sweep<T>(c, SWEEP_SUMS, true);
    SweepFn<T> fupd = pick_sweep<T>(c, SWEEP_UPDATE, plus_appr != 0);
    // From the second update on, the first one has stored the zeros of every
    // fiber with X == 0: with skip_zero_rows those updates sweep listed rows.
    SweepFn<T> flater = p->skip_zero ? pick_sweep<T>(c, SWEEP_COMPACT, plus_appr != 0) : fupd;
    if (!fsum || !fupd || !flater) return BLDM_ERR_UNSUPPORTED;
    const SweepParams<T> sp = sweep_params<T>(p, dX, dS, eps);
    const FinParams<T> fp = fin_params<T>(p, dalpha, dbeta, plus_appr, minus_appr);
    const dim3 grid_s(unsigned(c.n_bands) * unsigned(c.n_rr));
    const dim3 grid_f(unsigned(fp.f.nbB + fp.f.n_ablk));
    if (p->skip_zero) {
        const int rc = launch_nz_rows(p->dtype, dX, (long long)p->x, (long long)p->y, c.band_w,
                                      c.n_bands, p->nz_rows, p->nz_cnt, st);
        if (rc) return rc;
        p->launches += 2;
    }
    // Programmatic dependent launches: each kernel may begin while the one
    // before it drains (its preamble overlaps; it waits in grid_dep_wait()).
    // Not across the event records of a profiling run.
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    auto launch = [&](auto fn, dim3 grid, unsigned threads, size_t smem, const auto& prm) {
        cudaLaunchConfig_t lc = {};
        lc.gridDim = grid;
        lc.blockDim = dim3(threads);
        lc.dynamicSmemBytes = smem;
        lc.stream = st;
        lc.attrs = ev ? nullptr : attr;
        lc.numAttrs = ev ? 0 : 1;
        return cudaLaunchKernelEx(&lc, fn, prm);
    };
    cudaError_t e = launch(fsum, grid_s, kSweepThreads, c.smem_sums, sp);
    if (e == cudaSuccess) e = launch(finalize_kernel<T>, grid_f, kFinThreads, 0, fp);
    p->launches += 2;
    for (size_t it = 0; it < max_iter && e == cudaSuccess; ++it) {
        if (ev && 2 * it + 1 < nev) cudaEventRecord(ev[2 * it], st);
        e = launch(it == 0 ? fupd : flater, grid_s, kSweepThreads, c.smem_update, sp);
        if (ev && 2 * it + 1 < nev) cudaEventRecord(ev[2 * it + 1], st);
        p->launches += 1;
        if (e == cudaSuccess && it + 1 < max_iter) {
            e = launch(finalize_kernel<T>, grid_f, kFinThreads, 0, fp);
            p->launches += 1;
        }
    }
    if (e != cudaSuccess) return cuda_status(e);
    return cuda_status(cudaGetLastError());
}

// Axis-sum partials of S alone (the sums sweep): part_pjk[n_rr][y][z] and
// part_ipk[n_bands][x][z] of the plan's workspace; no X, no digamma tables.
int plan_sums(PlanImpl* p, const void* dS, cudaStream_t st) {
    if (!p || !p->ws || !dS) return BLDM_ERR_BAD_ARG;
    if (reinterpret_cast<uintptr_t>(dS) & 15) return BLDM_ERR_BAD_ARG;
    const SweepCfg& c = p->cfg;
    if (c.long_mode) {
        if (p->dtype == BLDM_F64) {
            const LongSweepParams<double> lp = long_params<double>(p, nullptr, const_cast<void*>(dS), 0.0);
            return launch_long_sweep(BLDM_F64, &lp, false, true, false, st, &p->launches);
        }
        const LongSweepParams<float> lp = long_params<float>(p, nullptr, const_cast<void*>(dS), 0.0);
        return launch_long_sweep(BLDM_F32, &lp, false, true, false, st, &p->launches);
    }
    const dim3 grid_s(unsigned(c.n_bands) * unsigned(c.n_rr));
    if (p->dtype == BLDM_F64) {
        SweepFn<double> f = pick_sweep<double>(c, SWEEP_SUMS, true);
        if (!f) return BLDM_ERR_UNSUPPORTED;
        f<<<grid_s, kSweepThreads, c.smem_sums, st>>>(
            sweep_params<double>(p, nullptr, const_cast<void*>(dS), 0.0));
    } else {
        SweepFn<float> f = pick_sweep<float>(c, SWEEP_SUMS, true);
        if (!f) return BLDM_ERR_UNSUPPORTED;
        f<<<grid_s, kSweepThreads, c.smem_sums, st>>>(
            sweep_params<float>(p, nullptr, const_cast<void*>(dS), 0.0));
    }
    p->launches += 1;
    return cuda_status(cudaGetLastError());
}

// Row-sharded solves (one plan per shard of rows): a sweep of the shard (the
// axis sums of S, or an update) followed by the finalize's reduction of the
// shard's partials into red; shard_finish tabulates the shared digamma
// values from red once it holds the sum over all shards.
template <typename T>
static int shard_step_typed(PlanImpl* p, const void* dX, void* dS, const double* dalpha,
                            double* d_red, bool update, int psi_mode, double eps,
                            cudaStream_t st) {
    const SweepCfg& c = p->cfg;
    const int plus_appr = psi_mode != BLDM_PSI_EXACT;
    const int minus_appr = psi_mode == BLDM_PSI_APPR;
    FinParams<T> fp = fin_params<T>(p, dalpha, nullptr, plus_appr, minus_appr);
    fp.f.red = d_red;
    const dim3 grid_f(unsigned(fp.f.nbB + fp.f.n_ablk));
    if (c.long_mode) {
        const LongSweepParams<T> lp = long_params<T>(p, dX, dS, eps);
        const int rc = launch_long_sweep(sizeof(T) == 8 ? BLDM_F64 : BLDM_F32, &lp, update,
                                         update ? plus_appr != 0 : true, false, st, &p->launches);
        if (rc) return rc;
    } else {
        SweepFn<T> f = pick_sweep<T>(c, update ? SWEEP_UPDATE : SWEEP_SUMS,
                                     update ? plus_appr != 0 : true);
        if (!f) return BLDM_ERR_UNSUPPORTED;
        const SweepParams<T> sp = sweep_params<T>(p, dX, dS, eps);
        const dim3 grid_s(unsigned(c.n_bands) * unsigned(c.n_rr));
        f<<<grid_s, kSweepThreads, update ? c.smem_update : c.smem_sums, st>>>(sp);
        p->launches += 1;
    }
    finalize_kernel<T><<<grid_f, kFinThreads, 0, st>>>(fp);
    p->launches += 1;
    return cuda_status(cudaGetLastError());
}

int plan_shard_step(PlanImpl* p, const void* dX, void* dS, const double* dalpha, double* d_red,
                    bool update, int psi_mode, double eps, cudaStream_t st) {
    if (!p || !p->ws || !dS || !dalpha || !d_red || (update && !dX)) return BLDM_ERR_BAD_ARG;
    if (psi_mode < 0 || psi_mode > 2) return BLDM_ERR_BAD_ARG;
    if ((reinterpret_cast<uintptr_t>(dX) | reinterpret_cast<uintptr_t>(dS)) & 15)
        return BLDM_ERR_BAD_ARG;
    return p->dtype == BLDM_F64
               ? shard_step_typed<double>(p, dX, dS, dalpha, d_red, update, psi_mode, eps, st)
               : shard_step_typed<float>(p, dX, dS, dalpha, d_red, update, psi_mode, eps, st);
}

int plan_shard_finish(PlanImpl* p, const double* dbeta, const double* d_red, int psi_mode,
                      cudaStream_t st) {
    if (!p || !p->ws || !dbeta || !d_red) return BLDM_ERR_BAD_ARG;
    if (psi_mode < 0 || psi_mode > 2) return BLDM_ERR_BAD_ARG;
    const long long y = (long long)p->y, z = (long long)p->z;
    const unsigned blocks = unsigned((std::max(y * z, z) + kFinThreads - 1) / kFinThreads);
    const int plus_appr = psi_mode != BLDM_PSI_EXACT;
    const int minus_appr = psi_mode == BLDM_PSI_APPR;
    if (p->dtype == BLDM_F64)
        shard_finish_kernel<double><<<blocks, kFinThreads, 0, st>>>(
            d_red, dbeta, y, z, static_cast<double*>(p->psiB), static_cast<double*>(p->psiAS),
            plus_appr, minus_appr);
    else
        shard_finish_kernel<float><<<blocks, kFinThreads, 0, st>>>(
            d_red, dbeta, y, z, static_cast<float*>(p->psiB), static_cast<float*>(p->psiAS),
            plus_appr, minus_appr);
    p->launches += 1;
    return cuda_status(cudaGetLastError());
}

int plan_run(PlanImpl* p, const void* dX, const double* dalpha, const double* dbeta, void* dS,
             size_t max_iter, int psi_mode, double eps, cudaStream_t st, cudaEvent_t* ev,
             size_t nev) {
    if (!p || !p->ws || !dX || !dalpha || !dbeta || !dS) return BLDM_ERR_BAD_ARG;
    if (psi_mode < 0 || psi_mode > 2) return BLDM_ERR_BAD_ARG;
    if ((reinterpret_cast<uintptr_t>(dX) | reinterpret_cast<uintptr_t>(dS)) & 15)
        return BLDM_ERR_BAD_ARG;
    if (max_iter == 0) return BLDM_OK;
    if (p->dtype == BLDM_F64)
        return run_typed<double>(p, dX, dalpha, dbeta, dS, max_iter, psi_mode, eps, st, ev, nev);
    return run_typed<float>(p, dX, dalpha, dbeta, dS, max_iter, psi_mode, eps, st, ev, nev);
}

int plan_init_S(PlanImpl* p, const void* dX, void* dS, uint64_t seed, cudaStream_t st) {
    const int rc = launch_init_S(p->dtype, dX, dS, (long long)(p->x * p->y), (long long)p->z,
                                 seed, st);
    p->launches += 1;
    return rc;
}

// One warp per (row, band): nz_rows[b][i] = 1 when row i has a nonzero X in
// band b's columns (lanes read the segment coalesced).
template <typename T>
__global__ void nz_flags_kernel(const T* X, long long x, long long y, int band_w, int n_bands,
                                int* flags) {
    const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (w >= x * n_bands) return;  // warp-uniform
    const long long i = w / n_bands;
    const int b = int(w % n_bands);
    const long long j0 = (long long)b * band_w;
    const long long j1 = min(y, j0 + band_w);
    bool nz = false;
    for (long long j = j0 + lane; j < j1; j += 32) nz = nz || X[i * y + j] != T(0);
    nz = __any_sync(0xffffffffu, nz);
    if (lane == 0) flags[(long long)b * x + i] = nz ? 1 : 0;
}

// One warp per band: compacts the band's flags into its ascending row list in
// place (an entry is written at or below the index it was read from, after
// the warp's reads of that chunk) and writes the running counts.
__global__ void nz_compact_kernel(long long x, int n_bands, int* nz_rows, int* nz_cnt) {
    const int b = int(((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    const int lane = threadIdx.x & 31;
    if (b >= n_bands) return;  // warp-uniform
    int* list = nz_rows + (long long)b * x;
    int* cnt = nz_cnt + (long long)b * (x + 1);
    int base = 0;
    for (long long i0 = 0; i0 < x; i0 += 32) {
        const long long i = i0 + lane;
        const bool nz = i < x && list[i] != 0;
        const unsigned m = __ballot_sync(0xffffffffu, nz);
        const int pre = __popc(m & ((1u << lane) - 1u));
        if (i < x) cnt[i] = base + pre;
        __syncwarp();
        if (nz) list[base + pre] = int(i);
        __syncwarp();
        base += __popc(m);
    }
    if (lane == 0) cnt[x] = base;
}

int launch_nz_rows(int dtype, const void* dX, long long x, long long y, int band_w, int n_bands,
                   int* nz_rows, int* nz_cnt, cudaStream_t st) {
    const long long warps = x * n_bands;
    const unsigned blocks = unsigned((warps * 32 + 255) / 256);
    if (dtype == BLDM_F64)
        nz_flags_kernel<double><<<blocks, 256, 0, st>>>(static_cast<const double*>(dX), x, y,
                                                        band_w, n_bands, nz_rows);
    else
        nz_flags_kernel<float><<<blocks, 256, 0, st>>>(static_cast<const float*>(dX), x, y,
                                                       band_w, n_bands, nz_rows);
    const unsigned cblocks = unsigned(((long long)n_bands * 32 + 255) / 256);
    nz_compact_kernel<<<cblocks, 256, 0, st>>>(x, n_bands, nz_rows, nz_cnt);
    return cuda_status(cudaGetLastError());
}

int launch_init_S(int dtype, const void* dX, void* dS, long long nf, long long z, uint64_t seed,
                  cudaStream_t st) {
    if (nf <= 0 || z <= 0) return BLDM_OK;
    int lpf = 1;
    while (lpf < 32 && lpf < z) lpf <<= 1;
    const long long warps = (nf + (32 / lpf) - 1) / (32 / lpf);
    const unsigned blocks = unsigned((warps * 32 + 255) / 256);
    if (dtype == BLDM_F64)
        init_S_kernel<double><<<blocks, 256, 0, st>>>(static_cast<const double*>(dX),
                                                      static_cast<double*>(dS), nf, z, seed, lpf);
    else
        init_S_kernel<float><<<blocks, 256, 0, st>>>(static_cast<const float*>(dX),
                                                     static_cast<float*>(dS), nf, z, seed, lpf);
    return cuda_status(cudaGetLastError());
}

// Reads the error word behind the work queued on `st` and clears it, all in
// the order of `st` (no legacy-stream copy that would wait for the device's
// other blocking streams).
int plan_check(PlanImpl* p, cudaStream_t st) {
    int herr = 0;
    BLDM_CU(cudaMemcpyAsync(&herr, p->err, sizeof(int), cudaMemcpyDeviceToHost, st));
    BLDM_CU(cudaStreamSynchronize(st));
    if (herr != 0) {
        BLDM_CU(cudaMemsetAsync(p->err, 0, sizeof(int), st));
        BLDM_CU(cudaStreamSynchronize(st));
        return BLDM_ERR_TIMEOUT;
    }
    return BLDM_OK;
}

// Row-sum conservation residual of (X, S): max over fibers of
// |sum_k S(i,j,k) - X(i,j)| / max(X(i,j), 1), in FP64.  Enqueued on `st`; the
// value lands in p->cons (the bits of a nonnegative double).
int plan_conservation_launch(PlanImpl* p, const void* dX, const void* dS, cudaStream_t st) {
    if (!p || !p->ws || !dX || !dS) return BLDM_ERR_BAD_ARG;
    BLDM_CU(cudaMemsetAsync(p->cons, 0, sizeof(unsigned long long), st));
    const int rc = launch_conservation(p->dtype, dX, dS, (long long)(p->x * p->y),
                                       (long long)p->z, p->cons, st);
    p->launches += 1;
    return rc;
}

}  // namespace bldm
