// C ABI: the drop-in host-buffer solve (bld::bld_mult_cuda,
// src/bld/bld_mult/bld_mult.hpp:225-324) and the device-buffer plan API.
#include <chrono>
#include <cmath>
#include <cstring>
#include <list>
#include <map>
#include <memory>
#include <mutex>
#include <tuple>
#include <vector>

#include "bldm_internal.h"
#include "bldm_kernels.h"

using namespace bldm;

struct bldm_plan {
    PlanImpl impl;
};

namespace {

#define BLDM_CU_RET(call)                               \
    do {                                                \
        cudaError_t e_ = (call);                        \
        if (e_ != cudaSuccess) return cuda_status(e_);  \
    } while (0)

// Device buffers of one drop-in call shape, reused by later calls of the same
// shape on the same device.  An entry is used by one call at a time.
struct CacheEntry {
    int device = 0;
    int dtype = 0;
    size_t x = 0, y = 0, z = 0;
    bool busy = false;
    PlanImpl plan;
    void* io = nullptr;  // X | S | alpha | beta
    void* dX = nullptr;
    void* dS = nullptr;
    double* dalpha = nullptr;
    double* dbeta = nullptr;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    // The iterations of a solve captured once per (max_iter, psi_mode, eps)
    // and replayed: the entry's buffers are fixed, so are the launches.
    struct Graph {
        cudaGraphExec_t exec = nullptr;
        uint64_t launches = 0;
    };
    std::map<std::tuple<size_t, int, uint64_t>, Graph> graphs;
    ~CacheEntry() {
        for (auto& g : graphs)
            if (g.second.exec) cudaGraphExecDestroy(g.second.exec);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (stream) cudaStreamDestroy(stream);
        if (io) cudaFree(io);
        plan_free(&plan);
    }
};

std::mutex g_mu;
std::list<std::unique_ptr<CacheEntry>> g_cache;  // most recently used first
constexpr size_t kMaxCached = 4;

size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

int make_entry(CacheEntry* e, int device, int dtype, size_t x, size_t y, size_t z) {
    e->device = device;
    e->dtype = dtype;
    e->x = x;
    e->y = y;
    e->z = z;
    int rc = plan_setup(&e->plan, x, y, z, dtype);
    if (rc) return rc;
    const size_t es = dtype == BLDM_F64 ? 8 : 4;
    const size_t bX = align_up(x * y * es, 256), bS = align_up(x * y * z * es, 256);
    const size_t bA = align_up(x * 8, 256), bB = align_up(z * 8, 256);
    BLDM_CU_RET(cudaMalloc(&e->io, bX + bS + bA + bB));
    char* base = static_cast<char*>(e->io);
    e->dX = base;
    e->dS = base + bX;
    e->dalpha = reinterpret_cast<double*>(base + bX + bS);
    e->dbeta = reinterpret_cast<double*>(base + bX + bS + bA);
    BLDM_CU_RET(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking));
    BLDM_CU_RET(cudaEventCreate(&e->ev0));
    BLDM_CU_RET(cudaEventCreate(&e->ev1));
    return BLDM_OK;
}

// Returns a reserved entry for (device, dtype, shape), creating it if needed.
int acquire(int device, int dtype, size_t x, size_t y, size_t z, CacheEntry** out) {
    std::lock_guard<std::mutex> lk(g_mu);
    for (auto it = g_cache.begin(); it != g_cache.end(); ++it) {
        CacheEntry* e = it->get();
        if (!e->busy && e->device == device && e->dtype == dtype && e->x == x && e->y == y &&
            e->z == z) {
            e->busy = true;
            g_cache.splice(g_cache.begin(), g_cache, it);
            *out = e;
            return BLDM_OK;
        }
    }
    // Evict idle entries beyond the cap (least recently used last).
    while (g_cache.size() >= kMaxCached) {
        auto victim = g_cache.end();
        for (auto it = g_cache.begin(); it != g_cache.end(); ++it)
            if (!(*it)->busy) victim = it;
        if (victim == g_cache.end()) break;
        g_cache.erase(victim);
    }
    std::unique_ptr<CacheEntry> e(new CacheEntry());
    int rc = make_entry(e.get(), device, dtype, x, y, z);
    if (rc) {
        // a failed allocation may be cured by dropping idle cached shapes
        for (auto it = g_cache.begin(); it != g_cache.end();) {
            if (!(*it)->busy) it = g_cache.erase(it);
            else ++it;
        }
        e.reset(new CacheEntry());
        rc = make_entry(e.get(), device, dtype, x, y, z);
        if (rc) return rc;
    }
    e->busy = true;
    *out = e.get();
    g_cache.push_front(std::move(e));
    return BLDM_OK;
}

void release(CacheEntry* e) {
    std::lock_guard<std::mutex> lk(g_mu);
    e->busy = false;
}

int check_params(size_t x, size_t z, const bldm_params* p, int psi_mode) {
    if (!p) return BLDM_ERR_BAD_ARG;
    if (psi_mode < BLDM_PSI_EXACT || psi_mode > BLDM_PSI_LEGACY_CUDA) return BLDM_ERR_BAD_ARG;
    // check_bld_params (src/bld/util_details.hpp:20-28)
    if (p->n_alpha != x || p->n_beta != z) return BLDM_ERR_BAD_ARG;
    if ((x > 0 && !p->alpha) || (z > 0 && !p->beta)) return BLDM_ERR_BAD_ARG;
    return BLDM_OK;
}

// plan_run on the entry's buffers, from a CUDA graph captured on first use.
// A capture that fails (e.g. inside a caller's own capture) falls back to
// launching directly.
int run_iterations(CacheEntry* e, size_t max_iter, int psi_mode, double eps) {
    cudaStream_t st = e->stream;
    if (max_iter == 0) return BLDM_OK;
    uint64_t eb;
    std::memcpy(&eb, &eps, sizeof eb);
    const auto key = std::make_tuple(max_iter, psi_mode, eb);
    auto it = e->graphs.find(key);
    if (it == e->graphs.end()) {
        CacheEntry::Graph g;
        const uint64_t l0 = e->plan.launches;
        cudaGraph_t graph = nullptr;
        int r = BLDM_ERR_CUDA;
        if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
            r = plan_run(&e->plan, e->dX, e->dalpha, e->dbeta, e->dS, max_iter, psi_mode, eps,
                         st, nullptr, 0);
            const cudaError_t ce = cudaStreamEndCapture(st, &graph);
            if (r == BLDM_OK && (ce != cudaSuccess ||
                                 cudaGraphInstantiate(&g.exec, graph, 0) != cudaSuccess))
                r = BLDM_ERR_CUDA;
            if (graph) cudaGraphDestroy(graph);
        }
        g.launches = e->plan.launches - l0;
        e->plan.launches = l0;
        if (r != BLDM_OK || !g.exec) {
            (void)cudaGetLastError();  // a failed capture leaves no sticky error
            if (g.exec) cudaGraphExecDestroy(g.exec);
            return plan_run(&e->plan, e->dX, e->dalpha, e->dbeta, e->dS, max_iter, psi_mode, eps,
                            st, nullptr, 0);
        }
        it = e->graphs.emplace(key, g).first;
    }
    const cudaError_t le = cudaGraphLaunch(it->second.exec, st);
    if (le != cudaSuccess) return cuda_status(le);
    e->plan.launches += it->second.launches;
    return BLDM_OK;
}

template <typename T>
int solve_impl(const T* X, size_t x, size_t y, size_t z, const bldm_params* params,
               size_t max_iter, int psi_mode, double eps, const T* S0, uint64_t seed, T* S_out,
               bldm_stats* stats) {
    const auto t0 = std::chrono::steady_clock::now();
    if (stats) std::memset(stats, 0, sizeof(*stats));
    int rc = check_params(x, z, params, psi_mode);
    if (rc) return rc;
    if ((x * y > 0 && !X) || (x * y * z > 0 && !S_out)) return BLDM_ERR_BAD_ARG;
    // X must be nonnegative (check_bld_params); NaN fails the check as in Eigen.
    for (size_t e = 0; e < x * y; ++e)
        if (!(X[e] >= T(0))) return BLDM_ERR_NEG_X;
    if (x * y * z == 0) return BLDM_OK;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return BLDM_ERR_NO_DEVICE;
    int device = 0;
    BLDM_CU_RET(cudaGetDevice(&device));
    const int dtype = sizeof(T) == 8 ? BLDM_F64 : BLDM_F32;
    CacheEntry* e = nullptr;
    rc = acquire(device, dtype, x, y, z, &e);
    if (rc) return rc;
    cudaStream_t st = e->stream;
    const uint64_t launches0 = e->plan.launches;
    auto body = [&]() -> int {
        BLDM_CU_RET(cudaMemcpyAsync(e->dX, X, x * y * sizeof(T), cudaMemcpyHostToDevice, st));
        BLDM_CU_RET(cudaMemcpyAsync(e->dalpha, params->alpha, x * sizeof(double),
                                    cudaMemcpyHostToDevice, st));
        BLDM_CU_RET(cudaMemcpyAsync(e->dbeta, params->beta, z * sizeof(double),
                                    cudaMemcpyHostToDevice, st));
        if (S0) {
            BLDM_CU_RET(cudaMemcpyAsync(e->dS, S0, x * y * z * sizeof(T), cudaMemcpyHostToDevice,
                                        st));
        } else {
            int r = plan_init_S(&e->plan, e->dX, e->dS, seed, st);
            if (r) return r;
        }
        BLDM_CU_RET(cudaEventRecord(e->ev0, st));
        int r = run_iterations(e, max_iter, psi_mode, eps);
        if (r) return r;
        BLDM_CU_RET(cudaEventRecord(e->ev1, st));
        // row-sum conservation of the result, one more read of S on the device
        r = plan_conservation_launch(&e->plan, e->dX, e->dS, st);
        if (r) return r;
        unsigned long long cons_bits = 0;
        BLDM_CU_RET(cudaMemcpyAsync(&cons_bits, e->plan.cons, sizeof cons_bits,
                                    cudaMemcpyDeviceToHost, st));
        BLDM_CU_RET(cudaMemcpyAsync(S_out, e->dS, x * y * z * sizeof(T), cudaMemcpyDeviceToHost,
                                    st));
        r = plan_check(&e->plan, st);
        if (r) return r;
        if (stats) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e->ev0, e->ev1);
            stats->device_ms = ms;
            stats->iterations = max_iter;
            stats->kernel_launches = e->plan.launches - launches0;
            stats->conservation_residual = cons_value(cons_bits);
        }
        return BLDM_OK;
    };
    rc = body();
    if (rc) cudaStreamSynchronize(st);
    release(e);
    if (stats)
        stats->total_ms = std::chrono::duration<double, std::milli>(
                              std::chrono::steady_clock::now() - t0)
                              .count();
    return rc;
}

}  // namespace

extern "C" {

int bldm_solve_f64(const double* X, size_t x, size_t y, size_t z, const bldm_params* params,
                   size_t max_iter, int psi_mode, double eps, const double* S0, uint64_t seed,
                   double* S_out, bldm_stats* stats) {
    return solve_impl<double>(X, x, y, z, params, max_iter, psi_mode, eps, S0, seed, S_out,
                              stats);
}

int bldm_solve_f32(const float* X, size_t x, size_t y, size_t z, const bldm_params* params,
                   size_t max_iter, int psi_mode, double eps, const float* S0, uint64_t seed,
                   float* S_out, bldm_stats* stats) {
    return solve_impl<float>(X, x, y, z, params, max_iter, psi_mode, eps, S0, seed, S_out,
                             stats);
}

int bldm_release_cache(void) {
    int device = 0;
    if (cudaGetDevice(&device) != cudaSuccess) return BLDM_ERR_NO_DEVICE;
    std::lock_guard<std::mutex> lk(g_mu);
    for (auto it = g_cache.begin(); it != g_cache.end();) {
        if (!(*it)->busy && (*it)->device == device) it = g_cache.erase(it);
        else ++it;
    }
    return BLDM_OK;
}

int bldm_plan_create(bldm_plan** plan, size_t x, size_t y, size_t z, int dtype) {
    if (!plan) return BLDM_ERR_BAD_ARG;
    *plan = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return BLDM_ERR_NO_DEVICE;
    std::unique_ptr<bldm_plan> p(new bldm_plan());
    int rc = plan_setup(&p->impl, x, y, z, dtype);
    if (rc) {
        plan_free(&p->impl);
        return rc;
    }
    *plan = p.release();
    return BLDM_OK;
}

int bldm_plan_create_tuned(bldm_plan** plan, size_t x, size_t y, size_t z, int dtype,
                           const bldm_tuning* tuning) {
    if (!plan) return BLDM_ERR_BAD_ARG;
    *plan = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return BLDM_ERR_NO_DEVICE;
    std::unique_ptr<bldm_plan> p(new bldm_plan());
    int rc = plan_setup(&p->impl, x, y, z, dtype, tuning);
    if (rc) {
        plan_free(&p->impl);
        return rc;
    }
    *plan = p.release();
    return BLDM_OK;
}

int bldm_plan_get_tuning(const bldm_plan* plan, bldm_tuning* out) {
    if (!plan || !out) return BLDM_ERR_BAD_ARG;
    out->stages = plan->impl.cfg.stages;
    out->ctas_per_sm = plan->impl.cfg.ctas_per_sm;
    out->row_ranges = plan->impl.cfg.n_rr;
    out->skip_zero_rows = plan->impl.skip_zero ? 1 : 0;
    return BLDM_OK;
}

int bldm_plan_destroy(bldm_plan* plan) {
    if (!plan) return BLDM_ERR_BAD_ARG;
    plan_free(&plan->impl);
    delete plan;
    return BLDM_OK;
}

int bldm_plan_workspace_bytes(const bldm_plan* plan, size_t* bytes) {
    if (!plan || !bytes) return BLDM_ERR_BAD_ARG;
    *bytes = plan->impl.ws_bytes;
    return BLDM_OK;
}

int bldm_plan_run(bldm_plan* plan, const void* d_X, const double* d_alpha, const double* d_beta,
                  void* d_S, size_t max_iter, int psi_mode, double eps, void* stream) {
    if (!plan) return BLDM_ERR_BAD_ARG;
    return plan_run(&plan->impl, d_X, d_alpha, d_beta, d_S, max_iter, psi_mode, eps,
                    static_cast<cudaStream_t>(stream), nullptr, 0);
}

int bldm_plan_conservation(bldm_plan* plan, const void* d_X, const void* d_S, void* stream,
                           double* residual) {
    if (!plan || !d_X || !d_S || !residual) return BLDM_ERR_BAD_ARG;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int rc = plan_conservation_launch(&plan->impl, d_X, d_S, st);
    if (rc) return rc;
    unsigned long long bits = 0;
    BLDM_CU_RET(cudaMemcpyAsync(&bits, plan->impl.cons, sizeof bits, cudaMemcpyDeviceToHost, st));
    BLDM_CU_RET(cudaStreamSynchronize(st));
    *residual = cons_value(bits);
    return BLDM_OK;
}

int bldm_plan_check(bldm_plan* plan, void* stream) {
    if (!plan) return BLDM_ERR_BAD_ARG;
    return plan_check(&plan->impl, static_cast<cudaStream_t>(stream));
}

int bldm_plan_init_S(bldm_plan* plan, const void* d_X, void* d_S, uint64_t seed, void* stream) {
    if (!plan || !d_X || !d_S) return BLDM_ERR_BAD_ARG;
    return plan_init_S(&plan->impl, d_X, d_S, seed, static_cast<cudaStream_t>(stream));
}

int bldm_plan_profile(bldm_plan* plan, const void* d_X, const double* d_alpha,
                      const double* d_beta, void* d_S, size_t iters, int psi_mode, double eps,
                      void* stream, double* update_kernel_ms, double* iteration_ms) {
    if (!plan || iters == 0 || !update_kernel_ms || !iteration_ms) return BLDM_ERR_BAD_ARG;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    std::vector<cudaEvent_t> ev(2 * iters + 2, nullptr);
    int rc = BLDM_OK;
    for (auto& e : ev)
        if (cudaEventCreate(&e) != cudaSuccess) rc = BLDM_ERR_CUDA;
    if (rc == BLDM_OK) {
        cudaEventRecord(ev[2 * iters], st);
        rc = plan_run(&plan->impl, d_X, d_alpha, d_beta, d_S, iters, psi_mode, eps, st, ev.data(),
                      2 * iters);
        cudaEventRecord(ev[2 * iters + 1], st);
    }
    if (rc == BLDM_OK) rc = plan_check(&plan->impl, st);
    if (rc == BLDM_OK) {
        double tot = 0.0;
        for (size_t i = 0; i < iters; ++i) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, ev[2 * i], ev[2 * i + 1]);
            tot += ms;
        }
        float all = 0.f;
        cudaEventElapsedTime(&all, ev[2 * iters], ev[2 * iters + 1]);
        *update_kernel_ms = tot / double(iters);
        *iteration_ms = double(all) / double(iters);
    }
    for (auto& e : ev)
        if (e) cudaEventDestroy(e);
    return rc;
}

int bldm_plan_shard_red_size(const bldm_plan* plan, size_t* n_doubles) {
    if (!plan || !n_doubles) return BLDM_ERR_BAD_ARG;
    *n_doubles = plan->impl.y * plan->impl.z + plan->impl.z;
    return BLDM_OK;
}

int bldm_plan_shard_sums(bldm_plan* plan, const void* d_S, const double* d_alpha, double* d_red,
                         int psi_mode, void* stream) {
    if (!plan) return BLDM_ERR_BAD_ARG;
    return plan_shard_step(&plan->impl, nullptr, const_cast<void*>(d_S), d_alpha, d_red, false,
                           psi_mode, 0.0, static_cast<cudaStream_t>(stream));
}

int bldm_plan_shard_update(bldm_plan* plan, const void* d_X, void* d_S, const double* d_alpha,
                           double* d_red, int psi_mode, double eps, void* stream) {
    if (!plan) return BLDM_ERR_BAD_ARG;
    return plan_shard_step(&plan->impl, d_X, d_S, d_alpha, d_red, true, psi_mode, eps,
                           static_cast<cudaStream_t>(stream));
}

int bldm_plan_shard_finish(bldm_plan* plan, const double* d_beta, const double* d_red,
                           int psi_mode, void* stream) {
    if (!plan) return BLDM_ERR_BAD_ARG;
    return plan_shard_finish(&plan->impl, d_beta, d_red, psi_mode,
                             static_cast<cudaStream_t>(stream));
}

int bldm_plan_launch_count(const bldm_plan* plan, uint64_t* count) {
    if (!plan || !count) return BLDM_ERR_BAD_ARG;
    *count = plan->impl.launches;
    return BLDM_OK;
}

const char* bldm_version(void) { return "bldm 0.1.0 (sm_100a)"; }

}  // extern "C"
