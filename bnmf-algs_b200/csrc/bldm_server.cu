// Serving loop: continuous batching of bld_mult requests (bldm_server_*).
//
// A worker thread owns the GPU work.  Each round it admits queued requests
// while a request slot and device memory (the configured budget, checked
// against the device's free memory) are available, allocates each admitted
// request's buffers stream-ordered, uploads X and draws the seeded initial S,
// runs `iters_per_round` iterations of every active request in shared
// launches (the multi-instance engine), and retires the requests whose
// relative change of S fell below `tol` or that reached `max_iter`: their S
// is copied back, their log-marginal is computed on the device in FP64, and
// their memory is freed.  S and the per-request state stay on the device
// between rounds.  A request's tiling and its iteration count depend only on
// itself, so its result is the same alone and in any mix.
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "bldm_engine.h"

using namespace bldm;

namespace {

using Clock = std::chrono::steady_clock;

enum ReqState { REQ_QUEUED = 0, REQ_ACTIVE = 1, REQ_DONE = 2, REQ_FAILED = 3 };

struct Request {
    uint64_t id = 0;
    size_t x = 0, y = 0, z = 0;
    std::vector<double> X, alpha, beta;
    double a = 1, b = 1;
    uint64_t seed = 0;
    int state = REQ_QUEUED;
    int status = BLDM_OK;
    std::atomic<bool> cancel{false};
    EngineInstance inst;
    void* dmem = nullptr;
    size_t dbytes = 0;
    int slot = -1;
    size_t iters = 0;
    double rel = 1.0;
    double log_marginal = 0.0;
    std::vector<double> S;
    Clock::time_point t_submit, t_admit, t_done;
};

double ms_between(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

}  // namespace

extern "C" int bldm_log_marginal_S(const void* d_S, int dtype, size_t x, size_t y, size_t z,
                                   const double* alpha, const double* beta, double a, double b,
                                   double* result, void* stream);

struct bldm_server {
    bldm_server_config cfg{};
    int device = 0;
    std::unique_ptr<Engine> eng;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request*> queue;
    std::unordered_map<uint64_t, std::unique_ptr<Request>> reqs;
    std::vector<Request*> active;
    std::vector<int> free_slots;
    double* d_rel = nullptr;
    std::vector<double> h_rel;
    size_t used = 0, peak = 0, budget = 0;
    uint64_t next_id = 1;
    bldm_server_stats st{};
    cudaStream_t stream = nullptr;
    std::thread worker;
    bool stop = false;
    std::atomic<size_t> n_active{0};

    void loop();
    int admit(Request* r);
    void retire(Request* r, int status);
};

int bldm_server::admit(Request* r) {
    int rc = eng->configure(r->inst, r->x, r->y, r->z);
    if (rc) return rc;
    cudaError_t e = cudaMallocAsync(&r->dmem, r->dbytes, stream);
    if (e != cudaSuccess) {
        r->dmem = nullptr;
        return cuda_status(e);
    }
    eng->bind(r->inst, r->dmem);
    r->inst.rel = d_rel + r->slot;
    e = cudaMemsetAsync(r->inst.counter, 0, 16, stream);
    if (e != cudaSuccess) return cuda_status(e);
    const size_t es = eng->es();
    if (es == 8) {
        e = cudaMemcpyAsync(r->inst.X, r->X.data(), r->x * r->y * 8, cudaMemcpyHostToDevice,
                            stream);
    } else {
        std::vector<float> tmp(r->X.begin(), r->X.end());
        e = cudaMemcpyAsync(r->inst.X, tmp.data(), r->x * r->y * 4, cudaMemcpyHostToDevice,
                            stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    }
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(r->inst.alpha, r->alpha.data(), r->x * 8, cudaMemcpyHostToDevice,
                            stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(r->inst.beta, r->beta.data(), r->z * 8, cudaMemcpyHostToDevice,
                            stream);
    if (e != cudaSuccess) return cuda_status(e);
    return launch_init_S(eng->dtype(), r->inst.X, r->inst.S, (long long)(r->x * r->y),
                         (long long)r->z, r->seed, stream);
}

void bldm_server::retire(Request* r, int status) {
    if (status == BLDM_OK && r->dmem) {
        const size_t n = r->x * r->y * r->z;
        r->S.resize(n);
        cudaError_t e;
        if (eng->es() == 8) {
            e = cudaMemcpyAsync(r->S.data(), r->inst.S, n * 8, cudaMemcpyDeviceToHost, stream);
            if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        } else {
            std::vector<float> tmp(n);
            e = cudaMemcpyAsync(tmp.data(), r->inst.S, n * 4, cudaMemcpyDeviceToHost, stream);
            if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
            for (size_t i = 0; i < n; ++i) r->S[i] = tmp[i];
        }
        if (e != cudaSuccess) status = cuda_status(e);
        if (status == BLDM_OK)
            status = bldm_log_marginal_S(r->inst.S, eng->dtype(), r->x, r->y, r->z,
                                         r->alpha.data(), r->beta.data(), r->a, r->b,
                                         &r->log_marginal, stream);
    }
    if (r->dmem) cudaFreeAsync(r->dmem, stream);
    r->dmem = nullptr;
    std::lock_guard<std::mutex> lk(mu);
    if (r->slot >= 0) free_slots.push_back(r->slot);
    r->slot = -1;
    used -= r->dbytes;
    r->status = status;
    r->state = status == BLDM_OK ? REQ_DONE : REQ_FAILED;
    r->t_done = Clock::now();
    if (status == BLDM_OK) st.completed += 1;
    else st.failed += 1;
    cv_done.notify_all();
}

void bldm_server::loop() {
    cudaSetDevice(device);
    bool rebuild = true;
    while (true) {
        std::vector<Request*> admitted;
        {
            std::unique_lock<std::mutex> lk(mu);
            if (active.empty() && queue.empty() && !stop)
                cv_work.wait_for(lk, std::chrono::milliseconds(20));
            if (stop) break;
            while (!queue.empty() && !free_slots.empty()) {
                Request* r = queue.front();
                if (r->cancel) {
                    queue.pop_front();
                    r->state = REQ_FAILED;
                    r->status = BLDM_ERR_NOT_FOUND;
                    r->t_done = Clock::now();
                    cv_done.notify_all();
                    continue;
                }
                size_t free_b = 0, total_b = 0;
                cudaMemGetInfo(&free_b, &total_b);
                if (used + r->dbytes > budget || r->dbytes + (64u << 20) > free_b) break;
                queue.pop_front();
                r->slot = free_slots.back();
                free_slots.pop_back();
                used += r->dbytes;
                if (used > peak) peak = used;
                r->state = REQ_ACTIVE;
                r->t_admit = Clock::now();
                admitted.push_back(r);
            }
        }
        for (Request* r : admitted) {
            const int rc = admit(r);
            if (rc) {
                retire(r, rc);
                continue;
            }
            active.push_back(r);
            n_active = active.size();
            rebuild = true;
        }
        if (active.empty()) continue;
        int rc = BLDM_OK;
        if (rebuild) {
            std::vector<EngineInstance*> ptrs;
            for (Request* r : active) ptrs.push_back(&r->inst);
            rc = eng->build(ptrs, stream);
            rebuild = false;
        }
        if (rc == BLDM_OK)
            rc = eng->run(cfg.iters_per_round, cfg.psi_mode, cfg.eps, false, stream);
        if (rc == BLDM_OK) rc = eng->check(stream);
        if (rc == BLDM_OK)
            rc = cuda_status(cudaMemcpy(h_rel.data(), d_rel, h_rel.size() * 8,
                                        cudaMemcpyDeviceToHost));
        {
            std::lock_guard<std::mutex> lk(mu);
            st.rounds += 1;
            st.iterations += cfg.iters_per_round * active.size();
        }
        std::vector<Request*> keep;
        for (Request* r : active) {
            if (rc != BLDM_OK) {
                retire(r, rc);
                continue;
            }
            r->iters += cfg.iters_per_round;
            r->rel = h_rel[r->slot];
            if (r->rel < cfg.tol || r->iters >= cfg.max_iter || r->cancel)
                retire(r, r->cancel ? BLDM_ERR_NOT_FOUND : BLDM_OK);
            else
                keep.push_back(r);
        }
        if (keep.size() != active.size()) rebuild = true;
        active.swap(keep);
        n_active = active.size();
    }
    for (Request* r : active) retire(r, BLDM_ERR_NOT_FOUND);
    active.clear();
    cudaStreamSynchronize(stream);
}

extern "C" {

int bldm_server_create(bldm_server** out, const bldm_server_config* cfg) {
    if (!out || !cfg) return BLDM_ERR_BAD_ARG;
    *out = nullptr;
    if (cfg->dtype != BLDM_F64 && cfg->dtype != BLDM_F32) return BLDM_ERR_BAD_ARG;
    if (cfg->psi_mode < BLDM_PSI_EXACT || cfg->psi_mode > BLDM_PSI_LEGACY_CUDA)
        return BLDM_ERR_BAD_ARG;
    if (cfg->iters_per_round == 0 || cfg->max_active == 0 || cfg->max_iter == 0)
        return BLDM_ERR_BAD_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return BLDM_ERR_NO_DEVICE;
    std::unique_ptr<bldm_server> s(new bldm_server());
    s->cfg = *cfg;
    cudaGetDevice(&s->device);
    s->eng.reset(new Engine(cfg->dtype, cfg->rows_per_tile));
    cudaError_t e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) return cuda_status(e);
    e = cudaMalloc(&s->d_rel, cfg->max_active * sizeof(double));
    if (e != cudaSuccess) return cuda_status(e);
    s->h_rel.assign(cfg->max_active, 1.0);
    for (size_t i = cfg->max_active; i > 0; --i) s->free_slots.push_back(int(i - 1));
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    s->budget = cfg->memory_budget ? cfg->memory_budget : size_t(0.8 * double(free_b));
    bldm_server* raw = s.get();
    s->worker = std::thread([raw] { raw->loop(); });
    *out = s.release();
    return BLDM_OK;
}

int bldm_server_destroy(bldm_server* s) {
    if (!s) return BLDM_ERR_BAD_ARG;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    if (s->worker.joinable()) s->worker.join();
    s->eng.reset();
    if (s->d_rel) cudaFree(s->d_rel);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
    return BLDM_OK;
}

int bldm_server_submit(bldm_server* s, const double* X, size_t x, size_t y, size_t z,
                       const bldm_params* p, uint64_t seed, uint64_t* id) {
    if (!s || !X || !p || !id || x == 0 || y == 0 || z == 0) return BLDM_ERR_BAD_ARG;
    if (p->n_alpha != x || p->n_beta != z || !p->alpha || !p->beta) return BLDM_ERR_BAD_ARG;
    for (size_t e = 0; e < x * y; ++e)
        if (!(X[e] >= 0.0)) return BLDM_ERR_NEG_X;
    std::unique_ptr<Request> r(new Request());
    int rc = s->eng->configure(r->inst, x, y, z);
    if (rc) return rc;
    r->dbytes = s->eng->bytes(r->inst).total(256);
    if (r->dbytes > s->budget) return BLDM_ERR_TOO_LARGE;
    r->x = x;
    r->y = y;
    r->z = z;
    r->X.assign(X, X + x * y);
    r->alpha.assign(p->alpha, p->alpha + x);
    r->beta.assign(p->beta, p->beta + z);
    r->a = p->a;
    r->b = p->b;
    r->seed = seed;
    r->t_submit = Clock::now();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        r->id = s->next_id++;
        *id = r->id;
        s->queue.push_back(r.get());
        s->reqs.emplace(r->id, std::move(r));
        s->st.submitted += 1;
    }
    s->cv_work.notify_all();
    return BLDM_OK;
}

int bldm_server_poll(bldm_server* s, uint64_t id, int* state) {
    if (!s || !state) return BLDM_ERR_BAD_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return BLDM_ERR_NOT_FOUND;
    *state = it->second->state;
    return BLDM_OK;
}

int bldm_server_wait(bldm_server* s, uint64_t id, double timeout_s) {
    if (!s) return BLDM_ERR_BAD_ARG;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return BLDM_ERR_NOT_FOUND;
    Request* r = it->second.get();
    const bool ok = s->cv_done.wait_for(
        lk, std::chrono::duration<double>(timeout_s),
        [r] { return r->state == REQ_DONE || r->state == REQ_FAILED; });
    return ok ? BLDM_OK : BLDM_ERR_BUSY;
}

int bldm_server_fetch(bldm_server* s, uint64_t id, double* S_out, bldm_request_stats* rs) {
    if (!s) return BLDM_ERR_BAD_ARG;
    std::unique_ptr<Request> r;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        auto it = s->reqs.find(id);
        if (it == s->reqs.end()) return BLDM_ERR_NOT_FOUND;
        if (it->second->state != REQ_DONE && it->second->state != REQ_FAILED)
            return BLDM_ERR_BUSY;
        r = std::move(it->second);
        s->reqs.erase(it);
    }
    if (rs) {
        rs->queue_ms = r->state == REQ_DONE ? ms_between(r->t_submit, r->t_admit) : 0.0;
        rs->latency_ms = ms_between(r->t_submit, r->t_done);
        rs->iterations = r->iters;
        rs->rel_change = r->rel;
        rs->log_marginal = r->log_marginal;
        rs->status = r->status;
    }
    if (r->state == REQ_DONE && S_out) std::memcpy(S_out, r->S.data(), r->S.size() * 8);
    return r->status;
}

int bldm_server_cancel(bldm_server* s, uint64_t id) {
    if (!s) return BLDM_ERR_BAD_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->reqs.find(id);
    if (it == s->reqs.end()) return BLDM_ERR_NOT_FOUND;
    it->second->cancel = true;
    s->cv_work.notify_all();
    return BLDM_OK;
}

int bldm_server_get_stats(bldm_server* s, bldm_server_stats* out) {
    if (!s || !out) return BLDM_ERR_BAD_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    *out = s->st;
    out->active = s->n_active.load();
    out->queued = s->queue.size();
    out->bytes_in_use = s->used;
    out->bytes_peak = s->peak;
    out->budget = s->budget;
    return BLDM_OK;
}

}  // extern "C"
