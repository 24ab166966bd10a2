// Serving loop: continuous batching of bld_mult requests (bldm_server_*).
//
// A worker thread owns the rounds.  Each round it admits queued requests
// while a request slot and device memory (the configured budget, checked
// against the device's free memory) are available: it allocates each admitted
// request's buffers stream-ordered, uploads X, draws the seeded initial S and
// computes the new requests' axis sums and digamma tables on their own (a
// small primer engine), so that the round's launches carry every other
// request's tables over from its previous round.  It then runs
// `iters_per_round` iterations of every active request in shared launches
// (the multi-instance engine) and hands the requests whose relative change of
// S fell below `tol`, or that reached `max_iter`, to a retirement thread.
// That thread waits for the round on its own stream, copies S to the host in
// the storage type, computes the log-marginal on the device in FP64 and frees
// the request's device memory, while the worker goes on with the next round.
// A request's tiling and its iteration count depend only on itself, so its
// result is the same alone and in any mix.
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdint>
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
    std::vector<double> X;   // FP64 storage: uploaded as is
    std::vector<float> Xf;   // FP32 storage: converted at submit (client thread)
    std::vector<double> alpha, beta;
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
    std::vector<double> S;   // result, FP64 storage
    std::vector<float> Sf;   // result, FP32 storage (converted by fetch)
    Clock::time_point t_submit, t_admit, t_done;
};

// Requests finished on the device after the round that `done` marks.
struct RetireBatch {
    std::vector<Request*> reqs;
    cudaEvent_t done = nullptr;
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
    std::unique_ptr<Engine> eng;     // every active request
    std::unique_ptr<Engine> primer;  // the requests admitted this round
    std::mutex mu;
    std::condition_variable cv_work, cv_done, cv_retire;
    std::deque<Request*> queue;
    std::unordered_map<uint64_t, std::unique_ptr<Request>> reqs;
    std::vector<Request*> active;  // worker thread only
    std::vector<int> free_slots;
    std::deque<RetireBatch> retire_q;
    size_t retiring = 0;
    double* d_rel = nullptr;
    std::vector<double> h_rel;
    size_t used = 0, peak = 0, budget = 0;
    uint64_t next_id = 1;
    bldm_server_stats st{};
    cudaStream_t stream = nullptr;   // rounds
    cudaStream_t rstream = nullptr;  // retirement
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::thread worker, retirer;
    bool stop = false, stop_retire = false;
    std::atomic<size_t> n_active{0};

    void loop();
    void retire_loop();
    int admit(Request* r);
    void finish(Request* r, int status);
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
    if (e == cudaSuccess)
        e = eng->es() == 8 ? cudaMemcpyAsync(r->inst.X, r->X.data(), r->x * r->y * 8,
                                             cudaMemcpyHostToDevice, stream)
                           : cudaMemcpyAsync(r->inst.X, r->Xf.data(), r->x * r->y * 4,
                                             cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(r->inst.alpha, r->alpha.data(), r->x * 8, cudaMemcpyHostToDevice,
                            stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(r->inst.beta, r->beta.data(), r->z * 8, cudaMemcpyHostToDevice,
                            stream);
    if (e != cudaSuccess) return cuda_status(e);
    rc = eng->set_row_lists(r->inst, stream);
    if (rc) return rc;
    return launch_init_S(eng->dtype(), r->inst.X, r->inst.S, (long long)(r->x * r->y),
                         (long long)r->z, r->seed, stream);
}

// Marks a request done or failed and releases its slot and budget.  Its
// device memory must already be freed (stream-ordered) by the caller.
void bldm_server::finish(Request* r, int status) {
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
    cv_work.notify_all();  // a slot and memory are free again
}

void bldm_server::retire_loop() {
    cudaSetDevice(device);
    while (true) {
        RetireBatch rb;
        {
            std::unique_lock<std::mutex> lk(mu);
            cv_retire.wait(lk, [this] { return stop_retire || !retire_q.empty(); });
            if (retire_q.empty()) break;  // stop_retire and nothing left
            rb = retire_q.front();
            retire_q.pop_front();
        }
        cudaError_t e = cudaStreamWaitEvent(rstream, rb.done, 0);
        for (Request* r : rb.reqs) {
            int status = cuda_status(e);
            const size_t n = r->x * r->y * r->z;
            if (status == BLDM_OK) {
                cudaError_t ce;
                if (eng->es() == 8) {
                    r->S.resize(n);
                    ce = cudaMemcpyAsync(r->S.data(), r->inst.S, n * 8, cudaMemcpyDeviceToHost,
                                         rstream);
                } else {
                    r->Sf.resize(n);
                    ce = cudaMemcpyAsync(r->Sf.data(), r->inst.S, n * 4, cudaMemcpyDeviceToHost,
                                         rstream);
                }
                status = cuda_status(ce);
            }
            if (status == BLDM_OK)
                status = bldm_log_marginal_S(r->inst.S, eng->dtype(), r->x, r->y, r->z,
                                             r->alpha.data(), r->beta.data(), r->a, r->b,
                                             &r->log_marginal, rstream);
            if (r->dmem) cudaFreeAsync(r->dmem, rstream);
            r->dmem = nullptr;
            if (status == BLDM_OK) status = cuda_status(cudaStreamSynchronize(rstream));
            {
                std::lock_guard<std::mutex> lk(mu);
                retiring -= 1;
            }
            finish(r, r->cancel ? BLDM_ERR_NOT_FOUND : status);
        }
        cudaEventDestroy(rb.done);
    }
}

void bldm_server::loop() {
    cudaSetDevice(device);
    bool rebuild = true;
    while (true) {
        std::vector<Request*> admitted;
        {
            std::unique_lock<std::mutex> lk(mu);
            if (active.empty() && !stop && (queue.empty() || free_slots.empty()))
                cv_work.wait_for(lk, std::chrono::milliseconds(20));
            if (stop) break;
            size_t free_b = 0, total_b = 0;
            bool have_free = false;
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
                if (!have_free) {
                    cudaMemGetInfo(&free_b, &total_b);
                    have_free = true;
                }
                if (used + r->dbytes > budget || r->dbytes + (64u << 20) > free_b) break;
                free_b -= r->dbytes;
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
        const Clock::time_point h0 = Clock::now();
        std::vector<Request*> fresh;
        for (Request* r : admitted) {
            const int rc = admit(r);
            if (rc) {
                if (r->dmem) cudaFreeAsync(r->dmem, stream);
                r->dmem = nullptr;
                finish(r, rc);
                continue;
            }
            fresh.push_back(r);
        }
        int rc = BLDM_OK;
        if (!fresh.empty()) {
            // axis sums and digamma tables of the new requests' initial S
            std::vector<EngineInstance*> ptrs;
            for (Request* r : fresh) ptrs.push_back(&r->inst);
            rc = primer->build(ptrs, stream);
            if (rc == BLDM_OK) rc = primer->prime(cfg.psi_mode, stream);
            for (Request* r : fresh) active.push_back(r);
            n_active = active.size();
            rebuild = true;
        }
        if (active.empty()) {
            // nothing admitted (memory still held by retiring requests): wait
            // for a retirement or a new request instead of polling
            std::unique_lock<std::mutex> lk(mu);
            if (!stop) cv_work.wait_for(lk, std::chrono::milliseconds(5));
            continue;
        }
        if (rc == BLDM_OK && rebuild) {
            std::vector<EngineInstance*> ptrs;
            for (Request* r : active) ptrs.push_back(&r->inst);
            rc = eng->build(ptrs, stream);
            rebuild = false;
        }
        const double host_ms = ms_between(h0, Clock::now());
        if (rc == BLDM_OK) rc = cuda_status(cudaEventRecord(ev0, stream));
        // requests admitted this round have not had an update yet
        if (rc == BLDM_OK)
            rc = eng->run(cfg.iters_per_round, cfg.psi_mode, cfg.eps, false, stream, false,
                          fresh.empty());
        if (rc == BLDM_OK) rc = cuda_status(cudaEventRecord(ev1, stream));
        if (rc == BLDM_OK) rc = eng->check(stream);
        if (rc == BLDM_OK)
            rc = cuda_status(cudaMemcpy(h_rel.data(), d_rel, h_rel.size() * 8,
                                        cudaMemcpyDeviceToHost));
        float gpu_ms = 0.f;
        if (rc == BLDM_OK) cudaEventElapsedTime(&gpu_ms, ev0, ev1);
        std::vector<Request*> keep, done;
        for (Request* r : active) {
            if (rc != BLDM_OK) {
                if (r->dmem) cudaFreeAsync(r->dmem, stream);
                r->dmem = nullptr;
                finish(r, rc);
                continue;
            }
            r->iters += cfg.iters_per_round;
            r->rel = h_rel[r->slot];
            if (r->rel < cfg.tol || r->iters >= cfg.max_iter || r->cancel)
                done.push_back(r);
            else
                keep.push_back(r);
        }
        {
            std::lock_guard<std::mutex> lk(mu);
            st.rounds += 1;
            st.iterations += cfg.iters_per_round * active.size();
            st.gpu_ms += gpu_ms;
            st.host_ms += host_ms;
        }
        if (!done.empty()) {
            RetireBatch rb;
            rb.reqs = done;
            cudaError_t e = cudaEventCreateWithFlags(&rb.done, cudaEventDisableTiming);
            if (e == cudaSuccess) e = cudaEventRecord(rb.done, stream);
            if (e != cudaSuccess) {
                for (Request* r : done) {
                    if (r->dmem) cudaFreeAsync(r->dmem, stream);
                    r->dmem = nullptr;
                    finish(r, cuda_status(e));
                }
            } else {
                std::lock_guard<std::mutex> lk(mu);
                retire_q.push_back(rb);
                retiring += done.size();
                cv_retire.notify_all();
            }
        }
        if (keep.size() != active.size()) rebuild = true;
        active.swap(keep);
        n_active = active.size();
    }
    for (Request* r : active) {
        if (r->dmem) cudaFreeAsync(r->dmem, stream);
        r->dmem = nullptr;
        finish(r, BLDM_ERR_NOT_FOUND);
    }
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
    s->primer.reset(new Engine(cfg->dtype, cfg->rows_per_tile));
    cudaError_t e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->rstream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&s->ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&s->ev1);
    if (e == cudaSuccess) e = cudaMalloc(&s->d_rel, cfg->max_active * sizeof(double));
    if (e != cudaSuccess) {
        if (s->d_rel) cudaFree(s->d_rel);
        if (s->ev0) cudaEventDestroy(s->ev0);
        if (s->ev1) cudaEventDestroy(s->ev1);
        if (s->rstream) cudaStreamDestroy(s->rstream);
        if (s->stream) cudaStreamDestroy(s->stream);
        return cuda_status(e);
    }
    // Keep freed request memory in the device's stream-ordered pool instead of
    // returning it at every synchronisation: admissions reuse it without new
    // mappings.
    cudaMemPool_t pool = nullptr;
    if (cudaDeviceGetDefaultMemPool(&pool, s->device) == cudaSuccess) {
        uint64_t keep = UINT64_MAX;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    s->h_rel.assign(cfg->max_active, 1.0);
    for (size_t i = cfg->max_active; i > 0; --i) s->free_slots.push_back(int(i - 1));
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    s->budget = cfg->memory_budget ? cfg->memory_budget : size_t(0.8 * double(free_b));
    bldm_server* raw = s.get();
    s->worker = std::thread([raw] { raw->loop(); });
    s->retirer = std::thread([raw] { raw->retire_loop(); });
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
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop_retire = true;
    }
    s->cv_retire.notify_all();
    if (s->retirer.joinable()) s->retirer.join();
    s->eng.reset();
    s->primer.reset();
    cudaStreamSynchronize(s->rstream);
    if (s->d_rel) cudaFree(s->d_rel);
    if (s->ev0) cudaEventDestroy(s->ev0);
    if (s->ev1) cudaEventDestroy(s->ev1);
    if (s->rstream) cudaStreamDestroy(s->rstream);
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
    if (s->cfg.dtype == BLDM_F64)
        r->X.assign(X, X + x * y);
    else
        r->Xf.assign(X, X + x * y);
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
    if (r->state == REQ_DONE && S_out) {
        if (!r->S.empty())
            std::memcpy(S_out, r->S.data(), r->S.size() * 8);
        else
            for (size_t i = 0; i < r->Sf.size(); ++i) S_out[i] = r->Sf[i];
    }
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
    out->retiring = s->retiring;
    return BLDM_OK;
}

}  // extern "C"
