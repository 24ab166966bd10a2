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
// That thread (one per lane) waits for the round on its own high-priority
// stream, copies S to the host in the storage type, computes the log-marginal
// on the device in FP64 and frees the request's device memory, while the
// worker goes on with the next round.
// A request's tiling and its iteration count depend only on itself, so its
// result is the same alone and in any mix.
//
// Requests of at least `large_elements` S elements are served in a second
// lane: its own worker, engines and a lower-priority stream.  A round of
// small requests then does not last as long as a round of a large one (a
// 4096x4096x32 iteration takes about a millisecond, a round of the small ones
// a fraction of that), and each lane's host work (admission, launch tables,
// reading the convergence values) overlaps the other lane's kernels.
#include <algorithm>
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
    int lane = 0;
    size_t iters = 0;
    double rel = 1.0;
    double log_marginal = 0.0;
    double conservation = 0.0;
    // result in the storage type (fetch converts FP32 to FP64); left
    // uninitialised until the copy fills it (a zero fill of a GiB-sized result
    // would cost as much as the copy)
    std::unique_ptr<double[]> S;
    std::unique_ptr<float[]> Sf;
    size_t n_out = 0;
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

// One worker's share of the server: small requests in lane 0, large ones in
// lane 1.
struct Lane {
    std::unique_ptr<Engine> eng;     // every active request of the lane
    std::unique_ptr<Engine> primer;  // the requests admitted this round
    std::deque<Request*> queue;      // guarded by bldm_server::mu
    std::vector<Request*> active;    // the lane's worker only
    std::vector<double> h_rel;       // the lane's copy of the convergence values
    cudaStream_t stream = nullptr;   // the lane's rounds
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::thread worker;
    // the lane's retirement: its own thread and stream, so that the results of
    // small requests never wait behind a large one's copy
    std::deque<RetireBatch> retire_q;  // guarded by bldm_server::mu
    cudaStream_t rstream = nullptr;
    std::thread retirer;
    std::atomic<size_t> n_active{0};
    // Results leave the device through two pinned staging buffers: a pageable
    // copy of a large result would fault its pages in inside the driver and
    // hold up the other threads' CUDA calls meanwhile.
    void* pin[2] = {nullptr, nullptr};
    cudaEvent_t pin_ev[2] = {nullptr, nullptr};

    int copy_out(void* dst, const void* src, size_t bytes);
};

// Copies `bytes` of device memory to pageable host memory in chunks through
// the staging buffers; the copy of chunk c+1 overlaps the host copy of c.
constexpr size_t kPinBytes = size_t(32) << 20;
int Lane::copy_out(void* dst, const void* src, size_t bytes) {
    const size_t nch = (bytes + kPinBytes - 1) / kPinBytes;
    auto issue = [&](size_t c) {
        const size_t off = c * kPinBytes;
        const size_t len = std::min(kPinBytes, bytes - off);
        cudaError_t e = cudaMemcpyAsync(pin[c & 1], static_cast<const char*>(src) + off, len,
                                        cudaMemcpyDeviceToHost, rstream);
        if (e == cudaSuccess) e = cudaEventRecord(pin_ev[c & 1], rstream);
        return e;
    };
    cudaError_t e = nch ? issue(0) : cudaSuccess;
    for (size_t c = 0; c < nch && e == cudaSuccess; ++c) {
        if (c + 1 < nch) e = issue(c + 1);
        if (e == cudaSuccess) e = cudaEventSynchronize(pin_ev[c & 1]);
        if (e == cudaSuccess) {
            const size_t off = c * kPinBytes;
            std::memcpy(static_cast<char*>(dst) + off, pin[c & 1],
                        std::min(kPinBytes, bytes - off));
        }
    }
    return cuda_status(e);
}

struct bldm_server {
    bldm_server_config cfg{};
    int device = 0;
    size_t large_elems = 0;  // lane 1 from this many S elements on
    Lane lanes[2];
    std::mutex mu;
    std::condition_variable cv_work, cv_done, cv_retire;
    std::unordered_map<uint64_t, std::unique_ptr<Request>> reqs;
    std::vector<int> free_slots;
    size_t retiring = 0;
    double* d_rel = nullptr;  // [max_active] by slot
    unsigned long long* d_cons = nullptr;  // [2] conservation residual bits, by lane
    size_t used = 0, peak = 0, budget = 0;
    uint64_t next_id = 1;
    bldm_server_stats st{};
    bool stop = false, stop_retire = false;

    void loop(int lane);
    void retire_loop(int lane);
    int admit(Lane& L, Request* r);
    void finish(Request* r, int status);
    int es() const { return cfg.dtype == BLDM_F64 ? 8 : 4; }
};

int bldm_server::admit(Lane& L, Request* r) {
    Engine* eng = L.eng.get();
    cudaStream_t stream = L.stream;
    int rc = eng->configure(r->inst, r->x, r->y, r->z);
    if (rc) return rc;
    cudaError_t e = cudaMallocAsync(&r->dmem, r->dbytes, stream);
    if (e != cudaSuccess) {
        r->dmem = nullptr;
        return cuda_status(e);
    }
    eng->bind(r->inst, r->dmem);
    r->inst.rel = d_rel + r->slot;
    e = cudaMemsetAsync(r->inst.counter, 0, eng->bytes(r->inst).counter, stream);
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

void bldm_server::retire_loop(int lane) {
    cudaSetDevice(device);
    std::deque<RetireBatch>& retire_q = lanes[lane].retire_q;
    cudaStream_t rstream = lanes[lane].rstream;
    while (true) {
        RetireBatch rb;
        {
            std::unique_lock<std::mutex> lk(mu);
            cv_retire.wait(lk, [&] { return stop_retire || !retire_q.empty(); });
            if (retire_q.empty()) break;  // stop_retire and nothing left
            rb = retire_q.front();
            retire_q.pop_front();
        }
        const Clock::time_point r0 = Clock::now();
        cudaError_t e = cudaStreamWaitEvent(rstream, rb.done, 0);
        for (Request* r : rb.reqs) {
            int status = cuda_status(e);
            const size_t n = r->x * r->y * r->z;
            if (status == BLDM_OK) {
                r->n_out = n;
                if (es() == 8) {
                    r->S.reset(new double[n]);
                    status = lanes[lane].copy_out(r->S.get(), r->inst.S, n * 8);
                } else {
                    r->Sf.reset(new float[n]);
                    status = lanes[lane].copy_out(r->Sf.get(), r->inst.S, n * 4);
                }
            }
            unsigned long long cons_bits = 0;
            if (status == BLDM_OK)
                status = cuda_status(cudaMemsetAsync(d_cons + lane, 0, 8, rstream));
            if (status == BLDM_OK)
                status = launch_conservation(cfg.dtype, r->inst.X, r->inst.S,
                                             (long long)(r->x * r->y), (long long)r->z,
                                             d_cons + lane, rstream);
            if (status == BLDM_OK)
                status = cuda_status(cudaMemcpyAsync(&cons_bits, d_cons + lane, 8,
                                                     cudaMemcpyDeviceToHost, rstream));
            if (status == BLDM_OK)
                status = bldm_log_marginal_S(r->inst.S, cfg.dtype, r->x, r->y, r->z,
                                             r->alpha.data(), r->beta.data(), r->a, r->b,
                                             &r->log_marginal, rstream);
            if (r->dmem) cudaFreeAsync(r->dmem, rstream);
            r->dmem = nullptr;
            if (status == BLDM_OK) status = cuda_status(cudaStreamSynchronize(rstream));
            if (status == BLDM_OK) r->conservation = cons_value(cons_bits);
            {
                std::lock_guard<std::mutex> lk(mu);
                retiring -= 1;
            }
            finish(r, r->cancel ? BLDM_ERR_NOT_FOUND : status);
        }
        cudaEventDestroy(rb.done);
        {
            std::lock_guard<std::mutex> lk(mu);
            st.retire_ms += ms_between(r0, Clock::now());
        }
    }
}

void bldm_server::loop(int lane) {
    cudaSetDevice(device);
    Lane& L = lanes[lane];
    Engine* eng = L.eng.get();
    Engine* primer = L.primer.get();
    cudaStream_t stream = L.stream;
    std::deque<Request*>& queue = L.queue;
    std::vector<Request*>& active = L.active;
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
            const int rc = admit(L, r);
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
            L.n_active = active.size();
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
        if (rc == BLDM_OK) rc = cuda_status(cudaEventRecord(L.ev0, stream));
        // requests admitted this round have not had an update yet
        if (rc == BLDM_OK)
            rc = eng->run(cfg.iters_per_round, cfg.psi_mode, cfg.eps, false, stream, false,
                          fresh.empty());
        if (rc == BLDM_OK) rc = cuda_status(cudaEventRecord(L.ev1, stream));
        // the whole array (the other lane's entries are read and ignored); the
        // check below waits for the stream
        if (rc == BLDM_OK)
            rc = cuda_status(cudaMemcpyAsync(L.h_rel.data(), d_rel, L.h_rel.size() * 8,
                                             cudaMemcpyDeviceToHost, stream));
        if (rc == BLDM_OK) rc = eng->check(stream);
        float gpu_ms = 0.f;
        if (rc == BLDM_OK) cudaEventElapsedTime(&gpu_ms, L.ev0, L.ev1);
        std::vector<Request*> keep, done;
        for (Request* r : active) {
            if (rc != BLDM_OK) {
                if (r->dmem) cudaFreeAsync(r->dmem, stream);
                r->dmem = nullptr;
                finish(r, rc);
                continue;
            }
            r->iters += cfg.iters_per_round;
            r->rel = L.h_rel[r->slot];
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
            if (lane == 1) st.gpu_ms_large += gpu_ms;
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
                L.retire_q.push_back(rb);
                retiring += done.size();
                cv_retire.notify_all();
            }
        }
        if (keep.size() != active.size()) rebuild = true;
        active.swap(keep);
        L.n_active = active.size();
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
    s->large_elems = cfg->large_elements ? cfg->large_elements : (size_t(1) << 25);
    cudaGetDevice(&s->device);
    // small requests' rounds first when both lanes have work waiting; the
    // retirement's copies and log-marginal kernels (short, and on every
    // request's latency) ahead of both
    int prio_low = 0, prio_high = 0;
    cudaDeviceGetStreamPriorityRange(&prio_low, &prio_high);
    cudaError_t e = cudaSuccess;
    for (int l = 0; l < 2 && e == cudaSuccess; ++l) {
        Lane& L = s->lanes[l];
        L.eng.reset(new Engine(cfg->dtype, cfg->rows_per_tile));
        L.primer.reset(new Engine(cfg->dtype, cfg->rows_per_tile));
        // the worker launches each round directly (its set of requests changes
        // from round to round): the joined form's fewer launches
        L.eng->set_per_class_rounds(false);
        L.primer->set_per_class_rounds(false);
        L.h_rel.assign(cfg->max_active, 1.0);
        e = cudaStreamCreateWithPriority(&L.stream, cudaStreamNonBlocking,
                                         l == 0 ? prio_high : prio_low);
        if (e == cudaSuccess)
            e = cudaStreamCreateWithPriority(&L.rstream, cudaStreamNonBlocking, prio_high);
        for (int b = 0; b < 2 && e == cudaSuccess; ++b) {
            e = cudaHostAlloc(&L.pin[b], kPinBytes, cudaHostAllocDefault);
            if (e == cudaSuccess)
                e = cudaEventCreateWithFlags(&L.pin_ev[b], cudaEventDisableTiming);
        }
        if (e == cudaSuccess) e = cudaEventCreate(&L.ev0);
        if (e == cudaSuccess) e = cudaEventCreate(&L.ev1);
    }
    if (e == cudaSuccess) e = cudaMalloc(&s->d_rel, cfg->max_active * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&s->d_cons, 2 * sizeof(unsigned long long));
    if (e != cudaSuccess) {
        if (s->d_rel) cudaFree(s->d_rel);
        if (s->d_cons) cudaFree(s->d_cons);
        for (Lane& L : s->lanes) {
            if (L.ev0) cudaEventDestroy(L.ev0);
            if (L.ev1) cudaEventDestroy(L.ev1);
            if (L.stream) cudaStreamDestroy(L.stream);
            if (L.rstream) cudaStreamDestroy(L.rstream);
            for (int b = 0; b < 2; ++b) {
                if (L.pin[b]) cudaFreeHost(L.pin[b]);
                if (L.pin_ev[b]) cudaEventDestroy(L.pin_ev[b]);
            }
        }
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
    for (size_t i = cfg->max_active; i > 0; --i) s->free_slots.push_back(int(i - 1));
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    s->budget = cfg->memory_budget ? cfg->memory_budget : size_t(0.8 * double(free_b));
    bldm_server* raw = s.get();
    for (int l = 0; l < 2; ++l) {
        s->lanes[l].worker = std::thread([raw, l] { raw->loop(l); });
        s->lanes[l].retirer = std::thread([raw, l] { raw->retire_loop(l); });
    }
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
    for (Lane& L : s->lanes)
        if (L.worker.joinable()) L.worker.join();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop_retire = true;
    }
    s->cv_retire.notify_all();
    for (Lane& L : s->lanes) {
        if (L.retirer.joinable()) L.retirer.join();
        cudaStreamSynchronize(L.rstream);
    }
    for (Lane& L : s->lanes) {
        L.eng.reset();
        L.primer.reset();
        if (L.ev0) cudaEventDestroy(L.ev0);
        if (L.ev1) cudaEventDestroy(L.ev1);
        if (L.stream) cudaStreamDestroy(L.stream);
        if (L.rstream) cudaStreamDestroy(L.rstream);
        for (int b = 0; b < 2; ++b) {
            if (L.pin[b]) cudaFreeHost(L.pin[b]);
            if (L.pin_ev[b]) cudaEventDestroy(L.pin_ev[b]);
        }
    }
    if (s->d_rel) cudaFree(s->d_rel);
    if (s->d_cons) cudaFree(s->d_cons);
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
    int rc = s->lanes[0].eng->configure(r->inst, x, y, z);
    if (rc) return rc;
    r->dbytes = s->lanes[0].eng->bytes(r->inst).total(256);
    if (r->dbytes > s->budget) return BLDM_ERR_TOO_LARGE;
    r->x = x;
    r->y = y;
    r->z = z;
    r->lane = x * y * z >= s->large_elems ? 1 : 0;
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
        s->lanes[r->lane].queue.push_back(r.get());
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
        rs->conservation_residual = r->conservation;
        rs->status = r->status;
    }
    if (r->state == REQ_DONE && S_out) {
        if (r->S)
            std::memcpy(S_out, r->S.get(), r->n_out * 8);
        else if (r->Sf)
            for (size_t i = 0; i < r->n_out; ++i) S_out[i] = r->Sf[i];
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
    out->active = s->lanes[0].n_active.load() + s->lanes[1].n_active.load();
    out->queued = s->lanes[0].queue.size() + s->lanes[1].queue.size();
    out->bytes_in_use = s->used;
    out->bytes_peak = s->peak;
    out->budget = s->budget;
    out->retiring = s->retiring;
    return BLDM_OK;
}

}  // extern "C"
