// C ABI of the batched solver: many independent bld_mult instances of
// different shapes solved together (bldm_batch_*).  The reference solves one
// instance per call (bld::bld_mult_cuda, src/bld/bld_mult/bld_mult.hpp:225-324);
// a batch runs the same iterations for all its instances in shared launches.
#include <algorithm>
#include <cstring>
#include <map>
#include <memory>
#include <vector>

#include "bldm_engine.h"

using namespace bldm;

struct bldm_batch {
    std::unique_ptr<Engine> eng;
    std::vector<EngineInstance> inst;
    std::vector<EngineInstance*> ptrs;
    void* arena = nullptr;
    size_t arena_bytes = 0;
    int dtype = BLDM_F64;
    bool clean = false;  // every instance has been updated since its S was set
    bool reorder = false;  // an X was set since the last build: re-sort the tiles
    void* cons_buf = nullptr;  // conservation: ConsInst[n] | block_off[n+1] | residual bits[n]
    ~bldm_batch() {
        eng.reset();
        if (arena) cudaFree(arena);
        if (cons_buf) cudaFree(cons_buf);
    }
};

namespace {

template <typename T>
int upload(const double* src, size_t n, void* dst) {
    if (sizeof(T) == 8) return cuda_status(cudaMemcpy(dst, src, n * 8, cudaMemcpyHostToDevice));
    std::vector<float> tmp(src, src + n);
    return cuda_status(cudaMemcpy(dst, tmp.data(), n * 4, cudaMemcpyHostToDevice));
}

template <typename T>
int download(const void* src, size_t n, double* dst) {
    if (sizeof(T) == 8) return cuda_status(cudaMemcpy(dst, src, n * 8, cudaMemcpyDeviceToHost));
    std::vector<float> tmp(n);
    const int rc = cuda_status(cudaMemcpy(tmp.data(), src, n * 4, cudaMemcpyDeviceToHost));
    for (size_t i = 0; i < n; ++i) dst[i] = tmp[i];
    return rc;
}

// Re-tiles every instance from the engine's class tunings and rebuilds.
int rebuild(bldm_batch* b, cudaStream_t st) {
    for (auto& in : b->inst) b->eng->retile(in);
    const int rc = b->eng->build(b->ptrs, st);
    if (rc == BLDM_OK) b->reorder = false;
    return rc;
}

}  // namespace

extern "C" {

int bldm_batch_create(bldm_batch** out, int dtype, size_t n, const size_t* xs, const size_t* ys,
                      const size_t* zs, int rows_per_tile) {
    if (!out || n == 0 || !xs || !ys || !zs) return BLDM_ERR_BAD_ARG;
    *out = nullptr;
    if (dtype != BLDM_F64 && dtype != BLDM_F32) return BLDM_ERR_BAD_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return BLDM_ERR_NO_DEVICE;
    std::unique_ptr<bldm_batch> b(new bldm_batch());
    b->dtype = dtype;
    b->eng.reset(new Engine(dtype, rows_per_tile));
    b->inst.resize(n);
    std::vector<size_t> off(n);
    size_t total = 0;
    for (size_t i = 0; i < n; ++i) {
        const int rc = b->eng->configure(b->inst[i], xs[i], ys[i], zs[i]);
        if (rc) return rc;
        off[i] = total;
        total += b->eng->bytes(b->inst[i]).total(256);
    }
    cudaError_t e = cudaMalloc(&b->arena, total);
    if (e != cudaSuccess) {
        b->arena = nullptr;
        return cuda_status(e);
    }
    b->arena_bytes = total;
    b->ptrs.resize(n);
    for (size_t i = 0; i < n; ++i) {
        b->eng->bind(b->inst[i], static_cast<char*>(b->arena) + off[i]);
        b->ptrs[i] = &b->inst[i];
    }
    for (size_t i = 0; i < n; ++i) {
        e = cudaMemset(b->inst[i].counter, 0, b->eng->bytes(b->inst[i]).counter);
        // empty row lists until bldm_batch_set fills them from X
        if (e == cudaSuccess)
            e = cudaMemset(b->inst[i].nz_cnt, 0, b->eng->bytes(b->inst[i]).nzc);
        if (e != cudaSuccess) return cuda_status(e);
    }
    int rc = b->eng->build(b->ptrs, nullptr);
    if (rc) return rc;
    rc = cuda_status(cudaDeviceSynchronize());
    if (rc) return rc;
    *out = b.release();
    return BLDM_OK;
}

int bldm_batch_destroy(bldm_batch* b) {
    if (!b) return BLDM_ERR_BAD_ARG;
    delete b;
    return BLDM_OK;
}

int bldm_batch_set(bldm_batch* b, size_t idx, const double* X, const double* alpha,
                   const double* beta, const double* S0, uint64_t seed) {
    if (!b || idx >= b->inst.size() || !X || !alpha || !beta) return BLDM_ERR_BAD_ARG;
    EngineInstance& in = b->inst[idx];
    for (size_t e = 0; e < in.x * in.y; ++e)
        if (!(X[e] >= 0.0)) return BLDM_ERR_NEG_X;
    const bool f64 = b->dtype == BLDM_F64;
    b->clean = false;
    int rc = f64 ? upload<double>(X, in.x * in.y, in.X) : upload<float>(X, in.x * in.y, in.X);
    if (rc) return rc;
    rc = b->eng->set_row_lists(in, nullptr);
    if (rc) return rc;
    b->eng->set_work(in, X, true);
    b->reorder = true;
    rc = cuda_status(cudaMemcpy(in.alpha, alpha, in.x * 8, cudaMemcpyHostToDevice));
    if (rc) return rc;
    rc = cuda_status(cudaMemcpy(in.beta, beta, in.z * 8, cudaMemcpyHostToDevice));
    if (rc) return rc;
    const size_t ns = in.x * in.y * in.z;
    if (S0) {
        rc = f64 ? upload<double>(S0, ns, in.S) : upload<float>(S0, ns, in.S);
        if (rc) return rc;
        return cuda_status(cudaDeviceSynchronize());
    }
    rc = launch_init_S(b->dtype, in.X, in.S, (long long)(in.x * in.y), (long long)in.z, seed,
                       nullptr);
    if (rc) return rc;
    return cuda_status(cudaDeviceSynchronize());
}

int bldm_batch_run(bldm_batch* b, size_t iters, int psi_mode, double eps, int use_graph,
                   void* stream) {
    if (!b) return BLDM_ERR_BAD_ARG;
    if (b->reorder) {
        // the tiles in the order of the work estimates of the X values set
        const int rr = rebuild(b, static_cast<cudaStream_t>(stream));
        if (rr) return rr;
    }
    const int rc = b->eng->run(iters, psi_mode, eps, use_graph != 0,
                               static_cast<cudaStream_t>(stream), true, b->clean);
    if (rc == BLDM_OK && iters > 0) b->clean = true;
    return rc;
}

int bldm_batch_set_launch_mode(bldm_batch* b, int persistent, double wait_limit_s,
                               int stall_test) {
    if (!b || !(wait_limit_s > 0.0) || wait_limit_s > 60.0) return BLDM_ERR_BAD_ARG;
    b->eng->set_persistent(persistent != 0, (unsigned long long)(wait_limit_s * 1e9),
                           stall_test != 0);
    return BLDM_OK;
}

int bldm_batch_get_launch_mode(const bldm_batch* b, int* persistent) {
    if (!b || !persistent) return BLDM_ERR_BAD_ARG;
    *persistent = b->eng->persistent_active() ? 1 : 0;
    return BLDM_OK;
}

int bldm_batch_check(bldm_batch* b, void* stream) {
    if (!b) return BLDM_ERR_BAD_ARG;
    return b->eng->check(static_cast<cudaStream_t>(stream));
}

int bldm_batch_get(bldm_batch* b, size_t idx, double* S_out, double* rel_change) {
    if (!b || idx >= b->inst.size()) return BLDM_ERR_BAD_ARG;
    EngineInstance& in = b->inst[idx];
    int rc = BLDM_OK;
    if (S_out) {
        const size_t ns = in.x * in.y * in.z;
        rc = b->dtype == BLDM_F64 ? download<double>(in.S, ns, S_out)
                                  : download<float>(in.S, ns, S_out);
        if (rc) return rc;
    }
    if (rel_change) rc = cuda_status(cudaMemcpy(rel_change, in.rel, 8, cudaMemcpyDeviceToHost));
    return rc;
}

int bldm_batch_conservation(bldm_batch* b, double* residuals, void* stream) {
    if (!b || !residuals) return BLDM_ERR_BAD_ARG;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t n = b->inst.size();
    const size_t o_off = (n * sizeof(ConsInst) + 255) / 256 * 256;
    const size_t o_out = (o_off + (n + 1) * sizeof(int) + 255) / 256 * 256;
    const size_t bytes = o_out + n * sizeof(unsigned long long);
    if (!b->cons_buf) {
        const cudaError_t e = cudaMalloc(&b->cons_buf, bytes);
        if (e != cudaSuccess) {
            b->cons_buf = nullptr;
            return cuda_status(e);
        }
    }
    char* base = static_cast<char*>(b->cons_buf);
    unsigned long long* d_out = reinterpret_cast<unsigned long long*>(base + o_out);
    std::vector<char> host(bytes, 0);
    ConsInst* ci = reinterpret_cast<ConsInst*>(host.data());
    int* boff = reinterpret_cast<int*>(host.data() + o_off);
    int blocks = 0;
    for (size_t i = 0; i < n; ++i) {
        const EngineInstance& in = b->inst[i];
        ci[i] = cons_inst(b->dtype, in.X, in.S, (long long)(in.x * in.y), (long long)in.z,
                          d_out + i);
        boff[i] = blocks;
        blocks += conservation_blocks(b->dtype, in.S, (long long)(in.x * in.y), (long long)in.z);
    }
    boff[n] = blocks;
    int rc = cuda_status(cudaMemcpyAsync(base, host.data(), bytes, cudaMemcpyHostToDevice, st));
    if (rc) return rc;
    rc = launch_conservation_multi(b->dtype, reinterpret_cast<const ConsInst*>(base),
                                   reinterpret_cast<const int*>(base + o_off), int(n), blocks, st);
    if (rc) return rc;
    std::vector<unsigned long long> bits(n);
    rc = cuda_status(cudaMemcpyAsync(bits.data(), d_out, n * sizeof(unsigned long long),
                                     cudaMemcpyDeviceToHost, st));
    if (rc) return rc;
    rc = cuda_status(cudaStreamSynchronize(st));
    if (rc) return rc;
    for (size_t i = 0; i < n; ++i) residuals[i] = cons_value(bits[i]);
    return BLDM_OK;
}

int bldm_batch_device_ptrs(bldm_batch* b, size_t idx, void** d_X, void** d_S) {
    if (!b || idx >= b->inst.size()) return BLDM_ERR_BAD_ARG;
    if (d_X) *d_X = b->inst[idx].X;
    if (d_S) *d_S = b->inst[idx].S;
    return BLDM_OK;
}

int bldm_batch_class_info(const bldm_batch* b, size_t idx, bldm_batch_class* out) {
    if (!b || !out) return BLDM_ERR_BAD_ARG;
    ClassKey k;
    ClassTune t;
    size_t tiles = 0;
    if (!b->eng->class_info(idx, &k, &t, &tiles)) return BLDM_ERR_BAD_ARG;
    out->vec = k.vec;
    out->lanes_per_fiber = k.lpf;
    out->chunks = k.mch;
    out->multirow = k.multirow ? 1 : 0;
    out->rows_per_tile = t.rows_per_tile;
    out->stages = t.stages;
    out->tiles = tiles;
    out->instances = 0;
    for (const auto& in : b->inst)
        if (Engine::key_of(in) == k) ++out->instances;
    return BLDM_OK;
}

int bldm_batch_set_class(bldm_batch* b, const bldm_batch_class* c) {
    if (!b || !c) return BLDM_ERR_BAD_ARG;
    if ((c->rows_per_tile != 0 && c->rows_per_tile < kMinTileRows) || c->stages < 0 ||
        c->stages == 1)
        return BLDM_ERR_BAD_ARG;
    ClassTune t;
    t.rows_per_tile = c->rows_per_tile;
    t.stages = c->stages;
    b->eng->set_tune(ClassKey{c->vec, c->lanes_per_fiber, c->chunks, c->multirow != 0}, t);
    return rebuild(b, nullptr);
}

int bldm_batch_autotune(bldm_batch* b, size_t probe_iters, int psi_mode, double eps,
                        void* stream, double* default_ms, double* tuned_ms) {
    if (!b || probe_iters == 0) return BLDM_ERR_BAD_ARG;
    if (psi_mode < BLDM_PSI_EXACT || psi_mode > BLDM_PSI_LEGACY_CUDA) return BLDM_ERR_BAD_ARG;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const size_t es = b->dtype == BLDM_F64 ? 8 : 4;
    // Save S: the caller's S is restored at the end.  The probes time the steady
    // state of a run: from the S after one update (which has stored the zeros
    // of the fibers with X == 0), with the zero-row skipping of the later
    // iterations from the first probe iteration on, as in the bulk of a long run.
    size_t sbytes = 0;
    for (const auto& in : b->inst) sbytes += in.x * in.y * in.z * es;
    void* save = nullptr;
    int rc = cuda_status(cudaMalloc(&save, 2 * sbytes));
    if (rc) return rc;
    void* start = static_cast<char*>(save) + sbytes;
    auto copy_S = [&](void* buf, bool to_buf) -> int {
        size_t off = 0;
        for (const auto& in : b->inst) {
            const size_t nb = in.x * in.y * in.z * es;
            char* sv = static_cast<char*>(buf) + off;
            const cudaError_t e =
                to_buf ? cudaMemcpyAsync(sv, in.S, nb, cudaMemcpyDeviceToDevice, st)
                       : cudaMemcpyAsync(in.S, sv, nb, cudaMemcpyDeviceToDevice, st);
            if (e != cudaSuccess) return cuda_status(e);
            off += nb;
        }
        return BLDM_OK;
    };
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    // Probe time of the current tunings; a configuration that does not fit
    // (shared memory, ring too shallow for a multi-row stage) reports
    // BLDM_ERR_UNSUPPORTED and is skipped.
    auto probe = [&](double* ms) -> int {
        int r = rebuild(b, st);
        if (r) return r;
        double best = 1e300;
        for (int rep = 0; rep < 3; ++rep) {
            r = copy_S(start, false);
            if (r) return r;
            cudaEventRecord(e0, st);
            r = b->eng->run(probe_iters, psi_mode, eps, false, st, true, true);
            if (r) return r;
            cudaEventRecord(e1, st);
            r = b->eng->check(st);
            if (r) return r;
            float t = 0.f;
            cudaEventElapsedTime(&t, e0, e1);
            best = std::min(best, double(t));
        }
        *ms = best;
        return BLDM_OK;
    };
    // Classes by S elements, largest first, with their largest row count.
    std::map<ClassKey, std::pair<size_t, size_t>> cls;  // key -> (elements, max x)
    for (const auto& in : b->inst) {
        auto& c = cls[Engine::key_of(in)];
        c.first += in.x * in.y * in.z;
        c.second = std::max(c.second, in.x);
    }
    std::vector<std::pair<ClassKey, std::pair<size_t, size_t>>> order(cls.begin(), cls.end());
    std::stable_sort(order.begin(), order.end(),
                     [](const auto& a, const auto& c) { return a.second.first > c.second.first; });
    rc = copy_S(save, true);
    if (!rc) rc = b->eng->run(1, psi_mode, eps, false, st);
    if (!rc) rc = b->eng->check(st);
    if (!rc) rc = copy_S(start, true);
    double best = 0.0;
    if (!rc) rc = probe(&best);
    if (!rc && default_ms) *default_ms = best;
    for (size_t ci = 0; !rc && ci < order.size(); ++ci) {
        const ClassKey key = order[ci].first;
        const size_t xmax = order[ci].second.second;
        ClassTune cur = b->eng->tune_of(key);
        for (int R : {32, 64, 128, 256, 512}) {
            // tile heights at or above every instance's row count tile alike
            if (R == cur.rows_per_tile || (size_t(R) >= xmax && size_t(cur.rows_per_tile) >= xmax))
                continue;
            b->eng->set_tune(key, ClassTune{R, cur.stages});
            double ms = 0.0;
            const int r = probe(&ms);
            if (r == BLDM_ERR_UNSUPPORTED) continue;
            if (r) {
                rc = r;
                break;
            }
            if (ms < 0.97 * best) {
                best = ms;
                cur.rows_per_tile = R;
            }
        }
        b->eng->set_tune(key, cur);
        for (int S : {2, 3, 4, 6, 8}) {
            if (rc || S == cur.stages) continue;
            b->eng->set_tune(key, ClassTune{cur.rows_per_tile, S});
            double ms = 0.0;
            const int r = probe(&ms);
            if (r == BLDM_ERR_UNSUPPORTED) continue;
            if (r) {
                rc = r;
                break;
            }
            if (ms < 0.97 * best) {
                best = ms;
                cur.stages = S;
            }
        }
        b->eng->set_tune(key, cur);
    }
    if (!rc) rc = rebuild(b, st);
    if (!rc) rc = copy_S(save, false);
    if (!rc) rc = cuda_status(cudaStreamSynchronize(st));
    b->clean = false;  // S is the one from before the probes
    if (!rc && tuned_ms) *tuned_ms = best;
    if (rc) {
        (void)copy_S(save, false);
        cudaStreamSynchronize(st);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(save);
    return rc;
}

int bldm_batch_info(const bldm_batch* b, size_t* n_classes, size_t* device_bytes,
                    uint64_t* launches) {
    if (!b) return BLDM_ERR_BAD_ARG;
    if (n_classes) *n_classes = b->eng->n_classes();
    if (device_bytes) *device_bytes = b->arena_bytes + b->eng->table_bytes();
    if (launches) *launches = b->eng->launches();
    return BLDM_OK;
}

}  // extern "C"
