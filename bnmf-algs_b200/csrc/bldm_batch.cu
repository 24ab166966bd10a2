// C ABI of the batched solver: many independent bld_mult instances of
// different shapes solved together (bldm_batch_*).  The reference solves one
// instance per call (bld::bld_mult_cuda, src/bld/bld_mult/bld_mult.hpp:225-324);
// a batch runs the same iterations for all its instances in shared launches.
#include <cstring>
#include <memory>
#include <vector>

#include "bldm_engine.h"

using namespace bldm;

struct bldm_batch {
    std::unique_ptr<Engine> eng;
    std::vector<EngineInstance> inst;
    void* arena = nullptr;
    size_t arena_bytes = 0;
    int dtype = BLDM_F64;
    ~bldm_batch() {
        eng.reset();
        if (arena) cudaFree(arena);
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
    std::vector<EngineInstance*> ptrs(n);
    for (size_t i = 0; i < n; ++i) {
        b->eng->bind(b->inst[i], static_cast<char*>(b->arena) + off[i]);
        ptrs[i] = &b->inst[i];
    }
    for (size_t i = 0; i < n; ++i) {
        e = cudaMemset(b->inst[i].counter, 0, 16);
        if (e != cudaSuccess) return cuda_status(e);
    }
    int rc = b->eng->build(ptrs, nullptr);
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
    int rc = f64 ? upload<double>(X, in.x * in.y, in.X) : upload<float>(X, in.x * in.y, in.X);
    if (rc) return rc;
    rc = cuda_status(cudaMemcpy(in.alpha, alpha, in.x * 8, cudaMemcpyHostToDevice));
    if (rc) return rc;
    rc = cuda_status(cudaMemcpy(in.beta, beta, in.z * 8, cudaMemcpyHostToDevice));
    if (rc) return rc;
    const size_t ns = in.x * in.y * in.z;
    if (S0) return f64 ? upload<double>(S0, ns, in.S) : upload<float>(S0, ns, in.S);
    rc = launch_init_S(b->dtype, in.X, in.S, (long long)(in.x * in.y), (long long)in.z, seed,
                       nullptr);
    if (rc) return rc;
    return cuda_status(cudaDeviceSynchronize());
}

int bldm_batch_run(bldm_batch* b, size_t iters, int psi_mode, double eps, int use_graph,
                   void* stream) {
    if (!b) return BLDM_ERR_BAD_ARG;
    return b->eng->run(iters, psi_mode, eps, use_graph != 0, static_cast<cudaStream_t>(stream));
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

int bldm_batch_device_ptrs(bldm_batch* b, size_t idx, void** d_X, void** d_S) {
    if (!b || idx >= b->inst.size()) return BLDM_ERR_BAD_ARG;
    if (d_X) *d_X = b->inst[idx].X;
    if (d_S) *d_S = b->inst[idx].S;
    return BLDM_OK;
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
