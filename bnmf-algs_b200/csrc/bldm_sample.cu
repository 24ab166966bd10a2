// Device data generation of the allocation model: bnmf_priors and sample_S
// (src/alloc_model/alloc_model_funcs.hpp:461-552).
//
//   L_j ~ Gamma(a, scale b)      (gsl_ran_gamma(r, a, b) takes b as the scale)
//   W(:,k) ~ Dirichlet(alpha)    (over the x rows, one draw per column k)
//   H(:,j) ~ Dirichlet(beta)     (over the z rows, one draw per column j)
//   S_ijk ~ Poisson(W_ik H_kj L_j)
//
// The reference draws from GSL's taus generator in one host thread; here
// every variate comes from a counter-based stream: a SplitMix64 hash of the
// seed, the variate's kind and index, and a per-variate draw counter, so the
// tensors do not depend on the launch layout.  Algorithms (from their
// publications): gamma by Marsaglia & Tsang (ACM TOMS 26(3), 2000) with the
// shape-below-one boost G(a) = G(a+1) U^(1/a); normal deviates by Box-Muller;
// Dirichlet as normalised gammas; Poisson by inversion below mean 10 and by
// Hormann's transformed rejection with squeeze, PTRS (Insurance: Mathematics
// and Economics 12, 1993) above.  Every rejection loop is bounded.
#include <cstdint>
#include <memory>

#include "bldm_internal.h"

namespace bldm {
namespace {

enum : uint64_t { TAG_L = 1, TAG_W = 2, TAG_H = 3, TAG_S = 4, TAG_X = 5 };
constexpr int kMaxTries = 256;

__device__ __forceinline__ uint64_t mix64(uint64_t v) {
    v += 0x9E3779B97F4A7C15ull;
    v = (v ^ (v >> 30)) * 0xBF58476D1CE4E5B9ull;
    v = (v ^ (v >> 27)) * 0x94D049BB133111EBull;
    return v ^ (v >> 31);
}

// Uniform (0, 1) deviates of one variate's stream.
struct Stream {
    uint64_t key;
    uint64_t n = 0;
    __device__ Stream(uint64_t seed, uint64_t tag, uint64_t idx)
        : key(mix64(mix64(seed ^ (tag << 56)) ^ idx)) {}
    __device__ double uniform() {
        const uint64_t h = mix64(key + 0xD1B54A32D192ED03ull * (++n));
        return (double(h >> 11) + 0.5) * (1.0 / 9007199254740992.0);
    }
    __device__ double normal() {
        const double u1 = uniform(), u2 = uniform();
        return sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
    }
};

// Gamma(shape a, scale 1).
__device__ double gamma_variate(Stream& r, double a) {
    if (!(a > 0.0)) return 0.0;
    double boost = 1.0;
    if (a < 1.0) {
        boost = pow(r.uniform(), 1.0 / a);
        a += 1.0;
    }
    const double d = a - 1.0 / 3.0;
    const double c = 1.0 / sqrt(9.0 * d);
    for (int t = 0; t < kMaxTries; ++t) {
        const double xn = r.normal();
        double v = 1.0 + c * xn;
        if (v <= 0.0) continue;
        v = v * v * v;
        const double u = r.uniform();
        const double x2 = xn * xn;
        if (u < 1.0 - 0.0331 * x2 * x2) return boost * d * v;
        if (log(u) < 0.5 * x2 + d * (1.0 - v + log(v))) return boost * d * v;
    }
    return boost * d;  // not reached in practice (acceptance > 95% per try)
}

__device__ double poisson_variate(Stream& r, double mu) {
    if (!(mu > 0.0)) return 0.0;
    if (mu < 10.0) {
        // inversion: the smallest k with F(k) >= u
        const double u = r.uniform();
        double p = exp(-mu), F = p;
        int k = 0;
        while (u > F && k < 1000) {
            ++k;
            p *= mu / double(k);
            F += p;
        }
        return double(k);
    }
    const double slam = sqrt(mu), loglam = log(mu);
    const double b = 0.931 + 2.53 * slam;
    const double a = -0.059 + 0.02483 * b;
    const double invalpha = 1.1239 + 1.1328 / (b - 3.4);
    const double vr = 0.9277 - 3.6224 / (b - 2.0);
    for (int t = 0; t < kMaxTries; ++t) {
        const double U = r.uniform() - 0.5;
        const double V = r.uniform();
        const double us = 0.5 - fabs(U);
        const double k = floor((2.0 * a / us + b) * U + mu + 0.43);
        if (us >= 0.07 && V <= vr) return k;
        if (k < 0.0 || (us < 0.013 && V > us)) continue;
        if (log(V) + log(invalpha) - log(a / (us * us) + b) <= -mu + k * loglam - lgamma(k + 1.0))
            return k;
    }
    return floor(mu);
}

template <typename T>
__global__ void prior_L_kernel(long long y, double a, double b, uint64_t seed, T* L) {
    const long long j = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= y) return;
    Stream r(seed, TAG_L, (uint64_t)j);
    L[j] = T(b * gamma_variate(r, a));
}

// Unnormalised Dirichlet components: g[i][c] = Gamma(conc[i]) for an n x m
// matrix whose columns are the draws (W: n = x rows, m = z; H: n = z, m = y).
__global__ void dirichlet_gamma_kernel(long long n, long long m, const double* conc,
                                       uint64_t seed, uint64_t tag, double* g) {
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n * m) return;
    Stream r(seed, tag, (uint64_t)e);
    g[e] = gamma_variate(r, conc[e / m]);
}

// Column c of the n x m matrix divided by its sum (one thread per column;
// the rows are read with stride m, coalesced across the warp's columns).
template <typename T>
__global__ void normalize_columns_kernel(long long n, long long m, const double* g, T* out) {
    const long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m) return;
    double s = 0.0;
    for (long long i = 0; i < n; ++i) s += g[i * m + c];
    const double inv = s > 0.0 ? 1.0 / s : 0.0;
    for (long long i = 0; i < n; ++i) out[i * m + c] = T(g[i * m + c] * inv);
}

template <typename T>
__global__ void sample_S_kernel(const T* W, const T* H, const T* L, long long x, long long y,
                                long long z, uint64_t seed, T* S) {
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= x * y * z) return;
    const long long k = e % z, j = (e / z) % y, i = e / (y * z);
    const double mu = double(W[i * z + k]) * double(H[k * y + j]) * double(L[j]);
    Stream r(seed, TAG_S, (uint64_t)e);
    S[e] = T(poisson_variate(r, mu));
}

template <typename T>
__global__ void sample_X_kernel(const T* W, const T* H, const T* L, long long x, long long y,
                                long long z, uint64_t seed, T* X) {
    const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= x * y) return;
    const long long j = e % y, i = e / y;
    double mu = 0.0;
    for (long long k = 0; k < z; ++k) mu += double(W[i * z + k]) * double(H[k * y + j]);
    Stream r(seed, TAG_X, (uint64_t)e);
    X[e] = T(poisson_variate(r, mu * double(L[j])));
}

unsigned blocks_for(long long n) { return unsigned((n + 255) / 256); }

template <typename T>
int priors_typed(size_t x, size_t y, size_t z, const bldm_params* p, uint64_t seed, void* d_W,
                 void* d_H, void* d_L, cudaStream_t st) {
    double* ws = nullptr;
    const size_t n = x + z + x * z + z * y;
    int rc = cuda_status(cudaMallocAsync(reinterpret_cast<void**>(&ws), n * 8, st));
    if (rc) return rc;
    double* alpha = ws;
    double* beta = ws + x;
    double* gW = beta + z;
    double* gH = gW + x * z;
    rc = cuda_status(cudaMemcpyAsync(alpha, p->alpha, x * 8, cudaMemcpyHostToDevice, st));
    if (!rc) rc = cuda_status(cudaMemcpyAsync(beta, p->beta, z * 8, cudaMemcpyHostToDevice, st));
    if (!rc) {
        prior_L_kernel<T><<<blocks_for((long long)y), 256, 0, st>>>((long long)y, p->a, p->b,
                                                                    seed, static_cast<T*>(d_L));
        dirichlet_gamma_kernel<<<blocks_for((long long)(x * z)), 256, 0, st>>>(
            (long long)x, (long long)z, alpha, seed, TAG_W, gW);
        normalize_columns_kernel<T><<<blocks_for((long long)z), 256, 0, st>>>(
            (long long)x, (long long)z, gW, static_cast<T*>(d_W));
        dirichlet_gamma_kernel<<<blocks_for((long long)(z * y)), 256, 0, st>>>(
            (long long)z, (long long)y, beta, seed, TAG_H, gH);
        normalize_columns_kernel<T><<<blocks_for((long long)y), 256, 0, st>>>(
            (long long)z, (long long)y, gH, static_cast<T*>(d_H));
        rc = cuda_status(cudaGetLastError());
    }
    // the host alpha/beta are read by the copies above
    const cudaError_t se = cudaStreamSynchronize(st);
    cudaFreeAsync(ws, st);
    return rc ? rc : cuda_status(se);
}

}  // namespace
}  // namespace bldm

using namespace bldm;

extern "C" int bldm_bnmf_priors(size_t x, size_t y, size_t z, const bldm_params* params,
                                uint64_t seed, int dtype, void* d_W, void* d_H, void* d_L,
                                void* stream) {
    if (!params || !d_W || !d_H || !d_L || x == 0 || y == 0 || z == 0) return BLDM_ERR_BAD_ARG;
    if (!params->alpha || !params->beta || params->n_alpha != x || params->n_beta != z)
        return BLDM_ERR_BAD_ARG;
    if (!(params->a > 0.0) || !(params->b > 0.0)) return BLDM_ERR_BAD_ARG;
    for (size_t i = 0; i < x; ++i)
        if (!(params->alpha[i] > 0.0)) return BLDM_ERR_BAD_ARG;
    for (size_t k = 0; k < z; ++k)
        if (!(params->beta[k] > 0.0)) return BLDM_ERR_BAD_ARG;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (dtype == BLDM_F64) return priors_typed<double>(x, y, z, params, seed, d_W, d_H, d_L, st);
    if (dtype == BLDM_F32) return priors_typed<float>(x, y, z, params, seed, d_W, d_H, d_L, st);
    return BLDM_ERR_BAD_ARG;
}

extern "C" int bldm_sample_S(const void* d_W, const void* d_H, const void* d_L, size_t x,
                             size_t y, size_t z, uint64_t seed, int dtype, void* d_S,
                             void* stream) {
    if (!d_W || !d_H || !d_L || !d_S || x == 0 || y == 0 || z == 0) return BLDM_ERR_BAD_ARG;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const long long n = (long long)(x * y * z);
    if (dtype == BLDM_F64)
        sample_S_kernel<double><<<blocks_for(n), 256, 0, st>>>(
            static_cast<const double*>(d_W), static_cast<const double*>(d_H),
            static_cast<const double*>(d_L), (long long)x, (long long)y, (long long)z, seed,
            static_cast<double*>(d_S));
    else if (dtype == BLDM_F32)
        sample_S_kernel<float><<<blocks_for(n), 256, 0, st>>>(
            static_cast<const float*>(d_W), static_cast<const float*>(d_H),
            static_cast<const float*>(d_L), (long long)x, (long long)y, (long long)z, seed,
            static_cast<float*>(d_S));
    else
        return BLDM_ERR_BAD_ARG;
    return cuda_status(cudaGetLastError());
}

extern "C" int bldm_sample_X(const void* d_W, const void* d_H, const void* d_L, size_t x,
                             size_t y, size_t z, uint64_t seed, int dtype, void* d_X,
                             void* stream) {
    if (!d_W || !d_H || !d_L || !d_X || x == 0 || y == 0 || z == 0) return BLDM_ERR_BAD_ARG;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const long long n = (long long)(x * y);
    if (dtype == BLDM_F64)
        sample_X_kernel<double><<<blocks_for(n), 256, 0, st>>>(
            static_cast<const double*>(d_W), static_cast<const double*>(d_H),
            static_cast<const double*>(d_L), (long long)x, (long long)y, (long long)z, seed,
            static_cast<double*>(d_X));
    else if (dtype == BLDM_F32)
        sample_X_kernel<float><<<blocks_for(n), 256, 0, st>>>(
            static_cast<const float*>(d_W), static_cast<const float*>(d_H),
            static_cast<const float*>(d_L), (long long)x, (long long)y, (long long)z, seed,
            static_cast<float*>(d_X));
    else
        return BLDM_ERR_BAD_ARG;
    return cuda_status(cudaGetLastError());
}
