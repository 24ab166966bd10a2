// bld_fact on the device: the factorisation the reference derives from a BLD
// solution, bld::bld_fact (src/bld/bld_fact.hpp:36-80):
//   W(i,k) = (alpha_i + S_i+k - 1) / (sum_i' (alpha_i' + S_i'+k - 1) + eps)
//   H(k,j) = (beta_k + S_+jk - 1) / (sum_k' (beta_k' + S_+jk' - 1) + eps)
//   L(j)   = (a + S_+j+ - 1) / (b + 1 + eps)
// The axis sums come from the fused sums sweep (deterministic partials); the
// three small kernels below reduce them in a fixed order in FP64 and write W,
// H and L in the storage type.
#include <algorithm>
#include <memory>

#include "bldm_internal.h"
#include "bldm_kernels.h"

namespace bldm {
namespace {

constexpr int kFactThreads = 256;

// H and L: one warp per column j.  Pass 1 sums h(k,j) = beta_k + S_+jk - 1 and
// S_+jk over k; pass 2 re-forms h from the partials and divides.
template <typename T>
__global__ void fact_HL_kernel(const double* part_pjk, int n_rr, long long y, long long z,
                               const double* beta, double a, double b, double eps, T* H, T* L) {
    const long long j = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (j >= y) return;  // warp-uniform
    auto pjk = [&](long long k) {
        double s = 0.0;
        for (int r = 0; r < n_rr; ++r) s += part_pjk[((long long)r * y + j) * z + k];
        return s;
    };
    double hs = 0.0, ps = 0.0;
    for (long long k = lane; k < z; k += 32) {
        const double v = pjk(k);
        hs += beta[k] + v - 1.0;
        ps += v;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        hs += __shfl_xor_sync(0xffffffffu, hs, o);
        ps += __shfl_xor_sync(0xffffffffu, ps, o);
    }
    const double cs = hs + eps;
    for (long long k = lane; k < z; k += 32) H[k * y + j] = T((beta[k] + pjk(k) - 1.0) / cs);
    if (lane == 0) L[j] = T((a + ps - 1.0) / (b + 1.0 + eps));
}

// w(i,k) = alpha_i + S_i+k - 1 from the band partials, in FP64.
__device__ __forceinline__ double fact_w(const double* part_ipk, int n_bands, long long x,
                                         long long z, const double* alpha, long long i,
                                         long long k) {
    double s = 0.0;
    for (int bd = 0; bd < n_bands; ++bd) s += part_ipk[((long long)bd * x + i) * z + k];
    return alpha[i] + s - 1.0;
}

// Column partials of W: block blk sums w over its rows; threads (k, sub).
__global__ void fact_Wpart_kernel(const double* part_ipk, int n_bands, long long x, long long z,
                                  const double* alpha, int rows, double* wpart) {
    __shared__ double acc[kFactThreads];
    const int KT = (int)min(z, (long long)kFactThreads);
    const int R = kFactThreads / KT;
    const int sub = threadIdx.x / KT;
    const long long i0 = (long long)blockIdx.x * rows;
    const long long i1 = min(x, i0 + rows);
    for (long long k0 = 0; k0 < z; k0 += KT) {
        const long long k = k0 + threadIdx.x % KT;
        double a = 0.0;
        if (sub < R && k < z)
            for (long long i = i0 + sub; i < i1; i += R) a += fact_w(part_ipk, n_bands, x, z, alpha, i, k);
        __syncthreads();
        if (sub < R) acc[threadIdx.x] = a;
        __syncthreads();
        if (threadIdx.x < KT && k < z) {
            double t = 0.0;
            for (int r = 0; r < R; ++r) t += acc[r * KT + threadIdx.x];
            wpart[(long long)blockIdx.x * z + k] = t;
        }
    }
}

// W: every block sums the column partials (fixed order) into shared memory,
// then divides its rows' w(i,k) by them.
template <typename T>
__global__ void fact_W_kernel(const double* part_ipk, int n_bands, long long x, long long z,
                              const double* alpha, const double* wpart, int n_blk, double eps,
                              long long rows_per_block, T* W) {
    extern __shared__ double colsum[];  // [z]
    for (long long k = threadIdx.x; k < z; k += blockDim.x) {
        double t = 0.0;
        for (int bb = 0; bb < n_blk; ++bb) t += wpart[(long long)bb * z + k];
        colsum[k] = t + eps;
    }
    __syncthreads();
    const long long i0 = (long long)blockIdx.x * rows_per_block;
    const long long i1 = min(x, i0 + rows_per_block);
    for (long long e = i0 * z + threadIdx.x; e < i1 * z; e += blockDim.x) {
        const long long i = e / z, k = e % z;
        W[e] = T(fact_w(part_ipk, n_bands, x, z, alpha, i, k) / colsum[k]);
    }
}

template <typename T>
int fact_typed(PlanImpl& p, const double* d_alpha, const double* d_beta, double a, double b,
               double eps, double* wpart, int rows, int n_blk, void* d_W, void* d_H, void* d_L,
               cudaStream_t st) {
    const long long x = (long long)p.x, y = (long long)p.y, z = (long long)p.z;
    const unsigned hl_blocks = unsigned((y * 32 + kFactThreads - 1) / kFactThreads);
    fact_HL_kernel<T><<<hl_blocks, kFactThreads, 0, st>>>(p.part_pjk, p.cfg.n_rr, y, z, d_beta,
                                                          a, b, eps, static_cast<T*>(d_H),
                                                          static_cast<T*>(d_L));
    fact_Wpart_kernel<<<unsigned(n_blk), kFactThreads, 0, st>>>(p.part_ipk, p.cfg.n_bands, x, z,
                                                               d_alpha, rows, wpart);
    const long long rpb = std::max(1LL, 4096 / z);
    const unsigned w_blocks = unsigned((x + rpb - 1) / rpb);
    fact_W_kernel<T><<<w_blocks, kFactThreads, size_t(z) * 8, st>>>(
        p.part_ipk, p.cfg.n_bands, x, z, d_alpha, wpart, n_blk, eps, rpb, static_cast<T*>(d_W));
    return cuda_status(cudaGetLastError());
}

}  // namespace
}  // namespace bldm

using namespace bldm;

extern "C" int bldm_bld_fact(const void* d_S, int dtype, size_t x, size_t y, size_t z,
                             const bldm_params* params, double eps, void* d_W, void* d_H,
                             void* d_L, void* stream) {
    if (!d_S || !params || !d_W || !d_H || !d_L || x == 0 || y == 0 || z == 0)
        return BLDM_ERR_BAD_ARG;
    if (dtype != BLDM_F64 && dtype != BLDM_F32) return BLDM_ERR_BAD_ARG;
    if (!params->alpha || !params->beta || params->n_alpha != x || params->n_beta != z)
        return BLDM_ERR_BAD_ARG;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    struct PlanGuard {
        PlanImpl p;
        ~PlanGuard() { plan_free(&p); }
    } g;
    int rc = plan_setup(&g.p, x, y, z, dtype);
    if (rc) return rc;
    const int rows = int(std::max<size_t>(8, (x + 255) / 256));
    const int n_blk = int((x + rows - 1) / rows);
    // device copies of alpha and beta, and the W column partials
    const size_t n_dbl = x + z + size_t(n_blk) * z;
    double* ws = nullptr;
    rc = cuda_status(cudaMallocAsync(reinterpret_cast<void**>(&ws), n_dbl * 8, st));
    if (rc) return rc;
    double* d_alpha = ws;
    double* d_beta = ws + x;
    double* wpart = ws + x + z;
    rc = cuda_status(cudaMemcpyAsync(d_alpha, params->alpha, x * 8, cudaMemcpyHostToDevice, st));
    if (!rc)
        rc = cuda_status(cudaMemcpyAsync(d_beta, params->beta, z * 8, cudaMemcpyHostToDevice, st));
    if (!rc) rc = plan_sums(&g.p, d_S, st);
    if (!rc)
        rc = dtype == BLDM_F64
                 ? fact_typed<double>(g.p, d_alpha, d_beta, params->a, params->b, eps, wpart,
                                      rows, n_blk, d_W, d_H, d_L, st)
                 : fact_typed<float>(g.p, d_alpha, d_beta, params->a, params->b, eps, wpart,
                                     rows, n_blk, d_W, d_H, d_L, st);
    // the host arrays and the plan's workspace are in use until the stream gets here
    const cudaError_t se = cudaStreamSynchronize(st);
    cudaFreeAsync(ws, st);
    if (!rc) rc = cuda_status(se);
    if (!rc) rc = plan_check(&g.p, st);
    return rc;
}

extern "C" int bldm_bld_fact_f64(const double* S, size_t x, size_t y, size_t z,
                                 const bldm_params* params, double eps, double* W, double* H,
                                 double* L) {
    if (!S || !params || !W || !H || !L || x == 0 || y == 0 || z == 0) return BLDM_ERR_BAD_ARG;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return BLDM_ERR_NO_DEVICE;
    const size_t nS = x * y * z, nW = x * z, nH = z * y;
    char* d = nullptr;
    const size_t bytes = (nS + nW + nH + y) * 8;
    int rc = cuda_status(cudaMalloc(reinterpret_cast<void**>(&d), bytes));
    if (rc) return rc;
    double* dS = reinterpret_cast<double*>(d);
    double* dW = dS + nS;
    double* dH = dW + nW;
    double* dL = dH + nH;
    rc = cuda_status(cudaMemcpy(dS, S, nS * 8, cudaMemcpyHostToDevice));
    if (!rc) rc = bldm_bld_fact(dS, BLDM_F64, x, y, z, params, eps, dW, dH, dL, nullptr);
    if (!rc) rc = cuda_status(cudaMemcpy(W, dW, nW * 8, cudaMemcpyDeviceToHost));
    if (!rc) rc = cuda_status(cudaMemcpy(H, dH, nH * 8, cudaMemcpyDeviceToHost));
    if (!rc) rc = cuda_status(cudaMemcpy(L, dL, y * 8, cudaMemcpyDeviceToHost));
    cudaFree(d);
    return rc;
}
