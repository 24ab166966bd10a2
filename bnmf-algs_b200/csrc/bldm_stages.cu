// Per-stage device functions and the device log-marginal.
//
// The stage kernels expose each formula of the reference's CUDA path on its
// own, so the tests can compare every stage with the CPU restatement the way
// test/bld/bld_mult/test_bld_mult_cuda_funcs.cpp does.  They share the digamma
// device functions with the fused sweep.  They are straightforward one-thread-
// per-output kernels: the production path is the fused sweep in
// bldm_sweep.cu, not these.
#include <cmath>
#include <vector>

#include "bldm_device.cuh"
#include "bldm_internal.h"

namespace bldm {

namespace {

constexpr int kT = 256;

inline unsigned nblocks(long long n) { return unsigned((n + kT - 1) / kT); }

// cuda::tensor_sums (cuda_src/tensor_ops.cu:10-55, kernel
// cuda_src/tensor_ops_kernels.cu:7-58), FP64 accumulation for any storage T.
template <typename T>
__global__ void sum_pjk_kernel(const T* S, long long x, long long y, long long z, double* pjk) {
    const long long idx = (long long)blockIdx.x * kT + threadIdx.x;  // (j,k)
    if (idx >= y * z) return;
    double s = 0.0;
    for (long long i = 0; i < x; ++i) s += double(S[i * y * z + idx]);
    pjk[idx] = s;
}
template <typename T>
__global__ void sum_ipk_kernel(const T* S, long long x, long long y, long long z, double* ipk) {
    const long long idx = (long long)blockIdx.x * kT + threadIdx.x;  // (i,k)
    if (idx >= x * z) return;
    const long long i = idx / z, k = idx % z;
    double s = 0.0;
    for (long long j = 0; j < y; ++j) s += double(S[(i * y + j) * z + k]);
    ipk[idx] = s;
}
template <typename T>
__global__ void sum_ijp_kernel(const T* S, long long x, long long y, long long z, double* ijp) {
    const long long idx = (long long)blockIdx.x * kT + threadIdx.x;  // (i,j)
    if (idx >= x * y) return;
    double s = 0.0;
    for (long long k = 0; k < z; ++k) s += double(S[idx * z + k]);
    ijp[idx] = s;
}

// update_grad_plus kernel (cuda_src/bld_mult/bld_mult_cuda_kernels.cu:86-117).
__global__ void grad_plus_kernel(const double* S, const double* beta_eph, long long x,
                                 long long y, long long z, int appr, double* gp) {
    const long long e = (long long)blockIdx.x * kT + threadIdx.x;
    if (e >= x * y * z) return;
    const long long k = e % z;
    const long long j = (e / z) % y;
    const double b = beta_eph[j * z + k];
    gp[e] = appr ? psi_appr_f64(b) - psi_appr_f64(S[e] + 1.0)
                 : psi_exact_f64(b) - psi_exact_f64(S[e] + 1.0);
}

// update_grad_minus (src/bld/bld_mult/bld_mult_funcs.hpp:205-229), two passes.
__global__ void psi_colsum_kernel(const double* alpha_eph, long long x, long long z, int appr,
                                  double* psi_sum) {
    const long long k = (long long)blockIdx.x * kT + threadIdx.x;
    if (k >= z) return;
    double s = 0.0;
    for (long long i = 0; i < x; ++i) s += alpha_eph[i * z + k];
    psi_sum[k] = psi_mode_f64(s, appr != 0);
}
__global__ void grad_minus_kernel(const double* alpha_eph, const double* psi_sum, long long x,
                                  long long z, int appr, double* gm) {
    const long long e = (long long)blockIdx.x * kT + threadIdx.x;
    if (e >= x * z) return;
    gm[e] = psi_sum[e % z] - psi_mode_f64(alpha_eph[e], appr != 0);
}

// update_nom kernel (bld_mult_cuda_kernels.cu:120-159).
__global__ void nom_kernel(const double* Xr, const double* gm, const double* S, long long x,
                           long long y, long long z, double* nom) {
    const long long f = (long long)blockIdx.x * kT + threadIdx.x;  // (i,j)
    if (f >= x * y) return;
    const long long i = f / y;
    double s = 0.0;
    for (long long k = 0; k < z; ++k) s += S[f * z + k] * Xr[f] * gm[i * z + k];
    nom[f] = s;
}

// update_denom kernel (bld_mult_cuda_kernels.cu:162-200).
__global__ void denom_kernel(const double* Xr, const double* gp, const double* S, long long x,
                             long long y, long long z, double* denom) {
    const long long f = (long long)blockIdx.x * kT + threadIdx.x;
    if (f >= x * y) return;
    double s = 0.0;
    for (long long k = 0; k < z; ++k) s += S[f * z + k] * Xr[f] * gp[f * z + k];
    denom[f] = s;
}

// update_S kernel (bld_mult_cuda_kernels.cu:203-255) with the caller's eps.
__global__ void update_S_kernel(const double* X, const double* nom, const double* denom,
                                const double* gm, const double* gp, const double* ijp,
                                long long x, long long y, long long z, double eps, double* S) {
    const long long e = (long long)blockIdx.x * kT + threadIdx.x;
    if (e >= x * y * z) return;
    const long long f = e / z;
    const long long k = e % z;
    const long long i = f / y;
    S[e] *= (gp[e] + nom[f]) * (X[f] / (ijp[f] + eps)) / (gm[i * z + k] + denom[f] + eps);
}

__global__ void psi_f64_kernel(const double* in, long long n, int appr, double* out) {
    __shared__ double2 ltab[kLogTabN];
    if (appr == 2) {
        log_tab_init(ltab, threadIdx.x, kT);
        __syncthreads();
    }
    const long long e = (long long)blockIdx.x * kT + threadIdx.x;
    if (appr == 2) {
        // the fused sweep's evaluation (all lanes take part)
        const double xv[1] = {e < n ? in[e] : 1.0};
        double r[1];
        psi_appr_batch<1>(xv, r, ltab);
        if (e < n) out[e] = r[0];
        return;
    }
    if (e < n) out[e] = appr ? psi_appr_f64(in[e]) : psi_exact_f64(in[e]);
}
__global__ void psi_f32_kernel(const float* in, long long n, int mode, float* out) {
    const long long e = (long long)blockIdx.x * kT + threadIdx.x;
    if (e >= n) return;
    if (mode == 1) {
        const float a[1] = {in[e]};
        float o[1];
        psi_f32_batch<1>(a, o);
        out[e] = o[0];
    } else {
        out[e] = psi_f32(in[e]);
    }
}

// ---- log_marginal_S (src/alloc_model/alloc_model_funcs.hpp:33-194,573-586).
// Block-level partial sums in a fixed order; the final kernel adds the
// partials of every term in order, so the result is deterministic.
__device__ __forceinline__ double block_sum(double v, double* sh) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    if (lane == 0) sh[w] = v;
    __syncthreads();
    double r = 0.0;
    if (threadIdx.x == 0)
        for (int i = 0; i < kT / 32; ++i) r += sh[i];
    __syncthreads();
    return r;
}

template <typename T>
__global__ void lgamma_S1_kernel(const T* S, long long n, double* part) {
    __shared__ double sh[kT / 32];
    double acc = 0.0;
    for (long long e = (long long)blockIdx.x * kT + threadIdx.x; e < n;
         e += (long long)gridDim.x * kT)
        acc += lgamma(double(S[e]) + 1.0);
    const double r = block_sum(acc, sh);
    if (threadIdx.x == 0) part[blockIdx.x] = r;
}

// first term per k (column of S_ipk): sum_i lgamma(alpha_i + S_ipk(i,k))
// - lgamma(sum_i (alpha_i + S_ipk(i,k))).  second term per j likewise with beta.
// third term per j: lgamma(a + S_pjp(j)) - (a + S_pjp(j)) log(b+1).
__global__ void small_terms_kernel(const double* ipk, const double* pjk, const double* alpha,
                                   const double* beta, long long x, long long y, long long z,
                                   double a, double b, double* part_first,
                                   double* part_second) {
    const long long t = (long long)blockIdx.x * kT + threadIdx.x;
    if (t < z) {
        const long long k = t;
        double tot = 0.0, acc = 0.0;
        for (long long i = 0; i < x; ++i) {
            const double v = alpha[i] + ipk[i * z + k];
            tot += v;
            acc += lgamma(v);
        }
        part_first[k] = acc - lgamma(tot);
    }
    if (t < y) {
        const long long j = t;
        double tot = 0.0, acc = 0.0, pjp = 0.0;
        for (long long k = 0; k < z; ++k) {
            const double v = beta[k] + pjk[j * z + k];
            pjp += pjk[j * z + k];
            tot += v;
            acc += lgamma(v);
        }
        const double sa = a + pjp;
        part_second[2 * j] = acc - lgamma(tot);
        part_second[2 * j + 1] = lgamma(sa) - sa * log(b + 1.0);
    }
}

__global__ void lm_final_kernel(const double* part_first, long long z, const double* part_second,
                                long long y, const double* part_fourth, int n4, double base,
                                double* out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double first = 0.0, second = 0.0, third = 0.0, fourth = 0.0;
    for (long long k = 0; k < z; ++k) first += part_first[k];
    for (long long j = 0; j < y; ++j) {
        second += part_second[2 * j];
        third += part_second[2 * j + 1];
    }
    for (int i = 0; i < n4; ++i) fourth += part_fourth[i];
    out[0] = base + first + second + third - fourth;
}

}  // namespace

template <typename T>
int tensor_sums_dev(const T* S, size_t x, size_t y, size_t z, double* pjk, double* ipk,
                    double* ijp, cudaStream_t st) {
    const long long X = (long long)x, Y = (long long)y, Z = (long long)z;
    if (pjk) sum_pjk_kernel<T><<<nblocks(Y * Z), kT, 0, st>>>(S, X, Y, Z, pjk);
    if (ipk) sum_ipk_kernel<T><<<nblocks(X * Z), kT, 0, st>>>(S, X, Y, Z, ipk);
    if (ijp) sum_ijp_kernel<T><<<nblocks(X * Y), kT, 0, st>>>(S, X, Y, Z, ijp);
    return cuda_status(cudaGetLastError());
}

}  // namespace bldm

using namespace bldm;

#define BLDM_CHECK_PTR(p) \
    if (!(p)) return BLDM_ERR_BAD_ARG

extern "C" {

int bldm_tensor_sums_f64(const double* d_S, size_t x, size_t y, size_t z, double* d_pjk,
                         double* d_ipk, double* d_ijp, void* stream) {
    BLDM_CHECK_PTR(d_S);
    if (x * y * z == 0) return BLDM_OK;
    return tensor_sums_dev<double>(d_S, x, y, z, d_pjk, d_ipk, d_ijp,
                                   static_cast<cudaStream_t>(stream));
}

int bldm_update_grad_plus_f64(const double* d_S, const double* d_beta_eph, size_t x, size_t y,
                              size_t z, int appr, double* d_grad_plus, void* stream) {
    BLDM_CHECK_PTR(d_S);
    BLDM_CHECK_PTR(d_beta_eph);
    BLDM_CHECK_PTR(d_grad_plus);
    const long long n = (long long)(x * y * z);
    if (n == 0) return BLDM_OK;
    grad_plus_kernel<<<nblocks(n), kT, 0, static_cast<cudaStream_t>(stream)>>>(
        d_S, d_beta_eph, (long long)x, (long long)y, (long long)z, appr, d_grad_plus);
    return cuda_status(cudaGetLastError());
}

int bldm_update_grad_minus_f64(const double* d_alpha_eph, size_t x, size_t z, int appr,
                               double* d_grad_minus, void* stream) {
    BLDM_CHECK_PTR(d_alpha_eph);
    BLDM_CHECK_PTR(d_grad_minus);
    if (x * z == 0) return BLDM_OK;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    double* psi_sum = nullptr;
    cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(&psi_sum), z * sizeof(double), st);
    if (e != cudaSuccess) return cuda_status(e);
    psi_colsum_kernel<<<nblocks((long long)z), kT, 0, st>>>(d_alpha_eph, (long long)x,
                                                             (long long)z, appr, psi_sum);
    grad_minus_kernel<<<nblocks((long long)(x * z)), kT, 0, st>>>(
        d_alpha_eph, psi_sum, (long long)x, (long long)z, appr, d_grad_minus);
    e = cudaGetLastError();
    cudaFreeAsync(psi_sum, st);
    return cuda_status(e);
}

int bldm_update_nom_f64(const double* d_X_reciprocal, const double* d_grad_minus,
                        const double* d_S, size_t x, size_t y, size_t z, double* d_nom,
                        void* stream) {
    BLDM_CHECK_PTR(d_X_reciprocal);
    BLDM_CHECK_PTR(d_grad_minus);
    BLDM_CHECK_PTR(d_S);
    BLDM_CHECK_PTR(d_nom);
    if (x * y == 0) return BLDM_OK;
    nom_kernel<<<nblocks((long long)(x * y)), kT, 0, static_cast<cudaStream_t>(stream)>>>(
        d_X_reciprocal, d_grad_minus, d_S, (long long)x, (long long)y, (long long)z, d_nom);
    return cuda_status(cudaGetLastError());
}

int bldm_update_denom_f64(const double* d_X_reciprocal, const double* d_grad_plus,
                          const double* d_S, size_t x, size_t y, size_t z, double* d_denom,
                          void* stream) {
    BLDM_CHECK_PTR(d_X_reciprocal);
    BLDM_CHECK_PTR(d_grad_plus);
    BLDM_CHECK_PTR(d_S);
    BLDM_CHECK_PTR(d_denom);
    if (x * y == 0) return BLDM_OK;
    denom_kernel<<<nblocks((long long)(x * y)), kT, 0, static_cast<cudaStream_t>(stream)>>>(
        d_X_reciprocal, d_grad_plus, d_S, (long long)x, (long long)y, (long long)z, d_denom);
    return cuda_status(cudaGetLastError());
}

int bldm_update_S_f64(const double* d_X, const double* d_nom, const double* d_denom,
                      const double* d_grad_minus, const double* d_grad_plus,
                      const double* d_S_ijp, size_t x, size_t y, size_t z, double eps,
                      double* d_S, void* stream) {
    BLDM_CHECK_PTR(d_X);
    BLDM_CHECK_PTR(d_nom);
    BLDM_CHECK_PTR(d_denom);
    BLDM_CHECK_PTR(d_grad_minus);
    BLDM_CHECK_PTR(d_grad_plus);
    BLDM_CHECK_PTR(d_S_ijp);
    BLDM_CHECK_PTR(d_S);
    const long long n = (long long)(x * y * z);
    if (n == 0) return BLDM_OK;
    update_S_kernel<<<nblocks(n), kT, 0, static_cast<cudaStream_t>(stream)>>>(
        d_X, d_nom, d_denom, d_grad_minus, d_grad_plus, d_S_ijp, (long long)x, (long long)y,
        (long long)z, eps, d_S);
    return cuda_status(cudaGetLastError());
}

int bldm_psi_f64(const double* d_in, size_t n, int appr, double* d_out, void* stream) {
    BLDM_CHECK_PTR(d_in);
    BLDM_CHECK_PTR(d_out);
    if (n == 0) return BLDM_OK;
    psi_f64_kernel<<<nblocks((long long)n), kT, 0, static_cast<cudaStream_t>(stream)>>>(
        d_in, (long long)n, appr, d_out);
    return cuda_status(cudaGetLastError());
}

int bldm_psi_f32_mode(const float* d_in, size_t n, int mode, float* d_out, void* stream) {
    BLDM_CHECK_PTR(d_in);
    BLDM_CHECK_PTR(d_out);
    if (mode != 0 && mode != 1) return BLDM_ERR_BAD_ARG;
    if (n == 0) return BLDM_OK;
    psi_f32_kernel<<<nblocks((long long)n), kT, 0, static_cast<cudaStream_t>(stream)>>>(
        d_in, (long long)n, mode, d_out);
    return cuda_status(cudaGetLastError());
}

int bldm_psi_f32(const float* d_in, size_t n, float* d_out, void* stream) {
    return bldm_psi_f32_mode(d_in, n, 0, d_out, stream);
}

int bldm_log_marginal_S(const void* d_S, int dtype, size_t x, size_t y, size_t z,
                        const double* alpha, const double* beta, double a, double b,
                        double* result, void* stream) {
    BLDM_CHECK_PTR(d_S);
    BLDM_CHECK_PTR(alpha);
    BLDM_CHECK_PTR(beta);
    BLDM_CHECK_PTR(result);
    if (dtype != BLDM_F64 && dtype != BLDM_F32) return BLDM_ERR_BAD_ARG;
    if (x * y * z == 0) return BLDM_ERR_BAD_ARG;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // Host-side constant parts (lgamma of the parameters).
    double sa = 0, lga = 0, sb = 0, lgb = 0;
    for (size_t i = 0; i < x; ++i) {
        sa += alpha[i];
        lga += std::lgamma(alpha[i]);
    }
    for (size_t k = 0; k < z; ++k) {
        sb += beta[k];
        lgb += std::lgamma(beta[k]);
    }
    const double base = (std::lgamma(sa) - lga) * double(z) + (std::lgamma(sb) - lgb) * double(y) +
                        (-std::lgamma(a) + a * std::log(b)) * double(y);
    const int n4 = 592;
    const size_t n_doubles = x * z + y * z + z + 2 * y + n4 + x + z + 1;
    double* ws = nullptr;
    cudaError_t e = cudaMallocAsync(reinterpret_cast<void**>(&ws), n_doubles * sizeof(double), st);
    if (e != cudaSuccess) return cuda_status(e);
    double* ipk = ws;
    double* pjk = ipk + x * z;
    double* pfirst = pjk + y * z;
    double* psecond = pfirst + z;
    double* pfourth = psecond + 2 * y;
    double* dalpha = pfourth + n4;
    double* dbeta = dalpha + x;
    double* dout = dbeta + z;
    int rc = BLDM_OK;
    e = cudaMemcpyAsync(dalpha, alpha, x * sizeof(double), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(dbeta, beta, z * sizeof(double), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        const long long n = (long long)(x * y * z);
        if (dtype == BLDM_F64) {
            rc = tensor_sums_dev<double>(static_cast<const double*>(d_S), x, y, z, pjk, ipk,
                                         nullptr, st);
            lgamma_S1_kernel<double><<<n4, kT, 0, st>>>(static_cast<const double*>(d_S), n,
                                                         pfourth);
        } else {
            rc = tensor_sums_dev<float>(static_cast<const float*>(d_S), x, y, z, pjk, ipk,
                                        nullptr, st);
            lgamma_S1_kernel<float><<<n4, kT, 0, st>>>(static_cast<const float*>(d_S), n,
                                                        pfourth);
        }
        const long long m = (long long)(y > z ? y : z);
        small_terms_kernel<<<nblocks(m), kT, 0, st>>>(ipk, pjk, dalpha, dbeta, (long long)x,
                                                      (long long)y, (long long)z, a, b, pfirst,
                                                      psecond);
        lm_final_kernel<<<1, 32, 0, st>>>(pfirst, (long long)z, psecond, (long long)y, pfourth,
                                          n4, base, dout);
        e = cudaGetLastError();
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(result, dout, sizeof(double), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    }
    cudaFreeAsync(ws, st);
    if (rc != BLDM_OK) return rc;
    return cuda_status(e);
}

}  // extern "C"
