// Row-sum conservation residual of a solution.
//
// The reference's tests check, after a solve, that S summed over k gives X back
// (test/bld/bld_mult/test_bld_mult.cpp:67-71,80-84: S_ij+ isApprox X).  The
// update uses the pre-update sums S_ij+ (bld_mult_funcs.hpp:307-327), so the
// sums equal X only at the fixed point; the residual
//   max_ij |sum_k S(i,j,k) - X(i,j)| / max(X(i,j), 1)
// is therefore reported with every solve rather than asserted to be zero.  One
// read of S: lane groups of lpf = min(32, pow2ceil(z)) lanes per fiber add the
// fiber in FP64 (consecutive lanes read consecutive elements), the group's
// first lane forms the fiber's ratio, and each block contributes its maximum
// with one atomicMax on the bits of the (nonnegative) double.
#include <cstring>

#include "bldm_device.cuh"
#include "bldm_internal.h"
#include "bldm_kernels.h"

namespace bldm {

namespace {

constexpr int kConsThreads = 256;
constexpr int kConsRounds = 8;  // fiber groups per warp per block

// max that keeps a NaN from either side
__device__ __forceinline__ double nan_max(double a, double b) {
    return (a != a || a > b) ? a : b;
}

int lpf_of(long long z) {
    int l = 1;
    while (l < 32 && l < z) l <<= 1;
    return l;
}

long long fibers_per_block(int lpf) { return (long long)(kConsThreads / lpf) * kConsRounds; }

// Fibers [f0, f1) of one instance; every thread of the block calls it.
template <typename T>
__device__ void cons_fibers(const T* X, const T* S, long long f0, long long f1, long long z,
                            int lpf, unsigned long long* out) {
    __shared__ double wmax[kConsThreads / 32];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int q = lane % lpf;
    const int gpw = 32 / lpf;  // fibers per warp per round
    double m = 0.0;
    for (int r = 0; r < kConsRounds; ++r) {
        const long long f =
            f0 + ((long long)r * (kConsThreads / 32) + warp) * gpw + lane / lpf;
        const bool on = f < f1;
        double s = 0.0;
        if (on)
            for (long long k = q; k < z; k += lpf) s += double(S[f * z + k]);
        for (int o = 1; o < lpf; o <<= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (on && q == 0) {
            const double xv = double(X[f]);
            m = nan_max(m, fabs(s - xv) / fmax(xv, 1.0));
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = nan_max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if (lane == 0) wmax[warp] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        double b = 0.0;
        for (int w = 0; w < kConsThreads / 32; ++w) b = nan_max(b, wmax[w]);
        atomicMax(out, (unsigned long long)__double_as_longlong(b));
    }
}

template <typename T>
__global__ void __launch_bounds__(kConsThreads)
    conservation_kernel(const T* X, const T* S, long long nf, long long z, int lpf,
                        unsigned long long* out) {
    const long long per = (long long)(kConsThreads / lpf) * kConsRounds;
    const long long f0 = (long long)blockIdx.x * per;
    cons_fibers<T>(X, S, f0, min(nf, f0 + per), z, lpf, out);
}

template <typename T>
__global__ void __launch_bounds__(kConsThreads)
    conservation_multi_kernel(const ConsInst* insts, const int* block_off, int n_inst) {
    int lo = 0, hi = n_inst - 1;
    const int b = int(blockIdx.x);
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (block_off[mid] <= b) lo = mid;
        else hi = mid - 1;
    }
    const ConsInst in = insts[lo];
    const long long per = (long long)(kConsThreads / in.lpf) * kConsRounds;
    const long long f0 = (long long)(b - block_off[lo]) * per;
    cons_fibers<T>(static_cast<const T*>(in.X), static_cast<const T*>(in.S), f0,
                   min(in.nf, f0 + per), in.z, in.lpf, in.out);
}

}  // namespace

int conservation_blocks(long long nf, long long z) {
    const long long per = fibers_per_block(lpf_of(z));
    return int((nf + per - 1) / per);
}

int launch_conservation(int dtype, const void* dX, const void* dS, long long nf, long long z,
                        unsigned long long* out, cudaStream_t st) {
    if (nf <= 0 || z <= 0) return BLDM_OK;
    const int lpf = lpf_of(z);
    const unsigned blocks = unsigned(conservation_blocks(nf, z));
    if (dtype == BLDM_F64)
        conservation_kernel<double><<<blocks, kConsThreads, 0, st>>>(
            static_cast<const double*>(dX), static_cast<const double*>(dS), nf, z, lpf, out);
    else
        conservation_kernel<float><<<blocks, kConsThreads, 0, st>>>(
            static_cast<const float*>(dX), static_cast<const float*>(dS), nf, z, lpf, out);
    return cuda_status(cudaGetLastError());
}

int launch_conservation_multi(int dtype, const ConsInst* d_insts, const int* d_block_off,
                              int n_inst, int n_blocks, cudaStream_t st) {
    if (n_inst <= 0 || n_blocks <= 0) return BLDM_OK;
    if (dtype == BLDM_F64)
        conservation_multi_kernel<double><<<n_blocks, kConsThreads, 0, st>>>(d_insts, d_block_off,
                                                                             n_inst);
    else
        conservation_multi_kernel<float><<<n_blocks, kConsThreads, 0, st>>>(d_insts, d_block_off,
                                                                            n_inst);
    return cuda_status(cudaGetLastError());
}

// ConsInst of one instance (lane-group width from its depth).
ConsInst cons_inst(const void* X, const void* S, long long nf, long long z,
                   unsigned long long* out) {
    ConsInst c;
    c.X = X;
    c.S = S;
    c.nf = nf;
    c.z = z;
    c.out = out;
    c.lpf = lpf_of(z);
    c.pad = 0;
    return c;
}

double cons_value(unsigned long long bits) {
    double v;
    static_assert(sizeof v == sizeof bits, "64-bit double");
    memcpy(&v, &bits, sizeof v);
    return v;
}

}  // namespace bldm
