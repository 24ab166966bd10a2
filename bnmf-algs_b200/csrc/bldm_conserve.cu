// Row-sum conservation residual of a solution.
//
// The reference's tests check, after a solve, that S summed over k gives X back
// (test/bld/bld_mult/test_bld_mult.cpp:67-71,80-84: S_ij+ isApprox X).  The
// update uses the pre-update sums S_ij+ (bld_mult_funcs.hpp:307-327), so the
// sums equal X only at the fixed point; the residual
//   max_ij |sum_k S(i,j,k) - X(i,j)| / max(X(i,j), 1)
// is therefore reported with every solve rather than asserted to be zero.  One
// read of S: lane groups of up to 32 lanes per fiber add the fiber in FP64
// from 16-byte streaming loads (consecutive lanes read consecutive vectors),
// eight fibers per group at a time reduced by one transposing butterfly, and
// each block contributes its maximum with one atomicMax on the bits of the
// (nonnegative) double.
#include <algorithm>
#include <cstdint>
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

// Lane layout of a fiber: VEC-element vectors (16 bytes when S starts on a
// 16-byte boundary and the fiber's bytes are a multiple of 16), lpf =
// min(32, pow2ceil(vectors)) lanes.
int vec_of(const void* S, long long z, size_t es) {
    const bool aligned = (reinterpret_cast<uintptr_t>(S) & 15) == 0;
    return aligned && (z * (long long)es) % 16 == 0 ? int(16 / es) : 1;
}
int lpf_of(long long z, int vec) {
    const long long nv = (z + vec - 1) / vec;
    int l = 1;
    while (l < 32 && l < nv) l <<= 1;
    return l;
}

long long fibers_per_block(int lpf) { return (long long)(kConsThreads / lpf) * kConsRounds; }

template <typename T, int VEC> struct Vec;
template <typename T> struct Vec<T, 1> {
    __device__ __forceinline__ static double sum(const T* p) { return double(__ldcs(p)); }
};
template <> struct Vec<double, 2> {
    __device__ __forceinline__ static double sum(const double* p) {
        const double2 v = __ldcs(reinterpret_cast<const double2*>(p));
        return v.x + v.y;
    }
};
template <> struct Vec<float, 4> {
    __device__ __forceinline__ static double sum(const float* p) {
        const float4 v = __ldcs(reinterpret_cast<const float4*>(p));
        return (double(v.x) + double(v.y)) + (double(v.z) + double(v.w));
    }
};

// Fibers [f0, f1) of one instance: the largest ratio of the calling thread's
// fibers folded into m.  Every thread of the block calls it.  A warp takes
// 32 / LPF fibers per round, kConsRounds rounds; all S loads are issued before
// any sum is reduced (streaming loads, 16 bytes per lane where aligned).  The
// U = kConsRounds per-lane partials are reduced over each lane group by a
// transposing butterfly: at each offset o while more than one partial is left,
// a lane keeps half of its partials (the upper half when its bit o is set) and
// adds the partner's matching half, so the U sums take U - 1 shuffles instead
// of U log2(LPF); the remaining offsets add plainly.  A lane then holds
// max(1, U / LPF) complete fiber sums, rounds base .. base + H - 1 of its group
// (lanes that differ only in the plain offsets hold the same ones, which the
// max does not mind); their X values are loaded with the S loads.
template <typename T, int VEC, int LPF>
__device__ void cons_fibers(const T* X, const T* S, long long f0, long long f1, long long z,
                            double& m_out) {
    constexpr int U = kConsRounds;
    constexpr int GPW = 32 / LPF;  // fibers per warp per round
    constexpr int H = U / LPF > 1 ? U / LPF : 1;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int q = lane % LPF;
    const int g = lane / LPF;
    const long long nv = z / VEC;  // VEC > 1 only when it divides z
    auto fiber = [&](int u) { return f0 + ((long long)u * (kConsThreads / 32) + warp) * GPW + g; };
    // rounds this lane holds after the butterfly
    int base = 0;
    {
        int cur = U;
#pragma unroll
        for (int o = LPF / 2; o > 0; o >>= 1)
            if (cur > 1) {
                cur >>= 1;
                if (lane & o) base += cur;
            }
    }
    double xv[H];
#pragma unroll
    for (int j = 0; j < H; ++j) {
        const long long f = fiber(base + j);
        xv[j] = f < f1 ? double(X[f]) : 0.0;
    }
    double s[U];
#pragma unroll
    for (int u = 0; u < U; ++u) s[u] = 0.0;
    for (long long v = q; v < nv; v += LPF) {
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const long long f = fiber(u);
            if (f < f1) s[u] += Vec<T, VEC>::sum(S + f * z + v * VEC);
        }
    }
    {
        int cur = U;
#pragma unroll
        for (int o = LPF / 2; o > 0; o >>= 1) {
            if (cur > 1) {
                const int half = cur >> 1;
                const bool hi = (lane & o) != 0;
#pragma unroll
                for (int j = 0; j < half; ++j) {
                    const double send = hi ? s[j] : s[j + half];
                    const double keep = hi ? s[j + half] : s[j];
                    s[j] = keep + __shfl_xor_sync(0xffffffffu, send, o);
                }
                cur = half;
            } else {
                s[0] += __shfl_xor_sync(0xffffffffu, s[0], o);
            }
        }
    }
    double m = m_out;
#pragma unroll
    for (int j = 0; j < H; ++j)
        if (fiber(base + j) < f1) m = nan_max(m, fabs(s[j] - xv[j]) / fmax(xv[j], 1.0));
    m_out = m;
}

// The block's maximum to *out: one atomicMax per CTA (the blocks of a launch
// loop over the fiber blocks, so the atomics on the one word stay few).
__device__ __forceinline__ void cons_block_max(double m, unsigned long long* out) {
    __shared__ double wmax[kConsThreads / 32];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
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

template <typename T, int VEC, int LPF>
__global__ void __launch_bounds__(kConsThreads)
    conservation_kernel(const T* X, const T* S, long long nf, long long z, long long nblocks,
                        unsigned long long* out) {
    constexpr long long per = (long long)(kConsThreads / LPF) * kConsRounds;
    double m = 0.0;
    for (long long vb = blockIdx.x; vb < nblocks; vb += gridDim.x) {
        const long long f0 = vb * per;
        cons_fibers<T, VEC, LPF>(X, S, f0, min(nf, f0 + per), z, m);
    }
    cons_block_max(m, out);
}

// The fibers [f0, f1) of one instance with the lane layout (vec, lpf) chosen at
// run time.
template <typename T>
__device__ void cons_fibers_rt(const T* X, const T* S, long long f0, long long f1, long long z,
                               int vec, int lpf, double& m) {
    constexpr int V = 16 / int(sizeof(T));
    if (vec == 1) {
        switch (lpf) {
            case 1: cons_fibers<T, 1, 1>(X, S, f0, f1, z, m); break;
            case 2: cons_fibers<T, 1, 2>(X, S, f0, f1, z, m); break;
            case 4: cons_fibers<T, 1, 4>(X, S, f0, f1, z, m); break;
            case 8: cons_fibers<T, 1, 8>(X, S, f0, f1, z, m); break;
            case 16: cons_fibers<T, 1, 16>(X, S, f0, f1, z, m); break;
            default: cons_fibers<T, 1, 32>(X, S, f0, f1, z, m); break;
        }
    } else {
        switch (lpf) {
            case 1: cons_fibers<T, V, 1>(X, S, f0, f1, z, m); break;
            case 2: cons_fibers<T, V, 2>(X, S, f0, f1, z, m); break;
            case 4: cons_fibers<T, V, 4>(X, S, f0, f1, z, m); break;
            case 8: cons_fibers<T, V, 8>(X, S, f0, f1, z, m); break;
            case 16: cons_fibers<T, V, 16>(X, S, f0, f1, z, m); break;
            default: cons_fibers<T, V, 32>(X, S, f0, f1, z, m); break;
        }
    }
}

// One fiber block (of block_off's numbering) per CTA: each instance has its own
// output word, so the atomics are spread over the instances.
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
    double m = 0.0;
    cons_fibers_rt<T>(static_cast<const T*>(in.X), static_cast<const T*>(in.S), f0,
                      min(in.nf, f0 + per), in.z, in.pad, in.lpf, m);
    cons_block_max(m, in.out);
}

template <typename T, int VEC, int LPF>
void launch_one(const T* X, const T* S, long long nf, long long z, long long nb, int sms,
                unsigned long long* out, cudaStream_t st) {
    // one wave of resident CTAs, each looping over fiber blocks
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, conservation_kernel<T, VEC, LPF>,
                                                      kConsThreads, 0) != cudaSuccess ||
        per_sm < 1)
        per_sm = 1;
    const unsigned grid = unsigned(std::min<long long>(nb, (long long)std::max(sms, 1) * per_sm));
    conservation_kernel<T, VEC, LPF><<<grid, kConsThreads, 0, st>>>(X, S, nf, z, nb, out);
}

template <typename T, int VEC>
void launch_lpf(const T* X, const T* S, long long nf, long long z, long long nb, int lpf, int sms,
                unsigned long long* out, cudaStream_t st) {
    switch (lpf) {
        case 1: launch_one<T, VEC, 1>(X, S, nf, z, nb, sms, out, st); break;
        case 2: launch_one<T, VEC, 2>(X, S, nf, z, nb, sms, out, st); break;
        case 4: launch_one<T, VEC, 4>(X, S, nf, z, nb, sms, out, st); break;
        case 8: launch_one<T, VEC, 8>(X, S, nf, z, nb, sms, out, st); break;
        case 16: launch_one<T, VEC, 16>(X, S, nf, z, nb, sms, out, st); break;
        default: launch_one<T, VEC, 32>(X, S, nf, z, nb, sms, out, st); break;
    }
}

}  // namespace

int conservation_blocks(int dtype, const void* dS, long long nf, long long z) {
    const size_t es = dtype == BLDM_F64 ? 8 : 4;
    const long long per = fibers_per_block(lpf_of(z, vec_of(dS, z, es)));
    return int((nf + per - 1) / per);
}

int launch_conservation(int dtype, const void* dX, const void* dS, long long nf, long long z,
                        unsigned long long* out, cudaStream_t st) {
    if (nf <= 0 || z <= 0) return BLDM_OK;
    const size_t es = dtype == BLDM_F64 ? 8 : 4;
    const int vec = vec_of(dS, z, es);
    const int lpf = lpf_of(z, vec);
    const long long nb = conservation_blocks(dtype, dS, nf, z);
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess)
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (dtype == BLDM_F64) {
        const double* X = static_cast<const double*>(dX);
        const double* S = static_cast<const double*>(dS);
        if (vec == 2)
            launch_lpf<double, 2>(X, S, nf, z, nb, lpf, sms, out, st);
        else
            launch_lpf<double, 1>(X, S, nf, z, nb, lpf, sms, out, st);
    } else {
        const float* X = static_cast<const float*>(dX);
        const float* S = static_cast<const float*>(dS);
        if (vec == 4)
            launch_lpf<float, 4>(X, S, nf, z, nb, lpf, sms, out, st);
        else
            launch_lpf<float, 1>(X, S, nf, z, nb, lpf, sms, out, st);
    }
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

// ConsInst of one instance (lane layout from its depth and S's alignment; pad
// holds the elements per vector load, 1 or 16 bytes' worth).
ConsInst cons_inst(int dtype, const void* X, const void* S, long long nf, long long z,
                   unsigned long long* out) {
    const size_t es = dtype == BLDM_F64 ? 8 : 4;
    ConsInst c;
    c.X = X;
    c.S = S;
    c.nf = nf;
    c.z = z;
    c.out = out;
    c.pad = vec_of(S, z, es);
    c.lpf = lpf_of(z, c.pad);
    return c;
}

double cons_value(unsigned long long bits) {
    double v;
    static_assert(sizeof v == sizeof bits, "64-bit double");
    memcpy(&v, &bits, sizeof v);
    return v;
}

}  // namespace bldm
