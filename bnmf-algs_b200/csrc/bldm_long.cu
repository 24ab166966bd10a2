// Long fibers: the update for depths z beyond the fused sweep's lane layout.
//
// The fused sweep holds one fiber S(i,j,:) in the registers of one lane group
// (at most 32 lanes x 8 chunks x one 16-byte vector: 512 FP64 / 1024 FP32
// elements, 256 for odd z).  The reference accepts any depth: its kernels loop k
// over the whole fiber (cuda_src/bld_mult/bld_mult_cuda_kernels.cu:120-159,
// 203-255).  For longer fibers an iteration here is two passes over S:
//
//   long_fiber_sums_kernel  one warp per fiber: the three fiber sums the update
//                           needs before it can change any element,
//                             S_ij+ = sum_k S,  an = sum_k S gm(i,k),
//                             ad = sum_k S gp(i,j,k),
//                           with gp = psi(beta_eph(j,k)) - psi(S+1) and
//                           gm = psi(sum_i alpha_eph(i,k)) - psi(alpha_eph(i,k))
//                           (update_nom / update_denom, bld_mult_funcs.hpp:242-290);
//   long_sweep_kernel       tiles of (k-chunk of 256, band of kLongBand columns,
//                           row range): each thread owns one k of the chunk,
//                           applies update_S (bld_mult_funcs.hpp:307-327) to the
//                           band's fibers row by row, and accumulates the new
//                           tensor's S_+jk (over the tile's rows) and S_i+k (over
//                           the band) partials in the fused sweep's layout, so
//                           the same finalize kernel sums them.  With UPDATE =
//                           false it only accumulates the sums of S (the start
//                           of a solve).
//
// HBM traffic per iteration: S read twice and written once (1.5x the fused
// sweep) plus the partials, 1/kLongBand of S in FP64 each way.  Fibers whose X
// is zero skip the digamma arithmetic (their update is zero), warp- or
// block-uniformly.
#include "bldm_device.cuh"
#include "bldm_internal.h"
#include "bldm_kernels.h"

namespace bldm {

namespace {

template <typename T>
__device__ __forceinline__ T psi_plus(T v);
template <>
__device__ __forceinline__ double psi_plus<double>(double v) { return psi_appr_f64(v); }
template <>
__device__ __forceinline__ float psi_plus<float>(float v) { return psi_f32(v); }

template <typename T, bool APPR>
__device__ __forceinline__ T psi_of(T v) {
    if (sizeof(T) == 8 && !APPR) return T(psi_exact_f64(double(v)));
    return psi_plus<T>(v);
}

template <typename T, bool APPR>
__global__ void __launch_bounds__(kLongThreads) long_fiber_sums_kernel(const LongSweepParams<T> p) {
    grid_dep_wait();  // S and the digamma tables of the previous kernels
    const long long f = ((long long)blockIdx.x * kLongThreads + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (f >= p.x * p.y) return;  // warp-uniform
    const long long i = f / p.y, j = f % p.y;
    double as = 0.0, an = 0.0, ad = 0.0;
    // a fiber with X == 0 updates to zero: its sums are not needed
    if (p.X[f] != T(0)) {
        const T* s = p.S + f * p.z;
        const T* pa = p.psiA + i * p.z;
        const T* pb = p.psiB + j * p.z;
        for (long long k = lane; k < p.z; k += 32) {
            const T e = s[k];
            const T gm = p.psiAS[k] - pa[k];
            const T gp = pb[k] - psi_of<T, APPR>(e + T(1));
            as += double(e);
            an += double(e) * double(gm);
            ad += double(e) * double(gp);
        }
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            as += __shfl_xor_sync(0xffffffffu, as, o);
            an += __shfl_xor_sync(0xffffffffu, an, o);
            ad += __shfl_xor_sync(0xffffffffu, ad, o);
        }
    }
    if (lane == 0) p.fsum[f] = make_double4(as, an, ad, 0.0);
}

template <typename T, bool UPDATE, bool APPR>
__global__ void __launch_bounds__(kLongThreads, 2) long_sweep_kernel(const LongSweepParams<T> p) {
    grid_dep_wait();
    const int tile = int(blockIdx.x);
    const int kc = tile % p.n_kc;
    const int rest = tile / p.n_kc;
    const int band = rest % p.n_bands;
    const int rr = rest / p.n_bands;
    const long long z = p.z;
    const long long k = (long long)kc * kLongThreads + threadIdx.x;
    const bool kon = k < z;
    const long long c0 = (long long)band * kLongBand;
    const int cw = int(min((long long)kLongBand, p.y - c0));
    const long long r0 = (long long)rr * p.rr_base + min(rr, p.rr_extra);
    const int nrows = int(min((long long)(p.rr_base + (rr < p.rr_extra ? 1 : 0)), p.x - r0));
    const T teps = T(p.eps);
    const T sAS = (UPDATE && kon) ? p.psiAS[k] : T(0);
    double pj[kLongBand];
#pragma unroll
    for (int c = 0; c < kLongBand; ++c) pj[c] = 0.0;
    for (int r = 0; r < nrows; ++r) {
        const long long i = r0 + r;
        // every fiber of the row's band segment at this thread's k, loads first
        T s[kLongBand];
#pragma unroll
        for (int c = 0; c < kLongBand; ++c)
            s[c] = (kon && c < cw) ? p.S[((i * p.y) + c0 + c) * z + k] : T(0);
        double ip = 0.0;
        if (UPDATE) {
            const T gm = kon ? sAS - p.psiA[i * z + k] : T(0);
#pragma unroll
            for (int c = 0; c < kLongBand; ++c) {
                if (c >= cw) break;
                const long long f = i * p.y + c0 + c;
                const T xe = p.X[f];  // block-uniform
                T sn = T(0);
                if (xe != T(0)) {
                    const double4 fs = p.fsum[f];
                    const T as = T(fs.x), an = T(fs.y), ad = T(fs.z);
                    const T be = kon ? p.psiB[(c0 + c) * z + k] : T(0);
                    const T gp = be - psi_of<T, APPR>(s[c] + T(1));
                    const T xr = Rcp<T>::of(xe + teps);
                    const T nom = an * xr;
                    const T den = ad * xr + teps;
                    const T xos = xe * Rcp<T>::of(as + teps);
                    sn = (as == T(0)) ? T(0)
                                      : s[c] * (((gp + nom) * xos) * Rcp<T>::of(gm + den));
                }
                if (kon) p.S[f * z + k] = sn;
                pj[c] += double(sn);
                ip += double(sn);
            }
        } else {
#pragma unroll
            for (int c = 0; c < kLongBand; ++c) {
                pj[c] += double(s[c]);
                ip += double(s[c]);
            }
        }
        if (kon) p.part_ipk[((long long)band * p.x + i) * z + k] = ip;
    }
    if (kon)
#pragma unroll
        for (int c = 0; c < kLongBand; ++c)
            if (c < cw) p.part_pjk[((long long)rr * p.y + c0 + c) * z + k] = pj[c];
}

template <typename T>
int launch_long_typed(const LongSweepParams<T>& p, bool update, bool appr, bool pdl,
                      cudaStream_t st, uint64_t* launches) {
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    auto launch = [&](auto fn, unsigned grid) {
        cudaLaunchConfig_t lc = {};
        lc.gridDim = dim3(grid);
        lc.blockDim = dim3(kLongThreads);
        lc.dynamicSmemBytes = 0;
        lc.stream = st;
        lc.attrs = pdl ? attr : nullptr;
        lc.numAttrs = pdl ? 1 : 0;
        return cudaLaunchKernelEx(&lc, fn, p);
    };
    const unsigned tiles = unsigned(p.n_kc) * unsigned(p.n_bands) * unsigned(p.n_rr);
    cudaError_t e = cudaSuccess;
    if (update) {
        const long long nf = p.x * p.y;
        const unsigned gs = unsigned((nf * 32 + kLongThreads - 1) / kLongThreads);
        e = appr ? launch(long_fiber_sums_kernel<T, true>, gs)
                 : launch(long_fiber_sums_kernel<T, false>, gs);
        if (e == cudaSuccess)
            e = appr ? launch(long_sweep_kernel<T, true, true>, tiles)
                     : launch(long_sweep_kernel<T, true, false>, tiles);
        *launches += 2;
    } else {
        e = launch(long_sweep_kernel<T, false, true>, tiles);
        *launches += 1;
    }
    return cuda_status(e);
}

}  // namespace

int launch_long_sweep(int dtype, const void* params, bool update, bool appr, bool pdl,
                      cudaStream_t st, uint64_t* launches) {
    if (dtype == BLDM_F64)
        return launch_long_typed<double>(*static_cast<const LongSweepParams<double>*>(params),
                                         update, appr, pdl, st, launches);
    return launch_long_typed<float>(*static_cast<const LongSweepParams<float>*>(params), update,
                                    appr, pdl, st, launches);
}

}  // namespace bldm
