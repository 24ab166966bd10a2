// Fused multiplicative-update sweep over the allocation tensor S.
//
// One iteration of the reference (src/bld/bld_mult/bld_mult.hpp:123-147;
// stage formulas in bld_mult_funcs.hpp:130-327) is two launches here:
//
//   sweep<UPDATE>  reads every fiber S(i,j,:) once from HBM (bulk copies of a
//                  row segment into a shared-memory ring), computes
//                  S_ijp = sum_k S, psi(S+1), grad_plus, nom and denom in
//                  registers with lane-group shuffles, applies update_S, writes
//                  the fiber once, and accumulates the NEW tensor's axis sums
//                  S_pjk (over the CTA's rows) and S_ipk (over the CTA's band
//                  of columns) as deterministic per-region partials;
//   finalize       sums the partials in a fixed order, forms beta_eph and
//                  alpha_eph, and tabulates psi(beta_eph) (y*z), psi(alpha_eph)
//                  (x*z) and psi(sum_i alpha_eph) (z) for the next sweep, which
//                  rebuilds grad_minus(i,k) = psi(sum) - psi(alpha_eph) per row.
//
// HBM traffic per iteration is one read and one write of S plus one read of X
// and the small partial/table arrays, against eleven S-sized passes in the
// reference GPU path (tensor_sums 3, grad_plus 2, denom 2, nom 1, update_S 3).
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>

#include "bldm_device.cuh"
#include "bldm_internal.h"

namespace bldm {

constexpr int kSweepWarps = 8;
constexpr int kSweepThreads = kSweepWarps * 32;
constexpr int kFinThreads = 256;

// fiber passes per warp per row, from the bytes a lane holds per fiber
__host__ __device__ constexpr int cpw_for(int bytes) { return bytes <= 16 ? 4 : (bytes <= 32 ? 2 : 1); }

template <typename T> struct SweepParams {
    T* S;
    const T* X;
    const T* psiB;   // psi(beta_eph) [y][z]
    const T* psiA;   // psi(alpha_eph) [x][z]
    const T* psiAS;  // psi(sum_i alpha_eph) [z]
    double* part_pjk;
    double* part_ipk;
    int* err;
    long long x, y, z;
    int n_bands, band_w, rr_base, rr_extra, stages;
    uint32_t capS, capX, stage_bytes;
    double eps;
};

template <typename T, int VEC> struct VecIO {
    __device__ __forceinline__ static void load(const T* p, T (&v)[VEC]) {
#pragma unroll
        for (int e = 0; e < VEC; ++e) v[e] = p[e];
    }
    __device__ __forceinline__ static void store(T* p, const T (&v)[VEC]) {
#pragma unroll
        for (int e = 0; e < VEC; ++e) __stcs(p + e, v[e]);
    }
};
template <> struct VecIO<double, 2> {
    __device__ __forceinline__ static void load(const double* p, double (&v)[2]) {
        const double2 t = *reinterpret_cast<const double2*>(p);
        v[0] = t.x;
        v[1] = t.y;
    }
    __device__ __forceinline__ static void store(double* p, const double (&v)[2]) {
        __stcs(reinterpret_cast<double2*>(p), make_double2(v[0], v[1]));
    }
};
template <> struct VecIO<float, 4> {
    __device__ __forceinline__ static void load(const float* p, float (&v)[4]) {
        const float4 t = *reinterpret_cast<const float4*>(p);
        v[0] = t.x;
        v[1] = t.y;
        v[2] = t.z;
        v[3] = t.w;
    }
    __device__ __forceinline__ static void store(float* p, const float (&v)[4]) {
        __stcs(reinterpret_cast<float4*>(p), make_float4(v[0], v[1], v[2], v[3]));
    }
};

__device__ __forceinline__ uintptr_t align_down16(uintptr_t a) { return a & ~uintptr_t(15); }
__device__ __forceinline__ uintptr_t align_up16(uintptr_t a) {
    return (a + 15) & ~uintptr_t(15);
}

// Block layout: blockIdx.x = rr * n_bands + band.  Lane layout: lane = g*LPF+q
// handles fiber slot g of the warp and elements k = (m*LPF + q)*VEC + v.
template <typename T, int VEC, int LPF, int MCH, bool UPDATE, bool APPR>
__global__ void __launch_bounds__(kSweepThreads, 2) sweep_kernel(const SweepParams<T> p) {
    constexpr int NW = kSweepWarps;
    constexpr int FPW = 32 / LPF;
    constexpr int CPW = cpw_for(MCH * VEC * int(sizeof(T)));
    extern __shared__ __align__(128) unsigned char smem[];

    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int g = lane / LPF;
    const int q = lane % LPF;

    const int band = blockIdx.x % p.n_bands;
    const int rr = blockIdx.x / p.n_bands;
    const long long z = p.z;
    const long long c0 = (long long)band * p.band_w;
    const int cw = (int)min((long long)p.band_w, p.y - c0);
    const long long r0 = (long long)rr * p.rr_base + min(rr, p.rr_extra);
    const int nrows = p.rr_base + (rr < p.rr_extra ? 1 : 0);

    unsigned char* stage0 = smem;
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + (size_t)p.stages * p.stage_bytes);
    double* red = reinterpret_cast<double*>(bars + 8);         // [stages][NW][z]
    T* sAS = reinterpret_cast<T*>(red + (size_t)p.stages * NW * z);  // [z]
    __shared__ int cnt[8];  // per-stage arrivals of warps (monotonic)

    if (tid == 0) {
        for (int s = 0; s < p.stages; ++s) mbar_init(&bars[s], 1);
        mbar_fence_init();
    }
    if (tid < 8) cnt[tid] = 0;
    __shared__ double2 ltab[kLogTabN];  // ln table of the FP64 digamma
    if (UPDATE) {
        for (long long k = tid; k < z; k += kSweepThreads) sAS[k] = p.psiAS[k];
        if (sizeof(T) == 8 && APPR) log_tab_init(ltab, tid, kSweepThreads);
    }
    __syncthreads();

    const uint64_t pol_stream = policy_evict_first();
    const uint64_t pol_keep = policy_evict_last();

    // Stage t holds row r0+t: the S segment of the band, the X segment and
    // (UPDATE) the psi(alpha_eph) row, each copied as its enclosing
    // 16-byte-aligned byte range.
    auto issue = [&](int t) {
        const long long i = r0 + t;
        const int s = t % p.stages;
        unsigned char* st = stage0 + (size_t)s * p.stage_bytes;
        const uintptr_t aS = reinterpret_cast<uintptr_t>(p.S + (i * p.y + c0) * z);
        const uintptr_t loS = align_down16(aS);
        const uintptr_t hiS = align_up16(aS + (uintptr_t)cw * z * sizeof(T));
        const uintptr_t aX = reinterpret_cast<uintptr_t>(p.X + i * p.y + c0);
        const uintptr_t loX = align_down16(aX);
        const uintptr_t hiX = align_up16(aX + (uintptr_t)cw * sizeof(T));
        uint32_t tot = uint32_t(hiS - loS) + uint32_t(hiX - loX);
        uintptr_t loA = 0, hiA = 0;
        if (UPDATE) {
            const uintptr_t aA = reinterpret_cast<uintptr_t>(p.psiA + i * z);
            loA = align_down16(aA);
            hiA = align_up16(aA + (uintptr_t)z * sizeof(T));
            tot += uint32_t(hiA - loA);
        }
        mbar_arrive_expect_tx(&bars[s], tot);
        bulk_g2s(st, reinterpret_cast<const void*>(loS), uint32_t(hiS - loS), &bars[s],
                 pol_stream);
        bulk_g2s(st + p.capS, reinterpret_cast<const void*>(loX), uint32_t(hiX - loX), &bars[s],
                 pol_keep);
        if (UPDATE)
            bulk_g2s(st + p.capS + p.capX, reinterpret_cast<const void*>(loA),
                     uint32_t(hiA - loA), &bars[s], pol_keep);
    };

    if (tid == 0) {
        const int n0 = min(p.stages, nrows);
        for (int t = 0; t < n0; ++t) issue(t);
    }

    // Per-lane constants for the band: psi(beta_eph) of the lane's fibers.
    T pB[CPW][MCH][VEC];
    Acc<T> pj[CPW][MCH][VEC];
#pragma unroll
    for (int c = 0; c < CPW; ++c) {
        const int jl = (warp * CPW + c) * FPW + g;
#pragma unroll
        for (int m = 0; m < MCH; ++m) {
#pragma unroll
            for (int v = 0; v < VEC; ++v) {
                const long long k = (long long)(m * LPF + q) * VEC + v;
                pj[c][m][v].init();
                if (UPDATE)
                    pB[c][m][v] = (jl < cw && k < z) ? p.psiB[(c0 + jl) * z + k] : T(0);
            }
        }
    }

    for (int t = 0; t < nrows; ++t) {
        const int s = t % p.stages;
        // warp-uniform: the lane-group shuffles below need every lane of the warp
        const bool ok =
            __all_sync(0xffffffffu, mbar_wait_bounded(&bars[s], (uint32_t)((t / p.stages) & 1)));
        if (!ok) {
            // Give up: flag the error and wait (bounded) for the copies that
            // may still be landing in this CTA's shared memory.
            if (lane == 0) {
                atomicOr(p.err, DEV_ERR_WAIT_TIMEOUT);
                const int issued = min(nrows, t + p.stages);
                for (int u = t; u < issued; ++u)
                    (void)mbar_wait_bounded(&bars[u % p.stages], (uint32_t)((u / p.stages) & 1));
            }
            return;
        }
        const long long i = r0 + t;
        const unsigned char* st = stage0 + (size_t)s * p.stage_bytes;
        const uintptr_t aS = reinterpret_cast<uintptr_t>(p.S + (i * p.y + c0) * z);
        const uintptr_t aX = reinterpret_cast<uintptr_t>(p.X + i * p.y + c0);
        const T* sS = reinterpret_cast<const T*>(st + (aS & 15));
        const T* sX = reinterpret_cast<const T*>(st + p.capS + (aX & 15));

        T gm[MCH][VEC];
        if (UPDATE) {
            const uintptr_t aA = reinterpret_cast<uintptr_t>(p.psiA + i * z);
            const T* sA = reinterpret_cast<const T*>(st + p.capS + p.capX + (aA & 15));
#pragma unroll
            for (int m = 0; m < MCH; ++m)
#pragma unroll
                for (int v = 0; v < VEC; ++v) {
                    const long long k = (long long)(m * LPF + q) * VEC + v;
                    gm[m][v] = (k < z) ? sAS[k] - sA[k] : T(0);
                }
        }

        Acc<T> ip[MCH][VEC];
#pragma unroll
        for (int m = 0; m < MCH; ++m)
#pragma unroll
            for (int v = 0; v < VEC; ++v) ip[m][v].init();

        if (ok) {
            T sv[CPW][MCH][VEC];
            T xv[CPW];
#pragma unroll
            for (int c = 0; c < CPW; ++c) {
                const int jl = (warp * CPW + c) * FPW + g;
                const bool fv = jl < cw;
#pragma unroll
                for (int m = 0; m < MCH; ++m) {
                    const long long k0 = (long long)(m * LPF + q) * VEC;
                    // VEC > 1 only when z*sizeof(T) is a multiple of 16, so a
                    // chunk is entirely inside or entirely outside the fiber.
                    if (fv && k0 < z) {
                        VecIO<T, VEC>::load(sS + (long long)jl * z + k0, sv[c][m]);
                    } else {
#pragma unroll
                        for (int v = 0; v < VEC; ++v) sv[c][m][v] = T(0);
                    }
                }
                xv[c] = (UPDATE && fv) ? sX[jl] : T(0);
            }
            if (UPDATE) {
                const T teps = T(p.eps);
#pragma unroll
                for (int c = 0; c < CPW; ++c) {
                    const int jl = (warp * CPW + c) * FPW + g;
                    const bool fv = jl < cw;
                    T sn[MCH][VEC];
                    // A fiber with X == 0 updates to zero whatever its digamma
                    // values (the reference formula multiplies by X/(S_ijp+eps));
                    // a pass whose fibers all have X == 0 skips the arithmetic.
                    if (__any_sync(0xffffffffu, xv[c] != T(0))) {
                        T arg[MCH * VEC], ps[MCH * VEC];
#pragma unroll
                        for (int m = 0; m < MCH; ++m)
#pragma unroll
                            for (int v = 0; v < VEC; ++v) arg[m * VEC + v] = sv[c][m][v] + T(1);
                        PsiPass<T, APPR>::template run<MCH * VEC>(arg, ps, ltab);
                        T gp[MCH][VEC];
                        T as = T(0), an = T(0), ad = T(0);
#pragma unroll
                        for (int m = 0; m < MCH; ++m)
#pragma unroll
                            for (int v = 0; v < VEC; ++v) {
                                const T e = sv[c][m][v];
                                gp[m][v] = pB[c][m][v] - ps[m * VEC + v];
                                as += e;
                                an += e * gm[m][v];
                                ad += e * gp[m][v];
                            }
                        as = group_sum<LPF>(as);
                        an = group_sum<LPF>(an);
                        ad = group_sum<LPF>(ad);
                        const T xr = T(1) / (xv[c] + teps);
                        const T nom = an * xr;
                        const T den = ad * xr + teps;
                        const T xos = xv[c] / (as + teps);
                        // X == 0 (or an all-zero fiber) keeps the fiber at zero: the
                        // reference's FP64 result, and no 0 * inf in FP32 where
                        // eps = 1e-50 underflows to zero.
                        const bool zero = (xv[c] == T(0)) || (as == T(0));
#pragma unroll
                        for (int m = 0; m < MCH; ++m)
#pragma unroll
                            for (int v = 0; v < VEC; ++v)
                                sn[m][v] = zero ? T(0)
                                                : sv[c][m][v] * (((gp[m][v] + nom) * xos) *
                                                                 Rcp<T>::of(gm[m][v] + den));
                    } else {
#pragma unroll
                        for (int m = 0; m < MCH; ++m)
#pragma unroll
                            for (int v = 0; v < VEC; ++v) sn[m][v] = T(0);
                    }
#pragma unroll
                    for (int m = 0; m < MCH; ++m) {
#pragma unroll
                        for (int v = 0; v < VEC; ++v) {
                            pj[c][m][v].add(sn[m][v]);
                            ip[m][v].add(sn[m][v]);
                        }
                        const long long k0 = (long long)(m * LPF + q) * VEC;
                        if (fv && k0 < z)
                            VecIO<T, VEC>::store(p.S + ((i * p.y + c0 + jl) * z + k0), sn[m]);
                    }
                }
            } else {
#pragma unroll
                for (int c = 0; c < CPW; ++c)
#pragma unroll
                    for (int m = 0; m < MCH; ++m)
#pragma unroll
                        for (int v = 0; v < VEC; ++v) {
                            pj[c][m][v].add(sv[c][m][v]);
                            ip[m][v].add(sv[c][m][v]);
                        }
            }
        }

        // S_ipk partial of row i over this band: fiber slots -> warp -> red[s][warp].
        double* redw = red + ((size_t)s * NW + warp) * z;
#pragma unroll
        for (int m = 0; m < MCH; ++m)
#pragma unroll
            for (int v = 0; v < VEC; ++v) {
                double val = ip[m][v].value();
                if (FPW > 1) val = cross_group_sum<LPF>(val);
                const long long k = (long long)(m * LPF + q) * VEC + v;
                if (g == 0 && k < z) redw[k] = val;
            }
        __syncwarp();
        // No CTA barrier per row: each warp counts itself done with stage s;
        // the last of the NW warps (the count reaches a multiple of NW) adds the
        // warps' partials in warp order, writes the S_ipk partial of row i and
        // refills the stage.  Warps drift apart by up to `stages` rows.
        int last = 0;
        if (lane == 0) {
            __threadfence_block();
            last = (atomicAdd(&cnt[s], 1) == (t / p.stages + 1) * NW - 1) ? 1 : 0;
        }
        last = __shfl_sync(0xffffffffu, last, 0);
        if (last) {
            __threadfence_block();
            const double* reds = red + (size_t)s * NW * z;
            for (long long k = lane; k < z; k += 32) {
                double sum = 0.0;
#pragma unroll
                for (int w = 0; w < NW; ++w) sum += reds[(size_t)w * z + k];
                p.part_ipk[((long long)band * p.x + i) * z + k] = sum;
            }
            __syncwarp();
            if (lane == 0 && t + p.stages < nrows) issue(t + p.stages);
        }
    }

    // S_pjk partial of the band over this CTA's rows: each (j,k) has one owner.
#pragma unroll
    for (int c = 0; c < CPW; ++c) {
        const int jl = (warp * CPW + c) * FPW + g;
#pragma unroll
        for (int m = 0; m < MCH; ++m)
#pragma unroll
            for (int v = 0; v < VEC; ++v) {
                const long long k = (long long)(m * LPF + q) * VEC + v;
                if (jl < cw && k < z)
                    p.part_pjk[((long long)rr * p.y + c0 + jl) * z + k] = pj[c][m][v].value();
            }
    }
}

template <typename T> struct FinParams {
    const double* part_pjk;
    const double* part_ipk;
    const double* alpha;
    const double* beta;
    T* psiB;
    T* psiA;
    T* psiAS;
    double* asum_part;
    unsigned* counter;
    long long x, y, z;
    int n_rr, n_bands, nbB, n_ablk, rows_per_ablk;
    int plus_appr, minus_appr;
};

// Blocks [0, nbB): psi(beta_eph) for every (j,k).  Blocks [nbB, nbB+n_ablk):
// psi(alpha_eph) for a block of rows plus that block's sum of alpha_eph over
// rows; the last block to finish sums the block sums in order and tabulates
// psi(sum_i alpha_eph(i,k)).
template <typename T>
__global__ void __launch_bounds__(kFinThreads) finalize_kernel(const FinParams<T> p) {
    const long long z = p.z;
    const int tid = threadIdx.x;
    if ((int)blockIdx.x < p.nbB) {
        const long long idx = (long long)blockIdx.x * kFinThreads + tid;
        if (idx < p.y * z) {
            const long long k = idx % z;
            double s = 0.0;
            for (int r = 0; r < p.n_rr; ++r) s += p.part_pjk[(long long)r * p.y * z + idx];
            p.psiB[idx] = T(psi_mode_f64(s + p.beta[k], p.plus_appr != 0));
        }
        return;
    }
    __shared__ double acc[1024];
    __shared__ unsigned last;
    const int b = (int)blockIdx.x - p.nbB;
    const long long i0 = (long long)b * p.rows_per_ablk;
    const long long i1 = min(p.x, i0 + p.rows_per_ablk);
    const int KT = (int)min(z, (long long)kFinThreads);
    const int R = kFinThreads / KT;
    const int sub = tid / KT;
    if (sub < R) {
        for (long long k = tid % KT; k < z; k += KT) {
            double a = 0.0;
            for (long long i = i0 + sub; i < i1; i += R) {
                double s = 0.0;
                for (int bd = 0; bd < p.n_bands; ++bd)
                    s += p.part_ipk[((long long)bd * p.x + i) * z + k];
                const double ae = s + p.alpha[i];
                p.psiA[i * z + k] = T(psi_mode_f64(ae, p.minus_appr != 0));
                a += ae;
            }
            acc[sub * z + k] = a;
        }
    }
    __syncthreads();
    for (long long k = tid; k < z; k += kFinThreads) {
        double a = 0.0;
        for (int r = 0; r < R; ++r) a += acc[r * z + k];
        p.asum_part[(long long)b * z + k] = a;
    }
    __threadfence();
    __syncthreads();
    if (tid == 0) last = (atomicAdd(p.counter, 1u) == (unsigned)(p.n_ablk - 1)) ? 1u : 0u;
    __syncthreads();
    if (last) {
        __threadfence();
        for (long long k = tid; k < z; k += kFinThreads) {
            double a = 0.0;
            for (int bb = 0; bb < p.n_ablk; ++bb) a += __ldcg(&p.asum_part[(long long)bb * z + k]);
            p.psiAS[k] = T(psi_mode_f64(a, p.minus_appr != 0));
        }
        if (tid == 0) *p.counter = 0u;
    }
}

// Seeded initial S: S(i,j,:) = X(i,j) * Dirichlet(1_z), the Dirichlet draw
// being normalised Exp(1) variates of a SplitMix64 counter hash.
__device__ __forceinline__ uint64_t splitmix64(uint64_t v) {
    v += 0x9E3779B97F4A7C15ull;
    v = (v ^ (v >> 30)) * 0xBF58476D1CE4E5B9ull;
    v = (v ^ (v >> 27)) * 0x94D049BB133111EBull;
    return v ^ (v >> 31);
}
__device__ __forceinline__ double exp1_variate(uint64_t hseed, uint64_t fiber, uint64_t k) {
    const uint64_t h = splitmix64(hseed ^ splitmix64(fiber * 0x100000001B3ull + k));
    const double u = (double(h >> 11) + 0.5) * (1.0 / 9007199254740992.0);
    return -log(u);
}

template <typename T>
__global__ void init_S_kernel(const T* X, T* S, long long nf, long long z, uint64_t seed) {
    const long long f = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (f >= nf) return;
    const uint64_t hs = splitmix64(seed ^ 0x5DEECE66Dull);
    double tot = 0.0;
    for (long long k = 0; k < z; ++k) tot += exp1_variate(hs, (uint64_t)f, (uint64_t)k);
    const double xv = double(X[f]);
    for (long long k = 0; k < z; ++k)
        S[f * z + k] = T(xv * (exp1_variate(hs, (uint64_t)f, (uint64_t)k) / tot));
}

// ---------------------------------------------------------------------------
// Host side.
// ---------------------------------------------------------------------------
int cuda_status(cudaError_t e) {
    if (e == cudaSuccess) return BLDM_OK;
    if (e == cudaErrorMemoryAllocation) return BLDM_ERR_OOM;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return BLDM_ERR_NO_DEVICE;
    return BLDM_ERR_CUDA;
}

#define BLDM_CU(call)                                   \
    do {                                                \
        cudaError_t e_ = (call);                        \
        if (e_ != cudaSuccess) return cuda_status(e_);  \
    } while (0)

template <typename T> using SweepFn = void (*)(const SweepParams<T>);

// Instantiated lane shapes: (LPF, MCH) with LPF*MCH a power of two.
#define BLDM_SHAPE_CASES(T, VEC, UPD, APPR)                                      \
    case 1 * 16 + 1: return &sweep_kernel<T, VEC, 1, 1, UPD, APPR>;            \
    case 2 * 16 + 1: return &sweep_kernel<T, VEC, 2, 1, UPD, APPR>;            \
    case 4 * 16 + 1: return &sweep_kernel<T, VEC, 4, 1, UPD, APPR>;            \
    case 8 * 16 + 1: return &sweep_kernel<T, VEC, 8, 1, UPD, APPR>;            \
    case 16 * 16 + 1: return &sweep_kernel<T, VEC, 16, 1, UPD, APPR>;          \
    case 32 * 16 + 1: return &sweep_kernel<T, VEC, 32, 1, UPD, APPR>;          \
    case 32 * 16 + 2: return &sweep_kernel<T, VEC, 32, 2, UPD, APPR>;          \
    case 32 * 16 + 4: return &sweep_kernel<T, VEC, 32, 4, UPD, APPR>;          \
    case 32 * 16 + 8: return &sweep_kernel<T, VEC, 32, 8, UPD, APPR>;

template <typename T, int VEC, bool UPD, bool APPR> SweepFn<T> pick_shape(int lpf, int mch) {
    switch (lpf * 16 + mch) { BLDM_SHAPE_CASES(T, VEC, UPD, APPR) default: return nullptr; }
}

template <typename T> SweepFn<T> pick_sweep(const SweepCfg& c, bool update, bool appr);
template <> SweepFn<double> pick_sweep<double>(const SweepCfg& c, bool update, bool appr) {
    if (c.vec == 2) {
        if (!update) return pick_shape<double, 2, false, true>(c.lpf, c.mch);
        return appr ? pick_shape<double, 2, true, true>(c.lpf, c.mch)
                    : pick_shape<double, 2, true, false>(c.lpf, c.mch);
    }
    if (!update) return pick_shape<double, 1, false, true>(c.lpf, c.mch);
    return appr ? pick_shape<double, 1, true, true>(c.lpf, c.mch)
                : pick_shape<double, 1, true, false>(c.lpf, c.mch);
}
template <> SweepFn<float> pick_sweep<float>(const SweepCfg& c, bool update, bool) {
    if (c.vec == 4) {
        if (!update) return pick_shape<float, 4, false, true>(c.lpf, c.mch);
        return pick_shape<float, 4, true, true>(c.lpf, c.mch);
    }
    if (!update) return pick_shape<float, 1, false, true>(c.lpf, c.mch);
    return pick_shape<float, 1, true, true>(c.lpf, c.mch);
}

static int pow2ceil(long v) {
    int p = 1;
    while (p < v) p <<= 1;
    return p;
}
static size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

static int num_sms_of(int dev) {
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0)
        n = 148;
    return n;
}

static int choose_cfg(SweepCfg& c, size_t x, size_t y, size_t z, size_t es, int num_sms,
                      const bldm_tuning* tune) {
    const bool aligned = (z * es) % 16 == 0;
    c.vec = aligned ? int(16 / es) : 1;
    const long nch = long((z + c.vec - 1) / c.vec);
    if (nch <= 32) {
        c.lpf = pow2ceil(nch);
        c.mch = 1;
    } else {
        c.lpf = 32;
        c.mch = pow2ceil((nch + 31) / 32);
        if (c.mch > 8) return BLDM_ERR_UNSUPPORTED;
    }
    c.cpw = cpw_for(int(c.mch * c.vec * es));
    c.warps = kSweepWarps;
    const int fpw = 32 / c.lpf;
    c.band_w = c.warps * c.cpw * fpw;
    c.n_bands = int((y + c.band_w - 1) / c.band_w);
    c.capS = uint32_t(align_up(size_t(c.band_w) * z * es + 32, 16));
    c.capX = uint32_t(align_up(size_t(c.band_w) * es + 32, 16));
    c.capA = uint32_t(align_up(z * es + 32, 16));
    c.stage_bytes = c.capS + c.capX + c.capA;
    // each stage also owns a [warps][z] slice of S_ipk partials (FP64)
    const size_t per_stage = c.stage_bytes + size_t(kSweepWarps) * z * 8;
    const size_t fixed = 64 + z * es + 128;
    // Shared memory per SM is 228 KB; each CTA also holds 1 KB reserved and
    // the 2 KB static log table.  Registers (<= 128 per thread) allow at most
    // two 256-thread CTAs per SM.
    int cps = (tune && tune->ctas_per_sm > 0) ? tune->ctas_per_sm : 2;
    if (cps > 2) return BLDM_ERR_UNSUPPORTED;
    const size_t budget = (cps == 2 ? 110 : 220) * 1024;
    long st = budget > fixed ? long((budget - fixed) / per_stage) : 0;
    st = std::min(8L, st);
    if (tune && tune->stages > 0) {
        if (tune->stages > st || tune->stages < 2) return BLDM_ERR_UNSUPPORTED;
        st = tune->stages;
    }
    if (st < 2) {
        if (tune && tune->ctas_per_sm == 2) return BLDM_ERR_UNSUPPORTED;
        // large slabs: one CTA per SM
        cps = 1;
        st = std::min(8L, long((220 * 1024 - fixed) / per_stage));
        if (st < 2) return BLDM_ERR_UNSUPPORTED;
    }
    c.stages = int(st);
    c.smem_update = size_t(c.stages) * per_stage + fixed;
    c.smem_sums = c.smem_update;
    c.ctas_per_sm = cps;
    // Row ranges: fill the resident CTA slots in one wave (a partial second
    // wave of a bandwidth-bound sweep costs a whole tail).
    const long target = long(c.ctas_per_sm) * num_sms;
    long nrr = target / c.n_bands;
    if (tune && tune->row_ranges > 0) nrr = tune->row_ranges;
    nrr = std::max(1L, std::min(long(x), nrr));
    c.n_rr = int(nrr);
    c.rr_base = int(x / nrr);
    c.rr_extra = int(x % nrr);
    // finalize row blocks
    const int KT = int(std::min<size_t>(z, kFinThreads));
    const int R = kFinThreads / KT;
    long rows = std::max<long>(R, long((x + 127) / 128));
    c.rows_per_ablk = int(rows);
    c.n_ablk = int((x + rows - 1) / rows);
    c.fin_threads = kFinThreads;
    return BLDM_OK;
}

int plan_setup(PlanImpl* p, size_t x, size_t y, size_t z, int dtype, const bldm_tuning* tune) {
    if (x == 0 || y == 0 || z == 0) return BLDM_ERR_BAD_ARG;
    if (z > 1024) return BLDM_ERR_UNSUPPORTED;
    if (dtype != BLDM_F64 && dtype != BLDM_F32) return BLDM_ERR_BAD_ARG;
    BLDM_CU(cudaGetDevice(&p->device));
    p->dtype = dtype;
    p->x = x;
    p->y = y;
    p->z = z;
    p->esize = dtype == BLDM_F64 ? 8 : 4;
    int rc = choose_cfg(p->cfg, x, y, z, p->esize, num_sms_of(p->device), tune);
    if (rc) return rc;
    const SweepCfg& c = p->cfg;
    const size_t a = 256;
    size_t off = 0;
    const size_t o_pjk = off;
    off = align_up(off + size_t(c.n_rr) * y * z * 8, a);
    const size_t o_ipk = off;
    off = align_up(off + size_t(c.n_bands) * x * z * 8, a);
    const size_t o_psiB = off;
    off = align_up(off + y * z * p->esize, a);
    const size_t o_psiA = off;
    off = align_up(off + x * z * p->esize, a);
    const size_t o_psiAS = off;
    off = align_up(off + z * p->esize, a);
    const size_t o_asum = off;
    off = align_up(off + size_t(c.n_ablk) * z * 8, a);
    const size_t o_cnt = off;
    off = align_up(off + 64, a);
    p->ws_bytes = off;
    cudaError_t e = cudaMalloc(&p->ws, p->ws_bytes);
    if (e != cudaSuccess) {
        p->ws = nullptr;
        return cuda_status(e);
    }
    char* base = static_cast<char*>(p->ws);
    p->part_pjk = reinterpret_cast<double*>(base + o_pjk);
    p->part_ipk = reinterpret_cast<double*>(base + o_ipk);
    p->psiB = base + o_psiB;
    p->psiA = base + o_psiA;
    p->psiAS = base + o_psiAS;
    p->asum_part = reinterpret_cast<double*>(base + o_asum);
    p->counter = reinterpret_cast<unsigned*>(base + o_cnt);
    p->err = reinterpret_cast<int*>(base + o_cnt + 16);
    BLDM_CU(cudaMemset(base + o_cnt, 0, 64));
    // Opt the selected kernels into large dynamic shared memory.
    for (int upd = 0; upd < 2; ++upd)
        for (int ap = 0; ap < 2; ++ap) {
            void* fn = nullptr;
            if (dtype == BLDM_F64)
                fn = reinterpret_cast<void*>(pick_sweep<double>(c, upd != 0, ap != 0));
            else
                fn = reinterpret_cast<void*>(pick_sweep<float>(c, upd != 0, ap != 0));
            if (!fn) return BLDM_ERR_UNSUPPORTED;
            BLDM_CU(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         int(c.smem_update)));
        }
    return BLDM_OK;
}

// Lays the plan's workspace out in caller-provided device memory `ws` of
// `ws_cap` bytes instead of allocating it.  Returns BLDM_ERR_TOO_LARGE (and the
// bytes needed in *ws_needed) when the workspace does not fit.  The counter and
// error word are cleared on `st`.
int plan_setup_in(PlanImpl* p, size_t x, size_t y, size_t z, int dtype, void* ws,
                  size_t ws_cap, size_t* ws_needed, cudaStream_t st) {
    if (x == 0 || y == 0 || z == 0 || !ws) return BLDM_ERR_BAD_ARG;
    if (z > 1024) return BLDM_ERR_UNSUPPORTED;
    if (dtype != BLDM_F64 && dtype != BLDM_F32) return BLDM_ERR_BAD_ARG;
    BLDM_CU(cudaGetDevice(&p->device));
    p->dtype = dtype;
    p->x = x;
    p->y = y;
    p->z = z;
    p->esize = dtype == BLDM_F64 ? 8 : 4;
    int rc = choose_cfg(p->cfg, x, y, z, p->esize, num_sms_of(p->device), nullptr);
    if (rc) return rc;
    const SweepCfg& c = p->cfg;
    const size_t a = 256;
    size_t off = 0;
    const size_t o_pjk = off;
    off = align_up(off + size_t(c.n_rr) * y * z * 8, a);
    const size_t o_ipk = off;
    off = align_up(off + size_t(c.n_bands) * x * z * 8, a);
    const size_t o_psiB = off;
    off = align_up(off + y * z * p->esize, a);
    const size_t o_psiA = off;
    off = align_up(off + x * z * p->esize, a);
    const size_t o_psiAS = off;
    off = align_up(off + z * p->esize, a);
    const size_t o_asum = off;
    off = align_up(off + size_t(c.n_ablk) * z * 8, a);
    const size_t o_cnt = off;
    off = align_up(off + 64, a);
    if (ws_needed) *ws_needed = off;
    if (off > ws_cap) return BLDM_ERR_TOO_LARGE;
    p->ws = ws;  // not owned: never pass this plan to plan_free
    p->ws_bytes = off;
    char* base = static_cast<char*>(ws);
    p->part_pjk = reinterpret_cast<double*>(base + o_pjk);
    p->part_ipk = reinterpret_cast<double*>(base + o_ipk);
    p->psiB = base + o_psiB;
    p->psiA = base + o_psiA;
    p->psiAS = base + o_psiAS;
    p->asum_part = reinterpret_cast<double*>(base + o_asum);
    p->counter = reinterpret_cast<unsigned*>(base + o_cnt);
    p->err = reinterpret_cast<int*>(base + o_cnt + 16);
    BLDM_CU(cudaMemsetAsync(base + o_cnt, 0, 64, st));
    for (int upd = 0; upd < 2; ++upd)
        for (int ap = 0; ap < 2; ++ap) {
            void* fn = nullptr;
            if (dtype == BLDM_F64)
                fn = reinterpret_cast<void*>(pick_sweep<double>(c, upd != 0, ap != 0));
            else
                fn = reinterpret_cast<void*>(pick_sweep<float>(c, upd != 0, ap != 0));
            if (!fn) return BLDM_ERR_UNSUPPORTED;
            BLDM_CU(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         int(c.smem_update)));
        }
    return BLDM_OK;
}

void plan_free(PlanImpl* p) {
    if (p->ws) cudaFree(p->ws);
    p->ws = nullptr;
}

template <typename T>
static SweepParams<T> sweep_params(PlanImpl* p, const void* dX, void* dS, double eps) {
    const SweepCfg& c = p->cfg;
    SweepParams<T> s;
    s.S = static_cast<T*>(dS);
    s.X = static_cast<const T*>(dX);
    s.psiB = static_cast<const T*>(p->psiB);
    s.psiA = static_cast<const T*>(p->psiA);
    s.psiAS = static_cast<const T*>(p->psiAS);
    s.part_pjk = p->part_pjk;
    s.part_ipk = p->part_ipk;
    s.err = p->err;
    s.x = (long long)p->x;
    s.y = (long long)p->y;
    s.z = (long long)p->z;
    s.n_bands = c.n_bands;
    s.band_w = c.band_w;
    s.rr_base = c.rr_base;
    s.rr_extra = c.rr_extra;
    s.stages = c.stages;
    s.capS = c.capS;
    s.capX = c.capX;
    s.stage_bytes = c.stage_bytes;
    s.eps = eps;
    return s;
}

template <typename T>
static FinParams<T> fin_params(PlanImpl* p, const double* dalpha, const double* dbeta,
                               int plus_appr, int minus_appr) {
    const SweepCfg& c = p->cfg;
    FinParams<T> f;
    f.part_pjk = p->part_pjk;
    f.part_ipk = p->part_ipk;
    f.alpha = dalpha;
    f.beta = dbeta;
    f.psiB = static_cast<T*>(p->psiB);
    f.psiA = static_cast<T*>(p->psiA);
    f.psiAS = static_cast<T*>(p->psiAS);
    f.asum_part = p->asum_part;
    f.counter = p->counter;
    f.x = (long long)p->x;
    f.y = (long long)p->y;
    f.z = (long long)p->z;
    f.n_rr = c.n_rr;
    f.n_bands = c.n_bands;
    f.nbB = int((p->y * p->z + kFinThreads - 1) / kFinThreads);
    f.n_ablk = c.n_ablk;
    f.rows_per_ablk = c.rows_per_ablk;
    f.plus_appr = plus_appr;
    f.minus_appr = minus_appr;
    return f;
}

template <typename T>
static int run_typed(PlanImpl* p, const void* dX, const double* dalpha, const double* dbeta,
                     void* dS, size_t max_iter, int psi_mode, double eps, cudaStream_t st,
                     cudaEvent_t* ev, size_t nev) {
    const SweepCfg& c = p->cfg;
    const int plus_appr = psi_mode != BLDM_PSI_EXACT;
    const int minus_appr = psi_mode == BLDM_PSI_APPR;
    SweepFn<T> fsum = pick_sweep<T>(c, false, true);
    SweepFn<T> fupd = pick_sweep<T>(c, true, plus_appr != 0);
    if (!fsum || !fupd) return BLDM_ERR_UNSUPPORTED;
    const SweepParams<T> sp = sweep_params<T>(p, dX, dS, eps);
    const FinParams<T> fp = fin_params<T>(p, dalpha, dbeta, plus_appr, minus_appr);
    const dim3 grid_s(unsigned(c.n_bands) * unsigned(c.n_rr));
    const dim3 grid_f(unsigned(fp.nbB + fp.n_ablk));
    fsum<<<grid_s, kSweepThreads, c.smem_sums, st>>>(sp);
    finalize_kernel<T><<<grid_f, kFinThreads, 0, st>>>(fp);
    p->launches += 2;
    for (size_t it = 0; it < max_iter; ++it) {
        if (ev && 2 * it + 1 < nev) cudaEventRecord(ev[2 * it], st);
        fupd<<<grid_s, kSweepThreads, c.smem_update, st>>>(sp);
        if (ev && 2 * it + 1 < nev) cudaEventRecord(ev[2 * it + 1], st);
        p->launches += 1;
        if (it + 1 < max_iter) {
            finalize_kernel<T><<<grid_f, kFinThreads, 0, st>>>(fp);
            p->launches += 1;
        }
    }
    return cuda_status(cudaGetLastError());
}

int plan_run(PlanImpl* p, const void* dX, const double* dalpha, const double* dbeta, void* dS,
             size_t max_iter, int psi_mode, double eps, cudaStream_t st, cudaEvent_t* ev,
             size_t nev) {
    if (!p || !p->ws || !dX || !dalpha || !dbeta || !dS) return BLDM_ERR_BAD_ARG;
    if (psi_mode < 0 || psi_mode > 2) return BLDM_ERR_BAD_ARG;
    if ((reinterpret_cast<uintptr_t>(dX) | reinterpret_cast<uintptr_t>(dS)) & 15)
        return BLDM_ERR_BAD_ARG;
    if (max_iter == 0) return BLDM_OK;
    if (p->dtype == BLDM_F64)
        return run_typed<double>(p, dX, dalpha, dbeta, dS, max_iter, psi_mode, eps, st, ev, nev);
    return run_typed<float>(p, dX, dalpha, dbeta, dS, max_iter, psi_mode, eps, st, ev, nev);
}

int plan_init_S(PlanImpl* p, const void* dX, void* dS, uint64_t seed, cudaStream_t st) {
    const long long nf = (long long)(p->x * p->y);
    const unsigned blocks = unsigned((nf + 255) / 256);
    if (p->dtype == BLDM_F64)
        init_S_kernel<double><<<blocks, 256, 0, st>>>(static_cast<const double*>(dX),
                                                      static_cast<double*>(dS), nf,
                                                      (long long)p->z, seed);
    else
        init_S_kernel<float><<<blocks, 256, 0, st>>>(static_cast<const float*>(dX),
                                                     static_cast<float*>(dS), nf,
                                                     (long long)p->z, seed);
    p->launches += 1;
    return cuda_status(cudaGetLastError());
}

int plan_check(PlanImpl* p, cudaStream_t st) {
    BLDM_CU(cudaStreamSynchronize(st));
    int herr = 0;
    BLDM_CU(cudaMemcpy(&herr, p->err, sizeof(int), cudaMemcpyDeviceToHost));
    if (herr != 0) {
        BLDM_CU(cudaMemset(p->err, 0, sizeof(int)));
        return BLDM_ERR_TIMEOUT;
    }
    return BLDM_OK;
}

}  // namespace bldm
