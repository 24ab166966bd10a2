// The fused sweep kernels (templates).  Instantiated by lane shape in
// bldm_pick_{f64,f32}_{plain,batch}.cu so that they compile in parallel.
#pragma once

#include "bldm_device.cuh"
#include "bldm_finalize.cuh"
#include "bldm_kernels.h"

namespace bldm {

template <typename T, int VEC> struct VecIO {
    __device__ __forceinline__ static void load(const T* p, T (&v)[VEC]) {
#pragma unroll
        for (int e = 0; e < VEC; ++e) v[e] = p[e];
    }
    __device__ __forceinline__ static void store(T* p, const T (&v)[VEC]) {
#pragma unroll
        for (int e = 0; e < VEC; ++e) __stcs(p + e, v[e]);
    }
    // through the read-only data cache
    __device__ __forceinline__ static void ldg(const T* p, T (&v)[VEC]) {
#pragma unroll
        for (int e = 0; e < VEC; ++e) v[e] = __ldg(p + e);
    }
    // from L2, bypassing L1
    __device__ __forceinline__ static void ldcg(const T* p, T (&v)[VEC]) {
#pragma unroll
        for (int e = 0; e < VEC; ++e) v[e] = __ldcg(p + e);
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
    __device__ __forceinline__ static void ldg(const double* p, double (&v)[2]) {
        const double2 t = __ldg(reinterpret_cast<const double2*>(p));
        v[0] = t.x;
        v[1] = t.y;
    }
    __device__ __forceinline__ static void ldcg(const double* p, double (&v)[2]) {
        const double2 t = __ldcg(reinterpret_cast<const double2*>(p));
        v[0] = t.x;
        v[1] = t.y;
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
    __device__ __forceinline__ static void ldg(const float* p, float (&v)[4]) {
        const float4 t = __ldg(reinterpret_cast<const float4*>(p));
        v[0] = t.x;
        v[1] = t.y;
        v[2] = t.z;
        v[3] = t.w;
    }
    __device__ __forceinline__ static void ldcg(const float* p, float (&v)[4]) {
        const float4 t = __ldcg(reinterpret_cast<const float4*>(p));
        v[0] = t.x;
        v[1] = t.y;
        v[2] = t.z;
        v[3] = t.w;
    }
};

__device__ __forceinline__ uintptr_t align_down16(uintptr_t a) { return a & ~uintptr_t(15); }
__device__ __forceinline__ uintptr_t align_up16(uintptr_t a) {
    return (a + 15) & ~uintptr_t(15);
}

// The sweep over one tile (band, row range) of one instance.  Lane layout:
// lane = g*LPF + q handles fiber slot g of its warp and elements
// k = (m*LPF + q)*VEC + v; warp w works on row slot w / wpr and column group
// w % wpr of the band.  Returns false when a bounded wait gave up (the error
// word is set).  COHERENT: psi(beta_eph) through coherent loads instead of the
// read-only cache (a persistent kernel reads tables that other CTAs of the
// same launch rewrote).  FUSED: the tile finalizes its share of the instance in
// its epilogue (tile_finalize) instead of leaving it to a finalize launch.
template <typename T, int VEC, int LPF, int MCH, bool UPDATE, bool APPR, bool BATCH, bool MULTIROW,
          bool COMPACT, bool COHERENT = false, bool FUSED = false>
__device__ __forceinline__ bool sweep_tile(const SweepInst<T>& in, const SweepLaunch& L, int band,
                                           int rr, int tile, unsigned char* smem) {
    constexpr int NW = kSweepWarps;
    constexpr int FPW = 32 / LPF;
    constexpr int CPW = cpw_for(MCH * VEC * int(sizeof(T)));

    const int tid = threadIdx.x;
    const int lane = tid & 31;
    const int warp = tid >> 5;
    const int g = lane / LPF;
    const int q = lane % LPF;
    // MULTIROW == false: one row per stage (wpr == NW), the common wide-row case
    // compiled without the row-slot arithmetic.
    const int wpr = MULTIROW ? in.wpr : NW;
    const int RPS = MULTIROW ? NW / wpr : 1;
    const int rs = MULTIROW ? warp / wpr : 0;      // row slot of this warp
    const int cg = MULTIROW ? warp % wpr : warp;   // column group of this warp

    const long long z = in.z;
    const long long c0 = (long long)band * in.band_w;
    const int cw = (int)min((long long)in.band_w, in.y - c0);
    const long long r0 = (long long)rr * in.rr_base + min(rr, in.rr_extra);
    const int nrows = (int)min((long long)(in.rr_base + (rr < in.rr_extra ? 1 : 0)), in.x - r0);
    const SlotLayout lay(in.band_w, z, int(sizeof(T)));
    // COMPACT (an update after an earlier one has stored the zeros of every
    // fiber with X == 0): zero passes store nothing, and with row lists only
    // the tile's rows whose band segment of X has a nonzero are swept; the
    // others' update is zero and their S_ipk partials are the zeros stored
    // before.
    static_assert(UPDATE || !COMPACT, "compact sweeps are updates");
    const bool compact = COMPACT && in.nz_rows != nullptr;
    constexpr bool clean = COMPACT;

    unsigned char* stage0 = smem;
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + (size_t)L.stages * L.stage_bytes);
    double* red = reinterpret_cast<double*>(bars + 8);                    // [stages][NW][z]
    T* sAS = reinterpret_cast<T*>(red + (size_t)L.stages * NW * z);         // [z]
    __shared__ int cnt[8];             // per-stage arrivals of warps (monotonic)
    __shared__ int srow[8][8];         // compact update: row of (stage, row slot)
    __shared__ int nzr[2];             // compact update: the tile's row-list range
    __shared__ double2 ltab[kLogTabN];  // ln table of the FP64 digamma
    __shared__ double dsum[NW][2];

    if (tid == 0) {
        for (int s = 0; s < L.stages; ++s) mbar_init(&bars[s], 1);
        mbar_fence_init();
    }
    if (tid < 8) cnt[tid] = 0;
    if (UPDATE && sizeof(T) == 8 && APPR) log_tab_init(ltab, tid, kSweepThreads);
    // everything below reads what the previous kernels of the stream wrote
    grid_dep_wait();
    if (compact && tid == 0) {
        const int* cb = in.nz_cnt + (long long)band * (in.x + 1);
        nzr[0] = cb[r0];
        nzr[1] = cb[r0 + nrows];
    }
    if (UPDATE)
        for (long long k = tid; k < z; k += kSweepThreads)
            sAS[k] = COHERENT ? __ldcg(in.psiAS + k) : in.psiAS[k];
    __syncthreads();
    // entries of the row sequence: the tile's rows, or its listed rows
    const int nlist = compact ? nzr[1] - nzr[0] : nrows;
    const int* rowlist = compact ? in.nz_rows + (long long)band * in.x + nzr[0] : nullptr;
    const int nrounds = (nlist + RPS - 1) / RPS;

    const uint64_t pol_stream = policy_evict_first();
    const uint64_t pol_keep = policy_evict_last();

    auto slotS = [&](unsigned char* st, int r) { return st + (size_t)r * lay.capS; };
    auto slotX = [&](unsigned char* st, int r) {
        return st + (size_t)RPS * lay.capS + (size_t)r * lay.capX;
    };
    auto slotA = [&](unsigned char* st, int r) {
        return st + (size_t)RPS * (lay.capS + lay.capX) + (size_t)r * lay.capA;
    };

    // Round t holds entries t*RPS + r, r < RPS, of the row sequence; a compact
    // update records their rows in srow[stage] for the consumers (published
    // by the stage's mbarrier arrival, read after its wait).
    auto issue = [&](int t, int s) {
        unsigned char* st = stage0 + (size_t)s * L.stage_bytes;
        const int nr = min(RPS, nlist - t * RPS);
        uint32_t tot = 0;
        for (int r = 0; r < nr; ++r) {
            const long long i = compact ? (long long)rowlist[t * RPS + r] : r0 + (long long)t * RPS + r;
            if (compact) srow[s][r] = int(i);
            const uintptr_t aS = reinterpret_cast<uintptr_t>(in.S + (i * in.y + c0) * z);
            tot += uint32_t(align_up16(aS + (uintptr_t)cw * z * sizeof(T)) - align_down16(aS));
            if (UPDATE) {  // the axis sums of S do not read X
                const uintptr_t aX = reinterpret_cast<uintptr_t>(in.X + i * in.y + c0);
                tot += uint32_t(align_up16(aX + (uintptr_t)cw * sizeof(T)) - align_down16(aX));
            }
            if (UPDATE) {
                const uintptr_t aA = reinterpret_cast<uintptr_t>(in.psiA + i * z);
                tot += uint32_t(align_up16(aA + (uintptr_t)z * sizeof(T)) - align_down16(aA));
            }
        }
        mbar_arrive_expect_tx(&bars[s], tot);
        for (int r = 0; r < nr; ++r) {
            const long long i = compact ? (long long)srow[s][r] : r0 + (long long)t * RPS + r;
            const uintptr_t aS = reinterpret_cast<uintptr_t>(in.S + (i * in.y + c0) * z);
            const uintptr_t aX = reinterpret_cast<uintptr_t>(in.X + i * in.y + c0);
            bulk_g2s(slotS(st, r), reinterpret_cast<const void*>(align_down16(aS)),
                     uint32_t(align_up16(aS + (uintptr_t)cw * z * sizeof(T)) - align_down16(aS)),
                     &bars[s], pol_stream);
            if (UPDATE)
                bulk_g2s(slotX(st, r), reinterpret_cast<const void*>(align_down16(aX)),
                         uint32_t(align_up16(aX + (uintptr_t)cw * sizeof(T)) - align_down16(aX)),
                         &bars[s], pol_keep);
            if (UPDATE) {
                const uintptr_t aA = reinterpret_cast<uintptr_t>(in.psiA + i * z);
                bulk_g2s(slotA(st, r), reinterpret_cast<const void*>(align_down16(aA)),
                         uint32_t(align_up16(aA + (uintptr_t)z * sizeof(T)) - align_down16(aA)),
                         &bars[s], pol_keep);
            }
        }
    };

    if (tid == 0) {
        const int n0 = min(L.stages, nrounds);
        for (int t = 0; t < n0; ++t) issue(t, t);
    }

    // S_pjk accumulators of the lane's fibers over the tile's rows.
    Acc<T> pj[CPW][MCH][VEC];
#pragma unroll
    for (int c = 0; c < CPW; ++c)
#pragma unroll
        for (int m = 0; m < MCH; ++m)
#pragma unroll
            for (int v = 0; v < VEC; ++v) pj[c][m][v].init();
    // only multi-instance sweeps track the relative change
    const bool track = BATCH && UPDATE && in.delta_part != nullptr;
    double d_abs = 0.0, d_new = 0.0;

    // round t uses stage s = t % stages in its lap-th pass over the ring
    // (counted, not divided: the ring depth is a launch parameter)
    int s = 0, lap = 0;
    for (int t = 0; t < nrounds; ++t) {
        // warp-uniform: the lane-group shuffles below need every lane of the warp
        const bool ok = __all_sync(0xffffffffu, mbar_wait_bounded(&bars[s], (uint32_t)(lap & 1)));
        if (!ok) {
            // Give up: flag the error and wait (bounded) for the copies that
            // may still be landing in this CTA's shared memory.
            if (lane == 0) {
                atomicOr(L.err, DEV_ERR_WAIT_TIMEOUT);
                const int issued = min(nrounds, t + L.stages);
                for (int u = t; u < issued; ++u)
                    (void)mbar_wait_bounded(&bars[u % L.stages], (uint32_t)((u / L.stages) & 1));
            }
            return false;
        }
        unsigned char* st = stage0 + (size_t)s * L.stage_bytes;
        const bool row_ok = t * RPS + rs < nlist;  // warp-uniform
        const long long i =
            compact ? (row_ok ? (long long)srow[s][rs] : 0) : r0 + (long long)t * RPS + rs;

        // S_ipk of row i over this warp's passes: at most CPW terms per lane,
        // accumulated in FP64 (exact for so few storage-type terms, and cheaper
        // than a Kahan pair in FP32)
        double ip[MCH][VEC];
#pragma unroll
        for (int m = 0; m < MCH; ++m)
#pragma unroll
            for (int v = 0; v < VEC; ++v) ip[m][v] = 0.0;
        // warp-uniform: an update round without a pass with X != 0 leaves ip at zero
        bool ip_live = !UPDATE;

        if (row_ok) {
            const uintptr_t aS = reinterpret_cast<uintptr_t>(in.S + (i * in.y + c0) * z);
            const uintptr_t aX = reinterpret_cast<uintptr_t>(in.X + i * in.y + c0);
            const T* sS = reinterpret_cast<const T*>(slotS(st, rs) + (aS & 15));
            const T* sX = reinterpret_cast<const T*>(slotX(st, rs) + (aX & 15));
            // grad_minus of the row's k from the stage's psi(alpha_eph) row
            const T* sA = nullptr;
            if (UPDATE) {
                const uintptr_t aA = reinterpret_cast<uintptr_t>(in.psiA + i * z);
                sA = reinterpret_cast<const T*>(slotA(st, rs) + (aA & 15));
            }
            auto load_gm = [&](T (&gm)[MCH][VEC]) {
#pragma unroll
                for (int m = 0; m < MCH; ++m)
#pragma unroll
                    for (int v = 0; v < VEC; ++v) {
                        const long long k = (long long)(m * LPF + q) * VEC + v;
                        gm[m][v] = (k < z) ? sAS[k] - sA[k] : T(0);
                    }
            };
            // The fiber values of pass c from the stage.  VEC > 1 only when
            // z*sizeof(T) is a multiple of 16, so a chunk is entirely inside or
            // entirely outside the fiber.
            auto load_pass = [&](const int c, T (&se)[MCH][VEC]) {
                const int jl = (cg * CPW + c) * FPW + g;
#pragma unroll
                for (int m = 0; m < MCH; ++m) {
                    const long long k0 = (long long)(m * LPF + q) * VEC;
                    if (jl < cw && k0 < z) {
                        VecIO<T, VEC>::load(sS + (long long)jl * z + k0, se[m]);
                    } else {
#pragma unroll
                        for (int v = 0; v < VEC; ++v) se[m][v] = T(0);
                    }
                }
            };
            // An update reads a pass's fibers when it needs them (they stay in
            // the stage until this warp's arrival); the sums read them all.
            T sv[CPW][MCH][VEC];
            auto x_of = [&](const int c) {
                const int jl = (cg * CPW + c) * FPW + g;
                return jl < cw ? sX[jl] : T(0);
            };
            if (!UPDATE)
#pragma unroll
                for (int c = 0; c < CPW; ++c) load_pass(c, sv[c]);
            if (UPDATE) {
                const T teps = T(L.eps);
                // A fiber with X == 0 updates to zero whatever its digamma values
                // (the reference formula multiplies by X/(S_ijp+eps)).  Passes
                // whose fibers all have X == 0 only store zeros; the others form
                // a warp-uniform work list that runs one copy of the arithmetic.
                unsigned work = 0;
#pragma unroll
                for (int c = 0; c < CPW; ++c)
                    if (__any_sync(0xffffffffu, x_of(c) != T(0))) work |= 1u << c;
                ip_live = work != 0;

                // The update of one pass from its fiber values se, psi(beta_eph)
                // values be and X value xe.
                auto pass_math = [&](const T (&se)[MCH][VEC], const T (&be)[MCH][VEC], const T xe,
                                     T (&sn)[MCH][VEC]) {
                    // digamma in chunks of at most 4 elements per lane (bounds
                    // the live registers of long fibers)
                    constexpr int NE = MCH * VEC;
                    constexpr int NC = NE < 4 ? NE : 4;
                    T ps[NE];
#pragma unroll
                    for (int e0 = 0; e0 < NE; e0 += NC) {
                        T arg[NC], out[NC];
#pragma unroll
                        for (int e = 0; e < NC; ++e)
                            arg[e] = se[(e0 + e) / VEC][(e0 + e) % VEC] + T(1);
                        PsiPass<T, APPR>::template run<NC>(arg, out, ltab);
#pragma unroll
                        for (int e = 0; e < NC; ++e) ps[e0 + e] = out[e];
                    }
                    T gp[MCH][VEC];
                    T gm[MCH][VEC];
                    load_gm(gm);
                    T as = T(0), an = T(0), ad = T(0);
#pragma unroll
                    for (int m = 0; m < MCH; ++m)
#pragma unroll
                        for (int v = 0; v < VEC; ++v) {
                            const T e = se[m][v];
                            gp[m][v] = be[m][v] - ps[m * VEC + v];
                            as += e;
                            an += e * gm[m][v];
                            ad += e * gp[m][v];
                        }
                    as = group_sum<LPF>(as);
                    an = group_sum<LPF>(an);
                    ad = group_sum<LPF>(ad);
                    const T xr = Rcp<T>::of(xe + teps);
                    const T nom = an * xr;
                    const T den = ad * xr + teps;
                    const T xos = xe * Rcp<T>::of(as + teps);
                    // X == 0 (or an all-zero fiber) keeps the fiber at zero: the
                    // reference's FP64 result, and no 0 * inf in FP32 where
                    // eps = 1e-50 underflows to zero.
                    const bool zero = (xe == T(0)) || (as == T(0));
#pragma unroll
                    for (int m = 0; m < MCH; ++m)
#pragma unroll
                        for (int v = 0; v < VEC; ++v)
                            sn[m][v] = zero ? T(0)
                                            : se[m][v] * (((gp[m][v] + nom) * xos) *
                                                          Rcp<T>::of(gm[m][v] + den));
                };
                // Accumulates and stores the new values of pass c.
                auto pass_out = [&](const int c, const T (&se)[MCH][VEC], const T (&sn)[MCH][VEC]) {
                    const int jl = (cg * CPW + c) * FPW + g;
#pragma unroll
                    for (int m = 0; m < MCH; ++m) {
#pragma unroll
                        for (int v = 0; v < VEC; ++v) {
                            ip[m][v] += double(sn[m][v]);
                            if (track) {
                                d_abs += fabs(double(sn[m][v]) - double(se[m][v]));
                                d_new += fabs(double(sn[m][v]));
                            }
                        }
                        const long long k0 = (long long)(m * LPF + q) * VEC;
                        if (jl < cw && k0 < z)
                            VecIO<T, VEC>::store(in.S + ((i * in.y + c0 + jl) * z + k0), sn[m]);
                    }
                };

#pragma unroll
                for (int c = 0; c < CPW; ++c) {
                    // a compact update finds the zeros of these fibers stored already
                    if (((work >> c) & 1u) || clean) continue;
                    const int jl = (cg * CPW + c) * FPW + g;
                    T zs[VEC];
#pragma unroll
                    for (int v = 0; v < VEC; ++v) zs[v] = T(0);
                    T so[MCH][VEC];
                    if (track) load_pass(c, so);
#pragma unroll
                    for (int m = 0; m < MCH; ++m) {
                        if (track) {
#pragma unroll
                            for (int v = 0; v < VEC; ++v) d_abs += fabs(double(so[m][v]));
                        }
                        const long long k0 = (long long)(m * LPF + q) * VEC;
                        if (jl < cw && k0 < z)
                            VecIO<T, VEC>::store(in.S + ((i * in.y + c0 + jl) * z + k0), zs);
                    }
                }
#pragma unroll 1
                while (work) {
                    const int c = __ffs(work) - 1;
                    work &= work - 1;
                    T se[MCH][VEC], be[MCH][VEC];
                    const T xe = x_of(c);
                    load_pass(c, se);
                    {
                        // psi(beta_eph) of the pass's fibers through the read-only
                        // cache (the band's slice stays in L1 over the tile); kept
                        // out of registers, which the digamma arithmetic needs more
                        const int jl = (cg * CPW + c) * FPW + g;
#pragma unroll
                        for (int m = 0; m < MCH; ++m) {
                            const long long k0 = (long long)(m * LPF + q) * VEC;
                            if (jl < cw && k0 < z) {
                                if (COHERENT)
                                    VecIO<T, VEC>::ldcg(in.psiB + (c0 + jl) * z + k0, be[m]);
                                else
                                    VecIO<T, VEC>::ldg(in.psiB + (c0 + jl) * z + k0, be[m]);
                            } else {
#pragma unroll
                                for (int v = 0; v < VEC; ++v) be[m][v] = T(0);
                            }
                        }
                    }
                    T sn[MCH][VEC];
                    pass_math(se, be, xe, sn);
#pragma unroll
                    for (int cc = 0; cc < CPW; ++cc) {
                        if (cc == c) {
#pragma unroll
                            for (int m = 0; m < MCH; ++m)
#pragma unroll
                                for (int v = 0; v < VEC; ++v) pj[cc][m][v].add(sn[m][v]);
                        }
                    }
                    pass_out(c, se, sn);
                }
            } else {
#pragma unroll
                for (int c = 0; c < CPW; ++c)
#pragma unroll
                    for (int m = 0; m < MCH; ++m)
#pragma unroll
                        for (int v = 0; v < VEC; ++v) {
                            pj[c][m][v].add(sv[c][m][v]);
                            ip[m][v] += double(sv[c][m][v]);
                        }
            }
        }

        // S_ipk partial of row i over this warp's columns -> red[s][warp].
        // (zeros stored directly when ip is zero: no conversion, no shuffles)
        double* redw = red + ((size_t)s * NW + warp) * z;
#pragma unroll
        for (int m = 0; m < MCH; ++m)
#pragma unroll
            for (int v = 0; v < VEC; ++v) {
                double val = 0.0;
                if (ip_live) {
                    val = ip[m][v];
                    if (FPW > 1) val = cross_group_sum<LPF>(val);
                }
                const long long k = (long long)(m * LPF + q) * VEC + v;
                if (g == 0 && k < z) redw[k] = val;
            }
        __syncwarp();
        // No CTA barrier per round: each warp counts itself done with stage s;
        // the last of the NW warps (the count reaches a multiple of NW) adds, per
        // row slot, its warps' partials in column-group order, writes the S_ipk
        // partials of the round's rows and refills the stage.  Warps drift apart
        // by up to `stages` rounds.
        int last = 0;
        if (lane == 0) {
            __threadfence_block();
            last = (atomicAdd(&cnt[s], 1) == (lap + 1) * NW - 1) ? 1 : 0;
        }
        last = __shfl_sync(0xffffffffu, last, 0);
        if (last) {
            __threadfence_block();
            const double* reds = red + (size_t)s * NW * z;
            const int nr = min(RPS, nlist - t * RPS);
            for (int r = 0; r < nr; ++r) {
                const long long ir = compact ? (long long)srow[s][r] : r0 + (long long)t * RPS + r;
                const double* redr = reds + (size_t)r * wpr * z;
                for (long long k = lane; k < z; k += 32) {
                    // all loads issued together; warps beyond wpr add nothing
                    double part[NW];
#pragma unroll
                    for (int w = 0; w < NW; ++w) part[w] = w < wpr ? redr[(size_t)w * z + k] : 0.0;
                    double sum = 0.0;
#pragma unroll
                    for (int w = 0; w < NW; ++w) sum += part[w];
                    in.part_ipk[((long long)band * in.x + ir) * z + k] = sum;
                }
            }
            __syncwarp();
            if (lane == 0 && t + L.stages < nrounds) issue(t + L.stages, s);
        }
        if (++s == L.stages) {
            s = 0;
            ++lap;
        }
    }

    // S_pjk partial of the band over this tile's rows.  With one row slot every
    // (j,k) has a single owner lane; otherwise the row slots' partials are added
    // in slot order through shared memory (the drained stage ring).
    if (RPS == 1) {
#pragma unroll
        for (int c = 0; c < CPW; ++c) {
            const int jl = (cg * CPW + c) * FPW + g;
#pragma unroll
            for (int m = 0; m < MCH; ++m)
#pragma unroll
                for (int v = 0; v < VEC; ++v) {
                    const long long k = (long long)(m * LPF + q) * VEC + v;
                    if (jl < cw && k < z)
                        in.part_pjk[((long long)rr * in.y + c0 + jl) * z + k] = pj[c][m][v].value();
                }
        }
    } else {
        __syncthreads();  // every warp is done with the ring
        double* pjbuf = reinterpret_cast<double*>(stage0);  // [RPS][band_w][z]
#pragma unroll
        for (int c = 0; c < CPW; ++c) {
            const int jl = (cg * CPW + c) * FPW + g;
#pragma unroll
            for (int m = 0; m < MCH; ++m)
#pragma unroll
                for (int v = 0; v < VEC; ++v) {
                    const long long k = (long long)(m * LPF + q) * VEC + v;
                    if (jl < in.band_w && k < z)
                        pjbuf[((size_t)rs * in.band_w + jl) * z + k] = pj[c][m][v].value();
                }
        }
        __syncthreads();
        const long long n = (long long)cw * z;
        for (long long e = tid; e < n; e += kSweepThreads) {
            double sum = 0.0;
            for (int r = 0; r < RPS; ++r) sum += pjbuf[(size_t)r * in.band_w * z + e];
            in.part_pjk[((long long)rr * in.y + c0) * z + e] = sum;
        }
    }

    if (track) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            d_abs += __shfl_xor_sync(0xffffffffu, d_abs, o);
            d_new += __shfl_xor_sync(0xffffffffu, d_new, o);
        }
        if (lane == 0) {
            dsum[warp][0] = d_abs;
            dsum[warp][1] = d_new;
        }
        __syncthreads();
        if (tid == 0) {
            double a = 0.0, b = 0.0;
            for (int w = 0; w < NW; ++w) {
                a += dsum[w][0];
                b += dsum[w][1];
            }
            in.delta_part[2 * tile] = a;
            in.delta_part[2 * tile + 1] = b;
        }
    }
    // the fused finalize in the tile's epilogue (the ring is drained)
    if (FUSED) tile_finalize<T>(in, L, band, rr, r0, nrows, c0, cw, reinterpret_cast<double*>(stage0));
    return true;
}

template <typename T, int VEC, int LPF, int MCH, bool UPDATE, bool APPR, bool MULTIROW,
          bool COMPACT>
__global__ void __launch_bounds__(kSweepThreads, 2) sweep_kernel(const SweepParams<T> p) {
    extern __shared__ __align__(128) unsigned char smem[];
    const int band = blockIdx.x % p.in.n_bands;
    const int rr = blockIdx.x / p.in.n_bands;
    sweep_tile<T, VEC, LPF, MCH, UPDATE, APPR, false, MULTIROW, COMPACT>(p.in, p.L, band, rr,
                                                                        int(blockIdx.x), smem);
}

template <typename T, int VEC, int LPF, int MCH, bool UPDATE, bool APPR, bool MULTIROW,
          bool COMPACT>
__global__ void __launch_bounds__(kSweepThreads, 2) sweep_batch_kernel(const BatchSweepParams<T> p) {
    extern __shared__ __align__(128) unsigned char smem[];
    const BatchTile tl = p.tiles[blockIdx.x];
    SweepInst<T> in = p.insts[tl.inst];
    if (!p.track) in.delta_part = nullptr;
    sweep_tile<T, VEC, LPF, MCH, UPDATE, APPR, true, MULTIROW, COMPACT>(
        in, p.L, tl.band, tl.rr, tl.rr * in.n_bands + tl.band, smem);
}


}  // namespace bldm
