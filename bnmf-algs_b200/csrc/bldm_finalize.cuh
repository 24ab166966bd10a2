// The finalize step of an iteration (shared by the plain, multi-instance and
// persistent launches): sums the sweep's partial axis sums in a fixed order,
// forms beta_eph / alpha_eph (update_alpha_eph / update_beta_eph,
// src/bld/bld_mult/bld_mult_funcs.hpp:130-163) and tabulates the digamma
// values the next sweep needs (grad_plus's psi(beta_eph), grad_minus's
// psi(alpha_eph) and psi(sum_i alpha_eph), bld_mult_funcs.hpp:177-229).
#pragma once

#include "bldm_device.cuh"
#include "bldm_kernels.h"

namespace bldm {

constexpr int kFinAccDoubles = 2 * kFinThreads;

// Sum of p[r * stride], r < n, in increasing r (the order of a plain loop),
// with the loads of W terms issued before their adds so that a thread keeps W
// reads of the partial buffers in flight (the partials were just written, so
// the finalize waits on L2 round trips, not on bandwidth).  Terms past n load
// nothing and add an exact 0.0.  W = 16 for the single-instance finalize (few
// blocks, long sums); 8 for the multi-instance one, whose tens of thousands of
// short blocks need the occupancy that fewer registers give.
template <bool CG, int W>
__device__ __forceinline__ double sum_strided(const double* p, long long stride, int n) {
    double s = 0.0;
    for (int r = 0; r < n; r += W) {
        double v[W];
#pragma unroll
        for (int u = 0; u < W; ++u) {
            const double* a = p + (long long)(r + u) * stride;
            v[u] = (r + u < n) ? (CG ? __ldcg(a) : *a) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < W; ++u) s += v[u];
    }
    return s;
}

// Block `blk` of an instance's finalize.  Blocks [0, nbB): psi(beta_eph) for
// every (j,k).  Blocks [nbB, nbB + n_ablk): psi(alpha_eph) for a block of rows
// plus that block's sum of alpha_eph over rows; the last block to finish sums
// the block sums (R interleaved groups of blocks, then the groups in order),
// tabulates psi(sum_i alpha_eph(i,k)) and, when the sweep tracked it, the
// relative change of S.
//
// CG: every load of the partials bypasses L1 (a persistent launch reads
// partials that other CTAs of the same launch have just rewritten).
//
// acc: 2 * kFinThreads doubles of shared memory for the row groups' sums.
template <typename T, int W, bool CG = false>
__device__ __forceinline__ void finalize_block(const FinInst<T>& p, int blk, int plus_appr,
                                               int minus_appr, double* acc) {
    const long long z = p.z;
    const int tid = threadIdx.x;
    if (blk < p.nbB) {
        const long long idx = (long long)blk * kFinThreads + tid;
        if (idx < p.y * z) {
            const long long k = idx % z;
            const double s = sum_strided<CG, W>(p.part_pjk + idx, p.y * z, p.n_rr);
            if (p.red)
                p.red[idx] = s;
            else
                p.psiB[idx] = T(psi_mode_f64(s + p.beta[k], plus_appr != 0));
        }
        return;
    }
    __shared__ unsigned last;
    const int b = blk - p.nbB;
    const long long i0 = (long long)b * p.rows_per_ablk;
    const long long i1 = min(p.x, i0 + p.rows_per_ablk);
    const int KT = (int)min(z, (long long)kFinThreads);
    const int R = kFinThreads / KT;
    const int sub = tid / KT;
    // R > 1 (z < 256): R row groups of KT threads, combined through acc
    // (R * z <= 2 * kFinThreads entries); R == 1: a thread's sum over the
    // block's rows is the block's partial itself (any z)
    if (sub < R) {
        for (long long k = tid % KT; k < z; k += KT) {
            double a = 0.0;
            for (long long i = i0 + sub; i < i1; i += R) {
                const double s = sum_strided<CG, W>(p.part_ipk + i * z + k, p.x * z, p.n_bands);
                const double ae = s + p.alpha[i];
                p.psiA[i * z + k] = T(psi_mode_f64(ae, minus_appr != 0));
                a += ae;
            }
            if (R == 1)
                p.asum_part[(long long)b * z + k] = a;
            else
                acc[sub * z + k] = a;
        }
    }
    if (R > 1) {
        __syncthreads();
        for (long long k = tid; k < z; k += kFinThreads) {
            double a = 0.0;
            for (int r = 0; r < R; ++r) a += acc[r * z + k];
            p.asum_part[(long long)b * z + k] = a;
        }
    }
    __threadfence();
    __syncthreads();
    if (tid == 0) last = (atomicAdd(p.counter, 1u) == (unsigned)(p.n_ablk - 1)) ? 1u : 0u;
    __syncthreads();
    if (last) {
        __threadfence();
        // group r < R sums blocks r, r + R, r + 2R, ... of column k
        if (R == 1) {
            for (long long k = tid; k < z; k += kFinThreads) {
                const double a = sum_strided<true, W>(p.asum_part + k, z, p.n_ablk);
                if (p.red)
                    p.red[p.y * z + k] = a;
                else
                    p.psiAS[k] = T(psi_mode_f64(a, minus_appr != 0));
            }
        } else {
            if (sub < R) {
                for (long long k = tid % KT; k < z; k += KT) {
                    const int nb = (p.n_ablk - sub + R - 1) / R;
                    acc[sub * z + k] = sum_strided<true, W>(p.asum_part + (long long)sub * z + k,
                                                            (long long)R * z, nb);
                }
            }
            __syncthreads();
            for (long long k = tid; k < z; k += kFinThreads) {
                double a = 0.0;
                for (int r = 0; r < R; ++r) a += acc[r * z + k];
                if (p.red)
                    p.red[p.y * z + k] = a;
                else
                    p.psiAS[k] = T(psi_mode_f64(a, minus_appr != 0));
            }
        }
        if (p.delta_part && tid < 32) {
            // lanes take tiles t = lane, lane + 32, ...; then a fixed-order tree
            double d = 0.0, n = 0.0;
            for (int t = tid; t < p.n_tiles; t += 32) {
                d += __ldcg(&p.delta_part[2 * t]);
                n += __ldcg(&p.delta_part[2 * t + 1]);
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                d += __shfl_xor_sync(0xffffffffu, d, o);
                n += __shfl_xor_sync(0xffffffffu, n, o);
            }
            if (tid == 0) *p.rel_change = n > 0.0 ? d / n : (d > 0.0 ? 1.0 : 0.0);
        }
        if (tid == 0) *p.counter = 0u;
    }
}

// The finalize of a multi-instance sweep, run by each tile after it has written
// its partials.  Three arrival counters per instance (SweepInst::fcnt) pick the
// CTAs that do the work, each the last of its kind to arrive:
//   * the last of a band's n_rr tiles: psi(beta_eph(j,k)) for the band's columns,
//     the band's S_+jk partials summed in row-range order;
//   * the last of a row range's n_bands tiles: psi(alpha_eph(i,k)) for the range's
//     rows, S_i+k partials summed in band order, and the range's sum of alpha_eph
//     over its rows (row groups, then the groups in order);
//   * the last of all the instance's tiles, once every tile has done the above:
//     psi(sum_i alpha_eph(i,k)) from the ranges' sums in range order, and the
//     relative change of S from the tiles' partials.
// Every sum runs in a fixed order, so the result does not depend on which CTA
// arrives last.  A counter is reset by its last arrival (no more arrivals come
// in this round).  With in.done, the instance's round count is published at the
// end (persistent launches wait on it).  All threads of the CTA call this; acc
// is kFinAccDoubles doubles of shared memory no longer in use.
template <typename T>
__device__ __forceinline__ void tile_finalize(const SweepInst<T>& in, const SweepLaunch& L,
                                              int band, int rr, long long r0, int nrows,
                                              long long c0, int cw, double* acc) {
    __shared__ unsigned s_flags;
    const int tid = threadIdx.x;
    const long long z = in.z;
    const bool plus = L.plus_appr != 0, minus = L.minus_appr != 0;
    __syncthreads();  // the tile's partials are written
    if (tid == 0) {
        __threadfence();
        unsigned f = 0;
        unsigned* bc = in.fcnt + 1 + band;
        unsigned* rc = in.fcnt + 1 + in.n_bands + rr;
        if (atomicAdd(bc, 1u) == unsigned(in.n_rr - 1)) {
            f |= 1u;
            *bc = 0u;
        }
        if (atomicAdd(rc, 1u) == unsigned(in.n_bands - 1)) {
            f |= 2u;
            *rc = 0u;
        }
        if (f) __threadfence();
        s_flags = f;
    }
    __syncthreads();
    const unsigned f = s_flags;
    if (f & 1u) {
        T* psiB = const_cast<T*>(in.psiB);
        const long long n = (long long)cw * z;
        for (long long e = tid; e < n; e += kSweepThreads) {
            const long long idx = c0 * z + e;
            const double s = sum_strided<true, 8>(in.part_pjk + idx, in.y * z, in.n_rr);
            psiB[idx] = T(psi_mode_f64(s + in.beta[idx % z], plus));
        }
    }
    if (f & 2u) {
        T* psiA = const_cast<T*>(in.psiA);
        const int KT = (int)min(z, (long long)kSweepThreads);
        const int R = kSweepThreads / KT;
        const int sub = tid / KT;
        if (sub < R) {
            for (long long k = tid % KT; k < z; k += KT) {
                double a = 0.0;
                for (long long i = r0 + sub; i < r0 + nrows; i += R) {
                    const double s =
                        sum_strided<true, 8>(in.part_ipk + i * z + k, in.x * z, in.n_bands);
                    const double ae = s + in.alpha[i];
                    psiA[i * z + k] = T(psi_mode_f64(ae, minus));
                    a += ae;
                }
                if (R == 1)
                    in.asum_rr[(long long)rr * z + k] = a;
                else
                    acc[sub * z + k] = a;
            }
        }
        if (R > 1) {
            __syncthreads();
            for (long long k = tid; k < z; k += kSweepThreads) {
                double a = 0.0;
                for (int r = 0; r < R; ++r) a += acc[r * z + k];
                in.asum_rr[(long long)rr * z + k] = a;
            }
        }
    }
    __syncthreads();  // this CTA's tables are written
    if (tid == 0) {
        __threadfence();
        const unsigned nt = unsigned(in.n_rr) * unsigned(in.n_bands);
        unsigned g = 0;
        if (atomicAdd(in.fcnt, 1u) == nt - 1u) {
            g = 4u;
            in.fcnt[0] = 0u;
            __threadfence();
        }
        s_flags = g;
    }
    __syncthreads();
    if (s_flags & 4u) {
        T* psiAS = const_cast<T*>(in.psiAS);
        for (long long k = tid; k < z; k += kSweepThreads) {
            const double a = sum_strided<true, 8>(in.asum_rr + k, z, in.n_rr);
            psiAS[k] = T(psi_mode_f64(a, minus));
        }
        if (in.delta_part && tid < 32) {
            // lanes take tiles t = lane, lane + 32, ...; then a fixed-order tree
            const int n_tiles = in.n_rr * in.n_bands;
            double d = 0.0, n = 0.0;
            for (int t = tid; t < n_tiles; t += 32) {
                d += __ldcg(&in.delta_part[2 * t]);
                n += __ldcg(&in.delta_part[2 * t + 1]);
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                d += __shfl_xor_sync(0xffffffffu, d, o);
                n += __shfl_xor_sync(0xffffffffu, n, o);
            }
            if (tid == 0) *in.rel_change = n > 0.0 ? d / n : (d > 0.0 ? 1.0 : 0.0);
        }
        if (in.done) {
            __syncthreads();
            if (tid == 0) {
                __threadfence();
                atomicAdd(in.done, 1u);
            }
        }
    }
}

}  // namespace bldm
