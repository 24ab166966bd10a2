// Persistent multi-instance launch: every round (iteration) of every instance of
// one lane-shape class in a single launch.
//
// The launch-per-round form (Engine::launch_sequence) issues, per iteration, one
// sweep launch per class and one finalize launch for all instances, so every
// instance waits at every iteration for the slowest tile of the whole batch and
// for the launch gaps.  Here the CTAs of one launch take items from an ordered
// queue (PersistParams): round r's sweep tiles of the class, largest first, then
// round r + 1's, and so on.  Each tile finalizes its share of its instance's
// round in its epilogue (tile_finalize); the last tile of the instance publishes
// the round's completion.  A tile of round r waits until its instance has
// completed r rounds, so an instance that finishes a round early moves on while
// others still sweep.  Each wait is one thread's acquire loop on a completion counter,
// bounded by %globaltimer (PersistParams::wait_ns); on expiry the CTA sets the
// error word and the class's abort flag, and every CTA stops taking items.
//
// Coherence: the producer of a counter fences its writes (__threadfence) before
// the counter's atomic increment; the consumer's acquire load, a fence and a
// proxy fence (the next bulk copies of S, X and psi(alpha_eph) go through the
// async proxy) precede the item's reads; tables rewritten within the launch
// (psi(beta_eph), psi(sum alpha_eph), the partials) are read from L2 (.cg).
#pragma once

#include "bldm_finalize.cuh"
#include "bldm_sweep_kernels.cuh"

namespace bldm {

// One CTA of the class's persistent launch.  Only called with 256 threads and at
// least kFinAccDoubles doubles of dynamic shared memory.
template <typename T, int VEC, int LPF, int MCH, bool APPR, bool MULTIROW>
__global__ void __launch_bounds__(kSweepThreads, 2) persist_kernel(const PersistParams<T> p) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ unsigned s_item;
    __shared__ int s_ok;
    const int tid = threadIdx.x;
    const unsigned total = unsigned(p.P) * unsigned(p.rounds);
    uint64_t* bars = reinterpret_cast<uint64_t*>(smem + (size_t)p.L.stages * p.L.stage_bytes);
    while (true) {
        __syncthreads();  // every thread is done with the previous item's shared memory
        if (tid == 0) {
            unsigned q = 0xffffffffu;
            if (ld_acquire_gpu(&p.ctl->abort) == 0u) q = atomicAdd(&p.ctl->next, 1u);
            s_item = q;
        }
        __syncthreads();
        const unsigned q = s_item;
        if (q >= total) break;
        const int round = int(q / unsigned(p.P));
        const PItem w = p.items[q % unsigned(p.P)];
        if (tid == 0) {
            // the instance's previous rounds are complete (its tables are written)
            unsigned target = unsigned(round);
            // test hook: wait for this round's completion, which needs this tile
            if (p.stall_test && w.inst == 0 && round == 0) target = 1u;
            const bool ok = wait_counter_bounded(p.done + w.inst, target, &p.ctl->abort, p.wait_ns);
            if (!ok) {
                atomicOr(p.L.err, DEV_ERR_WAIT_TIMEOUT);
                atomicExch(&p.ctl->abort, 1u);
            }
            __threadfence();
            fence_proxy_async_global();
            s_ok = ok ? 1 : 0;
        }
        __syncthreads();
        if (!s_ok) break;
        SweepInst<T> in = p.sinst[w.inst];
        in.done = p.done + w.inst;
        const bool update = !(p.prime && round == 0);
        // the relative change is taken over the last round only
        if (!(update && round + 1 == p.rounds)) in.delta_part = nullptr;
        const int tile = w.b * in.n_bands + w.a;
        bool ok;
        if (!update)
            ok = sweep_tile<T, VEC, LPF, MCH, false, true, true, MULTIROW, false, true, true>(
                in, p.L, w.a, w.b, tile, smem);
        else if (round >= p.compact_from)
            ok = sweep_tile<T, VEC, LPF, MCH, true, APPR, true, MULTIROW, true, true, true>(
                in, p.L, w.a, w.b, tile, smem);
        else
            ok = sweep_tile<T, VEC, LPF, MCH, true, APPR, true, MULTIROW, false, true, true>(
                in, p.L, w.a, w.b, tile, smem);
        // every warp of the CTA has left the tile (a warp that gave up waits for
        // its copies in flight before it returns)
        const int all_ok = __syncthreads_and(ok ? 1 : 0);
        if (tid == 0) {
            if (all_ok)
                for (int s = 0; s < p.L.stages; ++s) mbar_inval(&bars[s]);
            else
                atomicExch(&p.ctl->abort, 1u);
        }
        if (!all_ok) break;
    }
}

}  // namespace bldm
