// Parameter blocks of the sweep and finalize kernels, shared by the
// single-instance plan (bldm_sweep.cu) and the multi-instance engine
// (bldm_batch.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace bldm {

constexpr int kSweepWarps = 8;
constexpr int kSweepThreads = kSweepWarps * 32;
constexpr int kFinThreads = 256;

// fiber passes per warp per row, from the bytes a lane holds per fiber
__host__ __device__ constexpr int cpw_for(int bytes) { return bytes <= 16 ? 4 : (bytes <= 32 ? 2 : 1); }

// One instance as a sweep sees it.  Rows are split into row ranges of
// rr_base (+1 for the first rr_extra ranges) rows, clamped to x; columns into
// bands of band_w = wpr * CPW * (32 / LPF) columns; wpr warps share one row,
// so a stage holds 8 / wpr rows.
template <typename T> struct SweepInst {
    T* S;
    const T* X;
    const T* psiB;       // psi(beta_eph) [y][z]
    const T* psiA;       // psi(alpha_eph) [x][z]
    const T* psiAS;      // psi(sum_i alpha_eph) [z]
    double* part_pjk;    // [n_rr][y][z]
    double* part_ipk;    // [n_bands][x][z]
    double* delta_part;  // [n_rr * n_bands][2] (sum |S_new - S|, sum |S_new|) or null
    // Rows with some X != 0 in a band's columns, for updates that skip the
    // others: nz_rows[b][0 .. nz_cnt[b][x]) ascending, nz_cnt[b][i] = entries
    // of band b below row i.  null: every row is swept.
    const int* nz_rows;  // [n_bands][x]
    const int* nz_cnt;   // [n_bands][x + 1]
    long long x, y, z;
    int n_bands, band_w, wpr;
    int n_rr, rr_base, rr_extra;
    // Finalize in the tiles' epilogue (multi-instance sweeps, tile_finalize in
    // bldm_finalize.cuh): the last tile of a band tabulates the band's
    // psi(beta_eph), the last tile of a row range its rows' psi(alpha_eph) and
    // their sum over the rows, the last tile of the instance psi(sum_i
    // alpha_eph) and the relative change.  Unused by the single-instance plan.
    const double* alpha;   // [x]
    const double* beta;    // [z]
    unsigned* fcnt;        // [1 + n_bands + n_rr] arrivals: instance | per band | per row range
    double* asum_rr;       // [n_rr][z] sum of alpha_eph over a row range's rows
    double* rel_change;    // sum |S_new - S| / sum |S_new| of a tracked sweep
    unsigned* done;        // rounds the instance completed (persistent launches) or null
};

// Launch-wide constants: ring depth, bytes per stage, eps, error word, and the
// digamma of the fused finalize (grad_plus's psi(beta_eph), grad_minus's
// psi(alpha_eph)).
struct SweepLaunch {
    int stages;
    uint32_t stage_bytes;
    double eps;
    int* err;
    int plus_appr, minus_appr;
};

template <typename T> struct SweepParams {
    SweepInst<T> in;
    SweepLaunch L;
};

// Multi-instance launch: CTA b works on tile tiles[b] of instance insts[.].
struct BatchTile {
    int inst, band, rr, pad;
};
template <typename T> struct BatchSweepParams {
    const SweepInst<T>* insts;
    const BatchTile* tiles;
    SweepLaunch L;
    int track;  // accumulate the relative-change partials in this sweep
};

// Stage layout for an instance: RPS = 8 / wpr row slots, each with the S
// segment of the band, the X segment and (UPDATE) the psi(alpha_eph) row, each
// copied as its enclosing 16-byte-aligned byte range.
struct SlotLayout {
    uint32_t capS, capX, capA;
    __host__ __device__ static uint32_t a16(unsigned long long v) {
        return uint32_t((v + 15) & ~15ull);
    }
    __host__ __device__ SlotLayout(long long band_w, long long z, int es)
        : capS(a16((unsigned long long)(band_w * z * es + 32))),
          capX(a16((unsigned long long)(band_w * es + 32))),
          capA(a16((unsigned long long)(z * es + 32))) {}
};

// One instance as the finalize step sees it.
template <typename T> struct FinInst {
    const double* part_pjk;
    const double* part_ipk;
    const double* alpha;
    const double* beta;
    T* psiB;
    T* psiA;
    T* psiAS;
    double* asum_part;
    unsigned* counter;
    const double* delta_part;  // [n_tiles][2] or null
    double* rel_change;        // sum |S_new - S| / sum |S_new| of the last sweep
    // Row-sharded solves: red[y*z + z] receives this shard's S_+jk and
    // sum_i alpha_eph(i,k) instead of the digamma tables of those shared sums
    // (psi(alpha_eph) of the shard's own rows is still tabulated); null: the
    // whole instance is here.
    double* red;
    long long x, y, z;
    int n_rr, n_bands, nbB, n_ablk, rows_per_ablk, n_tiles;
};

template <typename T> struct FinParams {
    FinInst<T> f;
    int plus_appr, minus_appr;
};

template <typename T> struct BatchFinParams {
    const FinInst<T>* insts;
    const int* block_off;  // [n_inst + 1] first block of each instance
    int n_inst;
    int plus_appr, minus_appr;
};


// Persistent multi-instance launch (bldm_persist.cuh): one launch per lane-shape
// class runs every round (iteration) of every instance of the class from an
// ordered work queue of the class's sweep tiles, round after round; item q of
// the queue is items[q % P] in round q / P.  A tile of round r waits until its
// instance has completed r rounds (the fused finalize of the instance's last
// tile of a round publishes it).  Every wait points to earlier items of the
// queue, held by CTAs that are running, so the queue always drains.
struct PItem {
    int kind;  // reserved (0)
    int inst;  // instance index (into the engine's instance tables)
    int a, b;  // band, row range of the tile
};
struct PersistCtl {
    unsigned next;   // queue head
    unsigned abort;  // set when a wait gave up: every CTA stops taking items
    unsigned pad[2];
};
template <typename T> struct PersistParams {
    const SweepInst<T>* sinst;
    const PItem* items;     // [P] one round of the class's tiles, largest first
    unsigned* done;         // [n_inst] rounds completed per instance (cleared before the launch)
    PersistCtl* ctl;        // this class's queue (cleared before the launch)
    SweepLaunch L;          // ring depth and bytes per stage of the class, eps, error word
    int P;                  // items per round
    int rounds;             // prime round (if any) + update rounds
    int prime;              // round 0 takes the axis sums of the current S
    int compact_from;       // first update round that may skip zero rows (rounds if none)
    unsigned long long wait_ns;  // limit of a dependency wait
    int stall_test;         // test: instance 0's round-0 tiles wait for that round's completion
};
// The persistent kernel of a lane shape (nullptr when not instantiated).
void* pick_persist_fn(int dtype, int vec, int lpf, int mch, bool multirow, bool appr);

// Long fibers (depths beyond the fused sweep's lane layout; bldm_long.cu):
// tiles of (k-chunk of kLongThreads, band of kLongBand columns, row range).
constexpr int kLongThreads = 256;
constexpr int kLongBand = 8;
template <typename T> struct LongSweepParams {
    T* S;
    const T* X;
    const T* psiB;       // psi(beta_eph) [y][z]
    const T* psiA;       // psi(alpha_eph) [x][z]
    const T* psiAS;      // psi(sum_i alpha_eph) [z]
    double* part_pjk;    // [n_rr][y][z]
    double* part_ipk;    // [n_bands][x][z]
    double4* fsum;       // [x*y] (S_ij+, an, ad, -) of the fiber before the update
    long long x, y, z;
    int n_kc, n_bands, n_rr, rr_base, rr_extra;
    double eps;
};
// update: the fiber sums pass and the update pass (2 launches); otherwise the
// axis sums of S alone (1 launch).  params points to LongSweepParams<T> of the
// dtype.  pdl: launch with programmatic stream serialisation.
int launch_long_sweep(int dtype, const void* params, bool update, bool appr, bool pdl,
                      cudaStream_t st, uint64_t* launches);

// Kernel entry points by lane shape (defined in bldm_sweep.cu).  mode: 0 the
// axis sums of S, 1 the update, 2 the compact update (rows listed in
// SweepInst::nz_rows only, no stores of zeros: valid once an update has
// stored them).
enum SweepMode : int { SWEEP_SUMS = 0, SWEEP_UPDATE = 1, SWEEP_COMPACT = 2 };
void* pick_sweep_fn(int dtype, int vec, int lpf, int mch, int mode, bool appr, bool batch,
                    bool multirow);
void* finalize_batch_fn(int dtype);
void* pick_sweep_f64_plain(int vec, int lpf, int mch, int mode, bool appr, bool mr);
void* pick_sweep_f64_batch(int vec, int lpf, int mch, int mode, bool appr, bool mr);
void* pick_sweep_f32_plain(int vec, int lpf, int mch, int mode, bool mr);
void* pick_sweep_f32_batch(int vec, int lpf, int mch, int mode, bool mr);
// Row lists of SweepInst::nz_rows / nz_cnt from X (row-major x*y, storage
// type per dtype) for bands of band_w columns.
int launch_nz_rows(int dtype, const void* dX, long long x, long long y, int band_w, int n_bands,
                   int* nz_rows, int* nz_cnt, cudaStream_t st);
// Row-sum conservation residual max_f |sum_k S(f,k) - X(f)| / max(X(f), 1)
// over nf fibers of depth z, atomically maxed into *out (the bits of a
// nonnegative double; clear it first).  A NaN sum yields a NaN residual.
int launch_conservation(int dtype, const void* dX, const void* dS, long long nf, long long z,
                        unsigned long long* out, cudaStream_t st);
// The same over many instances in one launch: block b works on instance
// i = max{i : block_off[i] <= b}.
struct ConsInst {
    const void* X;
    const void* S;
    long long nf, z;
    unsigned long long* out;
    int lpf, pad;  // lanes per fiber; pad: elements per vector load
};
int launch_conservation_multi(int dtype, const ConsInst* d_insts, const int* d_block_off,
                              int n_inst, int n_blocks, cudaStream_t st);
int conservation_blocks(int dtype, const void* dS, long long nf, long long z);
ConsInst cons_inst(int dtype, const void* X, const void* S, long long nf, long long z,
                   unsigned long long* out);
// The residual from the bits launch_conservation left.
double cons_value(unsigned long long bits);
int launch_init_S(int dtype, const void* dX, void* dS, long long nf, long long z, uint64_t seed,
                  cudaStream_t st);

}  // namespace bldm
