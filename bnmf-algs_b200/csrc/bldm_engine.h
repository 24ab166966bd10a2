// Multi-instance engine: runs the fused sweep and finalize over many
// independent BLD instances of different shapes at once.  Used by the batched
// solver (bldm_batch_*) and the serving loop (bldm_server_*).
//
// An iteration of the instances of one lane-shape class (instances whose z
// maps to the same kernel) is one sweep launch and one finalize launch; each
// class runs its iterations on its own forked stream, the classes joining at
// the end of a run.  Or, persistent, one launch per class for a whole run
// whose tiles finalize their instances in their epilogues.
// Tiles (band x row range) of every instance of a class form the class grid;
// the tiling of an instance depends only on its own shape, so its results do
// not depend on which other instances share the launches.
#pragma once

#include <cstddef>
#include <cstdint>
#include <map>
#include <tuple>
#include <vector>

#include "bldm_internal.h"
#include "bldm_kernels.h"

namespace bldm {

// Lane-shape class of an instance: the sweep kernel it runs on.
struct ClassKey {
    int vec = 0, lpf = 0, mch = 0;
    bool multirow = false;  // fewer than 8 warps per row (narrow rows share a stage)
    bool operator<(const ClassKey& o) const {
        return std::tie(vec, lpf, mch, multirow) < std::tie(o.vec, o.lpf, o.mch, o.multirow);
    }
    bool operator==(const ClassKey& o) const {
        return vec == o.vec && lpf == o.lpf && mch == o.mch && multirow == o.multirow;
    }
};

// Tunable launch shape of a class: rows of S per tile (the tile height) and
// the depth of the bulk-copy stage ring (0 = as deep as shared memory allows).
struct ClassTune {
    int rows_per_tile = 0;
    int stages = 0;
};

// One instance: shape, derived geometry and device buffers.
struct EngineInstance {
    size_t x = 0, y = 0, z = 0;
    SweepCfg cfg{};      // lane shape, wpr, band_w, n_bands, n_rr, rr_base, n_ablk...
    int rr_cap = 0;      // row ranges the partial buffers hold (any tile height >= kMinTileRows)
    int nbB = 0;         // finalize-launch blocks for psi(beta_eph)
    uint32_t stage_need = 0;
    // device buffers (owned by the engine's user)
    void* X = nullptr;
    void* S = nullptr;
    double* alpha = nullptr;
    double* beta = nullptr;
    double* part_pjk = nullptr;
    double* part_ipk = nullptr;
    void* psiB = nullptr;
    void* psiA = nullptr;
    void* psiAS = nullptr;
    double* asum = nullptr;       // [rr_cap][z] fused finalize: alpha_eph summed per row range
    unsigned* counter = nullptr;  // [1 + n_bands + rr_cap] fused finalize arrival counters
    double* delta = nullptr;
    double* rel = nullptr;
    int* nz_rows = nullptr;  // [n_bands][x] rows with X != 0 per band, ascending
    int* nz_cnt = nullptr;   // [n_bands][x + 1] running counts of nz_rows
    // Host-side work estimate (Engine::set_work; empty: tiles weigh their bytes):
    // per band, running counts over the rows of the rows whose band segment of X
    // has a nonzero and of the nonzero passes.  [n_bands][x + 1] each.
    std::vector<int> work_rows, work_pass;
};

// Byte sizes of an instance's buffers, in the order of EngineInstance's fields.
struct InstanceBytes {
    size_t X, S, alpha, beta, pjk, ipk, psiB, psiA, psiAS, asum, counter, delta, rel, nzr, nzc;
    size_t total(size_t align) const;
};

// Smallest tile height a tuning may set; partial buffers are sized for it.
constexpr int kMinTileRows = 32;

class Engine {
  public:
    // skip_zero: once an update of every instance has stored the zeros of its
    // fibers with X == 0, later updates skip those fibers' stores and the rows
    // whose band segment of X is all zero (the result is the same).
    Engine(int dtype, int rows_per_tile, bool skip_zero = true);
    ~Engine();
    Engine(const Engine&) = delete;
    Engine& operator=(const Engine&) = delete;

    // Geometry of an instance of this shape (no device work).
    int configure(EngineInstance& in, size_t x, size_t y, size_t z) const;
    // Re-derives the row ranges of a configured instance from its class's
    // current tile height (within the capacity its buffers were sized for).
    void retile(EngineInstance& in) const;
    static ClassKey key_of(const EngineInstance& in);
    // Per-class launch shape; takes effect for instances configured or
    // retiled afterwards and at the next build.
    void set_tune(const ClassKey& k, const ClassTune& t) { tune_[k] = t; }
    ClassTune tune_of(const ClassKey& k) const;
    int default_rows_per_tile() const { return rows_per_tile_; }
    // Launch shape in effect for class i of the last build.
    bool class_info(size_t i, ClassKey* k, ClassTune* t, size_t* tiles) const;
    InstanceBytes bytes(const EngineInstance& in) const;
    // Points the instance's buffers into `base` (InstanceBytes layout, 256-aligned).
    void bind(EngineInstance& in, void* base) const;

    // Row lists of the instance's band segments with X != 0 (after X is set).
    int set_row_lists(EngineInstance& in, cudaStream_t st) const;
    // Work estimate of the instance's tiles from its X on the host (x * y
    // elements, FP64 or FP32 by f64), used to order the tiles of the next
    // builds (the batch sets it; the server, whose rounds hold few instances
    // and whose admission is on every request's latency path, does not).  A compact update sweeps only the rows of a band segment with a
    // nonzero and runs the update arithmetic only for the passes (32 / lpf
    // adjacent columns) with one, so instances of equal shape can differ in
    // work many times over.
    void set_work(EngineInstance& in, const void* X, bool f64) const;
    // (Re)builds the launch tables for the given instances; the pointers must
    // stay valid until the next build.  Clears the per-instance counters on st.
    int build(const std::vector<EngineInstance*>& insts, cudaStream_t st);
    // Runs `iters` iterations of every instance (from the S currently in the
    // buffers), tracking the relative change of the last one.  With prime,
    // the run first computes the axis sums and digamma tables of the current
    // S; without, it relies on those the last update (or prime()) left.
    // clean_first: every instance has had an update since its S was set, so
    // even the first update of this run may skip zero rows and stores.
    int run(size_t iters, int psi_mode, double eps, bool use_graph, cudaStream_t st,
            bool prime = true, bool clean_first = false);
    // Axis sums and digamma tables of the current S of every instance.
    int prime(int psi_mode, cudaStream_t st);
    int check(cudaStream_t st);

    // Persistent launches (one per class for a whole run; bldm_persist.cuh)
    // instead of one launch per class and round (the default, faster on mixes
    // of small instances).  Used when every class has a persistent kernel;
    // wait_ns bounds each dependency wait; stall_test makes instance 0's
    // first-round tiles wait for a round that cannot complete before them
    // (failure-detection tests).
    void set_persistent(bool on, unsigned long long wait_ns, bool stall_test) {
        persistent_ = on;
        wait_ns_ = wait_ns;
        stall_test_ = stall_test;
        drop_graphs();
    }
    bool persistent_active() const { return persistent_ && persist_ok_; }
    // Per-iteration launches: every class on its own stream with its own
    // finalize launch, joining once per run (the default: fewest waits, best in
    // a captured graph), or, joined, the classes' sweeps side by side and one
    // finalize launch for all instances per iteration (fewer launches, for
    // callers that launch rounds directly).  Both give bitwise the same results.
    void set_per_class_rounds(bool on) {
        per_class_rounds_ = on;
        drop_graphs();
    }

    int dtype() const { return dtype_; }
    size_t es() const { return es_; }
    size_t n_classes() const { return classes_.size(); }
    uint64_t launches() const { return launches_; }
    size_t table_bytes() const { return table_bytes_; }

  private:
    struct ShapeClass {
        int vec, lpf, mch;
        bool multirow;  // instances with fewer than 8 warps per row
        size_t max_z = 0;
        uint32_t stage_bytes = 0;
        int stages = 0;
        size_t smem = 0;
        std::vector<BatchTile> tiles;
        BatchTile* d_tiles = nullptr;
        cudaStream_t stream = nullptr;
        cudaEvent_t done = nullptr;
        // persistent launch of the class
        // the class's instances and its slice of the finalize tables
        std::vector<int> inst_ids;
        int fin_first = 0;   // first FinInst of the class
        int boff_first = 0;  // first block offset of the class
        int fin_blocks = 0;  // finalize blocks of the class
        void* pfn[2] = {nullptr, nullptr};  // by digamma of grad_plus: exact, psi_appr
        std::vector<PItem> items;  // one round: the tiles, largest first
        PItem* d_items = nullptr;
        int grid = 0;
    };
    int launch_persistent(size_t iters, int psi_mode, double eps, cudaStream_t st, bool prime,
                          bool clean_first);
    int launch_sequence(size_t iters, int psi_mode, double eps, cudaStream_t st, bool prime,
                        bool clean_first);
    int launch_class_sweep(ShapeClass& k, cudaStream_t s, bool update, int psi_mode, bool track,
                           double eps, bool clean);
    int launch_class_finalize(ShapeClass& k, cudaStream_t s, int psi_mode);
    int launch_rounds(size_t iters, int psi_mode, double eps, cudaStream_t st, bool prime,
                      bool clean_first);
    int launch_finalize_all(cudaStream_t st, int psi_mode);
    int launch_rounds_joined(size_t iters, int psi_mode, double eps, cudaStream_t st,
                             bool prime, bool clean_first);
    void free_tables();
    void drop_graphs();

    int dtype_;
    size_t es_;
    int rows_per_tile_;
    bool skip_zero_;
    int num_sms_;
    std::vector<EngineInstance*> insts_;
    std::vector<ShapeClass> classes_;
    void* d_tables_ = nullptr;  // SweepInst[n] | FinInst[n] | block_off[n+1] | err | tiles | items
    size_t table_bytes_ = 0;    // bytes in use
    size_t table_cap_ = 0;      // bytes allocated (grow-only across builds)
    void* h_stage_ = nullptr;   // pinned host staging of the tables
    size_t h_cap_ = 0;
    void* d_sinst_ = nullptr;
    void* d_finst_ = nullptr;
    int* d_block_off_ = nullptr;
    int* d_err_ = nullptr;
    cudaEvent_t fork_ = nullptr;
    uint64_t launches_ = 0;
    std::map<std::tuple<size_t, int, uint64_t, bool, bool>, cudaGraphExec_t> graphs_;
    // persistent launches: the counters cleared before every run (rounds done
    // per instance [n] | queue control per class)
    bool persistent_ = false;
    bool per_class_rounds_ = true;
    int fin_blocks_all_ = 0;
    int boff_all_first_ = 0;
    bool persist_ok_ = false;
    bool stall_test_ = false;
    unsigned long long wait_ns_ = 1000000000ull;
    void* d_counters_ = nullptr;
    size_t counter_bytes_ = 0;
    std::map<ClassKey, ClassTune> tune_;
};

}  // namespace bldm
