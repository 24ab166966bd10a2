// Multi-instance engine (see bldm_engine.h).
#include <algorithm>
#include <cstring>

#include "bldm_engine.h"
#include "bldm_finalize.cuh"

namespace bldm {

namespace {

size_t a256(size_t v) { return (v + 255) & ~size_t(255); }

// Cost of an element of a nonzero pass's update arithmetic relative to an
// element swept, chosen by timing the 512-instance uneven batch (FP32, X
// densities 1% to 89%) and its z = 64 class alone: weights 0 (bytes order), 2,
// 6, 16, 40 and 120 gave 113.5, 113.3, 112.4, 111.7, 110.7 and 110.9 ms per
// 150-iteration run of the batch and 506, 521, 469, 444, 415 and 408 us per
// iteration of the class.
constexpr double kPassWork = 40.0;

int sms_of_current_device() {
    int dev = 0, n = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 148;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0)
        return 148;
    return n;
}

#define ENG_CU(call)                                    \
    do {                                                \
        cudaError_t e_ = (call);                        \
        if (e_ != cudaSuccess) return cuda_status(e_);  \
    } while (0)

}  // namespace

size_t InstanceBytes::total(size_t align) const {
    const size_t parts[] = {X, S, alpha, beta, pjk, ipk, psiB, psiA, psiAS, asum, counter, delta,
                            rel, nzr, nzc};
    size_t t = 0;
    for (size_t p : parts) t += (p + align - 1) / align * align;
    return t;
}

Engine::Engine(int dtype, int rows_per_tile, bool skip_zero)
    : dtype_(dtype), es_(dtype == BLDM_F64 ? 8 : 4),
      rows_per_tile_(rows_per_tile > 0 ? rows_per_tile : 64), skip_zero_(skip_zero),
      num_sms_(sms_of_current_device()) {
    cudaEventCreateWithFlags(&fork_, cudaEventDisableTiming);
}

Engine::~Engine() {
    drop_graphs();
    free_tables();
    if (d_counters_) cudaFree(d_counters_);
    for (auto& c : classes_) {
        if (c.stream) cudaStreamDestroy(c.stream);
        if (c.done) cudaEventDestroy(c.done);
    }
    if (fork_) cudaEventDestroy(fork_);
}

int Engine::configure(EngineInstance& in, size_t x, size_t y, size_t z) const {
    if (x == 0 || y == 0 || z == 0) return BLDM_ERR_BAD_ARG;
    if (z > 1024) return BLDM_ERR_UNSUPPORTED;
    in.x = x;
    in.y = y;
    in.z = z;
    SweepCfg& c = in.cfg;
    if (lane_config(z, es_, c) != BLDM_OK) return BLDM_ERR_UNSUPPORTED;
    const int fpw = 32 / c.lpf;
    c.warps = kSweepWarps;
    c.wpr = kSweepWarps;
    while (c.wpr > 1 && size_t(c.wpr / 2) * c.cpw * fpw >= y) c.wpr /= 2;
    c.band_w = c.wpr * c.cpw * fpw;
    c.n_bands = int((y + c.band_w - 1) / c.band_w);
    const int rps = kSweepWarps / c.wpr;
    const int Rmin = std::max(rps, (kMinTileRows + rps - 1) / rps * rps);
    in.rr_cap = int((x + Rmin - 1) / Rmin);
    retile(in);
    const SlotLayout lay((long long)c.band_w, (long long)z, int(es_));
    in.stage_need = uint32_t(rps) * (lay.capS + lay.capX + lay.capA);
    // finalize launch geometry (the per-iteration form)
    const int KT = int(std::min<size_t>(z, kFinThreads));
    const int Rf = kFinThreads / KT;
    const long rows = std::max<long>(Rf, long((x + 127) / 128));
    c.rows_per_ablk = int(rows);
    c.n_ablk = int((x + rows - 1) / rows);
    in.nbB = int((y * z + kFinThreads - 1) / kFinThreads);
    return BLDM_OK;
}

ClassKey Engine::key_of(const EngineInstance& in) {
    ClassKey k;
    k.vec = in.cfg.vec;
    k.lpf = in.cfg.lpf;
    k.mch = in.cfg.mch;
    k.multirow = in.cfg.wpr < kSweepWarps;
    return k;
}

ClassTune Engine::tune_of(const ClassKey& k) const {
    auto it = tune_.find(k);
    ClassTune t = it == tune_.end() ? ClassTune{} : it->second;
    if (t.rows_per_tile <= 0) t.rows_per_tile = rows_per_tile_;
    return t;
}

// Row ranges of ceil(x / n_rr) rows rounded up to whole stages; since that is
// at most the tile height, the last range is never empty.
void Engine::retile(EngineInstance& in) const {
    SweepCfg& c = in.cfg;
    const int rps = kSweepWarps / c.wpr;
    const int want = std::max(kMinTileRows, tune_of(key_of(in)).rows_per_tile);
    const int R = std::max(rps, (want + rps - 1) / rps * rps);
    c.n_rr = std::min(in.rr_cap, int((in.x + R - 1) / R));
    c.rr_base = int((in.x + c.n_rr - 1) / c.n_rr);
    c.rr_base = (c.rr_base + rps - 1) / rps * rps;
    c.rr_extra = 0;
}

bool Engine::class_info(size_t i, ClassKey* k, ClassTune* t, size_t* tiles) const {
    if (i >= classes_.size()) return false;
    const ShapeClass& c = classes_[i];
    ClassKey key;
    key.vec = c.vec;
    key.lpf = c.lpf;
    key.mch = c.mch;
    key.multirow = c.multirow;
    if (k) *k = key;
    if (t) {
        *t = tune_of(key);
        t->stages = c.stages;
    }
    if (tiles) *tiles = c.tiles.size();
    return true;
}

InstanceBytes Engine::bytes(const EngineInstance& in) const {
    const SweepCfg& c = in.cfg;
    InstanceBytes b;
    b.X = in.x * in.y * es_;
    b.S = in.x * in.y * in.z * es_;
    b.alpha = in.x * 8;
    b.beta = in.z * 8;
    b.pjk = size_t(in.rr_cap) * in.y * in.z * 8;
    b.ipk = size_t(c.n_bands) * in.x * in.z * 8;
    b.psiB = in.y * in.z * es_;
    b.psiA = in.x * in.z * es_;
    b.psiAS = in.z * es_;
    // sums of alpha_eph over row blocks (finalize launch) or row ranges (fused
    // finalize), and the last-arrival counters: word 0 of the finalize launch,
    // or instance | per band | per row range of the fused finalize
    b.asum = size_t(std::max(c.n_ablk, in.rr_cap)) * in.z * 8;
    b.counter = std::max<size_t>(16, (1 + size_t(c.n_bands) + size_t(in.rr_cap)) * sizeof(unsigned));
    b.delta = size_t(in.rr_cap) * c.n_bands * 16;
    b.rel = 8;
    b.nzr = size_t(c.n_bands) * in.x * 4;
    b.nzc = size_t(c.n_bands) * (in.x + 1) * 4;
    return b;
}

void Engine::set_work(EngineInstance& in, const void* X, bool f64) const {
    const SweepCfg& c = in.cfg;
    const size_t x = in.x, y = in.y;
    const int fpw = 32 / c.lpf;
    in.work_rows.assign(size_t(c.n_bands) * (x + 1), 0);
    in.work_pass.assign(size_t(c.n_bands) * (x + 1), 0);
    auto nonzero = [&](size_t e) {
        return f64 ? static_cast<const double*>(X)[e] != 0.0
                   : static_cast<const float*>(X)[e] != 0.0f;
    };
    for (int b = 0; b < c.n_bands; ++b) {
        const size_t c0 = size_t(b) * c.band_w;
        const size_t c1 = std::min(y, c0 + size_t(c.band_w));
        int* wr = &in.work_rows[size_t(b) * (x + 1)];
        int* wp = &in.work_pass[size_t(b) * (x + 1)];
        for (size_t i = 0; i < x; ++i) {
            int passes = 0;
            for (size_t p0 = c0; p0 < c1; p0 += size_t(fpw)) {
                bool any = false;
                for (size_t j = p0; j < std::min(c1, p0 + size_t(fpw)) && !any; ++j)
                    any = nonzero(i * y + j);
                passes += any ? 1 : 0;
            }
            wr[i + 1] = wr[i] + (passes > 0 ? 1 : 0);
            wp[i + 1] = wp[i] + passes;
        }
    }
}

int Engine::set_row_lists(EngineInstance& in, cudaStream_t st) const {
    return launch_nz_rows(dtype_, in.X, (long long)in.x, (long long)in.y, in.cfg.band_w,
                          in.cfg.n_bands, in.nz_rows, in.nz_cnt, st);
}

void Engine::bind(EngineInstance& in, void* base) const {
    const InstanceBytes b = bytes(in);
    char* p = static_cast<char*>(base);
    auto take = [&](size_t n) {
        char* q = p;
        p += a256(n);
        return q;
    };
    in.X = take(b.X);
    in.S = take(b.S);
    in.alpha = reinterpret_cast<double*>(take(b.alpha));
    in.beta = reinterpret_cast<double*>(take(b.beta));
    in.part_pjk = reinterpret_cast<double*>(take(b.pjk));
    in.part_ipk = reinterpret_cast<double*>(take(b.ipk));
    in.psiB = take(b.psiB);
    in.psiA = take(b.psiA);
    in.psiAS = take(b.psiAS);
    in.asum = reinterpret_cast<double*>(take(b.asum));
    in.counter = reinterpret_cast<unsigned*>(take(b.counter));
    in.delta = reinterpret_cast<double*>(take(b.delta));
    in.rel = reinterpret_cast<double*>(take(b.rel));
    in.nz_rows = reinterpret_cast<int*>(take(b.nzr));
    in.nz_cnt = reinterpret_cast<int*>(take(b.nzc));
}

void Engine::free_tables() {
    for (auto& c : classes_) c.d_tiles = nullptr;
    if (d_tables_) cudaFree(d_tables_);
    if (h_stage_) cudaFreeHost(h_stage_);
    d_tables_ = nullptr;
    h_stage_ = nullptr;
    table_bytes_ = table_cap_ = h_cap_ = 0;
}

void Engine::drop_graphs() {
    for (auto& g : graphs_) cudaGraphExecDestroy(g.second);
    graphs_.clear();
}

// SweepInst[n] in instance order; FinInst entries in `fin_order` (the instances
// of each class together, so that a class's finalize launch takes a slice).
template <typename T>
static void fill_tables(const std::vector<EngineInstance*>& insts, std::vector<char>& host,
                        size_t o_sinst, size_t o_finst, bool skip_zero,
                        const std::vector<int>& fin_pos) {
    SweepInst<T>* si = reinterpret_cast<SweepInst<T>*>(host.data() + o_sinst);
    FinInst<T>* fi = reinterpret_cast<FinInst<T>*>(host.data() + o_finst);
    for (size_t n = 0; n < insts.size(); ++n) {
        const EngineInstance& in = *insts[n];
        const SweepCfg& c = in.cfg;
        SweepInst<T>& s = si[n];
        s.S = static_cast<T*>(in.S);
        s.X = static_cast<const T*>(in.X);
        s.psiB = static_cast<const T*>(in.psiB);
        s.psiA = static_cast<const T*>(in.psiA);
        s.psiAS = static_cast<const T*>(in.psiAS);
        s.part_pjk = in.part_pjk;
        s.part_ipk = in.part_ipk;
        s.delta_part = in.delta;
        s.nz_rows = skip_zero ? in.nz_rows : nullptr;
        s.nz_cnt = skip_zero ? in.nz_cnt : nullptr;
        s.x = (long long)in.x;
        s.y = (long long)in.y;
        s.z = (long long)in.z;
        s.n_bands = c.n_bands;
        s.band_w = c.band_w;
        s.wpr = c.wpr;
        s.n_rr = c.n_rr;
        s.rr_base = c.rr_base;
        s.rr_extra = c.rr_extra;
        s.alpha = in.alpha;
        s.beta = in.beta;
        s.fcnt = in.counter;
        s.asum_rr = in.asum;
        s.rel_change = in.rel;
        s.done = nullptr;
        FinInst<T>& f = fi[fin_pos[n]];
        f.red = nullptr;
        f.part_pjk = in.part_pjk;
        f.part_ipk = in.part_ipk;
        f.alpha = in.alpha;
        f.beta = in.beta;
        f.psiB = static_cast<T*>(in.psiB);
        f.psiA = static_cast<T*>(in.psiA);
        f.psiAS = static_cast<T*>(in.psiAS);
        f.asum_part = in.asum;
        f.counter = in.counter;
        f.delta_part = in.delta;
        f.rel_change = in.rel;
        f.x = (long long)in.x;
        f.y = (long long)in.y;
        f.z = (long long)in.z;
        f.n_rr = c.n_rr;
        f.n_bands = c.n_bands;
        f.nbB = in.nbB;
        f.n_ablk = c.n_ablk;
        f.rows_per_ablk = c.rows_per_ablk;
        f.n_tiles = c.n_rr * c.n_bands;
    }
}

int Engine::build(const std::vector<EngineInstance*>& insts, cudaStream_t st) {
    drop_graphs();
    // The previous tables may still be read by work queued on st; the new ones
    // are written on st behind it, so the device buffer can be reused.
    for (auto& c : classes_) c.d_tiles = nullptr;
    insts_ = insts;
    // Lane-shape classes, keeping streams of classes that already exist.
    std::vector<ShapeClass> old;
    old.swap(classes_);
    auto class_of = [&](const SweepCfg& c) -> ShapeClass& {
        for (auto& k : classes_)
            if (k.vec == c.vec && k.lpf == c.lpf && k.mch == c.mch &&
                k.multirow == (c.wpr < kSweepWarps))
                return k;
        ShapeClass k;
        k.vec = c.vec;
        k.lpf = c.lpf;
        k.mch = c.mch;
        k.multirow = c.wpr < kSweepWarps;
        classes_.push_back(k);
        return classes_.back();
    };
    for (EngineInstance* in : insts) {
        ShapeClass& k = class_of(in->cfg);
        k.max_z = std::max(k.max_z, in->z);
        k.stage_bytes = std::max(k.stage_bytes, in->stage_need);
    }
    for (size_t i = 0; i < classes_.size(); ++i) {
        if (i < old.size()) {
            classes_[i].stream = old[i].stream;
            classes_[i].done = old[i].done;
            old[i].stream = nullptr;
            old[i].done = nullptr;
        } else {
            ENG_CU(cudaStreamCreateWithFlags(&classes_[i].stream, cudaStreamNonBlocking));
            ENG_CU(cudaEventCreateWithFlags(&classes_[i].done, cudaEventDisableTiming));
        }
    }
    for (auto& k : old) {
        if (k.stream) cudaStreamDestroy(k.stream);
        if (k.done) cudaEventDestroy(k.done);
    }
    // Ring depth and shared memory per class (2 CTAs/SM when they fit).
    for (auto& k : classes_) {
        const size_t per_stage = k.stage_bytes + size_t(kSweepWarps) * k.max_z * 8;
        const size_t fixed = 64 + k.max_z * es_ + 128;
        long s = long((110 * 1024 - std::min<size_t>(fixed, 110 * 1024)) / per_stage);
        if (s < 2) s = long((220 * 1024 - std::min<size_t>(fixed, 220 * 1024)) / per_stage);
        if (s < 2) return BLDM_ERR_UNSUPPORTED;
        k.stages = int(std::min(8L, s));
        const ClassTune t = tune_of(ClassKey{k.vec, k.lpf, k.mch, k.multirow});
        if (t.stages >= 2) k.stages = std::min(k.stages, t.stages);
        k.smem = size_t(k.stages) * per_stage + fixed;
        // a persistent launch's finalize items keep their row sums in the ring
        k.smem = std::max(k.smem, size_t(kFinAccDoubles) * sizeof(double));
        for (int mode = SWEEP_SUMS; mode <= SWEEP_COMPACT; ++mode)
            for (int ap = 0; ap < 2; ++ap) {
                void* fn = pick_sweep_fn(dtype_, k.vec, k.lpf, k.mch, mode, ap != 0, true,
                                         k.multirow);
                if (!fn) return BLDM_ERR_UNSUPPORTED;
                const int rc_attr = ensure_smem_attr(fn, k.smem);
                if (rc_attr) return rc_attr;
            }
    }
    // Tiles of every instance, per class.
    for (size_t n = 0; n < insts.size(); ++n) {
        const EngineInstance& in = *insts[n];
        const SweepCfg& c = in.cfg;
        ShapeClass& k = class_of(c);
        const int rps = kSweepWarps / c.wpr;
        if (rps > 1 &&
            size_t(rps) * c.band_w * in.z * 8 > size_t(k.stages) * size_t(k.stage_bytes))
            return BLDM_ERR_UNSUPPORTED;
        for (int rr = 0; rr < c.n_rr; ++rr)
            for (int b = 0; b < c.n_bands; ++b) k.tiles.push_back(BatchTile{int(n), b, rr, 0});
    }
    // Largest tiles first: blocks start in index order as slots free up, so a
    // class grid of several waves ends with its smallest tiles (longest
    // processing time first).  A tile weighs the elements of the rows a compact
    // update sweeps plus kPassWork times those of its nonzero passes (the update
    // arithmetic), from the instance's work estimate, else its elements.  The
    // order depends only on the instances' shapes and X and changes no result.
    for (auto& k : classes_) {
        auto work = [&](const BatchTile& t) -> double {
            const EngineInstance& in = *insts[size_t(t.inst)];
            const SweepCfg& c = in.cfg;
            const long long r0 = (long long)t.rr * c.rr_base;
            const long long rows = std::min<long long>(c.rr_base, (long long)in.x - r0);
            const long long cols =
                std::min<long long>(c.band_w, (long long)in.y - (long long)t.band * c.band_w);
            if (in.work_rows.empty()) return double(rows * cols * (long long)in.z);
            const size_t o = size_t(t.band) * (in.x + 1);
            const double swept = in.work_rows[o + size_t(r0 + rows)] - in.work_rows[o + size_t(r0)];
            const double passes = in.work_pass[o + size_t(r0 + rows)] - in.work_pass[o + size_t(r0)];
            return (swept * double(cols) + kPassWork * passes * double(32 / c.lpf)) *
                   double(in.z);
        };
        std::stable_sort(k.tiles.begin(), k.tiles.end(),
                         [&](const BatchTile& a, const BatchTile& b) { return work(a) > work(b); });
    }
    // Persistent launches: every class needs its persistent kernel (short
    // fibers); a round of a class is its tiles in the order above.
    const size_t n = insts.size();
    persist_ok_ = !classes_.empty();
    for (auto& k : classes_) {
        k.items.clear();
        for (int ap = 0; ap < 2; ++ap)
            k.pfn[ap] = pick_persist_fn(dtype_, k.vec, k.lpf, k.mch, k.multirow, ap != 0);
        if (!k.pfn[0] || !k.pfn[1]) {
            persist_ok_ = false;
            continue;
        }
        for (const BatchTile& bt : k.tiles) k.items.push_back(PItem{0, bt.inst, bt.band, bt.rr});
        for (int ap = 0; ap < 2; ++ap) {
            const int rc_attr = ensure_smem_attr(k.pfn[ap], k.smem);
            if (rc_attr) return rc_attr;
        }
    }
    if (persist_ok_) {
        // A class's launch gets at most one wave of CTAs (at most one round's
        // tiles); launched side by side, a later class takes the SMs as an
        // earlier one drains.  (Measured: splitting one wave between the classes
        // in proportion to their bytes starves the classes of small instances,
        // whose rounds are bound by latency, not bytes.)
        for (auto& k : classes_) {
            int per_sm = 0;
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k.pfn[1], kSweepThreads,
                                                              k.smem) != cudaSuccess ||
                per_sm < 1)
                per_sm = 1;
            const long cap = long(per_sm) * num_sms_;
            k.grid = int(std::max(1L, std::min(cap, long(k.items.size()))));
        }
        // Every class but the one with the most tiles gets half that: a
        // persistent CTA keeps its SM while it waits for its instance's
        // previous round, and the small classes' rounds, bound by latency, can
        // take two passes over their tiles and still end before the large
        // class.  (Uneven 512-instance batch, 150 iterations: 131.6 ms against
        // 152-157 ms with a full share, 136 ms at 2/3, 146 ms at 1/4.)
        {
            size_t big = 0;
            for (size_t c = 1; c < classes_.size(); ++c)
                if (classes_[c].items.size() > classes_[big].items.size()) big = c;
            for (size_t c = 0; c < classes_.size(); ++c)
                if (c != big) classes_[c].grid = std::max(1, (classes_[c].grid + 1) / 2);
        }
        const size_t cb = (n + 4 * classes_.size()) * sizeof(unsigned);
        if (cb > counter_bytes_) {
            if (d_counters_) cudaFree(d_counters_);
            d_counters_ = nullptr;
            counter_bytes_ = 0;
            ENG_CU(cudaMalloc(&d_counters_, cb * 2));
            counter_bytes_ = cb * 2;
        }
    }
    // Each class's instances, in instance order: the class's finalize launch takes
    // their FinInst entries (stored together) and block offsets.
    std::vector<int> fin_pos(n, 0);
    {
        int pos = 0;
        size_t boff_at = 0;
        for (auto& k : classes_) {
            k.inst_ids.clear();
            k.fin_first = pos;
            k.boff_first = int(boff_at);
            k.fin_blocks = 0;
            for (size_t i = 0; i < n; ++i) {
                const SweepCfg& c = insts[i]->cfg;
                if (k.vec == c.vec && k.lpf == c.lpf && k.mch == c.mch &&
                    k.multirow == (c.wpr < kSweepWarps)) {
                    k.inst_ids.push_back(int(i));
                    fin_pos[i] = pos++;
                }
            }
            boff_at += k.inst_ids.size() + 1;
        }
    }
    // Device tables: SweepInst[n] | FinInst[n] (by class) | block offsets (per
    // class, n_c + 1 each) | err | tiles per class | (persistent) items per class.
    const size_t s_sz = dtype_ == BLDM_F64 ? sizeof(SweepInst<double>) : sizeof(SweepInst<float>);
    const size_t f_sz = dtype_ == BLDM_F64 ? sizeof(FinInst<double>) : sizeof(FinInst<float>);
    const size_t o_sinst = 0;
    const size_t o_finst = a256(o_sinst + n * s_sz);
    const size_t o_boff = a256(o_finst + n * f_sz);
    // per-class offsets (n_c + 1 each), then the offsets of all instances (n + 1)
    const size_t n_boff = (n + classes_.size()) + (n + 1);
    const size_t o_err = a256(o_boff + n_boff * sizeof(int));
    size_t off = a256(o_err + 64);
    std::vector<size_t> o_tiles(classes_.size()), o_items(classes_.size());
    for (size_t c = 0; c < classes_.size(); ++c) {
        o_tiles[c] = off;
        off = a256(off + classes_[c].tiles.size() * sizeof(BatchTile));
    }
    for (size_t c = 0; c < classes_.size(); ++c) {
        o_items[c] = off;
        off = a256(off + classes_[c].items.size() * sizeof(PItem));
    }
    table_bytes_ = off;
    if (table_bytes_ > h_cap_) {
        // a pinned staging buffer may still feed an earlier async copy
        ENG_CU(cudaStreamSynchronize(st));
        if (h_stage_) cudaFreeHost(h_stage_);
        h_stage_ = nullptr;
        h_cap_ = 0;
        ENG_CU(cudaMallocHost(&h_stage_, table_bytes_ * 2));
        h_cap_ = table_bytes_ * 2;
    } else {
        ENG_CU(cudaStreamSynchronize(st));  // the staging buffer is free again
    }
    if (table_bytes_ > table_cap_) {
        if (d_tables_) cudaFree(d_tables_);
        d_tables_ = nullptr;
        table_cap_ = 0;
        ENG_CU(cudaMalloc(&d_tables_, table_bytes_ * 2));
        table_cap_ = table_bytes_ * 2;
    }
    char* host = static_cast<char*>(h_stage_);
    std::memset(host, 0, table_bytes_);
    std::vector<char> hv;  // fill_tables works on a vector view of the staging buffer
    hv.resize(o_boff);
    if (dtype_ == BLDM_F64)
        fill_tables<double>(insts, hv, o_sinst, o_finst, skip_zero_, fin_pos);
    else
        fill_tables<float>(insts, hv, o_sinst, o_finst, skip_zero_, fin_pos);
    std::memcpy(host, hv.data(), o_boff);
    int* boff = reinterpret_cast<int*>(host + o_boff);
    for (auto& k : classes_) {
        int* kb = boff + k.boff_first;
        int blocks = 0;
        for (size_t j = 0; j < k.inst_ids.size(); ++j) {
            kb[j] = blocks;
            const EngineInstance& in = *insts[size_t(k.inst_ids[j])];
            blocks += in.nbB + in.cfg.n_ablk;
        }
        kb[k.inst_ids.size()] = blocks;
        k.fin_blocks = blocks;
    }
    {
        // all instances in the FinInst order (the classes one after the other)
        int* ab = boff + n + classes_.size();
        int blocks = 0, j = 0;
        for (auto& k : classes_)
            for (int i : k.inst_ids) {
                ab[j++] = blocks;
                blocks += insts[size_t(i)]->nbB + insts[size_t(i)]->cfg.n_ablk;
            }
        ab[n] = blocks;
        fin_blocks_all_ = blocks;
        boff_all_first_ = int(n + classes_.size());
    }
    char* base = static_cast<char*>(d_tables_);
    for (size_t c = 0; c < classes_.size(); ++c) {
        std::memcpy(host + o_tiles[c], classes_[c].tiles.data(),
                    classes_[c].tiles.size() * sizeof(BatchTile));
        classes_[c].d_tiles = reinterpret_cast<BatchTile*>(base + o_tiles[c]);
        std::memcpy(host + o_items[c], classes_[c].items.data(),
                    classes_[c].items.size() * sizeof(PItem));
        classes_[c].d_items = reinterpret_cast<PItem*>(base + o_items[c]);
    }

    d_sinst_ = base + o_sinst;
    d_finst_ = base + o_finst;
    d_block_off_ = reinterpret_cast<int*>(base + o_boff);
    d_err_ = reinterpret_cast<int*>(base + o_err);
    ENG_CU(cudaMemcpyAsync(d_tables_, host, table_bytes_, cudaMemcpyHostToDevice, st));
    (void)st;
    return BLDM_OK;
}

template <typename T>
static void launch_class_kernel(void* fn, unsigned grid, size_t smem, cudaStream_t s,
                                const void* d_sinst, const BatchTile* d_tiles, int stages,
                                uint32_t stage_bytes, double eps, int* err, bool track,
                                int plus_appr, int minus_appr) {
    BatchSweepParams<T> p;
    p.insts = static_cast<const SweepInst<T>*>(d_sinst);
    p.tiles = d_tiles;
    p.L.stages = stages;
    p.L.stage_bytes = stage_bytes;
    p.L.eps = eps;
    p.L.err = err;
    p.L.plus_appr = plus_appr;
    p.L.minus_appr = minus_appr;
    p.track = track ? 1 : 0;
    reinterpret_cast<void (*)(const BatchSweepParams<T>)>(fn)<<<grid, kSweepThreads, smem, s>>>(p);
}

// One sweep launch of class k on stream s.
int Engine::launch_class_sweep(ShapeClass& k, cudaStream_t s, bool update, int psi_mode,
                               bool track, double eps, bool clean) {
    const int plus_appr = psi_mode != BLDM_PSI_EXACT;
    const int minus_appr = psi_mode == BLDM_PSI_APPR;
    const int mode = !update ? SWEEP_SUMS : (clean ? SWEEP_COMPACT : SWEEP_UPDATE);
    void* fn = pick_sweep_fn(dtype_, k.vec, k.lpf, k.mch, mode, plus_appr != 0, true, k.multirow);
    if (dtype_ == BLDM_F64)
        launch_class_kernel<double>(fn, unsigned(k.tiles.size()), k.smem, s, d_sinst_, k.d_tiles,
                                    k.stages, k.stage_bytes, eps, d_err_, track, plus_appr,
                                    minus_appr);
    else
        launch_class_kernel<float>(fn, unsigned(k.tiles.size()), k.smem, s, d_sinst_, k.d_tiles,
                                   k.stages, k.stage_bytes, eps, d_err_, track, plus_appr,
                                   minus_appr);
    launches_ += 1;
    return cuda_status(cudaGetLastError());
}

template <typename T>
static void launch_fin_kernel(unsigned grid, cudaStream_t s, const void* d_finst,
                              const int* d_boff, int n, int plus_appr, int minus_appr) {
    BatchFinParams<T> p;
    p.insts = static_cast<const FinInst<T>*>(d_finst);
    p.block_off = d_boff;
    p.n_inst = n;
    p.plus_appr = plus_appr;
    p.minus_appr = minus_appr;
    void* fn = finalize_batch_fn(sizeof(T) == 8 ? BLDM_F64 : BLDM_F32);
    reinterpret_cast<void (*)(const BatchFinParams<T>)>(fn)<<<grid, kFinThreads, 0, s>>>(p);
}

// The finalize of class k's instances on stream s (block_off maps blocks to them).
int Engine::launch_class_finalize(ShapeClass& k, cudaStream_t s, int psi_mode) {
    const int plus_appr = psi_mode != BLDM_PSI_EXACT;
    const int minus_appr = psi_mode == BLDM_PSI_APPR;
    const int* boff = d_block_off_ + k.boff_first;
    const int nk = int(k.inst_ids.size());
    if (dtype_ == BLDM_F64)
        launch_fin_kernel<double>(unsigned(k.fin_blocks), s,
                                  static_cast<const FinInst<double>*>(d_finst_) + k.fin_first,
                                  boff, nk, plus_appr, minus_appr);
    else
        launch_fin_kernel<float>(unsigned(k.fin_blocks), s,
                                 static_cast<const FinInst<float>*>(d_finst_) + k.fin_first, boff,
                                 nk, plus_appr, minus_appr);
    launches_ += 1;
    return cuda_status(cudaGetLastError());
}

// Each class's rounds on its own forked stream: an instance's round needs only
// its own class's previous finalize, so the classes never wait for each other
// until the run's join (a class of small, latency-bound instances overlaps the
// others instead of adding to every round).
int Engine::launch_rounds(size_t iters, int psi_mode, double eps, cudaStream_t st, bool prime,
                          bool clean_first) {
    const bool fork = classes_.size() > 1;
    if (fork) ENG_CU(cudaEventRecord(fork_, st));
    for (auto& k : classes_) {
        if (k.tiles.empty()) continue;
        cudaStream_t s = fork ? k.stream : st;
        if (fork) ENG_CU(cudaStreamWaitEvent(s, fork_, 0));
        int rc = BLDM_OK;
        if (prime) {
            rc = launch_class_sweep(k, s, false, psi_mode, false, eps, false);
            if (!rc) rc = launch_class_finalize(k, s, psi_mode);
        }
        for (size_t it = 0; it < iters && !rc; ++it) {
            const bool clean = skip_zero_ && (clean_first || it > 0);
            rc = launch_class_sweep(k, s, true, psi_mode, it + 1 == iters, eps, clean);
            if (!rc) rc = launch_class_finalize(k, s, psi_mode);
        }
        if (rc) return rc;
        if (fork) ENG_CU(cudaEventRecord(k.done, s));
    }
    if (fork)
        for (auto& k : classes_)
            if (!k.tiles.empty()) ENG_CU(cudaStreamWaitEvent(st, k.done, 0));
    return BLDM_OK;
}

// One finalize launch for every instance (the joined form).
int Engine::launch_finalize_all(cudaStream_t st, int psi_mode) {
    const int plus_appr = psi_mode != BLDM_PSI_EXACT;
    const int minus_appr = psi_mode == BLDM_PSI_APPR;
    const int* boff = d_block_off_ + boff_all_first_;
    const int n = int(insts_.size());
    if (dtype_ == BLDM_F64)
        launch_fin_kernel<double>(unsigned(fin_blocks_all_), st,
                                  static_cast<const FinInst<double>*>(d_finst_), boff, n,
                                  plus_appr, minus_appr);
    else
        launch_fin_kernel<float>(unsigned(fin_blocks_all_), st,
                                 static_cast<const FinInst<float>*>(d_finst_), boff, n,
                                 plus_appr, minus_appr);
    launches_ += 1;
    return cuda_status(cudaGetLastError());
}

// The joined form: per iteration, the classes' sweeps side by side on forked
// streams, a join, and one finalize launch for every instance (fewer launches
// than the per-class form: for callers that launch rounds directly).
int Engine::launch_rounds_joined(size_t iters, int psi_mode, double eps, cudaStream_t st,
                                 bool prime, bool clean_first) {
    const bool fork = classes_.size() > 1;
    auto sweeps = [&](bool update, bool track, bool clean) -> int {
        if (fork) ENG_CU(cudaEventRecord(fork_, st));
        for (auto& k : classes_) {
            if (k.tiles.empty()) continue;
            cudaStream_t s = fork ? k.stream : st;
            if (fork) ENG_CU(cudaStreamWaitEvent(s, fork_, 0));
            const int rc = launch_class_sweep(k, s, update, psi_mode, track, eps, clean);
            if (rc) return rc;
            if (fork) ENG_CU(cudaEventRecord(k.done, s));
        }
        if (fork)
            for (auto& k : classes_)
                if (!k.tiles.empty()) ENG_CU(cudaStreamWaitEvent(st, k.done, 0));
        return launch_finalize_all(st, psi_mode);
    };
    int rc = BLDM_OK;
    if (prime) rc = sweeps(false, false, false);
    for (size_t it = 0; it < iters && !rc; ++it)
        rc = sweeps(true, it + 1 == iters, skip_zero_ && (clean_first || it > 0));
    return rc;
}

int Engine::prime(int psi_mode, cudaStream_t st) {
    if (psi_mode < BLDM_PSI_EXACT || psi_mode > BLDM_PSI_LEGACY_CUDA) return BLDM_ERR_BAD_ARG;
    if (insts_.empty()) return BLDM_OK;
    return per_class_rounds_ ? launch_rounds(0, psi_mode, 0.0, st, true, false)
                             : launch_rounds_joined(0, psi_mode, 0.0, st, true, false);
}

template <typename T>
static int launch_persist_class(void* fn, int grid, size_t smem, cudaStream_t s,
                                const PersistParams<T>& p) {
    reinterpret_cast<void (*)(const PersistParams<T>)>(fn)<<<grid, kSweepThreads, smem, s>>>(p);
    return cuda_status(cudaGetLastError());
}

// One launch per class for the whole run (rounds = prime round + iters).
int Engine::launch_persistent(size_t iters, int psi_mode, double eps, cudaStream_t st,
                              bool prime, bool clean_first) {
    const int plus_appr = psi_mode != BLDM_PSI_EXACT;
    const int minus_appr = psi_mode == BLDM_PSI_APPR;
    const size_t n = insts_.size();
    const int rounds = int(iters) + (prime ? 1 : 0);
    unsigned* ctr = static_cast<unsigned*>(d_counters_);
    ENG_CU(cudaMemsetAsync(ctr, 0, (n + 4 * classes_.size()) * sizeof(unsigned), st));
    const bool fork = classes_.size() > 1;
    if (fork) ENG_CU(cudaEventRecord(fork_, st));
    // Classes with the fewest tiles per round first: a launch whose CTAs are
    // resident keeps its SMs for the whole run, so the large class taking the
    // SMs last lets the small, latency-bound classes run beside it (uneven
    // 512-instance batch: 157 ms per 150-iteration run against 167 ms in
    // class order and 172 ms largest first).
    std::vector<size_t> ord(classes_.size());
    for (size_t c = 0; c < ord.size(); ++c) ord[c] = c;
    std::stable_sort(ord.begin(), ord.end(), [&](size_t a, size_t b) {
        return classes_[a].items.size() < classes_[b].items.size();
    });
    for (size_t oc = 0; oc < ord.size(); ++oc) {
        const size_t c = ord[oc];
        ShapeClass& k = classes_[c];
        if (k.items.empty()) continue;
        cudaStream_t s = fork ? k.stream : st;
        if (fork) ENG_CU(cudaStreamWaitEvent(s, fork_, 0));
        int rc;
        auto fill = [&](auto& p) {
            p.items = k.d_items;
            p.done = ctr;
            p.ctl = reinterpret_cast<PersistCtl*>(ctr + n) + c;
            p.L.stages = k.stages;
            p.L.stage_bytes = k.stage_bytes;
            p.L.eps = eps;
            p.L.err = d_err_;
            p.L.plus_appr = plus_appr;
            p.L.minus_appr = minus_appr;
            p.P = int(k.items.size());
            p.rounds = rounds;
            p.prime = prime ? 1 : 0;
            p.compact_from = !skip_zero_ ? rounds : (prime ? 1 : 0) + (clean_first ? 0 : 1);
            p.wait_ns = wait_ns_;
            p.stall_test = stall_test_ ? 1 : 0;
        };
        void* fn = k.pfn[plus_appr ? 1 : 0];
        if (dtype_ == BLDM_F64) {
            PersistParams<double> p;
            p.sinst = static_cast<const SweepInst<double>*>(d_sinst_);
            fill(p);
            rc = launch_persist_class<double>(fn, k.grid, k.smem, s, p);
        } else {
            PersistParams<float> p;
            p.sinst = static_cast<const SweepInst<float>*>(d_sinst_);
            fill(p);
            rc = launch_persist_class<float>(fn, k.grid, k.smem, s, p);
        }
        if (rc) return rc;
        launches_ += 1;
        if (fork) ENG_CU(cudaEventRecord(k.done, s));
    }
    if (fork)
        for (auto& k : classes_)
            if (!k.items.empty()) ENG_CU(cudaStreamWaitEvent(st, k.done, 0));
    return BLDM_OK;
}

int Engine::launch_sequence(size_t iters, int psi_mode, double eps, cudaStream_t st,
                            bool prime, bool clean_first) {
    if (persistent_active())
        return launch_persistent(iters, psi_mode, eps, st, prime, clean_first);
    if (!per_class_rounds_)
        return launch_rounds_joined(iters, psi_mode, eps, st, prime, clean_first);
    return launch_rounds(iters, psi_mode, eps, st, prime, clean_first);
}

int Engine::run(size_t iters, int psi_mode, double eps, bool use_graph, cudaStream_t st,
                bool prime, bool clean_first) {
    if (psi_mode < BLDM_PSI_EXACT || psi_mode > BLDM_PSI_LEGACY_CUDA) return BLDM_ERR_BAD_ARG;
    if (iters == 0 || insts_.empty()) return BLDM_OK;
    if (!use_graph || st == nullptr)
        return launch_sequence(iters, psi_mode, eps, st, prime, clean_first);
    uint64_t eb;
    std::memcpy(&eb, &eps, sizeof eb);
    const auto key = std::make_tuple(iters, psi_mode, eb, prime, clean_first);
    auto it = graphs_.find(key);
    if (it == graphs_.end()) {
        const uint64_t l0 = launches_;
        ENG_CU(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
        const int rc = launch_sequence(iters, psi_mode, eps, st, prime, clean_first);
        cudaGraph_t g = nullptr;
        const cudaError_t ce = cudaStreamEndCapture(st, &g);
        launches_ = l0;
        if (rc) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        ENG_CU(ce);
        cudaGraphExec_t exec = nullptr;
        const cudaError_t ie = cudaGraphInstantiate(&exec, g, 0);
        cudaGraphDestroy(g);
        ENG_CU(ie);
        it = graphs_.emplace(key, exec).first;
    }
    ENG_CU(cudaGraphLaunch(it->second, st));
    size_t active_classes = 0;
    for (const auto& k : classes_) active_classes += k.tiles.empty() ? 0 : 1;
    launches_ += persistent_active()   ? active_classes
                 : per_class_rounds_ ? (iters + (prime ? 1 : 0)) * 2 * active_classes
                                     : (iters + (prime ? 1 : 0)) * (active_classes + 1);
    return BLDM_OK;
}

int Engine::check(cudaStream_t st) {
    ENG_CU(cudaStreamSynchronize(st));
    if (!d_err_) return BLDM_OK;
    int herr = 0;
    ENG_CU(cudaMemcpyAsync(&herr, d_err_, sizeof(int), cudaMemcpyDeviceToHost, st));
    ENG_CU(cudaStreamSynchronize(st));
    if (herr) {
        // A run that gave up may have left an instance's finalize half counted:
        // clear every instance's last-block counter with the error word.
        ENG_CU(cudaMemsetAsync(d_err_, 0, sizeof(int), st));
        for (EngineInstance* in : insts_)
            ENG_CU(cudaMemsetAsync(in->counter, 0, bytes(*in).counter, st));
        ENG_CU(cudaStreamSynchronize(st));
        return BLDM_ERR_TIMEOUT;
    }
    return BLDM_OK;
}

}  // namespace bldm
