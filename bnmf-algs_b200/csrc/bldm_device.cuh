// Device building blocks shared by the bld_mult kernels: digamma in FP64 and
// FP32, warp reductions, and thin wrappers over the sm_100a bulk-copy (TMA
// engine, non-tensor form) and mbarrier PTX used to stage S slabs in shared
// memory.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace bldm {

enum PsiMode : int { PSI_EXACT = 0, PSI_APPR = 1, PSI_LEGACY_CUDA = 2 };

// Error bits written into the device error word.
enum DevErr : int { DEV_ERR_WAIT_TIMEOUT = 1, DEV_ERR_BAD_LAUNCH = 2 };

// A bounded wait gives up after this many nanoseconds of %globaltimer.
constexpr unsigned long long kWaitLimitNs = 1000000000ull;

// ---------------------------------------------------------------------------
// Digamma.
//
// psi_appr restates util::psi_appr (src/util/util.hpp:440-514): unit shifts by
// psi(x) = psi(x + 1) - 1/x until the argument is >= 6 (x < 1 shifts by 6,
// [n, n+1) by 6 - n), then the asymptotic series
//   ln x - 1/(2x) - 1/(12x^2) + 1/(120x^4) - 1/(252x^6) + 1/(240x^8)
//        - 1/(132x^10) + 691/(32760x^12) - 1/(12x^14).
// The exact digamma (the reference calls gsl_sf_psi) is the same published
// method (Abramowitz & Stegun 6.3.5 and 6.3.18) with threshold 10 and one more
// term, 3617/(8160x^16); its truncation error is below 5e-17.
//
// Both are branch-free: the shift sum sum_m 1/(x+m) is accumulated as one
// fraction N/D and a single division 1/(x' D) yields both 1/x' and N/D.
// ---------------------------------------------------------------------------
template <int THRESH, bool EXTRA_TERM>
__device__ __forceinline__ double psi_f64(double x) {
    double n = 0.0;
    if (x < double(THRESH)) {
        n = double(THRESH) - floor(x);
        n = n > double(THRESH) ? double(THRESH) : n;  // x < 1 shifts by THRESH
    }
    double num = 0.0, den = 1.0;
#pragma unroll
    for (int m = 0; m < THRESH; ++m) {
        const bool act = double(m) < n;
        const double f = act ? x + double(m) : 1.0;
        num = act ? fma(num, f, den) : num;
        den = den * f;
    }
    const double xs = x + n;
    const double inv = 1.0 / (xs * den);
    const double r = den * inv;       // 1 / xs
    const double shift = num * xs * inv;  // sum_m 1/(x+m)
    const double r2 = r * r;
    double t;
    if (EXTRA_TERM) {
        t = fma(r2, -3617.0 / 8160.0, 1.0 / 12.0);
        t = fma(r2, -t, 691.0 / 32760.0);
    } else {
        t = fma(r2, -1.0 / 12.0, 691.0 / 32760.0);
    }
    t = fma(r2, -t, 1.0 / 132.0);
    t = fma(r2, -t, 1.0 / 240.0);
    t = fma(r2, -t, 1.0 / 252.0);
    t = fma(r2, -t, 1.0 / 120.0);
    t = fma(r2, -t, 1.0 / 12.0);
    return log(xs) - 0.5 * r - r2 * t - shift;
}

__device__ __forceinline__ double psi_appr_f64(double x) { return psi_f64<6, false>(x); }
__device__ __forceinline__ double psi_exact_f64(double x) {
    return x > 0.0 ? psi_f64<10, true>(x) : __longlong_as_double(0x7ff8000000000000ll);
}

// FP32 digamma for FP32 storage: the same shift rule (threshold 6) and the
// series truncated after the x^-8 term, whose omitted remainder at x >= 6 is
// below 2e-10, far under FP32 resolution.  Written in 1/x so that it does not
// overflow for large counts.
__device__ __forceinline__ float psi_f32(float x) {
    float n = 0.f;
    if (x < 6.f) {
        n = 6.f - floorf(x);
        n = n > 6.f ? 6.f : n;
    }
    float num = 0.f, den = 1.f;
#pragma unroll
    for (int m = 0; m < 6; ++m) {
        const bool act = float(m) < n;
        const float f = act ? x + float(m) : 1.f;
        num = act ? fmaf(num, f, den) : num;
        den = den * f;
    }
    const float xs = x + n;
    const float inv = 1.f / (xs * den);
    const float r = den * inv;
    const float shift = n > 0.f ? num * xs * inv : 0.f;  // no 0 * inf at x = inf
    const float r2 = r * r;
    float t = fmaf(r2, -1.f / 240.f, 1.f / 252.f);
    t = fmaf(r2, -t, 1.f / 120.f);
    t = fmaf(r2, -t, 1.f / 12.f);
    return logf(xs) - 0.5f * r - r2 * t - shift;
}

template <typename T> struct Psi;
template <> struct Psi<double> {
    __device__ __forceinline__ static double appr(double v) { return psi_appr_f64(v); }
    __device__ __forceinline__ static double exact(double v) { return psi_exact_f64(v); }
};
template <> struct Psi<float> {
    __device__ __forceinline__ static float appr(float v) { return psi_f32(v); }
    __device__ __forceinline__ static float exact(float v) { return psi_f32(v); }
};

__device__ __forceinline__ double psi_mode_f64(double v, bool appr) {
    return appr ? psi_appr_f64(v) : psi_exact_f64(v);
}

// ---------------------------------------------------------------------------
// Throughput versions for the fused sweep, where FP64 issue slots bound the
// kernel.  Same mathematical functions as above; only the evaluation differs.
// ---------------------------------------------------------------------------

// 1/d by two Newton-Raphson steps y <- y (2 - d y) from the hardware
// reciprocal approximation (each step squares the relative error, so a seed
// good to 2^-16 is already below double rounding after two steps).  Normal
// finite d only (the seed flushes subnormals).
__device__ __forceinline__ double rcp_nr(double d) {
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(d));
    double e = fma(-d, y, 1.0);
    y = fma(y, e, y);
    e = fma(-d, y, 1.0);
    return fma(y, e, y);
}

// Natural logarithm by the table-driven method of P. T. P. Tang ("Table-driven
// implementation of the logarithm function in IEEE floating-point
// arithmetic", ACM TOMS 16(4), 1990): x = 2^e m, m in [1,2); R_j = 1/c_j with
// c_j = 1 + j/128 the nearest of 129 breakpoints; r = m R_j - 1 (one fused
// rounding), |r| <= 2^-8; ln x = e ln2 + ln(1/R_j) + log1p(r) with log1p as
// its Taylor series to r^6 (remainder below 2^-59).  ln2 is split in a
// 32-bit-exact high part and a low part so that e*ln2_hi is exact.
constexpr int kLogTabN = 129;
constexpr double kLn2Hi = 6.93147180369123816490e-01;  // ln2 to 32 significant bits
constexpr double kLn2Lo = 1.90821492927058770002e-10;  // ln2 - kLn2Hi

// Fills tab[j] = {ln(1/R_j), R_j}; call once per CTA before use.
__device__ __forceinline__ void log_tab_init(double2* tab, int tid, int nthreads) {
    for (int j = tid; j < kLogTabN; j += nthreads) {
        const double R = 1.0 / (1.0 + double(j) * (1.0 / 128.0));
        tab[j] = make_double2(-log(R), R);
    }
}

__device__ __forceinline__ double log_tab(double x, const double2* tab) {
    if (!(x >= 2.2250738585072014e-308 && x <= 1.7976931348623157e308)) return log(x);
    const long long b = __double_as_longlong(x);
    const int ex = int(b >> 52) - 1023;
    const long long mb = (b & 0x000FFFFFFFFFFFFFll) | 0x3FF0000000000000ll;
    const double m = __longlong_as_double(mb);
    const int j = (int((mb >> 44) & 0xFF) + 1) >> 1;  // nearest breakpoint, 0..128
    const double2 t = tab[j];
    const double r = fma(m, t.y, -1.0);
    double q = fma(r, -1.0 / 6.0, 1.0 / 5.0);
    q = fma(q, r, -1.0 / 4.0);
    q = fma(q, r, 1.0 / 3.0);
    q = fma(q, r, -1.0 / 2.0);
    const double l1 = fma(q, r * r, r);
    const double de = double(ex);
    return fma(de, kLn2Hi, t.x) + fma(de, kLn2Lo, l1);
}

// Reciprocal used by the update and the sweep's digamma.
template <typename T> struct Rcp;
template <> struct Rcp<double> {
    __device__ __forceinline__ static double of(double d) {
        const double a = fabs(d);
        return (a >= 2.2250738585072014e-308 && a <= 4.49423283715578976932e307) ? rcp_nr(d)
                                                                                 : 1.0 / d;
    }
};
// FP32: the hardware approximation refined by one Newton-Raphson step.  Where
// the step is undefined (d = 0 or a subnormal d, whose seed is inf; d = inf,
// whose seed is 0) the refinement gives NaN and the seed itself is returned:
// inf as 1/d overflows, 0 for an infinite divisor.  A reciprocal in the
// subnormal range (|d| >= 2^126) flushes to 0.
template <> struct Rcp<float> {
    __device__ __forceinline__ static float of(float d) {
        float y;
        asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(d));
        const float r = fmaf(y, fmaf(-d, y, 1.0f), y);
        return r == r ? r : y;
    }
};

// psi(arg) for the NE elements of one pass, every lane of the warp together.
template <int NE>
__device__ __forceinline__ void psi_appr_batch(const double (&x)[NE], double (&out)[NE],
                                               const double2* ltab) {
    int n[NE];
    double num[NE], den[NE];
    bool six = false;
#pragma unroll
    for (int e = 0; e < NE; ++e) {
        n[e] = (x[e] < 1.0) ? 6 : ((x[e] < 6.0) ? 6 - __double2int_rz(x[e]) : 0);
        six |= n[e] == 6;
        num[e] = 0.0;
        den[e] = 1.0;
    }
    // Arguments >= 1 need at most five unit shifts; a sixth (argument < 1,
    // i.e. S < 0) is taken only when some lane of the warp needs it.
    const int steps = __any_sync(0xffffffffu, six) ? 6 : 5;
#pragma unroll
    for (int m = 0; m < 6; ++m) {
        if (m == 5 && steps == 5) break;
#pragma unroll
        for (int e = 0; e < NE; ++e) {
            const bool act = m < n[e];
            const double f = act ? x[e] + double(m) : 1.0;
            num[e] = act ? fma(num[e], f, den[e]) : num[e];
            den[e] *= f;
        }
    }
#pragma unroll
    for (int e = 0; e < NE; ++e) {
        const double xs = x[e] + double(n[e]);
        const double inv = Rcp<double>::of(xs * den[e]);
        const double r = den[e] * inv;
        const double shift = num[e] * xs * inv;
        const double r2 = r * r;
        double t = fma(r2, -1.0 / 12.0, 691.0 / 32760.0);
        t = fma(r2, -t, 1.0 / 132.0);
        t = fma(r2, -t, 1.0 / 240.0);
        t = fma(r2, -t, 1.0 / 252.0);
        t = fma(r2, -t, 1.0 / 120.0);
        t = fma(r2, -t, 1.0 / 12.0);
        out[e] = log_tab(xs, ltab) - 0.5 * r - r2 * t - shift;
    }
}

template <typename T, bool APPR> struct PsiPass;
template <> struct PsiPass<double, true> {
    template <int NE>
    __device__ __forceinline__ static void run(const double (&x)[NE], double (&out)[NE],
                                               const double2* ltab) {
        psi_appr_batch<NE>(x, out, ltab);
    }
};
template <> struct PsiPass<double, false> {
    template <int NE>
    __device__ __forceinline__ static void run(const double (&x)[NE], double (&out)[NE],
                                               const double2*) {
#pragma unroll
        for (int e = 0; e < NE; ++e) out[e] = psi_exact_f64(x[e]);
    }
};
// FP32 digamma for the sweep.  Arguments below 4 take exactly three steps of
// the recurrence psi(v) = psi(v + 3) - (1/v + 1/(v+1) + 1/(v+2)), the three
// reciprocals summed as one rational function (3v^2 + 6v + 2) / (v (v+1) (v+2));
// at v + 3 >= 4 (and at v >= 4 unshifted) the asymptotic series
// ln x - 1/(2x) - sum_k B_2k / (2k x^2k), truncated after the x^-10 term,
// leaves a remainder below 1.3e-9, under FP32 resolution.  One reciprocal of
// x q serves both 1/x and the shift's division: the hardware approximation
// alone (about one ulp; a Newton step would not show beside the logarithm's
// error, and FP32 S computed with it is as unbiased against FP64 as with the
// refined reciprocal).  The logarithm is the hardware base-2 one (relative
// error about 2^-21, at the resolution of FP32 S).  No per-step selects: the
// shift is a fixed polynomial evaluation.
template <int NE>
__device__ __forceinline__ void psi_f32_batch(const float (&x)[NE], float (&out)[NE]) {
#pragma unroll
    for (int e = 0; e < NE; ++e) {
        const float v = x[e];
        const bool lo = v < 4.0f;
        const float q = lo ? fmaf(v + 3.0f, v, 2.0f) * v : 1.0f;   // v (v+1) (v+2)
        const float p = lo ? fmaf(fmaf(3.0f, v, 6.0f), v, 2.0f) : 0.0f;
        const float xs = lo ? v + 3.0f : v;
        float inv;
        asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(inv) : "f"(xs * q));
        const float r = q * inv;              // 1 / xs
        const float shift = lo ? (p * xs) * inv : 0.0f;   // p / q (no 0 * inf at v = inf)
        const float r2 = r * r;
        float t = fmaf(r2, -1.f / 132.f, 1.f / 240.f);
        t = fmaf(r2, -t, 1.f / 252.f);
        t = fmaf(r2, -t, 1.f / 120.f);
        t = fmaf(r2, -t, 1.f / 12.f);
        out[e] = __logf(xs) - 0.5f * r - r2 * t - shift;
    }
}

template <bool APPR> struct PsiPass<float, APPR> {
    template <int NE>
    __device__ __forceinline__ static void run(const float (&x)[NE], float (&out)[NE],
                                               const double2*) {
        psi_f32_batch<NE>(x, out);
    }
};


// ---------------------------------------------------------------------------
// Programmatic dependent launch: a kernel launched with programmatic stream
// serialisation may start while the previous kernel of the stream finishes;
// it waits here before touching that kernel's results.  launch_dependents lets
// the next kernel start its own preamble.  Both are no-ops otherwise.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void grid_dep_wait() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
}
__device__ __forceinline__ void grid_dep_launch() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// ---------------------------------------------------------------------------
// Timers, bounded waits, bulk copies.
// ---------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
                 : "memory");
}

__device__ __forceinline__ void mbar_fence_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Wait for the phase with the given parity to complete; false after
// kWaitLimitNs without completion.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
    if (mbar_try_wait(bar, parity)) return true;
    const unsigned long long t0 = global_ns();
    while (true) {
        if (mbar_try_wait(bar, parity)) return true;
        if (global_ns() - t0 > kWaitLimitNs) return false;
    }
}

// Invalidates an mbarrier whose phases have all completed, so that its shared
// memory can hold a new mbarrier (a persistent CTA re-initialises its ring for
// every tile).
__device__ __forceinline__ void mbar_inval(uint64_t* bar) {
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_addr(bar)) : "memory");
}

// Acquire load of a counter written by other CTAs (gpu scope).
__device__ __forceinline__ unsigned ld_acquire_gpu(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Orders this thread's generic-proxy accesses (and what they synchronised
// with) before its later bulk copies (async proxy), and the reverse.
__device__ __forceinline__ void fence_proxy_async_global() {
    asm volatile("fence.proxy.async.global;" ::: "memory");
}

// Waits until *ctr >= target: false after limit_ns of %globaltimer or when
// *abort is set.  One thread calls it.
__device__ __forceinline__ bool wait_counter_bounded(const unsigned* ctr, unsigned target,
                                                     const unsigned* abort,
                                                     unsigned long long limit_ns) {
    if (ld_acquire_gpu(ctr) >= target) return true;
    const unsigned long long t0 = global_ns();
    while (true) {
        if (ld_acquire_gpu(ctr) >= target) return true;
        if (ld_acquire_gpu(abort) != 0u) return false;
        if (global_ns() - t0 > limit_ns) return false;
        __nanosleep(64);
    }
}

__device__ __forceinline__ uint64_t policy_evict_first() {
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}

__device__ __forceinline__ uint64_t policy_evict_last() {
    uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
    return p;
}

// Global -> shared bulk copy (no tensor map, no multicast), completing on the
// mbarrier's transaction count.  dst/src 16-byte aligned, bytes % 16 == 0.
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes,
                                         uint64_t* bar, uint64_t policy) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint"
        " [%0], [%1], %2, [%3], %4;" ::"r"(smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar)), "l"(policy)
        : "memory");
}

// ---------------------------------------------------------------------------
// Warp reductions over aligned lane groups of width W (power of two).
// ---------------------------------------------------------------------------
template <int W, typename V> __device__ __forceinline__ V group_sum(V v) {
#pragma unroll
    for (int o = W / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Sum across lanes that share (lane % LPF): offsets LPF, 2 LPF, ..., 16.
template <int LPF, typename V> __device__ __forceinline__ V cross_group_sum(V v) {
#pragma unroll
    for (int o = LPF; o < 32; o <<= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Kahan-compensated FP32 accumulator (sum s, running compensation c).
struct KahanF {
    float s, c;
    __device__ __forceinline__ void init() { s = 0.f; c = 0.f; }
    __device__ __forceinline__ void add(float v) {
        const float yv = v - c;
        const float t = s + yv;
        c = (t - s) - yv;
        s = t;
    }
    __device__ __forceinline__ double value() const { return double(s) - double(c); }
};

// Accumulator selection: FP64 storage accumulates in double, FP32 storage in
// Kahan-compensated float pairs.
template <typename T> struct Acc;
template <> struct Acc<double> {
    double s;
    __device__ __forceinline__ void init() { s = 0.0; }
    __device__ __forceinline__ void add(double v) { s += v; }
    __device__ __forceinline__ double value() const { return s; }
};
template <> struct Acc<float> {
    KahanF k;
    __device__ __forceinline__ void init() { k.init(); }
    __device__ __forceinline__ void add(float v) { k.add(v); }
    __device__ __forceinline__ double value() const { return k.value(); }
};

}  // namespace bldm
