// TEST INFRASTRUCTURE ONLY — the CPU oracle for the bld_mult path.
//
// A restatement, in plain C++/OpenMP without Eigen or GSL, of eozd/bnmf-algs'
// multiplicative-update Best Latent Decomposition solver.  Only tests/, the
// smoke check and bench.py's CPU-baseline leg load this library; the product
// (libbldm.so) never links or calls it.
//
// Every function names the reference file:line it restates (paths relative to
// the reference project root).  The reference itself cannot be compiled in this
// image (Eigen3 and GSL are absent), so parity of this restatement is pinned by
// the reference's own known-answer tests (test/bld/bld_mult/test_bld_mult.cpp,
// test/util/test_util.cpp) re-expressed under tests/, and by scipy/mpmath for
// the digamma function.
//
// Storage is row-major like the reference's tensor_t/matrix_t
// (src/defs.hpp:40-52): S(i,j,k) lives at ((i*y)+j)*z+k, X(i,j) at i*y+j.

#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#include <omp.h>

namespace {

// ---------------------------------------------------------------------------
// Digamma.
// ---------------------------------------------------------------------------

// Asymptotic expansion of psi at x >= threshold (Abramowitz & Stegun 6.3.18):
//   psi(x) ~ ln x - 1/(2x) - sum_n B_2n / (2n x^2n)
// truncated after the x^-14 term, evaluated in Horner form in r^2 = 1/x^2.
template <typename R> R psi_series14(R x) {
    const R r = R(1) / x;
    const R r2 = r * r;
    const R tail =
        r2 * (R(1) / R(12) -
              r2 * (R(1) / R(120) -
                    r2 * (R(1) / R(252) -
                          r2 * (R(1) / R(240) -
                                r2 * (R(1) / R(132) -
                                      r2 * (R(691) / R(32760) -
                                            r2 / R(12)))))));
    return std::log(x) - r / R(2) - tail;
}

// util::psi_appr (src/util/util.hpp:440-514): shift the argument with the
// recurrence psi(x) = psi(x + 1) - 1/x until it is >= 6 (the reference's
// branches shift x < 1 by 6, [1,2) by 5, ..., [5,6) by 1), then apply the
// expansion truncated after the x^-14 term (the reference's combined rational
// form at util.hpp:500-511 is the same series).
template <typename R> R psi_appr(R x) {
    R shift = 0;
    if (x < R(6)) {
        const int n = (x < R(1)) ? 6 : 6 - static_cast<int>(std::floor(x));
        for (int m = 0; m < n; ++m) shift += R(1) / (x + R(m));
        x += R(n);
    }
    return psi_series14(x) - shift;
}

// Exact digamma (replaces gsl_sf_psi, used via details::gsl_psi_wrapper,
// src/bld/util_details.hpp:71-73).  Same published method with a larger shift
// threshold (10) and one more series term (3617/(8160 x^16)); the truncation
// error at x >= 10 is below 5e-17.  Defined for x > 0 (every argument on the
// bld_mult path is positive); returns NaN otherwise.
double psi_exact(double x) {
    if (!(x > 0)) return NAN;
    double shift = 0;
    while (x < 10.0) {
        shift += 1.0 / x;
        x += 1.0;
    }
    const double r = 1.0 / x;
    const double r2 = r * r;
    const double tail =
        r2 * (1.0 / 12 -
              r2 * (1.0 / 120 -
                    r2 * (1.0 / 252 -
                          r2 * (1.0 / 240 -
                                r2 * (1.0 / 132 -
                                      r2 * (691.0 / 32760 -
                                            r2 * (1.0 / 12 -
                                                  r2 * (3617.0 / 8160))))))));
    return std::log(x) - 0.5 * r - tail - shift;
}

enum { PSI_EXACT = 0, PSI_APPR = 1, PSI_LEGACY_CUDA = 2 };

template <typename T> T psi_by(int appr, T v) {
    return appr ? psi_appr<T>(v) : static_cast<T>(psi_exact(double(v)));
}

// ---------------------------------------------------------------------------
// Stage functions, src/bld/bld_mult/bld_mult_funcs.hpp.
// ---------------------------------------------------------------------------

// Three axis sums of S (bld_mult.hpp:126-128): S_pjk (y x z) = sum over i,
// S_ipk (x x z) = sum over j, S_ijp (x x y) = sum over k.
template <typename T>
void tensor_sums(const T* S, size_t x, size_t y, size_t z, T* pjk, T* ipk,
                 T* ijp) {
#pragma omp parallel for schedule(static)
    for (long j = 0; j < long(y); ++j) {
        for (size_t k = 0; k < z; ++k) {
            T s = T();
            for (size_t i = 0; i < x; ++i) s += S[(i * y + j) * z + k];
            pjk[j * z + k] = s;
        }
    }
#pragma omp parallel for schedule(static)
    for (long i = 0; i < long(x); ++i) {
        for (size_t k = 0; k < z; ++k) {
            T s = T();
            for (size_t j = 0; j < y; ++j) s += S[(i * y + j) * z + k];
            ipk[i * z + k] = s;
        }
        for (size_t j = 0; j < y; ++j) {
            T s = T();
            for (size_t k = 0; k < z; ++k) s += S[(i * y + j) * z + k];
            ijp[i * y + j] = s;
        }
    }
}

// X_reciprocal (bld_mult_funcs.hpp:87-100): Xr = 1 / (X + eps).
template <typename T>
void x_reciprocal(const T* X, size_t x, size_t y, double eps, T* Xr) {
#pragma omp parallel for schedule(static)
    for (long i = 0; i < long(x); ++i)
        for (size_t j = 0; j < y; ++j)
            Xr[i * y + j] = T(1.0 / (X[i * y + j] + eps));
}

// update_alpha_eph (bld_mult_funcs.hpp:130-141).
template <typename T>
void update_alpha_eph(const T* ipk, const T* alpha, size_t x, size_t z,
                      T* alpha_eph) {
#pragma omp parallel for schedule(static)
    for (long i = 0; i < long(x); ++i)
        for (size_t k = 0; k < z; ++k)
            alpha_eph[i * z + k] = ipk[i * z + k] + alpha[i];
}

// update_beta_eph (bld_mult_funcs.hpp:152-163).
template <typename T>
void update_beta_eph(const T* pjk, const T* beta, size_t y, size_t z,
                     T* beta_eph) {
#pragma omp parallel for schedule(static)
    for (long j = 0; j < long(y); ++j)
        for (size_t k = 0; k < z; ++k)
            beta_eph[j * z + k] = pjk[j * z + k] + beta[k];
}

// update_grad_plus (bld_mult_funcs.hpp:177-192):
//   gp(i,j,k) = psi(beta_eph(j,k)) - psi(S(i,j,k) + 1).
template <typename T>
void update_grad_plus(const T* S, const T* beta_eph, size_t x, size_t y,
                      size_t z, int appr, T* gp) {
#pragma omp parallel for schedule(static)
    for (long i = 0; i < long(x); ++i)
        for (size_t j = 0; j < y; ++j)
            for (size_t k = 0; k < z; ++k) {
                const size_t e = (i * y + j) * z + k;
                gp[e] = psi_by<T>(appr, beta_eph[j * z + k]) -
                        psi_by<T>(appr, S[e] + T(1));
            }
}

// update_grad_minus (bld_mult_funcs.hpp:205-229):
//   gm(i,k) = psi(sum_i' alpha_eph(i',k)) - psi(alpha_eph(i,k)).
template <typename T>
void update_grad_minus(const T* alpha_eph, size_t x, size_t z, int appr,
                       T* gm) {
    std::vector<T> psi_sum(z);
#pragma omp parallel for schedule(static)
    for (long k = 0; k < long(z); ++k) {
        T s = T();
        for (size_t i = 0; i < x; ++i) s += alpha_eph[i * z + k];
        psi_sum[k] = psi_by<T>(appr, s);
    }
#pragma omp parallel for schedule(static)
    for (long i = 0; i < long(x); ++i)
        for (size_t k = 0; k < z; ++k)
            gm[i * z + k] = psi_sum[k] - psi_by<T>(appr, alpha_eph[i * z + k]);
}

// update_nom_mult (bld_mult_funcs.hpp:242-259):
//   nom(i,j) = sum_k S(i,j,k) * Xr(i,j) * gm(i,k).
template <typename T>
void update_nom(const T* Xr, const T* gm, const T* S, size_t x, size_t y,
                size_t z, T* nom) {
#pragma omp parallel for schedule(static)
    for (long i = 0; i < long(x); ++i)
        for (size_t j = 0; j < y; ++j) {
            T s = T();
            for (size_t k = 0; k < z; ++k)
                s += S[(i * y + j) * z + k] * Xr[i * y + j] * gm[i * z + k];
            nom[i * y + j] = s;
        }
}

// update_denom_mult (bld_mult_funcs.hpp:272-290):
//   denom(i,j) = sum_k S(i,j,k) * Xr(i,j) * gp(i,j,k).
template <typename T>
void update_denom(const T* Xr, const T* gp, const T* S, size_t x, size_t y,
                  size_t z, T* denom) {
#pragma omp parallel for schedule(static)
    for (long i = 0; i < long(x); ++i)
        for (size_t j = 0; j < y; ++j) {
            T s = T();
            for (size_t k = 0; k < z; ++k) {
                const size_t e = (i * y + j) * z + k;
                s += S[e] * Xr[i * y + j] * gp[e];
            }
            denom[i * y + j] = s;
        }
}

// update_S (bld_mult_funcs.hpp:307-327):
//   S(i,j,k) *= (gp + nom(i,j)) * X(i,j)/(S_ijp(i,j)+eps) / (gm(i,k)+denom(i,j)+eps)
// with S_ijp taken from before the update.
template <typename T>
void update_S(const T* X, const T* nom, const T* denom, const T* gm,
              const T* gp, const T* ijp, size_t x, size_t y, size_t z,
              double eps, T* S) {
#pragma omp parallel for schedule(static)
    for (long i = 0; i < long(x); ++i)
        for (size_t j = 0; j < y; ++j) {
            const T x_over_s = T(X[i * y + j] / (ijp[i * y + j] + eps));
            for (size_t k = 0; k < z; ++k) {
                const size_t e = (i * y + j) * z + k;
                S[e] *= T((gp[e] + nom[i * y + j]) * x_over_s /
                          (gm[i * z + k] + denom[i * y + j] + eps));
            }
        }
}

// The bld_mult driver (src/bld/bld_mult/bld_mult.hpp:82-150), with init_S
// replaced by an injected S0 (the reference's init_S draws from GSL's taus
// generator with its default seed, per OpenMP thread, so it is not
// reproducible across thread counts).  psi_mode: PSI_APPR uses psi_appr
// everywhere; PSI_EXACT uses the exact digamma everywhere (bld_mult with
// use_psi_appr=false); PSI_LEGACY_CUDA reproduces bld_mult_cuda with
// use_psi_appr=false, whose grad_plus always uses psi_appr on the device
// (bld_mult.hpp:284-286 and cuda_src/bld_mult/bld_mult_cuda_kernels.cu:116)
// while grad_minus uses the exact digamma on the host.
template <typename T>
void bld_mult(const T* X, size_t x, size_t y, size_t z, const T* alpha,
              const T* beta, size_t max_iter, int psi_mode, double eps,
              const T* S0, T* S) {
    const size_t n = x * y * z;
    std::memcpy(S, S0, n * sizeof(T));
    std::vector<T> Xr(x * y), gp(n), nom(x * y), denom(x * y), gm(x * z),
        alpha_eph(x * z), beta_eph(y * z), pjk(y * z), ipk(x * z), ijp(x * y);
    x_reciprocal(X, x, y, eps, Xr.data());
    const int appr_plus = (psi_mode != PSI_EXACT) ? 1 : 0;
    const int appr_minus = (psi_mode == PSI_APPR) ? 1 : 0;
    for (size_t eph = 0; eph < max_iter; ++eph) {
        tensor_sums(S, x, y, z, pjk.data(), ipk.data(), ijp.data());
        update_alpha_eph(ipk.data(), alpha, x, z, alpha_eph.data());
        update_beta_eph(pjk.data(), beta, y, z, beta_eph.data());
        update_grad_plus(S, beta_eph.data(), x, y, z, appr_plus, gp.data());
        update_grad_minus(alpha_eph.data(), x, z, appr_minus, gm.data());
        update_nom(Xr.data(), gm.data(), S, x, y, z, nom.data());
        update_denom(Xr.data(), gp.data(), S, x, y, z, denom.data());
        update_S(X, nom.data(), denom.data(), gm.data(), gp.data(), ijp.data(),
                 x, y, z, eps, S);
    }
}

// ---------------------------------------------------------------------------
// log_marginal_S, src/alloc_model/alloc_model_funcs.hpp:33-194,573-586.
// std::lgamma replaces gsl_sf_lngamma.  All arithmetic in double.
// ---------------------------------------------------------------------------
template <typename T>
double log_marginal_S(const T* S, size_t x, size_t y, size_t z,
                      const double* alpha, const double* beta, double a,
                      double b) {
    // first term (alloc_model_funcs.hpp:33-77)
    double alpha_sum = 0, lg_alpha_sum = 0;
    for (size_t i = 0; i < x; ++i) {
        alpha_sum += alpha[i];
        lg_alpha_sum += std::lgamma(alpha[i]);
    }
    double first = 0;
#pragma omp parallel for reduction(+ : first)
    for (long k = 0; k < long(z); ++k) {
        double tot = 0;
        double acc = 0;
        for (size_t i = 0; i < x; ++i) {
            double row = alpha[i];
            for (size_t j = 0; j < y; ++j) row += double(S[(i * y + j) * z + k]);
            tot += row;
            acc += std::lgamma(row);
        }
        first += acc - std::lgamma(tot);
    }
    first += (std::lgamma(alpha_sum) - lg_alpha_sum) * double(z);

    // second term (alloc_model_funcs.hpp:90-132)
    double beta_sum = 0, lg_beta_sum = 0;
    for (size_t k = 0; k < z; ++k) {
        beta_sum += beta[k];
        lg_beta_sum += std::lgamma(beta[k]);
    }
    double second = 0;
#pragma omp parallel for reduction(+ : second)
    for (long j = 0; j < long(y); ++j) {
        double tot = 0, acc = 0;
        for (size_t k = 0; k < z; ++k) {
            double col = beta[k];
            for (size_t i = 0; i < x; ++i) col += double(S[(i * y + j) * z + k]);
            tot += col;
            acc += std::lgamma(col);
        }
        second += acc - std::lgamma(tot);
    }
    second += (std::lgamma(beta_sum) - lg_beta_sum) * double(y);

    // third term (alloc_model_funcs.hpp:145-169), rate parameterisation of b
    double third = 0;
    const double log_b1 = std::log(b + 1);
#pragma omp parallel for reduction(+ : third)
    for (long j = 0; j < long(y); ++j) {
        double s = a;
        for (size_t i = 0; i < x; ++i)
            for (size_t k = 0; k < z; ++k) s += double(S[(i * y + j) * z + k]);
        third += std::lgamma(s) - s * log_b1;
    }
    third += (-std::lgamma(a) + a * std::log(b)) * double(y);

    // fourth term (alloc_model_funcs.hpp:179-194)
    double fourth = 0;
    const long n = long(x * y * z);
#pragma omp parallel for reduction(+ : fourth)
    for (long e = 0; e < n; ++e) fourth += std::lgamma(double(S[e]) + 1);

    return first + second + third - fourth;
}

// util::sparseness (src/util/util.hpp:270-298): Hoyer sparseness.
template <typename T> double sparseness(const T* S, size_t x, size_t y, size_t z) {
    double sum = 0, sq = 0;
    const long n = long(x * y * z);
#pragma omp parallel for reduction(+ : sum, sq)
    for (long e = 0; e < n; ++e) {
        sum += double(S[e]);
        sq += double(S[e]) * double(S[e]);
    }
    if (sq < 2.220446049250313e-16) return 1.79769313486231570e+308;
    const double frob = std::sqrt(sq);
    const double axis = std::sqrt(double(n));
    return (axis - sum / frob) / (axis - 1);
}

// bld_fact (src/bld/bld_fact.hpp:36-80): S -> (W x*z, H z*y, L y).
template <typename T>
void bld_fact(const T* S, size_t x, size_t y, size_t z, const double* alpha,
              const double* beta, double a, double b, double eps, T* W, T* H,
              T* L) {
    std::vector<T> pjk(y * z), ipk(x * z), ijp(x * y);
    tensor_sums(S, x, y, z, pjk.data(), ipk.data(), ijp.data());
    for (size_t i = 0; i < x; ++i)
        for (size_t k = 0; k < z; ++k) W[i * z + k] = T(alpha[i] + ipk[i * z + k] - 1);
    for (size_t k = 0; k < z; ++k)
        for (size_t j = 0; j < y; ++j) H[k * y + j] = T(beta[k] + pjk[j * z + k] - 1);
    for (size_t j = 0; j < y; ++j) {
        T pjp = T();
        for (size_t k = 0; k < z; ++k) pjp += pjk[j * z + k];
        L[j] = T((a + pjp - 1) / (b + 1 + eps));
    }
    for (size_t k = 0; k < z; ++k) {
        T cs = T();
        for (size_t i = 0; i < x; ++i) cs += W[i * z + k];
        cs = T(cs + eps);
        for (size_t i = 0; i < x; ++i) W[i * z + k] /= cs;
    }
    for (size_t j = 0; j < y; ++j) {
        T cs = T();
        for (size_t k = 0; k < z; ++k) cs += H[k * y + j];
        cs = T(cs + eps);
        for (size_t k = 0; k < z; ++k) H[k * y + j] /= cs;
    }
}

// ---------------------------------------------------------------------------
// Seeded initial S.  The reference's init_S (bld_mult_funcs.hpp:36-74) sets
// S(i,j,:) = X(i,j) * Dirichlet(1_z); this restatement draws the Dirichlet
// sample as normalised Exp(1) variates from a counter-based generator
// (SplitMix64 finaliser of seed, fiber index and k), so that the device
// implementation can produce the same tensor independent of thread layout.
// ---------------------------------------------------------------------------
inline uint64_t splitmix64(uint64_t v) {
    v += 0x9E3779B97F4A7C15ull;
    v = (v ^ (v >> 30)) * 0xBF58476D1CE4E5B9ull;
    v = (v ^ (v >> 27)) * 0x94D049BB133111EBull;
    return v ^ (v >> 31);
}
inline double unit_open(uint64_t h) {  // (0,1), never 0
    return (double(h >> 11) + 0.5) * (1.0 / 9007199254740992.0);
}
inline double exp1_variate(uint64_t seed, uint64_t fiber, uint64_t k) {
    const uint64_t h = splitmix64(splitmix64(seed ^ 0x5DEECE66Dull) ^
                                  splitmix64(fiber * 0x100000001B3ull + k));
    return -std::log(unit_open(h));
}

template <typename T>
void init_S(const T* X, size_t x, size_t y, size_t z, uint64_t seed, T* S) {
#pragma omp parallel for schedule(static)
    for (long f = 0; f < long(x * y); ++f) {
        double tot = 0;
        for (size_t k = 0; k < z; ++k) tot += exp1_variate(seed, f, k);
        for (size_t k = 0; k < z; ++k)
            S[f * z + k] = T(double(X[f]) * (exp1_variate(seed, f, k) / tot));
    }
}

}  // namespace

extern "C" {

int oracle_set_threads(int n) {
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
}

double oracle_psi_appr_f64(double v) { return psi_appr<double>(v); }
float oracle_psi_appr_f32(float v) { return psi_appr<float>(v); }
double oracle_psi_exact(double v) { return psi_exact(v); }

void oracle_psi_array(const double* in, size_t n, int mode, double* out) {
#pragma omp parallel for schedule(static)
    for (long e = 0; e < long(n); ++e)
        out[e] = mode ? psi_appr<double>(in[e]) : psi_exact(in[e]);
}

void oracle_tensor_sums_f64(const double* S, size_t x, size_t y, size_t z,
                            double* pjk, double* ipk, double* ijp) {
    tensor_sums(S, x, y, z, pjk, ipk, ijp);
}
void oracle_tensor_sums_f32(const float* S, size_t x, size_t y, size_t z,
                            float* pjk, float* ipk, float* ijp) {
    tensor_sums(S, x, y, z, pjk, ipk, ijp);
}
void oracle_x_reciprocal_f64(const double* X, size_t x, size_t y, double eps,
                             double* Xr) {
    x_reciprocal(X, x, y, eps, Xr);
}
void oracle_update_alpha_eph_f64(const double* ipk, const double* alpha,
                                 size_t x, size_t z, double* out) {
    update_alpha_eph(ipk, alpha, x, z, out);
}
void oracle_update_beta_eph_f64(const double* pjk, const double* beta, size_t y,
                                size_t z, double* out) {
    update_beta_eph(pjk, beta, y, z, out);
}
void oracle_update_grad_plus_f64(const double* S, const double* beta_eph,
                                 size_t x, size_t y, size_t z, int appr,
                                 double* gp) {
    update_grad_plus(S, beta_eph, x, y, z, appr, gp);
}
void oracle_update_grad_minus_f64(const double* alpha_eph, size_t x, size_t z,
                                  int appr, double* gm) {
    update_grad_minus(alpha_eph, x, z, appr, gm);
}
void oracle_update_nom_f64(const double* Xr, const double* gm, const double* S,
                           size_t x, size_t y, size_t z, double* nom) {
    update_nom(Xr, gm, S, x, y, z, nom);
}
void oracle_update_denom_f64(const double* Xr, const double* gp,
                             const double* S, size_t x, size_t y, size_t z,
                             double* denom) {
    update_denom(Xr, gp, S, x, y, z, denom);
}
void oracle_update_S_f64(const double* X, const double* nom,
                         const double* denom, const double* gm,
                         const double* gp, const double* ijp, size_t x,
                         size_t y, size_t z, double eps, double* S) {
    update_S(X, nom, denom, gm, gp, ijp, x, y, z, eps, S);
}

void oracle_bld_mult_f64(const double* X, size_t x, size_t y, size_t z,
                         const double* alpha, const double* beta,
                         size_t max_iter, int psi_mode, double eps,
                         const double* S0, double* S) {
    bld_mult<double>(X, x, y, z, alpha, beta, max_iter, psi_mode, eps, S0, S);
}
void oracle_bld_mult_f32(const float* X, size_t x, size_t y, size_t z,
                         const float* alpha, const float* beta,
                         size_t max_iter, int psi_mode, double eps,
                         const float* S0, float* S) {
    bld_mult<float>(X, x, y, z, alpha, beta, max_iter, psi_mode, eps, S0, S);
}

double oracle_log_marginal_S_f64(const double* S, size_t x, size_t y, size_t z,
                                 const double* alpha, const double* beta,
                                 double a, double b) {
    return log_marginal_S(S, x, y, z, alpha, beta, a, b);
}
double oracle_log_marginal_S_f32(const float* S, size_t x, size_t y, size_t z,
                                 const double* alpha, const double* beta,
                                 double a, double b) {
    return log_marginal_S(S, x, y, z, alpha, beta, a, b);
}
double oracle_sparseness_f64(const double* S, size_t x, size_t y, size_t z) {
    return sparseness(S, x, y, z);
}
void oracle_bld_fact_f64(const double* S, size_t x, size_t y, size_t z,
                         const double* alpha, const double* beta, double a,
                         double b, double eps, double* W, double* H,
                         double* L) {
    bld_fact(S, x, y, z, alpha, beta, a, b, eps, W, H, L);
}
void oracle_init_S_f64(const double* X, size_t x, size_t y, size_t z,
                       uint64_t seed, double* S) {
    init_S(X, x, y, z, seed, S);
}

}  // extern "C"
