// Header-only C++14 host side of the B200-native bld_mult solver.
//
// A drop-in for eozd/bnmf-algs' bld::bld_mult_cuda and bld::bld_mult
// (src/bld/bld_mult/bld_mult.hpp:82-86, :225-229): same namespace, template
// parameters, arguments and defaults, and the same error contract (argument
// errors throw std::invalid_argument like BNMF_ASSERT in test builds,
// src/defs.hpp:12-20).  The work runs on the GPU through libbldm.so's C ABI
// (include/bldm.h); link with -lbldm.
//
// Types: with BLDM_USE_REFERENCE_TYPES defined, the reference's own headers
// (defs.hpp with the Eigen row-major matrix_t/tensor_t, and
// alloc_model/alloc_model_params.hpp) provide bnmf_algs::matrix_t, tensor_t
// and alloc_model::Params, and this header only adds the solver templates;
// include it instead of the reference's bld_mult.hpp.  Without it, the header
// defines minimal Eigen-free row-major containers with the members the
// reference's bld_mult path and its tests use.
#pragma once

#include <array>
#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <tuple>
#include <type_traits>
#include <vector>

#include "bldm.h"

#ifdef BLDM_USE_REFERENCE_TYPES
#include "alloc_model/alloc_model_params.hpp"
#include "defs.hpp"
#else
namespace bnmf_algs {

template <size_t N> using shape = std::array<size_t, N>;

// Row-major dense matrix (the reference's matrix_t is an Eigen RowMajor
// matrix, src/defs.hpp:40-41).
template <typename Scalar> class matrix_t {
  public:
    matrix_t() = default;
    matrix_t(size_t rows, size_t cols) : r_(rows), c_(cols), d_(rows * cols) {}
    static matrix_t Constant(size_t rows, size_t cols, Scalar v) {
        matrix_t m(rows, cols);
        for (auto& e : m.d_) e = v;
        return m;
    }
    static matrix_t Zero(size_t rows, size_t cols) { return Constant(rows, cols, Scalar(0)); }
    long rows() const { return long(r_); }
    long cols() const { return long(c_); }
    Scalar& operator()(size_t i, size_t j) { return d_[i * c_ + j]; }
    const Scalar& operator()(size_t i, size_t j) const { return d_[i * c_ + j]; }
    Scalar* data() { return d_.data(); }
    const Scalar* data() const { return d_.data(); }

  private:
    size_t r_ = 0, c_ = 0;
    std::vector<Scalar> d_;
};

// Row-major dense tensor (the reference's tensor_t is an Eigen RowMajor
// Tensor, src/defs.hpp:52).
template <typename Scalar, size_t N> class tensor_t {
  public:
    tensor_t() { dims_.fill(0); }
    template <typename... I> explicit tensor_t(I... dims) : dims_{{size_t(dims)...}} {
        static_assert(sizeof...(I) == N, "tensor_t: wrong number of dimensions");
        size_t n = 1;
        for (size_t d : dims_) n *= d;
        d_.assign(n, Scalar(0));
    }
    long dimension(size_t i) const { return long(dims_[i]); }
    long size() const { return long(d_.size()); }
    Scalar* data() { return d_.data(); }
    const Scalar* data() const { return d_.data(); }
    template <typename... I> Scalar& operator()(I... idx) { return d_[offset({{size_t(idx)...}})]; }
    template <typename... I> const Scalar& operator()(I... idx) const {
        return d_[offset({{size_t(idx)...}})];
    }

  private:
    size_t offset(const std::array<size_t, N>& ix) const {
        size_t o = 0;
        for (size_t a = 0; a < N; ++a) o = o * dims_[a] + ix[a];
        return o;
    }
    std::array<size_t, N> dims_;
    std::vector<Scalar> d_;
};

// Row vector (the reference's vector_t is an Eigen row vector, src/defs.hpp:27-32).
template <typename Scalar> class vector_t {
  public:
    vector_t() = default;
    explicit vector_t(size_t n) : d_(n) {}
    long size() const { return long(d_.size()); }
    long cols() const { return long(d_.size()); }
    Scalar& operator()(size_t i) { return d_[i]; }
    const Scalar& operator()(size_t i) const { return d_[i]; }
    Scalar* data() { return d_.data(); }
    const Scalar* data() const { return d_.data(); }

  private:
    std::vector<Scalar> d_;
};

namespace alloc_model {
// alloc_model::Params (src/alloc_model/alloc_model_params.hpp:25-84).
template <typename Scalar> struct Params {
    Scalar a;
    Scalar b;
    std::vector<Scalar> alpha;
    std::vector<Scalar> beta;
    Params(Scalar a, Scalar b, const std::vector<Scalar>& alpha, const std::vector<Scalar>& beta)
        : a(a), b(b), alpha(alpha), beta(beta) {}
    explicit Params(const shape<3>& tensor_shape)
        : a(static_cast<Scalar>(1)), b(static_cast<Scalar>(10)),
          alpha(tensor_shape[0], static_cast<Scalar>(1)),
          beta(tensor_shape[2], static_cast<Scalar>(1)) {}
    Params() = default;
};
}  // namespace alloc_model
}  // namespace bnmf_algs
#endif  // BLDM_USE_REFERENCE_TYPES

namespace bnmf_algs {
namespace bld {
namespace bldm_detail {

inline void throw_status(int rc, const char* where) {
    if (rc == BLDM_OK) return;
    const std::string msg = std::string(where) + ": bldm status " + std::to_string(rc);
    if (rc == BLDM_ERR_BAD_ARG || rc == BLDM_ERR_NEG_X) throw std::invalid_argument(msg);
    throw std::runtime_error(msg);
}

template <typename T> struct solver;
template <> struct solver<double> {
    static int run(const double* X, size_t x, size_t y, size_t z, const bldm_params* p,
                   size_t it, int mode, double eps, const double* S0, uint64_t seed,
                   double* out) {
        return bldm_solve_f64(X, x, y, z, p, it, mode, eps, S0, seed, out, nullptr);
    }
};
template <> struct solver<float> {
    static int run(const float* X, size_t x, size_t y, size_t z, const bldm_params* p,
                   size_t it, int mode, double eps, const float* S0, uint64_t seed, float* out) {
        return bldm_solve_f32(X, x, y, z, p, it, mode, eps, S0, seed, out, nullptr);
    }
};

template <typename T, typename Scalar>
tensor_t<T, 3> solve(const matrix_t<T>& X, size_t z, const alloc_model::Params<Scalar>& mp,
                     size_t max_iter, int psi_mode, double eps, const T* S0, uint64_t seed,
                     const char* where) {
    static_assert(std::is_same<T, double>::value || std::is_same<T, float>::value,
                  "bld_mult on the GPU supports double and float tensors");
    const size_t x = static_cast<size_t>(X.rows());
    const size_t y = static_cast<size_t>(X.cols());
    const std::vector<double> alpha(mp.alpha.begin(), mp.alpha.end());
    const std::vector<double> beta(mp.beta.begin(), mp.beta.end());
    bldm_params p;
    p.a = double(mp.a);
    p.b = double(mp.b);
    p.alpha = alpha.data();
    p.n_alpha = alpha.size();
    p.beta = beta.data();
    p.n_beta = beta.size();
    tensor_t<T, 3> S(x, y, z);
    throw_status(solver<T>::run(X.data(), x, y, z, &p, max_iter, psi_mode, eps, S0, seed,
                                S.data()),
                 where);
    return S;
}

}  // namespace bldm_detail

// bld::bld_mult_cuda (src/bld/bld_mult/bld_mult.hpp:225-324).  As in the
// reference, use_psi_appr=false keeps psi_appr for grad_plus (the reference's
// device kernel has no exact digamma) and uses the exact digamma for
// grad_minus.  The initial S is a seeded Dirichlet split of X (seed 0).
template <typename T, typename Scalar>
tensor_t<T, 3> bld_mult_cuda(const matrix_t<T>& X, const size_t z,
                             const alloc_model::Params<Scalar>& model_params,
                             size_t max_iter = 1000, bool use_psi_appr = false,
                             double eps = 1e-50) {
    return bldm_detail::solve<T, Scalar>(X, z, model_params, max_iter,
                                         use_psi_appr ? BLDM_PSI_APPR : BLDM_PSI_LEGACY_CUDA, eps,
                                         nullptr, 0, "bld_mult_cuda");
}

// bld::bld_mult (bld_mult.hpp:82-150) semantics — exact digamma everywhere
// unless use_psi_appr — computed on the GPU.
template <typename T, typename Scalar>
tensor_t<T, 3> bld_mult(const matrix_t<T>& X, const size_t z,
                        const alloc_model::Params<Scalar>& model_params, size_t max_iter = 1000,
                        bool use_psi_appr = false, double eps = 1e-50) {
    return bldm_detail::solve<T, Scalar>(X, z, model_params, max_iter,
                                         use_psi_appr ? BLDM_PSI_APPR : BLDM_PSI_EXACT, eps,
                                         nullptr, 0, "bld_mult");
}

// Extension: start from a given initial tensor S0 (x*y*z, row-major) instead
// of the seeded Dirichlet split; psi_mode is a bldm_psi_mode.
template <typename T, typename Scalar>
tensor_t<T, 3> bld_mult_from(const matrix_t<T>& X, const tensor_t<T, 3>& S0,
                             const alloc_model::Params<Scalar>& model_params, size_t max_iter,
                             int psi_mode, double eps = 1e-50) {
    if (S0.dimension(0) != X.rows() || S0.dimension(1) != X.cols())
        throw std::invalid_argument("bld_mult_from: S0 shape does not match X");
    return bldm_detail::solve<T, Scalar>(X, static_cast<size_t>(S0.dimension(2)), model_params,
                                         max_iter, psi_mode, eps, S0.data(), 0, "bld_mult_from");
}

// bld::bld_fact (src/bld/bld_fact.hpp:36-80): W (x*z), H (z*y) and L (y)
// from S, computed on the GPU (sums reduced in FP64).
template <typename T, typename Scalar>
std::tuple<matrix_t<T>, matrix_t<T>, vector_t<T>>
bld_fact(const tensor_t<T, 3>& S, const alloc_model::Params<Scalar>& model_params,
         double eps = 1e-50) {
    const size_t x = static_cast<size_t>(S.dimension(0));
    const size_t y = static_cast<size_t>(S.dimension(1));
    const size_t z = static_cast<size_t>(S.dimension(2));
    if (static_cast<size_t>(model_params.alpha.size()) != x)
        throw std::invalid_argument("Number of alpha parameters must be equal to S.dimension(0)");
    if (static_cast<size_t>(model_params.beta.size()) != z)
        throw std::invalid_argument("Number of beta parameters must be equal to z");
    const std::vector<double> alpha(model_params.alpha.data(),
                                    model_params.alpha.data() + x);
    const std::vector<double> beta(model_params.beta.data(), model_params.beta.data() + z);
    bldm_params p;
    p.a = double(model_params.a);
    p.b = double(model_params.b);
    p.alpha = alpha.data();
    p.n_alpha = x;
    p.beta = beta.data();
    p.n_beta = z;
    const std::vector<double> Sd(S.data(), S.data() + x * y * z);
    std::vector<double> Wd(x * z), Hd(z * y), Ld(y);
    bldm_detail::throw_status(
        bldm_bld_fact_f64(Sd.data(), x, y, z, &p, eps, Wd.data(), Hd.data(), Ld.data()),
        "bld_fact");
    matrix_t<T> W(x, z);
    matrix_t<T> H(z, y);
    vector_t<T> L(y);
    for (size_t e = 0; e < x * z; ++e) W.data()[e] = T(Wd[e]);
    for (size_t e = 0; e < z * y; ++e) H.data()[e] = T(Hd[e]);
    for (size_t e = 0; e < y; ++e) L.data()[e] = T(Ld[e]);
    return std::make_tuple(W, H, L);
}

}  // namespace bld
}  // namespace bnmf_algs
