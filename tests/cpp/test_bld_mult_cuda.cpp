// Re-expresses the reference's test/bld/bld_mult/test_bld_mult_cuda.cpp
// (parameter checks, zero matrix, the 8x10 known-answer case) against the
// header-only C++14 mirror, which runs on the GPU through libbldm.so.
//
// usage: test_bld_mult_cuda <kat_X.txt> <out_S_legacy.txt> <out_S_appr.txt>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <stdexcept>

#include "bnmf_algs_b200/bld_mult.hpp"

using namespace bnmf_algs;

#define REQUIRE(c)                                                             \
    do {                                                                       \
        if (!(c)) {                                                            \
            std::fprintf(stderr, "FAILED %s:%d: %s\n", __FILE__, __LINE__, #c); \
            return 1;                                                          \
        }                                                                      \
    } while (0)

template <typename F> static bool throws_invalid(F f) {
    try {
        f();
    } catch (const std::invalid_argument&) {
        return true;
    }
    return false;
}

// test_bld_mult_cuda.cpp:10-31
static int parameter_checks() {
    size_t x = 10, y = 5, z = 2;
    shape<3> tensor_shape{x, y, z};
    matrix_t<double> X = matrix_t<double>::Constant(x, y, 5);
    alloc_model::Params<double> model_params(tensor_shape);
    REQUIRE(!throws_invalid([&] { bld::bld_mult_cuda(X, z, model_params, 5); }));
    X(0, 0) = -5;
    REQUIRE(throws_invalid([&] { bld::bld_mult_cuda(X, z, model_params); }));
    X(0, 0) = 0;
    REQUIRE(!throws_invalid([&] { bld::bld_mult_cuda(X, z, model_params, 5); }));
    z++;
    REQUIRE(throws_invalid([&] { bld::bld_mult_cuda(X, z, model_params); }));
    z--;
    X = matrix_t<double>::Constant(x + 1, y, 5);
    REQUIRE(throws_invalid([&] { bld::bld_mult_cuda(X, z, model_params); }));
    // the same checks hold for the FP32 instantiation and for bld_mult
    matrix_t<float> Xf = matrix_t<float>::Constant(x, y, 5);
    alloc_model::Params<float> pf(tensor_shape);
    REQUIRE(!throws_invalid([&] { bld::bld_mult_cuda(Xf, z, pf, 5); }));
    Xf(1, 1) = -1;
    REQUIRE(throws_invalid([&] { bld::bld_mult(Xf, z, pf, 5); }));
    return 0;
}

// test_bld_mult_cuda.cpp:36-46
static int zero_matrix() {
    size_t x = 8, y = 10, z = 3;
    shape<3> tensor_shape{x, y, z};
    matrix_t<double> X = matrix_t<double>::Zero(x, y);
    alloc_model::Params<double> model_params(tensor_shape);
    tensor_t<double, 3> S = bld::bld_mult_cuda(X, z, model_params);
    for (long e = 0; e < S.size(); ++e) REQUIRE(S.data()[e] == 0.0);
    return 0;
}

static bool is_approx(const matrix_t<double>& X, const tensor_t<double, 3>& S, double prec) {
    const size_t x = X.rows(), y = X.cols(), z = S.dimension(2);
    double d2 = 0, a2 = 0, b2 = 0;
    for (size_t i = 0; i < x; ++i)
        for (size_t j = 0; j < y; ++j) {
            double s = 0;
            for (size_t k = 0; k < z; ++k) s += S(i, j, k);
            d2 += (X(i, j) - s) * (X(i, j) - s);
            a2 += X(i, j) * X(i, j);
            b2 += s * s;
        }
    return std::sqrt(d2) <= prec * std::sqrt(a2 < b2 ? a2 : b2);
}

static void write_tensor(const char* path, const tensor_t<double, 3>& S) {
    std::FILE* f = std::fopen(path, "w");
    for (long e = 0; e < S.size(); ++e) std::fprintf(f, "%.17g\n", S.data()[e]);
    std::fclose(f);
}

// test_bld_mult_cuda.cpp:48-84 (log_marginal and sparseness thresholds are
// checked by the calling test with the oracle's log_marginal_S).
static int known_answer(const char* xpath, const char* out_legacy, const char* out_appr) {
    size_t x = 8, y = 10, z = 3;
    matrix_t<double> X(x, y);
    std::ifstream in(xpath);
    for (size_t i = 0; i < x; ++i)
        for (size_t j = 0; j < y; ++j) in >> X(i, j);
    REQUIRE(bool(in));
    alloc_model::Params<double> model_params(40, 1, std::vector<double>(x, 1.0),
                                             std::vector<double>(z, 1.0));
    tensor_t<double, 3> S = bld::bld_mult_cuda(X, z, model_params, 2000);
    REQUIRE(is_approx(X, S, 1e-10));
    write_tensor(out_legacy, S);
    S = bld::bld_mult_cuda(X, z, model_params, 2000, true);
    REQUIRE(is_approx(X, S, 1e-4));
    write_tensor(out_appr, S);
    return 0;
}

// bld_fact (src/bld/bld_fact.hpp:36-80) of a small deterministic tensor
// against its definition evaluated here with plain loops.
static int factorization() {
    const size_t x = 7, y = 5, z = 3;
    tensor_t<double, 3> S(x, y, z);
    for (size_t i = 0; i < x; ++i)
        for (size_t j = 0; j < y; ++j)
            for (size_t k = 0; k < z; ++k) S(i, j, k) = double((i * 7 + j * 3 + k * 5) % 11);
    std::vector<double> alpha(x), beta(z);
    for (size_t i = 0; i < x; ++i) alpha[i] = 1.0 + 0.25 * double(i);
    for (size_t k = 0; k < z; ++k) beta[k] = 0.5 + double(k);
    alloc_model::Params<double> mp(2.0, 3.0, alpha, beta);
    auto f = bld::bld_fact(S, mp, 1e-50);
    const matrix_t<double>& W = std::get<0>(f);
    const matrix_t<double>& H = std::get<1>(f);
    const vector_t<double>& L = std::get<2>(f);
    for (size_t k = 0; k < z; ++k) {
        double cs = 0;
        for (size_t i = 0; i < x; ++i) {
            double s = 0;
            for (size_t j = 0; j < y; ++j) s += S(i, j, k);
            cs += alpha[i] + s - 1;
        }
        for (size_t i = 0; i < x; ++i) {
            double s = 0;
            for (size_t j = 0; j < y; ++j) s += S(i, j, k);
            REQUIRE(std::fabs(W(i, k) - (alpha[i] + s - 1) / (cs + 1e-50)) <= 1e-12);
        }
    }
    for (size_t j = 0; j < y; ++j) {
        double cs = 0, pjp = 0;
        for (size_t k = 0; k < z; ++k) {
            double s = 0;
            for (size_t i = 0; i < x; ++i) s += S(i, j, k);
            cs += beta[k] + s - 1;
            pjp += s;
        }
        for (size_t k = 0; k < z; ++k) {
            double s = 0;
            for (size_t i = 0; i < x; ++i) s += S(i, j, k);
            REQUIRE(std::fabs(H(k, j) - (beta[k] + s - 1) / (cs + 1e-50)) <= 1e-12);
        }
        REQUIRE(std::fabs(L(j) - (2.0 + pjp - 1) / (3.0 + 1 + 1e-50)) <= 1e-12 * std::fabs(L(j)));
    }
    alloc_model::Params<double> bad(2.0, 3.0, std::vector<double>(x + 1, 1.0), beta);
    REQUIRE(throws_invalid([&] { bld::bld_fact(S, bad); }));
    return 0;
}

int main(int argc, char** argv) {
    if (argc != 4) {
        std::fprintf(stderr, "usage: %s kat_X.txt out_legacy.txt out_appr.txt\n", argv[0]);
        return 2;
    }
    if (parameter_checks()) return 1;
    if (zero_matrix()) return 1;
    if (known_answer(argv[1], argv[2], argv[3])) return 1;
    if (factorization()) return 1;
    std::printf("ok\n");
    return 0;
}
