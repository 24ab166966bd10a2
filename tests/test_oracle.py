"""CPU tests that pin the oracle (the CPU restatement of the reference's
bld_mult path) against the reference's own known-answer tests, scipy/mpmath
digamma values, and independent numpy formulations of each stage."""

import numpy as np
import pytest
from scipy.special import digamma, gammaln


# ---- digamma: test/util/test_util.cpp:309-341 (psi_appr vs gsl_sf_psi) ----
def test_psi_appr_below_one_matches_reference_tolerance(oracle):
    xs = np.arange(1e-5, 1, 1e-5)
    err = np.abs(oracle.psi_array(xs, appr=True) - digamma(xs))
    assert err.max() <= 1e-10


def test_psi_appr_above_one_matches_reference_tolerance(oracle):
    xs = np.arange(1.0, 100.0, 1e-3)
    err = np.abs(oracle.psi_array(xs, appr=True) - digamma(xs))
    assert err.max() <= 1e-12


def test_psi_exact_against_mpmath(oracle, psi_points):
    for p, ref in zip(psi_points["points"], psi_points["digamma"]):
        got = oracle.psi_exact(p)
        assert abs(got - ref) <= 2e-15 * max(1.0, abs(ref)), (p, got, ref)


def test_psi_appr_golden_unchanged(oracle, psi_points):
    for p, ref in zip(psi_points["points"], psi_points["psi_appr_oracle"]):
        assert oracle.psi_appr(p) == ref


def test_psi_exact_domain(oracle):
    assert np.isnan(oracle.psi_exact(0.0))
    assert np.isnan(oracle.psi_exact(-1.5))


# ---- known-answer tests: test/bld/bld_mult/test_bld_mult.cpp:33-86 ----
def test_zero_X_gives_zero_S(oracle):
    X = np.zeros((8, 10))
    S = oracle.bld_mult(X, 3, np.ones(8), np.ones(3), 50, oracle.PSI_EXACT)
    assert np.all(S == 0)


@pytest.mark.parametrize("mode,tol_key", [(0, "rowsum_isapprox_exact"),
                                          (1, "rowsum_isapprox_appr")])
def test_kat_8x10_thresholds(oracle, kat, is_approx, mode, tol_key):
    X, z = kat["X"], kat["z"]
    x = X.shape[0]
    alpha, beta = np.ones(x), np.ones(z)
    S0 = oracle.init_S(X, z, kat["init_seed"])
    S = oracle.bld_mult(X, z, alpha, beta, kat["iters"], mode, 1e-50, S0=S0)
    assert oracle.log_marginal_S(S, alpha, beta, kat["a"], kat["b"]) >= kat["log_marginal_min"]
    assert oracle.sparseness(S) >= kat["sparseness_min"]
    assert is_approx(X, S.sum(axis=2), kat[tol_key])
    name = "exact" if mode == 0 else "appr"
    np.testing.assert_allclose(S.reshape(-1), kat[f"S_{name}"], rtol=1e-12, atol=1e-12)


def test_plain_small_golden(oracle, plain_small_golden, workloads):
    g = plain_small_golden
    prob = workloads.plain_small(0)
    np.testing.assert_array_equal(prob["X"], g["X"])
    S0 = oracle.init_S(g["X"], 8, 0)
    np.testing.assert_allclose(S0, g["S0"], rtol=1e-15, atol=0)
    S = oracle.bld_mult(g["X"], 8, g["alpha"], g["beta"], int(g["iters"]), oracle.PSI_APPR,
                        1e-50, S0=g["S0"])
    np.testing.assert_allclose(S, g["S"], rtol=1e-12, atol=1e-13)


# ---- stages vs independent numpy formulations ----
def _rand_problem(rng, x, y, z):
    S = rng.random((x, y, z)) + 1.0
    X = rng.random((x, y)) + 10.0
    return S, X


def test_tensor_sums_numpy(oracle):
    rng = np.random.default_rng(0)
    S = rng.random((37, 23, 9))
    pjk, ipk, ijp = oracle.tensor_sums(S)
    np.testing.assert_allclose(pjk, S.sum(0), rtol=1e-13)
    np.testing.assert_allclose(ipk, S.sum(1), rtol=1e-13)
    np.testing.assert_allclose(ijp, S.sum(2), rtol=1e-13)


def test_one_iteration_matches_numpy_formulation(oracle):
    rng = np.random.default_rng(1)
    x, y, z = 13, 17, 5
    S, X = _rand_problem(rng, x, y, z)
    alpha = rng.uniform(0.5, 2, x)
    beta = rng.uniform(0.5, 2, z)
    eps = 1e-50
    out = oracle.bld_mult(X, z, alpha, beta, 1, oracle.PSI_EXACT, eps, S0=S)
    # numpy restatement of bld_mult.hpp:123-147 with scipy's digamma
    pjk, ipk, ijp = S.sum(0), S.sum(1), S.sum(2)
    alpha_eph = ipk + alpha[:, None]
    beta_eph = pjk + beta[None, :]
    gp = digamma(beta_eph)[None, :, :] - digamma(S + 1)
    gm = digamma(alpha_eph.sum(0))[None, :] - digamma(alpha_eph)
    Xr = 1.0 / (X + eps)
    nom = np.einsum("ijk,ij,ik->ij", S, Xr, gm)
    den = np.einsum("ijk,ij,ijk->ij", S, Xr, gp)
    ref = S * (gp + nom[:, :, None]) * (X / (ijp + eps))[:, :, None] / (
        gm[:, None, :] + den[:, :, None] + eps)
    np.testing.assert_allclose(out, ref, rtol=1e-12)


def test_stage_functions_compose_to_driver(oracle):
    rng = np.random.default_rng(2)
    x, y, z = 9, 11, 4
    S, X = _rand_problem(rng, x, y, z)
    alpha, beta = np.ones(x), np.ones(z)
    pjk, ipk, ijp = oracle.tensor_sums(S)
    ae = oracle.update_alpha_eph(ipk, alpha)
    be = oracle.update_beta_eph(pjk, beta)
    gp = oracle.update_grad_plus(S, be, appr=True)
    gm = oracle.update_grad_minus(ae, appr=True)
    Xr = oracle.x_reciprocal(X)
    nom = oracle.update_nom(Xr, gm, S)
    den = oracle.update_denom(Xr, gp, S)
    S1 = oracle.update_S(X, nom, den, gm, gp, ijp, S)
    ref = oracle.bld_mult(X, z, alpha, beta, 1, oracle.PSI_APPR, 1e-50, S0=S)
    np.testing.assert_array_equal(S1, ref)


def test_legacy_mode_mixes_digammas(oracle):
    rng = np.random.default_rng(3)
    x, y, z = 6, 7, 3
    S, X = _rand_problem(rng, x, y, z)
    a, b = np.ones(x), np.ones(z)
    legacy = oracle.bld_mult(X, z, a, b, 3, oracle.PSI_LEGACY_CUDA, 1e-50, S0=S)
    exact = oracle.bld_mult(X, z, a, b, 3, oracle.PSI_EXACT, 1e-50, S0=S)
    appr = oracle.bld_mult(X, z, a, b, 3, oracle.PSI_APPR, 1e-50, S0=S)
    # all three agree to the digamma approximation error, but are not identical
    np.testing.assert_allclose(legacy, exact, rtol=1e-9)
    np.testing.assert_allclose(legacy, appr, rtol=1e-9)
    assert not np.array_equal(legacy, appr)


# ---- log_marginal_S, sparseness, bld_fact vs numpy/scipy ----
def test_log_marginal_numpy(oracle):
    rng = np.random.default_rng(4)
    x, y, z = 12, 9, 4
    S = rng.poisson(2.0, (x, y, z)).astype(float)
    alpha = rng.uniform(0.5, 2, x)
    beta = rng.uniform(0.5, 2, z)
    a, b = 3.0, 0.7
    ipk, pjk, pjp = S.sum(1), S.sum(0), S.sum((0, 2))
    first = z * (gammaln(alpha.sum()) - gammaln(alpha).sum()) + sum(
        gammaln(alpha + ipk[:, k]).sum() - gammaln((alpha + ipk[:, k]).sum()) for k in range(z))
    second = y * (gammaln(beta.sum()) - gammaln(beta).sum()) + sum(
        gammaln(beta + pjk[j]).sum() - gammaln((beta + pjk[j]).sum()) for j in range(y))
    third = y * (-gammaln(a) + a * np.log(b)) + np.sum(gammaln(a + pjp) - (a + pjp) * np.log(b + 1))
    fourth = gammaln(S + 1).sum()
    ref = first + second + third - fourth
    got = oracle.log_marginal_S(S, alpha, beta, a, b)
    assert abs(got - ref) <= 1e-10 * abs(ref)


def test_sparseness_numpy(oracle):
    rng = np.random.default_rng(5)
    S = rng.random((5, 6, 7))
    n = S.size
    ref = (np.sqrt(n) - S.sum() / np.linalg.norm(S)) / (np.sqrt(n) - 1)
    assert abs(oracle.sparseness(S) - ref) < 1e-14
    assert oracle.sparseness(np.zeros((2, 2, 2))) > 1e300


def test_bld_fact_numpy(oracle):
    rng = np.random.default_rng(6)
    x, y, z = 5, 6, 3
    S = rng.random((x, y, z)) * 4
    alpha, beta = rng.uniform(1, 2, x), rng.uniform(1, 2, z)
    a, b, eps = 2.0, 0.5, 1e-50
    W, H, L = oracle.bld_fact(S, alpha, beta, a, b, eps)
    W_ref = alpha[:, None] + S.sum(1) - 1
    H_ref = (beta[:, None] + S.sum(0).T - 1)
    L_ref = (a + S.sum((0, 2)) - 1) / (b + 1 + eps)
    np.testing.assert_allclose(W, W_ref / (W_ref.sum(0) + eps), rtol=1e-13)
    np.testing.assert_allclose(H, H_ref / (H_ref.sum(0) + eps), rtol=1e-13)
    np.testing.assert_allclose(L, L_ref, rtol=1e-13)


def test_init_S_is_dirichlet_split(oracle):
    rng = np.random.default_rng(7)
    X = rng.poisson(3.0, (20, 30)).astype(float)
    S = oracle.init_S(X, 6, 11)
    np.testing.assert_allclose(S.sum(2), X, rtol=1e-14, atol=1e-14)
    assert np.all(S >= 0)
    S2 = oracle.init_S(X, 6, 12)
    assert not np.array_equal(S, S2)


def test_fp32_sweep_digamma_formula_truncation():
    """The FP32 sweep's digamma (csrc/bldm_device.cuh, psi_f32_batch) as
    mathematics, evaluated here in float64: arguments below 4 shifted by three
    recurrence steps summed as one rational function, the asymptotic series
    through x^-10.  Its truncation error must sit far below FP32 resolution
    (the GPU test bounds the rounded FP32 evaluation at 2e-6)."""
    v = np.concatenate([np.linspace(1e-3, 12, 120001), np.geomspace(12, 1e9, 2000)])
    lo = v < 4
    q = np.where(lo, ((v + 3) * v + 2) * v, 1.0)
    p = np.where(lo, (3 * v + 6) * v + 2, 0.0)
    xs = np.where(lo, v + 3, v)
    r = 1 / xs
    r2 = r * r
    t = 1 / 240 - r2 / 132
    t = 1 / 252 - r2 * t
    t = 1 / 120 - r2 * t
    t = 1 / 12 - r2 * t
    got = np.log(xs) - 0.5 * r - r2 * t - p / q
    ref = digamma(v)
    assert (np.abs(got - ref) / np.maximum(1.0, np.abs(ref))).max() <= 3e-9
