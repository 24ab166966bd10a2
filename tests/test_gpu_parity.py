"""GPU parity of libbldm.so against the CPU oracle.

Tolerances (FP64 storage): per-stage results within Eigen's default isApprox
precision for double (1e-12), as the reference's
test/bld/bld_mult/test_bld_mult_cuda_funcs.cpp requires; whole solves within
1e-9 relative (max-norm relative error), the bar the reference's FP64 build
is held to.  FP32 storage is compared with the FP64 oracle at the tolerance
stated in each test.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def rel_err(a, b):
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    scale = max(np.abs(b).max(), 1e-300)
    return float(np.abs(a - b).max() / scale)


def dev(a, dtype=torch.float64):
    return torch.as_tensor(np.ascontiguousarray(a)).to(device="cuda", dtype=dtype)


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


# ---------------------------------------------------------------- digamma
def test_psi_appr_and_exact_match_oracle(bldm, oracle, psi_points):
    rng = np.random.default_rng(0)
    pts = np.concatenate([psi_points["points"], rng.uniform(1e-6, 1, 5000),
                          rng.uniform(1, 7, 5000), rng.lognormal(2, 3, 5000)])
    d = dev(pts)
    # 0: exact, 1: psi_appr, 2: psi_appr as the fused sweep evaluates it
    for mode in (0, 1, 2):
        got = host(bldm.psi(d, appr=mode))
        ref = oracle.psi_array(pts, appr=mode != 0)
        err = np.abs(got - ref) / np.maximum(1.0, np.abs(ref))
        assert err.max() <= 2e-14, (mode, err.max(), pts[err.argmax()])


@pytest.mark.parametrize("mode", [1, 2])   # 1: tabulating form, 2: the FP32 sweep's form
def test_psi_f32(bldm, mode):
    from scipy.special import digamma
    rng = np.random.default_rng(1)
    # the sweep evaluates psi(S + 1) >= 1; both forms also cover (0, 1) and
    # counts up to ~1e8 through the lognormal draws
    pts = np.concatenate([rng.uniform(1, 7, 4000), rng.uniform(3.9, 4.1, 2000),
                          rng.lognormal(2, 3, 4000), [1.0, 3.0, 4.0, 1e8]]).astype(np.float32)
    got = host(bldm.psi(dev(pts, torch.float32), appr=mode)).astype(np.float64)
    ref = digamma(pts.astype(np.float64))
    assert (np.abs(got - ref) / np.maximum(1.0, np.abs(ref))).max() <= 2e-6
    # psi(+inf) = +inf
    inf = host(bldm.psi(dev(np.array([np.inf], np.float32), torch.float32), appr=mode))
    assert np.isposinf(inf[0]), inf


# ------------------------------------------------- per-stage (reference funcs tests)
def test_tensor_sums_stage(bldm, oracle, is_approx):
    rng = np.random.default_rng(2)
    S = rng.uniform(-1, 1, (1024, 456, 17))       # Eigen setRandom range
    pjk, ipk, ijp = (host(t) for t in bldm.tensor_sums(dev(S)))
    rp, ri, rj = oracle.tensor_sums(S)
    assert is_approx(pjk, rp, 1e-12) and is_approx(ipk, ri, 1e-12) and is_approx(ijp, rj, 1e-12)


@pytest.mark.parametrize("appr", [True, False])
def test_grad_plus_stage(bldm, oracle, is_approx, appr):
    rng = np.random.default_rng(3)
    x, y, z = 131, 456, 89
    S = rng.uniform(-1, 1, (x, y, z)) + 1
    beta_eph = rng.uniform(-1, 1, (y, z)) + 1
    got = host(bldm.update_grad_plus(dev(S), dev(beta_eph), appr=appr))
    ref = oracle.update_grad_plus(S, beta_eph, appr=appr)
    assert is_approx(got, ref, 1e-12)


def test_grad_minus_stage(bldm, oracle, is_approx):
    rng = np.random.default_rng(4)
    ae = rng.uniform(0.5, 20, (356, 17))
    for appr in (True, False):
        got = host(bldm.update_grad_minus(dev(ae), appr=appr))
        assert is_approx(got, oracle.update_grad_minus(ae, appr=appr), 1e-12)


def _nom_inputs(rng, x=356, y=478, z=17):
    X = rng.uniform(-1, 1, (x, y)) + 10
    Xr = 1.0 / X
    gm = rng.uniform(-1, 1, (x, z)) + 2
    S = rng.uniform(-1, 1, (x, y, z)) + 1
    return X, Xr, gm, S


def test_nom_stage(bldm, oracle, is_approx):
    X, Xr, gm, S = _nom_inputs(np.random.default_rng(5))
    got = host(bldm.update_nom(dev(Xr), dev(gm), dev(S)))
    assert is_approx(got, oracle.update_nom(Xr, gm, S), 1e-12)


def test_denom_stage(bldm, oracle, is_approx):
    X, Xr, gm, S = _nom_inputs(np.random.default_rng(6))
    gp = S.copy()
    got = host(bldm.update_denom(dev(Xr), dev(gp), dev(S)))
    assert is_approx(got, oracle.update_denom(Xr, gp, S), 1e-12)


def test_update_S_stage(bldm, oracle, is_approx):
    rng = np.random.default_rng(7)
    X, Xr, gm, S = _nom_inputs(rng)
    x, y, z = S.shape
    nom = rng.uniform(-1, 1, (x, y)) + 3
    den = rng.uniform(-1, 1, (x, y)) + 5
    gp = S.copy()
    ijp = S.sum(2)
    dS = dev(S)
    bldm.update_S(dev(X), dev(nom), dev(den), dev(gm), dev(gp), dev(ijp), dS)
    ref = oracle.update_S(X, nom, den, gm, gp, ijp, S)
    assert is_approx(host(dS), ref, 1e-12)


# ------------------------------------------------------------- fused solver
def test_plain_small_golden_parity(bldm, plain_small_golden):
    g = plain_small_golden
    params = bldm.Params(5.0, 0.1, g["alpha"], g["beta"])
    S = bldm.bld_mult(g["X"], 8, params, int(g["iters"]), use_psi_appr=True, S0=g["S0"])
    assert rel_err(S, g["S"]) <= 1e-9


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_modes_match_oracle(bldm, oracle, workloads, mode):
    prob = workloads.plain_small(5)
    X, z = prob["X"], prob["z"]
    S0 = oracle.init_S(X, z, 3)
    ref = oracle.bld_mult(X, z, prob["alpha"], prob["beta"], 60, mode, 1e-50, S0=S0)
    params = bldm.Params(prob["a"], prob["b"], prob["alpha"], prob["beta"])
    S = bldm._solve(X, z, params, 60, mode, 1e-50, S0, 0, bldm.F64, None)
    assert rel_err(S, ref) <= 1e-9


SHAPES = [(1, 1, 1), (3, 5, 1), (2, 3, 2), (33, 65, 3), (65, 33, 17), (7, 300, 5),
          (5, 7, 33), (40, 41, 64), (9, 13, 100), (4, 9, 128), (3, 5, 256), (2, 3, 255), (2, 3, 512),
          (300, 7, 8), (17, 1000, 4),
          # fibers longer than the fused sweep's lane layout (the two-pass path):
          # odd z above 256, even z above 512
          (3, 5, 257), (3, 5, 513), (4, 9, 1000), (2, 3, 2048), (17, 11, 600), (70, 9, 777)]


@pytest.mark.parametrize("shape", SHAPES)
def test_odd_shapes_fp64(bldm, oracle, shape):
    x, y, z = shape
    rng = np.random.default_rng(x * 1000003 + y * 101 + z)
    X = rng.poisson(rng.uniform(0.2, 30), (x, y)).astype(np.float64)
    alpha = rng.uniform(0.5, 2, x)
    beta = rng.uniform(0.5, 2, z)
    S0 = oracle.init_S(X, z, 1)
    ref = oracle.bld_mult(X, z, alpha, beta, 12, oracle.PSI_APPR, 1e-50, S0=S0)
    S = bldm.bld_mult(X, z, bldm.Params(1, 1, alpha, beta), 12, True, S0=S0)
    assert rel_err(S, ref) <= 1e-9


@pytest.mark.parametrize("shape", [(3, 5, 1), (33, 65, 3), (40, 41, 4), (9, 13, 64), (5, 7, 17),
                                   (64, 48, 8), (4, 9, 512), (3, 4, 1000),
                                   (3, 4, 1500), (6, 10, 1025), (5, 3, 301)])
def test_odd_shapes_fp32(bldm, oracle, shape):
    x, y, z = shape
    rng = np.random.default_rng(x * 7 + y * 13 + z)
    X = rng.poisson(rng.uniform(0.5, 20), (x, y)).astype(np.float64)
    alpha, beta = np.ones(x), np.ones(z)
    S0 = oracle.init_S(X, z, 2)
    ref = oracle.bld_mult(X, z, alpha, beta, 12, oracle.PSI_APPR, 1e-50, S0=S0)
    S = bldm.bld_mult(X, z, bldm.Params(1, 1, alpha, beta), 12, True,
                      S0=S0.astype(np.float32), dtype=bldm.F32)
    # FP32 storage: within 1e-5 (max-norm relative) of FP64, or within 10x the
    # error of the FP32 restatement itself where the problem is ill-conditioned
    # in single precision (cancellation in psi(beta_eph) - psi(S+1)); two FP32
    # evaluations with different rounding then differ by the same order.
    ref32 = oracle.bld_mult(X, z, alpha, beta, 12, oracle.PSI_APPR, 1e-50, S0=S0,
                            dtype=np.float32)
    assert rel_err(S, ref) <= max(1e-5, 10 * rel_err(ref32, ref))


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_long_fibers_all_modes_match_oracle(bldm, oracle, mode):
    """The two-pass long-fiber path in every digamma mode, with rows of X that
    are all zero and fibers of several k-chunks, bands and row ranges."""
    rng = np.random.default_rng(90 + mode)
    x, y, z = 45, 21, 1100
    X = rng.poisson(3.0, (x, y)).astype(np.float64)
    X[7, :] = 0.0
    X[:, 4] = 0.0
    alpha = rng.uniform(0.5, 2, x)
    beta = rng.uniform(0.5, 2, z)
    S0 = oracle.init_S(X, z, 4)
    ref = oracle.bld_mult(X, z, alpha, beta, 15, mode, 1e-50, S0=S0)
    params = bldm.Params(1.0, 1.0, alpha, beta)
    stats = {}
    S = bldm._solve(X, z, params, 15, mode, 1e-50, S0, 0, bldm.F64, stats)
    assert rel_err(S, ref) <= 1e-9
    assert np.all(S[X == 0] == 0)
    want = float((np.abs(S.sum(axis=2) - X) / np.maximum(X, 1.0)).max())
    assert abs(stats["conservation_residual"] - want) <= 1e-12 * max(want, 1.0)
    # bld_fact of the long-fiber solution (the sums sweep of the same path)
    W0, H0, L0 = oracle.bld_fact(S, alpha, beta, 1.0, 1.0, 1e-50)
    W, H, L = bldm.bld_fact(S, params)
    for a, b in ((W, W0), (H, H0), (L, L0)):
        assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max()


def test_fp32_plain_small_vs_fp64_oracle(bldm, plain_small_golden):
    g = plain_small_golden
    params = bldm.Params(5.0, 0.1, g["alpha"], g["beta"])
    S = bldm.bld_mult(g["X"], 8, params, int(g["iters"]), use_psi_appr=True,
                      S0=g["S0"].astype(np.float32), dtype=bldm.F32)
    assert np.all(np.isfinite(S))
    # 200 iterations in FP32 with compensated sums: 1e-4 max-norm relative
    assert rel_err(S, g["S"]) <= 1e-4


def test_zero_X_gives_zero_S(bldm):
    for dt in (bldm.F64, bldm.F32):
        S = bldm.bld_mult_cuda(np.zeros((8, 10)), 3, bldm.Params.from_shape((8, 10, 3)), 1000,
                               dtype=dt)
        assert np.all(S == 0)


def test_zero_rows_cols_and_inconsistent_S0(bldm, oracle):
    rng = np.random.default_rng(9)
    X = rng.poisson(4.0, (20, 30)).astype(float)
    X[3, :] = 0
    X[:, 7] = 0
    S0 = oracle.init_S(X, 6, 5)
    S0[1, 2, :] = 0.0          # X > 0 but the initial fiber is empty
    S0[3, 4, :] = 1.0          # X == 0 but the initial fiber is not
    a, b = np.ones(20), np.ones(6)
    ref = oracle.bld_mult(X, 6, a, b, 20, oracle.PSI_APPR, 1e-50, S0=S0)
    S = bldm.bld_mult(X, 6, bldm.Params(1, 1, a, b), 20, True, S0=S0)
    assert np.all(np.isfinite(S))
    assert np.all(S[3] == 0) and np.all(S[:, 7] == 0) and np.all(S[1, 2] == 0)
    assert rel_err(S, ref) <= 1e-9
    S32 = bldm.bld_mult(X, 6, bldm.Params(1, 1, a, b), 20, True, S0=S0.astype(np.float32),
                        dtype=bldm.F32)
    assert np.all(np.isfinite(S32)) and np.all(S32[3] == 0) and np.all(S32[1, 2] == 0)


def test_solver_is_deterministic(bldm, workloads):
    prob = workloads.plain_small(1)
    params = bldm.Params(prob["a"], prob["b"], prob["alpha"], prob["beta"])
    a = bldm.bld_mult_cuda(prob["X"], prob["z"], params, 50, True, seed=4)
    b = bldm.bld_mult_cuda(prob["X"], prob["z"], params, 50, True, seed=4)
    np.testing.assert_array_equal(a, b)


def test_device_init_S_matches_oracle(bldm, oracle):
    rng = np.random.default_rng(10)
    X = rng.poisson(5.0, (50, 70)).astype(float)
    # lane groups narrower than a warp (z = 1, 9), four draws per lane kept in
    # registers (z = 64) and draws beyond them made again for the stores (z = 200)
    for zz in (1, 64, 200, 9):
        plan = bldm.Plan(50, 70, zz)
        dS = torch.empty((50, 70, zz), dtype=torch.float64, device="cuda")
        plan.init_S(dev(X), dS, seed=77)
        got = host(dS)
        ref = oracle.init_S(X, zz, 77)
        assert rel_err(got, ref) <= 1e-14, zz
        if zz != 9:
            plan.close()
    # a solve with S0=None starts from the same tensor
    params = bldm.Params(1, 1, np.ones(50), np.ones(9))
    S1 = bldm.bld_mult(X, 9, params, 3, True, seed=77)
    S2 = bldm.bld_mult(X, 9, params, 3, True, S0=ref)
    assert rel_err(S1, S2) <= 1e-13
    plan.close()


def test_plan_api_matches_host_api(bldm, workloads, oracle):
    prob = workloads.plain_small(2)
    X, z = prob["X"], prob["z"]
    x, y = X.shape
    S0 = oracle.init_S(X, z, 8)
    params = bldm.Params(prob["a"], prob["b"], prob["alpha"], prob["beta"])
    ref = bldm.bld_mult(X, z, params, 40, True, S0=S0)
    plan = bldm.Plan(x, y, z)
    dS = dev(S0)
    plan.run(dev(X), dev(prob["alpha"]), dev(prob["beta"]), dS, 40, bldm.PSI_APPR)
    plan.check()
    np.testing.assert_array_equal(host(dS), ref)
    assert plan.launch_count() == 2 + 40 + 39
    assert plan.workspace_bytes() > 0
    plan.close()


def test_full_size_one_iteration_parity(bldm, oracle, workloads):
    prob = workloads.plain_large(1)
    X, z = prob["X"], prob["z"]
    oracle.set_threads(0)
    S0 = oracle.init_S(X, z, 0)
    ref = oracle.bld_mult(X, z, prob["alpha"], prob["beta"], 1, oracle.PSI_APPR, 1e-50, S0=S0)
    params = bldm.Params(prob["a"], prob["b"], prob["alpha"], prob["beta"])
    S = bldm.bld_mult(X, z, params, 1, True, S0=S0)
    assert rel_err(S, ref) <= 1e-12
    # size-independent properties after more iterations: nonnegative, finite,
    # zero fibers of X stay zero, the row sums move toward X
    S5 = bldm.bld_mult(X, z, params, 5, True, S0=S0)
    assert np.all(np.isfinite(S5)) and S5.min() >= 0
    assert np.all(S5[X == 0] == 0)


def test_full_size_benchmarked_solve_parity(bldm, oracle, workloads):
    """The benchmarked solve itself: 1024x1024x64, FP64, psi_appr, 100
    iterations, within 1e-9 (max-norm relative) of the oracle from the same S0,
    through the drop-in host-buffer call; its conservation residual against
    numpy's."""
    prob = workloads.plain_large(1)
    X, z, iters = prob["X"], prob["z"], prob["iters"]
    assert (X.shape, z, iters) == ((1024, 1024), 64, 100)
    oracle.set_threads(0)
    S0 = oracle.init_S(X, z, 0)
    ref = oracle.bld_mult(X, z, prob["alpha"], prob["beta"], iters, oracle.PSI_APPR, 1e-50,
                          S0=S0)
    params = bldm.Params(prob["a"], prob["b"], prob["alpha"], prob["beta"])
    stats = {}
    S = bldm.bld_mult(X, z, params, iters, True, S0=S0, stats=stats)
    assert rel_err(S, ref) <= 1e-9, rel_err(S, ref)
    cons = np.abs(S.sum(axis=2) - X) / np.maximum(X, 1.0)
    assert abs(stats["conservation_residual"] - cons.max()) <= 1e-12 * max(cons.max(), 1.0)


def _cons_np(X, S):
    S = np.asarray(S, dtype=np.float64)
    return float((np.abs(S.sum(axis=2) - X) / np.maximum(X, 1.0)).max())


@pytest.mark.parametrize("dtype_name", ["f64", "f32"])
@pytest.mark.parametrize("shape", [(64, 48, 8), (37, 29, 3), (50, 41, 100), (9, 13, 1)])
def test_conservation_residual_matches_numpy(bldm, oracle, workloads, dtype_name, shape):
    x, y, z = shape
    f64 = dtype_name == "f64"
    rng = np.random.default_rng(x + y + z)
    X = workloads.allocation_model_X(x, y, z, 5.0, 0.05, rng) + rng.poisson(1.0, (x, y))
    S0 = oracle.init_S(X, z, 3)
    params = bldm.Params(1.0, 1.0, np.ones(x), np.ones(z))
    stats = {}
    S = bldm.bld_mult(X, z, params, 7, True, S0=S0, stats=stats,
                      dtype=bldm.F64 if f64 else bldm.F32)
    want = _cons_np(X.astype(S.dtype), S)
    tol = 1e-12 if f64 else 1e-5
    assert abs(stats["conservation_residual"] - want) <= tol * max(want, 1.0)
    assert want > 0.0  # 7 iterations from a random split are not at the fixed point
    # the plan API on device buffers, including an S0 that conserves exactly
    tt = torch.float64 if f64 else torch.float32
    plan = bldm.Plan(x, y, z, bldm.F64 if f64 else bldm.F32)
    dX = dev(X, tt)
    assert plan.conservation(dX, dev(S, tt)) == pytest.approx(want, rel=tol, abs=tol)
    assert plan.conservation(dX, dev(S0, tt)) <= (1e-14 if f64 else 1e-6)
    # S one element past a 16-byte boundary: scalar loads instead of 16-byte ones
    buf = torch.empty(S.size + 1, dtype=tt, device="cuda")
    buf[1:] = dev(S, tt).reshape(-1)
    assert buf[1:].data_ptr() % 16 != 0
    assert plan.conservation(dX, buf[1:]) == pytest.approx(want, rel=tol, abs=tol)
    plan.close()


def test_conservation_residual_reports_nan(bldm):
    x, y, z = 8, 8, 4
    X = np.ones((x, y))
    S = np.full((x, y, z), 0.25)
    S[3, 5, 2] = np.nan
    plan = bldm.Plan(x, y, z, bldm.F64)
    assert np.isnan(plan.conservation(dev(X), dev(S)))
    S[3, 5, 2] = 0.25
    assert plan.conservation(dev(X), dev(S)) == 0.0
    plan.close()


def test_log_marginal_device_matches_oracle(bldm, oracle):
    rng = np.random.default_rng(11)
    x, y, z = 70, 90, 12
    S = rng.poisson(1.5, (x, y, z)).astype(float) * rng.random((x, y, z))
    alpha = rng.uniform(0.5, 2, x)
    beta = rng.uniform(0.5, 2, z)
    params = bldm.Params(3.0, 0.5, alpha, beta)
    ref = oracle.log_marginal_S(S, alpha, beta, 3.0, 0.5)
    got = bldm.log_marginal_S(dev(S), params)
    assert abs(got - ref) <= 1e-11 * abs(ref)
    got32 = bldm.log_marginal_S(dev(S, torch.float32), params, dtype=bldm.F32)
    ref32 = oracle.log_marginal_S(S.astype(np.float32), alpha, beta, 3.0, 0.5)
    assert abs(got32 - ref32) <= 1e-11 * abs(ref32)


@pytest.mark.parametrize("use_appr", [False, True])
def test_kat_8x10_on_gpu(bldm, oracle, kat, is_approx, use_appr):
    X, z = kat["X"], kat["z"]
    x = X.shape[0]
    params = bldm.Params(kat["a"], kat["b"], np.ones(x), np.ones(z))
    S = bldm.bld_mult(X, z, params, kat["iters"], use_appr, seed=kat["init_seed"])
    name = "appr" if use_appr else "exact"
    assert oracle.log_marginal_S(S, np.ones(x), np.ones(z), kat["a"], kat["b"]) >= -262
    assert oracle.sparseness(S) >= kat["sparseness_min"]
    assert is_approx(X, S.sum(2), kat["rowsum_isapprox_" + name])
    assert rel_err(S.reshape(-1), kat["S_" + name]) <= 1e-9


@pytest.mark.parametrize("dtype_name", ["F64", "F32"])
def test_zero_row_skip_gives_the_same_S(bldm, workloads, dtype_name):
    """skip_zero_rows (later updates sweep only the rows whose band segment of
    X has a nonzero and store no zeros again) gives bitwise the S of the
    streaming sweep, also from an S0 with mass where X == 0."""
    import torch
    prob = workloads.plain_small(5)
    X, z = prob["X"], prob["z"]
    x, y = X.shape
    X = X.copy()
    X[: x // 2, :] = 0.0  # whole zero rows beside the model's scattered zeros
    X[x // 2 + 3, :] = 0.0
    rng = np.random.default_rng(4)
    S0 = rng.uniform(0.1, 1.0, (x, y, z))
    tt = torch.float64 if dtype_name == "F64" else torch.float32
    dt = getattr(bldm, dtype_name)
    out = []
    for skip in (False, True):
        plan = bldm.Plan(x, y, z, dt, skip_zero_rows=skip)
        assert plan.tuning()["skip_zero_rows"] == skip
        dS = torch.as_tensor(S0).to("cuda", tt)
        plan.run(torch.as_tensor(X).to("cuda", tt), dev(prob["alpha"]), dev(prob["beta"]), dS, 30,
                 bldm.PSI_APPR)
        plan.check()
        out.append(dS.cpu().numpy())
        plan.close()
    np.testing.assert_array_equal(out[0], out[1])
    assert not np.any(out[1][X == 0])


@pytest.mark.parametrize("dtype_name", ["F64", "F32"])
def test_bld_fact_matches_oracle(bldm, oracle, workloads, dtype_name):
    """bld_fact of a solved S on the device against the oracle's restatement
    (FP64 within 1e-12; FP32 storage within 1e-5 of the FP64 oracle)."""
    import torch
    prob = workloads.plain_small(7)
    X, z = prob["X"], prob["z"]
    x, y = X.shape
    params = bldm.Params(prob["a"], prob["b"], prob["alpha"], prob["beta"])
    S = bldm.bld_mult(X, z, params, 20, True, S0=oracle.init_S(X, z, 3))
    W0, H0, L0 = oracle.bld_fact(S, prob["alpha"], prob["beta"], prob["a"], prob["b"], 1e-50)
    if dtype_name == "F64":
        W, H, L = bldm.bld_fact(S, params)  # host FP64 path
        tol = 1e-12
    else:
        dS = torch.as_tensor(S).to("cuda", torch.float32)
        W, H, L = (t.double().cpu().numpy() for t in bldm.bld_fact(dS, params, dtype=bldm.F32))
        tol = 1e-5
    for a, b in ((W, W0), (H, H0), (L, L0)):
        assert np.abs(a - b).max() <= tol * np.abs(b).max()
    # device FP64 path on a larger shape with several row ranges and bands
    rng = np.random.default_rng(5)
    S2 = rng.gamma(0.3, 2.0, (300, 260, 16))
    a2, b2 = rng.uniform(1, 2, 300), rng.uniform(1, 2, 16)
    p2 = bldm.Params(3.0, 0.5, a2, b2)
    Wd, Hd, Ld = (t.cpu().numpy() for t in bldm.bld_fact(dev(S2), p2))
    Wr, Hr, Lr = oracle.bld_fact(S2, a2, b2, 3.0, 0.5, 1e-50)
    for a, b in ((Wd, Wr), (Hd, Hr), (Ld, Lr)):
        assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max()


def test_precision_study_crop_fp64_matches_oracle(bldm, oracle, workloads):
    """The FP64 GPU path is the reference for the FP32 precision study; it is
    validated here against the CPU oracle on a 256x256x32 crop of that
    workload (heavy-tailed counts, alpha, beta ~ U(0.5, 2)), all 300 iterations,
    within 1e-9 max-norm relative.  (A relative 1e-15 perturbation of S0 moves
    this crop, rows and columns 1024..1279, by 8.6e-12 after 300 iterations, so
    the bar is meaningful; other crops of this ill-conditioned workload amplify
    rounding up to 1e5-fold or reach NaN in the oracle itself.)"""
    p = workloads.precision_study(2)
    X = np.ascontiguousarray(p["X"][1024:1280, 1024:1280])
    z = p["z"]
    alpha = p["alpha"][1024:1280]
    oracle.set_threads(0)
    S0 = oracle.init_S(X, z, 1)
    ref = oracle.bld_mult(X, z, alpha, p["beta"], 300, oracle.PSI_APPR, 1e-50, S0=S0)
    params = bldm.Params(p["a"], p["b"], alpha, p["beta"])
    S = bldm.bld_mult(X, z, params, 300, True, S0=S0)
    assert rel_err(S, ref) <= 1e-9


@pytest.mark.parametrize("n_shards", [1, 3])
def test_row_sharded_solve_matches_plan(bldm, workloads, oracle, n_shards):
    """The row-sharded solve (bnmf_algs_b200.multi.sharded_solve over the plan's
    shard steps), emulated with several shards in one process on one GPU:
    one shard is bitwise the plan's solve; three shards agree to 1e-12 (the
    sums over rows are grouped by shard) and with the CPU oracle."""
    import torch
    import bnmf_algs_b200.multi as M
    prob = workloads.plain_small(9)
    X, z = prob["X"], prob["z"]
    x, y = X.shape
    S0 = oracle.init_S(X, z, 4)
    iters = 25
    full = bldm.Plan(x, y, z)
    dS_full = dev(S0)
    full.run(dev(X), dev(prob["alpha"]), dev(prob["beta"]), dS_full, iters, bldm.PSI_APPR)
    full.check()
    shards = []
    for i0, i1 in M.row_shards(x, n_shards):
        plan = bldm.Plan(i1 - i0, y, z)
        red = torch.empty(plan.shard_red_size(), dtype=torch.float64, device="cuda")
        shards.append(M.Shard(plan, dev(X[i0:i1]), dev(prob["alpha"][i0:i1]), dev(prob["beta"]),
                              dev(S0[i0:i1]), red))
    M.sharded_solve(shards, iters, bldm.PSI_APPR, 1e-50, M.local_allreduce)
    for sh in shards:
        sh.plan.check()
    S = np.concatenate([host(sh.dS) for sh in shards], axis=0)
    if n_shards == 1:
        np.testing.assert_array_equal(S, host(dS_full))
    else:
        assert rel_err(S, host(dS_full)) <= 1e-12
    ref = oracle.bld_mult(X, z, prob["alpha"], prob["beta"], iters, oracle.PSI_APPR, 1e-50, S0=S0)
    assert rel_err(S, ref) <= 1e-9
