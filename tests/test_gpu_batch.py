"""GPU tests of the batched solver (bldm_batch_*): many instances of different
shapes in shared launches.  Tolerances as in test_gpu_parity: FP64 within 1e-9
(max-norm relative) of the oracle; FP32 storage within 1e-5, or 10x the FP32
restatement's own error where that is larger.  An instance's result must not
depend on the batch it is solved in (bitwise)."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SHAPES = [(64, 48, 8), (33, 65, 3), (96, 80, 16), (130, 70, 8), (40, 41, 64), (7, 300, 5),
          (32, 32, 4), (200, 150, 32), (5, 7, 17), (70, 33, 4), (128, 256, 16), (48, 64, 64)]


def rel_err(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(np.abs(b).max(), 1e-300))


def _problems(workloads, oracle, shapes, seed0=0):
    out = []
    for k, (x, y, z) in enumerate(shapes):
        rng = np.random.default_rng(seed0 + k)
        X = workloads.allocation_model_X(x, y, z, 5.0, 0.05, rng) + rng.poisson(1.0, (x, y))
        alpha = rng.uniform(1.0, 2.0, x)
        beta = rng.uniform(1.0, 2.0, z)
        out.append((X, alpha, beta, oracle.init_S(X, z, seed0 + k)))
    return out


@pytest.mark.parametrize("use_graph", [True, False])
def test_batch_fp64_matches_oracle(bldm, oracle, workloads, use_graph):
    probs = _problems(workloads, oracle, SHAPES)
    b = bldm.Batch(SHAPES, dtype=bldm.F64)
    for k, (X, a, be, S0) in enumerate(probs):
        b.set(k, X, a, be, S0)
    import torch
    stream = torch.cuda.Stream()
    b.run(15, bldm.PSI_APPR, use_graph=use_graph, stream=stream)
    b.check(stream)
    for k, (X, a, be, S0) in enumerate(probs):
        ref = oracle.bld_mult(X, SHAPES[k][2], a, be, 15, oracle.PSI_APPR, 1e-50, S0=S0)
        S, _ = b.get(k)
        assert rel_err(S, ref) <= 1e-9, (SHAPES[k], rel_err(S, ref))
    info = b.info()
    assert info["classes"] >= 5
    b.close()


def test_batch_modes_exact_and_legacy(bldm, oracle, workloads):
    shapes = SHAPES[:4]
    probs = _problems(workloads, oracle, shapes, 100)
    for mode in (bldm.PSI_EXACT, bldm.PSI_LEGACY_CUDA):
        b = bldm.Batch(shapes, dtype=bldm.F64)
        for k, (X, a, be, S0) in enumerate(probs):
            b.set(k, X, a, be, S0)
        b.run(10, mode, use_graph=False)
        b.check()
        for k, (X, a, be, S0) in enumerate(probs):
            ref = oracle.bld_mult(X, shapes[k][2], a, be, 10, mode, 1e-50, S0=S0)
            assert rel_err(b.get(k)[0], ref) <= 1e-9
        b.close()


def test_instance_alone_equals_instance_in_mix(bldm, oracle, workloads):
    probs = _problems(workloads, oracle, SHAPES, 7)
    mix = bldm.Batch(SHAPES, dtype=bldm.F32)
    for k, (X, a, be, S0) in enumerate(probs):
        mix.set(k, X, a, be, S0)
    mix.run(20, use_graph=True, stream=None)
    mix.check()
    for k in (0, 4, 7, 11):
        alone = bldm.Batch([SHAPES[k]], dtype=bldm.F32)
        X, a, be, S0 = probs[k]
        alone.set(0, X, a, be, S0)
        alone.run(20, use_graph=False)
        alone.check()
        Sa, ra = alone.get(0)
        Sm, rm = mix.get(k)
        np.testing.assert_array_equal(Sa, Sm)
        assert ra == rm
        alone.close()
    mix.close()


def test_batch_fp32_vs_fp64(bldm, oracle, workloads):
    probs = _problems(workloads, oracle, SHAPES, 20)
    b = bldm.Batch(SHAPES, dtype=bldm.F32)
    for k, (X, a, be, S0) in enumerate(probs):
        b.set(k, X, a, be, S0)
    b.run(12, use_graph=False)
    b.check()
    for k, (X, a, be, S0) in enumerate(probs):
        z = SHAPES[k][2]
        ref = oracle.bld_mult(X, z, a, be, 12, oracle.PSI_APPR, 1e-50, S0=S0)
        ref32 = oracle.bld_mult(X, z, a, be, 12, oracle.PSI_APPR, 1e-50, S0=S0, dtype=np.float32)
        S, _ = b.get(k)
        assert np.all(np.isfinite(S))
        assert rel_err(S, ref) <= max(1e-5, 10 * rel_err(ref32, ref)), SHAPES[k]
    b.close()


def test_batch_relative_change(bldm, oracle, workloads):
    shapes = [(60, 50, 8), (30, 90, 16)]
    probs = _problems(workloads, oracle, shapes, 40)
    b = bldm.Batch(shapes, dtype=bldm.F64)
    for k, (X, a, be, S0) in enumerate(probs):
        b.set(k, X, a, be, S0)
    b.run(6, use_graph=False)
    b.check()
    for k, (X, a, be, S0) in enumerate(probs):
        s5 = oracle.bld_mult(X, shapes[k][2], a, be, 5, oracle.PSI_APPR, 1e-50, S0=S0)
        s6 = oracle.bld_mult(X, shapes[k][2], a, be, 6, oracle.PSI_APPR, 1e-50, S0=S0)
        ref = np.abs(s6 - s5).sum() / np.abs(s6).sum()
        S, rel = b.get(k)
        assert abs(rel - ref) <= 1e-9 * ref + 1e-15
    # a second run continues from the current S
    b.run(2, use_graph=False)
    b.check()
    s8 = oracle.bld_mult(probs[0][0], 8, probs[0][1], probs[0][2], 8, oracle.PSI_APPR, 1e-50,
                         S0=probs[0][3])
    assert rel_err(b.get(0)[0], s8) <= 1e-9
    b.close()


def test_batch_seeded_init_matches_oracle(bldm, oracle):
    rng = np.random.default_rng(3)
    X = rng.poisson(3.0, (20, 30)).astype(float)
    b = bldm.Batch([(20, 30, 6)], dtype=bldm.F64)
    b.set(0, X, np.ones(20), np.ones(6), None, seed=99)
    b.run(3, use_graph=False)
    ref = oracle.bld_mult(X, 6, np.ones(20), np.ones(6), 3, oracle.PSI_APPR, 1e-50,
                          S0=oracle.init_S(X, 6, 99))
    assert rel_err(b.get(0)[0], ref) <= 1e-9
    b.close()


def test_batch_rejects_bad_input(bldm):
    b = bldm.Batch([(4, 5, 3)], dtype=bldm.F64)
    X = np.ones((4, 5))
    X[0, 0] = -1
    with pytest.raises(ValueError):
        b.set(0, X, np.ones(4), np.ones(3))
    with pytest.raises(ValueError):
        b.set(3, np.ones((4, 5)), np.ones(4), np.ones(3))
    b.close()


def test_autotune_keeps_solution_and_reports_classes(bldm, oracle, workloads):
    """The autotuner times probe runs but restores S: the tuned batch then
    solves to the same tolerance, and every class reports a legal shape."""
    probs = _problems(workloads, oracle, SHAPES, 60)
    b = bldm.Batch(SHAPES, dtype=bldm.F64)
    for k, (X, a, be, S0) in enumerate(probs):
        b.set(k, X, a, be, S0)
    before = [b.get(k)[0] for k in range(len(SHAPES))]
    d_ms, t_ms = b.autotune(probe_iters=2)
    assert d_ms > 0 and 0 < t_ms <= d_ms
    for k in range(len(SHAPES)):
        np.testing.assert_array_equal(b.get(k)[0], before[k])
    cls = b.classes()
    assert sum(c["instances"] for c in cls) == len(SHAPES)
    for c in cls:
        assert c["rows_per_tile"] >= 32 and c["stages"] >= 2 and c["tiles"] >= 1
    b.run(10, use_graph=False)
    b.check()
    for k, (X, a, be, S0) in enumerate(probs):
        ref = oracle.bld_mult(X, SHAPES[k][2], a, be, 10, oracle.PSI_APPR, 1e-50, S0=S0)
        assert rel_err(b.get(k)[0], ref) <= 1e-9, SHAPES[k]
    b.close()


def test_class_shape_applies_alone_and_in_mix(bldm, oracle, workloads):
    """With the same class launch shapes an instance gives bitwise the same
    result alone and in a mix; a tile height below 32 is rejected."""
    probs = _problems(workloads, oracle, SHAPES, 80)
    mix = bldm.Batch(SHAPES, dtype=bldm.F32)
    for k, (X, a, be, S0) in enumerate(probs):
        mix.set(k, X, a, be, S0)
    shapes = []
    for c in mix.classes():
        c = dict(c, rows_per_tile=32, stages=2)
        mix.set_class(c)
        shapes.append(c)
    with pytest.raises(ValueError):
        mix.set_class(dict(shapes[0], rows_per_tile=16))
    mix.run(8, use_graph=True, stream=None)
    mix.check()
    for k in (3, 7):
        alone = bldm.Batch([SHAPES[k]], dtype=bldm.F32)
        X, a, be, S0 = probs[k]
        alone.set(0, X, a, be, S0)
        for c in shapes:
            alone.set_class(c)
        alone.run(8, use_graph=False)
        alone.check()
        np.testing.assert_array_equal(alone.get(0)[0], mix.get(k)[0])
        alone.close()
    mix.close()


def test_batch_zero_rows_from_dirty_S0(bldm, oracle, workloads):
    """The engine skips rows whose band segment of X is all zero once they
    hold zeros; an S0 with mass where X == 0 is still zeroed by the first
    update, the tracked change of a one-iteration run counts that mass, and
    later runs (which skip from their first update) stay on the oracle."""
    shapes = [(64, 40, 8), (50, 70, 16)]
    probs = []
    for k, (x, y, z) in enumerate(shapes):
        rng = np.random.default_rng(90 + k)
        X = workloads.allocation_model_X(x, y, z, 5.0, 0.05, rng)
        X[::3, :] = 0.0
        probs.append((X, rng.uniform(1.0, 2.0, x), rng.uniform(1.0, 2.0, z),
                      rng.uniform(0.1, 1.0, (x, y, z))))
    b = bldm.Batch(shapes, dtype=bldm.F64)
    for k, (X, a, be, S0) in enumerate(probs):
        b.set(k, X, a, be, S0)
    b.run(1, use_graph=False)
    b.check()
    for k, (X, a, be, S0) in enumerate(probs):
        s1 = oracle.bld_mult(X, shapes[k][2], a, be, 1, oracle.PSI_APPR, 1e-50, S0=S0)
        S, rel = b.get(k)
        assert rel_err(S, s1) <= 1e-9
        ref = np.abs(s1 - S0).sum() / np.abs(s1).sum()
        assert abs(rel - ref) <= 1e-9 * ref
    import torch
    stream = torch.cuda.Stream()
    b.run(9, use_graph=True, stream=stream)
    b.check(stream)
    for k, (X, a, be, S0) in enumerate(probs):
        s10 = oracle.bld_mult(X, shapes[k][2], a, be, 10, oracle.PSI_APPR, 1e-50, S0=S0)
        S, rel = b.get(k)
        assert rel_err(S, s10) <= 1e-9
        s9 = oracle.bld_mult(X, shapes[k][2], a, be, 9, oracle.PSI_APPR, 1e-50, S0=S0)
        ref = np.abs(s10 - s9).sum() / np.abs(s10).sum()
        assert abs(rel - ref) <= 1e-9 * ref + 1e-15
    b.close()


@pytest.fixture(scope="module")
def benchmarked_batch(workloads, oracle):
    """The 512-instance uneven batch the benchmark runs (x, y log-uniform in
    [32, 512], z in {4, 8, 16, 32, 64}, 150 iterations), with a seeded sample
    of 16 instances whose initial S is the oracle's and whose 150-iteration
    oracle solutions (FP64, psi_appr) are computed once here."""
    shapes = workloads.batch_shapes(512, 3)
    probs = [workloads.batch_instance(s, 1000 + 3 * 100003 + k) for k, s in enumerate(shapes)]
    sample = sorted(np.random.default_rng(2024).choice(len(shapes), 16, replace=False).tolist())
    oracle.set_threads(0)
    ref = {}
    for k in sample:
        pr = probs[k]
        S0 = oracle.init_S(pr["X"], pr["z"], k)
        S = oracle.bld_mult(pr["X"], pr["z"], pr["alpha"], pr["beta"], 150, oracle.PSI_APPR,
                            1e-50, S0=S0)
        ref[k] = (S0, S, oracle.log_marginal_S(S, pr["alpha"], pr["beta"], pr["a"], pr["b"]))
    return shapes, probs, sample, ref


def _run_benchmarked(bldm, shapes, probs, ref, dtype, persistent=False):
    import torch
    b = bldm.Batch(shapes, dtype=dtype)
    b.set_launch_mode(persistent)
    for k, pr in enumerate(probs):
        S0 = ref[k][0] if k in ref else None
        b.set(k, pr["X"], pr["alpha"], pr["beta"], S0, seed=k)
    stream = torch.cuda.Stream()
    b.autotune(probe_iters=3, stream=stream)
    b.run(150, bldm.PSI_APPR, 1e-50, True, stream)
    b.check(stream)
    return b


@pytest.mark.parametrize("persistent", [False, True])
def test_benchmarked_batch_sample_fp64_matches_oracle(bldm, oracle, benchmarked_batch, persistent):
    shapes, probs, sample, ref = benchmarked_batch
    b = _run_benchmarked(bldm, shapes, probs, ref, bldm.F64, persistent)
    assert b.persistent() == persistent
    cons = b.conservation()
    for k in sample:
        S, _ = b.get(k)
        assert rel_err(S, ref[k][1]) <= 1e-9, (k, shapes[k], rel_err(S, ref[k][1]))
        X = probs[k]["X"]
        want = float((np.abs(S.sum(axis=2) - X) / np.maximum(X, 1.0)).max())
        assert abs(cons[k] - want) <= 1e-12 * max(want, 1.0)
    b.close()


def test_benchmarked_batch_sample_fp32_log_marginal(bldm, oracle, benchmarked_batch):
    shapes, probs, sample, ref = benchmarked_batch
    b = _run_benchmarked(bldm, shapes, probs, ref, bldm.F32)
    for k in sample:
        pr = probs[k]
        S, _ = b.get(k)
        assert np.all(np.isfinite(S))
        lm = oracle.log_marginal_S(S.astype(np.float32), pr["alpha"], pr["beta"], pr["a"],
                                   pr["b"])
        assert abs(lm - ref[k][2]) <= 1e-5 * abs(ref[k][2]), (k, shapes[k], lm, ref[k][2])
    b.close()


def test_persistent_launch_matches_per_iteration_launches(bldm, oracle, workloads):
    """The persistent form (one launch per class for the whole run, each
    instance advancing through its own dependencies, the finalize in the tiles'
    epilogues) against the per-iteration form (a sweep launch per class and a
    finalize launch per iteration): each bitwise the same with and without the
    CUDA graph, the two within 1e-12 of each other in FP64 (they group the sum
    of alpha_eph over rows differently), over two consecutive runs (the second
    continues from the first's S and digamma tables)."""
    import torch
    probs = _problems(workloads, oracle, SHAPES, 61)
    out = {}
    for persistent in (True, False):
        for use_graph in (True, False):
            b = bldm.Batch(SHAPES, dtype=bldm.F64)
            b.set_launch_mode(persistent)
            assert b.persistent() == persistent
            for k, (X, a, be, S0) in enumerate(probs):
                b.set(k, X, a, be, S0)
            stream = torch.cuda.Stream()
            l0 = b.info()["launches"]
            b.run(9, use_graph=use_graph, stream=stream)
            b.run(4, use_graph=use_graph, stream=stream)
            b.check(stream)
            n_cls = b.info()["classes"]
            if persistent:
                assert b.info()["launches"] - l0 == 2 * n_cls  # one launch per class per run
            else:
                # a sweep and a finalize launch per class and iteration (prime included)
                assert b.info()["launches"] - l0 == (10 + 5) * 2 * n_cls
            out[(persistent, use_graph)] = [b.get(k) for k in range(len(SHAPES))]
            b.close()
    for persistent in (True, False):
        for (S, r), (S0, r0) in zip(out[(persistent, True)], out[(persistent, False)]):
            np.testing.assert_array_equal(S, S0)
            assert r == r0
    for k, ((S, r), (S0, r0)) in enumerate(zip(out[(True, False)], out[(False, False)])):
        assert rel_err(S, S0) <= 1e-12, (k, rel_err(S, S0))
        assert abs(r - r0) <= 1e-9 * abs(r0)
    # and both against the oracle
    for k, (X, a, be, S0) in enumerate(probs):
        ref = oracle.bld_mult(X, SHAPES[k][2], a, be, 13, oracle.PSI_APPR, 1e-50, S0=S0)
        assert rel_err(out[(True, True)][k][0], ref) <= 1e-9


def test_persistent_fp64_all_modes(bldm, oracle, workloads):
    probs = _problems(workloads, oracle, SHAPES[:6], 71)
    for mode in (0, 1, 2):
        b = bldm.Batch(SHAPES[:6], dtype=bldm.F64)
        b.set_launch_mode(True)
        assert b.persistent()
        for k, (X, a, be, S0) in enumerate(probs):
            b.set(k, X, a, be, S0)
        b.run(8, mode, use_graph=False)
        b.check()
        for k, (X, a, be, S0) in enumerate(probs):
            ref = oracle.bld_mult(X, SHAPES[k][2], a, be, 8, mode, 1e-50, S0=S0)
            assert rel_err(b.get(k)[0], ref) <= 1e-9, (mode, SHAPES[k])
        b.close()


def test_long_fiber_class_keeps_per_iteration_launches(bldm, oracle, workloads):
    shapes = [(20, 30, 300), (30, 20, 8)]  # z = 300 in FP32: four chunks per lane
    probs = _problems(workloads, oracle, shapes, 81)
    b = bldm.Batch(shapes, dtype=bldm.F32)
    b.set_launch_mode(True)
    assert not b.persistent()
    for k, (X, a, be, S0) in enumerate(probs):
        b.set(k, X, a, be, S0)
    b.run(5, use_graph=False)
    b.check()
    b.close()


def test_persistent_wait_runs_out_and_reports_timeout(bldm, oracle, workloads):
    """Failure detection without a GPU fault: with the test hook, instance 0's
    first-iteration tiles wait for the completion of that same iteration;
    the bounded wait (50 ms) runs out, the launch stops taking work and the
    host sees BLDM_ERR_TIMEOUT.  The context stays usable: the same batch then
    runs normally and matches the oracle."""
    import torch
    probs = _problems(workloads, oracle, SHAPES[:4], 91)
    b = bldm.Batch(SHAPES[:4], dtype=bldm.F64)
    for k, (X, a, be, S0) in enumerate(probs):
        b.set(k, X, a, be, S0)
    b.set_launch_mode(True, wait_limit_s=0.05, stall_test=True)
    stream = torch.cuda.Stream()
    b.run(3, use_graph=False, stream=stream)
    with pytest.raises(bldm.BldmError) as ei:
        b.check(stream)
    assert ei.value.status == bldm.ERR_TIMEOUT
    # the error is reported once and cleared; a normal run from fresh S0 works
    b.set_launch_mode(True, wait_limit_s=1.0, stall_test=False)
    for k, (X, a, be, S0) in enumerate(probs):
        b.set(k, X, a, be, S0)
    b.run(6, use_graph=False, stream=stream)
    b.check(stream)
    for k, (X, a, be, S0) in enumerate(probs):
        ref = oracle.bld_mult(X, SHAPES[k][2], a, be, 6, oracle.PSI_APPR, 1e-50, S0=S0)
        assert rel_err(b.get(k)[0], ref) <= 1e-9
    b.close()


def test_tile_order_follows_x_and_changes_no_result(bldm, oracle, workloads):
    """The engine orders a class's tiles by the work its X implies (rows with a
    nonzero, nonzero passes), not by bytes.  Instances of very different
    densities in forward and reversed order, and a batch re-sorted after one
    instance's X is set again, give every instance bitwise the same S as a
    batch set up with the final X from the start."""
    shapes = [(96, 130, 64), (64, 200, 64), (150, 90, 64), (40, 260, 64), (120, 120, 64)]
    probs = []
    for k, (x, y, z) in enumerate(shapes):
        rng = np.random.default_rng(50 + k)
        if k % 2 == 0:
            X = 1.0 + rng.poisson(10.0, (x, y)).astype(float)  # every fiber works
        else:
            X = workloads.allocation_model_X(x, y, z, 5.0, 0.05, rng)  # mostly zeros
        probs.append((X, rng.uniform(1.0, 2.0, x), rng.uniform(1.0, 2.0, z),
                      oracle.init_S(X, z, 50 + k)))

    def solve(order, iters=12):
        b = bldm.Batch([shapes[k] for k in order], dtype=bldm.F32)
        for i, k in enumerate(order):
            X, a, be, S0 = probs[k]
            b.set(i, X, a, be, S0)
        b.run(iters, use_graph=True)
        b.check()
        out = {k: b.get(i)[0] for i, k in enumerate(order)}
        return b, out

    fwd, S_fwd = solve(list(range(len(shapes))))
    rev, S_rev = solve(list(reversed(range(len(shapes)))))
    rev.close()
    for k in range(len(shapes)):
        np.testing.assert_array_equal(S_fwd[k], S_rev[k])
    # instance 1 becomes dense: the next run re-sorts the tiles
    x, y, z = shapes[1]
    X1 = 1.0 + np.random.default_rng(99).poisson(10.0, (x, y)).astype(float)
    probs[1] = (X1, probs[1][1], probs[1][2], oracle.init_S(X1, z, 99))
    for k in range(len(shapes)):
        X, a, be, S0 = probs[k]
        fwd.set(k, X, a, be, S0)
    fwd.run(12, use_graph=True)
    fwd.check()
    fresh, S_fresh = solve(list(range(len(shapes))))
    fresh.close()
    for k in range(len(shapes)):
        np.testing.assert_array_equal(fwd.get(k)[0], S_fresh[k])
    # and the FP32 solve of the dense instance keeps this file's FP32 bound
    ref = oracle.bld_mult(X1, z, probs[1][1], probs[1][2], 12, oracle.PSI_APPR, 1e-50,
                          S0=probs[1][3])
    ref32 = oracle.bld_mult(X1, z, probs[1][1], probs[1][2], 12, oracle.PSI_APPR, 1e-50,
                            S0=probs[1][3], dtype=np.float32)
    assert rel_err(S_fresh[1], ref) <= max(1e-5, 10 * rel_err(ref32, ref))
    fwd.close()
