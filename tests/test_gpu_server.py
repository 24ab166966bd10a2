"""GPU tests of the serving loop (bldm_server_*): continuous batching with
device-resident state, convergence retirement, memory admission, and the
property that a request's result is the same alone and in a mix."""

import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _req(workloads, shape, seed):
    x, y, z = shape
    rng = np.random.default_rng(seed)
    X = workloads.allocation_model_X(x, y, z, 5.0, 0.05, rng) + rng.poisson(0.5, (x, y))
    return X, z


SHAPES = [(64, 48, 8), (33, 65, 3), (96, 80, 16), (130, 70, 8), (40, 41, 64), (32, 32, 4)]


def _params(bldm, x, z):
    return bldm.Params(5.0, 0.1, np.ones(x), np.ones(z))


@pytest.mark.parametrize("target,seed", [(2, 5), (0, 17), (4, 23), (5, 31)])
def test_alone_equals_in_mix(bldm, workloads, target, seed):
    """A request's result is bitwise the same served alone and in a mix whose
    other requests arrive while it is on the GPU (a handful of seeds)."""
    reqs = [_req(workloads, s, 10 + k + seed) for k, s in enumerate(SHAPES)]
    alone = bldm.Server(dtype=bldm.F32, tol=1e-5, max_iter=200, iters_per_round=10)
    X, z = reqs[target]
    rid = alone.submit(X, z, _params(bldm, X.shape[0], z), seed=seed)
    assert alone.wait(rid)
    S_alone, st_alone = alone.fetch(rid)
    alone.close()
    mix = bldm.Server(dtype=bldm.F32, tol=1e-5, max_iter=200, iters_per_round=10)
    ids = {}
    for k, (X, z) in enumerate(reqs):
        ids[k] = mix.submit(X, z, _params(bldm, X.shape[0], z), seed=seed if k == target else k)
        if k == 1:
            time.sleep(0.05)  # later requests arrive while others are on the GPU
    for rid in ids.values():
        assert mix.wait(rid)
    S_mix, st_mix = mix.fetch(ids[target])
    for k, rid in ids.items():
        if k != target:
            S, st = mix.fetch(rid)
            assert S is not None and st["status"] == 0
    assert st_mix["iterations"] == st_alone["iterations"]
    np.testing.assert_array_equal(S_mix, S_alone)
    assert st_mix["log_marginal"] == st_alone["log_marginal"]
    mix.close()


def test_two_lanes_match_one_lane(bldm, workloads):
    """With a small large_elements the mix is split over both lanes (their own
    workers and streams, running concurrently); every request's result is
    bitwise the one of a single-lane server, and the large lane ran rounds."""
    reqs = [_req(workloads, s, 40 + k) for k, s in enumerate(SHAPES)]
    results = {}
    for lanes, large in (("one", 2**64 - 1), ("two", 40000)):
        srv = bldm.Server(dtype=bldm.F32, tol=1e-5, max_iter=200, iters_per_round=10,
                          large_elements=large)
        ids = [srv.submit(X, z, _params(bldm, X.shape[0], z), seed=k)
               for k, (X, z) in enumerate(reqs)]
        for rid in ids:
            assert srv.wait(rid)
        results[lanes] = [srv.fetch(rid) for rid in ids]
        st = srv.stats()
        if lanes == "two":
            assert st["gpu_ms_large"] > 0.0
        else:
            assert st["gpu_ms_large"] == 0.0
        srv.close()
    for (S1, st1), (S2, st2) in zip(results["one"], results["two"]):
        assert st1["status"] == 0 and st2["status"] == 0
        assert st1["iterations"] == st2["iterations"]
        np.testing.assert_array_equal(S1, S2)
    # both lanes had requests
    assert {x * y * z >= 40000 for x, y, z in SHAPES} == {False, True}


def test_server_fp64_matches_oracle_and_stops(bldm, workloads, oracle):
    srv = bldm.Server(dtype=bldm.F64, tol=1e-12, max_iter=30, iters_per_round=10)
    X, z = _req(workloads, (50, 60, 8), 3)
    p = _params(bldm, 50, z)
    rid = srv.submit(X, z, p, seed=11)
    assert srv.wait(rid)
    S, st = srv.fetch(rid)
    assert st["status"] == 0 and st["iterations"] == 30
    ref = oracle.bld_mult(X, z, p.alpha, p.beta, 30, oracle.PSI_APPR, 1e-50,
                          S0=oracle.init_S(X, z, 11))
    assert np.abs(S - ref).max() / np.abs(ref).max() <= 1e-9
    lm = oracle.log_marginal_S(S, p.alpha, p.beta, p.a, p.b)
    assert abs(st["log_marginal"] - lm) <= 1e-10 * abs(lm)
    # row-sum conservation residual computed on the device at retirement
    cons = float((np.abs(S.sum(axis=2) - X) / np.maximum(X, 1.0)).max())
    assert abs(st["conservation_residual"] - cons) <= 1e-12 * max(cons, 1.0)
    srv.close()


def test_converged_requests_retire_early(bldm, workloads):
    srv = bldm.Server(dtype=bldm.F64, tol=1e-3, max_iter=500, iters_per_round=10)
    X, z = _req(workloads, (40, 30, 4), 4)
    rid = srv.submit(X, z, _params(bldm, 40, z))
    assert srv.wait(rid)
    S, st = srv.fetch(rid)
    assert st["rel_change"] < 1e-3 and st["iterations"] < 500
    assert st["iterations"] % 10 == 0
    srv.close()


def test_memory_budget_bounds_concurrency(bldm, workloads):
    shapes = [(128, 128, 16)] * 6
    probe = bldm.Batch([shapes[0]], dtype=bldm.F32)
    one = probe.info()["device_bytes"]
    probe.close()
    srv = bldm.Server(dtype=bldm.F32, tol=0.0, max_iter=40, iters_per_round=10,
                      memory_budget=int(2.5 * one))
    ids = [srv.submit(*_req(workloads, s, 20 + k), _params(bldm, s[0], s[2]))
           for k, s in enumerate(shapes)]
    for rid in ids:
        assert srv.wait(rid)
        S, st = srv.fetch(rid)
        assert S is not None and st["iterations"] == 40
    stats = srv.stats()
    assert stats["completed"] == 6
    assert stats["bytes_peak"] <= stats["budget"]
    srv.close()


def test_bad_requests(bldm, workloads):
    srv = bldm.Server(dtype=bldm.F32, memory_budget=64 << 20)
    X = np.ones((10, 12))
    X[1, 1] = -1
    with pytest.raises(ValueError):
        srv.submit(X, 3, _params(bldm, 10, 3))
    with pytest.raises(ValueError):
        srv.submit(np.ones((10, 12)), 3, _params(bldm, 9, 3))
    with pytest.raises(bldm.BldmError) as e:
        srv.submit(np.ones((2048, 2048)), 64, _params(bldm, 2048, 64))
    assert e.value.status == bldm.ERR_TOO_LARGE
    srv.close()


def test_cancel(bldm, workloads):
    srv = bldm.Server(dtype=bldm.F32, tol=0.0, max_iter=100000, iters_per_round=10)
    X, z = _req(workloads, (64, 64, 8), 9)
    rid = srv.submit(X, z, _params(bldm, 64, z))
    time.sleep(0.2)
    srv.cancel(rid)
    assert srv.wait(rid, 30.0)
    S, st = srv.fetch(rid)
    assert S is None and st["status"] == bldm.ERR_NOT_FOUND
    srv.close()


def test_fp32_served_log_marginal_vs_fp64_oracle(bldm, workloads, oracle):
    """FP32 storage (Kahan axis sums) served to a fixed iteration count: the
    device FP64 log-marginal of the result is within 1e-5 relative of the CPU
    oracle's FP64 solve of the same request."""
    srv = bldm.Server(dtype=bldm.F32, tol=0.0, max_iter=60, iters_per_round=20)
    cases = []
    for k, shape in enumerate([(64, 48, 8), (96, 80, 16), (40, 41, 64)]):
        X, z = _req(workloads, shape, 50 + k)
        p = _params(bldm, X.shape[0], z)
        cases.append((srv.submit(X, z, p, seed=k), X, z, p, k))
    for rid, X, z, p, k in cases:
        assert srv.wait(rid)
        S, st = srv.fetch(rid)
        assert st["status"] == 0 and st["iterations"] == 60
        ref = oracle.bld_mult(X, z, p.alpha, p.beta, 60, oracle.PSI_APPR, 1e-50,
                              S0=oracle.init_S(X, z, k))
        lm = oracle.log_marginal_S(ref, p.alpha, p.beta, p.a, p.b)
        assert abs(st["log_marginal"] - lm) <= 1e-5 * abs(lm)
    srv.close()
