"""bldm_solve_device_noalloc: the allocation-free solve.

It serves callers that cannot allocate device memory while they solve (a
serving loop that must not let cudaMalloc/cudaFree synchronise the device, a
process whose HBM another allocator already holds).  Its scratch is a fixed
32 MiB array in the library's device data.  This test calls it through the C
ABI on device buffers that the test itself allocates, three times in a row
with different inputs (the array keeps the previous call's contents; the third
shape has fibers longer than the fused sweep's lane layout), and compares each
result with the plan API's (bldm_plan_run) at the solver tests' tolerance
(1e-9 max-norm relative for FP64, 1e-5 for FP32).  This file is
named so that pytest collects it last.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _problem(workloads, oracle, seed, x, y, z):
    rng = np.random.default_rng(seed)
    X = workloads.allocation_model_X(x, y, z, 5.0, 0.02, rng) + rng.poisson(2.0, (x, y))
    S0 = oracle.init_S(X, z, seed)
    return X, S0


def _noalloc(bldm, dX, da, db, dS, dtype, iters):
    x, y, z = dS.shape
    stream = torch.cuda.current_stream().cuda_stream
    p = lambda t: ctypes.c_void_p(t.data_ptr())
    return bldm.lib().bldm_solve_device_noalloc(p(dX), p(da), p(db), p(dS), x, y, z, dtype,
                                                iters, bldm.PSI_APPR, 1e-50,
                                                ctypes.c_void_p(stream))


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


@pytest.mark.parametrize("dtype,tol", [(0, 1e-9), (1, 1e-5)])
def test_noalloc_matches_plan_api_twice(bldm, workloads, oracle, dtype, tol):
    tt = torch.float64 if dtype == bldm.F64 else torch.float32
    for call, (seed, x, y, z, iters) in enumerate([(1, 96, 80, 16, 30), (2, 130, 70, 8, 25),
                                                   (3, 20, 12, 1300, 6)]):
        X, S0 = _problem(workloads, oracle, seed, x, y, z)
        dX = torch.as_tensor(X).to("cuda", tt)
        da = torch.ones(x, dtype=torch.float64, device="cuda")
        db = torch.ones(z, dtype=torch.float64, device="cuda")
        dS_ref = torch.as_tensor(S0).to("cuda", tt)
        plan = bldm.Plan(x, y, z, dtype)
        plan.run(dX, da, db, dS_ref, iters, bldm.PSI_APPR)
        plan.check()
        plan.close()
        dS = torch.as_tensor(S0).to("cuda", tt)
        rc = _noalloc(bldm, dX, da, db, dS, dtype, iters)
        assert rc == bldm.OK, (call, rc)
        got = dS.cpu().numpy().astype(np.float64)
        ref = dS_ref.cpu().numpy().astype(np.float64)
        assert _rel(got, ref) <= tol, (call, _rel(got, ref))


@pytest.mark.parametrize("dtype", [0, 1])
def test_noalloc_rejects_shapes_beyond_its_scratch(bldm, dtype):
    # 4096 x 4096 x 64 needs far more than the fixed 32 MiB scratch in either
    # storage type; the size check happens before any device work touches the
    # buffers.
    d = torch.zeros(16, dtype=torch.float64, device="cuda")
    p = ctypes.c_void_p(d.data_ptr())
    rc = bldm.lib().bldm_solve_device_noalloc(p, p, p, p, 4096, 4096, 64, dtype, 5,
                                              bldm.PSI_APPR, 1e-50, None)
    assert rc == bldm.ERR_TOO_LARGE


def test_noalloc_accepts_the_documented_fit(bldm):
    # 1024 x 1024 x 64 in FP64 needs 22.5 MB of scratch and fits.  With
    # max_iter = 0 the call sets up its scratch and returns without touching
    # the (deliberately small) buffers.
    d = torch.zeros(16, dtype=torch.float64, device="cuda")
    p = ctypes.c_void_p(d.data_ptr())
    rc = bldm.lib().bldm_solve_device_noalloc(p, p, p, p, 1024, 1024, 64, bldm.F64, 0,
                                              bldm.PSI_APPR, 1e-50, None)
    assert rc == bldm.OK
