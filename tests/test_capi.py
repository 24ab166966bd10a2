"""CPU tests of the C ABI: the library loads, exports every symbol include/bldm.h
declares, and rejects bad arguments before touching a device (the reference's
parameter checks, test/bld/bld_mult/test_bld_mult.cpp:10-31)."""

import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT


def header_symbols():
    text = open(os.path.join(ROOT, "include", "bldm.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(bldm_[A-Za-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol(bldm):
    lib = ctypes.CDLL(bldm.LIB_PATH)
    syms = header_symbols()
    assert len(syms) >= 20
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing
    # the Python binding declares exactly the header's entry points
    assert sorted(bldm.SIGNATURES) == syms


def test_version_string(bldm):
    assert "sm_100a" in bldm.version()


def _params(bldm, x, z):
    return bldm.Params(1.0, 10.0, np.ones(x), np.ones(z))


def test_negative_X_rejected(bldm):
    X = np.full((10, 5), 5.0)
    X[0, 0] = -5
    with pytest.raises(ValueError) as e:
        bldm.bld_mult_cuda(X, 2, _params(bldm, 10, 2), 5)
    assert e.value.status == bldm.ERR_NEG_X


def test_nan_X_rejected(bldm):
    X = np.full((10, 5), 5.0)
    X[3, 2] = np.nan
    with pytest.raises(ValueError):
        bldm.bld_mult(X, 2, _params(bldm, 10, 2), 5)


def test_wrong_z_rejected(bldm):
    X = np.full((10, 5), 5.0)
    with pytest.raises(ValueError) as e:
        bldm.bld_mult_cuda(X, 3, _params(bldm, 10, 2))
    assert e.value.status == bldm.ERR_BAD_ARG


def test_wrong_x_rejected(bldm):
    X = np.full((11, 5), 5.0)
    with pytest.raises(ValueError):
        bldm.bld_mult_cuda(X, 2, _params(bldm, 10, 2))


def test_fp32_checks_match(bldm):
    X = np.full((10, 5), 5.0)
    X[9, 4] = -1
    with pytest.raises(ValueError):
        bldm.bld_mult_cuda(X, 2, _params(bldm, 10, 2), 5, dtype=bldm.F32)


def test_bad_psi_mode_and_null_params(bldm):
    L = bldm.lib()
    X = np.ones((2, 2))
    out = np.empty((2, 2, 2))
    dp = ctypes.POINTER(ctypes.c_double)
    rc = L.bldm_solve_f64(X.ctypes.data_as(dp), 2, 2, 2, None, 1, 1, 1e-50, None, 0,
                          out.ctypes.data_as(dp), None)
    assert rc == bldm.ERR_BAD_ARG
    p = _params(bldm, 2, 2).c_struct()
    rc = L.bldm_solve_f64(X.ctypes.data_as(dp), 2, 2, 2, ctypes.byref(p), 1, 7, 1e-50, None, 0,
                          out.ctypes.data_as(dp), None)
    assert rc == bldm.ERR_BAD_ARG


def test_empty_problem_is_a_no_op(bldm):
    S = bldm.bld_mult_cuda(np.zeros((0, 4)), 3, bldm.Params(1, 1, np.ones(0), np.ones(3)), 5)
    assert S.shape == (0, 4, 3)


def test_params_default_ctor(bldm):
    p = bldm.Params.from_shape((4, 5, 6))
    assert (p.a, p.b) == (1.0, 10.0)
    assert p.alpha.shape == (4,) and p.beta.shape == (6,)
    assert np.all(p.alpha == 1) and np.all(p.beta == 1)


def test_plan_api_argument_checks(bldm):
    L = bldm.lib()
    h = ctypes.c_void_p()
    assert L.bldm_plan_create(None, 4, 4, 4, 0) == bldm.ERR_BAD_ARG
    assert L.bldm_plan_destroy(None) == bldm.ERR_BAD_ARG
    n = ctypes.c_size_t()
    assert L.bldm_plan_workspace_bytes(None, ctypes.byref(n)) == bldm.ERR_BAD_ARG
    assert L.bldm_plan_run(None, None, None, None, None, 1, 1, 1e-50, None) == bldm.ERR_BAD_ARG
    del h


def test_workloads_are_deterministic(workloads):
    a = workloads.plain_small(0)
    b = workloads.plain_small(0)
    np.testing.assert_array_equal(a["X"], b["X"])
    assert a["X"].shape == (64, 48) and a["z"] == 8 and a["iters"] == 200
    shapes = workloads.batch_shapes(512, 3)
    assert len(shapes) == 512
    assert all(32 <= x <= 512 and 32 <= y <= 512 and z in (4, 8, 16, 32, 64) for x, y, z in shapes)
    p = workloads.precision_study(2, x=256, y=256)
    assert 0.27 < np.mean(p["X"] == 0) < 0.33  # ~30% zeros in total
