"""TEST INFRASTRUCTURE ONLY: numpy bindings for the CPU oracle (liboracle.so).

The oracle restates eozd/bnmf-algs' bld_mult path on the CPU (see
bld_oracle.cpp for the reference file:line of every function).  Only tests/,
the smoke check and bench.py's CPU-baseline leg import this module; the
product library never does.
"""

import ctypes
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")

PSI_EXACT = 0
PSI_APPR = 1
PSI_LEGACY_CUDA = 2

_lib = None


def build():
    """Compile liboracle.so with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = ctypes.CDLL(_LIB_PATH)
        _declare(_lib)
    return _lib


_dp = ctypes.POINTER(ctypes.c_double)
_fp = ctypes.POINTER(ctypes.c_float)
_sz = ctypes.c_size_t


def _declare(L):
    L.oracle_set_threads.argtypes = [ctypes.c_int]
    L.oracle_set_threads.restype = ctypes.c_int
    L.oracle_psi_appr_f64.argtypes = [ctypes.c_double]
    L.oracle_psi_appr_f64.restype = ctypes.c_double
    L.oracle_psi_appr_f32.argtypes = [ctypes.c_float]
    L.oracle_psi_appr_f32.restype = ctypes.c_float
    L.oracle_psi_exact.argtypes = [ctypes.c_double]
    L.oracle_psi_exact.restype = ctypes.c_double
    L.oracle_psi_array.argtypes = [_dp, _sz, ctypes.c_int, _dp]
    L.oracle_tensor_sums_f64.argtypes = [_dp, _sz, _sz, _sz, _dp, _dp, _dp]
    L.oracle_tensor_sums_f32.argtypes = [_fp, _sz, _sz, _sz, _fp, _fp, _fp]
    L.oracle_x_reciprocal_f64.argtypes = [_dp, _sz, _sz, ctypes.c_double, _dp]
    L.oracle_update_alpha_eph_f64.argtypes = [_dp, _dp, _sz, _sz, _dp]
    L.oracle_update_beta_eph_f64.argtypes = [_dp, _dp, _sz, _sz, _dp]
    L.oracle_update_grad_plus_f64.argtypes = [_dp, _dp, _sz, _sz, _sz, ctypes.c_int, _dp]
    L.oracle_update_grad_minus_f64.argtypes = [_dp, _sz, _sz, ctypes.c_int, _dp]
    L.oracle_update_nom_f64.argtypes = [_dp, _dp, _dp, _sz, _sz, _sz, _dp]
    L.oracle_update_denom_f64.argtypes = [_dp, _dp, _dp, _sz, _sz, _sz, _dp]
    L.oracle_update_S_f64.argtypes = [_dp, _dp, _dp, _dp, _dp, _dp, _sz, _sz, _sz,
                                      ctypes.c_double, _dp]
    L.oracle_bld_mult_f64.argtypes = [_dp, _sz, _sz, _sz, _dp, _dp, _sz, ctypes.c_int,
                                      ctypes.c_double, _dp, _dp]
    L.oracle_bld_mult_f32.argtypes = [_fp, _sz, _sz, _sz, _fp, _fp, _sz, ctypes.c_int,
                                      ctypes.c_double, _fp, _fp]
    L.oracle_log_marginal_S_f64.argtypes = [_dp, _sz, _sz, _sz, _dp, _dp,
                                            ctypes.c_double, ctypes.c_double]
    L.oracle_log_marginal_S_f64.restype = ctypes.c_double
    L.oracle_log_marginal_S_f32.argtypes = [_fp, _sz, _sz, _sz, _dp, _dp,
                                            ctypes.c_double, ctypes.c_double]
    L.oracle_log_marginal_S_f32.restype = ctypes.c_double
    L.oracle_sparseness_f64.argtypes = [_dp, _sz, _sz, _sz]
    L.oracle_sparseness_f64.restype = ctypes.c_double
    L.oracle_bld_fact_f64.argtypes = [_dp, _sz, _sz, _sz, _dp, _dp, ctypes.c_double,
                                      ctypes.c_double, ctypes.c_double, _dp, _dp, _dp]
    L.oracle_init_S_f64.argtypes = [_dp, _sz, _sz, _sz, ctypes.c_uint64, _dp]


def _d(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(_dp)


def _f(a):
    a = np.ascontiguousarray(a, dtype=np.float32)
    return a, a.ctypes.data_as(_fp)


def set_threads(n=0):
    return lib().oracle_set_threads(int(n))


def psi_appr(v):
    return lib().oracle_psi_appr_f64(float(v))


def psi_appr_f32(v):
    return lib().oracle_psi_appr_f32(float(v))


def psi_exact(v):
    return lib().oracle_psi_exact(float(v))


def psi_array(values, appr=True):
    v, pv = _d(values)
    out = np.empty_like(v)
    lib().oracle_psi_array(pv, v.size, 1 if appr else 0, out.ctypes.data_as(_dp))
    return out


def tensor_sums(S):
    x, y, z = S.shape
    if S.dtype == np.float32:
        S, pS = _f(S)
        pjk, ipk, ijp = (np.empty((y, z), np.float32), np.empty((x, z), np.float32),
                         np.empty((x, y), np.float32))
        lib().oracle_tensor_sums_f32(pS, x, y, z, *[a.ctypes.data_as(_fp) for a in (pjk, ipk, ijp)])
        return pjk, ipk, ijp
    S, pS = _d(S)
    pjk, ipk, ijp = np.empty((y, z)), np.empty((x, z)), np.empty((x, y))
    lib().oracle_tensor_sums_f64(pS, x, y, z, *[a.ctypes.data_as(_dp) for a in (pjk, ipk, ijp)])
    return pjk, ipk, ijp


def x_reciprocal(X, eps=1e-50):
    X, pX = _d(X)
    out = np.empty_like(X)
    lib().oracle_x_reciprocal_f64(pX, X.shape[0], X.shape[1], eps, out.ctypes.data_as(_dp))
    return out


def update_alpha_eph(ipk, alpha):
    ipk, p1 = _d(ipk)
    alpha, p2 = _d(alpha)
    out = np.empty_like(ipk)
    lib().oracle_update_alpha_eph_f64(p1, p2, ipk.shape[0], ipk.shape[1], out.ctypes.data_as(_dp))
    return out


def update_beta_eph(pjk, beta):
    pjk, p1 = _d(pjk)
    beta, p2 = _d(beta)
    out = np.empty_like(pjk)
    lib().oracle_update_beta_eph_f64(p1, p2, pjk.shape[0], pjk.shape[1], out.ctypes.data_as(_dp))
    return out


def update_grad_plus(S, beta_eph, appr=True):
    S, pS = _d(S)
    beta_eph, pb = _d(beta_eph)
    out = np.empty_like(S)
    x, y, z = S.shape
    lib().oracle_update_grad_plus_f64(pS, pb, x, y, z, 1 if appr else 0, out.ctypes.data_as(_dp))
    return out


def update_grad_minus(alpha_eph, appr=True):
    a, pa = _d(alpha_eph)
    out = np.empty_like(a)
    lib().oracle_update_grad_minus_f64(pa, a.shape[0], a.shape[1], 1 if appr else 0,
                                       out.ctypes.data_as(_dp))
    return out


def update_nom(Xr, gm, S):
    Xr, p1 = _d(Xr)
    gm, p2 = _d(gm)
    S, p3 = _d(S)
    x, y, z = S.shape
    out = np.empty((x, y))
    lib().oracle_update_nom_f64(p1, p2, p3, x, y, z, out.ctypes.data_as(_dp))
    return out


def update_denom(Xr, gp, S):
    Xr, p1 = _d(Xr)
    gp, p2 = _d(gp)
    S, p3 = _d(S)
    x, y, z = S.shape
    out = np.empty((x, y))
    lib().oracle_update_denom_f64(p1, p2, p3, x, y, z, out.ctypes.data_as(_dp))
    return out


def update_S(X, nom, denom, gm, gp, ijp, S, eps=1e-50):
    """Returns the updated copy of S."""
    out = np.array(S, dtype=np.float64, copy=True, order="C")
    keep =[np.ascontiguousarray(a, dtype=np.float64) for a in (X, nom, denom, gm, gp, ijp)]
    args = [k.ctypes.data_as(_dp) for k in keep]
    x, y, z = out.shape
    lib().oracle_update_S_f64(*args, x, y, z, eps, out.ctypes.data_as(_dp))
    return out


def bld_mult(X, z, alpha, beta, max_iter, psi_mode=PSI_APPR, eps=1e-50, S0=None,
             dtype=np.float64, seed=0):
    """Oracle solve.  S0 defaults to the seeded initial S of init_S()."""
    X = np.ascontiguousarray(X, dtype=np.float64)
    x, y = X.shape
    if S0 is None:
        S0 = init_S(X, z, seed)
    if dtype == np.float32:
        Xf, pX = _f(X)
        af, pa = _f(alpha)
        bf, pb = _f(beta)
        S0f, pS0 = _f(S0)
        out = np.empty((x, y, z), np.float32)
        lib().oracle_bld_mult_f32(pX, x, y, z, pa, pb, max_iter, psi_mode, eps, pS0,
                                  out.ctypes.data_as(_fp))
        return out
    Xd, pX = _d(X)
    ad, pa = _d(alpha)
    bd, pb = _d(beta)
    S0d, pS0 = _d(S0)
    out = np.empty((x, y, z))
    lib().oracle_bld_mult_f64(pX, x, y, z, pa, pb, max_iter, psi_mode, eps, pS0,
                              out.ctypes.data_as(_dp))
    return out


def log_marginal_S(S, alpha, beta, a, b):
    x, y, z = S.shape
    alpha, pa = _d(alpha)
    beta, pb = _d(beta)
    if S.dtype == np.float32:
        S, pS = _f(S)
        return lib().oracle_log_marginal_S_f32(pS, x, y, z, pa, pb, a, b)
    S, pS = _d(S)
    return lib().oracle_log_marginal_S_f64(pS, x, y, z, pa, pb, a, b)


def sparseness(S):
    S, pS = _d(S)
    return lib().oracle_sparseness_f64(pS, *S.shape)


def bld_fact(S, alpha, beta, a, b, eps=1e-50):
    S, pS = _d(S)
    x, y, z = S.shape
    alpha, pa = _d(alpha)
    beta, pb = _d(beta)
    W, H, L = np.empty((x, z)), np.empty((z, y)), np.empty(y)
    lib().oracle_bld_fact_f64(pS, x, y, z, pa, pb, a, b, eps, W.ctypes.data_as(_dp),
                              H.ctypes.data_as(_dp), L.ctypes.data_as(_dp))
    return W, H, L


def init_S(X, z, seed=0):
    X, pX = _d(X)
    x, y = X.shape
    out = np.empty((x, y, z))
    lib().oracle_init_S_f64(pX, x, y, z, seed, out.ctypes.data_as(_dp))
    return out
