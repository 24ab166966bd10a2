"""Python binding of libbldm.so, the B200-native bld_mult solver.

Mirrors the reference interface of eozd/bnmf-algs for this path:

* ``Params``          — alloc_model::Params (src/alloc_model/alloc_model_params.hpp:25-84)
* ``bld_mult_cuda``   — bld::bld_mult_cuda (src/bld/bld_mult/bld_mult.hpp:225-324)
* ``bld_mult``        — bld::bld_mult semantics (bld_mult.hpp:82-150), run on the GPU
* ``log_marginal_S``  — alloc_model::log_marginal_S (src/alloc_model/alloc_model_funcs.hpp:573-586)

Argument errors raise ``InvalidArgument`` (a ``ValueError``), the counterpart of
the reference's ``BNMF_ASSERT`` throwing ``std::invalid_argument`` in test builds
(src/defs.hpp:12-20).  Every call goes through the C ABI declared in
include/bldm.h; there is no CPU fallback: if libbldm.so is missing or no GPU is
present, the calls raise.
"""

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libbldm.so")

# bldm_status
OK, ERR_BAD_ARG, ERR_NEG_X, ERR_OOM, ERR_CUDA, ERR_TIMEOUT, ERR_NO_DEVICE, \
    ERR_UNSUPPORTED, ERR_BUSY, ERR_NOT_FOUND, ERR_TOO_LARGE = range(11)
STATUS_NAMES = {0: "OK", 1: "BAD_ARG", 2: "NEG_X", 3: "OOM", 4: "CUDA", 5: "TIMEOUT",
                6: "NO_DEVICE", 7: "UNSUPPORTED", 8: "BUSY", 9: "NOT_FOUND", 10: "TOO_LARGE"}
# bldm_psi_mode
PSI_EXACT, PSI_APPR, PSI_LEGACY_CUDA = 0, 1, 2
# bldm_dtype
F64, F32 = 0, 1


class BldmError(RuntimeError):
    def __init__(self, status, what=""):
        self.status = status
        super().__init__(f"bldm: {STATUS_NAMES.get(status, status)} {what}".strip())


class InvalidArgument(ValueError):
    """Raised where the reference's BNMF_ASSERT throws std::invalid_argument."""

    def __init__(self, status, what=""):
        self.status = status
        super().__init__(f"bldm: {STATUS_NAMES.get(status, status)} {what}".strip())


def _check(rc, what=""):
    if rc == OK:
        return
    if rc in (ERR_BAD_ARG, ERR_NEG_X):
        raise InvalidArgument(rc, what)
    raise BldmError(rc, what)


class bldm_params(ctypes.Structure):
    _fields_ = [("a", ctypes.c_double), ("b", ctypes.c_double),
                ("alpha", ctypes.POINTER(ctypes.c_double)), ("n_alpha", ctypes.c_size_t),
                ("beta", ctypes.POINTER(ctypes.c_double)), ("n_beta", ctypes.c_size_t)]


class bldm_tuning(ctypes.Structure):
    _fields_ = [("stages", ctypes.c_int), ("ctas_per_sm", ctypes.c_int),
                ("row_ranges", ctypes.c_int), ("skip_zero_rows", ctypes.c_int)]


class bldm_stats(ctypes.Structure):
    _fields_ = [("device_ms", ctypes.c_double), ("total_ms", ctypes.c_double),
                ("iterations", ctypes.c_uint64), ("kernel_launches", ctypes.c_uint64),
                ("rel_change", ctypes.c_double), ("conservation_residual", ctypes.c_double)]


class bldm_server_config(ctypes.Structure):
    _fields_ = [("dtype", ctypes.c_int), ("psi_mode", ctypes.c_int), ("eps", ctypes.c_double),
                ("tol", ctypes.c_double), ("max_iter", ctypes.c_size_t),
                ("iters_per_round", ctypes.c_size_t), ("max_active", ctypes.c_size_t),
                ("memory_budget", ctypes.c_size_t), ("rows_per_tile", ctypes.c_int),
                ("large_elements", ctypes.c_size_t)]


class bldm_request_stats(ctypes.Structure):
    _fields_ = [("queue_ms", ctypes.c_double), ("latency_ms", ctypes.c_double),
                ("iterations", ctypes.c_uint64), ("rel_change", ctypes.c_double),
                ("log_marginal", ctypes.c_double), ("status", ctypes.c_int),
                ("conservation_residual", ctypes.c_double)]


class bldm_server_stats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_uint64) for n in ("submitted", "completed", "failed", "rounds",
                                              "iterations")] + \
               [(n, ctypes.c_size_t) for n in ("active", "queued", "bytes_in_use", "bytes_peak",
                                              "budget")] + \
               [("gpu_ms", ctypes.c_double), ("host_ms", ctypes.c_double),
                ("retiring", ctypes.c_size_t), ("gpu_ms_large", ctypes.c_double),
                ("retire_ms", ctypes.c_double)]


_lib = None
_vp = ctypes.c_void_p
_sz = ctypes.c_size_t
_dp = ctypes.POINTER(ctypes.c_double)
_fp = ctypes.POINTER(ctypes.c_float)


def lib():
    """The loaded libbldm.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise BldmError(ERR_NO_DEVICE, f"{LIB_PATH} is missing; run build()")
        L = ctypes.CDLL(LIB_PATH)
        _declare(L)
        _lib = L
    return _lib


def build(force=False):
    import importlib.util
    spec = importlib.util.spec_from_file_location("_bldm_build", os.path.join(_HERE, "build.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.build(force=force)


class bldm_batch_class(ctypes.Structure):
    _fields_ = [("vec", ctypes.c_int), ("lanes_per_fiber", ctypes.c_int),
                ("chunks", ctypes.c_int), ("multirow", ctypes.c_int),
                ("rows_per_tile", ctypes.c_int), ("stages", ctypes.c_int),
                ("tiles", ctypes.c_size_t), ("instances", ctypes.c_size_t)]


# Every symbol include/bldm.h declares, with (restype, argtypes).
SIGNATURES = {
    "bldm_solve_f64": (ctypes.c_int, [_dp, _sz, _sz, _sz, ctypes.POINTER(bldm_params), _sz,
                                      ctypes.c_int, ctypes.c_double, _dp, ctypes.c_uint64, _dp,
                                      ctypes.POINTER(bldm_stats)]),
    "bldm_solve_f32": (ctypes.c_int, [_fp, _sz, _sz, _sz, ctypes.POINTER(bldm_params), _sz,
                                      ctypes.c_int, ctypes.c_double, _fp, ctypes.c_uint64, _fp,
                                      ctypes.POINTER(bldm_stats)]),
    "bldm_release_cache": (ctypes.c_int, []),
    "bldm_plan_create": (ctypes.c_int, [ctypes.POINTER(_vp), _sz, _sz, _sz, ctypes.c_int]),
    "bldm_plan_create_tuned": (ctypes.c_int, [ctypes.POINTER(_vp), _sz, _sz, _sz, ctypes.c_int,
                                              ctypes.POINTER(bldm_tuning)]),
    "bldm_plan_get_tuning": (ctypes.c_int, [_vp, ctypes.POINTER(bldm_tuning)]),
    "bldm_plan_destroy": (ctypes.c_int, [_vp]),
    "bldm_plan_workspace_bytes": (ctypes.c_int, [_vp, ctypes.POINTER(_sz)]),
    "bldm_plan_run": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _sz, ctypes.c_int, ctypes.c_double,
                                     _vp]),
    "bldm_plan_check": (ctypes.c_int, [_vp, _vp]),
    "bldm_plan_conservation": (ctypes.c_int, [_vp, _vp, _vp, _vp, _dp]),
    "bldm_solve_device_noalloc": (ctypes.c_int, [_vp, _vp, _vp, _vp, _sz, _sz, _sz, ctypes.c_int,
                                                 _sz, ctypes.c_int, ctypes.c_double, _vp]),
    "bldm_plan_init_S": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_uint64, _vp]),
    "bldm_plan_profile": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _sz, ctypes.c_int,
                                         ctypes.c_double, _vp, _dp, _dp]),
    "bldm_plan_launch_count": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_uint64)]),
    "bldm_plan_shard_red_size": (ctypes.c_int, [_vp, ctypes.POINTER(_sz)]),
    "bldm_plan_shard_sums": (ctypes.c_int, [_vp, _vp, _vp, _vp, ctypes.c_int, _vp]),
    "bldm_plan_shard_update": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, ctypes.c_int,
                                              ctypes.c_double, _vp]),
    "bldm_plan_shard_finish": (ctypes.c_int, [_vp, _vp, _vp, ctypes.c_int, _vp]),
    "bldm_tensor_sums_f64": (ctypes.c_int, [_vp, _sz, _sz, _sz, _vp, _vp, _vp, _vp]),
    "bldm_update_grad_plus_f64": (ctypes.c_int, [_vp, _vp, _sz, _sz, _sz, ctypes.c_int, _vp,
                                                 _vp]),
    "bldm_update_grad_minus_f64": (ctypes.c_int, [_vp, _sz, _sz, ctypes.c_int, _vp, _vp]),
    "bldm_update_nom_f64": (ctypes.c_int, [_vp, _vp, _vp, _sz, _sz, _sz, _vp, _vp]),
    "bldm_update_denom_f64": (ctypes.c_int, [_vp, _vp, _vp, _sz, _sz, _sz, _vp, _vp]),
    "bldm_update_S_f64": (ctypes.c_int, [_vp, _vp, _vp, _vp, _vp, _vp, _sz, _sz, _sz,
                                         ctypes.c_double, _vp, _vp]),
    "bldm_psi_f64": (ctypes.c_int, [_vp, _sz, ctypes.c_int, _vp, _vp]),
    "bldm_psi_f32": (ctypes.c_int, [_vp, _sz, _vp, _vp]),
    "bldm_psi_f32_mode": (ctypes.c_int, [_vp, _sz, ctypes.c_int, _vp, _vp]),
    "bldm_log_marginal_S": (ctypes.c_int, [_vp, ctypes.c_int, _sz, _sz, _sz, _dp, _dp,
                                           ctypes.c_double, ctypes.c_double, _dp, _vp]),
    "bldm_bld_fact": (ctypes.c_int, [_vp, ctypes.c_int, _sz, _sz, _sz, ctypes.POINTER(bldm_params),
                                     ctypes.c_double, _vp, _vp, _vp, _vp]),
    "bldm_bld_fact_f64": (ctypes.c_int, [_dp, _sz, _sz, _sz, ctypes.POINTER(bldm_params),
                                         ctypes.c_double, _dp, _dp, _dp]),
    "bldm_bnmf_priors": (ctypes.c_int, [_sz, _sz, _sz, ctypes.POINTER(bldm_params),
                                        ctypes.c_uint64, ctypes.c_int, _vp, _vp, _vp, _vp]),
    "bldm_sample_S": (ctypes.c_int, [_vp, _vp, _vp, _sz, _sz, _sz, ctypes.c_uint64, ctypes.c_int,
                                     _vp, _vp]),
    "bldm_sample_X": (ctypes.c_int, [_vp, _vp, _vp, _sz, _sz, _sz, ctypes.c_uint64, ctypes.c_int,
                                     _vp, _vp]),
    "bldm_batch_create": (ctypes.c_int, [ctypes.POINTER(_vp), ctypes.c_int, _sz,
                                         ctypes.POINTER(_sz), ctypes.POINTER(_sz),
                                         ctypes.POINTER(_sz), ctypes.c_int]),
    "bldm_batch_destroy": (ctypes.c_int, [_vp]),
    "bldm_batch_set": (ctypes.c_int, [_vp, _sz, _dp, _dp, _dp, _dp, ctypes.c_uint64]),
    "bldm_batch_run": (ctypes.c_int, [_vp, _sz, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                      _vp]),
    "bldm_batch_check": (ctypes.c_int, [_vp, _vp]),
    "bldm_batch_set_launch_mode": (ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_double,
                                                  ctypes.c_int]),
    "bldm_batch_get_launch_mode": (ctypes.c_int, [_vp, ctypes.POINTER(ctypes.c_int)]),
    "bldm_batch_get": (ctypes.c_int, [_vp, _sz, _dp, _dp]),
    "bldm_batch_conservation": (ctypes.c_int, [_vp, _dp, _vp]),
    "bldm_batch_device_ptrs": (ctypes.c_int, [_vp, _sz, ctypes.POINTER(_vp),
                                              ctypes.POINTER(_vp)]),
    "bldm_batch_info": (ctypes.c_int, [_vp, ctypes.POINTER(_sz), ctypes.POINTER(_sz),
                                       ctypes.POINTER(ctypes.c_uint64)]),
    "bldm_batch_class_info": (ctypes.c_int, [_vp, _sz, ctypes.POINTER(bldm_batch_class)]),
    "bldm_batch_set_class": (ctypes.c_int, [_vp, ctypes.POINTER(bldm_batch_class)]),
    "bldm_batch_autotune": (ctypes.c_int, [_vp, _sz, ctypes.c_int, ctypes.c_double, _vp, _dp,
                                           _dp]),
    "bldm_server_create": (ctypes.c_int, [ctypes.POINTER(_vp), ctypes.POINTER(bldm_server_config)]),
    "bldm_server_destroy": (ctypes.c_int, [_vp]),
    "bldm_server_submit": (ctypes.c_int, [_vp, _dp, _sz, _sz, _sz, ctypes.POINTER(bldm_params),
                                          ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64)]),
    "bldm_server_poll": (ctypes.c_int, [_vp, ctypes.c_uint64, ctypes.POINTER(ctypes.c_int)]),
    "bldm_server_wait": (ctypes.c_int, [_vp, ctypes.c_uint64, ctypes.c_double]),
    "bldm_server_fetch": (ctypes.c_int, [_vp, ctypes.c_uint64, _dp,
                                         ctypes.POINTER(bldm_request_stats)]),
    "bldm_server_cancel": (ctypes.c_int, [_vp, ctypes.c_uint64]),
    "bldm_server_get_stats": (ctypes.c_int, [_vp, ctypes.POINTER(bldm_server_stats)]),
    "bldm_version": (ctypes.c_char_p, []),
}


def _declare(L):
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args


def version():
    return lib().bldm_version().decode()


class Params:
    """alloc_model::Params: Gamma shape a, rate b, Dirichlet alpha (x) and beta (z)."""

    def __init__(self, a, b, alpha, beta):
        self.a = float(a)
        self.b = float(b)
        self.alpha = np.ascontiguousarray(alpha, dtype=np.float64).reshape(-1)
        self.beta = np.ascontiguousarray(beta, dtype=np.float64).reshape(-1)

    @classmethod
    def from_shape(cls, shape):
        """The reference's default ctor from a tensor shape: a=1, b=10, alpha=1, beta=1."""
        x, _, z = shape
        return cls(1.0, 10.0, np.ones(x), np.ones(z))

    def c_struct(self):
        p = bldm_params()
        p.a, p.b = self.a, self.b
        p.alpha = self.alpha.ctypes.data_as(_dp)
        p.n_alpha = self.alpha.size
        p.beta = self.beta.ctypes.data_as(_dp)
        p.n_beta = self.beta.size
        return p


def _solve(X, z, params, max_iter, psi_mode, eps, S0, seed, dtype, stats):
    np_t = np.float64 if dtype == F64 else np.float32
    X = np.ascontiguousarray(X, dtype=np_t)
    if X.ndim != 2:
        raise InvalidArgument(ERR_BAD_ARG, "X must be a matrix")
    x, y = X.shape
    out = np.empty((x, y, int(z)), dtype=np_t)
    S0p = None
    if S0 is not None:
        S0 = np.ascontiguousarray(S0, dtype=np_t)
        if S0.shape != out.shape:
            raise InvalidArgument(ERR_BAD_ARG, "S0 shape")
    cp = params.c_struct()
    st = bldm_stats()
    if dtype == F64:
        ptr = lambda a: a.ctypes.data_as(_dp) if a is not None else None
        rc = lib().bldm_solve_f64(ptr(X), x, y, int(z), ctypes.byref(cp), int(max_iter),
                                  int(psi_mode), float(eps), ptr(S0), int(seed), ptr(out),
                                  ctypes.byref(st))
    else:
        ptr = lambda a: a.ctypes.data_as(_fp) if a is not None else None
        rc = lib().bldm_solve_f32(ptr(X), x, y, int(z), ctypes.byref(cp), int(max_iter),
                                  int(psi_mode), float(eps), ptr(S0), int(seed), ptr(out),
                                  ctypes.byref(st))
    _check(rc, "bldm_solve")
    if stats is not None:
        stats.update(device_ms=st.device_ms, total_ms=st.total_ms, iterations=st.iterations,
                     kernel_launches=st.kernel_launches,
                     conservation_residual=st.conservation_residual)
    return out


def bld_mult_cuda(X, z, params, max_iter=1000, use_psi_appr=False, eps=1e-50, S0=None, seed=0,
                  dtype=F64, stats=None):
    """bld::bld_mult_cuda: with use_psi_appr=False the grad_plus digamma stays psi_appr,
    as in the reference's device kernel; grad_minus uses the exact digamma."""
    mode = PSI_APPR if use_psi_appr else PSI_LEGACY_CUDA
    return _solve(X, z, params, max_iter, mode, eps, S0, seed, dtype, stats)


def bld_mult(X, z, params, max_iter=1000, use_psi_appr=False, eps=1e-50, S0=None, seed=0,
             dtype=F64, stats=None):
    """bld::bld_mult semantics (exact digamma everywhere unless use_psi_appr), on the GPU."""
    mode = PSI_APPR if use_psi_appr else PSI_EXACT
    return _solve(X, z, params, max_iter, mode, eps, S0, seed, dtype, stats)


def release_cache():
    _check(lib().bldm_release_cache())


# ----------------------------------------------------------------------------
# Device-buffer API (torch CUDA tensors as the device allocator).
# ----------------------------------------------------------------------------
def _ptr(t):
    return ctypes.c_void_p(t.data_ptr())


def _stream_ptr(stream):
    if stream is None:
        import torch
        stream = torch.cuda.current_stream()
    return ctypes.c_void_p(stream.cuda_stream)


class Plan:
    """bldm_plan: workspace for one (x, y, z, dtype); runs on device tensors."""

    def __init__(self, x, y, z, dtype=F64, stages=0, ctas_per_sm=0, row_ranges=0,
                 skip_zero_rows=False):
        self._h = ctypes.c_void_p()
        self.shape = (x, y, z)
        self.dtype = dtype
        if stages or ctas_per_sm or row_ranges or skip_zero_rows:
            t = bldm_tuning(int(stages), int(ctas_per_sm), int(row_ranges),
                            1 if skip_zero_rows else 0)
            _check(lib().bldm_plan_create_tuned(ctypes.byref(self._h), x, y, z, dtype,
                                                ctypes.byref(t)), "plan_create_tuned")
        else:
            _check(lib().bldm_plan_create(ctypes.byref(self._h), x, y, z, dtype), "plan_create")

    def tuning(self):
        t = bldm_tuning()
        _check(lib().bldm_plan_get_tuning(self._h, ctypes.byref(t)))
        return {"stages": t.stages, "ctas_per_sm": t.ctas_per_sm, "row_ranges": t.row_ranges,
                "skip_zero_rows": bool(t.skip_zero_rows)}

    def close(self):
        if self._h:
            lib().bldm_plan_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def workspace_bytes(self):
        n = ctypes.c_size_t()
        _check(lib().bldm_plan_workspace_bytes(self._h, ctypes.byref(n)))
        return n.value

    def run(self, dX, dalpha, dbeta, dS, max_iter, psi_mode=PSI_APPR, eps=1e-50, stream=None):
        _check(lib().bldm_plan_run(self._h, _ptr(dX), _ptr(dalpha), _ptr(dbeta), _ptr(dS),
                                   int(max_iter), int(psi_mode), float(eps),
                                   _stream_ptr(stream)), "plan_run")

    def check(self, stream=None):
        _check(lib().bldm_plan_check(self._h, _stream_ptr(stream)), "plan_check")

    def conservation(self, dX, dS, stream=None):
        """max_ij |sum_k S - X| / max(X, 1) of device tensors, computed on the device."""
        out = ctypes.c_double()
        _check(lib().bldm_plan_conservation(self._h, _ptr(dX), _ptr(dS), _stream_ptr(stream),
                                            ctypes.byref(out)), "plan_conservation")
        return out.value

    def init_S(self, dX, dS, seed=0, stream=None):
        _check(lib().bldm_plan_init_S(self._h, _ptr(dX), _ptr(dS), int(seed),
                                      _stream_ptr(stream)))

    def profile(self, dX, dalpha, dbeta, dS, iters, psi_mode=PSI_APPR, eps=1e-50, stream=None):
        k = ctypes.c_double()
        it = ctypes.c_double()
        _check(lib().bldm_plan_profile(self._h, _ptr(dX), _ptr(dalpha), _ptr(dbeta), _ptr(dS),
                                       int(iters), int(psi_mode), float(eps), _stream_ptr(stream),
                                       ctypes.byref(k), ctypes.byref(it)), "plan_profile")
        return k.value, it.value

    def launch_count(self):
        n = ctypes.c_uint64()
        _check(lib().bldm_plan_launch_count(self._h, ctypes.byref(n)))
        return n.value

    # Row-sharded solve steps (see bnmf_algs_b200.multi.sharded_solve).
    def shard_red_size(self):
        n = ctypes.c_size_t()
        _check(lib().bldm_plan_shard_red_size(self._h, ctypes.byref(n)))
        return n.value

    def shard_sums(self, dS, dalpha, dred, psi_mode=PSI_APPR, stream=None):
        _check(lib().bldm_plan_shard_sums(self._h, _ptr(dS), _ptr(dalpha), _ptr(dred),
                                          int(psi_mode), _stream_ptr(stream)), "shard_sums")

    def shard_update(self, dX, dS, dalpha, dred, psi_mode=PSI_APPR, eps=1e-50, stream=None):
        _check(lib().bldm_plan_shard_update(self._h, _ptr(dX), _ptr(dS), _ptr(dalpha),
                                            _ptr(dred), int(psi_mode), float(eps),
                                            _stream_ptr(stream)), "shard_update")

    def shard_finish(self, dbeta, dred, psi_mode=PSI_APPR, stream=None):
        _check(lib().bldm_plan_shard_finish(self._h, _ptr(dbeta), _ptr(dred), int(psi_mode),
                                            _stream_ptr(stream)), "shard_finish")


def bld_fact(S, params, eps=1e-50, dtype=F64, stream=None):
    """bld::bld_fact (src/bld/bld_fact.hpp:36-80): (W x*z, H z*y, L y) from S.

    S is a host array (FP64 in and out, as the reference) or a device tensor
    (outputs are device tensors of its dtype)."""
    x, y, z = S.shape
    if isinstance(S, np.ndarray):
        S = np.ascontiguousarray(S, dtype=np.float64)
        W, H, L = np.empty((x, z)), np.empty((z, y)), np.empty(y)
        cp = params.c_struct()
        _check(lib().bldm_bld_fact_f64(S.ctypes.data_as(_dp), x, y, z, ctypes.byref(cp),
                                       float(eps), W.ctypes.data_as(_dp), H.ctypes.data_as(_dp),
                                       L.ctypes.data_as(_dp)), "bld_fact")
        return W, H, L
    import torch
    W = torch.empty((x, z), dtype=S.dtype, device=S.device)
    H = torch.empty((z, y), dtype=S.dtype, device=S.device)
    L = torch.empty((y,), dtype=S.dtype, device=S.device)
    cp = params.c_struct()
    _check(lib().bldm_bld_fact(_ptr(S), dtype, x, y, z, ctypes.byref(cp), float(eps), _ptr(W),
                               _ptr(H), _ptr(L), _stream_ptr(stream)), "bld_fact")
    return W, H, L


def bnmf_priors(shape, params, seed=0, dtype=F64, stream=None):
    """alloc_model::bnmf_priors on the device: (W x*z, H z*y, L y) torch tensors."""
    import torch
    x, y, z = (int(v) for v in shape)
    tt = torch.float64 if dtype == F64 else torch.float32
    W = torch.empty((x, z), dtype=tt, device="cuda")
    H = torch.empty((z, y), dtype=tt, device="cuda")
    L = torch.empty((y,), dtype=tt, device="cuda")
    cp = params.c_struct()
    _check(lib().bldm_bnmf_priors(x, y, z, ctypes.byref(cp), int(seed), dtype, _ptr(W), _ptr(H),
                                  _ptr(L), _stream_ptr(stream)), "bnmf_priors")
    return W, H, L


def _sample(fn, W, H, L, seed, shape, stream, what):
    import torch
    x, z = W.shape
    y = L.shape[0]
    dtype = F64 if W.dtype == torch.float64 else F32
    out = torch.empty(shape(x, y, z), dtype=W.dtype, device=W.device)
    _check(fn(_ptr(W), _ptr(H), _ptr(L), x, y, z, int(seed), dtype, _ptr(out),
              _stream_ptr(stream)), what)
    return out


def sample_S(W, H, L, seed=0, stream=None):
    """alloc_model::sample_S on the device: S_ijk ~ Poisson(W_ik H_kj L_j)."""
    return _sample(lib().bldm_sample_S, W, H, L, seed, lambda x, y, z: (x, y, z), stream,
                   "sample_S")


def sample_X(W, H, L, seed=0, stream=None):
    """X_ij ~ Poisson(sum_k W_ik H_kj L_j) on the device."""
    return _sample(lib().bldm_sample_X, W, H, L, seed, lambda x, y, z: (x, y), stream, "sample_X")


def log_marginal_S(dS, params, dtype=F64, stream=None):
    """alloc_model::log_marginal_S of a device tensor, on the device (FP64)."""
    x, y, z = dS.shape
    out = ctypes.c_double()
    _check(lib().bldm_log_marginal_S(_ptr(dS), dtype, x, y, z,
                                     params.alpha.ctypes.data_as(_dp),
                                     params.beta.ctypes.data_as(_dp), params.a, params.b,
                                     ctypes.byref(out), _stream_ptr(stream)), "log_marginal_S")
    return out.value


# Per-stage device functions (FP64 torch tensors), mirroring the reference's
# update_*_cuda host functions.
def tensor_sums(dS, stream=None):
    import torch
    x, y, z = dS.shape
    pjk = torch.empty((y, z), dtype=torch.float64, device=dS.device)
    ipk = torch.empty((x, z), dtype=torch.float64, device=dS.device)
    ijp = torch.empty((x, y), dtype=torch.float64, device=dS.device)
    _check(lib().bldm_tensor_sums_f64(_ptr(dS), x, y, z, _ptr(pjk), _ptr(ipk), _ptr(ijp),
                                      _stream_ptr(stream)))
    return pjk, ipk, ijp


def update_grad_plus(dS, dbeta_eph, appr=True, stream=None):
    import torch
    x, y, z = dS.shape
    out = torch.empty_like(dS)
    _check(lib().bldm_update_grad_plus_f64(_ptr(dS), _ptr(dbeta_eph), x, y, z, int(appr),
                                           _ptr(out), _stream_ptr(stream)))
    return out


def update_grad_minus(dalpha_eph, appr=True, stream=None):
    import torch
    x, z = dalpha_eph.shape
    out = torch.empty_like(dalpha_eph)
    _check(lib().bldm_update_grad_minus_f64(_ptr(dalpha_eph), x, z, int(appr), _ptr(out),
                                            _stream_ptr(stream)))
    return out


def update_nom(dXr, dgm, dS, stream=None):
    import torch
    x, y, z = dS.shape
    out = torch.empty((x, y), dtype=torch.float64, device=dS.device)
    _check(lib().bldm_update_nom_f64(_ptr(dXr), _ptr(dgm), _ptr(dS), x, y, z, _ptr(out),
                                     _stream_ptr(stream)))
    return out


def update_denom(dXr, dgp, dS, stream=None):
    import torch
    x, y, z = dS.shape
    out = torch.empty((x, y), dtype=torch.float64, device=dS.device)
    _check(lib().bldm_update_denom_f64(_ptr(dXr), _ptr(dgp), _ptr(dS), x, y, z, _ptr(out),
                                       _stream_ptr(stream)))
    return out


def update_S(dX, dnom, ddenom, dgm, dgp, dijp, dS, eps=1e-50, stream=None):
    """In place on dS."""
    x, y, z = dS.shape
    _check(lib().bldm_update_S_f64(_ptr(dX), _ptr(dnom), _ptr(ddenom), _ptr(dgm), _ptr(dgp),
                                   _ptr(dijp), x, y, z, float(eps), _ptr(dS),
                                   _stream_ptr(stream)))
    return dS


def psi(d_in, appr=True, stream=None):
    import torch
    out = torch.empty_like(d_in)
    if d_in.dtype == torch.float64:
        _check(lib().bldm_psi_f64(_ptr(d_in), d_in.numel(), int(appr), _ptr(out),
                                  _stream_ptr(stream)))
    else:
        # FP32: appr == 2 selects the fused sweep's form, anything else the
        # tabulating form
        _check(lib().bldm_psi_f32_mode(_ptr(d_in), d_in.numel(), 1 if appr == 2 else 0,
                                       _ptr(out), _stream_ptr(stream)))
    return out


class Batch:
    """bldm_batch: independent instances of different shapes solved together."""

    def __init__(self, shapes, dtype=F32, rows_per_tile=0):
        n = len(shapes)
        arr = lambda v: (ctypes.c_size_t * n)(*v)
        self.shapes = [tuple(int(v) for v in s) for s in shapes]
        self.dtype = dtype
        self._h = ctypes.c_void_p()
        _check(lib().bldm_batch_create(ctypes.byref(self._h), dtype, n,
                                       arr([s[0] for s in self.shapes]),
                                       arr([s[1] for s in self.shapes]),
                                       arr([s[2] for s in self.shapes]), int(rows_per_tile)),
               "batch_create")

    def close(self):
        if self._h:
            lib().bldm_batch_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set(self, idx, X, alpha, beta, S0=None, seed=0):
        X = np.ascontiguousarray(X, dtype=np.float64)
        alpha = np.ascontiguousarray(alpha, dtype=np.float64)
        beta = np.ascontiguousarray(beta, dtype=np.float64)
        S0p = None
        if S0 is not None:
            S0 = np.ascontiguousarray(S0, dtype=np.float64)
            S0p = S0.ctypes.data_as(_dp)
        _check(lib().bldm_batch_set(self._h, idx, X.ctypes.data_as(_dp),
                                    alpha.ctypes.data_as(_dp), beta.ctypes.data_as(_dp), S0p,
                                    int(seed)), "batch_set")

    def run(self, iters, psi_mode=PSI_APPR, eps=1e-50, use_graph=True, stream=None):
        _check(lib().bldm_batch_run(self._h, int(iters), int(psi_mode), float(eps),
                                    1 if use_graph else 0, _stream_ptr(stream)), "batch_run")

    def check(self, stream=None):
        _check(lib().bldm_batch_check(self._h, _stream_ptr(stream)), "batch_check")

    def set_launch_mode(self, persistent=True, wait_limit_s=1.0, stall_test=False):
        """Persistent launches per class (default) or one launch per class and iteration."""
        _check(lib().bldm_batch_set_launch_mode(self._h, 1 if persistent else 0,
                                                float(wait_limit_s), 1 if stall_test else 0),
               "batch_set_launch_mode")

    def persistent(self):
        v = ctypes.c_int()
        _check(lib().bldm_batch_get_launch_mode(self._h, ctypes.byref(v)))
        return bool(v.value)

    def get(self, idx):
        x, y, z = self.shapes[idx]
        S = np.empty((x, y, z))
        rel = ctypes.c_double()
        _check(lib().bldm_batch_get(self._h, idx, S.ctypes.data_as(_dp), ctypes.byref(rel)))
        return S, rel.value

    def conservation(self, stream=None):
        """Row-sum conservation residual of every instance's current S (numpy array)."""
        out = np.empty(len(self.shapes))
        _check(lib().bldm_batch_conservation(self._h, out.ctypes.data_as(_dp),
                                             _stream_ptr(stream)), "batch_conservation")
        return out

    def info(self):
        nc, nb, nl = ctypes.c_size_t(), ctypes.c_size_t(), ctypes.c_uint64()
        _check(lib().bldm_batch_info(self._h, ctypes.byref(nc), ctypes.byref(nb),
                                     ctypes.byref(nl)))
        return {"classes": nc.value, "device_bytes": nb.value, "launches": nl.value}

    def classes(self):
        """Launch shape of every lane-shape class (list of dicts)."""
        out = []
        for i in range(self.info()["classes"]):
            c = bldm_batch_class()
            _check(lib().bldm_batch_class_info(self._h, i, ctypes.byref(c)), "batch_class_info")
            out.append({f: getattr(c, f) for f, _ in bldm_batch_class._fields_})
        return out

    def set_class(self, cls):
        """Applies a class launch shape (a dict as classes() returns)."""
        c = bldm_batch_class(**{f: int(cls.get(f, 0)) for f, _ in bldm_batch_class._fields_})
        _check(lib().bldm_batch_set_class(self._h, ctypes.byref(c)), "batch_set_class")

    def autotune(self, probe_iters=3, psi_mode=PSI_APPR, eps=1e-50, stream=None):
        """Picks tile height and stage depth per class; returns (default_ms, tuned_ms)."""
        d, t = ctypes.c_double(), ctypes.c_double()
        _check(lib().bldm_batch_autotune(self._h, int(probe_iters), int(psi_mode), float(eps),
                                         _stream_ptr(stream), ctypes.byref(d), ctypes.byref(t)),
               "batch_autotune")
        return d.value, t.value


class Server:
    """bldm_server: continuous batching of solves; S stays on the device between rounds."""

    QUEUED, ACTIVE, DONE, FAILED = 0, 1, 2, 3

    def __init__(self, dtype=F32, psi_mode=PSI_APPR, eps=1e-50, tol=1e-6, max_iter=500,
                 iters_per_round=10, max_active=256, memory_budget=0, rows_per_tile=0,
                 large_elements=0):
        cfg = bldm_server_config(dtype, psi_mode, eps, tol, max_iter, iters_per_round, max_active,
                                 memory_budget, rows_per_tile, large_elements)
        self.dtype = dtype
        self._h = ctypes.c_void_p()
        self._shapes = {}
        _check(lib().bldm_server_create(ctypes.byref(self._h), ctypes.byref(cfg)),
               "server_create")

    def close(self):
        if self._h:
            lib().bldm_server_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, X, z, params, seed=0):
        X = np.ascontiguousarray(X, dtype=np.float64)
        x, y = X.shape
        cp = params.c_struct()
        rid = ctypes.c_uint64()
        _check(lib().bldm_server_submit(self._h, X.ctypes.data_as(_dp), x, y, int(z),
                                        ctypes.byref(cp), int(seed), ctypes.byref(rid)),
               "server_submit")
        self._shapes[rid.value] = (x, y, int(z))
        return rid.value

    def poll(self, rid):
        st = ctypes.c_int()
        _check(lib().bldm_server_poll(self._h, rid, ctypes.byref(st)))
        return st.value

    def wait(self, rid, timeout=120.0):
        return lib().bldm_server_wait(self._h, rid, float(timeout)) == OK

    def fetch(self, rid, want_S=True):
        """(S or None, stats dict); S is None when the request failed or want_S is False."""
        x, y, z = self._shapes.pop(rid)
        S = np.empty((x, y, z)) if want_S else None
        rs = bldm_request_stats()
        rc = lib().bldm_server_fetch(self._h, rid, S.ctypes.data_as(_dp) if want_S else None,
                                     ctypes.byref(rs))
        stats = {"queue_ms": rs.queue_ms, "latency_ms": rs.latency_ms,
                 "iterations": rs.iterations, "rel_change": rs.rel_change,
                 "log_marginal": rs.log_marginal, "status": rs.status,
                 "conservation_residual": rs.conservation_residual}
        return (S if rc == OK else None), stats

    def cancel(self, rid):
        _check(lib().bldm_server_cancel(self._h, rid))

    def stats(self):
        st = bldm_server_stats()
        _check(lib().bldm_server_get_stats(self._h, ctypes.byref(st)))
        return {n: getattr(st, n) for n, _ in bldm_server_stats._fields_}
