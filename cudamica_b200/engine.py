"""Python mirror of the engine's C ABI (include/amica_b200.h), over ctypes.

The reference has no Python or library API -- its EM loop is
``runamica()`` behind the ``cudaamica -f <params>`` executable
(src/cudaamica.cu:17-43, src/amica.cu:624) -- so this module mirrors the C ABI
one to one.  It needs the in-tree shared library built for sm_100a
(``python -m cudamica_b200.build``) and raises if it is missing: there is no
CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

PKG = os.path.dirname(os.path.abspath(__file__))
# the in-tree build; CUDAMICA_B200_LIB names another build of the same ABI
LIB_PATH = os.environ.get("CUDAMICA_B200_LIB") or os.path.join(PKG, "libamica_b200.so")

AMICA_PREC_FP32 = 0
AMICA_PREC_MIXED = 1

_i64 = C.c_int64
_dbl = C.c_double
_pd = C.POINTER(C.c_double)
_pf = C.POINTER(C.c_float)
_pu8 = C.POINTER(C.c_uint8)

CFG_INT_FIELDS = (
    "nchannels", "nsamples", "nmmodels", "nsdm", "maxiter", "do_sphere", "block_size", "fix_init",
    "do_newton", "update_rho", "rho_start_iter", "newt_start_iter", "maxdec", "update_gm",
    "update_alpha", "update_A", "update_mu", "update_beta", "do_reparm", "do_reject", "rejstart",
    "rejint", "maxrej", "precision", "device", "seed", "verbose", "max_clusters", "phi_split",
    "tc_shape")
CFG_DBL_FIELDS = ("lrate0", "lratemax", "lnatrate", "lratefact", "rho0", "rholrate", "rhomin",
                  "rhomax", "rejsig", "phi_split_rel")

EXPORTED = (
    "amica_default_cfg", "amica_create", "amica_destroy", "amica_load_data",
    "amica_load_data_device", "amica_preprocess", "amica_set_sphered", "amica_init",
    "amica_em_step", "amica_run", "amica_get_params", "amica_set_params", "amica_estep_stats",
    "amica_stats_len", "amica_get_loglik", "amica_loglik_adjoint", "amica_reject_now",
    "amica_write_outputs", "amica_status_string", "amica_kernel_name", "amica_get_p_relative",
    "amica_last_cuda_error", "amica_set_iter_state", "amica_get_sphere", "amica_time_estep",
    "amica_launches_per_iteration", "amica_selftest_umma", "amica_estep_stats_noalloc",
    "amica_run_async", "amica_run_wait", "amica_set_grid", "amica_cohort_create",
    "amica_cohort_run", "amica_cohort_destroy", "amica_test_arm_wait_fault",
    "amica_shard_estep", "amica_shard_mstep", "amica_shard_colsum", "amica_shard_scatter",
    "amica_shard_sphere", "amica_get_stream", "amica_set_tile_shape")


class Cfg(C.Structure):
    _fields_ = [(k, _i64) for k in CFG_INT_FIELDS] + [(k, _dbl) for k in CFG_DBL_FIELDS]


class IterOut(C.Structure):
    _fields_ = [("iter", _i64), ("ll", _dbl), ("lrate", _dbl), ("ll_decreased", _i64),
                ("newton", _i64), ("nkeep", _i64), ("nrejected", _i64), ("device_ms", _dbl),
                ("phi_split", _i64)]


class Paths(C.Structure):
    _fields_ = [(k, C.c_char_p) for k in (
        "weightsfile", "afile", "cfile", "ltallfile", "gmfile", "alphafile", "mufile",
        "betafile", "rhofile", "llfile", "spherefile")]


class AmicaError(RuntimeError):
    def __init__(self, code: int, where: str):
        self.code = code
        msg = lib().amica_status_string(code).decode()
        super().__init__(f"{where}: status {code} ({msg})")


_lib = None


def lib():
    """Load libamica_b200.so; raise if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"{LIB_PATH} is missing: build it with python -m cudamica_b200.build")
        L = C.CDLL(LIB_PATH)
        vp = C.c_void_p
        L.amica_default_cfg.argtypes = [C.POINTER(Cfg)]
        L.amica_create.argtypes = [C.POINTER(Cfg), C.POINTER(vp)]
        L.amica_destroy.argtypes = [vp]
        L.amica_load_data.argtypes = [vp, _pf, _i64, _i64]
        L.amica_load_data_device.argtypes = [vp, vp, _i64, _i64]
        L.amica_preprocess.argtypes = [vp]
        L.amica_set_sphered.argtypes = [vp, _pd, _pd, _pd, _dbl]
        L.amica_init.argtypes = [vp, _pd, _pd]
        L.amica_em_step.argtypes = [vp, C.POINTER(IterOut)]
        L.amica_run.argtypes = [vp, _i64, C.POINTER(IterOut)]
        L.amica_run_async.argtypes = [vp, _i64]
        L.amica_set_grid.argtypes = [vp, _i64, C.POINTER(_i64)]
        L.amica_test_arm_wait_fault.argtypes = [vp, _i64]
        L.amica_shard_estep.argtypes = [vp, vp]
        L.amica_shard_mstep.argtypes = [vp, vp, _i64, C.POINTER(IterOut)]
        L.amica_shard_colsum.argtypes = [vp, vp]
        L.amica_get_stream.argtypes = [vp, C.POINTER(vp)]
        L.amica_set_tile_shape.argtypes = [vp, _i64]
        L.amica_shard_scatter.argtypes = [vp, vp, _i64, vp]
        L.amica_shard_sphere.argtypes = [vp, vp, _i64]
        L.amica_run_wait.argtypes = [vp, C.POINTER(IterOut)]
        L.amica_cohort_create.argtypes = [C.POINTER(vp), _i64, C.POINTER(vp)]
        L.amica_cohort_run.argtypes = [vp, _i64, C.POINTER(IterOut), C.POINTER(_dbl)]
        L.amica_cohort_destroy.argtypes = [vp]
        L.amica_get_params.argtypes = [vp] + [_pd] * 8
        L.amica_set_params.argtypes = [vp] + [_pd] * 7
        L.amica_estep_stats.argtypes = [vp, _pd]
        L.amica_stats_len.restype = _i64
        L.amica_stats_len.argtypes = [_i64, _i64, _i64]
        L.amica_get_loglik.argtypes = [vp, _pd, _pd, _pu8]
        L.amica_loglik_adjoint.argtypes = [vp, _pd, _pd, _pd, _pd, _pd]
        L.amica_reject_now.argtypes = [vp, C.POINTER(_i64)]
        L.amica_write_outputs.argtypes = [vp, C.POINTER(Paths)]
        L.amica_status_string.restype = C.c_char_p
        L.amica_status_string.argtypes = [C.c_int]
        L.amica_kernel_name.restype = C.c_char_p
        L.amica_kernel_name.argtypes = [vp]
        L.amica_get_p_relative.argtypes = [vp, _pf]
        L.amica_set_iter_state.argtypes = [vp, _i64, _dbl, _dbl]
        L.amica_get_sphere.argtypes = [vp, _pd, _pd, _pd]
        L.amica_time_estep.argtypes = [vp, _i64, _pd, C.POINTER(_i64)]
        L.amica_launches_per_iteration.restype = _i64
        L.amica_launches_per_iteration.argtypes = [vp]
        L.amica_selftest_umma.argtypes = [C.c_int, C.c_int, C.c_int, _pf, _pf, _pf, C.POINTER(C.c_int)]
        L.amica_estep_stats_noalloc.argtypes = [vp, _i64, _i64, _i64, _i64, _i64, vp, vp, vp, vp,
                                                vp, vp, vp, _dbl, vp, _i64, _i64, vp, vp]
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(_pd)


def _chk(rc: int, where: str) -> None:
    if rc != 0:
        raise AmicaError(rc, where)


def default_cfg(**over) -> Cfg:
    c = Cfg()
    _chk(lib().amica_default_cfg(C.byref(c)), "amica_default_cfg")
    for k, v in over.items():
        setattr(c, k, v)
    return c


def selftest_umma(mode: int, A: np.ndarray, B: np.ndarray) -> np.ndarray:
    """Run one tensor-core contraction with the E-step's layouts (see header)."""
    A = np.ascontiguousarray(A, dtype=np.float32)
    B = np.ascontiguousarray(B, dtype=np.float32)
    K = A.shape[1]
    N = B.shape[0]
    D = np.empty((128, N), dtype=np.float32)
    derr = C.c_int(0)
    _chk(lib().amica_selftest_umma(mode, N, K, A.ctypes.data_as(_pf), B.ctypes.data_as(_pf),
                                   D.ctypes.data_as(_pf), C.byref(derr)), "amica_selftest_umma")
    if derr.value:
        raise AmicaError(-24, "amica_selftest_umma (device wait)")
    return D


def estep_stats_noalloc(x_ptr: int, ldx: int, n: int, T: int, M: int, m: int, A_ptr: int,
                        c_ptr: int, alpha_ptr: int, mu_ptr: int, beta_ptr: int, rho_ptr: int,
                        gm_ptr: int, ldetS: float, stats_ptr: int, keep_ptr: int = 0,
                        nkeep: int | None = None, update_rho: int = 1, stream: int = 0) -> None:
    """The allocation-free E-step statistics call; every pointer is a device
    address owned by the caller (see include/amica_b200.h)."""
    rc = lib().amica_estep_stats_noalloc(
        C.c_void_p(x_ptr), ldx, n, T, M, m, C.c_void_p(A_ptr), C.c_void_p(c_ptr),
        C.c_void_p(alpha_ptr), C.c_void_p(mu_ptr), C.c_void_p(beta_ptr), C.c_void_p(rho_ptr),
        C.c_void_p(gm_ptr), float(ldetS), C.c_void_p(keep_ptr or None), T if nkeep is None else nkeep,
        update_rho, C.c_void_p(stats_ptr), C.c_void_p(stream or None))
    _chk(rc, "amica_estep_stats_noalloc")


class Amica:
    """One fit on one GPU: a thin owner of an amica_ctx."""

    def __init__(self, n: int, T: int, M: int = 1, m: int = 3, **cfg_over):
        self.cfg = default_cfg(nchannels=n, nsamples=T, nmmodels=M, nsdm=m, **cfg_over)
        self.n, self.T, self.M, self.m = n, T, M, m
        self._ctx = C.c_void_p()
        _chk(lib().amica_create(C.byref(self.cfg), C.byref(self._ctx)), "amica_create")

    # -- lifecycle -------------------------------------------------------
    def close(self) -> None:
        if self._ctx:
            lib().amica_destroy(self._ctx)
            self._ctx = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def kernel(self) -> str:
        return lib().amica_kernel_name(self._ctx).decode()

    # -- data --------------------------------------------------------------
    def load_data(self, x: np.ndarray) -> None:
        x = np.ascontiguousarray(x, dtype=np.float32)
        assert x.shape == (self.T, self.n)
        _chk(lib().amica_load_data(self._ctx, x.ctypes.data_as(_pf), self.n, self.T),
             "amica_load_data")

    def load_data_device(self, ptr: int) -> None:
        _chk(lib().amica_load_data_device(self._ctx, C.c_void_p(ptr), self.n, self.T),
             "amica_load_data_device")

    def preprocess(self) -> None:
        _chk(lib().amica_preprocess(self._ctx), "amica_preprocess")

    def set_sphered(self, xs, means=None, sphere=None, ldetS: float = 0.0) -> None:
        xs = np.ascontiguousarray(xs, dtype=np.float64)
        mn = None if means is None else np.ascontiguousarray(means, dtype=np.float64)
        sp = None if sphere is None else np.ascontiguousarray(np.asarray(sphere).T, dtype=np.float64)
        _chk(lib().amica_set_sphered(self._ctx, _p(xs), _p(mn), _p(sp), float(ldetS)),
             "amica_set_sphered")

    def init(self, A0=None, c0=None) -> None:
        a = None if A0 is None else np.ascontiguousarray(A0, dtype=np.float64)
        c = None if c0 is None else np.ascontiguousarray(c0, dtype=np.float64)
        _chk(lib().amica_init(self._ctx, _p(a), _p(c)), "amica_init")

    # -- iterations --------------------------------------------------------
    def step(self) -> IterOut:
        out = IterOut()
        _chk(lib().amica_em_step(self._ctx, C.byref(out)), "amica_em_step")
        return out

    def run(self, iters: int) -> list:
        outs = (IterOut * max(iters, 1))()
        _chk(lib().amica_run(self._ctx, iters, outs), "amica_run")
        return [outs[k] for k in range(iters)]

    def shard_estep(self, d_stats: int) -> None:
        """This shard's E-step statistics into device memory at d_stats
        (stats_len doubles; amica_shard_estep), queued on self.stream."""
        _chk(lib().amica_shard_estep(self._ctx, C.c_void_p(d_stats)), "amica_shard_estep")

    def shard_mstep(self, d_stats: int, nkeep_total: int) -> IterOut:
        """The M-step from the statistics of all shards at d_stats (device;
        amica_shard_mstep)."""
        out = IterOut()
        _chk(lib().amica_shard_mstep(self._ctx, C.c_void_p(d_stats), int(nkeep_total), C.byref(out)),
             "amica_shard_mstep")
        return out

    @property
    def stream(self) -> int:
        """The context's cudaStream_t, as an integer handle."""
        h = C.c_void_p()
        _chk(lib().amica_get_stream(self._ctx, C.byref(h)), "amica_get_stream")
        return int(h.value or 0)

    def shard_colsum(self, d_sums: int) -> None:
        """Column sums of this shard's raw data into device memory (n doubles)."""
        _chk(lib().amica_shard_colsum(self._ctx, C.c_void_p(d_sums)), "amica_shard_colsum")

    def shard_scatter(self, d_sums_total: int, T_total: int, d_scatter: int) -> None:
        """Mean from the column sums of all shards; this shard's scatter about
        it into device memory (n x n doubles)."""
        _chk(lib().amica_shard_scatter(self._ctx, C.c_void_p(d_sums_total), int(T_total),
                                       C.c_void_p(d_scatter)), "amica_shard_scatter")

    def shard_sphere(self, d_scatter_total: int, T_total: int) -> None:
        """Sphering from the scatter of all shards, applied to this shard."""
        _chk(lib().amica_shard_sphere(self._ctx, C.c_void_p(d_scatter_total), int(T_total)),
             "amica_shard_sphere")

    @property
    def stats_len(self) -> int:
        return int(lib().amica_stats_len(self.n, self.M, self.m))

    def arm_wait_fault(self, wait_cycles: int) -> None:
        """Test hook: the next preprocess() has one missed grid-barrier arrival
        and waits bounded by wait_cycles (amica_test_arm_wait_fault)."""
        _chk(lib().amica_test_arm_wait_fault(self._ctx, int(wait_cycles)), "amica_test_arm_wait_fault")

    def set_tile_shape(self, shape: int) -> None:
        """The fused E-step's tile shape (amica_set_tile_shape): 0, 1 or 2."""
        _chk(lib().amica_set_tile_shape(self._ctx, int(shape)), "amica_set_tile_shape")

    def set_grid(self, max_clusters: int) -> int:
        """Cap the E-step grid at max_clusters clusters (0: all that fit); returns
        the grid in effect."""
        k = _i64()
        _chk(lib().amica_set_grid(self._ctx, max_clusters, C.byref(k)), "amica_set_grid")
        return int(k.value)

    def run_async(self, iters: int) -> None:
        """Enqueue `iters` iterations on this context's stream and return at once."""
        _chk(lib().amica_run_async(self._ctx, iters), "amica_run_async")
        self._pending = iters

    def run_wait(self) -> list:
        """Wait for the iterations of the last run_async and return their records."""
        iters = getattr(self, "_pending", 0)
        outs = (IterOut * max(iters, 1))()
        _chk(lib().amica_run_wait(self._ctx, outs), "amica_run_wait")
        self._pending = 0
        return [outs[k] for k in range(iters)]

    # -- state -------------------------------------------------------------
    def params(self) -> dict:
        n, M, m = self.n, self.M, self.m
        out = dict(A=np.empty((M, n, n)), W=np.empty((M, n, n)), c=np.empty((M, n)),
                   gm=np.empty(M), alpha=np.empty((M, m, n)), mu=np.empty((M, m, n)),
                   beta=np.empty((M, m, n)), rho=np.empty((M, m, n)))
        _chk(lib().amica_get_params(self._ctx, *[_p(out[k]) for k in
                                                 ("A", "W", "c", "gm", "alpha", "mu", "beta",
                                                  "rho")]), "amica_get_params")
        return out

    def set_params(self, **kw) -> None:
        args = []
        for k in ("A", "c", "gm", "alpha", "mu", "beta", "rho"):
            v = kw.get(k)
            args.append(None if v is None else np.ascontiguousarray(v, dtype=np.float64))
        self._keep = args
        _chk(lib().amica_set_params(self._ctx, *[_p(a) for a in args]), "amica_set_params")

    def estep_stats(self) -> np.ndarray:
        L = lib().amica_stats_len(self.n, self.M, self.m)
        s = np.empty(L)
        _chk(lib().amica_estep_stats(self._ctx, _p(s)), "amica_estep_stats")
        return s

    def loglik(self):
        Lt = np.empty((self.M, self.T))
        P = np.empty(self.T)
        keep = np.empty(self.T, dtype=np.uint8)
        _chk(lib().amica_get_loglik(self._ctx, _p(Lt), _p(P), keep.ctypes.data_as(_pu8)),
             "amica_get_loglik")
        return Lt, P, keep

    def p_relative(self) -> np.ndarray:
        P = np.empty(self.T, dtype=np.float32)
        _chk(lib().amica_get_p_relative(self._ctx, P.ctypes.data_as(_pf)), "amica_get_p_relative")
        return P

    def set_iter_state(self, iter: int, lrate: float, ll_prev: float) -> None:
        _chk(lib().amica_set_iter_state(self._ctx, iter, lrate, ll_prev), "amica_set_iter_state")

    def sphere(self):
        S = np.empty((self.n, self.n))
        means = np.empty(self.n)
        ld = np.empty(1)
        _chk(lib().amica_get_sphere(self._ctx, _p(S), _p(means), _p(ld)), "amica_get_sphere")
        return S.T.copy(), means, float(ld[0])

    def time_estep(self, reps: int = 10):
        ms = np.empty(1)
        nl = _i64()
        _chk(lib().amica_time_estep(self._ctx, reps, _p(ms), C.byref(nl)), "amica_time_estep")
        return float(ms[0]), int(nl.value)

    @property
    def launches_per_iteration(self) -> int:
        return int(lib().amica_launches_per_iteration(self._ctx))

    def reject_now(self) -> int:
        k = _i64()
        _chk(lib().amica_reject_now(self._ctx, C.byref(k)), "amica_reject_now")
        return int(k.value)

    def adjoint(self):
        n, M, m = self.n, self.M, self.m
        ll = np.empty(1)
        dW = np.empty((M, n, n))
        dmu = np.empty((M, m, n))
        dbeta = np.empty((M, m, n))
        drho = np.empty((M, m, n))
        _chk(lib().amica_loglik_adjoint(self._ctx, _p(ll), _p(dW), _p(dmu), _p(dbeta), _p(drho)),
             "amica_loglik_adjoint")
        return float(ll[0]), dict(W=dW, mu=dmu, beta=dbeta, rho=drho)

    def write_outputs(self, **paths) -> None:
        p = Paths(**{k: (v.encode() if v else None) for k, v in paths.items()})
        _chk(lib().amica_write_outputs(self._ctx, C.byref(p)), "amica_write_outputs")


class PersistentCohort:
    """Single-model fits (mixed form, same m) advanced together with one
    persistent E-step launch per iteration over all their sample tiles
    (amica_cohort_*).  The engines stay usable on their own; this object does
    not own them."""

    def __init__(self, engines):
        self.engines = list(engines)
        arr = (C.c_void_p * len(self.engines))(*[e._ctx for e in self.engines])
        h = C.c_void_p()
        _chk(lib().amica_cohort_create(arr, len(self.engines), C.byref(h)), "amica_cohort_create")
        self._h = h

    def run(self, iters: int):
        """`iters` iterations of every subject: (records per subject, ms per
        cohort iteration on the device)."""
        S = len(self.engines)
        outs = (IterOut * max(S * iters, 1))()
        ms = _dbl()
        _chk(lib().amica_cohort_run(self._h, iters, outs, C.byref(ms)), "amica_cohort_run")
        return [[outs[s * iters + k] for k in range(iters)] for s in range(S)], float(ms.value)

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().amica_cohort_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
