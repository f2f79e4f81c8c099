"""ctypes wrapper over liboracle.so -- TEST INFRASTRUCTURE ONLY.

The FP64 CPU oracle (amica_oracle.c) restates the reference's EM iteration
(fraimondo/cudamica src/amica.cu:820-2541).  Only tests/, the smoke check and
bench.py's CPU-baseline leg import this module, as the checker; the engine in
cudamica_b200/ never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
LIB32_PATH = os.path.join(HERE, "liboracle32.so")

_i64 = C.c_int64
_dbl = C.c_double
_pd = C.POINTER(C.c_double)
_pu8 = C.POINTER(C.c_uint8)


class Cfg(C.Structure):
    _fields_ = [(k, _i64) for k in (
        "n", "T", "M", "m", "do_newton", "update_rho", "rho_start_iter", "newt_start_iter",
        "maxdec", "update_gm", "update_alpha", "update_A", "update_mu", "update_beta",
        "do_reparm", "do_reject", "rejstart", "rejint", "maxrej", "ref_y_slab_bug", "nthreads")]
    _fields_ += [(k, _dbl) for k in (
        "lrate0", "lratemax", "lnatrate", "lratefact", "rho0", "rholrate", "rhomin", "rhomax",
        "rejsig")]


class State(C.Structure):
    _fields_ = [(k, _pd) for k in ("A", "c", "alpha", "mu", "beta", "rho", "gm", "W", "ldet")]
    _fields_ += [("keep", _pu8), ("Lt", _pd), ("P", _pd)]
    _fields_ += [(k, _dbl) for k in ("ldetS", "lrate", "lratemax", "ll_prev", "ll")]
    _fields_ += [(k, _i64) for k in ("numdec", "iter", "nrej", "newton", "nkeep")]


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE], check=True)


_libs = {}


def lib(fp32: bool = False):
    """liboracle.so, or with fp32=True liboracle32.so: the same iteration with
    its E-step's per-sample arithmetic in FP32 (sums over samples in FP64)."""
    if fp32 not in _libs:
        path = LIB32_PATH if fp32 else LIB_PATH
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        L.amo_stats_len.restype = _i64
        L.amo_stats_len.argtypes = [_i64, _i64, _i64]
        L.amo_default_cfg.argtypes = [C.POINTER(Cfg)]
        for f in ("amo_prepare",):
            getattr(L, f).argtypes = [C.POINTER(Cfg), C.POINTER(State)]
        for f in ("amo_estep", "amo_em_step"):
            getattr(L, f).argtypes = [C.POINTER(Cfg), C.POINTER(State), _pd, _pd]
        L.amo_mstep.argtypes = [C.POINTER(Cfg), C.POINTER(State), _pd]
        L.amo_reject.restype = _i64
        L.amo_reject.argtypes = [_pd, _pu8, _i64, _dbl, _pd, _pd]
        L.amo_preprocess.argtypes = [C.POINTER(C.c_float), _i64, _i64, _i64, _pd, _pd, _pd, _pd]
        L.amo_jacobi_eig.argtypes = [_pd, _i64, _pd, _pd]
        L.amo_psi.restype = _dbl
        L.amo_psi.argtypes = [_dbl]
        _libs[fp32] = L
    return _libs[fp32]


def _p(a):
    return a.ctypes.data_as(_pd)


def stats_len(n, M, m) -> int:
    return int(lib().amo_stats_len(n, M, m))


def stats_offsets(n: int, m: int) -> dict:
    mn = m * n
    o = dict(vs=0, cn=1, s2=1 + n, phi=1 + 2 * n)
    o["us"] = o["phi"] + n * n
    for k, nk in (("kn", "us"), ("ln", "kn"), ("mn", "ln"), ("md", "mn"), ("bd", "md"),
                  ("rn", "bd")):
        o[k] = o[nk] + mn
    o["S"] = o["rn"] + mn
    return o


def split_stats(stats: np.ndarray, n: int, M: int, m: int) -> dict:
    """Flat stats vector -> dict of named per-model arrays."""
    o = stats_offsets(n, m)
    out = {"llsum": float(stats[0])}
    names = {"vs": (1,), "cn": (n,), "s2": (n,), "phi": (n, n), "us": (m, n), "kn": (m, n),
             "ln": (m, n), "mn": (m, n), "md": (m, n), "bd": (m, n), "rn": (m, n)}
    for key, shp in names.items():
        sz = int(np.prod(shp))
        out[key] = np.stack([stats[1 + h * o["S"] + o[key]: 1 + h * o["S"] + o[key] + sz]
                             .reshape(shp) for h in range(M)])
    return out


def psi(x: float) -> float:
    return float(lib().amo_psi(float(x)))


def preprocess(x: np.ndarray, do_sphere: int = 1):
    x = np.ascontiguousarray(x, dtype=np.float32)
    T, n = x.shape
    xs = np.empty((T, n))
    means = np.empty(n)
    S = np.empty((n, n))
    ld = np.empty(1)
    lib().amo_preprocess(x.ctypes.data_as(C.POINTER(C.c_float)), n, T, do_sphere,
                         _p(xs), _p(means), _p(S), _p(ld))
    return xs, means, S.T.copy(), float(ld[0])   # S returned row-major (S[i, k])


def jacobi_eig(Cm: np.ndarray):
    Cm = np.ascontiguousarray(Cm, dtype=np.float64)
    n = Cm.shape[0]
    ev = np.empty(n)
    V = np.empty((n, n))
    lib().amo_jacobi_eig(_p(Cm), n, _p(ev), _p(V))
    return ev, V.T.copy()   # V[:, e] = eigenvector e


def reject(P: np.ndarray, keep: np.ndarray, rejsig: float):
    P = np.ascontiguousarray(P, dtype=np.float64)
    k = np.ascontiguousarray(keep, dtype=np.uint8).copy()
    mean = np.empty(1)
    sd = np.empty(1)
    dropped = lib().amo_reject(_p(P), k.ctypes.data_as(_pu8), P.shape[0], float(rejsig),
                               _p(mean), _p(sd))
    return k, int(dropped), float(mean[0]), float(sd[0])


class Oracle:
    """Holds the parameter arrays of one fit and steps it with the C oracle."""

    def __init__(self, xs: np.ndarray, M: int, m: int, A0: np.ndarray, c0: np.ndarray,
                 ldetS: float, nthreads: int = 8, keep_P: bool = True, keep_Lt: bool = False,
                 fp32: bool = False, **cfg_over):
        self.x = np.ascontiguousarray(xs, dtype=np.float64)
        T, n = self.x.shape
        self.n, self.T, self.M, self.m = n, T, M, m
        self._L = L = lib(fp32)
        self.cfg = Cfg()
        L.amo_default_cfg(C.byref(self.cfg))
        self.cfg.n, self.cfg.T, self.cfg.M, self.cfg.m = n, T, M, m
        self.cfg.nthreads = nthreads
        for k, v in cfg_over.items():
            setattr(self.cfg, k, v)
        self.A = np.ascontiguousarray(A0, dtype=np.float64).reshape(M, n, n).copy()
        self.c = np.ascontiguousarray(c0, dtype=np.float64).reshape(M, n).copy()
        self.alpha = np.full((M, m, n), 1.0 / m)
        # fix_init: mu_j = j - (m-1)/2, beta = 1, rho = rho0 (src/amica.cu:337-394)
        self.mu = np.repeat((np.arange(m) - (m - 1) / 2.0)[None, :, None], M, 0).repeat(n, 2).copy()
        self.beta = np.ones((M, m, n))
        self.rho = np.full((M, m, n), self.cfg.rho0)
        self.gm = np.full(M, 1.0 / M)
        self.W = np.zeros((M, n, n))
        self.ldet = np.zeros(M)
        self.keep = np.ones(T, dtype=np.uint8)
        self.P = np.zeros(T) if keep_P else None
        self.Lt = np.zeros((M, T)) if keep_Lt else None
        self.stats = np.zeros(stats_len(n, M, m))
        self.st = State()
        for k in ("A", "c", "alpha", "mu", "beta", "rho", "gm", "W", "ldet"):
            setattr(self.st, k, _p(getattr(self, k)))
        self.st.keep = self.keep.ctypes.data_as(_pu8)
        self.st.P = _p(self.P) if self.P is not None else _pd()
        self.st.Lt = _p(self.Lt) if self.Lt is not None else _pd()
        self.st.ldetS = ldetS
        self.st.lrate = self.cfg.lrate0
        self.st.lratemax = self.cfg.lratemax
        self.ll_hist: list[float] = []
        self.lrate_hist: list[float] = []

    def step(self) -> float:
        self.lrate_hist.append(self.st.lrate)
        rc = self._L.amo_em_step(C.byref(self.cfg), C.byref(self.st), _p(self.x), _p(self.stats))
        if rc != 0:
            raise RuntimeError(f"oracle step failed: {rc}")
        self.ll_hist.append(self.st.ll)
        return self.st.ll

    def prepare(self) -> None:
        rc = self._L.amo_prepare(C.byref(self.cfg), C.byref(self.st))
        if rc != 0:
            raise RuntimeError(f"oracle prepare failed: {rc}")

    def estep(self) -> np.ndarray:
        """Sufficient statistics at the current parameters (after prepare())."""
        rc = self._L.amo_estep(C.byref(self.cfg), C.byref(self.st), _p(self.x), _p(self.stats))
        if rc != 0:
            raise RuntimeError(f"oracle estep failed: {rc}")
        return self.stats.copy()

    def mstep(self, stats: np.ndarray, nkeep: int | None = None) -> float:
        """The M-step from a statistics vector (e.g. the sum of several shards'
        estep() vectors), normalised by nkeep samples (default: this oracle's)."""
        if nkeep is not None:
            self.st.nkeep = int(nkeep)
        self.lrate_hist.append(self.st.lrate)
        s = np.ascontiguousarray(stats, dtype=np.float64)
        rc = self._L.amo_mstep(C.byref(self.cfg), C.byref(self.st), _p(s))
        if rc != 0:
            raise RuntimeError(f"oracle mstep failed: {rc}")
        self.ll_hist.append(self.st.ll)
        return self.st.ll

    def params(self) -> dict:
        return dict(A=self.A.copy(), c=self.c.copy(), alpha=self.alpha.copy(), mu=self.mu.copy(),
                    beta=self.beta.copy(), rho=self.rho.copy(), gm=self.gm.copy(),
                    W=self.W.copy(), ldet=self.ldet.copy())
