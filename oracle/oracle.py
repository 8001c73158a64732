"""ctypes binding of the CPU FP64 oracle (TEST INFRASTRUCTURE ONLY).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference arm
import this module; the product path (libpmcmc_deer.so and the `pmcmc` package)
never does.  Parity status: "parity unpinned" against reference outputs (the
reference ships no golden vectors and Julia is absent); the restatement is
pinned by the reference's property tests and by the NumPy restatement in
np_oracle.py.

Array convention: a Julia D x T matrix (column t = state t, contiguous) is a
NumPy array of shape (D, T) in Fortran order, i.e. the transpose view of a
C-contiguous (T, D) buffer.  Logistic X is N x D Fortran-ordered, as in
bayes_logreg.jl.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

DIAG_GAUSS, DENSE_GAUSS, LOGISTIC = 0, 1, 2
JAC = {"stoch_diag": 0, "diag": 1, "full": 2}

_dp = C.POINTER(C.c_double)
_fp = C.POINTER(C.c_float)
_ip = C.POINTER(C.c_int32)


class _Target(C.Structure):
    _fields_ = [
        ("kind", C.c_int32), ("D", C.c_int64), ("N", C.c_int64),
        ("mean", _dp), ("prec", _dp), ("X", _dp), ("y", _dp), ("prior_prec", C.c_double),
    ]


class _Params(C.Structure):
    _fields_ = [
        ("eps", C.c_double), ("tol_abs", C.c_double), ("tol_rel", C.c_double),
        ("maxiter", C.c_int32), ("jacobian", C.c_int32), ("damping", C.c_double),
        ("probes", C.c_int32), ("batched", C.c_int32), ("scan_doubling", C.c_int32),
        ("window", C.c_int64), ("nthreads", C.c_int32),
    ]


class _Info(C.Structure):
    _fields_ = [("iters", C.c_int32), ("converged", C.c_int32), ("metric", C.c_double)]


def build() -> str:
    """Compile liboracle.so with the committed Makefile (gcc, OpenMP)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return os.path.join(_HERE, "liboracle.so")


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        src = os.path.join(_HERE, "pmcmc_oracle.c")
        if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
            build()
        L = C.CDLL(path)
        L.orc_philox4x32_10.argtypes = [C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                        C.POINTER(C.c_uint32)]
        L.orc_u01.restype = C.c_float
        L.orc_u01.argtypes = [C.c_uint32]
        L.orc_logf.restype = C.c_float
        L.orc_logf.argtypes = [C.c_float]
        L.orc_sincos2pi.argtypes = [C.c_float, _fp, _fp]
        L.orc_tape.argtypes = [C.c_uint64, C.c_uint64, C.c_int64, C.c_int64, _fp, _fp]
        L.orc_probe.argtypes = [C.c_uint64, C.c_uint64, C.c_int32, C.c_int32, C.c_int64,
                                C.c_int64, _dp]
        L.orc_logp.restype = C.c_double
        L.orc_logp.argtypes = [C.POINTER(_Target), _dp]
        L.orc_grad.argtypes = [C.POINTER(_Target), _dp, _dp]
        L.orc_hvp.argtypes = [C.POINTER(_Target), _dp, _dp, _dp]
        L.orc_logq.restype = C.c_double
        L.orc_logq.argtypes = [C.POINTER(_Target), _dp, _dp, _dp, C.c_double]
        L.orc_mala_step.restype = C.c_double
        L.orc_mala_step.argtypes = [C.POINTER(_Target), C.c_double, _dp, _dp, C.c_double,
                                    _dp, _ip]
        L.orc_mala_sequential.argtypes = [C.POINTER(_Target), C.c_double, _dp, _dp, _dp,
                                          C.c_int64, _dp, _ip, _dp]
        L.orc_mala_sequential_mass.argtypes = [C.POINTER(_Target), C.c_double, _dp, _dp, _dp,
                                               _dp, C.c_int64, _dp, _ip, _dp]
        L.orc_mala_sequential_logistic.argtypes = [C.POINTER(_Target), C.c_double, _dp, _dp,
                                                   _dp, C.c_int64, _dp, _ip, _dp, C.c_int32]
        L.orc_fwd_and_jvp.argtypes = [C.POINTER(_Target), C.c_double, _dp, _dp, C.c_double,
                                      _dp, _dp, _dp]
        L.orc_fwd_and_jvp_batched.argtypes = [C.POINTER(_Target), C.c_double, C.c_int64, _dp,
                                              _dp, _dp, _dp, _dp, _dp, C.c_int32]
        L.orc_jac_full.argtypes = [C.POINTER(_Target), C.c_double, _dp, _dp, C.c_double,
                                   _dp, _dp]
        L.orc_scan_seq.argtypes = [C.c_int64, C.c_int64, _dp, _dp, _dp, _dp]
        L.orc_scan_doubling.argtypes = [C.c_int64, C.c_int64, _dp, _dp, _dp, _dp, _dp]
        L.orc_scan_residual.restype = C.c_double
        L.orc_scan_residual.argtypes = [C.c_int64, C.c_int64, _dp, _dp, _dp, _dp]
        L.orc_scan_dense_seq.argtypes = [C.c_int64, C.c_int64, _dp, _dp, _dp, _dp]
        L.orc_deer_update.restype = C.c_int
        L.orc_deer_update.argtypes = [C.POINTER(_Target), C.POINTER(_Params), C.c_int64, _dp,
                                      _dp, _dp, _dp, C.c_uint64, C.c_uint64, C.c_int32, _dp,
                                      _dp, _dp]
        L.orc_deer_solve.restype = C.c_int
        L.orc_deer_solve.argtypes = [C.POINTER(_Target), C.POINTER(_Params), C.c_int64, _dp,
                                     _dp, _dp, C.c_uint64, C.c_uint64, _dp, C.POINTER(_Info)]
        _LIB = L
    return _LIB


def _p(a, ty=_dp):
    return a.ctypes.data_as(ty) if a is not None else None


def _col(a, D=None, T=None):
    """(D, T) array -> C-contiguous (T, D) float64 buffer (Julia column-major D x T)."""
    a = np.asarray(a, dtype=np.float64)
    if a.ndim == 1:
        return np.ascontiguousarray(a)
    return np.ascontiguousarray(a.T)


class Target:
    """Oracle-side target descriptor (keeps the arrays alive)."""

    def __init__(self, kind, D, prec=None, mean=None, X=None, y=None, prior_prec=1.0):
        self.kind, self.D = kind, int(D)
        self.mean = None if mean is None else np.ascontiguousarray(mean, dtype=np.float64)
        if kind == DENSE_GAUSS:
            self.prec = np.ascontiguousarray(np.asarray(prec, dtype=np.float64).T)  # col-major
        elif prec is not None:
            self.prec = np.ascontiguousarray(prec, dtype=np.float64)
        else:
            self.prec = None
        self.X = None if X is None else np.ascontiguousarray(np.asarray(X, np.float64).T)
        self.y = None if y is None else np.ascontiguousarray(y, dtype=np.float64)
        self.N = 0 if X is None else int(np.asarray(X).shape[0])
        self.prior_prec = float(prior_prec)
        self.s = _Target(kind, self.D, self.N, _p(self.mean), _p(self.prec), _p(self.X),
                         _p(self.y), self.prior_prec)

    @staticmethod
    def diag_gauss(prec, mean=None):
        return Target(DIAG_GAUSS, len(prec), prec=prec, mean=mean)

    @staticmethod
    def dense_gauss(prec, mean=None):
        return Target(DENSE_GAUSS, np.asarray(prec).shape[0], prec=prec, mean=mean)

    @staticmethod
    def logistic(X, y, prior_prec=1.0):
        return Target(LOGISTIC, np.asarray(X).shape[1], X=X, y=y, prior_prec=prior_prec)

    def ref(self):
        return C.byref(self.s)


# ---------------------------------------------------------------- tape / RNG
def philox(ctr, key):
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    lib().orc_philox4x32_10(c, k, o)
    return [o[i] for i in range(4)]


def tape(seed, block, D, T):
    """Tape (Xi as (D, T) float32 view of a (T, D) buffer, u as (T,) float32)."""
    Xi = np.empty((T, D), dtype=np.float32)
    u = np.empty(T, dtype=np.float32)
    lib().orc_tape(seed, block, D, T, _p(Xi, _fp), _p(u, _fp))
    return Xi.T, u


def probe(seed, block, it, k, D, T):
    Z = np.empty((T, D), dtype=np.float64)
    lib().orc_probe(seed, block, it, k, D, T, _p(Z))
    return Z.T


# ---------------------------------------------------------------- MALA
def logp(tg, x):
    x = np.ascontiguousarray(x, np.float64)
    return lib().orc_logp(tg.ref(), _p(x))


def grad(tg, x):
    x = np.ascontiguousarray(x, np.float64)
    g = np.empty_like(x)
    lib().orc_grad(tg.ref(), _p(x), _p(g))
    return g


def hvp(tg, x, v):
    x = np.ascontiguousarray(x, np.float64)
    v = np.ascontiguousarray(v, np.float64)
    o = np.empty_like(x)
    lib().orc_hvp(tg.ref(), _p(x), _p(v), _p(o))
    return o


def mala_step(tg, eps, x, xi, u):
    x = np.ascontiguousarray(x, np.float64)
    xi = np.ascontiguousarray(xi, np.float64)
    xn = np.empty_like(x)
    a = C.c_int32()
    la = lib().orc_mala_step(tg.ref(), eps, _p(x), _p(xi), float(u), _p(xn), C.byref(a))
    return xn, bool(a.value), la


def mala_sequential(tg, eps, x0, Xi, u):
    """Sequential taped MALA: returns S (D, T), accepted (T,), logalpha (T,)."""
    Xi_c = _col(Xi)
    T, D = Xi_c.shape
    u = np.ascontiguousarray(u, np.float64)
    x0 = np.ascontiguousarray(x0, np.float64)
    S = np.empty((T, D))
    acc = np.empty(T, np.int32)
    la = np.empty(T)
    lib().orc_mala_sequential(tg.ref(), eps, _p(x0), _p(Xi_c), _p(u), T, _p(S),
                              _p(acc, _ip), _p(la))
    return S.T, acc.astype(bool), la


def dual_average(eps_init, eps_bar, h_bar, m, la, target_accept=0.574, gamma=0.05, t0=10.0,
                 kappa=0.75):
    """_dual_average_update (src/interface.jl:962-984): (eps, eps_bar, H_bar)
    after step m (m >= 1) with log acceptance ratio la."""
    alpha = 1.0 if la >= 0 else math.exp(la)
    mu = math.log(10.0 * eps_init)
    w = 1.0 / (m + t0)
    h_new = (1.0 - w) * h_bar + w * (target_accept - alpha)
    log_eps = mu - math.sqrt(m) / gamma * h_new
    mk = m ** (-kappa)
    log_eps_bar = mk * log_eps + (1.0 - mk) * math.log(eps_bar)
    return math.exp(log_eps), math.exp(log_eps_bar), h_new


def mala_adaptive(tg, eps_init, x0, Xi, u, n_warmup, **settings):
    """AdaptiveMALASampler's chain (src/interface.jl:1024-1065) on a fixed tape:
    step m uses eps while m < n_warmup and eps_bar after, and during warmup is
    followed by dual_average with m + 1.  Returns S (D, T), accepted (T,),
    step sizes (T,) and the final (eps, eps_bar, H_bar)."""
    Xi_c = _col(Xi)
    T, D = Xi_c.shape
    x = np.asarray(x0, np.float64)
    eps = eps_bar = float(eps_init)
    h_bar = 0.0
    S = np.empty((D, T))
    acc = np.empty(T, bool)
    used = np.empty(T)
    for t in range(T):
        warm = t < n_warmup
        e = eps if warm else eps_bar
        x, acc[t], la = mala_step(tg, e, x, Xi_c[t], float(u[t]))
        if warm:
            eps, eps_bar, h_bar = dual_average(eps_init, eps_bar, h_bar, t + 1, la, **settings)
        S[:, t] = x
        used[t] = e
    return S, acc, used, (eps, eps_bar, h_bar)


def mala_sequential_mass(tg, eps, Lfac, x0, Xi, u):
    """Sequential MALA with mass matrix M = L L^T (L lower triangular): returns
    S (D, T), accepted (T,), logalpha (T,)."""
    Xi_c = _col(Xi)
    T, D = Xi_c.shape
    Lc = np.ascontiguousarray(np.asarray(Lfac, np.float64).T)  # column-major
    u = np.ascontiguousarray(u, np.float64)
    x0 = np.ascontiguousarray(x0, np.float64)
    S = np.empty((T, D))
    acc = np.empty(T, np.int32)
    la = np.empty(T)
    lib().orc_mala_sequential_mass(tg.ref(), eps, _p(Lc), _p(x0), _p(Xi_c), _p(u), T, _p(S),
                                   _p(acc, _ip), _p(la))
    return S.T, acc.astype(bool), la


def mala_sequential_logistic(tg, eps, x0, Xi, u, nthreads=0):
    """mala_sequential for a logistic target (the same results bit for bit),
    threaded and with the accepted proposal's log density and gradient reused."""
    Xi_c = _col(Xi)
    T, D = Xi_c.shape
    u = np.ascontiguousarray(u, np.float64)
    x0 = np.ascontiguousarray(x0, np.float64)
    S = np.empty((T, D))
    acc = np.empty(T, np.int32)
    la = np.empty(T)
    lib().orc_mala_sequential_logistic(tg.ref(), eps, _p(x0), _p(Xi_c), _p(u), T, _p(S),
                                       _p(acc, _ip), _p(la), int(nthreads))
    return S.T, acc.astype(bool), la


def fwd_and_jvp(tg, eps, x, xi, u, v):
    x, xi, v = (np.ascontiguousarray(a, np.float64) for a in (x, xi, v))
    f = np.empty_like(x)
    jv = np.empty_like(x)
    lib().orc_fwd_and_jvp(tg.ref(), eps, _p(x), _p(xi), float(u), _p(v), _p(f), _p(jv))
    return f, jv


def fwd_and_jvp_batched(tg, eps, X, Xi, u, Z, nthreads=0):
    Xc, Xic, Zc = _col(X), _col(Xi), _col(Z)
    T, D = Xc.shape
    u = np.ascontiguousarray(u, np.float64)
    FT = np.empty((T, D))
    Jt = np.empty((T, D))
    lib().orc_fwd_and_jvp_batched(tg.ref(), eps, T, _p(Xc), _p(Xic), _p(u), _p(Zc), _p(FT),
                                  _p(Jt), nthreads)
    return FT.T, Jt.T


def jac_full(tg, eps, x, xi, u):
    x, xi = (np.ascontiguousarray(a, np.float64) for a in (x, xi))
    D = x.shape[0]
    f = np.empty(D)
    J = np.empty((D, D))  # column-major in C == J.T here
    lib().orc_jac_full(tg.ref(), eps, _p(x), _p(xi), float(u), _p(f), _p(J))
    return f, J.T.copy()


# ---------------------------------------------------------------- scans
def scan_seq(A, B, s0):
    Ac, Bc = _col(A), _col(B)
    T, D = Ac.shape
    s0 = np.ascontiguousarray(s0, np.float64)
    S = np.empty((T, D))
    lib().orc_scan_seq(D, T, _p(Ac), _p(Bc), _p(s0), _p(S))
    return S.T


def scan_doubling(A, B, s0):
    Ac, Bc = _col(A), _col(B)
    T, D = Ac.shape
    s0 = np.ascontiguousarray(s0, np.float64)
    S = np.empty((T, D))
    ws = np.empty(4 * max(T * D, 1))
    lib().orc_scan_doubling(D, T, _p(Ac), _p(Bc), _p(s0), _p(S), _p(ws))
    return S.T


def scan_residual(S, A, B, s0):
    Sc, Ac, Bc = _col(S), _col(A), _col(B)
    T, D = Ac.shape
    s0 = np.ascontiguousarray(s0, np.float64)
    return lib().orc_scan_residual(D, T, _p(Sc), _p(Ac), _p(Bc), _p(s0))


def scan_dense_seq(J, B, s0):
    """J: (T, D, D) with J[t] the matrix of step t; B: (D, T)."""
    J = np.asarray(J, np.float64)
    T, D, _ = J.shape
    Jc = np.ascontiguousarray(np.transpose(J, (0, 2, 1)))  # column-major per step
    Bc = _col(B)
    s0 = np.ascontiguousarray(s0, np.float64)
    S = np.empty((T, D))
    lib().orc_scan_dense_seq(D, T, _p(Jc), _p(Bc), _p(s0), _p(S))
    return S.T


# ---------------------------------------------------------------- DEER
def _params(eps, tol_abs=1e-6, tol_rel=1e-5, maxiter=200, jacobian="stoch_diag",
            damping=0.5, probes=1, batched=1, scan_doubling=1, window=0, nthreads=0):
    return _Params(eps, tol_abs, tol_rel, maxiter, JAC[jacobian], damping, probes, batched,
                   scan_doubling, window, nthreads)


def deer_update(tg, eps, s0, S_in, Xi, u, seed, block, it, **kw):
    p = _params(eps, **kw)
    Sc, Xic = _col(S_in), _col(Xi)
    T, D = Sc.shape
    u = np.ascontiguousarray(u, np.float64)
    s0 = np.ascontiguousarray(s0, np.float64)
    So = np.empty((T, D))
    A = np.empty((T, D))
    B = np.empty((T, D))
    rc = lib().orc_deer_update(tg.ref(), C.byref(p), T, _p(s0), _p(Sc), _p(Xic), _p(u), seed,
                               block, it, _p(So), _p(A), _p(B))
    if rc:
        raise ValueError("invalid DEER arguments")
    return So.T, A.T, B.T


def deer_solve(tg, eps, s0, Xi, u, seed, block, **kw):
    """CPU DEER (DEER.jl:506-595); returns (S (D,T), info dict)."""
    p = _params(eps, **kw)
    Xic = _col(Xi)
    T, D = Xic.shape
    u = np.ascontiguousarray(u, np.float64)
    s0 = np.ascontiguousarray(s0, np.float64)
    S = np.empty((T, D))
    info = _Info()
    rc = lib().orc_deer_solve(tg.ref(), C.byref(p), T, _p(s0), _p(Xic), _p(u), seed, block,
                              _p(S), C.byref(info))
    if rc:
        raise ValueError("invalid DEER arguments")
    return S.T, {"iters": info.iters, "converged": bool(info.converged),
                 "metric": info.metric}
