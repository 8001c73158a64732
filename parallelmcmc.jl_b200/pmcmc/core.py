"""Host mirror of the reference's DEER-path API over the C ABI.

Mirrors (names, argument meaning, defaults and error classes):
  DensityModel          src/interface.jl:36-70
  ParallelMALASampler   src/interface.jl:248-290
  sample / mcmcsample   src/interface.jl:557-809 (block loop in libpmcmc_deer)
  step                  src/interface.jl:811-869
  DEER.solve            src/DEER/DEER.jl:506-595
  DEERScan.solve_affine_scan_diag   src/DEER/DEERScan.jl:102-191
Arrays follow the reference's layout: a D x T trajectory is returned as a
(D, T) array whose column t is state t (Fortran order in NumPy; a transposed
view of a contiguous (T, D) tensor for torch).  Host inputs may be NumPy
arrays; CUDA torch tensors are passed to the library as device pointers and
results come back as CUDA tensors.
"""
from __future__ import annotations

import ctypes as C
import hashlib
from dataclasses import dataclass, field
from typing import Any, Optional, Sequence

import numpy as np

from . import _lib as L
from ._lib import ArgumentError, DimensionMismatch


def _is_torch_cuda(x) -> bool:
    return type(x).__module__.startswith("torch") and getattr(x, "is_cuda", False)


def _torch_ready(x):
    """Wait for torch's current stream on x's device: the library runs on its
    handle's stream, which is not ordered after torch's work on x."""
    import torch
    torch.cuda.current_stream(x.device).synchronize()
    return x


def _dtype_code(dt) -> int:
    return L.F32 if np.dtype(dt) == np.float32 else L.F64


# --------------------------------------------------------------------------- mass matrix
class Cholesky:
    """cholesky(M): the lower factor L of a symmetric positive definite mass
    matrix M = L L^T, as the reference's `cholM = cholesky(M)` keyword takes it
    (src/interface.jl:84-100).  `.L` is lower, `.U` = L^T."""

    def __init__(self, M=None, *, L=None):
        if (M is None) == (L is None):
            raise ArgumentError("give the matrix M or its lower factor L")
        if L is None:
            Mm = np.asarray(M, dtype=np.float64)
            if Mm.ndim != 2 or Mm.shape[0] != Mm.shape[1]:
                raise DimensionMismatch("M must be a square matrix")
            try:
                L = np.linalg.cholesky(0.5 * (Mm + Mm.T))
            except np.linalg.LinAlgError as e:
                raise ArgumentError(f"M is not positive definite: {e}") from None
        self.L = _mass_factor(L)

    @property
    def U(self):
        return self.L.T

    @property
    def M(self):
        return self.L @ self.L.T


def cholesky(M) -> Cholesky:
    return Cholesky(M)


def _mass_factor(cholM, D: Optional[int] = None):
    """The lower factor of a cholM argument (a Cholesky, anything with `.L`, or
    a square lower-triangular array) as float64, checked."""
    Lm = getattr(cholM, "L", cholM)
    try:
        Lm = np.asarray(Lm, dtype=np.float64)
    except (TypeError, ValueError):
        raise ArgumentError("cholM must be a Cholesky factor (cholesky(M)) or a lower "
                            "triangular matrix") from None
    if Lm.ndim != 2 or Lm.shape[0] != Lm.shape[1]:
        raise DimensionMismatch("cholM must be a square factor")
    if D is not None and Lm.shape[0] != D:
        raise DimensionMismatch(f"cholM is {Lm.shape[0]} x {Lm.shape[0]}, the model has dim {D}")
    Lm = np.tril(Lm)
    if not np.all(np.isfinite(Lm)) or not np.all(np.diag(Lm) > 0):
        raise ArgumentError("cholM must be finite with a positive diagonal")
    return Lm


# --------------------------------------------------------------------------- model
class DensityModel:
    """DensityModel(logdensity, grad_logdensity, dim; param_names, hvp, *_batch).

    The device sampler needs one of the built-in targets (diag_gaussian,
    dense_gaussian, logistic); a model made only of Python closures is accepted
    for API compatibility but raises ArgumentError when sampled, because
    arbitrary closures cannot run inside the sweep kernels (no CPU fallback).
    """

    def __init__(self, logdensity=None, grad_logdensity=None, dim: Optional[int] = None, *,
                 param_names=None, hvp=None, logdensity_batch=None, grad_logdensity_batch=None,
                 hvp_batch=None, target: Optional[dict] = None):
        self.logdensity = logdensity
        self.grad_logdensity = grad_logdensity
        self.hvp = hvp
        self.logdensity_batch = logdensity_batch
        self.grad_logdensity_batch = grad_logdensity_batch
        self.hvp_batch = hvp_batch
        self.param_names = param_names
        self.target = target
        if dim is None and target is not None:
            dim = target["D"]
        if dim is None:
            raise ArgumentError("dim is required")
        self.dim = int(dim)
        self._dev: dict[int, Any] = {}
        self._mass: dict[tuple, Any] = {}

    # ---- built-in device targets
    @classmethod
    def diag_gaussian(cls, prec, mean=None, param_names=None):
        prec = np.ascontiguousarray(prec, dtype=np.float64).ravel()
        mean = None if mean is None else np.ascontiguousarray(mean, dtype=np.float64).ravel()
        D = prec.size
        if mean is not None and mean.size != D:
            raise DimensionMismatch("mean and prec must have the same length")
        m = np.zeros(D) if mean is None else mean
        return cls(lambda x: -0.5 * float(np.sum(prec * (np.asarray(x) - m) ** 2)),
                   lambda x: -prec * (np.asarray(x) - m), D, param_names=param_names,
                   hvp=lambda x, v: -prec * np.asarray(v),
                   target={"kind": "diag_gauss", "D": D, "prec": prec, "mean": mean})

    @classmethod
    def dense_gaussian(cls, prec, mean=None, param_names=None):
        P = np.asarray(prec, dtype=np.float64)
        if P.ndim != 2 or P.shape[0] != P.shape[1]:
            raise DimensionMismatch("prec must be a square matrix")
        D = P.shape[0]
        mean = None if mean is None else np.ascontiguousarray(mean, dtype=np.float64).ravel()
        if mean is not None and mean.size != D:
            raise DimensionMismatch("mean must have length D")
        m = np.zeros(D) if mean is None else mean
        return cls(lambda x: -0.5 * float((np.asarray(x) - m) @ P @ (np.asarray(x) - m)),
                   lambda x: -P @ (np.asarray(x) - m), D, param_names=param_names,
                   hvp=lambda x, v: -P @ np.asarray(v),
                   target={"kind": "dense_gauss", "D": D, "prec": P, "mean": mean})

    @classmethod
    def logistic(cls, X, y, prior_prec: float = 1.0, param_names=None):
        X = np.asarray(X, dtype=np.float64)
        y = np.ascontiguousarray(y, dtype=np.float64).ravel()
        if X.ndim != 2 or X.shape[0] != y.size:
            raise DimensionMismatch("X must be N x D with N = length(y)")
        return cls(None, None, X.shape[1], param_names=param_names,
                   target={"kind": "logistic", "D": X.shape[1], "X": X, "y": y,
                           "prior_prec": float(prior_prec)})

    def device_target(self, handle: L.Handle, cholM=None):
        """pmcmc_target* on the handle's device (created once, cached); with
        cholM, the target of the chain with that mass matrix
        (pmcmc_target_mass), cached per factor."""
        if cholM is not None:
            Lm = _mass_factor(cholM, self.dim)
            key = (id(handle), Lm.shape[0], hashlib.sha256(Lm.tobytes()).digest())
            if key not in self._mass:
                base = self.device_target(handle)
                Lf = np.asfortranarray(Lm)
                t = C.c_void_p()
                L.check(L.load().pmcmc_target_mass(handle.ptr, base, Lf.ctypes.data, C.byref(t)),
                        handle.ptr, "target_mass")
                self._mass[key] = (handle, t)
            return self._mass[key][1]
        if self.target is None:
            raise ArgumentError(
                "the GPU sampler needs a built-in device target (DensityModel.diag_gaussian, "
                ".dense_gaussian or .logistic); arbitrary closures cannot run on the device")
        key = id(handle)
        if key in self._dev:
            return self._dev[key][1]
        lib = L.load()
        t = C.c_void_p()
        tg = self.target
        if tg["kind"] == "diag_gauss":
            mean = tg["mean"]
            rc = lib.pmcmc_target_diag_gauss(handle.ptr, tg["D"],
                                             mean.ctypes.data if mean is not None else None,
                                             tg["prec"].ctypes.data, C.byref(t))
        elif tg["kind"] == "dense_gauss":
            mean = tg["mean"]
            P = np.ascontiguousarray(tg["prec"].T)  # column-major
            rc = lib.pmcmc_target_dense_gauss(handle.ptr, tg["D"],
                                              mean.ctypes.data if mean is not None else None,
                                              P.ctypes.data, C.byref(t))
        else:
            Xc = np.asfortranarray(tg["X"])
            rc = lib.pmcmc_target_logistic(handle.ptr, Xc.shape[0], Xc.shape[1], Xc.ctypes.data,
                                           tg["y"].ctypes.data, tg["prior_prec"], C.byref(t))
        L.check(rc, handle.ptr, "target")
        self._dev[key] = (handle, t)
        return t

    def eigen(self, handle: Optional[L.Handle] = None, device: int = 0):
        """(lam, Q): the precision P = Q diag(lam) Q^T of a Gaussian target as
        the :full mode and the adjoint use it (ascending lam for the dense
        target, the given order for the diagonal one)."""
        h = handle or L.default_handle(device)
        t = self.device_target(h)
        lam = np.empty(self.dim)
        Q = np.empty((self.dim, self.dim), order="F")
        L.check(L.load().pmcmc_target_eigen(t, lam.ctypes.data, Q.ctypes.data), h.ptr, "eigen")
        return lam, Q

    def __del__(self):
        try:
            for h, t in list(self._mass.values()) + list(self._dev.values()):
                if h.ptr:
                    L.load().pmcmc_target_destroy(t)
        except Exception:
            pass


# --------------------------------------------------------------------------- sampler
@dataclass
class ParallelMALASampler:
    """ParallelMALASampler(epsilon; T, maxiter, tol_abs, tol_rel, jacobian, damping,
    probes, cholM, backend) plus `window` (sliding window, 0 = off), `dtype`
    (working precision; defaults to the precision of epsilon, as
    FP = typeof(float(epsilon)) in the reference) and `exec` ("fused" product
    path or "plain" baseline)."""

    epsilon: float
    T: int = 64
    maxiter: int = 200
    tol_abs: float = 1e-6
    tol_rel: float = 1e-5
    jacobian: str = "stoch_diag"
    damping: float = 0.5
    probes: int = 1
    cholM: Any = None
    backend: Any = None
    window: int = 0
    dtype: Any = None
    exec: str = "fused"

    def __post_init__(self):
        if not (self.epsilon > 0):
            raise ArgumentError(f"epsilon must be > 0, got {self.epsilon}")
        jac = self.jacobian.lstrip(":") if isinstance(self.jacobian, str) else self.jacobian
        if jac not in ("stoch_diag", "diag", "full"):
            raise ArgumentError("jacobian must be :stoch_diag, :diag or :full")
        self.jacobian = jac
        if self.cholM is not None:
            self.cholM = Cholesky(L=_mass_factor(self.cholM))
        if self.exec not in L.EXEC:
            raise ArgumentError("exec must be 'fused' or 'plain'")
        if self.dtype is None:
            self.dtype = np.float32 if isinstance(self.epsilon, np.float32) else np.float64
        self.dtype = np.dtype(self.dtype).type
        if self.dtype not in (np.float32, np.float64):
            raise ArgumentError("dtype must be float32 or float64")
        self.epsilon = float(self.epsilon)

    def target(self, model: "DensityModel", handle: L.Handle):
        """The device target this sampler runs on `model` (with its mass matrix)."""
        return model.device_target(handle, self.cholM)

    def params(self) -> L.DeerParams:
        return L.DeerParams(self.epsilon, int(self.T), int(self.maxiter), float(self.tol_abs),
                            float(self.tol_rel), L.JAC[self.jacobian], float(self.damping),
                            int(self.probes), int(self.window), _dtype_code(self.dtype),
                            L.EXEC[self.exec])


# --------------------------------------------------------------------------- buffers
class _Out:
    """Output buffer on the device (torch) or on the host: a NumPy array backed by
    page-locked memory when torch can provide it (the library's device-to-host
    copies then run at DMA speed), else an ordinary NumPy array."""

    def __init__(self, shape, dtype, like_device: Optional[Any], pinned: bool = True):
        self.device = like_device
        tdt = None
        try:
            import torch
            tdt = {np.float32: torch.float32, np.float64: torch.float64,
                   np.uint8: torch.uint8}[np.dtype(dtype).type]
        except Exception:
            torch = None
        if like_device is not None:
            self.arr = torch.empty(shape, dtype=tdt, device=like_device)
            self.ptr = self.arr.data_ptr()
        elif pinned and torch is not None and torch.cuda.is_available():
            self._t = torch.empty(shape, dtype=tdt, pin_memory=True)
            self.arr = self._t.numpy()
            self.ptr = self.arr.ctypes.data
        else:
            self.arr = np.empty(shape, dtype=dtype)
            self.ptr = self.arr.ctypes.data


def _input_vector(x, D, dtype, device_like):
    if _is_torch_cuda(x):
        import torch
        tdt = torch.float32 if dtype == np.float32 else torch.float64
        x = x.detach().to(dtype=tdt).contiguous().reshape(-1)
        if x.numel() != D:
            raise DimensionMismatch(f"initial state must have length {D}")
        _torch_ready(x)
        return x, x.data_ptr(), L.MEM_DEVICE
    a = np.ascontiguousarray(np.asarray(x, dtype=dtype).ravel())
    if a.size != D:
        raise DimensionMismatch(f"initial state must have length {D}")
    return a, a.ctypes.data, L.MEM_HOST


@dataclass
class Chain:
    """Samples of sample(): values (N, D), logp (N,), accepted (N,), info."""
    values: Any
    logp: Any
    accepted: Any
    info: dict
    param_names: Any = None

    def __len__(self):
        return int(self.values.shape[0])


def _initial_params(model, sampler, initial_params, seed):
    if initial_params is not None:
        return initial_params
    # randn(rng, FP, dim) (interface.jl:526-530) from the seeded host RNG
    return np.random.default_rng(seed).standard_normal(model.dim).astype(sampler.dtype)


class MCMCThreads:
    """AbstractMCMC.MCMCThreads(): several chains side by side,
    sample(model, sampler, MCMCThreads(), N, nchains)."""


@dataclass
class ChainSet:
    """The chains of sample(model, sampler, MCMCThreads(), N, nchains)."""
    chains: list

    @property
    def nchains(self) -> int:
        return len(self.chains)

    @property
    def niters(self) -> int:
        return len(self.chains[0]) if self.chains else 0

    @property
    def values(self):  # (nchains, N, D)
        return np.stack([c.values for c in self.chains])


def chain_seed(seed: int, c: int) -> int:
    """Seed of chain c of a multi-chain sample() with master seed `seed`."""
    return (int(seed) * 1000003 + 7919 * int(c) + 1) % (1 << 63)


def _sample_threads(model, sampler, N, nchains, *, seed=0, initial_params=None, device=0,
                    handle=None, workers=8):
    """MCMCThreads (src/interface.jl:557-607 per chain, test/test-DEER-Interface.jl:300-318):
    chain c has seed chain_seed(seed, c) and runs exactly the blocks sample() runs for
    that seed; every round solves the next block of all chains together on the device
    fleet (pmcmc_fleet_solve), each chain continuing from its last state."""
    if N < 1 or nchains < 1:
        raise ArgumentError("N and nchains must be >= 1")
    h = handle or L.default_handle(device)
    seeds = [chain_seed(seed, c) for c in range(nchains)]
    if initial_params is None:
        x = [np.asarray(_initial_params(model, sampler, None, sd), sampler.dtype).ravel()
             for sd in seeds]
    else:
        ip = list(initial_params)
        if len(ip) != nchains:
            raise DimensionMismatch("one initial state per chain")
        x = [np.asarray(v, sampler.dtype).ravel() for v in ip]
    T = int(sampler.T)
    vals = [np.empty((N, model.dim), sampler.dtype) for _ in range(nchains)]
    logp = [np.empty(N, sampler.dtype) for _ in range(nchains)]
    acc = [np.empty(N, bool) for _ in range(nchains)]
    info = [{"iters": 0, "converged": True, "n_accept": 0} for _ in range(nchains)]
    for b in range((N + T - 1) // T):
        keep = min(T, N - b * T)
        res = fleet_solve([(model, sampler, x[c], seeds[c], b) for c in range(nchains)],
                          workers=workers, handle=h, errors="raise")
        for c, (S, inf, lp, ac) in enumerate(res):
            vals[c][b * T:b * T + keep] = S[:, :keep].T
            logp[c][b * T:b * T + keep] = lp[:keep]
            acc[c][b * T:b * T + keep] = ac[:keep]
            info[c]["iters"] += inf["iters"]
            info[c]["converged"] &= bool(inf["converged"])
            info[c]["n_accept"] += int(np.sum(ac[:keep]))
            x[c] = np.ascontiguousarray(S[:, keep - 1])
    return ChainSet([Chain(vals[c], logp[c], acc[c], dict(info[c], seed=seeds[c]),
                           model.param_names) for c in range(nchains)])


def sample(model: DensityModel, sampler: ParallelMALASampler, N, *rest, seed: int = 0,
           initial_params=None, device: int = 0, handle: Optional[L.Handle] = None,
           progress: bool = False, chain_type=None, **kw) -> Chain:
    """sample(rng, model, ParallelMALASampler(...), N): ceil(N/T) DEER blocks solved
    on the GPU, block b with tape block b of `seed` (interface.jl:557-607).  With an
    AdaptiveMALASampler: its sequential adaptive chain on the device
    (pmcmc.adapt.sample_adaptive)."""
    if isinstance(N, MCMCThreads):  # sample(model, sampler, MCMCThreads(), N, nchains)
        if len(rest) != 2:
            raise ArgumentError("sample(model, sampler, MCMCThreads(), N, nchains)")
        return _sample_threads(model, sampler, int(rest[0]), int(rest[1]), seed=seed,
                               initial_params=initial_params, device=device, handle=handle)
    if rest:
        raise ArgumentError("unexpected positional arguments")
    if type(sampler).__name__ == "AdaptiveMALASampler":
        from .adapt import sample_adaptive
        return sample_adaptive(model, sampler, N, seed=seed, initial_params=initial_params,
                               device=device, handle=handle)
    if kw.get("callback") is not None or kw.get("num_warmup", 0) or kw.get("thinning", 1) != 1 \
            or kw.get("discard_initial", 0):
        return _sample_generic(model, sampler, N, seed=seed, initial_params=initial_params,
                               device=device, handle=handle, **kw)
    if N < 1:
        raise ArgumentError("the number of samples must be >= 1")
    h = handle or L.default_handle(device)
    tgt = sampler.target(model, h)
    x0 = _initial_params(model, sampler, initial_params, seed)
    keep, x0p, mem = _input_vector(x0, model.dim, sampler.dtype, None)
    dev = x0.device if mem == L.MEM_DEVICE else None
    vals = _Out((N, model.dim), sampler.dtype, dev)
    logp = _Out((N,), sampler.dtype, dev)
    acc = _Out((N,), np.uint8, dev)
    info = L.Info()
    p = sampler.params()
    rc = L.load().pmcmc_sample(h.ptr, tgt, C.byref(p), x0p, int(seed), int(N), vals.ptr, logp.ptr,
                               acc.ptr, mem, C.byref(info))
    L.check(rc, h.ptr, "sample")
    return Chain(vals.arr, logp.arr, acc.arr.astype(bool) if dev is None else acc.arr.bool(),
                 info.as_dict(), model.param_names)


def _sample_generic(model, sampler, N, *, seed=0, initial_params=None, device=0, handle=None,
                    callback=None, num_warmup=0, discard_initial=None, thinning=1, **_):
    """The generic AbstractMCMC path (interface.jl:753-775): repeated step() calls."""
    discard_initial = num_warmup if discard_initial is None else discard_initial
    xs, lps = [], []
    state = None
    total = discard_initial + (N - 1) * thinning + 1
    for i in range(total):
        trans, state = step(model, sampler, state, seed=seed, initial_params=initial_params,
                            device=device, handle=handle)
        if callback is not None:
            callback(trans, state, i)
        if i >= discard_initial and (i - discard_initial) % thinning == 0:
            xs.append(np.asarray(trans.x))
            lps.append(float(trans.logp))
    return Chain(np.stack(xs), np.asarray(lps), None, {}, model.param_names)


@dataclass
class ParallelMALATransition:
    x: Any
    logp: float


@dataclass
class ParallelMALAState:
    x: Any
    logp: float
    trajectory: Any  # (D, T)
    logps: Any
    t: int
    block: int
    info: dict = field(default_factory=dict)


def step(model: DensityModel, sampler: ParallelMALASampler, state: Optional[ParallelMALAState] = None,
         *, seed: int = 0, initial_params=None, device: int = 0,
         handle: Optional[L.Handle] = None):
    """AbstractMCMC.step for ParallelMALASampler (interface.jl:811-869): the first
    call solves a block and returns column 1; later calls walk the cached
    trajectory and re-solve from column T when it is exhausted."""
    h = handle or L.default_handle(device)
    if state is not None and state.t + 1 <= sampler.T:
        t = state.t + 1
        x = state.trajectory[:, t - 1]
        lp = float(state.logps[t - 1])
        return ParallelMALATransition(x, lp), ParallelMALAState(
            x, lp, state.trajectory, state.logps, t, state.block, state.info)
    if state is None:
        x0 = _initial_params(model, sampler, initial_params, seed)
        blk = 0
    else:
        x0 = state.trajectory[:, sampler.T - 1]
        blk = state.block + 1
    S, info, logps, _ = solve(model, sampler, x0, seed=seed, block=blk, handle=h,
                              return_logp=True)
    x = S[:, 0]
    lp = float(logps[0])
    return ParallelMALATransition(x, lp), ParallelMALAState(x, lp, S, logps, 1, blk, info)


# --------------------------------------------------------------------------- DEER.solve
def solve(model: DensityModel, sampler: ParallelMALASampler, s0, *, seed: int = 0,
          block: int = 0, handle: Optional[L.Handle] = None, device: int = 0,
          return_logp: bool = False):
    """One DEER block (the body of _deer_solve_new_tape + DEER.solve with
    return_info=true): returns S (D, T), info and, with return_logp, logp (T,)
    and the accept flags (T,)."""
    h = handle or L.default_handle(device)
    tgt = sampler.target(model, h)
    keep, x0p, mem = _input_vector(s0, model.dim, sampler.dtype, None)
    dev = s0.device if mem == L.MEM_DEVICE else None
    T = int(sampler.T)
    S = _Out((T, model.dim), sampler.dtype, dev)
    lp = _Out((T,), sampler.dtype, dev)
    acc = _Out((T,), np.uint8, dev)
    info = L.Info()
    p = sampler.params()
    rc = L.load().pmcmc_deer_solve(h.ptr, tgt, C.byref(p), x0p, int(seed), int(block), S.ptr,
                                   lp.ptr, acc.ptr, mem, C.byref(info))
    L.check(rc, h.ptr, "deer_solve")
    Sv = S.arr.T
    accepted = acc.arr.astype(bool) if dev is None else acc.arr.bool()
    if return_logp:
        return Sv, info.as_dict(), lp.arr, accepted
    return Sv, info.as_dict()


# --------------------------------------------------------------------------- autotuning
def autotune(model: DensityModel, sampler: ParallelMALASampler, x0, *, seed: int = 0,
             handle: Optional[L.Handle] = None, device: int = 0) -> dict:
    """Time the candidate kernel shapes for this problem on the device and keep
    the fastest for later solves of the same shape (pmcmc_autotune).  Returns
    {"choice": kept value (CTAs a SM, or :full chunk count; 0 if nothing to
    tune), "ms": its time a solve}."""
    h = handle or L.default_handle(device)
    tgt = sampler.target(model, h)
    keep, x0p, mem = _input_vector(x0, model.dim, sampler.dtype, None)
    ch = C.c_int32(0)
    ms = C.c_double(0.0)
    p = sampler.params()
    L.check(L.load().pmcmc_autotune(h.ptr, tgt, C.byref(p), x0p, int(seed), mem, C.byref(ch),
                                    C.byref(ms)), h.ptr, "autotune")
    return {"choice": int(ch.value), "ms": float(ms.value)}


# --------------------------------------------------------------------------- sequential chains
def mala_chains(model: DensityModel, sampler: ParallelMALASampler, x0s, seeds, *,
                block: int = 0, handle: Optional[L.Handle] = None, device: int = 0):
    """n independent sequential MALA chains of sampler.T steps on the device,
    one warp a chain (the reference's MALASampler chains run side by side,
    MALA.jl:322-346, 377-411).  x0s: (n, D); seeds: (n,).  Chain c uses the
    tape of (seeds[c], block), the tape DEER uses for that seed and block.
    Returns S (n, T, D), logp (n, T) and accept flags (n, T)."""
    h = handle or L.default_handle(device)
    tgt = sampler.target(model, h)
    x = np.ascontiguousarray(np.asarray(x0s, dtype=sampler.dtype).reshape(-1, model.dim))
    n = x.shape[0]
    sd = np.ascontiguousarray(np.asarray(seeds, dtype=np.uint64).reshape(-1))
    if sd.size != n:
        raise DimensionMismatch("one seed per chain")
    T = int(sampler.T)
    S = np.empty((n, T, model.dim), sampler.dtype)
    lp = np.empty((n, T), sampler.dtype)
    acc = np.empty((n, T), np.uint8)
    p = sampler.params()
    rc = L.load().pmcmc_mala_chains(h.ptr, tgt, C.byref(p), n, x.ctypes.data, sd.ctypes.data,
                                    int(block), S.ctypes.data, lp.ctypes.data, acc.ctypes.data,
                                    L.MEM_HOST)
    L.check(rc, h.ptr, "mala_chains")
    return S, lp, acc.astype(bool)


# --------------------------------------------------------------------------- adjoint
def adjoint(model: DensityModel, sampler: ParallelMALASampler, s0, S, *, objective: str = "esjd",
            seed: int = 0, block: int = 0, handle: Optional[L.Handle] = None, device: int = 0):
    """Gradient of an objective of the solved trajectory S (D, T) with the
    accept decisions of S held fixed (one reverse scan on the device).

    objective "esjd":    (1/T) sum_t min(1, alpha_t) |y_t - x_{t-1}|^2
    objective "mean_sq": (1/T) sum_t |x_t|^2
    Returns {"d_epsilon": float, "d_log_s": (D,) or None}; d_log_s is the
    gradient with respect to the log covariance eigenvalues s_i = 1/lam_i in
    the order of DensityModel.eigen (mean_sq, Gaussian targets only).  The logistic
    target (FP32 or FP64 state) gives d_epsilon alone."""
    if objective not in L.OBJECTIVE:
        raise ArgumentError("objective must be 'esjd' or 'mean_sq'")
    h = handle or L.default_handle(device)
    tgt = sampler.target(model, h)
    keep, x0p, mem = _input_vector(s0, model.dim, sampler.dtype, None)
    if mem == L.MEM_DEVICE:
        Sc = _torch_ready(S.T.contiguous())
        sp = Sc.data_ptr()
    else:
        Sc = np.ascontiguousarray(np.asarray(S).T, dtype=sampler.dtype)
        sp = Sc.ctypes.data
    if tuple(Sc.shape) != (int(sampler.T), model.dim):
        raise DimensionMismatch("S must be D x T")
    g = np.zeros(model.dim + 1)
    p = sampler.params()
    rc = L.load().pmcmc_deer_adjoint(h.ptr, tgt, C.byref(p), x0p, int(seed), int(block), sp, mem,
                                     L.OBJECTIVE[objective], g.ctypes.data)
    L.check(rc, h.ptr, "deer_adjoint")
    gaussian = (model.target or {}).get("kind") != "logistic"
    return {"d_epsilon": float(g[0]),
            "d_log_s": g[1:].copy() if objective == "mean_sq" and gaussian else None}


# --------------------------------------------------------------------------- fleet
def fleet_solve(chains, *, workers: int = 8, handle: Optional[L.Handle] = None, device: int = 0,
                errors: str = "raise"):
    """Many independent chains of uneven size on one GPU (MCMCThreads-style):
    `chains` is a list of (model, sampler, x0, seed, block) tuples, one DEER
    block of sampler.T columns each.  Worker streams take chains largest-first;
    every chain converges on its own.  Returns a list of (S (D, T), info,
    logp (T,), accept (T,)); info["status"] is the chain's pmcmc status.
    errors="raise" raises for the first failing chain (after all chains ran);
    errors="report" returns every chain's result with its status."""
    if errors not in ("raise", "report"):
        raise ArgumentError("errors must be 'raise' or 'report'")
    h = handle or L.default_handle(device)
    arr = (L.FleetChain * len(chains))()
    keep = []
    outs = []
    for i, (model, sampler, x0, seed, block) in enumerate(chains):
        dt = sampler.dtype
        x = np.ascontiguousarray(np.asarray(x0, dtype=dt).ravel())
        if x.size != model.dim:
            raise DimensionMismatch(f"chain {i}: initial state must have length {model.dim}")
        T = int(sampler.T)
        S = np.empty((T, model.dim), dt)
        lp = np.empty(T, dt)
        acc = np.empty(T, np.uint8)
        keep.append(x)
        outs.append((S, lp, acc))
        c = arr[i]
        c.target = sampler.target(model, h)
        c.params = sampler.params()
        c.x0, c.seed, c.block = x.ctypes.data, int(seed), int(block)
        c.S_out, c.logp_out, c.accept_out = S.ctypes.data, lp.ctypes.data, acc.ctypes.data
    rc = L.load().pmcmc_fleet_solve(h.ptr, arr, len(chains), int(workers), L.MEM_HOST)
    if errors == "raise" or rc not in (L.OK, L.ERR_NONFINITE, L.ERR_TIMEOUT):
        L.check(rc, h.ptr, "fleet_solve")
    res = []
    for i, (S, lp, acc) in enumerate(outs):
        info = arr[i].info.as_dict()
        info["status"] = int(arr[i].status)
        res.append((S.T, info, lp, acc.astype(bool)))
    return res


# --------------------------------------------------------------------------- tape
def tape(D: int, T: int, seed: int, block: int = 0, *, handle: Optional[L.Handle] = None,
         device: int = 0):
    """Device tape of (seed, block): Xi (D, T) float32 and u (T,) float32."""
    h = handle or L.default_handle(device)
    Xi = np.empty((T, D), np.float32)
    u = np.empty(T, np.float32)
    rc = L.load().pmcmc_tape(h.ptr, int(D), int(T), int(seed), int(block), Xi.ctypes.data,
                             u.ctypes.data, L.MEM_HOST)
    L.check(rc, h.ptr, "tape")
    return Xi.T, u


# --------------------------------------------------------------------------- DEERScan
def solve_affine_scan_diag(A, B, s0, *, handle: Optional[L.Handle] = None, device: int = 0):
    """S[:,t] = A[:,t] .* S[:,t-1] + B[:,t] with S[:,0-1] = s0 (DEERScan.jl:102-191).

    A, B: (D, T) arrays (NumPy or CUDA torch tensors), s0: (D,)."""
    h = handle or L.default_handle(device)
    lib = L.load()
    if _is_torch_cuda(A):
        import torch
        D, T = A.shape
        if tuple(B.shape) != (D, T):
            raise DimensionMismatch("B must have the same size as A")
        if s0.numel() != D:
            raise DimensionMismatch("length(s0) must equal size(A,1)")
        dt = A.dtype
        if dt not in (torch.float32, torch.float64):
            raise ArgumentError("A must be float32 or float64")
        Ac = A.T.contiguous()
        Bc = B.to(dt).T.contiguous()
        sc = s0.to(dt).contiguous()
        S = torch.empty_like(Ac)
        _torch_ready(Ac)
        rc = lib.pmcmc_affine_scan_diag(h.ptr, L.F32 if dt == torch.float32 else L.F64, D, T,
                                        Ac.data_ptr(), Bc.data_ptr(), sc.data_ptr(),
                                        S.data_ptr(), L.MEM_DEVICE)
        L.check(rc, h.ptr, "solve_affine_scan_diag")
        return S.T
    A = np.asarray(A)
    B = np.asarray(B)
    s0 = np.asarray(s0).ravel()
    if A.ndim != 2:
        raise DimensionMismatch("A must be a D x T matrix")
    D, T = A.shape
    if B.shape != (D, T):
        raise DimensionMismatch("B must have the same size as A")
    if s0.size != D:
        raise DimensionMismatch("length(s0) must equal size(A,1)")
    dt = np.float32 if A.dtype == np.float32 else np.float64
    Ac = np.ascontiguousarray(A.T, dtype=dt)
    Bc = np.ascontiguousarray(B.T, dtype=dt)
    sc = np.ascontiguousarray(s0, dtype=dt)
    S = np.empty((T, D), dtype=dt)
    if T and D:
        rc = lib.pmcmc_affine_scan_diag(h.ptr, _dtype_code(dt), D, T, Ac.ctypes.data,
                                        Bc.ctypes.data, sc.ctypes.data, S.ctypes.data,
                                        L.MEM_HOST)
        L.check(rc, h.ptr, "solve_affine_scan_diag")
    return S.T
