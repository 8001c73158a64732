"""Step-size adaptation for the DEER sampler.

Two ways to pick epsilon before sampling, both block by block on the device:

* dual averaging (Hoffman & Gelman's scheme, as `_dual_average_update`,
  src/interface.jl:962-984, drives the reference's AdaptiveMALASampler,
  src/interface.jl:899-933, 1000-1065).  The reference updates after every
  sequential MALA step with that step's acceptance probability.  Here a block
  of T steps is solved at one epsilon, so one update follows each block, with
  the block's accept rate as the acceptance probability and m counting blocks
  (fed the T steps of a fixed-epsilon block one by one, the recursion would
  take T identical signals and overshoot by orders of magnitude);
* gradient ascent on the expected squared jump distance, with the gradient
  d ESJD / d epsilon from the adjoint reverse scan at each solved block
  (Gaussian device targets), a sign step on log epsilon with a step length
  that decays as 1 / sqrt(block).

A sequential MALA chain only rejects at a step size far too large; a DEER
solve there can fail with a non-finite trajectory.  So the epsilon a block
uses moves at most a factor `max_step_ratio` from the previous block's, and a
block that fails that way is solved again at half its epsilon.  The dual
averaging state itself follows the reference update.

Neither changes the sampling path: the adapted epsilon goes into an ordinary
ParallelMALASampler.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, replace
from typing import Any, Optional

import numpy as np

from . import _lib as L
from ._lib import ArgumentError, DimensionMismatch
from .core import Cholesky, DensityModel, ParallelMALASampler, _mass_factor, adjoint, solve


@dataclass
class AdaptiveMALASampler:
    """AdaptiveMALASampler(epsilon_init; n_warmup, target_accept, gamma, t0, kappa,
    cholM): the reference's dual-averaging settings and their validation
    (src/interface.jl:911-933)."""

    epsilon_init: float
    n_warmup: int = 1000
    target_accept: float = 0.574
    gamma: float = 0.05
    t0: float = 10.0
    kappa: float = 0.75
    cholM: Any = None

    def __post_init__(self):
        if not (self.epsilon_init > 0):
            raise ArgumentError(f"epsilon_init must be > 0, got {self.epsilon_init}")
        if not (0 < self.target_accept < 1):
            raise ArgumentError(f"target_accept must be in (0,1), got {self.target_accept}")
        if not (self.gamma > 0):
            raise ArgumentError(f"gamma must be > 0, got {self.gamma}")
        if not (self.t0 > 0):
            raise ArgumentError(f"t0 must be > 0, got {self.t0}")
        if not (0.5 < self.kappa <= 1.0):
            raise ArgumentError(f"kappa must be in (0.5, 1], got {self.kappa}")
        if self.cholM is not None:
            self.cholM = Cholesky(L=_mass_factor(self.cholM))


def _sampler_dtype(adaptive: "AdaptiveMALASampler"):
    # FP = typeof(float(epsilon_init)) (src/interface.jl:925-926)
    return np.float32 if isinstance(adaptive.epsilon_init, np.float32) else np.float64


def adaptive_chains(model: DensityModel, adaptive: "AdaptiveMALASampler", x0s, seeds, T: int, *,
                    block: int = 0, handle: Optional[L.Handle] = None, device: int = 0,
                    dtype=None) -> dict:
    """n AdaptiveMALASampler chains of T steps on the device, one warp a chain
    (pmcmc_mala_chains_adaptive): chain c starts at x0s[c] with the tape of
    (seeds[c], block) and adapts its own step size by dual averaging during its
    first n_warmup steps (src/interface.jl:1024-1065).  Returns a dict with S
    (n, T, D), logp (n, T), accepted (n, T), step_size (n, T), is_warmup (n, T)
    and epsilon, epsilon_bar, H_bar (n,): the chains' final adaptation state."""
    import ctypes as C

    h = handle or L.default_handle(device)
    dt = np.dtype(dtype or _sampler_dtype(adaptive)).type
    smp = ParallelMALASampler(float(adaptive.epsilon_init), T=int(T), dtype=dt,
                              cholM=adaptive.cholM)
    tgt = smp.target(model, h)
    x = np.ascontiguousarray(np.asarray(x0s, dtype=dt).reshape(-1, model.dim))
    n = x.shape[0]
    sd = np.ascontiguousarray(np.asarray(seeds, dtype=np.uint64).reshape(-1))
    if sd.size != n:
        raise DimensionMismatch("one seed per chain")
    S = np.empty((n, T, model.dim), dt)
    lp = np.empty((n, T), dt)
    acc = np.empty((n, T), np.uint8)
    eps = np.empty((n, T), np.float64)
    st = np.empty((n, 3), np.float64)
    ad = L.Adapt(int(adaptive.n_warmup), float(adaptive.target_accept), float(adaptive.gamma),
                 float(adaptive.t0), float(adaptive.kappa))
    p = smp.params()
    rc = L.load().pmcmc_mala_chains_adaptive(
        h.ptr, tgt, C.byref(p), n, x.ctypes.data, sd.ctypes.data, int(block), C.byref(ad),
        S.ctypes.data, lp.ctypes.data, acc.ctypes.data, eps.ctypes.data, st.ctypes.data,
        L.MEM_HOST)
    L.check(rc, h.ptr, "mala_chains_adaptive")
    return {"S": S, "logp": lp, "accepted": acc.astype(bool), "step_size": eps,
            "is_warmup": np.broadcast_to(np.arange(T) < adaptive.n_warmup, (n, T)).copy(),
            "epsilon": st[:, 0].copy(), "epsilon_bar": st[:, 1].copy(), "H_bar": st[:, 2].copy()}


def sample_adaptive(model: DensityModel, adaptive: "AdaptiveMALASampler", N: int, *,
                    seed: int = 0, initial_params=None, handle: Optional[L.Handle] = None,
                    device: int = 0, **_):
    """sample(rng, model, AdaptiveMALASampler(...), N) (src/interface.jl:987-1065)
    on the device: as AbstractMCMC runs it, transition 1 is the initial state
    (log density from the model, accepted, step size epsilon_init, warmup) and
    transitions 2..N are N - 1 adaptive MALA steps on tape block 0 of `seed`.
    The Chain's info carries step_size, is_warmup and the final epsilon_bar."""
    from .core import Chain, _initial_params

    if N < 1:
        raise ArgumentError("the number of samples must be >= 1")
    dt = _sampler_dtype(adaptive)
    x0 = np.asarray(_initial_params(model, ParallelMALASampler(1.0, dtype=dt), initial_params,
                                    seed), dt).ravel()
    if x0.size != model.dim:
        raise L.DimensionMismatch(f"initial state must have length {model.dim}")
    lp0 = model.logdensity(x0) if model.logdensity is not None else np.nan
    vals = np.empty((N, model.dim), dt)
    logp = np.empty(N, dt)
    acc = np.ones(N, bool)
    step = np.full(N, float(adaptive.epsilon_init))
    warm = np.ones(N, bool)
    vals[0], logp[0] = x0, lp0
    info = {"epsilon_bar": float(adaptive.epsilon_init)}
    if N > 1:
        r = adaptive_chains(model, adaptive, x0[None, :], [seed], N - 1, handle=handle,
                            device=device, dtype=dt)
        vals[1:], logp[1:], acc[1:] = r["S"][0], r["logp"][0], r["accepted"][0]
        step[1:], warm[1:] = r["step_size"][0], r["is_warmup"][0]
        info = {"epsilon": float(r["epsilon"][0]), "epsilon_bar": float(r["epsilon_bar"][0]),
                "H_bar": float(r["H_bar"][0])}
    info.update({"step_size": step, "is_warmup": warm})
    return Chain(vals, logp, acc, info, model.param_names)


def dual_average_update(epsilon_init: float, epsilon_bar: float, H_bar: float, m: int,
                        logalpha: float, sampler: AdaptiveMALASampler):
    """One dual-averaging step after step m (m >= 1) with log acceptance ratio
    logalpha: returns (epsilon, epsilon_bar, H_bar) (src/interface.jl:962-984)."""
    alpha = min(1.0, math.exp(logalpha)) if logalpha < 0 else 1.0
    mu = math.log(10.0 * epsilon_init)
    w = 1.0 / (m + sampler.t0)
    H_new = (1.0 - w) * H_bar + w * (sampler.target_accept - alpha)
    log_eps = mu - math.sqrt(m) / sampler.gamma * H_new
    mk = m ** (-sampler.kappa)
    log_eps_bar = mk * log_eps + (1.0 - mk) * math.log(epsilon_bar)
    return math.exp(log_eps), math.exp(log_eps_bar), H_new


def _esjd(S, x0) -> float:
    """Realised squared jump distance per step of a solved block, S (D, T)."""
    S = np.asarray(S, np.float64)
    prev = np.concatenate([np.asarray(x0, np.float64)[:, None], S[:, :-1]], axis=1)
    return float(np.mean(np.sum((S - prev) ** 2, axis=0)))


def _solve_block(model, sampler, eps, x, seed, b, h, retries=10):
    """One block at epsilon, halving epsilon while the solve is non-finite."""
    for _ in range(retries):
        smp = replace(sampler, epsilon=eps)
        try:
            S, info, _, acc = solve(model, smp, x, seed=seed, block=b, handle=h,
                                    return_logp=True)
            return smp, S, info, acc
        except L.DeviceError as e:
            if "non-finite" not in str(e):
                raise
            eps *= 0.5
    raise L.DeviceError(f"block {b}: non-finite trajectory down to epsilon {eps}")


def adapt_step_size(model: DensityModel, sampler: ParallelMALASampler, x0, *,
                    n_blocks: int = 20, method: str = "dual_averaging",
                    adaptive: Optional[AdaptiveMALASampler] = None, step0: float = 0.5,
                    max_step_ratio: float = 4.0, seed: int = 0,
                    handle: Optional[L.Handle] = None, device: int = 0) -> dict:
    """Adapt epsilon over n_blocks DEER blocks of sampler.T steps, the chain
    continuing from block to block (block b uses tape block b of `seed`).

    method "dual_averaging": `adaptive` holds the settings (default
      AdaptiveMALASampler(sampler.epsilon)); the result is epsilon_bar, as the
      reference uses after warmup.  The epsilon a block uses follows the dual
      averaging iterate within a factor max_step_ratio of the previous block's.
    method "esjd_gradient": log epsilon += step0 / sqrt(b + 1) * sign(d ESJD / d
      epsilon) after block b (Gaussian device targets).

    Returns {"epsilon": adapted value, "history": per-block dicts with the
    epsilon used, accept rate, realised ESJD and, for the gradient method, the
    gradient}."""
    if n_blocks < 1:
        raise ArgumentError("n_blocks must be >= 1")
    if method not in ("dual_averaging", "esjd_gradient"):
        raise ArgumentError("method must be 'dual_averaging' or 'esjd_gradient'")
    h = handle or L.default_handle(device)
    x = np.asarray(x0, sampler.dtype).copy()
    eps = float(sampler.epsilon)
    hist = []
    if method == "dual_averaging":
        ad = adaptive or AdaptiveMALASampler(eps)
        if ad.cholM is not None:
            # the adaptive sampler's mass matrix (src/interface.jl:1040) drives the blocks
            if sampler.cholM is not None and not np.array_equal(sampler.cholM.L, ad.cholM.L):
                raise ArgumentError("sampler and adaptive carry different mass matrices")
            sampler = replace(sampler, cholM=ad.cholM)
        eps_bar, H_bar, m = ad.epsilon_init, 0.0, 0
        eps = used = ad.epsilon_init
        for b in range(n_blocks):
            used = min(max(eps, used / max_step_ratio), used * max_step_ratio)
            smp, S, info, acc = _solve_block(model, sampler, used, x, seed, b, h)
            used = smp.epsilon
            hist.append({"epsilon": used, "accept_rate": float(np.mean(acc)),
                         "esjd": _esjd(S, x), "iters": info["iters"]})
            rate = float(np.mean(acc))
            m += 1
            eps, eps_bar, H_bar = dual_average_update(
                ad.epsilon_init, eps_bar, H_bar, m, math.log(rate) if rate > 0 else -math.inf, ad)
            x = np.asarray(S[:, -1], sampler.dtype).copy()
        return {"epsilon": eps_bar, "history": hist}
    log_eps = math.log(eps)
    for b in range(n_blocks):
        smp, S, info, acc = _solve_block(model, sampler, math.exp(log_eps), x, seed, b, h)
        log_eps = math.log(smp.epsilon)
        g = adjoint(model, smp, x, S, objective="esjd", seed=seed, block=b, handle=h)
        d = g["d_epsilon"]
        hist.append({"epsilon": smp.epsilon, "accept_rate": float(np.mean(acc)),
                     "esjd": _esjd(S, x), "d_esjd_d_epsilon": d, "iters": info["iters"]})
        if d != 0.0 and np.isfinite(d):
            log_eps += step0 / math.sqrt(b + 1.0) * math.copysign(1.0, d)
        x = np.asarray(S[:, -1], sampler.dtype).copy()
    return {"epsilon": math.exp(log_eps), "history": hist}


def adapt_fleet(chains, *, rounds: int = 8, T_adapt: int = 256, target_accept: float = 0.574,
                max_step_ratio: float = 4.0, retries: int = 6, workers: int = 8,
                handle: Optional[L.Handle] = None, device: int = 0, solve=None,
                method: str = "dual_averaging", step0: float = 0.5, grad=None):
    """Per-chain step-size adaptation for a fleet (`chains` as for
    pmcmc.fleet_solve), every round one short block of every chain solved
    together on the fleet.

    method "esjd_gradient": after round r, log epsilon += step0 / sqrt(r + 1) *
    sign(d ESJD / d epsilon) with the gradient from the adjoint at the block
    (pmcmc.adjoint; `grad(chain, x_start, S)` replaces it in tests), as
    adapt_step_size does for one chain; the result is the last epsilon.
    method "dual_averaging", the default, is described below.

    Round r: chain c solves tape block `block_c + 1 + r` of its seed, T_adapt
    steps at its current epsilon from its current state; the block's accept
    rate feeds dual_average_update (one update a block, m = r + 1, as
    adapt_step_size does for one chain) with epsilon_init = the chain's
    epsilon; the chain continues from the block's last column.  The epsilon a
    block uses stays within max_step_ratio of the chain's previous one; a block
    that goes non-finite is solved again at half its epsilon (at most `retries`
    times; a chain that still fails keeps its halved epsilon).  `solve`
    replaces fleet_solve (tests).

    Returns (adapted, history): the chains with sampler.epsilon = epsilon_bar
    and x0 = the state after the last round, and per chain the list of
    (epsilon, accept rate) of its rounds."""
    from .core import fleet_solve

    if rounds < 1 or T_adapt < 1:
        raise ArgumentError("rounds and T_adapt must be >= 1")
    if method not in ("dual_averaging", "esjd_gradient"):
        raise ArgumentError("method must be 'dual_averaging' or 'esjd_gradient'")
    h = None
    if solve is None or (method == "esjd_gradient" and grad is None):
        h = handle or L.default_handle(device)
    if solve is None:
        solve = lambda cs: fleet_solve(cs, workers=workers, handle=h, errors="report")
    if grad is None:
        grad = lambda ch, xs, S: adjoint(ch[0], ch[1], xs, S, objective="esjd", seed=ch[3],
                                         block=ch[4], handle=h)["d_epsilon"]
    n = len(chains)
    eps0 = [float(s.epsilon) for _, s, *_ in chains]
    ads = [AdaptiveMALASampler(e, target_accept=target_accept) for e in eps0]
    eps, used, eps_bar, h_bar = list(eps0), list(eps0), list(eps0), [0.0] * n
    x = [np.asarray(x0, s.dtype).copy() for _, s, x0, *_ in chains]
    hist = [[] for _ in range(n)]
    for r in range(rounds):
        todo = list(range(n))
        for c in todo:
            used[c] = min(max(eps[c], used[c] / max_step_ratio), used[c] * max_step_ratio)
        res = {}
        for _ in range(retries + 1):
            if not todo:
                break
            batch = [(chains[c][0], replace(chains[c][1], epsilon=used[c], T=int(T_adapt)), x[c],
                      chains[c][3], chains[c][4] + 1 + r) for c in todo]
            out = solve(batch)
            again = []
            for c, o in zip(todo, out):
                if o[1].get("status", 0) == L.ERR_NONFINITE:
                    used[c] *= 0.5
                    again.append(c)
                else:
                    res[c] = o
            todo = again
        for c in range(n):
            if c not in res:  # non-finite at every retry: keep the halved epsilon
                hist[c].append((used[c], float("nan")))
                eps[c] = eps_bar[c] = used[c]
                continue
            S, info, _, acc = res[c]
            rate = float(np.mean(acc))
            hist[c].append((used[c], rate))
            if method == "dual_averaging":
                eps[c], eps_bar[c], h_bar[c] = dual_average_update(
                    eps0[c], eps_bar[c], h_bar[c], r + 1,
                    math.log(rate) if rate > 0 else -math.inf, ads[c])
            else:
                ch = (chains[c][0], replace(chains[c][1], epsilon=used[c], T=int(T_adapt)),
                      None, chains[c][3], chains[c][4] + 1 + r)
                d = grad(ch, x[c], S)
                step = step0 / math.sqrt(r + 1.0) * (math.copysign(1.0, d)
                                                     if d != 0.0 and math.isfinite(d) else 0.0)
                eps[c] = eps_bar[c] = used[c] * math.exp(step)
            x[c] = np.asarray(S[:, -1], chains[c][1].dtype).copy()
    adapted = [(m, replace(s, epsilon=eps_bar[c]), x[c], seed, block)
               for c, (m, s, _, seed, block) in enumerate(chains)]
    return adapted, hist
