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
from ._lib import ArgumentError
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
