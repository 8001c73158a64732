"""Step-size adaptation through DEER blocks on the device: dual averaging
settles near the target accept rate, and ESJD gradient ascent (adjoint
gradients) moves a too-small step size up and raises the jump distance."""
import numpy as np
import pytest

import pmcmc

pytestmark = pytest.mark.gpu


def _problem():
    lam = 10 ** np.random.default_rng(7).uniform(-0.3, 0.3, 16)
    model = pmcmc.DensityModel.diag_gaussian(lam)
    x0 = (np.random.default_rng(8).standard_normal(16) / np.sqrt(lam)).astype(np.float32)
    return model, x0


def _accept_and_esjd(model, eps, x0, h, blocks=(100, 101, 102)):
    s = pmcmc.ParallelMALASampler(eps, T=1024, jacobian="diag", dtype=np.float32)
    rates, esjd = [], []
    for b in blocks:
        S, info, _, acc = pmcmc.solve(model, s, x0, seed=3, block=b, handle=h, return_logp=True)
        assert info["converged"]
        rates.append(acc.mean())
        prev = np.concatenate([x0[:, None], S[:, :-1]], axis=1).astype(np.float64)
        esjd.append(np.mean(np.sum((S - prev) ** 2, axis=0)))
    return float(np.mean(rates)), float(np.mean(esjd))


def test_dual_averaging_reaches_the_target_rate():
    model, x0 = _problem()
    h = pmcmc.Handle(0)
    s = pmcmc.ParallelMALASampler(0.01, T=512, jacobian="diag", dtype=np.float32)
    out = pmcmc.adapt_step_size(model, s, x0, n_blocks=16, method="dual_averaging", seed=1,
                                handle=h)
    assert len(out["history"]) == 16 and out["epsilon"] > 0.01
    rate, _ = _accept_and_esjd(model, out["epsilon"], x0, h)
    assert 0.45 <= rate <= 0.75, (out["epsilon"], rate)


def test_esjd_gradient_raises_a_small_step():
    model, x0 = _problem()
    h = pmcmc.Handle(0)
    s = pmcmc.ParallelMALASampler(0.005, T=512, jacobian="diag", dtype=np.float32)
    out = pmcmc.adapt_step_size(model, s, x0, n_blocks=10, method="esjd_gradient", seed=1,
                                handle=h)
    assert out["history"][0]["d_esjd_d_epsilon"] > 0  # ESJD grows with a small step
    assert out["epsilon"] > 0.05
    _, e0 = _accept_and_esjd(model, 0.005, x0, h)
    _, e1 = _accept_and_esjd(model, out["epsilon"], x0, h)
    assert e1 > 3 * e0, (out["epsilon"], e0, e1)


def test_esjd_gradient_on_the_logistic_target():
    # ESJD ascent with the logistic adjoint: a small step grows and the jump distance
    # with it (the per-chain adaptation config 5 describes)
    rng = np.random.default_rng(7)
    N, D = 800, 16
    X = rng.standard_normal((N, D)) / np.sqrt(D)
    y = (rng.random(N) < 1 / (1 + np.exp(-X @ rng.standard_normal(D)))).astype(float)
    model = pmcmc.DensityModel.logistic(X, y)
    h = pmcmc.Handle(0)
    x0 = np.zeros(D, np.float32)
    s = pmcmc.ParallelMALASampler(0.001, T=256, dtype=np.float32, tol_abs=1e-7, tol_rel=1e-6,
                                  maxiter=300)
    out = pmcmc.adapt_step_size(model, s, x0, n_blocks=8, method="esjd_gradient", seed=2,
                                handle=h)
    assert out["history"][0]["d_esjd_d_epsilon"] > 0
    assert out["epsilon"] > 0.004
    assert out["history"][-1]["esjd"] > 3 * out["history"][0]["esjd"]
