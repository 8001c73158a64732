"""Dual averaging of the step size (the reference's _dual_average_update,
src/interface.jl:962-984, and AdaptiveMALASampler's validation, :911-933):
host arithmetic, no GPU."""
import math

import numpy as np
import pytest

import pmcmc
from pmcmc import AdaptiveMALASampler, dual_average_update


def _restated(eps0, eps_bar, H_bar, m, logalpha, delta, gamma, t0, kappa):
    alpha = np.minimum(1.0, np.exp(logalpha))
    eta = 1.0 / (m + t0)
    H = (1 - eta) * H_bar + eta * (delta - alpha)
    le = np.log(10 * eps0) - np.sqrt(m) / gamma * H
    w = m ** (-kappa)
    return np.exp(le), np.exp(w * le + (1 - w) * np.log(eps_bar)), H


def test_update_matches_the_formula():
    rng = np.random.default_rng(0)
    for _ in range(200):
        ad = AdaptiveMALASampler(10 ** rng.uniform(-3, 0), target_accept=rng.uniform(0.2, 0.9),
                                 gamma=rng.uniform(0.01, 0.2), t0=rng.uniform(1, 20),
                                 kappa=rng.uniform(0.51, 1.0))
        args = (ad.epsilon_init, 10 ** rng.uniform(-3, 0), rng.normal(0, 0.1),
                int(rng.integers(1, 5000)), -abs(rng.normal(0, 2)))
        got = dual_average_update(*args, ad)
        ref = _restated(*args, ad.target_accept, ad.gamma, ad.t0, ad.kappa)
        np.testing.assert_allclose(got, ref, rtol=1e-12)


def test_direction_of_the_update():
    ad = AdaptiveMALASampler(0.1)
    e_hi = e_lo = (0.1, 0.1, 0.0)
    for m in range(1, 200):
        e_hi = dual_average_update(0.1, e_hi[1], e_hi[2], m, 0.0, ad)        # always accepted
        e_lo = dual_average_update(0.1, e_lo[1], e_lo[2], m, -math.inf, ad)  # never accepted
    assert e_hi[1] > 0.1 > e_lo[1]
    # at the target rate H stays 0 and epsilon sits at the prior centre 10 eps0
    e = dual_average_update(0.1, 0.1, 0.0, 1, math.log(ad.target_accept), ad)
    assert e[2] == pytest.approx(0.0, abs=1e-15) and e[0] == pytest.approx(1.0)


@pytest.mark.parametrize("kw", [dict(epsilon_init=0.0), dict(epsilon_init=0.1, target_accept=1.0),
                                dict(epsilon_init=0.1, gamma=0.0), dict(epsilon_init=0.1, t0=0.0),
                                dict(epsilon_init=0.1, kappa=0.5),
                                dict(epsilon_init=0.1, kappa=1.5)])
def test_validation_mirrors_the_reference(kw):
    with pytest.raises(pmcmc.ArgumentError):
        AdaptiveMALASampler(**kw)


def test_adapt_arguments_are_checked():
    model = pmcmc.DensityModel.diag_gaussian(np.ones(3))
    s = pmcmc.ParallelMALASampler(0.1, T=8)
    with pytest.raises(pmcmc.ArgumentError):
        pmcmc.adapt_step_size(model, s, np.zeros(3), method="newton")
    with pytest.raises(pmcmc.ArgumentError):
        pmcmc.adapt_step_size(model, s, np.zeros(3), n_blocks=0)


def test_oracle_adaptive_chain_has_the_reference_properties():
    # the oracle's AdaptiveMALASampler chain (the checker of the device chains) on a
    # standard normal, test-Adaptive-MALA.jl:117-168: the step size moves during warmup,
    # is frozen at epsilon_bar after it, and the adapted rate is near the target
    import oracle as O
    D, n_w, T = 5, 2000, 2500
    tg = O.Target.diag_gauss(np.ones(D))
    Xi, u = O.tape(42, 0, D, T)
    S, acc, used, (eps, eps_bar, h_bar) = O.mala_adaptive(tg, 0.5, np.zeros(D), Xi, u, n_w)
    assert len(set(used[:n_w].tolist())) > 100
    assert np.all(used[n_w:] == eps_bar)
    assert 0.35 < acc[n_w:].mean() < 0.80
    # the oracle's update and the product's host update are the same formula
    ad = AdaptiveMALASampler(0.5)
    np.testing.assert_allclose(O.dual_average(0.5, 0.3, 0.01, 7, -0.4),
                               dual_average_update(0.5, 0.3, 0.01, 7, -0.4, ad), rtol=1e-14)


def test_adapt_fleet_with_a_stand_in_solver():
    # the fleet-level dual averaging with a stand-in for fleet_solve: the accept rate
    # falls with epsilon (rate = exp(-eps / s_c)), a block above 4 s_c goes non-finite
    from pmcmc import _lib as L
    from pmcmc.adapt import adapt_fleet
    scales = [0.01, 0.05, 0.2]
    chains = [(pmcmc.DensityModel.diag_gaussian(np.ones(2)),
               pmcmc.ParallelMALASampler(1.0, T=64), np.zeros(2), 7 + c, 0) for c in range(3)]
    seen = []

    def solve(batch):
        out = []
        for m, smp, x0, seed, block in batch:
            s = scales[seed - 7]
            seen.append((seed, block, smp.T))
            if smp.epsilon > 4 * s:
                out.append((None, {"status": L.ERR_NONFINITE}, None, None))
                continue
            k = int(round(smp.T * np.exp(-smp.epsilon / s)))
            acc = np.arange(smp.T) < k
            out.append((np.full((2, smp.T), float(seed)), {"status": 0}, None, acc))
        return out

    adapted, hist = adapt_fleet(chains, rounds=40, T_adapt=200, solve=solve)
    for c, s in enumerate(scales):
        eps = adapted[c][1].epsilon
        # the target accept rate 0.574 is reached at eps = -s log(0.574) = 0.555 s
        assert 0.3 * s < eps < 1.2 * s, (c, eps / s)
        assert adapted[c][1].T == 64 and np.all(adapted[c][2] == 7 + c)
        assert all(e <= 4 * s * 4 for e, _ in hist[c])
    assert {b for _, b, _ in seen} == set(range(1, 41)) and {t for *_, t in seen} == {200}


def test_adapt_fleet_esjd_gradient_with_stand_ins():
    # the gradient method of adapt_fleet: sign steps on log epsilon toward the epsilon
    # where a stand-in ESJD gradient changes sign (eps* = 0.01 and 0.2)
    from pmcmc.adapt import adapt_fleet
    targets = [0.01, 0.2]
    chains = [(pmcmc.DensityModel.diag_gaussian(np.ones(2)),
               pmcmc.ParallelMALASampler(0.05, T=64), np.zeros(2), 30 + c, 0) for c in range(2)]

    def solve(batch):
        return [(np.zeros((2, smp.T)), {"status": 0}, None, np.ones(smp.T, bool))
                for _, smp, *_ in batch]

    def grad(ch, xs, S):
        return targets[ch[3] - 30] - ch[1].epsilon

    adapted, hist = adapt_fleet(chains, rounds=60, T_adapt=32, method="esjd_gradient",
                                solve=solve, grad=grad)
    for c, t in enumerate(targets):
        assert 0.8 * t < adapted[c][1].epsilon < 1.25 * t, (c, adapted[c][1].epsilon)
    with pytest.raises(pmcmc.ArgumentError):
        adapt_fleet(chains, method="newton", solve=solve)
