"""Run-to-run reproducibility of the per-sweep path: the decoupled look-back
composes each tile's carry in a fixed association, so the same (seed, block)
gives bit-identical trajectories and the same Newton iteration count on every
solve, whichever CTA finishes first (the reference's CPU DEER is deterministic:
src/DEER/DEER.jl:506-595)."""
import os

import numpy as np
import pytest

import pmcmc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def h_lookback():
    # narrow tiles: hundreds of tiles a solve, so the look-back joins them
    # (a column-width override also keeps the solve off the persistent kernel)
    old = os.environ.get("PMCMC_TILE_COLS")
    os.environ["PMCMC_TILE_COLS"] = "8"
    try:
        return pmcmc.Handle(0)
    finally:
        if old is None:
            del os.environ["PMCMC_TILE_COLS"]
        else:
            os.environ["PMCMC_TILE_COLS"] = old


def _solves(h, model, sampler, x0, n=3):
    out = [pmcmc.solve(model, sampler, x0, seed=5, block=2, handle=h, return_logp=True)
           for _ in range(n)]
    return out


def _same(out):
    S0, i0, lp0, a0 = out[0]
    for S, info, lp, acc in out[1:]:
        assert info["iters"] == i0["iters"]
        assert np.array_equal(S, S0)
        assert np.array_equal(lp, lp0)
        assert np.array_equal(acc, a0)


def test_logistic_solves_repeat_bit_for_bit(h_lookback):
    rng = np.random.default_rng(41)
    N, D, T = 1500, 64, 4096
    X = (rng.standard_normal((N, D)) / np.sqrt(D)).astype(np.float32).astype(np.float64)
    th = rng.standard_normal(D)
    y = (rng.random(N) < 1 / (1 + np.exp(-X @ th))).astype(np.float64)
    model = pmcmc.DensityModel.logistic(X, y)
    sampler = pmcmc.ParallelMALASampler(0.02, T=T, jacobian="stoch_diag", dtype=np.float32,
                                        maxiter=60)
    out = _solves(h_lookback, model, sampler, np.zeros(D, np.float32))
    assert out[0][1]["path"] & 8  # tensor-core contraction
    assert not out[0][1]["path"] & 2  # not the cooperative sweep: tiles joined by look-back
    _same(out)


def test_gaussian_per_sweep_solves_repeat_bit_for_bit(h_lookback):
    rng = np.random.default_rng(42)
    D, T = 100, 16384
    prec = 10.0 ** rng.uniform(-2, 2, D)
    model = pmcmc.DensityModel.diag_gaussian(prec)
    sampler = pmcmc.ParallelMALASampler(0.005, T=T, jacobian="diag", dtype=np.float32)
    out = _solves(h_lookback, model, sampler, rng.standard_normal(D).astype(np.float32))
    assert not out[0][1]["path"] & 32  # per-sweep kernel, not the persistent solve
    assert out[0][1]["iters"] > 5
    _same(out)
