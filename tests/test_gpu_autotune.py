"""pmcmc_autotune: the kept shape is one of the candidates, later solves of the
same shape use it and still reproduce the FP64 sequential chain, and paths with
nothing to tune report 0."""
import numpy as np
import pytest

import oracle as O
import pmcmc
from pmcmc import configs

pytestmark = pytest.mark.gpu


def trace_err(S, R):
    S = np.asarray(S, np.float64)
    R = np.asarray(R, np.float64)
    return float(np.max(np.linalg.norm(S - R, axis=0) /
                        np.maximum(np.linalg.norm(R, axis=0), 1e-30)))


def test_persistent_shape_is_tuned_and_used():
    lam = 10 ** np.random.default_rng(4).uniform(-1, 1, 100)
    model = pmcmc.DensityModel.diag_gaussian(lam)
    sampler = pmcmc.ParallelMALASampler(0.05, T=4096, jacobian="diag", dtype=np.float32,
                                        tol_abs=1e-7, tol_rel=1e-6)
    x0 = np.random.default_rng(5).standard_normal(100).astype(np.float32)
    h = pmcmc.Handle(0)
    r = pmcmc.autotune(model, sampler, x0, seed=2, handle=h)
    assert r["choice"] in (1, 2, 3, 4) and r["ms"] > 0
    S, info, _, acc = pmcmc.solve(model, sampler, x0, seed=2, block=3, handle=h,
                                  return_logp=True)
    assert "persistent" in info["path_names"] and info["converged"]
    Xi, u = O.tape(2, 3, 100, 4096)
    S_seq, acc_seq, _ = O.mala_sequential(O.Target.diag_gauss(lam), 0.05,
                                          x0.astype(np.float64), Xi, u)
    assert np.array_equal(acc, acc_seq)
    assert trace_err(S, S_seq) <= 1e-5


def test_full_chunk_count_is_tuned_and_used():
    model, sampler, x0, meta = configs.correlated_gauss_d64(T=1024)
    sampler.tol_abs, sampler.tol_rel = 1e-7, 1e-6
    h = pmcmc.Handle(0)
    r = pmcmc.autotune(model, sampler, x0, seed=3, handle=h)
    cands = {max(1, min(148, int(np.sqrt(f * 1024) + 0.5))) for f in (0.5, 1, 2, 4)}
    assert r["choice"] in cands and r["ms"] > 0
    S, info, _, acc = pmcmc.solve(model, sampler, x0, seed=3, block=0, handle=h,
                                  return_logp=True)
    assert info["converged"] and "full_jacobian" in info["path_names"]
    tg = O.Target.dense_gauss(model.target["prec"], model.target["mean"])
    Xi, u = O.tape(3, 0, 64, 1024)
    S_seq, acc_seq, _ = O.mala_sequential(tg, 0.05, np.asarray(x0, np.float64), Xi, u)
    assert np.array_equal(acc, acc_seq)
    assert trace_err(S, S_seq) <= 1e-5


def test_nothing_to_tune_on_the_plain_path():
    model = pmcmc.DensityModel.diag_gaussian(np.ones(8))
    sampler = pmcmc.ParallelMALASampler(0.1, T=256, exec="plain", dtype=np.float32)
    r = pmcmc.autotune(model, sampler, np.zeros(8, np.float32))
    assert r == {"choice": 0, "ms": 0.0}
