"""Bayesian logistic regression at full size: N = 10000, D = 256, T = 65536,
:stoch_diag with one probe, FP32 state, contractions on the tensor cores.

The reference's GPU test compares a logistic DEER trajectory with the
sequential chain on the same tape at rtol 1e-3 / atol 1e-4
(test/test-DEER-Turing-Logistic.jl:205-260) on a small problem.  Here the
whole block is checked against the FP64 sequential chain
(MALA.jl:322-346, 377-411): accept flags identical, trace error at most 1e-5.
The sampler's own stopping rule (1e-6 + 1e-5 max|S|, DEER.jl:567-578) bounds
the last Newton step, and the iterate then still sits about 1e-5 from the
fixed point (an FP64 solve at that rule gives 1.2e-5 on this block), so the
1e-5 bar is checked at a rule ten times tighter.
"""
import dataclasses

import numpy as np
import pytest

import oracle as O
import pmcmc
from pmcmc import configs

pytestmark = pytest.mark.gpu


def trace_err(S, R):
    return float(np.max(np.linalg.norm(S - R, axis=0) /
                        np.maximum(np.linalg.norm(R, axis=0), 1e-30)))


@pytest.fixture(scope="module")
def problem():
    model, sampler, x0, meta = configs.logistic_n10k_d256()
    tg = O.Target.logistic(model.target["X"], model.target["y"])
    block = 1000  # a block whose FP32 decisions meet near-ties (|log alpha - log u| ~ 1e-5)
    Xi, u = O.tape(meta["seed"], block, model.dim, sampler.T)
    S_seq, acc_seq, la_seq = O.mala_sequential_logistic(tg, sampler.epsilon,
                                                        np.zeros(model.dim), Xi, u)
    return model, sampler, x0, meta, block, tg, S_seq, acc_seq, la_seq - np.log(u.astype(np.float64))


def test_logistic_n10k_d256_matches_fp64_chain(problem):
    model, sampler, x0, meta, block, tg, S_seq, acc_seq, m_seq = problem
    smp = dataclasses.replace(sampler, tol_abs=1e-7, tol_rel=1e-6)
    h = pmcmc.Handle(0)
    S, info, lp, acc = pmcmc.solve(model, smp, x0, seed=meta["seed"], block=block, handle=h,
                                   return_logp=True)
    S = np.asarray(S, np.float64)
    assert info["converged"], info
    assert "tensor_core" in info["path_names"] and "tie_fp64" in info["path_names"]
    assert np.array_equal(acc, acc_seq), np.nonzero(acc != acc_seq)[0][:10]
    assert trace_err(S, S_seq) <= 1e-5
    # the verification pass at the returned trajectory
    assert np.isfinite(info["max_defect"])
    assert info["max_defect"] <= 1e-5 * (1 + np.abs(S).max())
    assert info["n_accept"] == int(acc_seq.sum())
    # the smallest margin at the returned trajectory, within what its ~2e-6
    # distance from the FP64 chain moves a margin
    assert abs(info["min_margin"] - np.abs(m_seq).min()) <= 5e-6
    ref = np.array([O.logp(tg, S[:, t]) for t in range(0, sampler.T, 4099)])
    np.testing.assert_allclose(np.asarray(lp, np.float64)[::4099], ref, rtol=1e-6)


def test_logistic_n10k_d256_default_rule(problem):
    """At the sampler's default stopping rule: the same accept flags, and the
    trace error that rule allows (reported beside the 1e-5 bar above)."""
    model, sampler, x0, meta, block, tg, S_seq, acc_seq, m_seq = problem
    h = pmcmc.Handle(0)
    S, info, lp, acc = pmcmc.solve(model, sampler, x0, seed=meta["seed"], block=block, handle=h,
                                   return_logp=True)
    assert info["converged"], info
    assert np.array_equal(acc, acc_seq)
    assert trace_err(np.asarray(S, np.float64), S_seq) <= 5e-5
