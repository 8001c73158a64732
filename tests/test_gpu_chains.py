"""Independent sequential MALA chains on the device (pmcmc_mala_chains) against
the FP64 sequential oracle on the same tapes, and against DEER: a chain and a
DEER solve with the same seed and block follow the same trajectory."""
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


def test_fp64_diag_chains_match_the_sequential_oracle():
    lam = np.array([0.5, 1.0, 2.0, 4.0, 0.25])
    model = pmcmc.DensityModel.diag_gaussian(lam, mean=np.linspace(-1, 1, 5))
    sampler = pmcmc.ParallelMALASampler(0.2, T=300)
    seeds = [3, 4, 5, 6]
    x0 = np.random.default_rng(0).standard_normal((4, 5))
    S, lp, acc = pmcmc.mala_chains(model, sampler, x0, seeds, block=2)
    assert S.shape == (4, 300, 5) and lp.shape == acc.shape == (4, 300)
    tg = O.Target.diag_gauss(lam, np.linspace(-1, 1, 5))
    for c, sd in enumerate(seeds):
        Xi, u = O.tape(sd, 2, 5, 300)
        S_ref, acc_ref, _ = O.mala_sequential(tg, 0.2, x0[c], Xi, u)
        assert np.array_equal(acc[c], acc_ref), c
        np.testing.assert_allclose(S[c].T, S_ref, rtol=1e-12, atol=1e-12)
        lp_ref = np.array([O.logp(tg, S_ref[:, t]) for t in range(0, 300, 29)])
        np.testing.assert_allclose(lp[c, ::29], lp_ref, rtol=1e-12, atol=1e-12)
    assert 0.2 < acc.mean() < 1.0


def test_fp32_dense_chains_match_the_sequential_oracle():
    model, sampler, x0, meta = configs.correlated_gauss_d64(T=512, jacobian="diag")
    x0s = np.random.default_rng(1).standard_normal((3, 64)).astype(np.float32)
    S, lp, acc = pmcmc.mala_chains(model, sampler, x0s, [11, 12, 13], block=0)
    tg = O.Target.dense_gauss(model.target["prec"], model.target["mean"])
    for c, sd in enumerate([11, 12, 13]):
        Xi, u = O.tape(sd, 0, 64, 512)
        S_ref, acc_ref, _ = O.mala_sequential(tg, 0.05, x0s[c].astype(np.float64), Xi, u)
        assert np.array_equal(acc[c], acc_ref), c
        assert trace_err(S[c].T, S_ref) <= 1e-5
        lp_ref = np.array([O.logp(tg, np.asarray(S[c, t], np.float64)) for t in range(0, 512, 51)])
        np.testing.assert_allclose(lp[c, ::51], lp_ref, rtol=1e-5, atol=1e-4)


def test_a_chain_is_the_trajectory_deer_converges_to():
    lam = 10 ** np.random.default_rng(2).uniform(-1, 1, 100)
    model = pmcmc.DensityModel.diag_gaussian(lam)
    sampler = pmcmc.ParallelMALASampler(0.05, T=2048, jacobian="diag", dtype=np.float32,
                                        tol_abs=1e-7, tol_rel=1e-6)
    x0 = np.random.default_rng(3).standard_normal(100).astype(np.float32)
    S, _, acc = pmcmc.mala_chains(model, sampler, x0[None], [9], block=4)
    Sd, info, _, accd = pmcmc.solve(model, sampler, x0, seed=9, block=4, return_logp=True)
    assert info["converged"]
    assert np.array_equal(acc[0], accd)
    assert trace_err(Sd, S[0].T) <= 1e-5


def test_chain_arguments():
    model = pmcmc.DensityModel.diag_gaussian(np.ones(3))
    s = pmcmc.ParallelMALASampler(0.1, T=8)
    with pytest.raises(pmcmc.DimensionMismatch):
        pmcmc.mala_chains(model, s, np.zeros((2, 3)), [1])
