"""T-split slices on one GPU (pmcmc.distributed.local_tsplit: one handle per
slice, run in lockstep) against the single-device solve of the same block.

Bars: FP64 state -- the unfused plain path takes the same Newton steps, so
trajectories agree to 1e-10 and iteration counts are equal; FP32 state -- the
fused solve's trajectory to 1e-5 relative trace error, identical accepts."""
import numpy as np
import pytest

import oracle as O
import pmcmc
from pmcmc import configs
from pmcmc import distributed as Dd

pytestmark = pytest.mark.gpu


def trace_err(S, R):
    S, R = np.asarray(S, np.float64), np.asarray(R, np.float64)
    return float(np.max(np.linalg.norm(S - R, axis=0) / np.maximum(np.linalg.norm(R, axis=0),
                                                                   1e-30)))


@pytest.mark.parametrize("jac", ["diag", "stoch_diag"])
@pytest.mark.parametrize("nslices", [1, 3, 8])
def test_fp64_slices_match_plain_solve(jac, nslices):
    rng = np.random.default_rng(5)
    D, T = 10, 600
    lam = 10 ** rng.uniform(-1, 1, D)
    x0 = rng.standard_normal(D)
    model = pmcmc.DensityModel.diag_gaussian(lam)
    kw = dict(T=T, jacobian=jac, tol_abs=1e-10, tol_rel=1e-9, maxiter=500, dtype=np.float64)
    S_ref, info = pmcmc.solve(model, pmcmc.ParallelMALASampler(0.05, exec="plain", **kw), x0,
                              seed=9, block=2)
    S, acc, iters, conv = Dd.local_tsplit(model, pmcmc.ParallelMALASampler(0.05, **kw), x0,
                                          nslices, seed=9, block=2)
    assert conv and info["converged"]
    assert iters == info["iters"]
    np.testing.assert_allclose(S, S_ref, rtol=1e-10, atol=1e-12)
    Xi, u = O.tape(9, 2, D, T)
    _, acc_seq, _ = O.mala_sequential(O.Target.diag_gauss(lam), 0.05, x0, Xi, u)
    assert np.array_equal(acc, acc_seq.astype(bool))


def test_fp32_headline_workload_in_four_slices():
    model, sampler, x0, meta = configs.aniso_diag_d100()
    S_ref, info, lp, acc_ref = pmcmc.solve(model, sampler, x0, seed=meta["seed"],
                                           return_logp=True)
    S, acc, iters, conv = Dd.local_tsplit(model, sampler, x0, 4, seed=meta["seed"])
    assert conv
    assert np.array_equal(acc, acc_ref)
    assert trace_err(S, S_ref) <= 1e-5


def test_dense_target_slices():
    rng = np.random.default_rng(8)
    D, T = 12, 400
    Q = configs.haar_orthogonal(rng, D)
    s = 10 ** rng.uniform(-1, 1, D)
    P = (Q / s) @ Q.T
    P = 0.5 * (P + P.T)
    x0 = rng.standard_normal(D)
    model = pmcmc.DensityModel.dense_gaussian(P)
    kw = dict(T=T, jacobian="diag", tol_abs=1e-10, tol_rel=1e-9, maxiter=2000, dtype=np.float64)
    S_ref, info = pmcmc.solve(model, pmcmc.ParallelMALASampler(0.05, exec="plain", **kw), x0,
                              seed=4)
    S, acc, iters, conv = Dd.local_tsplit(model, pmcmc.ParallelMALASampler(0.05, **kw), x0, 5,
                                          seed=4)
    assert conv and iters == info["iters"]
    np.testing.assert_allclose(S, S_ref, rtol=1e-9, atol=1e-11)


def test_slice_argument_errors():
    h = pmcmc.Handle(0)
    X = np.random.default_rng(0).standard_normal((40, 3))
    lg = pmcmc.DensityModel.logistic(X, (X[:, 0] > 0).astype(float))
    s = pmcmc.ParallelMALASampler(0.05, T=64, dtype=np.float32)
    with pytest.raises(pmcmc.Unsupported):
        Dd.DeviceSlice(lg, s, h).begin(np.zeros(3), 0, 0, 0, 32)
    g = pmcmc.DensityModel.diag_gaussian(np.ones(3))
    with pytest.raises(pmcmc.DimensionMismatch):
        Dd.DeviceSlice(g, s, h).begin(np.zeros(3), 0, 0, 40, 32)
    with pytest.raises(pmcmc.Unsupported):
        Dd.DeviceSlice(g, pmcmc.ParallelMALASampler(0.05, T=64, jacobian="full",
                                                     dtype=np.float32), h).begin(
            np.zeros(3), 0, 0, 0, 32)
