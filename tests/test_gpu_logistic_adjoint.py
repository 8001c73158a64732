"""The logistic adjoint on the device (d objective / d epsilon at a returned
trajectory, accept decisions held fixed) against the dense FP64 restatement of
the oracle at the same trajectory (1e-8 relative for FP64 state, 1e-6 for FP32)
and against central finite differences of the sequential trace's objective
that flip no accept (1e-4 relative, the Gaussian adjoint's bar)."""
import numpy as np
import pytest

import np_oracle as NO
import oracle as O
import pmcmc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def h():
    return pmcmc.Handle(0)


def _problem(N, D, seed):
    rng = np.random.default_rng(seed)
    X = (rng.standard_normal((N, D)) / np.sqrt(D)).astype(np.float32).astype(np.float64)
    th = rng.standard_normal(D)
    y = (rng.random(N) < 1 / (1 + np.exp(-X @ th))).astype(np.float64)
    return X, y


@pytest.mark.parametrize("objective", ["esjd", "mean_sq"])
def test_fp64_adjoint_matches_the_restatement_and_fd(h, objective):
    N, D, T, eps, seed, block = 200, 8, 256, 0.05, 4, 1
    X, y = _problem(N, D, 51)
    model = pmcmc.DensityModel.logistic(X, y)
    sampler = pmcmc.ParallelMALASampler(eps, T=T, dtype=np.float64, tol_abs=1e-12,
                                        tol_rel=1e-10, maxiter=400)
    x0 = np.random.default_rng(2).standard_normal(D) * 0.3
    S, info = pmcmc.solve(model, sampler, x0, seed=seed, block=block, handle=h)
    assert info["converged"]
    g = pmcmc.adjoint(model, sampler, x0, S, objective=objective, seed=seed, block=block,
                      handle=h)
    assert g["d_log_s"] is None
    Xi, u = O.tape(seed, block, D, T)
    ref = NO.logistic_adjoint(X, y, eps, x0, Xi, u, np.asarray(S), objective)
    assert abs(g["d_epsilon"] - ref) <= 1e-8 * abs(ref)
    hh = 1e-6 * eps
    ep, mp, _, ap = NO.logistic_objectives(X, y, eps + hh, x0, Xi, u)
    em, mm, _, am = NO.logistic_objectives(X, y, eps - hh, x0, Xi, u)
    _, _, _, acc = NO.logistic_objectives(X, y, eps, x0, Xi, u)
    assert np.array_equal(ap, acc) and np.array_equal(am, acc) and 0 < (~acc).sum() < T
    fd = ((ep - em) if objective == "esjd" else (mp - mm)) / (2 * hh)
    assert abs(g["d_epsilon"] - fd) <= 1e-4 * abs(fd)


def test_fp32_adjoint_on_a_tensor_core_trajectory(h):
    # FP32 state solved on the tensor cores; the adjoint runs in FP64 at that trajectory
    N, D, T, eps = 600, 48, 1024, 0.02
    X, y = _problem(N, D, 52)
    model = pmcmc.DensityModel.logistic(X, y)
    sampler = pmcmc.ParallelMALASampler(eps, T=T, dtype=np.float32, tol_abs=1e-7,
                                        tol_rel=1e-6, maxiter=400)
    x0 = np.zeros(D, np.float32)
    S, info = pmcmc.solve(model, sampler, x0, seed=6, handle=h)
    assert info["converged"] and info["path"] & 8
    Xi, u = O.tape(6, 0, D, T)
    for objective in ("esjd", "mean_sq"):
        g = pmcmc.adjoint(model, sampler, x0, S, objective=objective, seed=6, handle=h)
        ref = NO.logistic_adjoint(X, y, eps, x0.astype(np.float64), Xi, u,
                                  np.asarray(S, np.float64), objective)
        assert abs(g["d_epsilon"] - ref) <= 1e-6 * abs(ref), objective


def test_adjoint_rejects_a_mass_matrix_on_logistic(h):
    X, y = _problem(50, 4, 53)
    model = pmcmc.DensityModel.logistic(X, y)
    s = pmcmc.ParallelMALASampler(0.05, T=16, dtype=np.float64)
    S, _ = pmcmc.solve(model, s, np.zeros(4), handle=h)
    with pytest.raises(pmcmc.Unsupported):
        pmcmc.adjoint(model, pmcmc.ParallelMALASampler(0.05, T=16, dtype=np.float64,
                                                       cholM=np.eye(4)), np.zeros(4), S,
                      handle=h)
