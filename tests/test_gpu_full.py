"""GPU parity of the dense-Jacobian (:full) mode and of the adjoint pass.

Bars (tolerances are written in each test):
  * accept/reject sequences: bit-exact against the FP64 sequential oracle;
  * trajectories: 1e-5 relative trace error (FP32 state vs the FP64 oracle);
  * Newton iterations: within 2 of the FP64 CPU DEER with the exact dense
    Jacobian (oracle deer_solve(jacobian="full")), which takes the same Newton
    steps in exact arithmetic;
  * adjoint: the FP64 adjoint restatement evaluated at the GPU trajectory to
    1e-4 relative, and central finite differences of the FP64 sequential
    trace (accept flags identical at +-h) to 1e-4 relative.
"""
import numpy as np
import pytest

import np_oracle as NP
import oracle as O
import pmcmc
from pmcmc import configs

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def h():
    return pmcmc.Handle(0)


def trace_err(S, R):
    S = np.asarray(S, np.float64)
    R = np.asarray(R, np.float64)
    return float(np.max(np.linalg.norm(S - R, axis=0) /
                        np.maximum(np.linalg.norm(R, axis=0), 1e-30)))


def _corr(D, seed):
    rng = np.random.default_rng(seed)
    s = 10.0 ** rng.uniform(-1.0, 1.0, D)
    Q = configs.haar_orthogonal(rng, D)
    P = (Q / s) @ Q.T
    return 0.5 * (P + P.T), Q, s, rng


def _sampler(T, **kw):
    base = dict(T=T, jacobian="full", dtype=np.float32, tol_abs=1e-7, tol_rel=1e-6, maxiter=200)
    base.update(kw)
    return pmcmc.ParallelMALASampler(0.05, **base)


@pytest.mark.parametrize("D,T,seed", [(8, 256, 1), (30, 1000, 2), (64, 2048, 3), (100, 700, 4)])
def test_full_dense_matches_sequential_and_cpu_newton(h, D, T, seed):
    P, Q, s, rng = _corr(D, seed)
    x0 = rng.standard_normal(D).astype(np.float32)
    model = pmcmc.DensityModel.dense_gaussian(P)
    S, info, lp, acc = pmcmc.solve(model, _sampler(T), x0, seed=seed, block=1, handle=h,
                                   return_logp=True)
    assert "full_jacobian" in info["path_names"] and "graph" in info["path_names"]
    tg = O.Target.dense_gauss(P)
    Xi, u = O.tape(seed, 1, D, T)
    S_seq, acc_seq, _ = O.mala_sequential(tg, 0.05, x0.astype(np.float64), Xi, u)
    assert info["converged"], info
    assert np.array_equal(acc, acc_seq.astype(bool)), np.nonzero(acc != acc_seq)[0][:5]
    assert 0.05 < acc.mean() < 1.0
    assert trace_err(S, S_seq) <= 1e-5
    if T <= 1000:
        _, icpu = O.deer_solve(tg, 0.05, x0.astype(np.float64), Xi, u, seed, 1, jacobian="full",
                               tol_abs=1e-7, tol_rel=1e-6, maxiter=200)
        assert icpu["converged"]
        assert abs(info["iters"] - icpu["iters"]) <= 2, (info["iters"], icpu["iters"])


def test_full_diag_target(h):
    rng = np.random.default_rng(7)
    D, T = 10, 900
    lam = 10 ** rng.uniform(-1, 1, D)
    x0 = rng.standard_normal(D).astype(np.float32)
    model = pmcmc.DensityModel.diag_gaussian(lam)
    S, info, lp, acc = pmcmc.solve(model, _sampler(T), x0, seed=5, handle=h, return_logp=True)
    Xi, u = O.tape(5, 0, D, T)
    S_seq, acc_seq, _ = O.mala_sequential(O.Target.diag_gauss(lam), 0.05, x0.astype(np.float64),
                                          Xi, u)
    assert info["converged"]
    assert np.array_equal(acc, acc_seq.astype(bool))
    assert trace_err(S, S_seq) <= 1e-5


def test_full_fewer_sweeps_than_diagonal_jacobian(h):
    model, sampler, x0, meta = configs.correlated_gauss_d64(T=1024)
    kw = dict(tol_abs=1e-7, tol_rel=1e-6, maxiter=2000)
    _, i_full = pmcmc.solve(model, _sampler(1024, **kw), x0, seed=3, handle=h)
    _, i_diag = pmcmc.solve(model, _sampler(1024, jacobian="diag", **kw), x0, seed=3, handle=h)
    assert i_full["converged"] and i_diag["converged"]
    assert i_full["iters"] < i_diag["iters"], (i_full["iters"], i_diag["iters"])


@pytest.mark.parametrize("chunks", ["1", "7", "300"])
def test_full_chunking_does_not_change_the_answer(monkeypatch, h, chunks):
    P, Q, s, rng = _corr(16, 12)
    x0 = rng.standard_normal(16).astype(np.float32)
    model = pmcmc.DensityModel.dense_gaussian(P)
    S0, i0 = pmcmc.solve(model, _sampler(600), x0, seed=2, handle=h)
    monkeypatch.setenv("PMCMC_FULL_CHUNKS", chunks)
    hc = pmcmc.Handle(0)
    monkeypatch.delenv("PMCMC_FULL_CHUNKS")
    model2 = pmcmc.DensityModel.dense_gaussian(P)
    S1, i1 = pmcmc.solve(model2, _sampler(600), x0, seed=2, handle=hc)
    assert i0["converged"] and i1["converged"]
    assert trace_err(S1, S0) <= 1e-5
    assert abs(i0["iters"] - i1["iters"]) <= 2


def test_full_eager_matches_graph(monkeypatch):
    monkeypatch.setenv("PMCMC_EAGER", "1")
    he = pmcmc.Handle(0)
    monkeypatch.delenv("PMCMC_EAGER")
    hg = pmcmc.Handle(0)
    P, Q, s, rng = _corr(12, 13)
    x0 = rng.standard_normal(12).astype(np.float32)
    model = pmcmc.DensityModel.dense_gaussian(P)
    Se, ie = pmcmc.solve(model, _sampler(500), x0, seed=4, handle=he)
    Sg, ig = pmcmc.solve(model, _sampler(500), x0, seed=4, handle=hg)
    assert ie["iters"] == ig["iters"]
    np.testing.assert_array_equal(Se, Sg)


def test_full_config4_full_size(h):
    """The D = 64, T = 8192 correlated-Gaussian workload against the FP64
    sequential oracle."""
    model, sampler, x0, meta = configs.correlated_gauss_d64()
    sampler.tol_abs, sampler.tol_rel = 1e-7, 1e-6
    S, info, lp, acc = pmcmc.solve(model, sampler, x0, seed=meta["seed"], handle=h,
                                   return_logp=True)
    tg = O.Target.dense_gauss(model.target["prec"])
    Xi, u = O.tape(meta["seed"], 0, 64, sampler.T)
    S_seq, acc_seq, la = O.mala_sequential(tg, 0.05, x0.astype(np.float64), Xi, u)
    assert info["converged"], info
    assert np.array_equal(acc, acc_seq.astype(bool)), np.nonzero(acc != acc_seq)[0][:5]
    assert trace_err(S, S_seq) <= 1e-5


def test_eigen_reconstructs_precision(h):
    P, Q, s, rng = _corr(20, 21)
    model = pmcmc.DensityModel.dense_gaussian(P)
    lam, V = model.eigen(handle=h)
    assert np.all(np.diff(lam) >= 0)
    np.testing.assert_allclose((V * lam) @ V.T, P, atol=1e-10 * np.abs(P).max())
    np.testing.assert_allclose(V.T @ V, np.eye(20), atol=1e-12)
    np.testing.assert_allclose(np.sort(1.0 / s), lam, rtol=1e-10)


def test_full_unsupported_modes(h):
    X = np.random.default_rng(0).standard_normal((50, 4))
    y = (X[:, 0] > 0).astype(float)
    with pytest.raises(pmcmc.Unsupported):
        pmcmc.solve(pmcmc.DensityModel.logistic(X, y), _sampler(64), np.zeros(4, np.float32),
                    handle=h)
    g = pmcmc.DensityModel.diag_gaussian(np.ones(4))
    with pytest.raises(pmcmc.Unsupported):
        pmcmc.solve(g, pmcmc.ParallelMALASampler(0.05, T=64, jacobian="full"), np.zeros(4),
                    handle=h)  # FP64 state
    with pytest.raises(pmcmc.Unsupported):
        pmcmc.solve(g, _sampler(64, window=16), np.zeros(4, np.float32), handle=h)
    with pytest.raises(pmcmc.Unsupported):
        pmcmc.solve(pmcmc.DensityModel.diag_gaussian(np.ones(200)), _sampler(64),
                    np.zeros(200, np.float32), handle=h)


# --------------------------------------------------------------------------- adjoint
def _adjoint_problem(D, T, seed, dense=True):
    P, Q, s, rng = _corr(D, seed)
    if not dense:
        s = 10.0 ** rng.uniform(-1.0, 1.0, D)
        P, Q = np.diag(1.0 / s), np.eye(D)
    x0 = rng.standard_normal(D).astype(np.float32)
    return P, Q, s, x0


@pytest.mark.parametrize("objective", ["esjd", "mean_sq"])
@pytest.mark.parametrize("dense", [True, False])
def test_adjoint_matches_oracle_and_fd(h, objective, dense):
    D, T, eps = 8, 256, 0.05
    P, Q, s, x0 = _adjoint_problem(D, T, 31, dense)
    model = (pmcmc.DensityModel.dense_gaussian(P) if dense
             else pmcmc.DensityModel.diag_gaussian(1.0 / s))
    sampler = _sampler(T, tol_abs=1e-8, tol_rel=1e-7)
    S, info = pmcmc.solve(model, sampler, x0, seed=6, handle=h)
    assert info["converged"]
    g = pmcmc.adjoint(model, sampler, x0, S, objective=objective, seed=6, handle=h)
    Xi, u = O.tape(6, 0, D, T)
    x0d = x0.astype(np.float64)
    # (1) the FP64 restatement evaluated at the GPU trajectory
    lam, V = model.eigen(handle=h)
    ge, gls = NP.gauss_adjoint(P, None, eps, x0d, Xi, u, np.asarray(S, np.float64), objective,
                               Q=V, s=1.0 / lam)
    assert abs(g["d_epsilon"] - ge) <= 1e-4 * max(1.0, abs(ge)), (g["d_epsilon"], ge)
    if objective == "mean_sq":
        np.testing.assert_allclose(g["d_log_s"], gls, rtol=1e-4, atol=1e-4 * np.abs(gls).max())
    # (2) central differences of the FP64 sequential trace
    _, _, _, acc = NP.gauss_objectives(P, None, eps, x0d, Xi, u)
    hh = 1e-6 * eps
    rp = NP.gauss_objectives(P, None, eps + hh, x0d, Xi, u)
    rm = NP.gauss_objectives(P, None, eps - hh, x0d, Xi, u)
    assert np.array_equal(rp[3], acc) and np.array_equal(rm[3], acc)
    k = 0 if objective == "esjd" else 1
    fd = (rp[k] - rm[k]) / (2 * hh)
    assert abs(g["d_epsilon"] - fd) <= 1e-4 * max(1.0, abs(fd)), (g["d_epsilon"], fd)


def test_adjoint_log_s_matches_fd(h):
    D, T, eps = 6, 200, 0.05
    P, Q, s, x0 = _adjoint_problem(D, T, 41)
    model = pmcmc.DensityModel.dense_gaussian(P)
    sampler = _sampler(T, tol_abs=1e-8, tol_rel=1e-7)
    S, info = pmcmc.solve(model, sampler, x0, seed=8, handle=h)
    g = pmcmc.adjoint(model, sampler, x0, S, objective="mean_sq", seed=8, handle=h)
    lam, V = model.eigen(handle=h)
    Xi, u = O.tape(8, 0, D, T)
    x0d = x0.astype(np.float64)
    _, _, _, acc = NP.gauss_objectives(P, None, eps, x0d, Xi, u)
    sv = 1.0 / lam
    for i in range(D):
        vals = []
        for sg in (1, -1):
            s2 = sv.copy()
            s2[i] *= np.exp(sg * 1e-6)
            P2 = (V / s2) @ V.T
            r = NP.gauss_objectives(0.5 * (P2 + P2.T), None, eps, x0d, Xi, u)
            assert np.array_equal(r[3], acc)
            vals.append(r[1])
        fd = (vals[0] - vals[1]) / 2e-6
        assert abs(g["d_log_s"][i] - fd) <= 1e-4 * max(1.0, abs(fd)), (i, g["d_log_s"][i], fd)


def test_adjoint_config4_full_size(h):
    """The adjoint at the D = 64, T = 8192 correlated-Gaussian workload against
    central differences of the FP64 sequential trace that flip no accept:
    d ESJD / d eps, d mean|x|^2 / d eps and d mean|x|^2 / d log s_i for eight
    eigenvalues across the spectrum, each within 1e-4 relative."""
    model, sampler, x0, meta = configs.correlated_gauss_d64()
    sampler.tol_abs, sampler.tol_rel = 1e-8, 1e-7
    eps, T, D = sampler.epsilon, sampler.T, model.dim
    S, info = pmcmc.solve(model, sampler, x0, seed=meta["seed"], handle=h)
    assert info["converged"], info
    P = model.target["prec"]
    Xi, u = O.tape(meta["seed"], 0, D, T)
    x0d = x0.astype(np.float64)
    _, _, _, acc = NP.gauss_objectives(P, None, eps, x0d, Xi, u)
    hh = 1e-6 * eps
    rp = NP.gauss_objectives(P, None, eps + hh, x0d, Xi, u)
    rm = NP.gauss_objectives(P, None, eps - hh, x0d, Xi, u)
    assert np.array_equal(rp[3], acc) and np.array_equal(rm[3], acc)
    for k, objective in enumerate(("esjd", "mean_sq")):
        g = pmcmc.adjoint(model, sampler, x0, S, objective=objective, seed=meta["seed"],
                          handle=h)
        fd = (rp[k] - rm[k]) / (2 * hh)
        assert abs(g["d_epsilon"] - fd) <= 1e-4 * max(1.0, abs(fd)), (objective, g["d_epsilon"], fd)
    lam, V = model.eigen(handle=h)
    sv = 1.0 / lam
    for i in np.linspace(0, D - 1, 8).astype(int):
        vals = []
        for sg in (1, -1):
            s2 = sv.copy()
            s2[i] *= np.exp(sg * 1e-6)
            P2 = (V / s2) @ V.T
            r = NP.gauss_objectives(0.5 * (P2 + P2.T), None, eps, x0d, Xi, u)
            assert np.array_equal(r[3], acc)
            vals.append(r[1])
        fd = (vals[0] - vals[1]) / 2e-6
        assert abs(g["d_log_s"][i] - fd) <= 1e-4 * max(1.0, abs(fd)), (i, g["d_log_s"][i], fd)
