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


@pytest.mark.parametrize("mass", [False, True])
def test_adaptive_chains_match_the_oracle(mass):
    # AdaptiveMALASampler chains on the device (src/interface.jl:1024-1065) against the
    # oracle's chain on the same tapes: FP64 state, every step size and decision
    from pmcmc import AdaptiveMALASampler
    lam = np.array([0.5, 1.0, 2.0, 4.0, 8.0, 0.25])
    D, T, n_w = 6, 600, 400
    model = pmcmc.DensityModel.diag_gaussian(lam)
    tg = O.Target.diag_gauss(lam)
    L = None
    if mass:
        B = np.random.default_rng(9).standard_normal((D, D))
        L = np.linalg.cholesky(0.2 * (B @ B.T / D + np.eye(D)))
    ad = AdaptiveMALASampler(0.01, n_warmup=n_w, cholM=L)
    seeds = [21, 22, 23]
    x0 = np.random.default_rng(4).standard_normal((3, D))
    r = pmcmc.adaptive_chains(model, ad, x0, seeds, T, block=1)
    for c, sd in enumerate(seeds):
        Xi, u = O.tape(sd, 1, D, T)
        if mass:
            # the oracle's adaptive chain on the whitened target, mapped back
            Pw = L.T @ np.diag(lam) @ L
            tw = O.Target.dense_gauss(0.5 * (Pw + Pw.T))
            Sw, acc_ref, used, fin = O.mala_adaptive(tw, 0.01, np.linalg.solve(L, x0[c]), Xi, u,
                                                     n_w)
            S_ref = L @ Sw
        else:
            S_ref, acc_ref, used, fin = O.mala_adaptive(tg, 0.01, x0[c], Xi, u, n_w)
        assert np.array_equal(r["accepted"][c], acc_ref), c
        # with a mass matrix the library and the oracle form L^T P L in different orders;
        # the dual averaging amplifies those last-bit differences of log alpha to ~3e-9
        rt = 1e-8 if mass else 1e-10
        np.testing.assert_allclose(r["step_size"][c], used, rtol=rt)
        np.testing.assert_allclose(S_ref, r["S"][c].T, rtol=10 * rt, atol=rt)
        np.testing.assert_allclose([r["epsilon"][c], r["epsilon_bar"][c], r["H_bar"][c]], fin,
                                   rtol=rt, atol=1e-13)
    assert np.all(r["step_size"][:, n_w:] == r["epsilon_bar"][:, None])
    assert np.array_equal(r["is_warmup"][0], np.arange(T) < n_w)


def test_sample_with_adaptive_sampler():
    # sample(model, AdaptiveMALASampler(...), N), test-Adaptive-MALA.jl:144-213: the
    # initial transition, warmup flags, a frozen step size after warmup, and the adapted
    # acceptance rate near its target
    from pmcmc import AdaptiveMALASampler
    model = pmcmc.DensityModel.diag_gaussian(np.ones(5))
    n_w = 2000
    ch = pmcmc.sample(model, AdaptiveMALASampler(0.5, n_warmup=n_w), n_w + 501, seed=42,
                      initial_params=np.zeros(5))
    assert len(ch) == n_w + 501
    assert np.array_equal(ch.values[0], np.zeros(5)) and ch.info["step_size"][0] == 0.5
    assert ch.info["is_warmup"][0] and not ch.info["is_warmup"][-1]
    post = ch.info["step_size"][~ch.info["is_warmup"]]
    assert np.all(post == ch.info["epsilon_bar"]) and np.all(ch.info["step_size"] > 0)
    assert 0.35 < ch.accepted[n_w + 1:].mean() < 0.80
    assert np.all(np.isfinite(ch.logp))


def test_adaptive_settings_are_checked_by_the_library():
    # the constructor checks of src/interface.jl:919-923, in the C ABI
    import ctypes as C
    from pmcmc import _lib as L
    h = pmcmc.default_handle(0)
    model = pmcmc.DensityModel.diag_gaussian(np.ones(3))
    smp = pmcmc.ParallelMALASampler(0.1, T=8)
    tgt = smp.target(model, h)
    x = np.zeros(3)
    sd = np.array([1], np.uint64)
    S = np.empty((8, 3))
    p = smp.params()
    for bad in (dict(target_accept=1.0), dict(gamma=0.0), dict(t0=-1.0), dict(kappa=0.5),
                dict(n_warmup=-1)):
        kw = dict(n_warmup=4, target_accept=0.574, gamma=0.05, t0=10.0, kappa=0.75)
        kw.update(bad)
        ad = L.Adapt(kw["n_warmup"], kw["target_accept"], kw["gamma"], kw["t0"], kw["kappa"])
        rc = L.load().pmcmc_mala_chains_adaptive(h.ptr, tgt, C.byref(p), 1, x.ctypes.data,
                                                 sd.ctypes.data, 0, C.byref(ad), S.ctypes.data,
                                                 None, None, None, None, L.MEM_HOST)
        assert rc == L.ERR_ARGUMENT, bad
