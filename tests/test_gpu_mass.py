"""GPU parity of the mass-matrix path (cholM = cholesky(M)) against the FP64 CPU
oracle's sequential MALA chain with mass M on the same tape.

The reference threads cholM through every MALA step of the DEER recursion
(src/interface.jl:395-406 -> src/MALA/MALA.jl:29-47).  Bars: accept/reject
sequences bit-exact; positions within 1e-8 relative trace error for FP64 state
(the reference's FP64 bar is rtol 1e-6, test-Deer-vs-MALA.jl:106) and 1e-5 for
FP32 state, at stopping tolerances tight enough for those bars.
"""
import dataclasses

import numpy as np
import pytest

import oracle as O
import pmcmc

pytestmark = pytest.mark.gpu

# test-MALA-Kernel.jl:199-204
M_REF = np.array([[1.7, 0.2, -0.1], [0.2, 1.3, 0.15], [-0.1, 0.15, 1.5]])


@pytest.fixture(scope="module")
def h():
    return pmcmc.Handle(0)


def trace_err(S, R):
    S = np.asarray(S, np.float64)
    R = np.asarray(R, np.float64)
    return float(np.max(np.linalg.norm(S - R, axis=0) /
                        np.maximum(np.linalg.norm(R, axis=0), 1e-30)))


def _dense_case(D, seed):
    rng = np.random.default_rng(seed)
    A = rng.standard_normal((D, D))
    P = A @ A.T / D + np.eye(D)
    mu = rng.standard_normal(D)
    B = rng.standard_normal((D, D))
    M = 0.25 * (B @ B.T / D + 0.5 * np.eye(D))
    return P, mu, M, rng.standard_normal(D)


CASES = {
    # the reference's own mass matrix on a 3-d standard normal, eps 0.08
    "ref_M_std_normal": lambda: (pmcmc.DensityModel.diag_gaussian(np.ones(3)),
                                 O.Target.diag_gauss(np.ones(3)), M_REF, 0.08,
                                 np.random.default_rng(20260201).standard_normal(3)),
    "dense_D16": lambda: (lambda P, mu, M, x0: (pmcmc.DensityModel.dense_gaussian(P, mu),
                                                O.Target.dense_gauss(P, mu), M, 0.25, x0))(
        *_dense_case(16, 4)),
}


@pytest.mark.parametrize("dtype", [np.float64, np.float32])
@pytest.mark.parametrize("case", sorted(CASES))
@pytest.mark.parametrize("jac", ["stoch_diag", "diag"])
def test_mass_block_matches_sequential_mass_chain(h, case, dtype, jac):
    model, tg, M, eps, x0 = CASES[case]()
    D, T = model.dim, 256
    # the 3-d case has columns of norm 0.135, where the rule 1e-7 + 1e-6 max|S| leaves even
    # the FP64 oracle DEER 2.1e-5 from the chain; at 1e-8 + 2e-7 max|S| it is 3.6e-6
    tol = (1e-12, 1e-10) if dtype == np.float64 else (1e-8, 2e-7)
    sampler = pmcmc.ParallelMALASampler(eps, T=T, jacobian=jac, tol_abs=tol[0], tol_rel=tol[1],
                                        maxiter=400, dtype=dtype, cholM=pmcmc.cholesky(M))
    S, info, lp, acc = pmcmc.solve(model, sampler, x0.astype(dtype), seed=11, block=3, handle=h,
                                   return_logp=True)
    Xi, u = O.tape(11, 3, D, T)
    Lf = np.linalg.cholesky(M)
    S_seq, acc_seq, _ = O.mala_sequential_mass(tg, eps, Lf, x0.astype(dtype), Xi, u)
    assert info["converged"]
    assert 0 < (~acc_seq).sum() < T
    assert np.array_equal(acc, acc_seq)
    assert trace_err(S, S_seq) <= (1e-8 if dtype == np.float64 else 1e-5)
    # log p is coordinate-free: the base target's density at the returned states
    lp_ref = np.array([O.logp(tg, np.asarray(S[:, t], np.float64)) for t in range(T)])
    # FP32: the device evaluates log p in whitened coordinates from FP32 state
    np.testing.assert_allclose(lp, lp_ref, rtol=1e-5 if dtype == np.float32 else 1e-11,
                               atol=1e-4 if dtype == np.float32 else 1e-11)


def test_mass_sample_blocks_host_and_device(h):
    # several blocks through sample(): block b continues from block b-1's last state
    # (interface.jl:557-607), on host and device buffers alike
    torch = pytest.importorskip("torch")
    P, mu, M, x0 = _dense_case(16, 5)
    model = pmcmc.DensityModel.dense_gaussian(P, mu)
    T, nb = 128, 3
    sampler = pmcmc.ParallelMALASampler(0.25, T=T, tol_abs=1e-12, tol_rel=1e-10, maxiter=400,
                                        dtype=np.float64, cholM=pmcmc.cholesky(M))
    ch = pmcmc.sample(model, sampler, T * nb, seed=9, initial_params=x0, handle=h)
    chd = pmcmc.sample(model, sampler, T * nb, seed=9,
                       initial_params=torch.tensor(x0, device="cuda"), handle=h)
    np.testing.assert_array_equal(ch.values, chd.values.cpu().numpy())
    np.testing.assert_array_equal(ch.accepted, chd.accepted.cpu().numpy())
    tg = O.Target.dense_gauss(P, mu)
    Lf = np.linalg.cholesky(M)
    x = x0
    for b in range(nb):
        Xi, u = O.tape(9, b, 16, T)
        S_seq, acc_seq, _ = O.mala_sequential_mass(tg, 0.25, Lf, x, Xi, u)
        assert np.array_equal(ch.accepted[b * T:(b + 1) * T], acc_seq)
        assert trace_err(ch.values[b * T:(b + 1) * T].T, S_seq) <= 1e-8
        x = ch.values[(b + 1) * T - 1]


def test_mass_sequential_device_chains(h):
    # the device's sequential chains with the same mass matrix (MALASampler(eps; cholM),
    # interface.jl:84-100) against the oracle's, chain by chain
    P, mu, M, _ = _dense_case(8, 6)
    model = pmcmc.DensityModel.dense_gaussian(P, mu)
    sampler = pmcmc.ParallelMALASampler(0.25, T=200, dtype=np.float64, cholM=pmcmc.cholesky(M))
    n = 5
    x0s = np.random.default_rng(2).standard_normal((n, 8))
    seeds = np.arange(100, 100 + n, dtype=np.uint64)
    S, lp, acc = pmcmc.mala_chains(model, sampler, x0s, seeds, block=1, handle=h)
    tg = O.Target.dense_gauss(P, mu)
    Lf = np.linalg.cholesky(M)
    for c in range(n):
        Xi, u = O.tape(int(seeds[c]), 1, 8, 200)
        S_seq, acc_seq, _ = O.mala_sequential_mass(tg, 0.25, Lf, x0s[c], Xi, u)
        assert np.array_equal(acc[c], acc_seq)
        assert np.max(np.abs(S[c].T - S_seq)) <= 1e-10


def test_identity_mass_is_the_plain_chain(h):
    D, T = 12, 128
    lam = 10 ** np.linspace(-0.5, 0.5, D)
    model = pmcmc.DensityModel.diag_gaussian(lam)
    x0 = np.random.default_rng(3).standard_normal(D)
    base = pmcmc.ParallelMALASampler(0.2, T=T, tol_abs=1e-12, tol_rel=1e-10, maxiter=400,
                                     dtype=np.float64)
    withI = dataclasses.replace(base, cholM=np.eye(D))
    S0, i0, _, a0 = pmcmc.solve(model, base, x0, seed=1, handle=h, return_logp=True)
    S1, i1, _, a1 = pmcmc.solve(model, withI, x0, seed=1, handle=h, return_logp=True)
    assert i0["converged"] and i1["converged"] and np.array_equal(a0, a1)
    assert trace_err(S1, S0) <= 1e-10


def test_mass_unsupported_paths(h):
    rng = np.random.default_rng(0)
    X = rng.standard_normal((50, 4))
    y = (rng.random(50) < 0.5).astype(float)
    lg = pmcmc.DensityModel.logistic(X, y)
    s = pmcmc.ParallelMALASampler(0.05, T=32, cholM=np.eye(4), dtype=np.float32)
    with pytest.raises(pmcmc.Unsupported):
        pmcmc.solve(lg, s, np.zeros(4, np.float32), handle=h)
    g = pmcmc.DensityModel.diag_gaussian(np.ones(4))
    S, _ = pmcmc.solve(g, s, np.zeros(4, np.float32), handle=h)
    with pytest.raises(pmcmc.Unsupported):
        pmcmc.adjoint(g, s, np.zeros(4, np.float32), S, handle=h)
    with pytest.raises(pmcmc.DimensionMismatch):
        pmcmc.solve(pmcmc.DensityModel.diag_gaussian(np.ones(5)), s, np.zeros(5, np.float32),
                    handle=h)


def test_mass_with_full_jacobian_and_in_the_fleet(h):
    # the whitened target is a dense Gaussian, so :full (eigenbasis scan) and the fleet
    # take it as they take any dense target
    P, mu, M, x0 = _dense_case(16, 8)
    model = pmcmc.DensityModel.dense_gaussian(P, mu)
    T, eps = 512, 0.25
    Lf = np.linalg.cholesky(M)
    tg = O.Target.dense_gauss(P, mu)
    full = pmcmc.ParallelMALASampler(eps, T=T, jacobian="full", dtype=np.float32, tol_abs=1e-8,
                                     tol_rel=2e-7, maxiter=400, cholM=pmcmc.cholesky(M))
    S, info, _, acc = pmcmc.solve(model, full, x0.astype(np.float32), seed=13, handle=h,
                                  return_logp=True)
    Xi, u = O.tape(13, 0, 16, T)
    S_seq, acc_seq, _ = O.mala_sequential_mass(tg, eps, Lf, x0.astype(np.float32), Xi, u)
    assert info["converged"] and info["path"] & 16
    assert np.array_equal(acc, acc_seq)
    assert trace_err(S, S_seq) <= 1e-5
    diag = dataclasses.replace(full, jacobian="diag", dtype=np.float64, tol_abs=1e-12,
                               tol_rel=1e-10)
    chains = [(model, diag, x0 + 0.1 * k, 20 + k, 0) for k in range(4)]
    res = pmcmc.fleet_solve(chains, workers=4, handle=h)
    for k, (Sk, ik, _, ak) in enumerate(res):
        Xi, u = O.tape(20 + k, 0, 16, T)
        S_ref, acc_ref, _ = O.mala_sequential_mass(tg, eps, Lf, x0 + 0.1 * k, Xi, u)
        assert ik["converged"] and np.array_equal(ak, acc_ref)
        assert trace_err(Sk, S_ref) <= 1e-8
