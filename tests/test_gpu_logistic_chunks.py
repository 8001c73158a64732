"""Logistic blocks solved in chunks (window W < T): chunk k is a DEER solve of
its own on tape columns [k W, k W + W) of the block, started from the end of
chunk k - 1.  The chain is Markov, so the chunks reproduce the block's
sequential chain: accept flags identical to the FP64 oracle chain, positions
within 1e-5 relative trace error (FP32 state) at a rule of 1e-8 + 1e-7 max|S|."""
import numpy as np
import pytest

import oracle as O
import pmcmc

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def h():
    return pmcmc.Handle(0)


def trace_err(S, R):
    S = np.asarray(S, np.float64)
    R = np.asarray(R, np.float64)
    return float(np.max(np.linalg.norm(S - R, axis=0) /
                        np.maximum(np.linalg.norm(R, axis=0), 1e-30)))


def _problem(N, D, seed):
    rng = np.random.default_rng(seed)
    X = (rng.standard_normal((N, D)) / np.sqrt(D)).astype(np.float32).astype(np.float64)
    th = rng.standard_normal(D)
    y = (rng.random(N) < 1 / (1 + np.exp(-X @ th))).astype(np.float64)
    return X, y


# the wide pass (D > 256) stalls about 2 ulp above a rule of 1e-8 + 1e-7 max|S| (an FP32
# floor, not the chunking): it is given 5e-8 + 5e-7 max|S|
@pytest.mark.parametrize("exec_,D,W,rtol", [("fused", 24, 96, 1e-7), ("fused", 300, 100, 5e-7),
                                            ("plain", 24, 128, 1e-7), ("fused", 24, 97, 1e-7)])
def test_chunks_reproduce_the_sequential_chain(h, exec_, D, W, rtol):
    N, T, eps = 400, 512, 0.02
    X, y = _problem(N, D, 41)
    model = pmcmc.DensityModel.logistic(X, y)
    sampler = pmcmc.ParallelMALASampler(eps, T=T, window=W, dtype=np.float32, exec=exec_,
                                        tol_abs=rtol / 10, tol_rel=rtol, maxiter=400)
    S, info, lp, acc = pmcmc.solve(model, sampler, np.zeros(D, np.float32), seed=5, block=2,
                                   handle=h, return_logp=True)
    tg = O.Target.logistic(X, y)
    Xi, u = O.tape(5, 2, D, T)
    S_seq, acc_seq, _ = O.mala_sequential(tg, eps, np.zeros(D), Xi, u)
    assert info["converged"], info
    assert 0 < (~acc_seq).sum() < T
    assert np.array_equal(acc, acc_seq)
    assert trace_err(S, S_seq) <= 1e-5
    assert info["n_accept"] == int(acc_seq.sum())
    lp_ref = np.array([O.logp(tg, np.asarray(S[:, t], np.float64)) for t in range(0, T, 31)])
    np.testing.assert_allclose(lp[::31], lp_ref, rtol=1e-5, atol=1e-4)


def test_chunked_sample_over_blocks_host_and_device(h):
    # sample() of 2.5 blocks (interface.jl:557-607) with chunked blocks, on host and
    # device buffers: the same chain, block b continuing from block b - 1
    torch = pytest.importorskip("torch")
    N, D, T, W, eps = 300, 16, 256, 64, 0.02
    X, y = _problem(N, D, 43)
    model = pmcmc.DensityModel.logistic(X, y)
    sampler = pmcmc.ParallelMALASampler(eps, T=T, window=W, dtype=np.float32,
                                        tol_abs=1e-8, tol_rel=1e-7, maxiter=400)
    n = 2 * T + T // 2
    ch = pmcmc.sample(model, sampler, n, seed=3, initial_params=np.zeros(D, np.float32),
                      handle=h)
    chd = pmcmc.sample(model, sampler, n, seed=3,
                       initial_params=torch.zeros(D, dtype=torch.float32, device="cuda"),
                       handle=h)
    np.testing.assert_array_equal(ch.values, chd.values.cpu().numpy())
    np.testing.assert_array_equal(ch.accepted, chd.accepted.cpu().numpy())
    assert ch.info["converged"]
    tg = O.Target.logistic(X, y)
    x = np.zeros(D)
    for b in range(3):
        keep = min(T, n - b * T)
        Xi, u = O.tape(3, b, D, T)
        S_seq, acc_seq, _ = O.mala_sequential(tg, eps, x, Xi, u)
        assert np.array_equal(ch.accepted[b * T:b * T + keep], acc_seq[:keep])
        assert trace_err(ch.values[b * T:b * T + keep].T, S_seq[:, :keep]) <= 1e-5
        x = np.asarray(ch.values[b * T + keep - 1], np.float64)
