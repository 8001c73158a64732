"""The oracle reproduces the committed known-answer fixtures (tests/golden/make_golden.py)."""
import os

import numpy as np

import oracle as O

G = np.load(os.path.join(os.path.dirname(__file__), "golden", "golden_v1.npz"))


def test_tape_fixtures_bit_exact():
    for (seed, block, D, T) in [(0, 0, 5, 8), (7, 3, 2, 16), (2**40 + 5, 9, 13, 4)]:
        Xi, u = O.tape(seed, block, D, T)
        assert np.array_equal(np.asarray(Xi), G[f"tape_{seed}_{block}_{D}_{T}_Xi"])
        assert np.array_equal(u, G[f"tape_{seed}_{block}_{D}_{T}_u"])
    assert np.array_equal(O.probe(3, 1, 2, 1, 300, 4), G["probe_3_1_2_1_300_4"])


def test_config1_fixture():
    D, T, N, eps = 2, 64, 500, 0.1
    tg = O.Target.diag_gauss(np.ones(D))
    x = np.zeros(D)
    vals, seqs, iters = [], [], []
    nsteps, b = 0, 0
    while nsteps < N:
        Xi, u = O.tape(0, b, D, T)
        S, acc, _ = O.mala_sequential(tg, eps, x, Xi, u)
        Sd, info = O.deer_solve(tg, eps, x, Xi, u, 0, b, tol_abs=1e-6, tol_rel=1e-5)
        nkeep = min(T, N - nsteps)
        vals.append(Sd[:, :nkeep])
        seqs.append(S[:, :nkeep])
        iters.append(info["iters"])
        x = Sd[:, nkeep - 1].copy()
        nsteps += nkeep
        b += 1
    np.testing.assert_allclose(np.concatenate(vals, axis=1), G["cfg1_deer_values"], rtol=1e-12,
                               atol=1e-12)
    np.testing.assert_allclose(np.concatenate(seqs, axis=1), G["cfg1_seq_values"], rtol=1e-13,
                               atol=1e-13)
    assert list(iters) == list(G["cfg1_deer_iters"])
    # DEER and the sequential chain agree to the solver tolerance
    assert np.max(np.abs(G["cfg1_deer_values"] - G["cfg1_seq_values"])) < 1e-3


def test_diag_and_dense_fixtures():
    tg = O.Target.diag_gauss(G["diag_lam"])
    Xi, u = O.tape(1, 0, 10, 96)
    S, acc, _ = O.mala_sequential(tg, 0.05, G["diag_x0"], Xi, u)
    np.testing.assert_allclose(S, G["diag_seq"], rtol=1e-13, atol=1e-13)
    assert np.array_equal(acc, G["diag_acc"])
    tg = O.Target.dense_gauss(G["dense_P"])
    Xi, u = O.tape(4, 2, 6, 64)
    S, acc, _ = O.mala_sequential(tg, 0.1, G["dense_x0"], Xi, u)
    np.testing.assert_allclose(S, G["dense_seq"], rtol=1e-13, atol=1e-13)
    assert np.array_equal(acc, G["dense_acc"])
    S, info = O.deer_solve(tg, 0.1, G["dense_x0"], Xi, u, 4, 2, jacobian="stoch_diag", probes=2,
                           damping=0.5, tol_abs=1e-10, tol_rel=1e-9, maxiter=400)
    np.testing.assert_allclose(S, G["dense_deer"], rtol=1e-12, atol=1e-12)
