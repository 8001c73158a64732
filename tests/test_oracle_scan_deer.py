"""Oracle pinning: DEERScan and DEER properties of test/test-DEERScan.jl,
test/test-Deer-vs-MALA.jl and test/test-Jacobian-Estimator.jl restated on the
FP64 CPU oracle (no GPU)."""
import numpy as np
import pytest

import np_oracle as NO
import oracle as O


def _affine(rng, D, T):
    # make_affine_problem (test-DEERScan.jl:25-35), stable branch
    A = 0.2 * (rng.random((D, T)) - 0.5)
    return A, rng.standard_normal((D, T)), rng.standard_normal(D)


@pytest.mark.parametrize("D,T", [(1, 1), (1, 2), (2, 3), (3, 4), (4, 5), (5, 17), (8, 31),
                                 (8, 64)])
def test_doubling_scan_matches_sequential(D, T):
    # test-DEERScan.jl:37-55
    A, B, s0 = _affine(np.random.default_rng(11 + D * T), D, T)
    S_ref = O.scan_seq(A, B, s0)
    S = O.scan_doubling(A, B, s0)
    np.testing.assert_allclose(S, S_ref, rtol=1e-12, atol=1e-12)
    np.testing.assert_allclose(S_ref, NO.scan_seq(A, B, s0), rtol=1e-14, atol=1e-14)


def test_scan_residual_helpers():
    # test-DEERScan.jl:57-96
    A, B, s0 = _affine(np.random.default_rng(12), 4, 9)
    S = O.scan_seq(A, B, s0)
    assert O.scan_residual(S, A, B, s0) <= 1e-12
    bad = S.copy()
    bad[1, 0] += 0.25
    assert abs(O.scan_residual(bad, A, B, s0) - 0.25) < 1e-12
    bad = S.copy()
    bad[2, 5] -= 0.5
    assert abs(O.scan_residual(bad, A, B, s0) - 0.5) < 1e-12
    Z = np.zeros((4, 0))
    assert O.scan_residual(Z, Z, Z, s0) == 0.0


def _stdnormal(D):
    return O.Target.diag_gauss(np.ones(D))


def test_rejections_occur():
    # test-Deer-vs-MALA.jl:50-69
    D, T, eps = 3, 32, 0.35
    Xi, u = O.tape(12345, 1, D, T)
    _, acc, _ = O.mala_sequential(_stdnormal(D), eps, np.ones(D), Xi, u)
    assert (~acc).sum() > 0


def test_deer_diag_recovers_sequential():
    # test-Deer-vs-MALA.jl:71-108
    D, T, eps = 3, 32, 0.05
    tg = _stdnormal(D)
    Xi, u = O.tape(12345, 1, D, T)
    x0 = np.random.default_rng(1).standard_normal(D)
    S_seq, _, _ = O.mala_sequential(tg, eps, x0, Xi, u)
    S, info = O.deer_solve(tg, eps, x0, Xi, u, 12345, 1, jacobian="diag", damping=0.5,
                           tol_abs=1e-10, tol_rel=1e-8, maxiter=200)
    assert info["converged"]
    for t in range(T):
        a, b = S[:, t], S_seq[:, t]
        assert np.linalg.norm(a - b) <= max(1e-8, 1e-6 * max(np.linalg.norm(a),
                                                                np.linalg.norm(b)))


def test_deer_stoch_diag_recovers_sequential_with_rejections():
    # test-Deer-vs-MALA.jl:161-215
    D, T, eps = 3, 32, 0.15
    tg = _stdnormal(D)
    for blk in range(20):
        Xi, u = O.tape(777, blk, D, T)
        x0 = np.random.default_rng(blk).standard_normal(D)
        S_seq, acc, _ = O.mala_sequential(tg, eps, x0, Xi, u)
        if (~acc).sum() > 0:
            break
    assert (~acc).sum() > 0
    S, info = O.deer_solve(tg, eps, x0, Xi, u, 42, blk, jacobian="stoch_diag", probes=2,
                           damping=0.5, tol_abs=1e-9, tol_rel=1e-7, maxiter=400)
    assert info["converged"]
    for t in range(T):
        a, b = S[:, t], S_seq[:, t]
        assert np.linalg.norm(a - b) <= max(1e-7, 1e-5 * max(np.linalg.norm(a),
                                                                np.linalg.norm(b)))


def test_recursion_defect():
    # test-Jacobian-Estimator.jl:187-232
    D, T, eps = 6, 80, 0.35
    tg = _stdnormal(D)
    Xi, u = O.tape(20251231, 0, D, T)
    x0 = np.random.default_rng(2).standard_normal(D)
    S, info = O.deer_solve(tg, eps, x0, Xi, u, 1, 0, jacobian="diag", damping=0.5,
                           tol_abs=1e-12, tol_rel=1e-10, maxiter=200)
    prev, md = x0, 0.0
    for t in range(T):
        nxt, _, _ = O.mala_step(tg, eps, prev, Xi[:, t], u[t])
        md = max(md, np.linalg.norm(S[:, t] - nxt))
        prev = S[:, t]
    assert info["converged"] and md <= 1e-9


@pytest.mark.parametrize("jac", ["stoch_diag", "diag", "full"])
def test_fixed_point_invariance(jac):
    """At the exact trajectory, one DEER update (damping 1) returns it unchanged."""
    rng = np.random.default_rng(8)
    D, T = 4, 20
    P = rng.standard_normal((D, D))
    P = P @ P.T / D + np.eye(D)
    tg = O.Target.dense_gauss(P)
    Xi, u = O.tape(4, 0, D, T)
    x0 = rng.standard_normal(D)
    S_seq, _, _ = O.mala_sequential(tg, 0.2, x0, Xi, u)
    S, _, _ = O.deer_update(tg, 0.2, x0, S_seq, Xi, u, 4, 0, 0, jacobian=jac, damping=1.0)
    np.testing.assert_allclose(S, S_seq, rtol=1e-12, atol=1e-12)


def test_update_scan_consistency():
    """S_out of one update equals solve_affine_seq(A, B, s0) (test-Jacobian-Estimator.jl:161-185)."""
    rng = np.random.default_rng(9)
    D, T = 7, 13
    tg = _stdnormal(D)
    Xi, u = O.tape(9, 0, D, T)
    s0, S_in = rng.standard_normal(D), rng.standard_normal((D, T))
    S, A, B = O.deer_update(tg, 0.2, s0, S_in, Xi, u, 9, 0, 0, damping=1.0)
    np.testing.assert_allclose(S, O.scan_seq(A, B, s0), rtol=1e-12, atol=1e-12)


def test_hutchinson_converges_to_exact_diag():
    # test-Jacobian-Estimator.jl:74-106 and test-Deer-vs-MALA.jl:205-214
    rng = np.random.default_rng(10)
    D, T = 6, 4
    P = rng.standard_normal((D, D))
    P = 0.3 * P @ P.T / D + np.eye(D)
    tg = O.Target.dense_gauss(P)
    Xi, u = O.tape(10, 0, D, T)
    x = rng.standard_normal(D)
    _, J = O.jac_full(tg, 0.3, x, Xi[:, 0], u[0])
    exact = np.diag(J)

    def est(K, rep):
        acc = np.zeros(D)
        for k in range(K):
            z = O.probe(1000 + rep, 0, 0, k, D, 1)[:, 0]
            _, jv = O.fwd_and_jvp(tg, 0.3, x, Xi[:, 0], u[0], z)
            acc += z * jv
        return acc / K

    mse = {K: np.mean([np.mean((est(K, r) - exact) ** 2) for r in range(25)])
           for K in (1, 8, 64)}
    assert mse[8] < mse[1] and mse[64] < mse[8]
    np.testing.assert_allclose(est(200, 0), exact, rtol=0.15, atol=0.15)


def test_full_and_window_reach_same_fixed_point():
    rng = np.random.default_rng(11)
    D, T = 5, 96
    P = rng.standard_normal((D, D))
    P = P @ P.T / D + np.eye(D)
    tg = O.Target.dense_gauss(P)
    Xi, u = O.tape(11, 0, D, T)
    x0 = rng.standard_normal(D)
    S_seq, _, _ = O.mala_sequential(tg, 0.1, x0, Xi, u)
    kw = dict(tol_abs=1e-11, tol_rel=1e-10, maxiter=500, damping=1.0)
    S_d, i_d = O.deer_solve(tg, 0.1, x0, Xi, u, 3, 0, jacobian="diag", **kw)
    S_f, i_f = O.deer_solve(tg, 0.1, x0, Xi, u, 3, 0, jacobian="full", **kw)
    S_w, i_w = O.deer_solve(tg, 0.1, x0, Xi, u, 3, 0, jacobian="diag", window=16, **kw)
    for S, inf in ((S_d, i_d), (S_f, i_f), (S_w, i_w)):
        assert inf["converged"]
        np.testing.assert_allclose(S, S_seq, rtol=1e-8, atol=1e-9)
    assert i_f["iters"] <= i_d["iters"]


def test_logistic_deer_matches_sequential():
    rng = np.random.default_rng(12)
    N, D, T = 80, 4, 48
    X = rng.standard_normal((N, D)) / np.sqrt(D)
    th = rng.standard_normal(D)
    y = (rng.random(N) < 1 / (1 + np.exp(-X @ th))).astype(float)
    tg = O.Target.logistic(X, y)
    Xi, u = O.tape(2, 0, D, T)
    x0 = np.zeros(D)
    S_seq, _, _ = O.mala_sequential(tg, 0.05, x0, Xi, u)
    S, info = O.deer_solve(tg, 0.05, x0, Xi, u, 2, 0, tol_abs=1e-10, tol_rel=1e-9,
                           maxiter=300)
    assert info["converged"]
    np.testing.assert_allclose(S, S_seq, rtol=1e-7, atol=1e-8)


def test_argument_validation():
    # test-Jacobian-Estimator.jl:124-159
    D, T = 3, 4
    tg = _stdnormal(D)
    Xi, u = O.tape(1, 0, D, T)
    s0 = np.zeros(D)
    S = np.zeros((D, T))
    with pytest.raises(ValueError):
        O.deer_update(tg, 0.1, s0, S, Xi, u, 1, 0, 0, damping=0.0)
    with pytest.raises(ValueError):
        O.deer_update(tg, 0.1, s0, S, Xi, u, 1, 0, 0, probes=0)
    with pytest.raises(ValueError):
        O.deer_solve(tg, 0.1, s0, Xi, u, 1, 0, maxiter=0)
    with pytest.raises(ValueError):
        O.deer_solve(tg, 0.1, s0, Xi, u, 1, 0, tol_abs=-1.0)
    with pytest.raises(ValueError):
        O.deer_solve(tg, 0.1, s0, Xi, u, 1, 0, tol_rel=-1.0)
