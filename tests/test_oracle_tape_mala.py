"""Oracle pinning: tape generator known answers and the MALA kernel properties of
test/test-MALA-Kernel.jl, restated on the FP64 CPU oracle (no GPU)."""
import numpy as np
import pytest

import np_oracle as NO
import oracle as O


# Published Philox4x32-10 known-answer vectors (Random123 kat_vectors).
KAT = [
    ([0, 0, 0, 0], [0, 0], [0x6627E8D5, 0xE169C58D, 0xBC57AC4C, 0x9B00DBD8]),
    ([0xFFFFFFFF] * 4, [0xFFFFFFFF] * 2, [0x408F276D, 0x41C83B0E, 0xA20BC7C6, 0x6D5451FD]),
    ([0x243F6A88, 0x85A308D3, 0x13198A2E, 0x03707344], [0xA4093822, 0x299F31D0],
     [0xD16CFE09, 0x94FDCCEB, 0x5001E420, 0x24126EA1]),
]


@pytest.mark.parametrize("ctr,key,want", KAT)
def test_philox_known_answers(ctr, key, want):
    assert O.philox(ctr, key) == want


def test_tape_deterministic_and_block_distinct():
    a, ua = O.tape(11, 2, 7, 33)
    b, ub = O.tape(11, 2, 7, 33)
    c, uc = O.tape(11, 3, 7, 33)
    assert np.array_equal(a, b) and np.array_equal(ua, ub)
    assert not np.array_equal(a, c)
    # a prefix of a longer tape is the shorter tape (counter-based, column-addressed)
    d, ud = O.tape(11, 2, 7, 50)
    assert np.array_equal(d[:, :33], a) and np.array_equal(ud[:33], ua)


def test_tape_distribution():
    Xi, u = O.tape(5, 0, 8, 40000)
    x = Xi.astype(np.float64).ravel()
    assert abs(x.mean()) < 0.01 and abs(x.var() - 1) < 0.01
    assert abs(((x - x.mean()) ** 4).mean() / x.var() ** 2 - 3) < 0.05
    assert u.min() > 0 and u.max() < 1 and abs(u.mean() - 0.5) < 0.01


def test_probe_rademacher():
    Z = O.probe(1, 0, 3, 1, 300, 50)
    assert set(np.unique(Z)) == {-1.0, 1.0}
    assert abs(Z.mean()) < 0.02
    assert not np.array_equal(Z, O.probe(1, 0, 4, 1, 300, 50))


def _std_normal(D):
    return O.Target.diag_gauss(np.ones(D)), NO.NPTarget("diag", prec=np.ones(D))


def test_determinism_with_fixed_tape():
    # test-MALA-Kernel.jl:46-80
    D, T, eps = 7, 250, 0.35
    tg, _ = _std_normal(D)
    Xi, u = O.tape(20251231, 0, D, T)
    x0 = np.random.default_rng(0).standard_normal(D)
    S1, a1, _ = O.mala_sequential(tg, eps, x0, Xi, u)
    S2, a2, _ = O.mala_sequential(tg, eps, x0, Xi, u)
    assert np.array_equal(S1, S2) and np.array_equal(a1, a2)


def test_stationary_moments():
    # test-MALA-Kernel.jl:82-113
    D, T, burn, eps = 3, 25000, 5000, 0.30
    tg, _ = _std_normal(D)
    Xi, u = O.tape(20251231, 1, D, T)
    S, _, _ = O.mala_sequential(tg, eps, np.zeros(D), Xi, u)
    X = S[:, burn:]
    mu = X.mean(axis=1)
    cov = np.cov(X)
    assert np.max(np.abs(mu)) < 0.08
    assert np.max(np.abs(np.diag(cov) - 1)) < 0.12
    assert np.max(np.abs(cov - np.diag(np.diag(cov)))) < 0.10


def test_forced_accept_and_reject():
    # test-MALA-Kernel.jl:115-167
    rng = np.random.default_rng(3)
    D, eps = 5, 0.45
    tg, nt = _std_normal(D)
    x = rng.standard_normal(D)
    for _ in range(2000):
        xi = rng.standard_normal(D)
        _, _, la = O.mala_step(tg, eps, x, xi, 0.5)
        if la < -1e-8:
            break
    assert la < -1e-8
    tau = np.exp(la)
    y = x + eps * O.grad(tg, x) + np.sqrt(2 * eps) * xi
    xa, acc, _ = O.mala_step(tg, eps, x, xi, tau / 2)
    xr, rej, _ = O.mala_step(tg, eps, x, xi, (tau + 1) / 2)
    assert acc and np.array_equal(xa, y)
    assert (not rej) and np.array_equal(xr, x)


def test_logalpha_vs_independent_formula():
    # test-MALA-Kernel.jl:169-197
    rng = np.random.default_rng(4)
    D, eps = 6, 0.40
    tg, nt = _std_normal(D)
    x, xi = rng.standard_normal(D), rng.standard_normal(D)
    _, _, la = O.mala_step(tg, eps, x, xi, 0.5)
    y = x + eps * (-x) + np.sqrt(2 * eps) * xi

    def lq(a, b, gb):
        r = a - (b + eps * gb)
        return -0.5 * r @ r / (2 * eps) - D / 2 * np.log(4 * np.pi * eps)

    ref = (-0.5 * y @ y + lq(x, y, -y)) - (-0.5 * x @ x + lq(y, x, -x))
    assert abs(la - ref) <= 1e-10 + 1e-10 * abs(ref)


def _targets(rng, D):
    lam = 10 ** rng.uniform(-1, 1, D)
    P = rng.standard_normal((D, D))
    P = P @ P.T / D + np.eye(D)
    N = 60
    X = rng.standard_normal((N, D)) / np.sqrt(D)
    y = (rng.random(N) < 0.5).astype(float)
    return [
        (O.Target.diag_gauss(lam), NO.NPTarget("diag", prec=lam), 0.3),
        (O.Target.dense_gauss(P), NO.NPTarget("dense", prec=P), 0.2),
        (O.Target.logistic(X, y), NO.NPTarget("logistic", X=X, y=y), 0.1),
    ]


def test_oracle_matches_numpy_restatement():
    rng = np.random.default_rng(5)
    D, T = 5, 40
    Xi, u = O.tape(3, 0, D, T)
    x0 = rng.standard_normal(D)
    v = rng.standard_normal(D)
    for tg, nt, eps in _targets(rng, D):
        S, acc, _ = O.mala_sequential(tg, eps, x0, Xi, u)
        S2, acc2 = NO.mala_sequential(nt, eps, x0, Xi, u)
        assert np.array_equal(acc, acc2)
        assert np.max(np.abs(S - S2)) < 1e-12
        f, jv = O.fwd_and_jvp(tg, eps, x0, Xi[:, 0], u[0], v)
        f2, jv2 = NO.fwd_and_jvp(nt, eps, x0, Xi[:, 0].astype(float), float(u[0]), v)
        assert np.max(np.abs(jv - jv2)) < 1e-12 and np.max(np.abs(f - f2)) < 1e-14


def test_full_jacobian_matches_jvp_and_batched():
    rng = np.random.default_rng(6)
    D, T = 5, 12
    Xi, u = O.tape(9, 0, D, T)
    X = rng.standard_normal((D, T))
    Z = O.probe(9, 0, 0, 0, D, T)
    for tg, nt, eps in _targets(rng, D):
        FT, Jt = O.fwd_and_jvp_batched(tg, eps, X, Xi, u, Z)
        for t in range(T):
            f, J = O.jac_full(tg, eps, X[:, t], Xi[:, t], u[t])
            f2, jv = O.fwd_and_jvp(tg, eps, X[:, t], Xi[:, t], u[t], Z[:, t])
            assert np.max(np.abs(J @ Z[:, t] - jv)) < 1e-12
            assert np.max(np.abs(Jt[:, t] - jv)) < 1e-12 and np.array_equal(FT[:, t], f)


# mass matrix of test-MALA-Kernel.jl:199-204 (D = 3, eps = 0.08, standard normal target)
M_REF = np.array([[1.7, 0.2, -0.1], [0.2, 1.3, 0.15], [-0.1, 0.15, 1.5]])


def test_mass_step_matches_reference_formulas():
    # test-MALA-Kernel.jl:199-217: y = x + eps L L^T g + sqrt(2 eps) L xi, and log q with
    # M^-1 and log det M (test-MALA-Kernel.jl:26-36)
    rng = np.random.default_rng(20260201)
    D, eps = 3, 0.08
    Lf = np.linalg.cholesky(M_REF)
    tg, _ = _std_normal(D)
    x, xi = rng.standard_normal(D), rng.standard_normal(D)
    S, acc, la = O.mala_sequential_mass(tg, eps, Lf, x, xi[:, None], np.array([1e-300]))
    y = x + eps * (Lf @ (Lf.T @ -x)) + np.sqrt(2 * eps) * (Lf @ xi)
    assert acc[0] and np.max(np.abs(S[:, 0] - y)) < 1e-12

    def lq(a, b, gb):
        r = a - b - eps * (M_REF @ gb)
        return (-0.5 * r @ np.linalg.solve(M_REF, r) / (2 * eps) - D / 2 * np.log(4 * np.pi * eps)
                - 0.5 * np.linalg.slogdet(M_REF)[1])

    ref = (-0.5 * y @ y + lq(x, y, -y)) - (-0.5 * x @ x + lq(y, x, -x))
    assert abs(la[0] - ref) <= 1e-10 + 1e-10 * abs(ref)


def test_mass_chain_is_the_whitened_chain():
    # the identity the device solve is built on: MALA with mass M = L L^T from x0 is
    # L times plain MALA on the whitened target (precision L^T P L, mean L^-1 mu) from
    # L^-1 x0, on the same tape, with the same log alpha
    rng = np.random.default_rng(8)
    D, T, eps = 6, 200, 0.25
    A = rng.standard_normal((D, D))
    P = A @ A.T / D + np.eye(D)
    mu = rng.standard_normal(D)
    B = rng.standard_normal((D, D))
    # eps * lambda_max(L^T P L) = 0.6: a stable chain, so roundoff does not grow
    Lf = np.linalg.cholesky(0.25 * (B @ B.T / D + 0.5 * np.eye(D)))
    Xi, u = O.tape(5, 0, D, T)
    x0 = rng.standard_normal(D)
    S, acc, la = O.mala_sequential_mass(O.Target.dense_gauss(P, mu), eps, Lf, x0, Xi, u)
    Pw = Lf.T @ P @ Lf
    tw = O.Target.dense_gauss(0.5 * (Pw + Pw.T), np.linalg.solve(Lf, mu))
    Sw, accw, law = O.mala_sequential(tw, eps, np.linalg.solve(Lf, x0), Xi, u)
    assert 0 < (~acc).sum() < T and np.array_equal(acc, accw)
    assert np.max(np.abs(S - Lf @ Sw)) < 1e-11
    assert np.max(np.abs(la - law)) < 1e-10
    # identity factor: the plain chain, bit for bit
    S1, acc1, la1 = O.mala_sequential_mass(O.Target.dense_gauss(P, mu), eps, np.eye(D), x0, Xi, u)
    S0, acc0, la0 = O.mala_sequential(O.Target.dense_gauss(P, mu), eps, x0, Xi, u)
    assert np.array_equal(acc1, acc0) and np.max(np.abs(S1 - S0)) < 1e-14
