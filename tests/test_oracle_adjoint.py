"""The FP64 adjoint restatement (oracle/np_oracle.gauss_adjoint) against
central finite differences of the sequential trace, with the accept flags
asserted identical at +-h (no accept flips inside the difference)."""
import numpy as np
import pytest

import np_oracle as NP
import oracle as O


def _problem(D=8, T=96, seed=5, eps=0.05):
    rng = np.random.default_rng(seed)
    s = 10.0 ** rng.uniform(-1.0, 1.0, D)
    Z = rng.standard_normal((D, D))
    Q, R = np.linalg.qr(Z)
    Q = Q * np.sign(np.diag(R))
    P = (Q / s) @ Q.T
    P = 0.5 * (P + P.T)
    x0 = rng.standard_normal(D)
    Xi, u = O.tape(11, 2, D, T)
    return P, Q, s, x0, Xi, u, eps


@pytest.mark.parametrize("objective", ["esjd", "mean_sq"])
def test_adjoint_d_eps_matches_fd(objective):
    P, Q, s, x0, Xi, u, eps = _problem()
    esjd, msq, S, acc = NP.gauss_objectives(P, None, eps, x0, Xi, u)
    assert 0 < acc.sum() < acc.size  # both branches exercised
    g, _ = NP.gauss_adjoint(P, None, eps, x0, Xi, u, S, objective)
    h = 1e-6 * eps
    ep = NP.gauss_objectives(P, None, eps + h, x0, Xi, u)
    em = NP.gauss_objectives(P, None, eps - h, x0, Xi, u)
    assert np.array_equal(ep[3], acc) and np.array_equal(em[3], acc)
    k = 0 if objective == "esjd" else 1
    fd = (ep[k] - em[k]) / (2 * h)
    assert abs(g - fd) <= 1e-5 * max(1.0, abs(fd)), (g, fd)


def test_adjoint_d_log_s_matches_fd():
    P, Q, s, x0, Xi, u, eps = _problem(D=6, T=80, seed=9)
    esjd, msq, S, acc = NP.gauss_objectives(P, None, eps, x0, Xi, u)
    _, gls = NP.gauss_adjoint(P, None, eps, x0, Xi, u, S, "mean_sq", Q=Q, s=s)
    h = 1e-6
    for i in range(s.size):
        vals = []
        for sgn in (1, -1):
            s2 = s.copy()
            s2[i] *= np.exp(sgn * h)
            P2 = (Q / s2) @ Q.T
            r = NP.gauss_objectives(0.5 * (P2 + P2.T), None, eps, x0, Xi, u)
            assert np.array_equal(r[3], acc)
            vals.append(r[1])
        fd = (vals[0] - vals[1]) / (2 * h)
        assert abs(gls[i] - fd) <= 1e-5 * max(1.0, abs(fd)), (i, gls[i], fd)


def test_objective_trace_matches_c_oracle():
    P, Q, s, x0, Xi, u, eps = _problem()
    _, _, S, acc = NP.gauss_objectives(P, None, eps, x0, Xi, u)
    S2, acc2, _ = O.mala_sequential(O.Target.dense_gauss(P), eps, x0, Xi, u)
    assert np.array_equal(acc, acc2.astype(bool))
    np.testing.assert_allclose(S, S2, rtol=1e-12, atol=1e-12)


@pytest.mark.parametrize("objective", ["esjd", "mean_sq"])
def test_logistic_adjoint_matches_fd(objective):
    # the logistic restatement against central differences of the sequential trace's
    # objective that flip no accept decision
    import np_oracle as NO
    rng = np.random.default_rng(12)
    N, D, T, eps = 60, 4, 80, 0.05
    X = rng.standard_normal((N, D)) / np.sqrt(D)
    y = (rng.random(N) < 1 / (1 + np.exp(-X @ rng.standard_normal(D)))).astype(float)
    Xi, u = O.tape(3, 0, D, T)
    x0 = rng.standard_normal(D) * 0.3
    e0, m0, S, acc = NO.logistic_objectives(X, y, eps, x0, Xi, u)
    assert 0 < (~acc).sum() < T
    g = NO.logistic_adjoint(X, y, eps, x0, Xi, u, S, objective)
    h = 1e-6 * eps
    ep, mp, _, ap = NO.logistic_objectives(X, y, eps + h, x0, Xi, u)
    em, mm, _, am = NO.logistic_objectives(X, y, eps - h, x0, Xi, u)
    assert np.array_equal(ap, acc) and np.array_equal(am, acc)
    fd = ((ep - em) if objective == "esjd" else (mp - mm)) / (2 * h)
    assert abs(g - fd) <= 1e-5 * abs(fd) + 1e-9
