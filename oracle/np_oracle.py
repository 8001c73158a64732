"""NumPy FP64 restatement of the reference's MALA/DEER formulas (TEST INFRASTRUCTURE ONLY).

An independent second restatement used to cross-check the C oracle on small
cases.  Each function cites the reference file:line it follows.  Arrays use the
(D, T) convention of oracle.py.
"""
from __future__ import annotations

import numpy as np


def _softplus(z):
    return np.maximum(z, 0.0) + np.log1p(np.exp(-np.abs(z)))


class NPTarget:
    """kind in {'diag', 'dense', 'logistic'} with logp/grad/hvp closures."""

    def __init__(self, kind, prec=None, mean=None, X=None, y=None, prior_prec=1.0):
        self.kind = kind
        if kind == "diag":
            lam = np.asarray(prec, float)
            m = np.zeros_like(lam) if mean is None else np.asarray(mean, float)
            self.D = lam.size
            self.logp = lambda x: -0.5 * np.sum(lam * (x - m) ** 2)
            self.grad = lambda x: -lam * (x - m)
            self.hvp = lambda x, v: -lam * v
        elif kind == "dense":
            P = np.asarray(prec, float)
            m = np.zeros(P.shape[0]) if mean is None else np.asarray(mean, float)
            self.D = P.shape[0]
            self.logp = lambda x: -0.5 * (x - m) @ P @ (x - m)
            self.grad = lambda x: -P @ (x - m)
            self.hvp = lambda x, v: -P @ v
        else:
            Xm = np.asarray(X, float)
            yv = np.asarray(y, float)
            tau = float(prior_prec)
            self.D = Xm.shape[1]
            # bayes_logreg.jl:37-58, 76-83
            self.logp = lambda b: float(np.sum(yv * -_softplus(-(Xm @ b)) +
                                               (1 - yv) * -_softplus(Xm @ b))
                                        - 0.5 * tau * b @ b)
            self.grad = lambda b: Xm.T @ (yv - 1 / (1 + np.exp(-(Xm @ b)))) - tau * b

            def hvp(b, v):
                p = 1 / (1 + np.exp(-(Xm @ b)))
                return -Xm.T @ (p * (1 - p) * (Xm @ v)) - tau * v

            self.hvp = hvp


def logq(tg, y, x, gx, eps):
    """logq_mala! (MALA.jl:172-193), identity mass matrix."""
    r = y - (x + eps * gx)
    return -0.5 * (r @ r) / (2 * eps) - (x.size / 2) * np.log(4 * np.pi * eps)


def mala_step(tg, eps, x, xi, u):
    """mala_step_with_logalpha! (MALA.jl:377-411)."""
    gx = tg.grad(x)
    y = x + eps * gx + np.sqrt(2 * eps) * xi
    gy = tg.grad(y)
    la = (tg.logp(y) + logq(tg, x, y, gy, eps)) - (tg.logp(x) + logq(tg, y, x, gx, eps))
    acc = np.log(u) < la
    return (y.copy() if acc else x.copy()), bool(acc), la


def mala_sequential(tg, eps, x0, Xi, u):
    """run_mala_sequential_taped (MALA.jl:322-346); S[:, t] = x_{t+1}."""
    D, T = Xi.shape
    S = np.empty((D, T))
    acc = np.zeros(T, bool)
    x = np.asarray(x0, float)
    for t in range(T):
        x, acc[t], _ = mala_step(tg, eps, x, Xi[:, t].astype(float), float(u[t]))
        S[:, t] = x
    return S, acc


def fwd_and_jvp(tg, eps, x, xi, u, v):
    """mala_step_taped_and_jvp! (MALA.jl:732-797)."""
    gx = tg.grad(x)
    y = x + eps * gx + np.sqrt(2 * eps) * xi
    gy = tg.grad(y)
    la = (tg.logp(y) + logq(tg, x, y, gy, eps)) - (tg.logp(x) + logq(tg, y, x, gx, eps))
    g = 1 / (1 + np.exp(-(la - np.log(u))))
    a = 1.0 if np.log(u) < la else 0.0
    w = v + eps * tg.hvp(x, v)
    r = x - y - eps * gy
    dr = v - w - eps * tg.hvp(y, w)
    dla = np.sum(gy * w - gx * v - (1 / (2 * eps)) * r * dr)
    dg = g * (1 - g) * dla
    return (y if a else x), a * w + (y - x) * dg + (1 - a) * v


def scan_seq(A, B, s0):
    """solve_affine_seq! (DEERScan.jl:51-68)."""
    D, T = A.shape
    S = np.empty((D, T))
    s = np.asarray(s0, float)
    for t in range(T):
        s = A[:, t] * s + B[:, t]
        S[:, t] = s
    return S


def deer_update(tg, eps, s0, S_in, Xi, u, Zs, jacobian="stoch_diag", damping=0.5):
    """deer_update! (DEER.jl:375-475) with explicit probes Zs (list of (D,T))."""
    D, T = S_in.shape
    Xbar = np.concatenate([np.asarray(s0, float)[:, None], S_in[:, :T - 1]], axis=1)
    A = np.zeros((D, T))
    B = np.zeros((D, T))
    for t in range(T):
        xb = Xbar[:, t]
        xi = Xi[:, t].astype(float)
        if jacobian == "stoch_diag":
            acc = np.zeros(D)
            for Z in Zs:
                ft, jv = fwd_and_jvp(tg, eps, xb, xi, float(u[t]), Z[:, t])
                acc += Z[:, t] * jv
            jt = acc / len(Zs)
        else:
            ft, _, _ = mala_step(tg, eps, xb, xi, float(u[t]))
            jt = np.array([fwd_and_jvp(tg, eps, xb, xi, float(u[t]), e)[1][i]
                           for i, e in enumerate(np.eye(D))])
        A[:, t] = jt
        B[:, t] = ft - jt * xb
    S = scan_seq(A, B, s0)
    if damping != 1.0:
        S = (1 - damping) * S_in + damping * S
    return S, A, B


# ---------------------------------------------------------------------------
# Objectives of a Gaussian trace and their adjoint (no counterpart in the
# reference; the checks of the device adjoint).  Target N(mean, P^-1).
# ---------------------------------------------------------------------------

def gauss_objectives(P, mean, eps, x0, Xi, u):
    """Sequential FP64 trace (mala_step above) and the two objectives
    esjd = (1/T) sum_t min(1, alpha_t) |y_t - x_{t-1}|^2 and
    msq  = (1/T) sum_t |x_t|^2.  Returns (esjd, msq, S, acc)."""
    P = np.asarray(P, float)
    tg = NPTarget("dense", P, mean)
    D, T = Xi.shape
    S = np.empty((D, T))
    acc = np.zeros(T, bool)
    x = np.asarray(x0, float)
    esjd = 0.0
    for t in range(T):
        xi = Xi[:, t].astype(float)
        gx = tg.grad(x)
        y = x + eps * gx + np.sqrt(2 * eps) * xi
        xn, acc[t], la = mala_step(tg, eps, x, xi, float(u[t]))
        esjd += min(1.0, np.exp(la)) * float((y - x) @ (y - x))
        x = xn
        S[:, t] = x
    return esjd / T, float(np.sum(S * S)) / T, S, acc


def gauss_adjoint(P, mean, eps, x0, Xi, u, S, objective, Q=None, s=None):
    """Adjoint of an objective at the trajectory S with its accept flags held
    fixed: lambda_t = dL/dx_t + C_{t+1}^T lambda_{t+1}, C = I - eps P (accepted)
    or I.  Returns (dL/deps, dL/dlog s or None) with P = Q diag(1/s) Q^T."""
    P = np.asarray(P, float)
    D, T = S.shape
    m = np.zeros(D) if mean is None else np.asarray(mean, float)
    tg = NPTarget("dense", P, m)
    M = np.eye(D) - eps * P
    c = np.zeros((D, T))
    acc = np.zeros(T, bool)
    direct = 0.0
    gxs = np.zeros((D, T))
    for t in range(T):
        xb = np.asarray(x0, float) if t == 0 else S[:, t - 1]
        xi = Xi[:, t].astype(float)
        gx = tg.grad(xb)
        y = xb + eps * gx + np.sqrt(2 * eps) * xi
        gy = tg.grad(y)
        la = (tg.logp(y) + logq(tg, xb, y, gy, eps)) - (tg.logp(xb) + logq(tg, y, xb, gx, eps))
        acc[t] = np.log(u[t]) < la
        gxs[:, t] = gx
        if objective == "mean_sq":
            c[:, t] += 2.0 * S[:, t] / T
            continue
        alpha = min(1.0, np.exp(la))
        dalpha = alpha if la < 0 else 0.0
        e2 = float((y - xb) @ (y - xb))
        dy = gx + xi / np.sqrt(2 * eps)
        q = xb - y - eps * gy
        dq = -(M @ dy) - gy
        dla = gy @ dy - q @ dq / (2 * eps) + (q @ q) / (4 * eps ** 2)
        direct += (dalpha * dla * e2 + alpha * 2.0 * ((y - xb) @ dy)) / T
        if t >= 1:
            v = M @ gy - gx - P @ q + 0.5 * eps * P @ (P @ q)
            c[:, t - 1] += (dalpha * e2 * v + alpha * 2.0 * eps * (-P @ (y - xb))) / T
    lam = np.zeros((D, T))
    lam[:, T - 1] = c[:, T - 1]
    for t in range(T - 2, -1, -1):
        lam[:, t] = c[:, t] + ((M @ lam[:, t + 1]) if acc[t + 1] else lam[:, t + 1])
    geps = direct
    gls = np.zeros(D) if (Q is not None and objective == "mean_sq") else None
    for t in range(T):
        if not acc[t]:
            continue
        xb = np.asarray(x0, float) if t == 0 else S[:, t - 1]
        geps += lam[:, t] @ (gxs[:, t] + Xi[:, t].astype(float) / np.sqrt(2 * eps))
        if gls is not None:
            gls += eps / np.asarray(s) * (Q.T @ lam[:, t]) * (Q.T @ (xb - m))
    return geps, gls


# --------------------------------------------------------------------------- batched CPU DEER
def logistic_batched_model(X, y, tau=1.0):
    """The batched model functions of bayes_logreg.jl:91-206 (make_problem_batched
    and make_problem_batched_with_hvp): every call is GEMM -> elementwise -> GEMM
    through BLAS, as the reference's batched DEER branch calls them.  The softplus
    is the stable form of docs/src/15-gpu.md:91-97."""
    X = np.ascontiguousarray(X, np.float64)
    yc = np.asarray(y, np.float64)[:, None]

    def logp_batch(B):  # bayes_logreg.jl:119-138
        L = X @ B
        res = yc * -_softplus(-L) + (1 - yc) * -_softplus(L)
        return res.sum(axis=0) - 0.5 * tau * (B * B).sum(axis=0)

    def grad_batch(B):  # :140-155
        L = X @ B
        return X.T @ (yc - 1.0 / (1.0 + np.exp(-L))) - tau * B

    def hvp_batch(B, V):  # :182-203
        P = 1.0 / (1.0 + np.exp(-(X @ B)))
        return -(X.T @ ((P * (1 - P)) * (X @ V))) - tau * V

    return logp_batch, grad_batch, hvp_batch


def fwd_and_jvp_batched(model, eps, Xb, Xi, u, Z):
    """mala_step_batched_fwd_and_jvp! (MALA.jl:556-628), identity mass matrix:
    gradlogp(X), logp(X), logp(Y), gradlogp(Y), hvp(X, Z), hvp(Y, W) -- twelve
    GEMMs for the logistic model -- then the column reductions."""
    logp_b, grad_b, hvp_b = model
    D = Xb.shape[0]
    c = np.sqrt(2 * eps)
    GX = grad_b(Xb)
    Y = Xb + eps * GX + c * Xi
    lpX, lpY = logp_b(Xb), logp_b(Y)
    GY = grad_b(Y)
    k = (D / 2) * np.log(4 * np.pi * eps)
    lq_yx = -0.5 * np.sum((Y - (Xb + eps * GX)) ** 2, axis=0) / (2 * eps) - k
    lq_xy = -0.5 * np.sum((Xb - (Y + eps * GY)) ** 2, axis=0) / (2 * eps) - k
    la = (lpY + lq_xy) - (lpX + lq_yx)
    logu = np.log(u)
    g = 1.0 / (1.0 + np.exp(-(la - logu)))
    acc = logu < la
    FT = np.where(acc[None, :], Y, Xb)
    W = Z + eps * hvp_b(Xb, Z)
    HvY = hvp_b(Y, W)
    R = Xb - Y - eps * GY
    dR = Z - W - eps * HvY
    dla = np.sum(GY * W, axis=0) - np.sum(GX * Z, axis=0) - (1 / (2 * eps)) * np.sum(R * dR, axis=0)
    dg = g * (1 - g) * dla
    Jt = np.where(acc[None, :], W, Z) + (Y - Xb) * dg[None, :]
    return FT, Jt


def scan_doubling(A, B, s0):
    """solve_affine_scan_diag! (DEERScan.jl:102-173): Hillis-Steele doubling over
    the maps (a, b), then s_t = a_t s0 + b_t."""
    a, b = A.copy(), B.copy()
    T = a.shape[1]
    off = 1
    while off < T:
        an, bn = a.copy(), b.copy()
        an[:, off:] = a[:, off:] * a[:, :-off]
        bn[:, off:] = a[:, off:] * b[:, :-off] + b[:, off:]
        a, b = an, bn
        off <<= 1
    return a * np.asarray(s0, float)[:, None] + b


def deer_solve_batched(model, eps, s0, Xi, u, probe, *, tol_abs=1e-6, tol_rel=1e-5, maxiter=200,
                       damping=0.5, chunk=4096):
    """DEER.solve (DEER.jl:506-595) on the batched :stoch_diag branch with one
    probe (DEER.jl:398-419): per sweep x_bar = [s0, S[:, :T-1]], Z = probe(iter),
    (FT, Jt) from fwd_and_jvp_batched over column chunks, A = Z .* Jt,
    B = FT - A .* x_bar, the doubling scan, damping, and the stopping rule
    max|dS| <= tol_abs + tol_rel max|S| (:567-578).  Returns (S, info)."""
    D, T = Xi.shape
    s0 = np.asarray(s0, np.float64)
    S = np.repeat(s0[:, None], T, axis=1)
    Xi = np.asarray(Xi, np.float64)
    u = np.asarray(u, np.float64)
    metric, it = np.inf, 0
    for it in range(1, maxiter + 1):
        Xbar = np.concatenate([s0[:, None], S[:, :T - 1]], axis=1)
        Z = probe(it - 1)
        A = np.empty((D, T))
        Bm = np.empty((D, T))
        for c0 in range(0, T, chunk):
            c1 = min(T, c0 + chunk)
            FT, Jt = fwd_and_jvp_batched(model, eps, Xbar[:, c0:c1], Xi[:, c0:c1], u[c0:c1],
                                         Z[:, c0:c1])
            A[:, c0:c1] = Z[:, c0:c1] * Jt
            Bm[:, c0:c1] = FT - A[:, c0:c1] * Xbar[:, c0:c1]
        Sn = scan_doubling(A, Bm, s0)
        if damping != 1.0:
            Sn = (1 - damping) * S + damping * Sn
        metric = np.max(np.abs(Sn - S)) / (tol_abs + tol_rel * np.max(np.abs(Sn)))
        S = Sn
        if not np.all(np.isfinite(S)):
            return S, {"iters": it, "converged": False, "metric": float("nan")}
        if metric <= 1:
            return S, {"iters": it, "converged": True, "metric": float(metric)}
    return S, {"iters": it, "converged": False, "metric": float(metric)}


# ---------------------------------------------------------------------------
# Objectives of a logistic-regression trace and their adjoint (no counterpart
# in the reference; the checks of the device adjoint).  The same recursion as
# gauss_adjoint with the state-dependent Jacobian J_t = I + eps H(x_{t-1}) of an
# accepted step, H the dense Hessian of bayes_logreg.jl:30-86 (prior N(0, I/tau)).
# ---------------------------------------------------------------------------

def logistic_parts(X, y, tau=1.0):
    """(logp, grad, hess) of the logistic target, dense, FP64."""
    X = np.asarray(X, np.float64)
    y = np.asarray(y, np.float64)

    def logp(th):
        L = X @ th
        return float(np.sum(y * L - _softplus(L)) - 0.5 * tau * th @ th)

    def grad(th):
        return X.T @ (y - 1.0 / (1.0 + np.exp(-(X @ th)))) - tau * th

    def hess(th):
        p = 1.0 / (1.0 + np.exp(-(X @ th)))
        return -(X.T * (p * (1 - p))) @ X - tau * np.eye(X.shape[1])

    return logp, grad, hess


def logistic_objectives(X, y, eps, x0, Xi, u, tau=1.0):
    """Sequential FP64 trace of the logistic target and its two objectives
    esjd = (1/T) sum_t min(1, alpha_t) |y_t - x_{t-1}|^2 and msq = (1/T) sum_t
    |x_t|^2.  Returns (esjd, msq, S, acc)."""
    logp, grad, _ = logistic_parts(X, y, tau)
    D, T = Xi.shape
    S = np.empty((D, T))
    acc = np.zeros(T, bool)
    x = np.asarray(x0, np.float64)
    esjd = 0.0
    c = np.sqrt(2 * eps)
    for t in range(T):
        xi = Xi[:, t].astype(np.float64)
        gx = grad(x)
        yv = x + eps * gx + c * xi
        gy = grad(yv)
        q = x - yv - eps * gy
        la = logp(yv) - logp(x) - q @ q / (4 * eps) + 0.5 * xi @ xi
        acc[t] = np.log(u[t]) < la
        esjd += min(1.0, np.exp(min(la, 0.0))) * float((yv - x) @ (yv - x))
        x = yv if acc[t] else x
        S[:, t] = x
    return esjd / T, float(np.sum(S * S)) / T, S, acc


def logistic_adjoint(X, y, eps, x0, Xi, u, S, objective, tau=1.0):
    """d objective / d eps at the trajectory S (D, T) with its accept flags held
    fixed: the local terms at every step, then lambda_t = c_t + J_{t+1}^T
    lambda_{t+1} with J_{t+1} = I + eps H(x_t) (accepted) or I, solved
    sequentially with dense Hessians."""
    logp, grad, hess = logistic_parts(X, y, tau)
    D, T = S.shape
    c2 = np.sqrt(2 * eps)
    cvec = np.zeros((D, T))
    acc = np.zeros(T, bool)
    dys = np.zeros((D, T))
    Hs = []
    direct = 0.0
    for t in range(T):
        xb = np.asarray(x0, float) if t == 0 else S[:, t - 1]
        xi = Xi[:, t].astype(float)
        gx = grad(xb)
        yv = xb + eps * gx + c2 * xi
        gy = grad(yv)
        q = xb - yv - eps * gy
        la = logp(yv) - logp(xb) - q @ q / (4 * eps) + 0.5 * xi @ xi
        acc[t] = np.log(u[t]) < la
        Hx, Hy = hess(xb), hess(yv)
        Hs.append(Hx)
        dy = gx + xi / c2
        dys[:, t] = dy
        if objective == "mean_sq":
            cvec[:, t] += 2.0 * S[:, t] / T
            continue
        alpha = min(1.0, np.exp(min(la, 0.0)))
        dalpha = alpha if la < 0 else 0.0
        e = yv - xb
        e2 = float(e @ e)
        dq = -(dy + eps * (Hy @ dy)) - gy
        dla = gy @ dy - q @ dq / (2 * eps) + (q @ q) / (4 * eps ** 2)
        direct += (dalpha * dla * e2 + alpha * 2.0 * (e @ dy)) / T
        if t >= 1:
            Jx = np.eye(D) + eps * Hx
            w = q + eps * (Hy @ q)
            v = Jx @ gy - gx - (q - Jx @ w) / (2 * eps)
            cvec[:, t - 1] += (dalpha * e2 * v + alpha * 2.0 * eps * (Hx @ e)) / T
    lam = np.zeros((D, T))
    lam[:, T - 1] = cvec[:, T - 1]
    for t in range(T - 2, -1, -1):
        nxt = lam[:, t + 1]
        lam[:, t] = cvec[:, t] + ((nxt + eps * (Hs[t + 1] @ nxt)) if acc[t + 1] else nxt)
    geps = direct + sum(float(lam[:, t] @ dys[:, t]) for t in range(T) if acc[t])
    return geps
