"""Seeded synthetic workloads with the shapes of the benchmark configurations.

Each function returns (model, sampler, x0, meta).  All data come from NumPy's
PCG64 seeded as stated; the MALA tape itself is the library's counter-based
tape of (seed, block).
"""
from __future__ import annotations

import numpy as np

from .core import DensityModel, ParallelMALASampler


def quickstart_2d(dtype=np.float64):
    """2-D standard normal, eps 0.1, T 64, :stoch_diag (1 probe), x0 = 0, 500 samples
    (the README quick start, README.md:59-66)."""
    model = DensityModel.diag_gaussian(np.ones(2))
    sampler = ParallelMALASampler(0.1, T=64, jacobian="stoch_diag", probes=1, dtype=dtype)
    return model, sampler, np.zeros(2, dtype=dtype), {"N": 500, "seed": 0,
                                                       "workload": "gauss2d_T64_stoch_diag"}


def aniso_diag_d100(T=16384, dtype=np.float32, seed=1):
    """Anisotropic diagonal Gaussian, D = 100, precisions log-uniform in [1e-2, 1e2]
    (seed 1), mean 0, eps 0.05, T = 16384, :diag, FP32 state, x0 ~ N(0, I)."""
    rng = np.random.default_rng(seed)
    lam = 10.0 ** rng.uniform(-2.0, 2.0, 100)
    x0 = rng.standard_normal(100).astype(dtype)
    model = DensityModel.diag_gaussian(lam)
    sampler = ParallelMALASampler(0.05, T=T, jacobian="diag", dtype=dtype)
    return model, sampler, x0, {"N": T, "seed": seed,
                                "workload": f"diag_gauss_D100_T{T}_diag_f32"}


def logistic_n10k_d256(T=65536, dtype=np.float32, seed=2, N=10_000, D=256):
    """Bayesian logistic regression: X iid N(0,1)/sqrt(D), theta* ~ N(0, I),
    y ~ Bernoulli(sigmoid(X theta*)), prior N(0, I), seed 2; eps 0.01, :stoch_diag."""
    rng = np.random.default_rng(seed)
    X = (rng.standard_normal((N, D)) / np.sqrt(D)).astype(np.float32).astype(np.float64)
    th = rng.standard_normal(D)
    y = (rng.random(N) < 1.0 / (1.0 + np.exp(-(X @ th)))).astype(np.float64)
    model = DensityModel.logistic(X, y, prior_prec=1.0)
    sampler = ParallelMALASampler(0.01, T=T, jacobian="stoch_diag", probes=1, dtype=dtype)
    return model, sampler, np.zeros(D, dtype=dtype), {"N": T, "seed": seed,
                                                      "workload": f"logistic_N{N}_D{D}_T{T}"}


def haar_orthogonal(rng, D):
    """Haar-random orthogonal matrix: QR of a Gaussian matrix with the sign of R's
    diagonal folded into Q."""
    Z = rng.standard_normal((D, D))
    Q, R = np.linalg.qr(Z)
    return Q * np.sign(np.diag(R))


def correlated_gauss_d64(T=8192, dtype=np.float32, seed=3, jacobian="full"):
    """Correlated Gaussian, D = 64: Sigma = Q diag(s) Q' with s log-uniform in
    [0.1, 10] and Q Haar (seed 3); eps 0.05, T = 8192."""
    rng = np.random.default_rng(seed)
    D = 64
    s = 10.0 ** rng.uniform(-1.0, 1.0, D)
    Q = haar_orthogonal(rng, D)
    P = (Q / s) @ Q.T
    P = 0.5 * (P + P.T)
    model = DensityModel.dense_gaussian(P)
    sampler = ParallelMALASampler(0.05, T=T, jacobian=jacobian, dtype=dtype)
    return model, sampler, np.zeros(D, dtype=dtype), {"N": T, "seed": seed, "s": s, "Q": Q,
                                                      "workload": f"corr_gauss_D64_T{T}"}


def logistic_fleet(n_chains=512, scale=1.0, dtype=np.float32, first=0):
    """Uneven fleet of independent logistic-regression chains: chain c (seed c)
    has D uniform on {16, 32, ..., 512}, N uniform in [1000, 20000], T uniform
    in [1024, 32768], eps = 0.5 / sqrt(D), :stoch_diag, data from the generative
    model of logistic_n10k_d256.  `scale` < 1 shrinks N and T (a bounded sample
    of the fleet); chains first .. first + n_chains - 1.
    Returns a list of (model, sampler, x0, seed, block)."""
    out = []
    for c in range(first, first + n_chains):
        rng = np.random.default_rng(c)
        D = int(16 * rng.integers(1, 33))
        N = max(16, int(rng.integers(1000, 20001) * scale))
        T = max(16, int(rng.integers(1024, 32769) * scale))
        X = (rng.standard_normal((N, D)) / np.sqrt(D)).astype(np.float32).astype(np.float64)
        th = rng.standard_normal(D)
        y = (rng.random(N) < 1.0 / (1.0 + np.exp(-(X @ th)))).astype(np.float64)
        model = DensityModel.logistic(X, y, prior_prec=1.0)
        sampler = ParallelMALASampler(0.5 / np.sqrt(D), T=T, jacobian="stoch_diag", probes=1,
                                      dtype=dtype)
        out.append((model, sampler, np.zeros(D, dtype=dtype), c, 0))
    return out
