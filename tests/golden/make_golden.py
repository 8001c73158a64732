"""Regenerate the committed known-answer fixtures in tests/golden/ from the FP64 oracle.

    python tests/golden/make_golden.py

The reference ships no golden vectors (all its tests draw from MersenneTwister
at run time), so these fixtures pin (a) the project tape generator and (b) the
oracle's outputs on small cases, for regression and for GPU parity.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(HERE)), "oracle"))
import oracle as O  # noqa: E402


def cases():
    out = {}
    # tape: seed 0 block 0 and an odd D (partial quad)
    for (seed, block, D, T) in [(0, 0, 5, 8), (7, 3, 2, 16), (2**40 + 5, 9, 13, 4)]:
        Xi, u = O.tape(seed, block, D, T)
        out[f"tape_{seed}_{block}_{D}_{T}_Xi"] = np.asarray(Xi, np.float32)
        out[f"tape_{seed}_{block}_{D}_{T}_u"] = u
    # probes
    out["probe_3_1_2_1_300_4"] = O.probe(3, 1, 2, 1, 300, 4)

    # config-1 quick start: D=2 standard normal, eps 0.1, T=64, stoch_diag, x0 = 0, 500 samples.
    # Blocks chain like the reference's block loop (interface.jl:584-599): block b+1
    # starts from the last kept column of block b's DEER solution.  The sequential
    # trace of each block starts from the same state.
    D, T, N, eps = 2, 64, 500, 0.1
    tg = O.Target.diag_gauss(np.ones(D))
    x = np.zeros(D)
    vals, seqs, accs, iters = [], [], [], []
    nsteps, b = 0, 0
    while nsteps < N:
        Xi, u = O.tape(0, b, D, T)
        S_seq, acc, _ = O.mala_sequential(tg, eps, x, Xi, u)
        S_deer, info = O.deer_solve(tg, eps, x, Xi, u, 0, b, jacobian="stoch_diag", probes=1,
                                    damping=0.5, tol_abs=1e-6, tol_rel=1e-5, maxiter=200)
        nkeep = min(T, N - nsteps)
        vals.append(S_deer[:, :nkeep])
        seqs.append(S_seq[:, :nkeep])
        accs.append(acc[:nkeep])
        iters.append(info["iters"])
        x = S_deer[:, nkeep - 1].copy()
        nsteps += nkeep
        b += 1
    out["cfg1_deer_values"] = np.concatenate(vals, axis=1)
    out["cfg1_seq_values"] = np.concatenate(seqs, axis=1)
    out["cfg1_seq_accept"] = np.concatenate(accs)
    out["cfg1_deer_iters"] = np.asarray(iters)

    # diag Gaussian (anisotropic), :diag, FP64
    rng = np.random.default_rng(1)
    D, T = 10, 96
    lam = 10 ** rng.uniform(-1, 1, D)
    x0 = rng.standard_normal(D)
    Xi, u = O.tape(1, 0, D, T)
    tg = O.Target.diag_gauss(lam)
    S_seq, acc, la = O.mala_sequential(tg, 0.05, x0, Xi, u)
    S_deer, info = O.deer_solve(tg, 0.05, x0, Xi, u, 1, 0, jacobian="diag", damping=0.5,
                                tol_abs=1e-10, tol_rel=1e-9, maxiter=300)
    out.update(diag_lam=lam, diag_x0=x0, diag_seq=S_seq, diag_acc=acc, diag_deer=S_deer,
               diag_iters=np.asarray([info["iters"]]))

    # dense Gaussian, stoch_diag with 2 probes, FP64
    D, T = 6, 64
    Q = rng.standard_normal((D, D))
    P = Q @ Q.T / D + np.eye(D)
    x0 = rng.standard_normal(D)
    Xi, u = O.tape(4, 2, D, T)
    tg = O.Target.dense_gauss(P)
    S_seq, acc, la = O.mala_sequential(tg, 0.1, x0, Xi, u)
    S_deer, info = O.deer_solve(tg, 0.1, x0, Xi, u, 4, 2, jacobian="stoch_diag", probes=2,
                                damping=0.5, tol_abs=1e-10, tol_rel=1e-9, maxiter=400)
    out.update(dense_P=P, dense_x0=x0, dense_seq=S_seq, dense_acc=acc, dense_deer=S_deer,
               dense_iters=np.asarray([info["iters"]]))
    return out


if __name__ == "__main__":
    data = cases()
    path = os.path.join(HERE, "golden_v1.npz")
    np.savez_compressed(path, **data)
    print(path, os.path.getsize(path), "bytes", len(data), "arrays")
