"""T-split host logic (pmcmc.distributed) on CPU: two gloo ranks, each owning
slices whose device work is replaced by the FP64 oracle (deer_update on the
slice), must reproduce the oracle's single-block DEER solve: same Newton
iterates in exact arithmetic, so trajectories to 1e-10 and equal iteration
counts."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import oracle as O
from pmcmc import distributed as Dd


class OracleSlice:
    """A slice backend computing with the FP64 oracle (exact :diag Jacobian)."""

    def __init__(self, lam, eps, damping, seed, block, T):
        self.tg = O.Target.diag_gauss(lam)
        self.eps, self.damping = eps, damping
        self.Xi, self.u = O.tape(seed, block, lam.size, T)

    def begin(self, x0, seed, block, t0, W):
        self.t0, self.W = t0, W
        self.S = np.repeat(np.asarray(x0, float)[:, None], W, axis=1)

    def local(self, xbar0):
        sl = slice(self.t0, self.t0 + self.W)
        _, self.A, self.B = O.deer_update(self.tg, self.eps, xbar0, self.S, self.Xi[:, sl],
                                          self.u[sl], 0, 0, 0, jacobian="diag", damping=1.0)
        b = O.scan_seq(self.A, self.B, np.zeros(self.A.shape[0]))[:, -1]
        return np.stack([np.prod(self.A, axis=1), b])

    def finish(self, carry):
        Sn = O.scan_seq(self.A, self.B, carry)
        Sn = (1 - self.damping) * self.S + self.damping * Sn
        dmax = float(np.max(np.abs(Sn - self.S)))
        self.S = Sn
        return dmax, float(np.max(np.abs(Sn))), Sn[:, -1].copy()

    def result(self, xbar0):
        return self.S, np.zeros(self.W), np.zeros(self.W, bool), {}


def _problem():
    rng = np.random.default_rng(17)
    D, T = 6, 120
    lam = 10 ** rng.uniform(-1, 1, D)
    x0 = rng.standard_normal(D)
    return lam, x0, D, T


class _Sampler:
    T, maxiter, tol_abs, tol_rel = 120, 300, 1e-11, 1e-10


def _worker(rank, world, port, per_process, out_path):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    lam, x0, D, T = _problem()
    slices = [OracleSlice(lam, 0.05, 0.5, 3, 1, T) for _ in range(per_process)]
    res = Dd.tsplit_solve(slices, x0, _Sampler(), seed=3, block=1,
                          exchange=Dd.Exchange(per_process=per_process))
    # gather every slice's trajectory on every rank (fixed-size, padded)
    ex = Dd.Exchange(per_process=per_process)
    wmax = max(Dd.slice_bounds(T, ex.world, r)[1] for r in range(ex.world))
    pad = [np.pad(r.S, ((0, 0), (0, wmax - r.S.shape[1]))).reshape(-1) for r in res]
    allS = ex.allgather(pad)
    if rank == 0:
        S = np.concatenate([allS[r].reshape(D, wmax)[:, :Dd.slice_bounds(T, ex.world, r)[1]]
                            for r in range(ex.world)], axis=1)
        np.savez(out_path, S=S, iters=res[0].iters, converged=res[0].converged)
    dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _reference():
    lam, x0, D, T = _problem()
    Xi, u = O.tape(3, 1, D, T)
    return O.deer_solve(O.Target.diag_gauss(lam), 0.05, x0, Xi, u, 3, 1, jacobian="diag",
                        damping=0.5, tol_abs=1e-11, tol_rel=1e-10, maxiter=300)


@pytest.mark.parametrize("world,per_process", [(2, 1), (2, 2)])
def test_gloo_tsplit_matches_single_block_deer(tmp_path, world, per_process):
    out = str(tmp_path / "res.npz")
    mp.start_processes(_worker, args=(world, _free_port(), per_process, out), nprocs=world,
                       join=True, start_method="spawn")
    r = np.load(out)
    S_ref, info = _reference()
    assert bool(r["converged"]) and info["converged"]
    assert int(r["iters"]) == info["iters"]
    np.testing.assert_allclose(r["S"], S_ref, rtol=1e-10, atol=1e-12)


@pytest.mark.parametrize("nslices", [1, 3, 7])
def test_local_tsplit_oracle_slices(nslices):
    lam, x0, D, T = _problem()
    slices = [OracleSlice(lam, 0.05, 0.5, 3, 1, T) for _ in range(nslices)]
    res = Dd.tsplit_solve(slices, x0, _Sampler(), seed=3, block=1)
    S = np.concatenate([r.S for r in res], axis=1)
    S_ref, info = _reference()
    assert res[0].iters == info["iters"]
    np.testing.assert_allclose(S, S_ref, rtol=1e-10, atol=1e-12)


def test_slice_bounds_cover_the_block():
    for T, n in [(10, 3), (16384, 8), (7, 7)]:
        b = [Dd.slice_bounds(T, n, r) for r in range(n)]
        assert b[0][0] == 0 and sum(w for _, w in b) == T
        assert all(b[i][0] + b[i][1] == b[i + 1][0] for i in range(n - 1))
        assert max(w for _, w in b) - min(w for _, w in b) <= 1
