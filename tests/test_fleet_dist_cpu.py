"""Independent chains across ranks (pmcmc.distributed.fleet_solve_distributed):
the partition, and a world-size-2 gloo run on CPU in which each chain is solved
by the CPU oracle in place of the device fleet."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import oracle as O
import pmcmc
from pmcmc import distributed as Dd


def _fleet():
    rng = np.random.default_rng(5)
    chains = []
    for c in range(9):
        D = int(rng.integers(2, 9))
        lam = 10 ** rng.uniform(-0.5, 0.5, D)
        model = pmcmc.DensityModel.diag_gaussian(lam)
        sampler = pmcmc.ParallelMALASampler(0.1, T=int(rng.integers(16, 97)), jacobian="diag",
                                            tol_abs=1e-11, tol_rel=1e-10, maxiter=300)
        chains.append((model, sampler, rng.standard_normal(D), 100 + c, c % 3))
    return chains


def _oracle_solve(chains):
    """What fleet_solve returns for each chain, from the CPU oracle's DEER."""
    out = []
    for model, smp, x0, seed, block in chains:
        Xi, u = O.tape(seed, block, model.dim, smp.T)
        tg = O.Target.diag_gauss(model.target["prec"])
        S, info = O.deer_solve(tg, smp.epsilon, x0, Xi, u, seed, block, jacobian="diag",
                               tol_abs=smp.tol_abs, tol_rel=smp.tol_rel, maxiter=smp.maxiter)
        out.append((S, {"iters": info["iters"], "converged": info["converged"], "status": 0},
                    None, None))
    return out


def _worker(rank, world, port, out_path):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    chains = _fleet()
    res = Dd.fleet_solve_distributed(chains, solve=_oracle_solve)
    mine = Dd.fleet_solve_distributed(chains, solve=_oracle_solve, gather=False)
    np.savez(out_path + f".{rank}.npz", *[r[0] for r in res],
             iters=np.array([r[1]["iters"] for r in res]), mine=np.array(sorted(mine)))
    dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_partition_is_balanced_and_covers_every_chain():
    rng = np.random.default_rng(0)
    for n, ranks in [(512, 8), (37, 4), (3, 5), (0, 2)]:
        costs = rng.uniform(1, 100, n)
        parts = Dd.partition_chains(costs, ranks)
        assert len(parts) == ranks
        assert sorted(i for p in parts for i in p) == list(range(n))
        assert parts == Dd.partition_chains(costs, ranks)  # the same on every rank
        if n:
            loads = [costs[p].sum() if p else 0.0 for p in parts]
            assert max(loads) - min(loads) <= costs.max() + 1e-9
    with pytest.raises(pmcmc.ArgumentError):
        Dd.partition_chains([1.0], 0)


def test_chain_cost_follows_the_target():
    X = np.zeros((50, 4))
    lg = pmcmc.DensityModel.logistic(X, np.zeros(50))
    s = pmcmc.ParallelMALASampler(0.1, T=10)
    assert Dd.chain_cost(lg, s) == 4 * 50 * 10
    assert Dd.chain_cost(pmcmc.DensityModel.dense_gaussian(np.eye(3)), s) == 90
    assert Dd.chain_cost(pmcmc.DensityModel.diag_gaussian(np.ones(3)), s) == 30


def test_gloo_fleet_matches_the_chains_solved_alone(tmp_path):
    world = 2
    out = str(tmp_path / "res")
    mp.start_processes(_worker, args=(world, _free_port(), out), nprocs=world, join=True,
                       start_method="spawn")
    alone = _oracle_solve(_fleet())
    parts = Dd.partition_chains([Dd.chain_cost(m, s) for m, s, *_ in _fleet()], world)
    for rank in range(world):
        r = np.load(out + f".{rank}.npz")
        assert list(r["mine"]) == sorted(parts[rank])
        assert list(r["iters"]) == [a[1]["iters"] for a in alone]
        for i, a in enumerate(alone):
            np.testing.assert_array_equal(r[f"arr_{i}"], a[0])
