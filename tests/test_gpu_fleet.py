"""Fleet of independent chains (pmcmc_fleet_solve) against the same chains
solved one at a time: every chain takes the same kernels on its own worker
stream, so trajectories agree to 1e-6 relative, accept flags and iteration
counts are equal."""
import numpy as np
import pytest

import pmcmc
from pmcmc import configs

pytestmark = pytest.mark.gpu


def test_fleet_matches_chains_solved_one_by_one():
    chains = configs.logistic_fleet(n_chains=6, scale=0.05)
    # a Gaussian chain in the same fleet
    g = pmcmc.DensityModel.diag_gaussian(10 ** np.random.default_rng(1).uniform(-1, 1, 20))
    chains.append((g, pmcmc.ParallelMALASampler(0.05, T=700, jacobian="diag", dtype=np.float32),
                   np.zeros(20, np.float32), 11, 0))
    h = pmcmc.Handle(0)
    fleet = pmcmc.fleet_solve(chains, workers=4, handle=h)
    assert any(m.dim > 256 for m, *_ in chains)  # both logistic contraction paths
    for (model, sampler, x0, seed, block), (S, info, lp, acc) in zip(chains, fleet):
        S1, i1, lp1, acc1 = pmcmc.solve(model, sampler, x0, seed=seed, block=block, handle=h,
                                        return_logp=True)
        assert info["converged"] == i1["converged"]
        assert info["iters"] == i1["iters"]
        assert np.array_equal(acc, acc1)
        np.testing.assert_allclose(S, S1, rtol=1e-6, atol=1e-6)


def test_fleet_reports_a_failing_chain():
    chains = configs.logistic_fleet(n_chains=2, scale=0.05)
    model, sampler, x0, seed, block = chains[1]
    bad = pmcmc.ParallelMALASampler(sampler.epsilon, T=sampler.T, probes=1, dtype=np.float32)
    bad.damping = 0.0  # invalid: ArgumentError from the library, not from the dataclass
    chains[1] = (model, bad, x0, seed, block)
    with pytest.raises(pmcmc.ArgumentError):
        pmcmc.fleet_solve(chains, workers=2)


def test_fleet_chains_match_the_fp64_sequential_chains():
    """Chains of the uneven fleet distribution (D on both tensor-core passes) solved
    together, each against its own FP64 sequential chain on the same tape
    (MALA.jl:322-346): identical accepts, trace error at most 1e-5."""
    import dataclasses

    import oracle as O
    chains = configs.logistic_fleet(n_chains=6, scale=0.05)
    # the FP32-state stopping rule of the 1e-5 trace bar (1e-7 + 1e-6 max|S|); a rule ten
    # times tighter sits at the FP32 rounding floor
    chains = [(m, dataclasses.replace(s, tol_abs=1e-7, tol_rel=1e-6, maxiter=400), x0, sd, b)
              for m, s, x0, sd, b in chains]
    assert any(m.dim > 256 for m, *_ in chains) and any(m.dim <= 256 for m, *_ in chains)
    fleet = pmcmc.fleet_solve(chains, workers=3, handle=pmcmc.Handle(0), errors="report")
    checked = 0
    for (model, sampler, x0, seed, block), (S, info, lp, acc) in zip(chains, fleet):
        if info["status"]:  # stiff chains that DEER itself cannot solve are reported
            continue
        assert info["converged"], info
        tg = O.Target.logistic(model.target["X"], model.target["y"])
        Xi, u = O.tape(seed, block, model.dim, sampler.T)
        S_seq, acc_seq, _ = O.mala_sequential_logistic(tg, sampler.epsilon, np.zeros(model.dim),
                                                       Xi, u)
        assert np.array_equal(np.asarray(acc, bool), acc_seq), (seed, model.dim)
        S = np.asarray(S, np.float64)
        err = np.max(np.linalg.norm(S - S_seq, axis=0) /
                     np.maximum(np.linalg.norm(S_seq, axis=0), 1e-30))
        assert err <= 1e-5, (seed, model.dim, err)
        checked += 1
    assert checked >= 4


def test_partitioned_fleet_on_one_rank_is_the_fleet():
    # fleet_solve_distributed on a world of one (gloo), the device fleet underneath: the
    # same results as fleet_solve, in chain order
    import os
    import socket

    import torch.distributed as dist
    from pmcmc import configs
    from pmcmc import distributed as Dd
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=0, world_size=1)
    try:
        chains = configs.logistic_fleet(n_chains=6, scale=0.05)
        h = pmcmc.Handle(0)
        got = Dd.fleet_solve_distributed(chains, device=0)
        ref = pmcmc.fleet_solve(chains, workers=8, handle=h, errors="report")
        assert len(got) == len(ref)
        for a, b in zip(got, ref):
            assert a[1]["status"] == b[1]["status"]
            np.testing.assert_array_equal(a[0], b[0])
            np.testing.assert_array_equal(a[3], b[3])
    finally:
        dist.destroy_process_group()
