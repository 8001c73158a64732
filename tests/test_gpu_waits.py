"""Bounded device waits: each wait kind the kernels use (the look-back spin of
the scans and sweeps, the mbarrier wait of the tensor-core pass) runs on a
flag that nothing sets, gives up at its bound and returns PMCMC_ERR_TIMEOUT;
the same handle then solves as before.  No fault, trap or hang is involved:
the kernel returns normally after the bound."""
import numpy as np
import pytest

import pmcmc
from pmcmc import _lib as L

pytestmark = pytest.mark.gpu


def _solve(h):
    prec = 10 ** np.random.default_rng(3).uniform(-1, 1, 16)
    model = pmcmc.DensityModel.diag_gaussian(prec)
    sampler = pmcmc.ParallelMALASampler(0.05, T=512, jacobian="diag", dtype=np.float32)
    return pmcmc.solve(model, sampler, np.zeros(16, np.float32), seed=5, block=0, handle=h,
                       return_logp=True)


@pytest.mark.parametrize("kind", ["lookback", "mbarrier"])
def test_wait_gives_up_at_its_bound_and_handle_stays_usable(kind):
    h = pmcmc.Handle(0)
    r = h.check_wait_bound(kind)
    assert r["status"] == L.ERR_TIMEOUT, r
    assert "reached its bound" in r["message"]
    # bounds: 2^22 look-back spins, 2e9 SM cycles for the mbarrier wait
    assert 1.0 <= r["wait_ms"] <= 20000.0, r
    S, info, lp, acc = _solve(h)
    S1, info1, lp1, acc1 = _solve(pmcmc.Handle(0))
    assert info["converged"] and info["iters"] == info1["iters"]
    assert np.array_equal(acc, acc1)
    np.testing.assert_array_equal(S, S1)


def test_unknown_wait_kind_is_an_argument_error():
    with pytest.raises(pmcmc.ArgumentError):
        pmcmc.Handle(0).check_wait_bound("spin")
