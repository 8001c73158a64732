"""One long DEER chain split along T across ranks (one slice per rank, one
exchange per Newton sweep).

The reference solves every block on one device (src/DEER/DEER.jl:506-595).
The Newton step's linear part is an affine scan, and affine maps compose
associatively (src/DEER/DEERScan.jl:102-173), so a block can be cut into
contiguous slices [t0, t0 + W) that evaluate and scan locally and exchange
only D-vectors:

    per sweep, on every slice r
      1. xbar0  = last column of slice r-1's iterate (x0 for slice 0)
      2. local  = A, B on the slice; map (prod_t A_t, b) of the slice
      3. carry  = maps of slices 0..r-1 applied to x0, in order         allgather
      4. finish = slice rescanned from carry, damped; its last column,
                  max|dS|, max|S|                                        allgather
      converged when max|dS| / (tol_abs + tol_rel max|S|) <= 1 (DEER.jl:567-578);
      the last columns gathered in 4 are the next sweep's left boundaries (1),
      so a sweep makes two exchanges

The iterates are those of the single-device solve in exact arithmetic.  The
device work of a slice runs in libpmcmc_deer.so (pmcmc_slice_*); this module is
the host-side plumbing: slice bounds, the exchanges and the convergence test.
`Exchange` wraps torch.distributed (NCCL between GPUs, gloo on CPU); several
slices may also live in one process (one handle each), run in lockstep.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import Optional, Sequence

import numpy as np

from . import _lib as L
from ._lib import ArgumentError


def slice_bounds(T: int, nslices: int, r: int) -> tuple[int, int]:
    """(t0, W) of slice r when T columns are split into nslices contiguous
    slices, the remainder spread over the first slices."""
    if not (1 <= nslices <= T):
        raise ArgumentError("need 1 <= nslices <= T")
    base, rem = divmod(T, nslices)
    t0 = r * base + min(r, rem)
    return t0, base + (1 if r < rem else 0)


class Exchange:
    """Collectives across processes for the slices this process owns.

    `group` is a torch.distributed process group (or None for the default
    group); `device` is where the exchanged tensors live ("cuda:k" for NCCL,
    "cpu" for gloo).  Every process owns the same number of slices, slice
    index = process rank * per_process + local index."""

    def __init__(self, per_process: int = 1, group=None, device: str = "cpu"):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        self.device = device
        self.per_process = per_process
        self.world = dist.get_world_size(group) * per_process
        self.first = dist.get_rank(group) * per_process

    def allgather(self, local: Sequence[np.ndarray]) -> list[np.ndarray]:
        import torch
        x = torch.as_tensor(np.stack(local), dtype=torch.float64, device=self.device)
        out = [torch.empty_like(x) for _ in range(self.dist.get_world_size(self.group))]
        self.dist.all_gather(out, x, group=self.group)
        return [v for t in out for v in t.cpu().numpy()]

    def allreduce_max(self, v: np.ndarray) -> np.ndarray:
        import torch
        x = torch.as_tensor(np.asarray(v, np.float64), device=self.device)
        self.dist.all_reduce(x, op=self.dist.ReduceOp.MAX, group=self.group)
        return x.cpu().numpy()


class LocalExchange:
    """All slices in this process: the collectives are list operations."""

    def __init__(self, nslices: int):
        self.world = nslices
        self.first = 0
        self.per_process = nslices

    def allgather(self, local):
        return [np.asarray(v, np.float64) for v in local]

    def allreduce_max(self, v):
        return np.asarray(v, np.float64)


class DeviceSlice:
    """Device work of one slice through the C ABI (host buffers, D-vectors)."""

    def __init__(self, model, sampler, handle: L.Handle):
        self.model = model
        self.sampler = sampler
        self.h = handle
        self.tgt = sampler.target(model, handle)
        self.dt = np.dtype(sampler.dtype)
        self.lib = L.load()

    def _vec(self, v):
        return np.ascontiguousarray(v, dtype=self.dt)

    def begin(self, x0, seed: int, block: int, t0: int, W: int):
        p = self.sampler.params()
        self.W = W
        self._x0 = self._vec(x0)
        L.check(self.lib.pmcmc_slice_begin(self.h.ptr, self.tgt, C.byref(p), self._x0.ctypes.data,
                                           int(seed), int(block), int(t0), int(W), L.MEM_HOST),
                self.h.ptr, "slice_begin")

    def local(self, xbar0) -> np.ndarray:
        xb = self._vec(xbar0)
        agg = np.empty((2, self.model.dim), self.dt)
        L.check(self.lib.pmcmc_slice_local(self.h.ptr, xb.ctypes.data, agg.ctypes.data,
                                           L.MEM_HOST), self.h.ptr, "slice_local")
        return agg.astype(np.float64)

    def finish(self, carry):
        c = self._vec(carry)
        last = np.empty(self.model.dim, self.dt)
        red = np.zeros(2)
        L.check(self.lib.pmcmc_slice_finish(self.h.ptr, c.ctypes.data, last.ctypes.data,
                                            red.ctypes.data, L.MEM_HOST), self.h.ptr,
                "slice_finish")
        return float(red[0]), float(red[1]), last.astype(np.float64)

    def result(self, xbar0):
        xb = self._vec(xbar0)
        D, W = self.model.dim, self.W
        S = np.empty((W, D), self.dt)
        lp = np.empty(W, self.dt)
        acc = np.empty(W, np.uint8)
        info = L.Info()
        L.check(self.lib.pmcmc_slice_result(self.h.ptr, xb.ctypes.data, S.ctypes.data,
                                            lp.ctypes.data, acc.ctypes.data, C.byref(info),
                                            L.MEM_HOST), self.h.ptr, "slice_result")
        return S.T, lp, acc.astype(bool), info.as_dict()


@dataclass
class SliceResult:
    rank: int
    t0: int
    S: np.ndarray       # (D, W)
    logp: np.ndarray    # (W,)
    accept: np.ndarray  # (W,)
    iters: int
    converged: bool
    metric: float
    info: dict


def tsplit_solve(slices: Sequence, x0, sampler, *, seed: int = 0, block: int = 0,
                 exchange=None) -> list[SliceResult]:
    """Solve one block with the T-split Newton iteration.

    `slices` are this process's slice backends (DeviceSlice or any object with
    begin/local/finish/result), in slice order; `exchange` joins processes
    (Exchange) or is None when this process owns every slice."""
    ex = exchange or LocalExchange(len(slices))
    if len(slices) != ex.per_process:
        raise ArgumentError("every process must own the same number of slices")
    x0 = np.asarray(x0, np.float64)
    ranks = [ex.first + i for i in range(len(slices))]
    bounds = [slice_bounds(int(sampler.T), ex.world, r) for r in ranks]
    for b, (t0, W) in zip(slices, bounds):
        b.begin(x0, seed, block, t0, W)
    # the iterate starts as x0 broadcast, so every slice's last column is x0: no
    # exchange before the first sweep
    D = x0.size
    lasts = [x0.copy() for _ in range(ex.world)]
    converged, metric, it = False, float("inf"), 0
    for it in range(1, int(sampler.maxiter) + 1):
        aggs_local = [b.local(x0 if r == 0 else lasts[r - 1]) for b, r in zip(slices, ranks)]
        aggs = ex.allgather([a.reshape(-1) for a in aggs_local])
        packed = []
        for b, r in zip(slices, ranks):
            carry = x0.copy()
            for q in range(r):
                a = aggs[q].reshape(2, -1)
                carry = a[0] * carry + a[1]
            dm, sm, last = b.finish(carry)
            packed.append(np.concatenate([np.asarray(last, np.float64).ravel(), [dm, sm]]))
        # one exchange: every slice's last column (the next sweep's left boundaries)
        # together with its maxima, whose max over the slices is the convergence test
        everyone = ex.allgather(packed)
        lasts = [v[:D] for v in everyone]
        dmax = max(float(v[D]) for v in everyone)
        smax = max(float(v[D + 1]) for v in everyone)
        metric = float(dmax / (sampler.tol_abs + sampler.tol_rel * smax))
        if metric <= 1.0:
            converged = True
            break
    out = []
    for b, r, (t0, W) in zip(slices, ranks, bounds):
        S, lp, acc, info = b.result(x0 if r == 0 else lasts[r - 1])
        out.append(SliceResult(r, t0, S, lp, acc, it, converged, metric, info))
    return out


def local_tsplit(model, sampler, x0, nslices: int, *, seed: int = 0, block: int = 0,
                 device: int = 0, handles: Optional[list] = None):
    """All slices of one block on one GPU (one handle each), run in lockstep:
    the T-split algorithm on a single device.  Returns (S (D, T), accept (T,),
    iters, converged)."""
    hs = handles or [L.Handle(device) for _ in range(nslices)]
    res = tsplit_solve([DeviceSlice(model, sampler, h) for h in hs], x0, sampler, seed=seed,
                       block=block)
    S = np.concatenate([r.S for r in res], axis=1)
    acc = np.concatenate([r.accept for r in res])
    return S, acc, res[0].iters, res[0].converged


# --------------------------------------------------------------------------- chains across GPUs
def chain_cost(model, sampler) -> float:
    """Work estimate of one chain's block: D N T for the logistic target (two
    contraction passes of N x D by T a sweep), D^2 T for the dense Gaussian,
    D T for the diagonal one."""
    tg = model.target or {}
    D, T = model.dim, int(sampler.T)
    if tg.get("kind") == "logistic":
        return float(D) * tg["X"].shape[0] * T
    if tg.get("kind") == "dense_gauss":
        return float(D) * D * T
    return float(D) * T


def partition_chains(costs: Sequence[float], nranks: int) -> list[list[int]]:
    """Longest-first assignment of independent chains to ranks: chains in
    descending cost (index breaks ties) each go to the rank with the least work
    so far (lowest rank breaks ties).  Every rank computes the same partition
    from the same costs, so no message is needed to agree on it.  Rank r's list
    is in assignment order (its largest chain first)."""
    if nranks < 1:
        raise ArgumentError("need at least one rank")
    order = sorted(range(len(costs)), key=lambda i: (-float(costs[i]), i))
    load = [0.0] * nranks
    parts: list[list[int]] = [[] for _ in range(nranks)]
    for i in order:
        r = min(range(nranks), key=lambda k: (load[k], k))
        parts[r].append(i)
        load[r] += float(costs[i])
    return parts


def fleet_solve_distributed(chains, *, group=None, workers: int = 8, device: Optional[int] = None,
                            errors: str = "report", gather: bool = True, solve=None):
    """Independent chains across ranks, one process per GPU (the MCMCThreads
    fleet of src/interface.jl:753-775, test/test-DEER-Interface.jl:300-318,
    spread over GPUs).  `chains` is the whole fleet, the same list on every
    rank, as for pmcmc.fleet_solve.  Every rank solves the chains
    partition_chains gives it with fleet_solve on its own GPU (`device`,
    default LOCAL_RANK); the chains share nothing, so no collective runs while
    they solve.  With gather=True the results are exchanged once at the end
    and every rank returns the list for all chains in their order; otherwise a
    dict {chain index: result} of this rank's chains.  `solve` replaces
    fleet_solve (tests on CPU)."""
    import os

    import torch.distributed as dist

    from . import core

    rank, world = dist.get_rank(group), dist.get_world_size(group)
    parts = partition_chains([chain_cost(m, s) for m, s, *_ in chains], world)
    mine = parts[rank]
    if solve is None:
        dev = int(os.environ.get("LOCAL_RANK", 0)) if device is None else device
        solve = lambda cs: core.fleet_solve(cs, workers=workers, device=dev, errors=errors)
    res = solve([chains[i] for i in mine]) if mine else []
    local = list(zip(mine, res))
    if not gather:
        return dict(local)
    every = [None] * world
    dist.all_gather_object(every, local, group=group)
    out = [None] * len(chains)
    for lst in every:
        for i, r in lst:
            out[i] = r
    return out
