"""The allocation-free scan entry point (pmcmc_affine_scan_diag_noalloc).

It exists for callers that may not call cudaMalloc once running -- a process
whose own memory pool already owns the device (a Julia session with CUDA.jl's
pool, a serving process with a fixed memory budget) or a latency-critical loop
that cannot take an allocation's implicit synchronisation.  Its scratch is a
static 4 MiB device array shared by all calls.  This file is collected last so
that a failure here comes after every other test has run; it also passes when
run alone in a fresh process.
"""
import numpy as np
import pytest

import oracle as O
import pmcmc
from pmcmc import _lib as L

pytestmark = pytest.mark.gpu


def _call(dt, D, T, A, B, s0, S, stream):
    return L.load().pmcmc_affine_scan_diag_noalloc(
        L.F32 if dt == np.float32 else L.F64, D, T, A.data_ptr(), B.data_ptr(), s0.data_ptr(),
        S.data_ptr(), stream)


def test_noalloc_matches_handle_scan_and_sequential_scan_on_two_calls_in_a_row():
    torch = pytest.importorskip("torch")
    stream = torch.cuda.current_stream().cuda_stream
    h = pmcmc.Handle(0)
    rng = np.random.default_rng(0)
    # the first call on a device places the static array (lazy module loading)
    one = torch.ones(1, device="cuda")
    out1 = torch.empty(1, device="cuda")
    assert _call(np.float32, 1, 1, one, one, one, out1, stream) == L.OK
    for (D, T, dt) in [(8, 4096, np.float32), (5, 3001, np.float32), (6, 2000, np.float64)]:
        A = (0.2 * (rng.random((D, T)) - 0.5)).astype(dt)
        B = rng.standard_normal((D, T)).astype(dt)
        s0 = rng.standard_normal(D).astype(dt)
        At, Bt, st = (torch.from_numpy(x).cuda() for x in (A, B, s0))
        # keep the transposed copies alive across the calls
        At_c, Bt_c = At.T.contiguous(), Bt.T.contiguous()
        ref = pmcmc.solve_affine_scan_diag(A, B, s0, handle=h)
        seq = O.scan_seq(A.astype(np.float64), B.astype(np.float64), s0.astype(np.float64))
        outs = [torch.empty((T, D), dtype=At.dtype, device="cuda") for _ in range(2)]
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info()[0]
        nalloc0 = torch.cuda.memory_stats().get("allocation.all.allocated", 0)
        for S in outs:  # two calls in a row: the shared scratch keeps state between them
            assert _call(dt, D, T, At_c, Bt_c, st, S, stream) == L.OK
        torch.cuda.synchronize()
        # the calls took no device memory: the device's free bytes are unchanged and
        # torch's allocator served no allocation in between
        assert torch.cuda.mem_get_info()[0] == free0
        assert torch.cuda.memory_stats().get("allocation.all.allocated", 0) == nalloc0
        tol = 1e-5 if dt == np.float32 else 1e-12
        for S in outs:
            got = S.T.cpu().numpy()
            np.testing.assert_allclose(got, ref, rtol=tol, atol=tol)
            np.testing.assert_allclose(got, seq, rtol=tol, atol=tol)


def test_noalloc_rejects_sizes_beyond_its_scratch():
    torch = pytest.importorskip("torch")
    stream = torch.cuda.current_stream().cuda_stream
    D, T = 1000, 100_000  # needs ~ 3 * 4 * D * T / 8 bytes of scratch >> 4 MiB
    A = torch.zeros((T, D), device="cuda")
    S = torch.empty_like(A)
    s0 = torch.zeros(D, device="cuda")
    assert _call(np.float32, D, T, A, A, s0, S, stream) == L.ERR_NOMEM
