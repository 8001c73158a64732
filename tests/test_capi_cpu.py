"""C-ABI library checks that need no GPU: it builds, loads, exports every symbol
declared in include/pmcmc_deer.h, and the host API validates like the reference."""
import ctypes
import os
import re
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "parallelmcmc.jl_b200")
LIB = os.path.join(PKG, "lib", "libpmcmc_deer.so")
HDR = os.path.join(ROOT, "include", "pmcmc_deer.h")


def _ensure_built():
    if not os.path.exists(LIB):
        subprocess.run([sys.executable, os.path.join(PKG, "build.py")], check=True)
    return LIB


def _declared():
    txt = open(HDR).read()
    return sorted(set(re.findall(r"^(?:int|const char\*)\s+(pmcmc_\w+)\s*\(", txt, re.M)))


def test_library_loads_and_exports_header_symbols():
    lib = ctypes.CDLL(_ensure_built())
    names = _declared()
    assert len(names) >= 12
    for n in names:
        assert hasattr(lib, n), f"{n} declared in pmcmc_deer.h but not exported"
    lib.pmcmc_abi_version.restype = ctypes.c_int
    assert lib.pmcmc_abi_version() == 1


def test_python_symbol_list_matches_header():
    from pmcmc import _lib
    assert set(_lib.SYMBOLS) <= set(_declared())
    assert set(_declared()) <= set(_lib.SYMBOLS)


def test_sampler_validation_mirrors_reference():
    # interface.jl:273-275, test-DEER-Interface.jl:22-36
    from pmcmc import ArgumentError, ParallelMALASampler
    s = ParallelMALASampler(0.05)
    assert (s.T, s.maxiter, s.jacobian, s.damping, s.probes) == (64, 200, "stoch_diag", 0.5, 1)
    assert (s.tol_abs, s.tol_rel) == (1e-6, 1e-5)
    s2 = ParallelMALASampler(0.1, T=32, jacobian=":stoch_diag", damping=0.8)
    assert s2.T == 32 and s2.damping == 0.8
    assert ParallelMALASampler(0.1, jacobian="full").jacobian == "full"
    for bad in (dict(epsilon=0.0), dict(epsilon=-1.0), dict(epsilon=0.1, jacobian="dense"),
                dict(epsilon=0.1, cholM=object())):
        with pytest.raises(ArgumentError):
            ParallelMALASampler(**bad)


def test_mass_matrix_arguments():
    # cholM = cholesky(M) (interface.jl:84-100): the factor is checked up front
    import numpy as np
    from pmcmc import ArgumentError, Cholesky, DimensionMismatch, ParallelMALASampler, cholesky
    from pmcmc.adapt import AdaptiveMALASampler
    rng = np.random.default_rng(3)
    A = rng.standard_normal((5, 5))
    M = A @ A.T + 5 * np.eye(5)
    c = cholesky(M)
    assert np.allclose(c.L @ c.L.T, M) and np.allclose(c.U, c.L.T)
    assert np.array_equal(c.L, np.tril(c.L))
    s = ParallelMALASampler(0.1, cholM=c)
    assert np.array_equal(s.cholM.L, c.L)
    # a plain lower factor is accepted; the strict upper part is ignored
    s2 = ParallelMALASampler(0.1, cholM=c.L + np.triu(np.ones((5, 5)), 1))
    assert np.array_equal(s2.cholM.L, c.L)
    assert np.array_equal(AdaptiveMALASampler(0.1, cholM=c).cholM.L, c.L)
    with pytest.raises(DimensionMismatch):
        ParallelMALASampler(0.1, cholM=np.ones((2, 3)))
    with pytest.raises(ArgumentError):
        ParallelMALASampler(0.1, cholM=np.diag([1.0, 0.0, 1.0]))
    with pytest.raises(ArgumentError):
        Cholesky(-np.eye(3))
    with pytest.raises(DimensionMismatch):
        from pmcmc.core import _mass_factor
        _mass_factor(c, 4)


def test_model_requires_device_target():
    import numpy as np
    from pmcmc import ArgumentError, DensityModel, DimensionMismatch
    m = DensityModel(lambda x: 0.0, lambda x: x, 3)
    with pytest.raises(ArgumentError):
        m.device_target(None)
    with pytest.raises(DimensionMismatch):
        DensityModel.diag_gaussian(np.ones(3), mean=np.zeros(2))
    with pytest.raises(DimensionMismatch):
        DensityModel.dense_gaussian(np.ones((2, 3)))


def test_no_silent_cpu_fallback_without_gpu():
    import numpy as np
    from conftest import cuda_available
    if cuda_available():
        pytest.skip("a GPU is present")
    import pmcmc
    m = pmcmc.DensityModel.diag_gaussian(np.ones(2))
    with pytest.raises(pmcmc.DeviceError):
        pmcmc.sample(m, pmcmc.ParallelMALASampler(0.1), 10)


def test_mcmcthreads_arguments():
    import numpy as np
    from pmcmc import ArgumentError, DensityModel, MCMCThreads, ParallelMALASampler, sample
    m = DensityModel.diag_gaussian(np.ones(2))
    s = ParallelMALASampler(0.1, T=8)
    with pytest.raises(ArgumentError):
        sample(m, s, MCMCThreads(), 10)
    with pytest.raises(ArgumentError):
        sample(m, s, MCMCThreads(), 0, 2)
    with pytest.raises(ArgumentError):
        sample(m, s, 10, 3)
