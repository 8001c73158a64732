"""pmcmc -- B200 DEER hot path of ParallelMCMC.jl behind the reference's sampler API.

The numerics run in libpmcmc_deer.so (hand-written sm_100a CUDA); this package
is the host-side mirror of the reference interface for that path.
"""
from types import SimpleNamespace

from ._lib import (ArgumentError, DeviceError, DimensionMismatch, Handle, Unsupported,
                   default_handle, load)
from .adapt import (AdaptiveMALASampler, adapt_step_size, adaptive_chains, dual_average_update,
                    sample_adaptive)
from .core import (Chain, ChainSet, Cholesky, DensityModel, MCMCThreads, ParallelMALASampler, ParallelMALAState,
                   ParallelMALATransition, adjoint, autotune, fleet_solve, mala_chains, sample,
                   solve,
                   cholesky, solve_affine_scan_diag, step, tape)

# Module-style aliases matching ParallelMCMC.DEER / ParallelMCMC.DEERScan.
DEER = SimpleNamespace(solve=solve, adjoint=adjoint, solve_affine_scan_diag=solve_affine_scan_diag)
DEERScan = SimpleNamespace(solve_affine_scan_diag=solve_affine_scan_diag)

__all__ = [
    "ArgumentError", "DimensionMismatch", "DeviceError", "Unsupported", "Handle",
    "default_handle", "load", "Chain", "DensityModel", "ParallelMALASampler",
    "ParallelMALAState", "ParallelMALATransition", "adjoint", "fleet_solve", "sample", "solve",
    "step", "tape", "mala_chains", "autotune", "AdaptiveMALASampler", "adapt_step_size", "dual_average_update",
    "adaptive_chains", "sample_adaptive",
    "solve_affine_scan_diag", "DEER", "DEERScan", "Cholesky", "cholesky", "MCMCThreads",
    "ChainSet",
]
