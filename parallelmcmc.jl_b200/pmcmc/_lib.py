"""ctypes binding of libpmcmc_deer.so (the C ABI declared in include/pmcmc_deer.h).

The product path has no CPU fallback: if the library or a CUDA device is
missing, every entry point raises.
"""
from __future__ import annotations

import ctypes as C
import os
import threading

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "lib", "libpmcmc_deer.so")

OK, ERR_ARGUMENT, ERR_DIMENSION, ERR_CUDA, ERR_NONFINITE, ERR_TIMEOUT, ERR_UNSUPPORTED, \
    ERR_NOMEM = range(8)
JAC = {"stoch_diag": 0, "diag": 1, "full": 2}
F32, F64 = 0, 1
MEM_HOST, MEM_DEVICE = 0, 1
EXEC = {"fused": 0, "plain": 1}

# Exported symbols (kept in step with include/pmcmc_deer.h; tests check both).
SYMBOLS = [
    "pmcmc_abi_version", "pmcmc_create", "pmcmc_destroy", "pmcmc_last_error",
    "pmcmc_target_diag_gauss", "pmcmc_target_dense_gauss", "pmcmc_target_logistic",
    "pmcmc_target_mass", "pmcmc_target_destroy", "pmcmc_tape", "pmcmc_deer_solve", "pmcmc_sample",
    "pmcmc_affine_scan_diag", "pmcmc_set_profiling", "pmcmc_get_profile",
    "pmcmc_affine_scan_diag_noalloc", "pmcmc_target_eigen", "pmcmc_deer_adjoint",
    "pmcmc_slice_begin", "pmcmc_slice_local", "pmcmc_slice_finish", "pmcmc_slice_result",
    "pmcmc_fleet_solve", "pmcmc_check_wait_bound", "pmcmc_mala_chains", "pmcmc_autotune",
    "pmcmc_mala_chains_adaptive",
]
OBJECTIVE = {"esjd": 0, "mean_sq": 1}
WAIT_KIND = {"lookback": 0, "mbarrier": 1}


class ArgumentError(ValueError):
    """Counterpart of Julia's ArgumentError (invalid sampler/solver arguments)."""


class DimensionMismatch(ValueError):
    """Counterpart of Julia's DimensionMismatch (inconsistent shapes)."""


class DeviceError(RuntimeError):
    """CUDA failure, bounded-wait timeout or non-finite trajectory."""


class Unsupported(NotImplementedError):
    """A valid request that this build does not implement."""


class DeerParams(C.Structure):
    _fields_ = [
        ("epsilon", C.c_double), ("T", C.c_int64), ("maxiter", C.c_int32),
        ("tol_abs", C.c_double), ("tol_rel", C.c_double), ("jacobian", C.c_int32),
        ("damping", C.c_double), ("probes", C.c_int32), ("window", C.c_int64),
        ("dtype", C.c_int32), ("exec", C.c_int32),
    ]


class Profile(C.Structure):
    _fields_ = [("sweep_launches", C.c_int64), ("sweep_ms", C.c_double),
                ("finalize_launches", C.c_int64), ("finalize_ms", C.c_double),
                ("pass_launches", C.c_int64), ("pass_ms", C.c_double),
                ("solve_launches", C.c_int64), ("solve_ms", C.c_double),
                ("solve_sweeps", C.c_int64)]


class Info(C.Structure):
    _fields_ = [
        ("iters", C.c_int32), ("converged", C.c_int32), ("metric", C.c_double),
        ("n_accept", C.c_int64), ("min_margin", C.c_double), ("max_defect", C.c_double),
        ("status", C.c_int32), ("path", C.c_int32),
    ]

    def as_dict(self):
        d = {k: getattr(self, k) for k, _ in self._fields_}
        d["path_names"] = [n for b, n in PATH_BITS if self.path & b]
        return d


class Adapt(C.Structure):
    _fields_ = [("n_warmup", C.c_int64), ("target_accept", C.c_double), ("gamma", C.c_double),
                ("t0", C.c_double), ("kappa", C.c_double)]


class FleetChain(C.Structure):
    _fields_ = [("target", C.c_void_p), ("params", DeerParams), ("x0", C.c_void_p),
                ("seed", C.c_uint64), ("block", C.c_uint64), ("S_out", C.c_void_p),
                ("logp_out", C.c_void_p), ("accept_out", C.c_void_p), ("info", Info),
                ("status", C.c_int32), ("pad0", C.c_int32)]


PATH_BITS = [(1, "fused_sweep"), (2, "cooperative"), (4, "graph"), (8, "tensor_core"),
             (16, "full_jacobian"), (32, "persistent"), (64, "tie_fp64")]


_vp = C.c_void_p
_lib = None
_lock = threading.Lock()


def load(path: str = LIB_PATH):
    """Load the library and declare signatures (no device work)."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(path):
            raise RuntimeError(
                f"{path} is missing: build it with `python parallelmcmc.jl_b200/build.py`")
        L = C.CDLL(path)
        L.pmcmc_abi_version.restype = C.c_int
        L.pmcmc_create.argtypes = [C.c_int, _vp, C.POINTER(_vp)]
        L.pmcmc_destroy.argtypes = [_vp]
        L.pmcmc_last_error.restype = C.c_char_p
        L.pmcmc_last_error.argtypes = [_vp]
        for fn in ("pmcmc_target_diag_gauss", "pmcmc_target_dense_gauss"):
            getattr(L, fn).argtypes = [_vp, C.c_int64, _vp, _vp, C.POINTER(_vp)]
        L.pmcmc_target_logistic.argtypes = [_vp, C.c_int64, C.c_int64, _vp, _vp, C.c_double,
                                            C.POINTER(_vp)]
        L.pmcmc_target_mass.argtypes = [_vp, _vp, _vp, C.POINTER(_vp)]
        L.pmcmc_target_destroy.argtypes = [_vp]
        L.pmcmc_tape.argtypes = [_vp, C.c_int64, C.c_int64, C.c_uint64, C.c_uint64, _vp, _vp,
                                 C.c_int32]
        L.pmcmc_deer_solve.argtypes = [_vp, _vp, C.POINTER(DeerParams), _vp, C.c_uint64,
                                       C.c_uint64, _vp, _vp, _vp, C.c_int32, C.POINTER(Info)]
        L.pmcmc_sample.argtypes = [_vp, _vp, C.POINTER(DeerParams), _vp, C.c_uint64, C.c_int64,
                                   _vp, _vp, _vp, C.c_int32, C.POINTER(Info)]
        L.pmcmc_affine_scan_diag.argtypes = [_vp, C.c_int32, C.c_int64, C.c_int64, _vp, _vp, _vp,
                                             _vp, C.c_int32]
        L.pmcmc_affine_scan_diag_noalloc.argtypes = [C.c_int32, C.c_int64, C.c_int64, _vp, _vp,
                                                     _vp, _vp, _vp]
        L.pmcmc_set_profiling.argtypes = [_vp, C.c_int32]
        L.pmcmc_get_profile.argtypes = [_vp, C.POINTER(Profile), C.c_int32]
        L.pmcmc_target_eigen.argtypes = [_vp, _vp, _vp]
        L.pmcmc_fleet_solve.argtypes = [_vp, C.POINTER(FleetChain), C.c_int64, C.c_int32,
                                        C.c_int32]
        L.pmcmc_slice_begin.argtypes = [_vp, _vp, C.POINTER(DeerParams), _vp, C.c_uint64,
                                        C.c_uint64, C.c_int64, C.c_int64, C.c_int32]
        L.pmcmc_slice_local.argtypes = [_vp, _vp, _vp, C.c_int32]
        L.pmcmc_slice_finish.argtypes = [_vp, _vp, _vp, _vp, C.c_int32]
        L.pmcmc_slice_result.argtypes = [_vp, _vp, _vp, _vp, _vp, C.POINTER(Info), C.c_int32]
        L.pmcmc_deer_adjoint.argtypes = [_vp, _vp, C.POINTER(DeerParams), _vp, C.c_uint64,
                                         C.c_uint64, _vp, C.c_int32, C.c_int32, _vp]
        L.pmcmc_check_wait_bound.argtypes = [_vp, C.c_int32, C.POINTER(C.c_double)]
        L.pmcmc_autotune.argtypes = [_vp, _vp, C.POINTER(DeerParams), _vp, C.c_uint64, C.c_int32,
                                     C.POINTER(C.c_int32), C.POINTER(C.c_double)]
        L.pmcmc_mala_chains.argtypes = [_vp, _vp, C.POINTER(DeerParams), C.c_int64, _vp, _vp,
                                        C.c_uint64, _vp, _vp, _vp, C.c_int32]
        L.pmcmc_mala_chains_adaptive.argtypes = [_vp, _vp, C.POINTER(DeerParams), C.c_int64, _vp,
                                                 _vp, C.c_uint64, C.POINTER(Adapt), _vp, _vp, _vp,
                                                 _vp, _vp, C.c_int32]
        for fn in SYMBOLS:
            if fn not in ("pmcmc_last_error", "pmcmc_abi_version"):
                getattr(L, fn).restype = C.c_int
        _lib = L
        return L


def check(rc: int, handle=None, what: str = ""):
    if rc == OK:
        return
    msg = ""
    if handle is not None:
        m = load().pmcmc_last_error(handle)
        msg = m.decode() if m else ""
    text = f"{what}: {msg}" if what else msg
    if rc == ERR_ARGUMENT:
        raise ArgumentError(text)
    if rc == ERR_DIMENSION:
        raise DimensionMismatch(text)
    if rc == ERR_UNSUPPORTED:
        raise Unsupported(text)
    raise DeviceError(f"status {rc}: {text}")


class Handle:
    """One device context: stream, workspace and cached CUDA graph
    (the DEERWorkspace of DEER.jl:47-90, owned on the device)."""

    def __init__(self, device: int = 0, stream: int | None = None):
        L = load()
        h = _vp()
        rc = L.pmcmc_create(int(device), _vp(stream) if stream else None, C.byref(h))
        if rc != OK:
            raise DeviceError(f"pmcmc_create(device={device}) failed with status {rc} "
                              "(no usable CUDA device?)")
        self.ptr = h
        self.device = int(device)

    def set_profiling(self, on: bool):
        check(load().pmcmc_set_profiling(self.ptr, int(bool(on))), self.ptr, "set_profiling")

    def profile(self, reset: bool = True) -> dict:
        p = Profile()
        check(load().pmcmc_get_profile(self.ptr, C.byref(p), int(reset)), self.ptr, "profile")
        return {k: getattr(p, k) for k, _ in p._fields_}

    def check_wait_bound(self, kind: str = "lookback") -> dict:
        """Run one of the library's bounded device waits ("lookback" or
        "mbarrier") on a flag that nothing sets.  A working bound returns
        status ERR_TIMEOUT with the device time the wait took; the handle
        stays usable afterwards."""
        if kind not in WAIT_KIND:
            raise ArgumentError(f"kind must be one of {sorted(WAIT_KIND)}")
        L = load()
        ms = C.c_double(0.0)
        rc = L.pmcmc_check_wait_bound(self.ptr, WAIT_KIND[kind], C.byref(ms))
        if rc not in (OK, ERR_TIMEOUT):
            check(rc, self.ptr, "check_wait_bound")
        m = L.pmcmc_last_error(self.ptr) if rc else b""
        return {"status": rc, "wait_ms": ms.value, "message": m.decode() if m else ""}

    def close(self):
        if getattr(self, "ptr", None):
            load().pmcmc_destroy(self.ptr)
            self.ptr = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_handles: dict[int, Handle] = {}


def default_handle(device: int = 0) -> Handle:
    with _lock:
        h = _handles.get(device)
    if h is None:
        h = Handle(device)
        with _lock:
            _handles[device] = h
    return h
