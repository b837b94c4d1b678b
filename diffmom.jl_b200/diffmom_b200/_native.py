"""ctypes binding of libdiffmom_b200.so (the C ABI declared in
include/diffmom_b200.h).

The library is the only compute path: there is no CPU fallback.  Loading fails
loudly when the shared object is missing, and every call checks its status and
raises the exception type the reference raises for the same condition.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
LIB_PATH = _HERE.parent / "lib" / "libdiffmom_b200.so"
HEADER_PATH = _HERE.parent.parent / "include" / "diffmom_b200.h"

DMB_OK = 0
DMB_ERR_ARGUMENT = 1
DMB_ERR_OVERFLOW = 2
DMB_ERR_DIMENSION = 3
DMB_ERR_BUDGET = 4
DMB_ERR_NOT_CONVERGED = 5
DMB_ERR_CUDA = 6
DMB_ERR_STATE = 7
DMB_ERR_BREAKDOWN = 8
DMB_ERR_TIMEOUT = 9

PREC_FP64 = 0
PREC_MIXED = 1

PRECOND_NONE = 0
PRECOND_NF_LU = 1
PRECOND_NF_DIAG = 2
PRECOND_LOCAL_INV = 3
PRECOND_LEARNED = 4
PRECOND_RING = 5

SIDE_LEFT = 0
SIDE_RIGHT = 1

OPT_TENSOR_CORES = 1
OPT_TC_MIN_RHS = 2
OPT_FAR_TILE = 3
OPT_EXACT_KRYLOV = 4
OPT_PRECOND_TF32_TERMS = 5
OPT_GMRES_GRAPHS = 6
OPT_OPERATOR = 7
OPT_TRUE_RESIDUAL = 8
OPT_SPIN_LIMIT = 9
OPT_TUNE_TC_GEMM = 10
OPT_TUNE_TC_SYRK = 11
OPT_PRECOND_BF16 = 12
OPT_INT8_SCHEME = 13
OPT_TUNE_INT8_TILE = 14


class DiffMoMError(RuntimeError):
    """Generic library failure (ErrorException in the reference)."""


class NotConvergedError(DiffMoMError):
    """GMRES did not reach the tolerance (IterativeSolve.jl:50-61)."""


class FactorizationBreakdown(DiffMoMError):
    """Zero or non-finite pivot in the near-field factorisation."""


class DimensionMismatch(ValueError):
    pass


class DeviceWaitTimeout(DiffMoMError, TimeoutError):
    """A bounded wait inside a kernel gave up (DMB_ERR_TIMEOUT): the call's
    results are invalid, the context stays usable."""


_EXC = {
    DMB_ERR_ARGUMENT: ValueError,          # ArgumentError
    DMB_ERR_OVERFLOW: OverflowError,       # OverflowError
    DMB_ERR_DIMENSION: DimensionMismatch,  # DimensionMismatch
    DMB_ERR_BUDGET: ValueError,            # ArgumentError (resource limit)
    DMB_ERR_NOT_CONVERGED: NotConvergedError,
    DMB_ERR_CUDA: DiffMoMError,
    DMB_ERR_STATE: DiffMoMError,
    DMB_ERR_BREAKDOWN: FactorizationBreakdown,
    DMB_ERR_TIMEOUT: DeviceWaitTimeout,
}


class GmresStats(ctypes.Structure):
    _fields_ = [("niter", ctypes.c_int32), ("solved", ctypes.c_int32),
                ("residual", ctypes.c_double), ("true_residual", ctypes.c_double),
                ("restarts", ctypes.c_int32), ("reserved", ctypes.c_int32)]


class Timings(ctypes.Structure):
    _fields_ = [("geometry_ms", ctypes.c_double), ("assembly_ms", ctypes.c_double),
                ("precond_ms", ctypes.c_double), ("rhs_ms", ctypes.c_double),
                ("solve_ms", ctypes.c_double), ("nnz_ratio", ctypes.c_double),
                ("kernels", ctypes.c_int64), ("gmres_ms", ctypes.c_double)]


class SolveParams(ctypes.Structure):
    _fields_ = [("k", ctypes.c_double), ("eta0", ctypes.c_double), ("cutoff", ctypes.c_double),
                ("tol", ctypes.c_double), ("quad_order", ctypes.c_int32), ("precision", ctypes.c_int32),
                ("precond_kind", ctypes.c_int32), ("precond_side", ctypes.c_int32),
                ("maxiter", ctypes.c_int32), ("reserved", ctypes.c_int32),
                ("kvec", ctypes.c_double * 3), ("pol", ctypes.c_double * 3), ("E0", ctypes.c_double)]


class BatchItem(ctypes.Structure):
    _fields_ = [("xyz", ctypes.c_void_p), ("tri", ctypes.c_void_p), ("nv", ctypes.c_int64),
                ("nt", ctypes.c_int64), ("n", ctypes.c_int64), ("tplus", ctypes.c_void_p),
                ("tminus", ctypes.c_void_p), ("evert", ctypes.c_void_p), ("vplus_opp", ctypes.c_void_p),
                ("vminus_opp", ctypes.c_void_p), ("len", ctypes.c_void_p), ("area_plus", ctypes.c_void_p),
                ("area_minus", ctypes.c_void_p), ("zs", ctypes.c_void_p), ("kvec", ctypes.c_double * 3),
                ("pol", ctypes.c_double * 3), ("E0", ctypes.c_double), ("I_out", ctypes.c_void_p),
                ("sigma", ctypes.c_double), ("stats", GmresStats), ("latency_ms", ctypes.c_double),
                ("solve_ms", ctypes.c_double)]


class AcaInfo(ctypes.Structure):
    _fields_ = [("n_dense", ctypes.c_int64), ("n_lowrank", ctypes.c_int64), ("n_fallback", ctypes.c_int64),
                ("max_rank_used", ctypes.c_int64), ("entries_stored", ctypes.c_int64),
                ("n_unconverged", ctypes.c_int64), ("build_ms", ctypes.c_double), ("plan_ms", ctypes.c_double),
                ("dense_ms", ctypes.c_double), ("lowrank_ms", ctypes.c_double)]


_P = ctypes.c_void_p
_D = ctypes.c_double
_I = ctypes.c_int
_L = ctypes.c_int64
_DP = ctypes.POINTER(ctypes.c_double)
_LP = ctypes.POINTER(ctypes.c_int64)
_FP = ctypes.POINTER(ctypes.c_float)
_IP = ctypes.POINTER(ctypes.c_int32)

SIGNATURES = {
    "dmb_version": ([], ctypes.c_char_p),
    "dmb_ctx_create": ([_I, ctypes.POINTER(_P)], _I),
    "dmb_ctx_destroy": ([_P], _I),
    "dmb_last_error": ([_P], ctypes.c_char_p),
    "dmb_get_timings": ([_P, ctypes.POINTER(Timings)], _I),
    "dmb_set_option": ([_P, _I, _I], _I),
    "dmb_get_far_tile": ([_P, ctypes.POINTER(ctypes.c_int)], _I),
    "dmb_tune_report": ([ctypes.c_char_p, ctypes.c_size_t, ctypes.POINTER(ctypes.c_size_t)], _I),
    "dmb_kernel_timing_family": ([_P, _I, _DP, ctypes.POINTER(ctypes.c_int64), _DP], _I),
    "dmb_batch_create": ([_I, _I, ctypes.POINTER(_P)], _I),
    "dmb_batch_destroy": ([_P], _I),
    "dmb_batch_last_error": ([_P], ctypes.c_char_p),
    "dmb_batch_assembly_ms": ([_P, _DP], _I),
    "dmb_batch_solve": ([_P, ctypes.POINTER(SolveParams), ctypes.POINTER(BatchItem), _L, _DP], _I),
    "dmb_mesh_upload": ([_P, _DP, _LP, _L, _L], _I),
    "dmb_rwg_upload": ([_P, _L, _LP, _LP, _LP, _LP, _LP, _DP, _DP, _DP], _I),
    "dmb_assemble_z": ([_P, _D, _D, _I, _I, _DP], _I),
    "dmb_z_entries": ([_P, _LP, _LP, _L, _DP], _I),
    "dmb_apply_impedance": ([_P, _DP], _I),
    "dmb_matvec": ([_P, _DP, _DP, _L], _I),
    "dmb_prepare_operator": ([_P, _D, _D, _I], _I),
    "dmb_matvec_free": ([_P, _DP, _DP], _I),
    "dmb_matvec_free_noalloc": ([_P, _P, _P], _I),
    "dmb_nf_build": ([_P, _D, _I, _DP], _I),
    "dmb_nf_apply": ([_P, _DP, _DP, _L], _I),
    "dmb_rhs_plane_waves": ([_P, _DP, _DP, _DP, _L, _I, _DP], _I),
    "dmb_gmres": ([_P, _DP, _DP, _L, _D, _I, _I, _I, _I, ctypes.POINTER(GmresStats)], _I),
    "dmb_rhs_pattern_feed": ([_P, _I, _DP, _I, _DP, _DP, _DP, _D, _DP, _I, _I, _DP], _I),
    "dmb_gradient_impedance": ([_P, _L, _DP, _DP, _IP, _L, _I, _I, _DP], _I),
    "dmb_rhs_dipoles": ([_P, _L, _DP, _DP, _IP, _DP, _I, _DP], _I),
    "dmb_gmres_adjoint": ([_P, _DP, _DP, _L, _D, _I, _I, _I, _I, ctypes.POINTER(GmresStats)], _I),
    "dmb_solve_direct": ([_P, _DP, _DP, _L, _DP], _I),
    "dmb_farfield": ([_P, _DP, _L, _D, _D, _I, _DP, _L, _DP], _I),
    "dmb_local_build": ([_P, _D, _I], _I),
    "dmb_net_train": ([_P, _D, _I, _I, _D, ctypes.c_uint64, _DP], _I),
    "dmb_net_param_count": ([], _I),
    "dmb_net_get": ([_P, _FP], _I),
    "dmb_net_set": ([_P, _FP], _I),
    "dmb_net_loss_grad": ([_P, _FP, _FP, _FP, _IP, _L, _FP, _FP], _I),
    "dmb_solve_resident": ([_P, ctypes.POINTER(SolveParams), ctypes.POINTER(GmresStats)], _I),
    "dmb_solve_resident_many": ([_P, ctypes.POINTER(SolveParams), _L, _DP, _DP, _DP, _DP,
                                 ctypes.POINTER(GmresStats)], _I),
    "dmb_copy_solution": ([_P, _DP], _I),
    "dmb_get_stream": ([_P, ctypes.POINTER(ctypes.c_void_p)], _I),
    "dmb_set_kernel_timing": ([_P, _I], _I),
    "dmb_kernel_timing": ([_P, _DP, _LP, _DP], _I),
    "dmb_aca_plan": ([_DP, _L, _I, _D, _L, _LP, _LP, _LP, _DP, _LP, _LP, _L], _I),
    "dmb_aca_admissible": ([_DP, _DP, _D, ctypes.POINTER(ctypes.c_int)], _I),
    "dmb_aca_build": ([_P, _D, _D, _I, _I, _D, _D, _I, _L, _L, ctypes.POINTER(AcaInfo)], _I),
    "dmb_aca_matvec": ([_P, _DP, _DP, _L, _I], _I),
    "dmb_aca_blocks": ([_P, _LP], _I),
    "dmb_aca_block_data": ([_P, _L, _DP, _DP], _I),
    "dmb_aca_entries": ([_P, _LP, _LP, _L, _DP], _I),
    "dmb_aca_tree": ([_P, _LP, _DP], _I),
    "dmb_aca_lowrank": ([_P, _D, _D, _I, _LP, _L, _LP, _L, _D, _I, _L, _DP, _DP, _LP], _I),
    "dmb_aca_nf_build": ([_P, _I, _I, _DP], _I),
}


def check_free(lib, status: int):
    """Raise for a failed entry point that takes no context."""
    if status == DMB_OK:
        return
    msg = (lib.dmb_last_error(None) or b"").decode()
    raise _EXC.get(status, DiffMoMError)(msg or f"libdiffmom_b200 status {status}")

_lib = None


def load_library(path: os.PathLike | str | None = None):
    """Load and type the shared library (raises if it is absent)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path is not None else LIB_PATH
    if not p.exists():
        raise DiffMoMError(
            f"libdiffmom_b200.so not found at {p}; build it with "
            "`make -C diffmom.jl_b200/csrc` (there is no CPU fallback)")
    lib = ctypes.CDLL(str(p))
    for name, (args, res) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    if path is None:
        _lib = lib
    return lib


def dptr(a: np.ndarray):
    if a is None:
        return None
    return a.ctypes.data_as(_DP)


def iptr(a: np.ndarray):
    if a is None:
        return None
    return a.ctypes.data_as(_IP)


def lptr(a: np.ndarray):
    if a is None:
        return None
    return a.ctypes.data_as(_LP)


def c128(a) -> np.ndarray:
    """Contiguous complex128 copy/view in Julia's column-major layout."""
    return np.asfortranarray(np.asarray(a, dtype=np.complex128))


class Context:
    """Owns one dmb_ctx (device buffers, stream)."""

    def __init__(self, device: int = 0):
        self.lib = load_library()
        h = ctypes.c_void_p()
        self._check(self.lib.dmb_ctx_create(device, ctypes.byref(h)), None)
        self.h = h

    def _check(self, status: int, h=...):
        if status == DMB_OK:
            return
        handle = self.h if h is ... else h
        msg = (self.lib.dmb_last_error(handle) or b"").decode() if handle is not None else ""
        exc = _EXC.get(status, DiffMoMError)
        raise exc(msg or f"libdiffmom_b200 status {status}")

    def call(self, name: str, *args):
        self._check(getattr(self.lib, name)(self.h, *args))

    def timings(self) -> Timings:
        t = Timings()
        self.call("dmb_get_timings", ctypes.byref(t))
        return t

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            self.lib.dmb_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def declared_symbols() -> list[str]:
    """Function names declared in include/diffmom_b200.h."""
    import re
    text = HEADER_PATH.read_text()
    return sorted(set(re.findall(r"\b(dmb_[a-z_0-9]+)\s*\(", text)))
