"""ctypes binding of the C ABI in ``include/ssn.h`` (``libssn.so``).

This is the only route from Python to the compute path: there is no CPU or
library fallback.  Loading fails loudly when the library is missing, and every
compute call requires CUDA float64 tensors on one device.  Arguments are raw
device pointers and sizes; kernels run on torch's current CUDA stream.
"""
from __future__ import annotations

import ctypes
from pathlib import Path

import torch

LIB_PATH = Path(__file__).resolve().parent / "libssn.so"

_P = ctypes.c_void_p
_I = ctypes.c_int
_I64 = ctypes.c_int64
_SZ = ctypes.c_size_t

# name: (restype, argtypes) -- mirrors include/ssn.h
PROTOTYPES = {
    "ssn_version": (_I, []),
    "ssn_status_string": (ctypes.c_char_p, [_I]),
    "ssn_default_options": (None, [_P]),
    "ssn_workspace_bytes": (_SZ, [_I, _I, _I]),
    "ssn_solve": (_I, [_P, _P, _P, _P, _P, _I, _I, _I, _P, _SZ, _P, _P]),
    "ssn_ragged_workspace_bytes": (_SZ, [_I, _P, _P]),
    "ssn_solve_ragged": (_I, [_P, _P, _P, _P, _P, _I, _P, _P, _P, _P, _P, _SZ, _P, _P]),
    "ssn_adjoint_workspace_bytes": (_SZ, [_I, _I, _I]),
    "ssn_adjoint": (_I, [_P, _P, _P, _P, _P, _P, _P, _I, _I, _I, _P, _SZ, _P, _P]),
    "ssn_gram_workspace_bytes": (_SZ, [_I, _I, _I]),
    "ssn_gram": (_I, [_P, _P, _I64, _P, _P, _I, _I, _I, _P, _SZ, _P, _P]),
    "ssn_gram_noalloc_scratch_bytes": (_SZ, []),
    "ssn_gram_noalloc": (_I, [_P, _P, _I64, _P, _P, _I, _I, _I, _P]),
    "ssn_cross_gram_workspace_bytes": (_SZ, [_I, _I, _I]),
    "ssn_cross_gram": (_I, [_P, _P, _I64, _P, _P, _I64, _P, _P, _I, _I, _I, _P, _SZ, _P]),
    "ssn_recover_workspace_bytes": (_SZ, [_I, _I, _I]),
    "ssn_recover": (_I, [_P, _P, _I64, _P, _P, _P, _P, _I64, _I, _I, _I, _P, _SZ, _P, _P]),
    "ssn_eigh_workspace_bytes": (_SZ, [_I, _I]),
    "ssn_eigh": (_I, [_P, _P, _P, _P, _P, _I, _I, _P, _SZ, _P, _P]),
    "ssn_dual_workspace_bytes": (_SZ, [_I, _I]),
    "ssn_dual": (_I, [_P, _P, _P, _P, _P, _P, _P, _I, _I, _P, _SZ, _P, _P]),
    "ssn_newton_workspace_bytes": (_SZ, [_I, _I]),
    "ssn_newton": (_I, [_P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _P, _I, _I, _P, _SZ, _P, _P]),
    "ssn_set_newton_events": (_I, [_P]),
    "ssn_probe_fp64_mma": (_I, [_P, _I, _P, _P]),
    "ssn_probe_s8_mma": (_I, [_P, _P, _P, _I, _I, _P, _P]),
    "ssn_inner_products": (_I, [_P, _P, _P, _P, _P, _I, _I, _P]),
    "ssn_outer_skew": (_I, [_P, _P, _P, _P, _P, _I, _I, _P]),
    "ssn_sandwich_front": (_I, [_P, _P, _P, _P, _P, _P, _I, _I, _P]),
    "ssn_line_change": (_I, [_P, _P, _P, _P, _P, _P, _P, _I, _I, _P]),
    "ssn_precondition": (_I, [_P, _P, _P, _I, _I, _P]),
    "ssn_cg_update": (_I, [_P, _P, _P, _P, _P, _P, _P, _I, _I, _P]),
    "ssn_cg_next": (_I, [_P, _P, _P, _P, _P, _I, _I, _P]),
    "ssn_inverse_from_cholesky": (_I, [_P, _P, _I, _I, _P]),
    "ssn_spd_inverse": (_I, [_P, _P, _P, _I, _I, _P]),
    "ssn_cholesky_k": (_I, [_P, _P, _P, _I, _I, _P]),
    "ssn_set_tuning": (_I, [_P, _I]),
    "ssn_get_tuning": (_I, [_P, _I]),
}

SSN_OK = 0
STATUS_NAMES = {0: "converged", 1: "invalid argument", 2: "CUDA error", 3: "Newton cap",
                4: "line search", 5: "non-finite", 6: "eigh", 7: "workspace", 8: "scratch limit"}


class Options(ctypes.Structure):
    """ssn_options (include/ssn.h)."""
    _fields_ = [("max_newton", ctypes.c_int), ("max_cg", ctypes.c_int),
                ("max_backtrack", ctypes.c_int), ("feas_tol", ctypes.c_double),
                ("precision", ctypes.c_int), ("eig_sweeps", ctypes.c_int),
                ("preconditioner", ctypes.c_int), ("fp32_newton", ctypes.c_int),
                ("reserved", ctypes.c_int * 4)]


class Tuning(ctypes.Structure):
    """ssn_tuning (include/ssn.h): launch parameters for one problem class; 0 = built-in rule."""
    _fields_ = [("precision", ctypes.c_int), ("m", ctypes.c_int), ("n_min", ctypes.c_int),
                ("n_max", ctypes.c_int), ("batch_min", ctypes.c_int), ("batch_max", ctypes.c_int),
                ("gram_splits", ctypes.c_int), ("gram_chunks", ctypes.c_int),
                ("recover_parts", ctypes.c_int), ("cluster", ctypes.c_int)]


# ssn_options.precision / .preconditioner values (include/ssn.h)
PRECISIONS = {"fp64": 0, "split": 1}
PRECONDITIONERS = {"eigenbasis": 0, "adaptive": 1}


_lib = None


def load() -> ctypes.CDLL:
    """Load libssn.so once; raise if it is absent (no fallback path exists)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(
                f"native library {LIB_PATH} is missing; build it with "
                "`python -c 'import __graft_entry__ as g; g.build()'` (nvcc, sm_100a)")
        lib = ctypes.CDLL(str(LIB_PATH))
        for name, (res, args) in PROTOTYPES.items():
            fn = getattr(lib, name)
            fn.restype = res
            fn.argtypes = args
        _lib = lib
        from . import autotune
        autotune.load()        # the committed per-(n, k) table, when present
    return _lib


def options(max_newton=100, max_cg=150, max_backtrack=40, feas_tol=1e-8, precision="fp64",
            eig_sweeps=0, preconditioner="eigenbasis", fp32_newton=True) -> Options:
    """ssn_options; fp32_newton (split form only): early Newton steps in FP32 (default) or all FP64."""
    if precision not in PRECISIONS:
        raise ValueError(f"precision must be one of {sorted(PRECISIONS)}")
    if preconditioner not in PRECONDITIONERS:
        raise ValueError(f"preconditioner must be one of {sorted(PRECONDITIONERS)}")
    opt = Options()
    load().ssn_default_options(ctypes.byref(opt))
    opt.max_newton, opt.max_cg, opt.max_backtrack, opt.feas_tol = max_newton, max_cg, max_backtrack, feas_tol
    opt.precision, opt.eig_sweeps = PRECISIONS[precision], eig_sweeps
    opt.preconditioner = PRECONDITIONERS[preconditioner]
    opt.fp32_newton = 0 if fp32_newton else -1
    return opt


def check(code: int, what: str) -> None:
    if code != SSN_OK:
        msg = load().ssn_status_string(code).decode()
        raise RuntimeError(f"{what}: {msg} (status {code})")


def ptr(t: torch.Tensor | None) -> int | None:
    return None if t is None else t.data_ptr()


def stream_handle(device: torch.device) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def row_halves(A: torch.Tensor, D: torch.Tensor):
    """(A, D, batch stride) for a pair of [batch, rows, m] operands of one kernel call.

    The C ABI takes both halves with one batch stride and densely packed rows, as
    the two halves T[:, :n] and T[:, n:] of a target batch are; such views pass
    without a copy.  Other layouts are made contiguous.
    """
    batch, rows, m = A.shape

    def packed(x):
        return x.stride(2) == 1 and x.stride(1) == m and x.data_ptr() % 16 == 0

    if packed(A) and packed(D):
        stride = rows * m if batch == 1 else A.stride(0)
        if (batch == 1 or D.stride(0) == stride) and stride >= rows * m and stride % 2 == 0:
            return A, D, stride
    return A.contiguous(), D.contiguous(), rows * m


def require_cuda_f64(*tensors: torch.Tensor) -> torch.device:
    dev = tensors[0].device
    for t in tensors:
        if not isinstance(t, torch.Tensor) or not t.is_cuda or t.dtype != torch.float64 or t.device != dev:
            raise ValueError("expected CUDA float64 tensors on one device")
    return dev
