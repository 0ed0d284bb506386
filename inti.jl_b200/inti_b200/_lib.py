"""ctypes binding of libinti_b200.so (declarations: include/inti_b200.h).

The shared library is the product; this module only declares argument types
and turns non-zero statuses into Python exceptions that mirror the Julia side:
``ArgumentError`` (invalid argument), ``DimensionMismatch`` (shapes) and
``Inti B200Error`` subclasses for device-side failures.  There is no fallback:
if the library is missing or no CUDA device is present the import of the
operator layer fails loudly.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

_HERE = Path(__file__).resolve().parent
LIB_PATH = Path(os.environ.get("INTI_B200_LIB", _HERE.parent / "_build" / "libinti_b200.so"))

OK, E_ARG, E_SHAPE, E_CUDA, E_NONFINITE, E_TIMEOUT, E_NOMEM, E_UNSUPPORTED, E_NOCONV, E_STATE = range(10)
LAPLACE, HELMHOLTZ = 0, 1
SL, DL, ADL, HS = 0, 1, 2, 3
FP64, FP32C, TF32 = 0, 1, 2
CF = 4
F64, C128 = 0, 1
H2D, D2H, D2D = 0, 1, 2
GMRES_FP64, GMRES_MIXED = 0, 1


class InticError(RuntimeError):
    """Failure reported by libinti_b200 (status code in ``.code``)."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class ArgumentError(InticError, ValueError):
    """Invalid argument (Julia's ArgumentError)."""


class DimensionMismatch(InticError, ValueError):
    """Incompatible sizes (Julia's DimensionMismatch)."""


class NonFiniteError(InticError, ValueError):
    """NaN or Inf in an input."""


class UnsupportedError(InticError, NotImplementedError):
    """A combination the library does not implement."""


class DeviceError(InticError):
    """CUDA failure, device allocation failure or a bounded device wait that ran out."""


_EXC = {
    E_ARG: ArgumentError,
    E_SHAPE: DimensionMismatch,
    E_NONFINITE: NonFiniteError,
    E_UNSUPPORTED: UnsupportedError,
    E_STATE: ArgumentError,
}


class GmresStats(C.Structure):
    _fields_ = [
        ("iterations", C.c_int32),
        ("outer", C.c_int32),
        ("fp64_applies", C.c_int32),
        ("fp32_applies", C.c_int32),
        ("converged", C.c_int32),
        ("reserved", C.c_int32),
        ("relres", C.c_double),
        ("seconds", C.c_double),
        ("setup_seconds", C.c_double),
    ]

    def as_dict(self) -> dict:
        return {f: getattr(self, f) for f, _ in self._fields_ if f != "reserved"}


P = C.c_void_p
PP = C.POINTER(C.c_void_p)
D = C.POINTER(C.c_double)
I64 = C.c_int64

# name: (restype, argtypes)
SIGNATURES = {
    "inti_version": (C.c_int, []),
    "inti_ctx_create": (C.c_int, [C.c_int, P, PP]),
    "inti_ctx_destroy": (C.c_int, [P]),
    "inti_last_error": (C.c_char_p, [P]),
    "inti_ctx_synchronize": (C.c_int, [P]),
    "inti_ctx_stream": (P, [P]),
    "inti_ctx_launch_count": (I64, [P]),
    "inti_ctx_set_profiling": (C.c_int, [P, C.c_int]),
    "inti_ctx_profile": (C.c_int, [P, C.c_char_p, D, C.POINTER(I64)]),
    "inti_dev_alloc": (C.c_int, [P, I64, PP]),
    "inti_dev_free": (C.c_int, [P, P]),
    "inti_memcpy": (C.c_int, [P, P, P, I64, C.c_int]),
    "inti_quad_create": (C.c_int, [P, C.c_int, I64, P, P, P, C.c_int32, PP]),
    "inti_quad_destroy": (C.c_int, [P]),
    "inti_quad_size": (I64, [P]),
    "inti_csr_create": (C.c_int, [P, I64, I64, I64, P, P, P, C.c_int, PP]),
    "inti_csr_create_from_csc": (C.c_int, [P, I64, I64, I64, P, P, P, C.c_int, PP]),
    "inti_csr_info": (C.c_int, [P, C.POINTER(I64), C.POINTER(I64), C.POINTER(I64), C.POINTER(C.c_int)]),
    "inti_csr_download": (C.c_int, [P, P, P, P]),
    "inti_csr_apply": (C.c_int, [P, P, P, D, D, C.c_int]),
    "inti_csr_destroy": (C.c_int, [P]),
    "inti_op_create": (C.c_int, [P, C.c_int, C.c_int, C.c_double, C.c_double, P, P, P, C.c_int, PP]),
    "inti_op_create_combined": (C.c_int, [P, C.c_int, C.c_double, C.c_double, P, P, P, P, D, D, C.c_int, PP]),
    "inti_op_info": (C.c_int, [P, C.POINTER(I64), C.POINTER(I64), C.POINTER(C.c_int)]),
    "inti_op_apply": (C.c_int, [P, P, I64, P, I64, C.c_int32, D, D, C.c_int]),
    "inti_op_apply_transpose": (C.c_int, [P, P, I64, P, I64, C.c_int32, D, D, C.c_int]),
    "inti_op_assemble": (C.c_int, [P, P, C.c_int]),
    "inti_op_destroy": (C.c_int, [P]),
    "inti_dim_correction": (C.c_int, [P, C.c_int, C.c_double, C.c_double, P, C.c_int, P, PP, PP]),
    "inti_dim_correction_targets": (C.c_int, [P, C.c_int, C.c_double, C.c_double, P, P, C.c_int, P, C.c_double,
                                              PP, PP]),
    "inti_gmres": (C.c_int, [P, C.c_int32, PP, D, D, P, P, C.c_double, C.c_int32, C.c_int32,
                             C.c_int32, C.c_int, P, C.POINTER(GmresStats)]),
    "inti_op_grad_sources": (C.c_int, [P, P, P, P, P, P, P, C.c_int]),
    "inti_measure_peaks": (C.c_int, [P, D, D, D]),
    "inti_measure_peak_tf32": (C.c_int, [P, D]),
    "inti_op_tuning": (C.c_int, [P, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]),
    "inti_ctx_set_autotune": (C.c_int, [P, C.c_int]),
    "inti_ctx_set_symmetric": (C.c_int, [P, C.c_int]),
    "inti_op_symmetric": (C.c_int, [P]),
    "inti_ctx_set_partial_budget": (C.c_int, [P, C.c_double]),
    "inti_op_panels": (C.c_int, [P]),
    "inti_ctx_set_single_launch": (C.c_int, [P, C.c_int]),
    "inti_ctx_set_gmres_small": (C.c_int, [P, I64]),
    "inti_op_single_launch": (C.c_int, [P]),
    "inti_op_set_shard": (C.c_int, [P, C.c_int, C.c_int]),
    "inti_selftest_math": (C.c_int, [P, D]),
    "inti_selftest_wait_timeout": (C.c_int, [P]),
    "inti_batch_create": (C.c_int, [P, C.c_int32, PP, C.c_int, C.c_int, C.c_double, C.c_double, D, D, PP, PP, PP]),
    "inti_batch_apply": (C.c_int, [P, C.c_int, P, I64, P, I64, C.c_int32, D, D, C.c_int]),
    "inti_batch_gmres": (C.c_int, [P, D, P, P, I64, C.c_int32, C.c_double, C.c_int32, C.c_int32, C.c_int32, C.c_int,
                                    P, C.POINTER(GmresStats)]),
    "inti_batch_size": (I64, [P]),
    "inti_batch_destroy": (C.c_int, [P]),
    "inti_apply_noalloc": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_double, C.c_int, I64, P, P, I64, P, P, P,
                                     P, P, P, P, P, D, D, P, C.c_int]),
}

_lib = None


def load(path: str | os.PathLike | None = None) -> C.CDLL:
    """Load (once) and declare the library.  Raises OSError if it is absent."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise OSError(f"libinti_b200.so not found at {p}; run inti.jl_b200/build.py")
    lib = C.CDLL(str(p))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def check(status: int, ctx_handle=None) -> None:
    if status == OK:
        return
    lib = load()
    msg = lib.inti_last_error(ctx_handle)
    msg = msg.decode() if msg else "unknown error"
    raise _EXC.get(status, DeviceError)(status, msg)


def dptr(a) -> int | None:
    """Address of a contiguous numpy array (or None)."""
    if a is None:
        return None
    return a.ctypes.data


_ONE = (C.c_double * 2)(1.0, 0.0)
_ZERO = (C.c_double * 2)(0.0, 0.0)


def cpair(z) -> C.Array:
    """A complex scalar as the (re, im) double pair the ABI takes (the ABI
    only reads it, so 1 and 0 share one array each)."""
    if z == 1:
        return _ONE
    if z == 0:
        return _ZERO
    z = complex(z)
    return (C.c_double * 2)(z.real, z.imag)
