"""ctypes binding of ``libqeb200.so`` (the C ABI of ``include/qe_b200.h``).

The library is the only compute path: when it is missing or no CUDA device
is visible, every entry point raises instead of falling back to the CPU.
"""

from __future__ import annotations

import ctypes
import os
import threading
from pathlib import Path

LIBRARY_PATH = Path(__file__).resolve().parent / "libqeb200.so"

QEB_F64 = 0
QEB_F32 = 1

STATUS_NAMES = {
    -1: "EINVAL",
    -2: "EUNSUPPORTED",
    -3: "ECUDA",
    -4: "ESCRATCH",
    -5: "ENOPLAN",
}

# (name, restype, argtypes) for every exported symbol of include/qe_b200.h.
_P = ctypes.c_void_p
_I = ctypes.c_int
_L = ctypes.c_int64
_D = ctypes.c_double
SIGNATURES: list[tuple[str, object, list]] = [
    ("qeb_last_error", ctypes.c_char_p, []),
    ("qeb_version", _I, []),
    ("qeb_launch_count", _L, []),
    ("qeb_qe_random_pairs", _I, [_L, _L, _P, _P, _P, _P, _P]),
    ("qeb_qe_random_draws", _I, [_L, _L, _P, _P, _P, _P, _P]),
    ("qeb_local_plan_create", _I, [ctypes.POINTER(_P), _I, _I, _I, _L, _P, _I]),
    ("qeb_local_plan_destroy", _I, [_P]),
    ("qeb_local_plan_info", _I, [_P, _P, _I]),
    ("qeb_local_scratch_bytes", _L, [_P, _L]),
    ("qeb_apply_local", _I, [_P, _P, _L, _P, _L, _L, _P, _P, _P, _L, _P]),
    ("qeb_apply_local_profiled", _I, [_P, _P, _L, _P, _L, _L, _P, _P, _P, _L, _P, _P]),
    ("qeb_accumulate_density", _I, [_P, _P, _L, _P, _L, _L, _P, _P, _P]),
    ("qeb_local_multi_scratch_bytes", _L, [_I, _P, _P]),
    ("qeb_apply_local_multi", _I, [_I, _P, _P, _L, _P, _P, _P, _P, _P, _P, _P, _P]),
    ("qeb_set_persistent_passes", _I, [_I]),
    ("qeb_persistent_passes", _I, []),
    ("qeb_zgemm_scratch_bytes", _L, [_I, _I, _I, _I, _I]),
    ("qeb_zgemm", _I, [_I, _I, _I, _I, _P, _P, _L, _P, _L, _P, _P, _L, _P, _L, _P]),
    ("qeb_cgemm", _I, [_I, _I, _I, _I, _P, _P, _L, _P, _L, _P, _P, _L, _P, _L, _P]),
    ("qeb_projector_basis", _I, [_L, _P, _P, _L, _I, _D, _I, _P, _P, _P, _P, _L, _P]),
    ("qeb_symmetrize_density", _I, [_I, _I, _I, _I, _P, _P, _P, _P, _P]),
    ("qeb_random_trials", _I, [_L, _L, _P, _P, _P, _P, _L, _I, _P]),
    ("qeb_zgemm_static_scratch_capacity", _L, []),
    ("qeb_zgemm_static_scratch", _I, [_I, _I, _I, _P, _P, _L, _P, _L, _P, _P, _L, _P]),
    ("qeb_block_coupling", _I, [_I, _I, _I, _I, _P, _P, _P, _P, _P, _P, _L, _P, _L, _P]),
    ("qeb_tf32_pack", _I, [_I, _I, _I, _I, _I, _P, _L, _P, _P, _L, _P]),
    ("qeb_tf32_gemm_scratch_bytes", _L, [_I, _I, _I]),
    ("qeb_tf32_gemm", _I, [_I, _I, _I, _P, _P, _L, _P, _P, _P, _P, _L, _P, _P, _P, _L, _P, _L,
                           _P]),
    ("qeb_tf32_gemm_error", _I, [_P]),
    ("qeb_cgemm_tf32x3_scratch_bytes", _L, [_I, _I, _I, _I]),
    ("qeb_cgemm_tf32x3", _I, [_I, _I, _I, _I, _P, _P, _L, _P, _L, _P, _P, _L, _P, _L, _P]),
    ("qeb_cgemm_tf32x3_default_splits", _I, [_I, _I, _I, _I]),
    ("qeb_cgemm_tf32x3_ex", _I, [_I, _I, _I, _I, _P, _P, _L, _P, _L, _P, _P, _L, _P, _L, _I, _P]),
    ("qeb_column_squared_norms", _I, [_I, _L, _L, _P, _L, _P, _P]),
    ("qeb_column_diagonal_expectations", _I, [_I, _L, _L, _P, _L, _P, _P, _P]),
    ("qeb_column_inner_products", _I, [_I, _L, _L, _P, _L, _P, _L, _P, _P]),
    ("qeb_precondition", _I, [_I, _L, _L, _P, _L, _P, _P, _P, _L, _P]),
    ("qeb_normalize_columns", _I, [_I, _L, _L, _P, _L, _P, _P, _P, _L, _P]),
    ("qeb_subtract_band_energies", _I, [_I, _L, _L, _P, _L, _P, _L, _P, _P]),
    ("qeb_accumulate_projector_diagonal", _I, [_I, _L, _L, _P, _L, _P, _L, _D, _P, _P]),
]


class NativeError(RuntimeError):
    """A qe_b200 entry point returned a failure status."""

    def __init__(self, function: str, status: int, message: str) -> None:
        self.status = status
        super().__init__(f"{function} failed ({STATUS_NAMES.get(status, status)}): {message}")


_LOCK = threading.Lock()
_HANDLE: ctypes.CDLL | None = None


def load(build_if_missing: bool = False) -> ctypes.CDLL:
    """Load (once) and return the CUDA library with typed signatures."""
    global _HANDLE
    if _HANDLE is not None:
        return _HANDLE
    with _LOCK:
        if _HANDLE is not None:
            return _HANDLE
        if not LIBRARY_PATH.exists():
            if build_if_missing or os.environ.get("QEB_BUILD_ON_IMPORT") == "1":
                from .build import build_library

                build_library()
            else:
                raise ImportError(
                    f"{LIBRARY_PATH.name} is not built; run `python -m qe_python_b200.build` "
                    "(there is no CPU fallback for the qe_b200 hot path)"
                )
        handle = ctypes.CDLL(str(LIBRARY_PATH))
        for name, restype, argtypes in SIGNATURES:
            function = getattr(handle, name)
            function.restype = restype
            function.argtypes = argtypes
        _HANDLE = handle
        return handle


def last_error() -> str:
    message = load().qeb_last_error()
    return message.decode(errors="replace") if message else ""


def check(function: str, status: int) -> None:
    if status != 0:
        raise NativeError(function, int(status), last_error())


def call(function: str, *args) -> int:
    status = getattr(load(), function)(*args)
    check(function, status)
    return status
