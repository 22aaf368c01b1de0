"""The C ABI library loads and exports every function include/qe_b200.h declares.

CPU-only: symbols are resolved with ctypes; nothing is launched.
"""

from __future__ import annotations

import ctypes
import re
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parents[1]
HEADER = REPO / "include" / "qe_b200.h"


def declared_functions() -> list[str]:
    text = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return sorted(set(re.findall(r"\b(qeb_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def library():
    from qe_python_b200.build import build_library

    path = build_library()
    return ctypes.CDLL(str(path))


def test_header_declares_the_hot_path(library):
    names = declared_functions()
    for required in ("qeb_local_plan_create", "qeb_apply_local", "qeb_accumulate_density",
                     "qeb_zgemm", "qeb_precondition", "qeb_column_squared_norms"):
        assert required in names


def test_every_declared_function_is_exported(library):
    missing = [name for name in declared_functions() if not hasattr(library, name)]
    assert not missing, f"symbols declared but not exported: {missing}"


def test_python_binding_covers_the_header():
    from qe_python_b200._lib import SIGNATURES

    bound = {name for name, _r, _a in SIGNATURES}
    assert set(declared_functions()) <= bound


def test_version_and_error_calls_need_no_gpu(library):
    from qe_python_b200 import _lib

    handle = _lib.load()
    assert handle.qeb_version() == 1
    assert isinstance(_lib.last_error(), str)
    # argument validation happens before any CUDA call
    plan = ctypes.c_void_p()
    status = handle.qeb_local_plan_create(ctypes.byref(plan), 0, 4, 4, 1, None, 0)
    assert status == -1
    assert "invalid grid" in _lib.last_error()


def test_setup_entry_points_validate_before_any_launch(library):
    """The projector-basis and symmetrisation entry points refuse bad
    arguments with a status and a message, without touching a GPU."""
    from qe_python_b200 import _lib

    handle = _lib.load()
    ints = (ctypes.c_int * 3)(0, 0, 0)
    # a radial table of fewer than four rows cannot be interpolated
    status = handle.qeb_projector_basis(10, 1, 1, 3, 1, 0.01, 1, ints, ints, ints, 1, 10, None)
    assert status == -1 and "invalid arguments" in _lib.last_error()
    # l = 3 channels are outside the harmonics this library tabulates
    bad_l = (ctypes.c_int * 1)(3)
    status = handle.qeb_projector_basis(10, 1, 1, 8, 1, 0.01, 1, ints, bad_l, ints, 1, 10, None)
    assert status == -1 and "channel 0" in _lib.last_error()
    offsets = (ctypes.c_int * (3 * 97))()
    coefficients = (ctypes.c_int * (9 * 97))()
    status = handle.qeb_symmetrize_density(4, 4, 4, 97, offsets, coefficients, 1, 2, None)
    assert status == -2 and "operations exceed" in _lib.last_error()
    status = handle.qeb_symmetrize_density(4, 4, 4, 2, offsets, coefficients, 1, 1, None)
    assert status == -1 and "must differ" in _lib.last_error()
