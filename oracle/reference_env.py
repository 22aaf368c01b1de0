"""Import the reference qepy-pw package with the oracle as its native module.

TEST INFRASTRUCTURE ONLY, like the rest of oracle/.  Used to generate golden fixtures and to pin the oracle against the
reference's own regression outputs (build container), and by the drop-in
test and ``bench.py --impl reference`` (GPU host).  The reference tree is
located through ``QEPY_REFERENCE_ROOT``, else the staged copy under
baseline/_ref (baseline/stage_reference.py; it travels with the repository
snapshot), else the read-only mount of the build container.
"""

from __future__ import annotations

import importlib
import os
import sys
from pathlib import Path

REPO = Path(__file__).resolve().parents[1]
STAGED_ROOT = REPO / "baseline" / "_ref"


def _locate() -> Path:
    if os.environ.get("QEPY_REFERENCE_ROOT"):
        return Path(os.environ["QEPY_REFERENCE_ROOT"])
    if (STAGED_ROOT / "qepy_pw" / "basis.py").is_file():
        return STAGED_ROOT
    return Path("/root/reference")


REFERENCE_ROOT = _locate()
# the full reference tree (its test inputs and recorded outputs); only the
# build container has it
SOURCE_ROOT = Path(os.environ.get("QEPY_REFERENCE_SOURCE", "/root/reference"))


def source_available() -> bool:
    return (SOURCE_ROOT / "tests" / "qe_reference").is_dir()


def reference_available() -> bool:
    return (REFERENCE_ROOT / "qepy_pw" / "basis.py").is_file()


def load_reference():
    """Return the ``qepy_pw`` package running on the NumPy oracle."""
    if not reference_available():
        raise RuntimeError(f"reference tree not found at {REFERENCE_ROOT}")
    os.environ.setdefault("PYTHONDONTWRITEBYTECODE", "1")
    sys.dont_write_bytecode = True
    if str(REPO) not in sys.path:
        sys.path.insert(0, str(REPO))
    if str(REFERENCE_ROOT) not in sys.path:
        sys.path.insert(0, str(REFERENCE_ROOT))
    oracle_native = importlib.import_module("oracle.native_fft")
    sys.modules["qepy_pw._native_fft"] = oracle_native
    package = importlib.import_module("qepy_pw")
    setattr(package, "_native_fft", oracle_native)
    return package
