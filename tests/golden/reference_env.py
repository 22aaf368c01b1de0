"""Import the reference qepy-pw package with the oracle as its native module.

Used only in the build container to generate golden fixtures and to pin the
oracle against the reference's own regression outputs.  The reference tree
is located through ``QEPY_REFERENCE_ROOT`` (default: the read-only mount of
the build container).  Nothing on the GPU side imports this file.
"""

from __future__ import annotations

import importlib
import os
import sys
from pathlib import Path

REPO = Path(__file__).resolve().parents[2]
REFERENCE_ROOT = Path(os.environ.get("QEPY_REFERENCE_ROOT", "/root/reference"))


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
