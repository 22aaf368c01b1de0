"""Stage the reference qepy-pw package under baseline/_ref (git-ignored).

The reference's own install command

    python -m pip install --no-index --no-build-isolation --no-deps \
        --find-links /opt/wheelhouse --target baseline/_ref <reference tree>

fails in this image: its setup.py imports mpi4py at module level to build
the mandatory Cython/MPI/FFTW extension (no MPI, mpi4py or FFTW here).
This script first tries that command (from a temporary copy, since the
reference tree is read-only) and, when it fails, stages what the install
would have placed next to the extension: the package's pure-Python modules,
unmodified, under baseline/_ref/qepy_pw.  Its native module is then
supplied by the oracle (tests/golden/reference_env.py registers
oracle.native_fft as qepy_pw._native_fft).  baseline/_ref/STAGED.json
records how the tree was staged and the SHA-256 of every staged file.

The staged tree travels with the repository snapshot to the GPU host, where
the drop-in test runs the reference's own SCF driver with this package's
GPU classes bound in, and ``bench.py --impl reference`` times the
reference's own PlaneWaveHamiltonian.apply_into on the oracle.

Usage: python baseline/stage_reference.py [reference tree]
"""

from __future__ import annotations

import hashlib
import json
import os
import shutil
import subprocess
import sys
import tempfile
from pathlib import Path

HERE = Path(__file__).resolve().parent
TARGET = HERE / "_ref"


def try_pip(source: Path) -> tuple[bool, str]:
    with tempfile.TemporaryDirectory() as tmp:
        copy = Path(tmp) / "src"
        shutil.copytree(source, copy, ignore=shutil.ignore_patterns(".git", "__pycache__"))
        cmd = [sys.executable, "-m", "pip", "install", "--no-index", "--no-build-isolation",
               "--no-deps", "--find-links", "/opt/wheelhouse", "--target", str(TARGET), str(copy)]
        done = subprocess.run(cmd, capture_output=True, text=True)
    lines = [line.strip() for line in (done.stdout + done.stderr).splitlines() if line.strip()]
    reason = next((line for line in lines if "ModuleNotFoundError" in line or "No module" in line),
                  None) or next((line for line in reversed(lines) if "rror" in line),
                                lines[-1] if lines else "")
    return done.returncode == 0, reason


def stage(source: Path) -> dict:
    package = source / "qepy_pw"
    if not (package / "basis.py").is_file():
        raise SystemExit(f"no qepy_pw package under {source}")
    if TARGET.exists():
        shutil.rmtree(TARGET)
    TARGET.mkdir(parents=True)
    installed, reason = try_pip(source)
    record = {"source": str(source), "pip_install": "ok" if installed else "failed",
              "pip_error": None if installed else reason}
    if not installed:
        if TARGET.exists():
            shutil.rmtree(TARGET)
        files = {}
        for path in sorted(package.rglob("*.py")):
            rel = path.relative_to(source)
            out = TARGET / rel
            out.parent.mkdir(parents=True, exist_ok=True)
            shutil.copy2(path, out)
            files[str(rel)] = hashlib.sha256(path.read_bytes()).hexdigest()
        record["staged"] = "pure-Python modules of qepy_pw, unmodified"
        record["files"] = files
    (TARGET / "STAGED.json").write_text(json.dumps(record, indent=1))
    return record


if __name__ == "__main__":
    root = Path(sys.argv[1] if len(sys.argv) > 1 else
                os.environ.get("QEPY_REFERENCE_ROOT", "/root/reference"))
    result = stage(root)
    print(json.dumps({k: v for k, v in result.items() if k != "files"}, indent=1))
    print(f"{len(result.get('files', {}))} files staged under {TARGET}")
