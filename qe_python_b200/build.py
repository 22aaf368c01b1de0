"""Compile the sm_100a CUDA library ``libqeb200.so`` in-tree with nvcc.

The shared library holds every kernel of the hot path and the C ABI declared
in ``include/qe_b200.h``.  It is built next to this file so that it travels
with the source tree; nothing is installed into site-packages.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PACKAGE = Path(__file__).resolve().parent
REPO = PACKAGE.parent
CSRC = PACKAGE / "csrc"
INCLUDE = REPO / "include"
LIBRARY = PACKAGE / "libqeb200.so"
BUILD_DIR = REPO / "_build"

ARCH_FLAGS = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON_FLAGS = [
    "-O3",
    "-lineinfo",
    "-std=c++17",
    "--expt-relaxed-constexpr",
    "-Xcompiler",
    "-fPIC",
]


def nvcc_path() -> str:
    candidates = [
        os.environ.get("NVCC"),
        shutil.which("nvcc"),
        "/usr/local/cuda/bin/nvcc",
    ]
    for candidate in candidates:
        if candidate and Path(candidate).exists():
            return candidate
    raise RuntimeError("nvcc not found; the CUDA toolkit is required to build qe_b200")


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def _stale() -> bool:
    if not LIBRARY.exists():
        return True
    built = LIBRARY.stat().st_mtime
    inputs = list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cuh")) + list(INCLUDE.glob("*.h"))
    return any(path.stat().st_mtime > built for path in inputs)


def build_library(force: bool = False, verbose: bool = False, jobs: int | None = None) -> Path:
    """Compile each ``csrc/*.cu`` to an object, then link ``libqeb200.so``."""
    if not force and not _stale():
        return LIBRARY
    nvcc = nvcc_path()
    BUILD_DIR.mkdir(exist_ok=True)
    objects = []
    processes = []
    for source in sources():
        obj = BUILD_DIR / (source.stem + ".o")
        objects.append(obj)
        cmd = [nvcc, *ARCH_FLAGS, *COMMON_FLAGS, f"-I{INCLUDE}", f"-I{CSRC}",
               "-c", str(source), "-o", str(obj)]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
            print(" ".join(cmd), file=sys.stderr)
        processes.append((source, subprocess.Popen(cmd, stdout=subprocess.PIPE,
                                                   stderr=subprocess.STDOUT, text=True)))
        limit = jobs or os.cpu_count() or 4
        while sum(p.poll() is None for _, p in processes) >= limit:
            processes[0][1].wait(timeout=600)
            break
    failures = []
    for source, process in processes:
        output, _ = process.communicate()
        if verbose and output:
            print(output, file=sys.stderr)
        if process.returncode != 0:
            failures.append(f"{source.name}:\n{output}")
    if failures:
        raise RuntimeError("nvcc failed:\n" + "\n".join(failures))
    tmp = LIBRARY.with_suffix(".so.tmp")
    link = [nvcc, *ARCH_FLAGS, "-shared", "-o", str(tmp), *map(str, objects), "-lcudart"]
    result = subprocess.run(link, capture_output=True, text=True)
    if result.returncode != 0:
        raise RuntimeError("nvcc link failed:\n" + result.stdout + result.stderr)
    os.replace(tmp, LIBRARY)
    return LIBRARY


if __name__ == "__main__":
    build_library(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIBRARY)
