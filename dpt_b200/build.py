"""Build the projector's CUDA library in-tree: ``dpt_b200/_lib/libdpt_b200.so``.

Each ``csrc/*.cu`` translation unit is compiled for sm_100a with nvcc and the
objects are linked into one shared library that exports the C ABI declared in
``include/dpt_b200.h``.  ``-fmad=false`` keeps every fused multiply-add explicit
(the arithmetic contract the kernels and the oracle share).

Run ``python -m dpt_b200.build`` (or ``__graft_entry__.build()``).
"""

from __future__ import annotations

import concurrent.futures
import os
import shutil
import subprocess
import sys
from pathlib import Path

PACKAGE = Path(__file__).resolve().parent
ROOT = PACKAGE.parent
SOURCES = sorted((PACKAGE / "csrc").glob("*.cu"))
HEADERS = sorted((PACKAGE / "csrc").glob("*.h")) + sorted((PACKAGE / "csrc").glob("*.cuh"))
HEADERS += [ROOT / "include" / "dpt_b200.h"]
BUILD = ROOT / "_build" / "dpt_b200"
LIBRARY = PACKAGE / "_lib" / "libdpt_b200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = [
    "-O3",
    "-std=c++17",
    "-lineinfo",
    "-fmad=false",
    "-Xcompiler",
    "-fPIC",
    "-Xcompiler",
    "-O3",
    "--expt-relaxed-constexpr",
]


def nvcc() -> str:
    found = shutil.which("nvcc")
    if found:
        return found
    candidate = Path("/usr/local/cuda/bin/nvcc")
    if candidate.exists():
        return str(candidate)
    raise RuntimeError("nvcc not found: the projector library needs the CUDA toolkit to build")


def _stale(target: Path, inputs: list[Path]) -> bool:
    if not target.exists():
        return True
    built = target.stat().st_mtime
    return any(path.stat().st_mtime > built for path in inputs)


def _compile(source: Path, verbose: bool) -> Path:
    obj = BUILD / (source.stem + ".o")
    if not _stale(obj, [source, *HEADERS]):
        return obj
    command = [nvcc(), *ARCH, *FLAGS, "-c", str(source), "-o", str(obj)]
    if verbose:
        command += ["-Xptxas", "-v"]
    result = subprocess.run(command, capture_output=True, text=True)
    if result.returncode != 0:
        raise RuntimeError(f"nvcc failed for {source.name}:\n{result.stdout}\n{result.stderr}")
    if verbose and result.stderr:
        sys.stderr.write(result.stderr)
    return obj


def build(verbose: bool = False) -> Path:
    """Compile every translation unit and link the shared library; return its path."""
    BUILD.mkdir(parents=True, exist_ok=True)
    LIBRARY.parent.mkdir(parents=True, exist_ok=True)
    workers = max(1, min(len(SOURCES), os.cpu_count() or 1))
    with concurrent.futures.ThreadPoolExecutor(workers) as pool:
        objects = list(pool.map(lambda source: _compile(source, verbose), SOURCES))
    if _stale(LIBRARY, objects):
        command = [nvcc(), *ARCH, "-shared", "-o", str(LIBRARY), *map(str, objects), "-lcudart"]
        result = subprocess.run(command, capture_output=True, text=True)
        if result.returncode != 0:
            raise RuntimeError(f"linking {LIBRARY.name} failed:\n{result.stdout}\n{result.stderr}")
    return LIBRARY


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
