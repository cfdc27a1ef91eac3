"""Compile the CPU oracle (``projector_oracle.c``, ``pointwise_oracle.c``) into
``oracle/_build/liboracle.so``.

TEST INFRASTRUCTURE ONLY.  ``-ffp-contract=off`` keeps every fused multiply-add
explicit so the oracle follows the same floating-point contract as the CUDA
kernels; ``-fopenmp`` parallelises over rays for the timed CPU baseline.
The target is x86-64-v3 (AVX2 + FMA) so the library also runs on the GPU hosts.
"""

from __future__ import annotations

import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
SOURCES = (HERE / "projector_oracle.c", HERE / "pointwise_oracle.c")
HEADER = HERE.parent / "include" / "dpt_b200.h"
LIBRARY = HERE / "_build" / "liboracle.so"


def build(force: bool = False) -> Path:
    """Build the oracle library if it is missing or older than its sources."""
    if (
        not force
        and LIBRARY.exists()
        and LIBRARY.stat().st_mtime >= max(path.stat().st_mtime for path in (*SOURCES, HEADER))
    ):
        return LIBRARY
    compiler = shutil.which("gcc") or shutil.which("cc")
    if compiler is None:
        raise RuntimeError("a C compiler is required to build the oracle")
    LIBRARY.parent.mkdir(parents=True, exist_ok=True)
    command = [
        compiler,
        "-O3",
        "-march=x86-64-v3",
        "-ffp-contract=off",
        "-fno-fast-math",
        "-fopenmp",
        "-fPIC",
        "-shared",
        "-std=c11",
        *(str(source) for source in SOURCES),
        "-o",
        str(LIBRARY),
        "-lm",
    ]
    result = subprocess.run(command, capture_output=True, text=True)
    if result.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{result.stdout}\n{result.stderr}")
    return LIBRARY


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
