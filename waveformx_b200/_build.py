"""Build the CUDA library in-tree: ``waveformx_b200/lib/libwaveformx_b200.so``
from ``csrc/kernels.cu``, for sm_100a only.

``python -m waveformx_b200._build`` (or ``__graft_entry__.build()``) runs
nvcc; the library is rebuilt when a source under ``csrc/`` or
``include/`` is newer than it.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PACKAGE = Path(__file__).resolve().parent
ROOT = PACKAGE.parent
SOURCE = PACKAGE / "csrc" / "kernels.cu"
LIBRARY = PACKAGE / "lib" / "libwaveformx_b200.so"

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-std=c++17", "-lineinfo",
    "-shared", "-Xcompiler", "-fPIC",
    "--expt-relaxed-constexpr",
]


def _nvcc() -> str:
    for candidate in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if candidate and Path(candidate).exists():
            return candidate
    raise FileNotFoundError("nvcc not found (set NVCC or add CUDA's bin to PATH)")


def _sources():
    return [p for d in (PACKAGE / "csrc", ROOT / "include") for p in d.glob("*") if p.suffix in (".cu", ".cuh", ".h")]


def stale() -> bool:
    """Whether the library is missing or older than a source."""
    if not LIBRARY.exists():
        return True
    built = LIBRARY.stat().st_mtime
    return any(p.stat().st_mtime > built for p in _sources())


def build(force: bool = False, verbose: bool = False) -> Path:
    """Compile the library (when stale, or always with ``force``)."""
    if not force and not stale():
        return LIBRARY
    LIBRARY.parent.mkdir(parents=True, exist_ok=True)
    tmp = LIBRARY.with_suffix(".so.tmp")
    cmd = [_nvcc(), *NVCC_FLAGS, "-o", str(tmp), str(SOURCE)]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
        print(" ".join(cmd), file=sys.stderr)
    subprocess.run(cmd, check=True, cwd=str(SOURCE.parent))
    os.replace(tmp, LIBRARY)
    return LIBRARY


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIBRARY)
