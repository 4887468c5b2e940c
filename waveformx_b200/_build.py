"""Build the CUDA library in-tree: ``waveformx_b200/lib/libwaveformx_b200.so``
from ``csrc/kernels.cu`` (the frequency kernels), ``csrc/setup.cu`` (the
per-binary set-up, compiled without FMA contraction) and ``csrc/match.cu``
(the matches), for sm_100a only.

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
LIBRARY = PACKAGE / "lib" / "libwaveformx_b200.so"

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-O3", "-std=c++17", "-lineinfo",
    "-Xcompiler", "-fPIC",
    "--expt-relaxed-constexpr",
]
#: The translation units and their own flags.
UNITS = {
    "kernels.cu": [],
    "setup.cu": ["-fmad=false"],
    "match.cu": [],
    "xhm.cu": [],
    "pipeline.cu": [],
}


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
    """Compile the library (when stale, or always with ``force``): the
    translation units in parallel, then one shared link."""
    if not force and not stale():
        return LIBRARY
    LIBRARY.parent.mkdir(parents=True, exist_ok=True)
    nvcc = _nvcc()
    objects, jobs = [], []
    for unit, flags in UNITS.items():
        obj = LIBRARY.parent / (Path(unit).stem + ".o")
        cmd = [nvcc, *NVCC_FLAGS, *flags, "-c", "-o", str(obj), str(PACKAGE / "csrc" / unit)]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
            print(" ".join(cmd), file=sys.stderr)
        jobs.append(subprocess.Popen(cmd, cwd=str(PACKAGE / "csrc")))
        objects.append(obj)
    failed = [job.args for job in jobs if job.wait() != 0]
    if failed:
        raise subprocess.CalledProcessError(1, failed[0])
    tmp = LIBRARY.with_suffix(".so.tmp")
    subprocess.run([nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-shared", "-o", str(tmp),
                    *map(str, objects)], check=True)
    os.replace(tmp, LIBRARY)
    return LIBRARY


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(LIBRARY)
