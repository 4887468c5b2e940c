"""The oracle's C restatement (``oracle/xas_eval.c``, built by
``oracle/Makefile`` into ``oracle/_build/liboracle.so``), bound with ctypes.
Test infrastructure, as the rest of ``oracle/``."""

from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIBRARY = HERE / "_build" / "liboracle.so"
_lib = None


def build(force: bool = False) -> Path:
    """Compile the C restatement (make) when it is missing or older than its source."""
    source = HERE / "xas_eval.c"
    if force or not LIBRARY.exists() or LIBRARY.stat().st_mtime < source.stat().st_mtime:
        subprocess.run(["make", "-s", "-C", str(HERE), "-B" if force else "_build/liboracle.so"], check=True)
    return LIBRARY


def library() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        build()
        lib = ctypes.CDLL(str(LIBRARY))
        lib.oracle_xas_evaluate.restype = ctypes.c_int
        lib.oracle_xas_evaluate.argtypes = [ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p, ctypes.c_int64,
                                            ctypes.c_int64, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
        _lib = lib
    return _lib


def xas_evaluate(flat_table, frequencies, threads: int = 0):
    """``(hplus, hcross)`` complex128 ``(B, N)`` of IMRPhenomXAS from the
    reference's flat tables ``(B, 86)`` at ``frequencies`` (``(N,)`` shared
    or ``(B, N)``), on ``threads`` OpenMP threads (0: all)."""
    tab = np.ascontiguousarray(np.atleast_2d(flat_table), dtype=np.float64)
    f = np.ascontiguousarray(frequencies, dtype=np.float64)
    b = tab.shape[0]
    n = f.shape[-1]
    stride = 0 if f.ndim == 1 else n
    hp = np.empty((b, n), dtype=np.complex128)
    hc = np.empty((b, n), dtype=np.complex128)
    rc = library().oracle_xas_evaluate(tab.ctypes.data, b, f.ctypes.data, n, stride, hp.ctypes.data, hc.ctypes.data,
                                       int(threads))
    if rc != 0:
        raise MemoryError("oracle_xas_evaluate")
    return hp, hc


def xas_polarizations(params, frequencies, threads: int = 0):
    """The whole path for ``params`` ``(B, 8)``: the NumPy oracle's table
    (vectorised over binaries), then the C evaluation."""
    from . import xas

    f = np.asarray(frequencies, dtype=np.float64)
    tab = xas.table(params, f[..., 0])
    return xas_evaluate(xas.flat(tab), f, threads)


def cores() -> int:
    """The host cores this process may use."""
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1
