"""The ctypes binding of the C ABI (``include/waveformx_b200.h``).

The library is the in-tree ``lib/libwaveformx_b200.so`` (``_build.py``). It
is loaded on first use; without it (or without a CUDA device) every entry
raises :class:`~waveformx_b200.exceptions.KernelError`: there is no CPU
fallback.
"""

from __future__ import annotations

import ctypes
import threading

from . import _build
from .exceptions import KernelError

__all__ = ["library", "check", "XAS", "PHENOMD", "TAYLORF2", "XHM", "FP64", "FP32", "TABLE_STRIDE", "GRAD_COLUMNS",
           "XHM_STRIDE64", "XHM_STRIDE32", "XHM_MODES", "OP_VJP",
           "OP_FUSED", "OP_POLARIZATIONS", "EXPORTS", "STATIC_SCRATCH_BYTES", "ESCRATCH",
           "EOFFSETS", "EINVAL", "EWORKSPACE"]

XAS, PHENOMD, TAYLORF2, XHM = 0, 1, 2, 3
FP64, FP32 = 0, 1
TABLE_STRIDE = 72
XHM_STRIDE64, XHM_STRIDE32, XHM_MODES = 544, 576, 5
GRAD_COLUMNS = 9
OP_VJP, OP_FUSED, OP_POLARIZATIONS = 0, 1, 2

_P = ctypes.c_void_p
_I64 = ctypes.c_int64
_D = ctypes.c_double
_INT = ctypes.c_int

#: name -> (restype, argtypes) of every entry point of the header.
EXPORTS = {
    "wfx_version": (_INT, []),
    "wfx_pipeline_create": (_INT, [ctypes.POINTER(ctypes.c_void_p)]),
    "wfx_pipeline_destroy": (_INT, [_P]),
    "wfx_pipeline_setup": (_INT, [_P, _INT, _INT, _P, _I64, _P, _I64, _D, _D, _P, _P, _P, _P]),
    "wfx_pipeline_forward": (_INT, [_P, _INT, _INT, _INT, _P, _P, _P, _I64, _I64, _I64, _P, _P, _P, _P,
                                    ctypes.c_size_t, _P]),
    "wfx_pipeline_join": (_INT, [_P, _P]),
    "wfx_pipeline_run": (_INT, [_P, _INT, _INT, _I64, _P, _I64, _P, _I64, _D, _D, _P, _P, _P, _P, _I64, _I64, _P,
                                _P, _P, _I64, _I64, _P, ctypes.c_size_t, _P]),
    "wfx_pipeline_setup_jvp": (_INT, [_P, _INT, _INT, _P, _I64, _P, _I64, _D, _D, _P, _P]),
    "wfx_pipeline_fused": (_INT, [_P, _INT, _INT, _P, _P, _P, _I64, _I64, _P, _P, _INT, _P, _INT, _D, _D, _D, _P,
                                  _P, _P, _P, ctypes.c_size_t, _P]),
    "wfx_pipeline_likelihood_run": (_INT, [_P, _INT, _I64, _P, _I64, _P, _I64, _D, _D, _P, _P, _P, _P, _P, _I64,
                                           _P, _P, _INT, _P, _INT, _D, _D, _D, _P, _P, _I64, _P, ctypes.c_size_t,
                                           _P]),
    "wfx_status_string": (ctypes.c_char_p, [_INT]),
    "wfx_setup": (_INT, [_INT, _P, _I64, _P, _I64, _D, _D, _P, _P, _P, _P]),
    "wfx_setup_jvp": (_INT, [_INT, _P, _I64, _P, _I64, _D, _D, _P, _P, _P, _P, _P]),
    "wfx_polarizations": (_INT, [_INT, _INT, _P, _P, _P, _I64, _I64, _P, _P, _P, _P, ctypes.c_size_t, _P]),
    "wfx_workspace_bytes": (ctypes.c_size_t, [_INT, _INT, _INT, _I64, _I64, _INT]),
    "wfx_ragged_status": (_INT, [_P, _P]),
    "wfx_vjp": (_INT, [_INT, _INT, _P, _P, _P, _P, _I64, _I64, _P, _P, _P, _P, _P, ctypes.c_size_t, _P]),
    "wfx_fused_loss": (_INT, [_INT, _INT, _P, _P, _P, _P, _I64, _I64, _P, _P, _INT, _P, _INT, _D, _D, _D, _P, _P,
                              _P, ctypes.c_size_t, _P]),
    "wfx_autotune_ragged": (_INT, [_INT, _P, _P, _P, _I64, _I64, _P, _P, _P, _P, ctypes.c_size_t, _P, _P]),
    "wfx_tuning": (_INT, [_INT, _I64, _I64, _P, _INT]),
    "wfx_fused_loss_noalloc": (_INT, [_INT, _INT, _P, _P, _P, _P, _I64, _I64, _P, _P, _INT, _P, _INT, _D, _D, _D, _P,
                                      _P, _P]),
    "wfx_fused_loss_partials": (_INT, [_INT, _P, _P, _P, _I64, _I64, _P, _P, _INT, _P, _INT, _D, _D, _D, _P,
                                       ctypes.c_size_t, _P]),
    "wfx_fused_loss_contract": (_INT, [_INT, _P, _P, _I64, _I64, _P, _P, _P, ctypes.c_size_t, _P]),
    "wfx_overlap": (_INT, [_INT, _P, _I64, _P, _I64, _P, _I64, _I64, _D, _P, _I64, _P, _P]),
    "wfx_template_overlap": (_INT, [_INT, _P, _P, _I64, _I64, _P, _D, _D, _P, _P, _D, _P, _I64, _P, _P]),
    "wfx_match_refine": (_INT, [_INT, _P, _P, _I64, _I64, _I64, _P, _D, _P, _INT, _INT, _INT, _P, _P, _P]),
    "wfx_match_grid_time": (_INT, [_P, _I64, _I64, _I64, _D, _P, _P]),
    "wfx_xhm_setup": (_INT, [_P, _I64, _P, _I64, _D, _D, _P, _P, _P, _P]),
    "wfx_xhm_setup_jvp": (_INT, [_P, _I64, _P, _I64, _D, _D, _P, _P, _P, _P, _P]),
    "wfx_phase_difference": (_INT, [_INT, _P, _I64, _P, _P, _P, _P]),
    "wfx_grid_vjp": (_INT, [_INT, _P, _P, _P, _I64, _I64, _P, _P, _P, _P, _P]),
    "wfx_xhm_vjp": (_INT, [_P, _P, _P, _P, _I64, _I64, _I64, _P, _P, _P, _P, _P]),
    "wfx_xhm_polarizations": (_INT, [_INT, _P, _P, _P, _I64, _I64, _I64, _P, _P, _P, _P, _P]),
    "wfx_polarization_overlap": (_INT, [_INT, _P, _I64, _P, _I64, _P, _I64, _P, _I64, _I64, _D, _P, _I64, _P, _P]),
    "wfx_template_polarization_overlap": (_INT, [_INT, _P, _P, _I64, _I64, _P, _P, _P, _D, _P, _I64, _P, _P]),
    "wfx_polarization_refine": (_INT, [_INT, _P, _P, _I64, _I64, _I64, _P, _D, _P, _INT, _INT, _P, _P, _P]),
}
#: WFX_STATIC_SCRATCH_BYTES: the static scratch of wfx_fused_loss_noalloc.
STATIC_SCRATCH_BYTES = 16777216
ESCRATCH = -5
#: WFX_EOFFSETS: ragged offsets that are not non-decreasing from >= 0 to n.
EOFFSETS = -2
#: WFX_EINVAL: a null pointer, a non-positive size or an unknown model.
EINVAL = -1
#: WFX_EWORKSPACE: a workspace missing or smaller than wfx_workspace_bytes().
EWORKSPACE = -3

_lock = threading.Lock()
_library = None


def library(build_if_missing: bool = False) -> ctypes.CDLL:
    """The loaded library (built first if ``build_if_missing`` and stale)."""
    global _library
    with _lock:
        if _library is None:
            path = _build.LIBRARY
            if build_if_missing and _build.stale():
                _build.build()
            if not path.exists():
                raise KernelError(f"the CUDA library {path} is missing: run `python -m waveformx_b200._build`")
            lib = ctypes.CDLL(str(path))
            for name, (restype, argtypes) in EXPORTS.items():
                fn = getattr(lib, name)
                fn.restype = restype
                fn.argtypes = argtypes
            _library = lib
        return _library


def check(name: str, code: int) -> None:
    """Raise :class:`KernelError` for a non-zero return code of ``name``."""
    if code != 0:
        message = library().wfx_status_string(int(code)).decode()
        raise KernelError(f"{name} failed ({code}): {message}")
