"""``batch_polarizations``: many binaries on one grid (or each on its own,
a ragged batch) with the reference's checks and result conventions
(``src/waveformx/_api.py:307-360``).

The reference checks each binary in a Python loop on the host; here the
common checks are one vectorised pass over the table and the model's own
checks (mass ratio, final mass and spin, f_MECO, the mass-scaled reference)
come back from the set-up kernel as a status word per binary.
"""

from __future__ import annotations

from typing import Any, Optional

import numpy as np
import torch

from . import _lib, ops
from ._binary import aligned_table, parameter_table, table_errors
from ._options import WaveformOptions, parse_options, strain_scale
from ._results import BatchPolarizations, FrequencyGrid, check_frequencies
from .exceptions import InvalidParameterError, KernelError, ModelError

__all__ = ["batch_polarizations", "status_errors"]

# the model's errors, in the order the reference's validate raises them
_STATUS_MESSAGES = (
    (64, "masses and distance must be positive"),
    (32, "with reference_mf, the reference frequency is reference_mf / M: f_ref must be zero "
         "(to_mass_scaled_reference converts a binary given at f_ref)"),
    (1, "{approximant} is not valid at mass ratios beyond 1000"),
    (4, "the fitted final mass is not physical"),
    (8, "the fitted final spin exceeds one"),
    (16, "f_MECO cannot be greater than f_ISCO"),
    (2, "|chi| must be at most one"),
    (128, "a collocation system of the set-up is singular"),
)


def status_errors(status: np.ndarray, approximant: str) -> dict:
    """``{row: InvalidParameterError}`` from the set-up's status words."""
    errors = {}
    for i in np.flatnonzero(status):
        word = int(status[i])
        for bit, message in _STATUS_MESSAGES:
            if word & bit:
                if bit == 8 and approximant == "IMRPhenomD":
                    message = "the final spin of IMRPhenomD exceeds one"
                errors[int(i)] = InvalidParameterError(message.format(approximant=approximant))
                break
    return errors


def _device(device) -> torch.device:
    if device is not None:
        device = torch.device(device)
        if device.type != "cuda":
            raise KernelError("waveformx_b200 runs on a CUDA device")
        return device
    if not torch.cuda.is_available():
        raise KernelError("waveformx_b200 runs on a CUDA device and none is available")
    return torch.device("cuda", torch.cuda.current_device())


def batch_polarizations(approximant: str, grid: Any, parameters: Any, *, threads: int = 1, strict: bool = False,
                        exact: bool = False, chunk_size: Optional[int] = None,
                        options: Optional[WaveformOptions] = None, device=None, dtype=torch.float64,
                        output: str = "torch", t_c: Any = None, **option_keywords) -> BatchPolarizations:
    """Polarizations of many binaries, as the reference's
    ``batch_polarizations``: ``parameters`` is a mapping of arrays, a
    structured array, a ``DataFrame`` or an ``(n, 12)`` table; binaries that
    fail the checks or whose waveform is not finite are reported in ``ok``
    and ``errors`` and left as zeros, unless ``strict`` (the first error is
    raised). ``threads`` and ``exact`` are accepted and ignored.

    ``grid`` is a :class:`FrequencyGrid` or frequencies shared by every
    binary, or a list of one grid per binary (a ragged batch: ``hplus`` and
    ``hcross`` are then lists of rows). Extensions: ``device`` (a CUDA
    device), ``dtype`` (``torch.float64``: complex128 by the plain FP64
    kernels, as the reference; ``torch.float32``: complex64 by the FP32
    kernels with double-float phase), ``output`` (``"torch"`` tensors on the
    device, or ``"numpy"``), ``t_c`` (per-binary time shifts, s).
    """
    ops.model_code(approximant)
    options = parse_options(options, option_keywords)
    dev = _device(device)
    precision = _lib.FP32 if dtype == torch.float32 else _lib.FP64
    real = torch.float32 if precision == _lib.FP32 else torch.float64
    cplx = torch.complex64 if precision == _lib.FP32 else torch.complex128
    table = parameter_table(parameters)
    n = len(table)
    ragged = isinstance(grid, (list, tuple)) and len(grid) > 0 and np.ndim(grid[0]) == 1 and not isinstance(
        grid, FrequencyGrid)
    if ragged:
        if len(grid) != n:
            raise ValueError("a ragged batch needs one grid per binary")
        rows = [check_frequencies(g) for g in grid]
        lengths = np.array([len(r) for r in rows], dtype=np.int64)
        offsets_np = np.concatenate([[0], np.cumsum(lengths)]).astype(np.int64)
        flat = np.concatenate(rows) if offsets_np[-1] else np.zeros(0)
        f_min_np = np.array([r[0] if len(r) else 1.0 for r in rows])
    else:
        frequencies = grid.frequencies if isinstance(grid, FrequencyGrid) else check_frequencies(grid)
        flat = frequencies
        f_min_np = np.full(n, frequencies[0] if len(frequencies) else 1.0)
    errors = table_errors(table, approximant)
    if options.reference_mf is not None:
        for i in np.flatnonzero(table[:, 11] != 0.0):
            errors.setdefault(int(i), InvalidParameterError(
                "with reference_mf, the reference frequency is reference_mf / M: f_ref must be zero "
                "(to_mass_scaled_reference converts a binary given at f_ref)"))
    ok = np.ones(n, dtype=bool)
    for i in errors:
        ok[i] = False
    if strict and errors:
        raise errors[min(errors)]
    params_np = aligned_table(table)
    # rows that fail the common checks are replaced by a valid one (as the
    # reference does) and zeroed afterwards
    if ok.any() and not ok.all():
        params_np[~ok] = params_np[np.argmax(ok)]
    tc_np = None if t_c is None else np.broadcast_to(np.asarray(t_c, dtype=np.float64), (n,))
    rmf = options.reference_mf
    scale = strain_scale(options)
    out_p, out_c = [], []
    status_all = np.zeros(n, dtype=np.int32)
    step = n if chunk_size is None else max(1, int(chunk_size))
    if n and len(flat):
        f_dev_all = torch.as_tensor(flat, dtype=real, device=dev)
        for start in range(0, n, step):
            stop = min(n, start + step)
            params = torch.as_tensor(params_np[start:stop], dtype=torch.float64, device=dev)
            f_min = torch.as_tensor(f_min_np[start:stop], dtype=torch.float64, device=dev)
            tables = ops.setup(approximant, params, f_min, amp_scale=scale, reference_mf=rmf, precision=precision)
            tc = None if tc_np is None else torch.as_tensor(tc_np[start:stop], dtype=real, device=dev)
            if ragged:
                lo, hi = int(offsets_np[start]), int(offsets_np[stop])
                offs = torch.as_tensor(offsets_np[start:stop + 1] - lo, dtype=torch.int64, device=dev)
                hp, hc = ops.polarizations(approximant, tables.table, f_dev_all[lo:hi].contiguous(), offs, tc)
            else:
                hp, hc = ops.polarizations(approximant, tables.table, f_dev_all, None, tc)
            status_all[start:stop] = tables.status.cpu().numpy()
            out_p.append(hp)
            out_c.append(hc)
        hplus = torch.cat(out_p)
        hcross = torch.cat(out_c)
    else:
        hplus = torch.zeros((n, len(flat)) if not ragged else (0,), dtype=cplx, device=dev)
        hcross = torch.zeros_like(hplus)
    # the model's own checks, from the set-up's status words
    for i, error in status_errors(status_all, approximant).items():
        if ok[i]:
            ok[i] = False
            errors[i] = error
    if ragged:
        row_of = torch.repeat_interleave(torch.arange(n, device=dev), torch.as_tensor(lengths, device=dev))
        bad = ~(torch.isfinite(torch.view_as_real(hplus)).all(-1) & torch.isfinite(torch.view_as_real(hcross)).all(-1))
        finite = torch.ones(n, dtype=torch.bool, device=dev)
        if bad.any():
            finite[row_of[bad]] = False
        finite = finite.cpu().numpy()
    else:
        # ((n, N, 2) -> (n,): also for no binary or no frequency)
        finite = (torch.isfinite(torch.view_as_real(hplus)).all(-1).all(-1)
                  & torch.isfinite(torch.view_as_real(hcross)).all(-1).all(-1)).cpu().numpy()
    for i in np.flatnonzero(ok & ~finite):
        ok[i] = False
        errors[int(i)] = ModelError(f"{approximant} could not be evaluated for binary {i}")
    if strict and errors:
        raise errors[min(errors)]
    mask = torch.as_tensor(~ok, device=dev)
    if ragged:
        zero_rows = mask[row_of] if len(flat) else mask[:0]
        hplus[zero_rows] = 0
        hcross[zero_rows] = 0
        hplus = list(torch.tensor_split(hplus, offsets_np[1:-1].tolist()))
        hcross = list(torch.tensor_split(hcross, offsets_np[1:-1].tolist()))
    else:
        hplus[mask] = 0
        hcross[mask] = 0
    if output == "numpy":
        conv = lambda x: x.cpu().numpy()  # noqa: E731
        hplus = [conv(x) for x in hplus] if ragged else conv(hplus)
        hcross = [conv(x) for x in hcross] if ragged else conv(hcross)
    elif output != "torch":
        raise ValueError('output must be "torch" or "numpy"')
    return BatchPolarizations(hplus, hcross, ok, errors)
