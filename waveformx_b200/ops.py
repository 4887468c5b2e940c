"""Tensor-level operations on CUDA tensors: the per-binary tables, the
polarizations, their vector-Jacobian product and the fused likelihood, each
one call of the C ABI on the current stream of the tensors' device.

All inputs are CUDA tensors (the caller moves host data); outputs are new
CUDA tensors. FP32 runs the FP32 kernels with the double-float phase (float32
tables, frequencies and ``t_c``, complex64 strain); FP64 the plain FP64 form
(float64 everywhere, complex128 strain). The set-up is FP64 in both.
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass
from typing import Optional

import torch

from . import _lib
from .exceptions import UnknownApproximantError, UnsupportedError

__all__ = ["APPROXIMANTS", "model_code", "Tables", "setup", "polarizations", "vjp", "fused_loss", "workspace",
           "setup_jvp_async", "fused_loss_from_params", "fft_length", "overlap", "template_overlap",
           "grid_time_supported", "match_grid_time", "match_refine",
           "polarization_overlap", "template_polarization_overlap", "polarization_refine", "xhm_modes",
           "XHM_MODES", "xhm_dtable", "xhm_vjp", "grid_vjp", "check_offsets", "check_per_frequency",
           "offsets_problem"]

#: The approximants of this path and their codes in the C ABI.
APPROXIMANTS = {"IMRPhenomXAS": _lib.XAS, "IMRPhenomD": _lib.PHENOMD, "TaylorF2": _lib.TAYLORF2,
                "IMRPhenomXHM": _lib.XHM}
#: The reference's other approximants: known, not on this path.
OTHER_APPROXIMANTS = ("IMRPhenomXPNR", "IMRPhenomXPNR_NNLO", "IMRPhenomXPNR_MSA", "NRSur7dq4")
#: IMRPhenomXHM's modes, in the order of its outputs (models/xhm/core.py:56-57).
XHM_MODES = ((2, 2), (2, 1), (3, 3), (3, 2), (4, 4))


def model_code(approximant: str) -> int:
    """The C-ABI model of an approximant (errors as the reference's registry,
    ``models/__init__.py:74-84``)."""
    if isinstance(approximant, str) and approximant in APPROXIMANTS:
        return APPROXIMANTS[approximant]
    if isinstance(approximant, str) and approximant in OTHER_APPROXIMANTS:
        raise UnsupportedError(f"{approximant} is not on the aligned-spin B200 path ({', '.join(APPROXIMANTS)})")
    raise UnknownApproximantError(
        f"unknown approximant {approximant!r}: waveformx_b200 implements {', '.join(APPROXIMANTS)}")


def _differentiable(model: int) -> None:
    """IMRPhenomXHM has no table-based backward or fused likelihood: they
    raise UnsupportedError (its gradient is :func:`xhm_vjp`)."""
    if model == _lib.XHM:
        raise UnsupportedError("IMRPhenomXHM: no table-based backward or fused likelihood "
                               "(its gradient: ops.xhm_vjp)")


def _ptr(t: Optional[torch.Tensor]):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def _stream(device: torch.device):
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def _require(t: torch.Tensor, name: str, dtype=None):
    if not isinstance(t, torch.Tensor) or t.device.type != "cuda":
        raise TypeError(f"{name} must be a CUDA tensor")
    if dtype is not None and t.dtype != dtype:
        raise TypeError(f"{name} must be {dtype}, got {t.dtype}")
    if not t.is_contiguous():
        raise ValueError(f"{name} must be contiguous")
    return t


def workspace(op: int, model: int, precision: int, batch: int, n: int, ragged: bool,
              device: torch.device) -> Optional[torch.Tensor]:
    """A scratch buffer for ``op`` (None if none is needed)."""
    nbytes = int(_lib.library().wfx_workspace_bytes(op, model, precision, batch, n, int(ragged)))
    return None if nbytes == 0 else torch.empty(nbytes, dtype=torch.uint8, device=device)


@dataclass
class Tables:
    """The per-binary tables of a batch: ``table`` (B x 72, float32 or
    float64), ``dtable`` (B x 72 x 8 float64, or None), ``status`` (B
    int32), and the precision code."""

    table: torch.Tensor
    dtable: Optional[torch.Tensor]
    status: torch.Tensor
    precision: int


def setup(approximant: str, params: torch.Tensor, f_min: torch.Tensor, *, amp_scale: float = 1e21,
          reference_mf: Optional[float] = None, precision: int = _lib.FP32, jvp: bool = False) -> Tables:
    """The tables of ``params`` (``(B, 8)`` float64: masses, aligned spins,
    distance, inclination, phi_ref, f_ref) with first frequencies ``f_min``
    (``(B,)``, or one value); with ``jvp``, their derivatives too."""
    model = model_code(approximant)
    _require(params, "params", torch.float64)
    _require(f_min, "f_min", torch.float64)
    batch = params.shape[0]
    if params.ndim != 2 or params.shape[1] != 8 or batch == 0:
        raise ValueError("params must be (B, 8) with B > 0")
    stride = 0 if f_min.numel() == 1 else 1
    if stride and f_min.numel() != batch:
        raise ValueError("f_min must have one value or one per binary")
    device = params.device
    dtype = torch.float32 if precision == _lib.FP32 else torch.float64
    rmf = math.nan if reference_mf is None else float(reference_mf)
    lib = _lib.library()
    if model == _lib.XHM:
        # IMRPhenomXHM: its own rows (the (2,2), the head, the higher modes)
        # (with jvp, d row64 / d params: B x 544 x 8 float64, from the set-up
        # on dual numbers)
        stride = _lib.XHM_STRIDE32 if precision == _lib.FP32 else _lib.XHM_STRIDE64
        table = torch.empty((batch, stride), dtype=dtype, device=device)
        status = torch.empty(batch, dtype=torch.int32, device=device)
        t64 = table if precision == _lib.FP64 else None
        t32 = table if precision == _lib.FP32 else None
        f_stride = 0 if f_min.numel() == 1 else 1
        if jvp:
            dtable = torch.empty((batch, _lib.XHM_STRIDE64, 8), dtype=torch.float64, device=device)
            _lib.check("wfx_xhm_setup_jvp", lib.wfx_xhm_setup_jvp(
                _ptr(params), batch, _ptr(f_min), f_stride, float(amp_scale), rmf, _ptr(t64), _ptr(t32),
                _ptr(dtable), _ptr(status), _stream(device)))
            return Tables(table, dtable, status, precision)
        _lib.check("wfx_xhm_setup", lib.wfx_xhm_setup(_ptr(params), batch, _ptr(f_min), f_stride, float(amp_scale),
                                                      rmf, _ptr(t64), _ptr(t32), _ptr(status), _stream(device)))
        return Tables(table, None, status, precision)
    table = torch.empty((batch, _lib.TABLE_STRIDE), dtype=dtype, device=device)
    status = torch.empty(batch, dtype=torch.int32, device=device)
    t64 = table if precision == _lib.FP64 else None
    t32 = table if precision == _lib.FP32 else None
    if jvp:
        dtable = torch.empty((batch, _lib.TABLE_STRIDE, 8), dtype=torch.float64, device=device)
        _lib.check("wfx_setup_jvp", lib.wfx_setup_jvp(model, _ptr(params), batch, _ptr(f_min), stride,
                                                      float(amp_scale), rmf, _ptr(t64), _ptr(t32), _ptr(dtable),
                                                      _ptr(status), _stream(device)))
    else:
        dtable = None
        _lib.check("wfx_setup", lib.wfx_setup(model, _ptr(params), batch, _ptr(f_min), stride, float(amp_scale), rmf,
                                              _ptr(t64), _ptr(t32), _ptr(status), _stream(device)))
    return Tables(table, dtable, status, precision)


def _precision_of(table: torch.Tensor) -> int:
    return _lib.FP32 if table.dtype == torch.float32 else _lib.FP64


def check_offsets(offsets: torch.Tensor, batch: int, n: int) -> None:
    """Raise ValueError unless ``offsets`` (``B + 1`` int64) run from
    ``offsets[0] >= 0``, non-decreasing, to ``offsets[B] == n`` (the rows
    check of the reference's batch API, ``src/waveformx/_api.py:292-305``).
    Reads the offsets to the host once per tensor and version (in-place
    changes bump the version); the kernels check them again on the device."""
    _require(offsets, "offsets", torch.int64)
    key = (offsets._version, int(n), offsets.data_ptr())
    if getattr(offsets, "_wfx_checked", None) == key:
        return
    problem = offsets_problem(offsets.cpu(), batch, n)
    if problem is not None:
        raise ValueError(problem)
    offsets._wfx_checked = key


def offsets_problem(offsets, batch: int, n: int) -> Optional[str]:
    """Why host ``offsets`` (a CPU tensor or array) cannot index ``batch``
    binaries' grids in ``n`` flattened frequencies, or None if they can."""
    o = torch.as_tensor(offsets)
    if o.ndim != 1 or o.numel() != batch + 1:
        return f"offsets must have B + 1 = {batch + 1} entries, got shape {tuple(o.shape)}"
    if int(o[0]) < 0 or int(o[-1]) != n or bool((o[1:] < o[:-1]).any()):
        return (f"offsets must be non-decreasing from offsets[0] >= 0 to offsets[B] == {n} "
                f"(the number of flattened frequencies)")
    return None


def check_per_frequency(t: torch.Tensor, name: str, batch: int, n: int, ragged: bool) -> int:
    """The stride code of ``data`` or ``weights`` of the fused likelihood:
    0 for one value per frequency of a shared grid (``n``), 1 for one per
    element of the batch's strain (``B n``, or the ``n`` flattened
    frequencies of a ragged batch); ValueError for any other size."""
    if ragged:
        if t.numel() != n:
            raise ValueError(f"{name} must have one value per flattened frequency ({n}), got {t.numel()}")
        return 1
    if t.numel() == n:
        return 0
    if t.numel() == batch * n:
        return 1
    raise ValueError(f"{name} must have {n} values (shared) or {batch * n} (per binary), got {t.numel()}")


def _grid(table, freqs, offsets, t_c):
    precision = _precision_of(table)
    real = table.dtype
    _require(table, "table", real)
    _require(freqs, "freqs", real)
    batch = table.shape[0]
    if offsets is not None:
        check_offsets(offsets, batch, freqs.numel())
    if t_c is not None:
        _require(t_c, "t_c", real)
        if t_c.numel() != batch:
            raise ValueError("t_c must have one value per binary")
    return precision, batch, freqs.numel()


def polarizations(approximant: str, table: torch.Tensor, freqs: torch.Tensor, offsets: Optional[torch.Tensor] = None,
                  t_c: Optional[torch.Tensor] = None):
    """``(hplus, hcross)``: ``(B, N)`` complex on a shared grid ``freqs``
    ``(N,)``, or flat ``(offsets[B],)`` for a ragged batch."""
    model = model_code(approximant)
    if model == _lib.XHM:
        if offsets is not None:
            return _xhm_ragged(table, freqs, offsets, t_c)
        hp, hc, _ = xhm_modes(table, freqs, t_c, modes=False)
        return hp, hc
    precision, batch, n = _grid(table, freqs, offsets, t_c)
    complex_dtype = torch.complex64 if precision == _lib.FP32 else torch.complex128
    shape = (batch, n) if offsets is None else (n,)
    hp = torch.empty(shape, dtype=complex_dtype, device=table.device)
    hc = torch.empty(shape, dtype=complex_dtype, device=table.device)
    ws = workspace(_lib.OP_POLARIZATIONS, model, precision, batch, n, offsets is not None, table.device)
    lib = _lib.library()
    _lib.check("wfx_polarizations", lib.wfx_polarizations(
        model, precision, _ptr(table), _ptr(freqs), _ptr(offsets), batch, n, _ptr(t_c), _ptr(hp), _ptr(hc),
        _ptr(ws), 0 if ws is None else ws.numel(), _stream(table.device)))
    return hp, hc


def grid_vjp(approximant: str, table: torch.Tensor, freqs: torch.Tensor, offsets: Optional[torch.Tensor],
             t_c: Optional[torch.Tensor], cot_hp: torch.Tensor, cot_hc: torch.Tensor) -> torch.Tensor:
    """``dL/df`` (float64, ``(N,)`` summed over the binaries of a shared grid,
    or flat ragged) for the cotangents of (hplus, hcross), from the FP64
    evaluation of the FP64 ``table`` (IMRPhenomXHM: its FP64 rows)."""
    model = model_code(approximant)
    _require(table, "table", torch.float64)
    _require(freqs, "freqs", torch.float64)
    batch, n = table.shape[0], freqs.numel()
    if t_c is not None:
        _require(t_c, "t_c", torch.float64)
    if offsets is not None:
        check_offsets(offsets, batch, n)
    cp = cot_hp.to(torch.complex128).contiguous()
    cc = cot_hc.to(torch.complex128).contiguous()
    out = torch.empty(n, dtype=torch.float64, device=table.device)
    _lib.check("wfx_grid_vjp", _lib.library().wfx_grid_vjp(
        model, _ptr(table), _ptr(freqs), _ptr(offsets), batch, n, _ptr(t_c), _ptr(cp), _ptr(cc), _ptr(out),
        _stream(table.device)))
    return out


def xhm_modes(table: torch.Tensor, freqs: torch.Tensor, t_c: Optional[torch.Tensor] = None, *, modes: bool = True):
    """IMRPhenomXHM from its tables (:func:`setup`) on a shared grid ``freqs``
    ``(N,)``: ``(hplus, hcross, modes)``, ``(B, N)`` complex each and the
    modes ``h_{l,-m}`` of :data:`XHM_MODES` ``(B, 5, N)`` (None without
    ``modes``)."""
    precision, batch, n = _grid(table, freqs, None, t_c)
    stride = _lib.XHM_STRIDE32 if precision == _lib.FP32 else _lib.XHM_STRIDE64
    if table.ndim != 2 or table.shape[1] != stride:
        raise ValueError(f"an IMRPhenomXHM table has {stride} columns in this precision")
    complex_dtype = torch.complex64 if precision == _lib.FP32 else torch.complex128
    hp = torch.empty((batch, n), dtype=complex_dtype, device=table.device)
    hc = torch.empty((batch, n), dtype=complex_dtype, device=table.device)
    out = torch.empty((batch, _lib.XHM_MODES, n), dtype=complex_dtype, device=table.device) if modes else None
    _lib.check("wfx_xhm_polarizations", _lib.library().wfx_xhm_polarizations(
        precision, _ptr(table), _ptr(freqs), None, batch, n, n, _ptr(t_c), _ptr(hp), _ptr(hc), _ptr(out),
        _stream(table.device)))
    return hp, hc, out


def xhm_dtable(params: torch.Tensor, f_min: torch.Tensor, *, amp_scale: float = 1e21,
               reference_mf: Optional[float] = None) -> torch.Tensor:
    """IMRPhenomXHM's ``d table / d params`` ``(B, 544, 8)`` float64 of its
    FP64 row: its set-up on dual numbers (one thread per binary, part and
    parameter); zero along ``f_ref`` where ``f_ref = 0`` (the first frequency
    or ``reference_mf / M`` then stands for it, as in the reference)."""
    _require(params, "params", torch.float64)
    _require(f_min, "f_min", torch.float64)
    batch = params.shape[0]
    if params.ndim != 2 or params.shape[1] != 8 or batch == 0:
        raise ValueError("params must be (B, 8) with B > 0")
    if f_min.numel() not in (1, batch):
        raise ValueError("f_min must have one value or one per binary")
    dtable = torch.empty((batch, _lib.XHM_STRIDE64, 8), dtype=torch.float64, device=params.device)
    _lib.check("wfx_xhm_setup_jvp", _lib.library().wfx_xhm_setup_jvp(
        _ptr(params), batch, _ptr(f_min), 0 if f_min.numel() == 1 else 1, float(amp_scale),
        math.nan if reference_mf is None else float(reference_mf), None, None, _ptr(dtable), None,
        _stream(params.device)))
    return dtable


def xhm_vjp(params: torch.Tensor, f_min: torch.Tensor, freqs: torch.Tensor, offsets: Optional[torch.Tensor],
            t_c: Optional[torch.Tensor], cot_hp: torch.Tensor, cot_hc: torch.Tensor, *, amp_scale: float = 1e21,
            reference_mf: Optional[float] = None) -> torch.Tensor:
    """IMRPhenomXHM's ``(B, 9)`` float64 gradients of ``L`` with respect to
    (mass_1, mass_2, chi_1, chi_2, luminosity_distance, inclination, phi_ref,
    f_ref, t_c) for the cotangents ``dL/dRe h + i dL/dIm h`` of (hplus,
    hcross), from the FP64 evaluation on ``freqs`` (float64; ragged with
    ``offsets``): its forward-mode derivatives along the set-up's tangents
    (the set-up on dual numbers, :func:`xhm_dtable`), contracted with the
    cotangents in the kernel."""
    _require(params, "params", torch.float64)
    _require(freqs, "freqs", torch.float64)
    tables = setup("IMRPhenomXHM", params, f_min, amp_scale=amp_scale, reference_mf=reference_mf,
                   precision=_lib.FP64, jvp=True)
    table, dtable = tables.table, tables.dtable
    batch, n = params.shape[0], freqs.numel()
    if t_c is not None:
        _require(t_c, "t_c", torch.float64)
    cp = cot_hp.to(torch.complex128).contiguous()
    cc = cot_hc.to(torch.complex128).contiguous()
    max_len = n
    if offsets is not None:
        check_offsets(offsets, batch, n)
        max_len = int((offsets[1:] - offsets[:-1]).max())
    grad = torch.empty((batch, _lib.GRAD_COLUMNS), dtype=torch.float64, device=params.device)
    _lib.check("wfx_xhm_vjp", _lib.library().wfx_xhm_vjp(
        _ptr(table), _ptr(dtable), _ptr(freqs), _ptr(offsets), batch, n, max_len, _ptr(t_c), _ptr(cp), _ptr(cc),
        _ptr(grad), _stream(params.device)))
    return grad


def _xhm_ragged(table, freqs, offsets, t_c):
    """IMRPhenomXHM's (hplus, hcross) on per-binary grids: flat
    ``(offsets[B],)`` each."""
    precision, batch, n = _grid(table, freqs, offsets, t_c)
    complex_dtype = torch.complex64 if precision == _lib.FP32 else torch.complex128
    hp = torch.empty(n, dtype=complex_dtype, device=table.device)
    hc = torch.empty(n, dtype=complex_dtype, device=table.device)
    max_len = int((offsets[1:] - offsets[:-1]).max()) if batch else 0
    if n == 0 or max_len <= 0:
        return hp, hc
    _lib.check("wfx_xhm_polarizations", _lib.library().wfx_xhm_polarizations(
        precision, _ptr(table), _ptr(freqs), _ptr(offsets), batch, n, max_len, _ptr(t_c), _ptr(hp), _ptr(hc),
        None, _stream(table.device)))
    return hp, hc


def vjp(approximant: str, table: torch.Tensor, dtable: torch.Tensor, freqs: torch.Tensor,
        offsets: Optional[torch.Tensor], t_c: Optional[torch.Tensor], cot_hp: torch.Tensor,
        cot_hc: torch.Tensor) -> torch.Tensor:
    """``(B, 9)`` gradients of ``L`` with respect to (mass_1, mass_2, chi_1,
    chi_2, luminosity_distance, inclination, phi_ref, f_ref, t_c) for the
    cotangents ``dL/dRe h + i dL/dIm h`` of (hplus, hcross)."""
    model = model_code(approximant)
    _differentiable(model)
    precision, batch, n = _grid(table, freqs, offsets, t_c)
    complex_dtype = torch.complex64 if precision == _lib.FP32 else torch.complex128
    _require(dtable, "dtable", torch.float64)
    _require(cot_hp, "cot_hp", complex_dtype)
    _require(cot_hc, "cot_hc", complex_dtype)
    grad = torch.empty((batch, _lib.GRAD_COLUMNS), dtype=table.dtype, device=table.device)
    ws = workspace(_lib.OP_VJP, model, precision, batch, n, offsets is not None, table.device)
    lib = _lib.library()
    _lib.check("wfx_vjp", lib.wfx_vjp(model, precision, _ptr(table), _ptr(dtable), _ptr(freqs), _ptr(offsets), batch,
                                      n, _ptr(t_c), _ptr(cot_hp), _ptr(cot_hc), _ptr(grad), _ptr(ws),
                                      0 if ws is None else ws.numel(), _stream(table.device)))
    return grad


def fused_loss(approximant: str, table: torch.Tensor, dtable: Optional[torch.Tensor], freqs: torch.Tensor,
               offsets: Optional[torch.Tensor], t_c: Optional[torch.Tensor], data: torch.Tensor,
               weights: torch.Tensor, *, antenna=(1.0, 0.0), scale: float = 1.0):
    """``loss[b] = scale * sum_f w(f) |F+ h+ + Fx hx - d(f)|^2`` and, with
    ``dtable``, its ``(B, 9)`` gradient, without writing the strain. ``data``
    and ``weights`` are shared (one per frequency of the shared grid) or per
    binary (laid out like the strain)."""
    model = model_code(approximant)
    _differentiable(model)
    precision, batch, n = _grid(table, freqs, offsets, t_c)
    complex_dtype = torch.complex64 if precision == _lib.FP32 else torch.complex128
    _require(data, "data", complex_dtype)
    _require(weights, "weights", table.dtype)
    data_stride = check_per_frequency(data, "data", batch, n, offsets is not None)
    weights_stride = check_per_frequency(weights, "weights", batch, n, offsets is not None)
    loss = torch.empty(batch, dtype=table.dtype, device=table.device)
    grad = None
    if dtable is not None:
        _require(dtable, "dtable", torch.float64)
        grad = torch.empty((batch, _lib.GRAD_COLUMNS), dtype=table.dtype, device=table.device)
    ws = workspace(_lib.OP_FUSED, model, precision, batch, n, offsets is not None, table.device)
    lib = _lib.library()
    _lib.check("wfx_fused_loss", lib.wfx_fused_loss(
        model, precision, _ptr(table), _ptr(dtable), _ptr(freqs), _ptr(offsets), batch, n, _ptr(t_c), _ptr(data),
        data_stride, _ptr(weights), weights_stride, float(antenna[0]), float(antenna[1]), float(scale), _ptr(loss),
        _ptr(grad), _ptr(ws), 0 if ws is None else ws.numel(), _stream(table.device)))
    return loss, grad


_SIDE_STREAMS: dict = {}


def _side_stream(device: torch.device) -> torch.cuda.Stream:
    """A second stream of ``device`` (one per device, kept)."""
    key = torch.device(device).index
    stream = _SIDE_STREAMS.get(key)
    if stream is None:
        stream = torch.cuda.Stream(device=device)
        _SIDE_STREAMS[key] = stream
    return stream


def setup_jvp_async(approximant: str, params: torch.Tensor, f_min: torch.Tensor, *, amp_scale: float = 1e21,
                    reference_mf: Optional[float] = None, out: Optional[torch.Tensor] = None):
    """``dtable`` (``(B, 72, 8)`` float64) by the dual-number set-up on a
    second stream of the device, after the work queued so far on the current
    one: ``(dtable, event)``. Work that reads ``dtable`` waits for ``event``
    (``torch.cuda.current_stream().wait_event(event)``); the current stream
    is free meanwhile (the value set-up, the forward or the reverse pass).
    ``out``: a buffer of that shape allocated on the current stream, which
    must then wait for ``event`` before it frees or reuses it (the form a
    CUDA-graph capture takes: nothing is allocated on the second stream)."""
    model = model_code(approximant)
    _differentiable(model)
    _require(params, "params", torch.float64)
    _require(f_min, "f_min", torch.float64)
    batch = params.shape[0]
    stride = 0 if f_min.numel() == 1 else 1
    device = params.device
    rmf = math.nan if reference_mf is None else float(reference_mf)
    main = torch.cuda.current_stream(device)
    if out is not None:
        _require(out, "out", torch.float64)
        if tuple(out.shape) != (batch, _lib.TABLE_STRIDE, 8):
            raise ValueError(f"out must be ({batch}, {_lib.TABLE_STRIDE}, 8)")
    side = _side_stream(device)
    side.wait_stream(main)
    with torch.cuda.stream(side):
        dtable = out if out is not None else torch.empty((batch, _lib.TABLE_STRIDE, 8), dtype=torch.float64,
                                                         device=device)
        _lib.check("wfx_setup_jvp", _lib.library().wfx_setup_jvp(
            model, _ptr(params), batch, _ptr(f_min), stride, float(amp_scale), rmf, None, None, _ptr(dtable), None,
            _stream(device)))
        event = torch.cuda.Event()
        event.record(side)
    if out is None:
        dtable.record_stream(main)
    return dtable, event


def fused_loss_from_params(approximant: str, params: torch.Tensor, f_min: torch.Tensor, freqs: torch.Tensor,
                           offsets: Optional[torch.Tensor], t_c: Optional[torch.Tensor], data: torch.Tensor,
                           weights: torch.Tensor, *, antenna=(1.0, 0.0), scale: float = 1.0, amp_scale: float = 1e21,
                           reference_mf: Optional[float] = None, dtable_out: Optional[torch.Tensor] = None):
    """The FP32 fused likelihood and its ``(B, 9)`` gradient from the
    binaries' parameters, with the dual-number set-up of ``dtable`` on a
    second stream while the value set-up and the reverse pass run on the
    current one (they do not need it): ``(loss, grad, status)``. The same
    results as :func:`setup` with ``jvp`` followed by :func:`fused_loss`.
    ``dtable_out``: the ``out`` of :func:`setup_jvp_async`."""
    model = model_code(approximant)
    device = params.device
    lib = _lib.library()
    main = torch.cuda.current_stream(device)
    dtable, ready = setup_jvp_async(approximant, params, f_min, amp_scale=amp_scale, reference_mf=reference_mf,
                                    out=dtable_out)
    tables = setup(approximant, params, f_min, amp_scale=amp_scale, reference_mf=reference_mf, precision=_lib.FP32)
    _, batch, n = _grid(tables.table, freqs, offsets, t_c)
    _require(data, "data", torch.complex64)
    _require(weights, "weights", torch.float32)
    data_stride = check_per_frequency(data, "data", batch, n, offsets is not None)
    weights_stride = check_per_frequency(weights, "weights", batch, n, offsets is not None)
    ws = workspace(_lib.OP_FUSED, model, _lib.FP32, batch, n, offsets is not None, device)
    _lib.check("wfx_fused_loss_partials", lib.wfx_fused_loss_partials(
        model, _ptr(tables.table), _ptr(freqs), _ptr(offsets), batch, n, _ptr(t_c), _ptr(data), data_stride,
        _ptr(weights), weights_stride, float(antenna[0]), float(antenna[1]), float(scale), _ptr(ws), ws.numel(),
        _stream(device)))
    main.wait_event(ready)
    loss = torch.empty(batch, dtype=torch.float32, device=device)
    grad = torch.empty((batch, _lib.GRAD_COLUMNS), dtype=torch.float32, device=device)
    _lib.check("wfx_fused_loss_contract", lib.wfx_fused_loss_contract(
        model, _ptr(dtable), _ptr(offsets), batch, n, _ptr(loss), _ptr(grad), _ptr(ws), ws.numel(), _stream(device)))
    return loss, grad, tables.status


# ---------------------------------------------------------------------------
# matches (src/waveformx/match.py:71-147)

def fft_length(n: int, pad: int) -> int:
    """The length of the time grid of a match: ``pad`` times the power of two
    at or above the number of frequencies (match.py:95-96)."""
    return int(pad) * (1 << (int(n) - 1).bit_length())


def overlap(a: torch.Tensor, b: torch.Tensor, psd: torch.Tensor, delta_f: float, series: torch.Tensor):
    """The overlap series of the rows of ``a`` and ``b`` (``(rows, n)`` or
    ``(n,)`` for one vector for every row; complex64 or complex128) into the
    first ``n`` columns of ``series`` (``(rows, n_fft)``, its other columns
    zero), and the ``(rows, 2)`` float64 norms ``<a, a>``, ``<b, b>``."""
    precision = _lib.FP64 if a.dtype == torch.complex128 else _lib.FP32
    real = torch.float64 if precision == _lib.FP64 else torch.float32
    _require(a, "a", a.dtype)
    _require(b, "b", a.dtype)
    _require(psd, "psd", real)
    _require(series, "series", a.dtype)
    n = psd.numel()
    rows = series.shape[0]
    norms = torch.empty((rows, 2), dtype=torch.float64, device=series.device)
    lib = _lib.library()
    _lib.check("wfx_overlap", lib.wfx_overlap(
        precision, _ptr(a), n if a.ndim == 2 else 0, _ptr(b), n if b.ndim == 2 else 0, _ptr(psd), rows, n,
        float(delta_f), _ptr(series), series.shape[1], _ptr(norms), _stream(series.device)))
    return norms


def template_overlap(approximant: str, table: torch.Tensor, freqs: torch.Tensor, signal: torch.Tensor,
                     psd: torch.Tensor, delta_f: float, series: torch.Tensor, *, t_c: Optional[torch.Tensor] = None,
                     antenna=(1.0, 0.0)):
    """The overlap series of the templates ``F+ h+ + Fx hx`` of the FP32
    ``table`` (``(B, 72)``) on the shared grid ``freqs`` with ``signal``
    (complex64, ``(n,)``) into ``series`` (``(B, n_fft)`` complex64, its
    columns from ``n`` zero), without writing the templates; returns the
    ``(B, 2)`` norms."""
    model = model_code(approximant)
    _require(table, "table", torch.float32)
    _require(freqs, "freqs", torch.float32)
    _require(signal, "signal", torch.complex64)
    _require(psd, "psd", torch.float32)
    _require(series, "series", torch.complex64)
    batch, n = table.shape[0], freqs.numel()
    if t_c is not None:
        _require(t_c, "t_c", torch.float32)
    norms = torch.empty((batch, 2), dtype=torch.float64, device=table.device)
    lib = _lib.library()
    _lib.check("wfx_template_overlap", lib.wfx_template_overlap(
        model, _ptr(table), _ptr(freqs), batch, n, _ptr(t_c), float(antenna[0]), float(antenna[1]), _ptr(signal),
        _ptr(psd), float(delta_f), _ptr(series), series.shape[1], _ptr(norms), _stream(table.device)))
    return norms


def grid_time_supported(n: int, n_fft: int) -> bool:
    """Whether :func:`match_grid_time` takes ``n`` frequencies on a grid of
    ``n_fft`` times: the power of two ``L >= max(n, 2048)`` is at most 16384
    and divides ``n_fft`` (the library's rule, ``wfx_match_grid_time``)."""
    length = max(2048, 1 << (int(n) - 1).bit_length())
    return length <= 16384 and int(n_fft) % length == 0


def match_grid_time(series: torch.Tensor, n: int, delta_f: float) -> torch.Tensor:
    """The best time of each row's grid (largest ``|z|``) by the inverse FFT
    in shared memory, for complex64 ``series`` whose rows are zero from
    ``n`` on (see :func:`grid_time_supported`): float64 ``(rows,)``."""
    _require(series, "series", torch.complex64)
    rows, n_fft = series.shape
    t = torch.empty(rows, dtype=torch.float64, device=series.device)
    _lib.check("wfx_match_grid_time", _lib.library().wfx_match_grid_time(
        _ptr(series), rows, int(n), n_fft, float(delta_f), _ptr(t), _stream(series.device)))
    return t


def match_refine(series: torch.Tensor, zgrid: Optional[torch.Tensor], freqs: torch.Tensor, delta_f: float,
                 norms: torch.Tensor, *, time: bool = True, phase: bool = True, steps: int = 3,
                 t_start: Optional[torch.Tensor] = None):
    """The matches of the rows of ``series`` (with ``time``: from its
    unnormalised inverse FFT ``zgrid``, or from the grid times ``t_start`` of
    :func:`match_grid_time`) at the float64 frequencies ``freqs``:
    ``(match, t)``, float64 ``(rows,)``."""
    precision = _lib.FP64 if series.dtype == torch.complex128 else _lib.FP32
    _require(series, "series", series.dtype)
    _require(freqs, "freqs", torch.float64)
    _require(norms, "norms", torch.float64)
    mode = 0
    if time:
        mode = 2 if t_start is not None else 1
        if mode == 1:
            _require(zgrid, "zgrid", series.dtype)
    rows, n_fft = series.shape
    out = torch.empty(rows, dtype=torch.float64, device=series.device)
    t = t_start if mode == 2 else torch.empty(rows, dtype=torch.float64, device=series.device)
    lib = _lib.library()
    _lib.check("wfx_match_refine", lib.wfx_match_refine(
        precision, _ptr(series), _ptr(zgrid) if mode == 1 else None, rows, freqs.numel(), n_fft, _ptr(freqs),
        float(delta_f), _ptr(norms), mode, int(bool(phase)), int(steps), _ptr(out), _ptr(t),
        _stream(series.device)))
    return out, t


def polarization_overlap(signal: torch.Tensor, hplus: torch.Tensor, hcross: torch.Tensor, psd: torch.Tensor,
                         delta_f: float, series: torch.Tensor):
    """polarization_match's series of each row (rows ``2 r`` and ``2 r + 1``
    of ``series``, ``(2 rows, n_fft)``, its columns from ``n`` zero) and the
    ``(rows, 4)`` norms ``<s, s>, <h+, h+>, <hx, hx>, <h+, hx>``; a
    one-dimensional input is one vector for every row."""
    precision = _lib.FP64 if signal.dtype == torch.complex128 else _lib.FP32
    real = torch.float64 if precision == _lib.FP64 else torch.float32
    for name, t in (("signal", signal), ("hplus", hplus), ("hcross", hcross)):
        _require(t, name, signal.dtype)
    _require(psd, "psd", real)
    _require(series, "series", signal.dtype)
    n = psd.numel()
    rows = series.shape[0] // 2
    norms = torch.empty((rows, 4), dtype=torch.float64, device=series.device)
    stride = lambda t: n if t.ndim == 2 else 0  # noqa: E731
    _lib.check("wfx_polarization_overlap", _lib.library().wfx_polarization_overlap(
        precision, _ptr(signal), stride(signal), _ptr(hplus), stride(hplus), _ptr(hcross), stride(hcross), _ptr(psd),
        rows, n, float(delta_f), _ptr(series), series.shape[1], _ptr(norms), _stream(series.device)))
    return norms


def template_polarization_overlap(approximant: str, table: torch.Tensor, freqs: torch.Tensor, signal: torch.Tensor,
                                  psd: torch.Tensor, delta_f: float, series: torch.Tensor, *,
                                  t_c: Optional[torch.Tensor] = None):
    """polarization_match's series of the binaries of the FP32 ``table``
    against ``signal`` (``series`` ``(2 B, n_fft)`` complex64), without
    their strain; returns the ``(B, 4)`` norms."""
    model = model_code(approximant)
    _require(table, "table", torch.float32)
    _require(freqs, "freqs", torch.float32)
    _require(signal, "signal", torch.complex64)
    _require(psd, "psd", torch.float32)
    _require(series, "series", torch.complex64)
    batch, n = table.shape[0], freqs.numel()
    norms = torch.empty((batch, 4), dtype=torch.float64, device=table.device)
    _lib.check("wfx_template_polarization_overlap", _lib.library().wfx_template_polarization_overlap(
        model, _ptr(table), _ptr(freqs), batch, n, _ptr(t_c), _ptr(signal), _ptr(psd), float(delta_f), _ptr(series),
        series.shape[1], _ptr(norms), _stream(table.device)))
    return norms


def polarization_refine(series: torch.Tensor, zgrid: Optional[torch.Tensor], freqs: torch.Tensor, delta_f: float,
                        norms: torch.Tensor, *, time: bool = True, steps: int = 3):
    """The polarization matches of the ``series.shape[0] // 2`` rows:
    ``(match, t)``, float64."""
    precision = _lib.FP64 if series.dtype == torch.complex128 else _lib.FP32
    _require(series, "series", series.dtype)
    _require(freqs, "freqs", torch.float64)
    _require(norms, "norms", torch.float64)
    if time:
        _require(zgrid, "zgrid", series.dtype)
    rows, n_fft = series.shape[0] // 2, series.shape[1]
    out = torch.empty(rows, dtype=torch.float64, device=series.device)
    t = torch.empty(rows, dtype=torch.float64, device=series.device)
    _lib.check("wfx_polarization_refine", _lib.library().wfx_polarization_refine(
        precision, _ptr(series), _ptr(zgrid) if time else None, rows, freqs.numel(), n_fft, _ptr(freqs),
        float(delta_f), _ptr(norms), int(bool(time)), int(steps), _ptr(out), _ptr(t), _stream(series.device)))
    return out, t
