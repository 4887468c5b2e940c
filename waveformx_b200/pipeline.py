"""Polarizations of a stream of batches, each batch's set-up overlapping the
previous batch's forward.

A batch's FP64 set-up is one latency-bound chain per binary (about 33 us
for IMRPhenomXAS at any batch size: one warp on each of 128 SMs, waiting on
instruction fetch), while the FP32 forward of a 4096 x 4017 batch takes
about 66 us over every SM. One after the other, the set-up is a third of a
batch's time. :func:`polarizations_stream` runs the set-up of batch k + 1
on a second stream of higher priority while batch k's forward runs on the
current one: the set-up's blocks take one warp's registers on the SMs they
land on, next to three of the forward's four blocks. Two table buffers
alternate; each is rewritten only after the forward that read it has
finished. Every batch still gets its own set-up and forward, with the same
results as :func:`ops.setup` followed by :func:`ops.polarizations`.
"""

from __future__ import annotations

import ctypes
from typing import Iterable, Iterator, Optional

import torch

from . import _lib, ops

__all__ = ["polarizations_stream"]

_HIGH_PRIORITY_STREAMS: dict = {}


def _setup_stream(device: torch.device) -> torch.cuda.Stream:
    """A second stream of ``device`` at the highest priority (one per device,
    kept), so that a set-up's blocks are placed before the forward's."""
    key = torch.device(device).index
    stream = _HIGH_PRIORITY_STREAMS.get(key)
    if stream is None:
        high, _ = torch.cuda.Stream.priority_range()
        stream = torch.cuda.Stream(device=device, priority=high)
        _HIGH_PRIORITY_STREAMS[key] = stream
    return stream


def _split(item):
    if isinstance(item, (tuple, list)):
        if len(item) != 2:
            raise ValueError("a batch is params or (params, t_c)")
        return item[0], item[1]
    return item, None


def polarizations_stream(approximant: str, batches: Iterable, freqs: torch.Tensor,
                         offsets: Optional[torch.Tensor] = None, *, f_min: Optional[torch.Tensor] = None,
                         amp_scale: float = 1e21, reference_mf: Optional[float] = None,
                         precision: int = _lib.FP32) -> Iterator:
    """``(hplus, hcross, status)`` of each batch of ``batches``, in order.

    A batch is a ``(B, 8)`` float64 CUDA tensor of parameters (masses,
    aligned spins, distance, inclination, phi_ref, f_ref), or ``(params,
    t_c)``; every batch has the same B. ``freqs``: the shared grid, or with
    ``offsets`` the flat grids of a ragged batch, in the precision's real
    type. ``f_min``: the first frequency of each binary (default: the grid's
    first). The outputs of a batch are ready on the current stream when it is
    yielded, as those of :func:`ops.polarizations`, and so is the batch's own
    ``status`` tensor."""
    model = ops.model_code(approximant)
    if model == _lib.XHM:
        stride = _lib.XHM_STRIDE32 if precision == _lib.FP32 else _lib.XHM_STRIDE64
    else:
        stride = _lib.TABLE_STRIDE
    real = torch.float32 if precision == _lib.FP32 else torch.float64
    device = freqs.device
    if f_min is None:
        if offsets is None:
            f_min = freqs[:1].to(torch.float64)
        else:
            first = offsets[:-1].clamp(max=max(freqs.numel() - 1, 0))
            f_min = freqs[first].to(torch.float64)
    f_min = f_min.to(device, torch.float64).contiguous()
    rmf = float("nan") if reference_mf is None else float(reference_mf)
    lib = _lib.library()
    main = torch.cuda.current_stream(device)
    side = _setup_stream(device)
    main_handle = ctypes.c_void_p(main.cuda_stream)
    side_handle = ctypes.c_void_p(side.cuda_stream)
    fstride = 0 if f_min.numel() == 1 else 1
    f_min_ptr = ops._ptr(f_min)
    complex_dtype = torch.complex64 if precision == _lib.FP32 else torch.complex128
    n = freqs.numel()
    shape_of = None
    tables = None
    ws = None
    fork = [torch.cuda.Event(), torch.cuda.Event()]
    ready = [torch.cuda.Event(), torch.cuda.Event()]
    batch = None

    def launch_setup(slot, params):
        """Batch ``params``'s set-up into table ``slot`` on the second stream;
        its status, allocated on the current stream."""
        nonlocal tables, batch, shape_of, ws
        ops._require(params, "params", torch.float64)
        if params.ndim != 2 or params.shape[1] != 8 or params.shape[0] == 0:
            raise ValueError("params must be (B, 8) with B > 0")
        if batch is None:
            batch = params.shape[0]
            if f_min.numel() not in (1, batch):
                raise ValueError("f_min must have one value or one per binary")
            # (allocated on the current stream, which every set-up waits for)
            tables = [torch.empty((batch, stride), dtype=real, device=device) for _ in range(2)]
            if model != _lib.XHM:
                ops._grid(tables[0], freqs, offsets, None)
                shape_of = (batch, n) if offsets is None else (n,)
                # (the forwards run one after the other on the current stream)
                ws = ops.workspace(_lib.OP_POLARIZATIONS, model, precision, batch, n, offsets is not None, device)
        elif params.shape[0] != batch:
            raise ValueError("every batch must have the same number of binaries")
        status = torch.empty(batch, dtype=torch.int32, device=device)
        table = tables[slot]
        t64 = ops._ptr(table) if precision == _lib.FP64 else None
        t32 = ops._ptr(table) if precision == _lib.FP32 else None
        # after everything queued so far on the current stream: the batch's
        # parameters, and the forward that last read this slot
        fork[slot].record(main)
        side.wait_event(fork[slot])
        if model == _lib.XHM:
            rc = lib.wfx_xhm_setup(ops._ptr(params), batch, f_min_ptr, fstride, float(amp_scale), rmf, t64, t32,
                                   ops._ptr(status), side_handle)
            _lib.check("wfx_xhm_setup", rc)
        else:
            rc = lib.wfx_setup(model, ops._ptr(params), batch, f_min_ptr, fstride, float(amp_scale), rmf, t64, t32,
                               ops._ptr(status), side_handle)
            _lib.check("wfx_setup", rc)
        ready[slot].record(side)
        return status

    def forward(slot, t_c):
        if t_c is not None:
            t_c = torch.as_tensor(t_c, dtype=real, device=device)
        if model == _lib.XHM:
            return ops.polarizations(approximant, tables[slot], freqs, offsets, t_c)
        if t_c is not None:
            ops._require(t_c, "t_c", real)
            if t_c.numel() != batch:
                raise ValueError("t_c must have one value per binary")
        hp = torch.empty(shape_of, dtype=complex_dtype, device=device)
        hc = torch.empty(shape_of, dtype=complex_dtype, device=device)
        _lib.check("wfx_polarizations", lib.wfx_polarizations(
            model, precision, ops._ptr(tables[slot]), ops._ptr(freqs), ops._ptr(offsets), batch, n, ops._ptr(t_c),
            ops._ptr(hp), ops._ptr(hc), ops._ptr(ws), 0 if ws is None else ws.numel(), main_handle))
        return hp, hc

    it = iter(batches)
    try:
        current = _split(next(it))
    except StopIteration:
        return
    slot = 0
    try:
        status = launch_setup(0, current[0])
        while current is not None:
            try:
                following = _split(next(it))
            except StopIteration:
                following = None
            next_status = launch_setup(1 - slot, following[0]) if following is not None else None
            main.wait_event(ready[slot])
            hp, hc = forward(slot, current[1])
            yield hp, hc, status
            current, status = following, next_status
            slot = 1 - slot
    finally:
        # (a set-up still writing a buffer when the stream is left: the
        # buffers are freed on the current stream, after it)
        main.wait_stream(side)
