"""Polarizations of a stream of batches, each batch's set-up overlapping the
previous batch's forward.

A batch's FP64 set-up is one latency-bound chain per binary (about 33 us
for IMRPhenomXAS at any batch size, waiting on instruction fetch), while
the FP32 forward of a 4096 x 4017 batch takes
about 66 us over every SM. One after the other, the set-up is a third of a
batch's time. :func:`polarizations_stream` runs the set-up of batch k + 1
on a second stream of higher priority while batch k's forward runs on the
current one: the set-up's blocks (four warps, 4096 binaries on 32 SMs)
take two of the forward's four block slots on the SMs they land on. Two
table buffers alternate; each is rewritten only after the forward that read
it has finished. Each batch costs two calls into the library
(``wfx_pipeline_setup``, ``wfx_pipeline_forward``: the events and launches
in C), so that the host keeps ahead of the device. Every batch still gets
its own set-up and forward, with the same results as :func:`ops.setup`
followed by :func:`ops.polarizations`.
"""

from __future__ import annotations

import ctypes
from typing import Iterable, Iterator, Optional

import torch

from . import _lib, ops

__all__ = ["likelihood_stream", "likelihood_batches", "polarizations_stream", "polarizations_batches", "Pipeline"]


def _split(item):
    if isinstance(item, (tuple, list)):
        if len(item) != 2:
            raise ValueError("a batch is params or (params, t_c)")
        return item[0], item[1]
    return item, None


#: The binaries that one set-up launch of polarizations_batches takes by
#: default (IMRPhenomXAS on a B200: the set-up takes 36 us for 4096 or 16384
#: binaries, 109 us for 81920; 20 batches of 4096 x 4017 take 67.3-67.7 us a
#: batch with one batch a set-up, 67.3-67.9 with 2, 68.0-68.4 with 4,
#: 70.2-70.7 with 20, against 62.5 us for the forwards alone).
SETUP_BINARIES = 8192

#: The binaries that one dual-number set-up launch of likelihood_batches
#: takes by default (IMRPhenomXAS on a B200, batches of 1024 x 4017: 109 us
#: a batch with one batch a launch, 95 with 2, 91 with 4, 96 with 8, 94 with
#: 16; the dual-number set-up of 16384 binaries runs in several waves).
LIKELIHOOD_SETUP_BINARIES = 4096


class Pipeline:
    """A pipeline's streams and events on one device (``wfx_pipeline_create``),
    kept for repeated :func:`polarizations_batches` and
    :func:`likelihood_batches` calls so that none of them pays for creating
    streams. One sequence of batches at a time; a context manager (closed on
    exit)."""

    def __init__(self, device=None):
        self.device = torch.device("cuda", torch.cuda.current_device()) if device is None else torch.device(device)
        self.handle = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            _lib.check("wfx_pipeline_create", _lib.library().wfx_pipeline_create(ctypes.byref(self.handle)))

    def close(self):
        """Release the streams and events (waits for the pipeline's streams)."""
        if self.handle:
            with torch.cuda.device(self.device):
                _lib.library().wfx_pipeline_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
        return False

    def __del__(self):
        try:
            self.close()
        except Exception:  # interpreter shutdown
            pass


def polarizations_batches(approximant: str, params: torch.Tensor, freqs: torch.Tensor,
                          offsets: Optional[torch.Tensor] = None, *, t_c: Optional[torch.Tensor] = None,
                          f_min: Optional[torch.Tensor] = None, amp_scale: float = 1e21,
                          reference_mf: Optional[float] = None, precision: int = _lib.FP32, ring: Optional[int] = None,
                          group: Optional[int] = None, out=None, pipeline: Optional[Pipeline] = None,
                          status: Optional[torch.Tensor] = None, tables: Optional[torch.Tensor] = None):
    """K batches of ``params`` (``(K, B, 8)`` float64 CUDA) through the
    pipeline in one library call (``wfx_pipeline_run``): each batch's set-up
    on the pipeline's second stream during the previous batch's forward, the
    forwards in order on the current stream. ``t_c``: ``(K, B)`` or None.
    Batch k's ``(hplus, hcross)`` go to slot ``k % ring`` of the returned
    ``(ring, B, N)`` (ragged: ``(ring, n)``) outputs (``ring`` defaults to K;
    complex64 slots of an odd size are one element apart, so every slot is
    16-byte aligned; ``out``: a previous call's pair to fill again);
    ``status`` is ``(K, B)``. ``group``: the batches whose set-ups run in one
    launch, during the previous group's forwards (default: as many as make
    up to 8192 binaries, when every binary has the same ``f_min``; the
    set-up's time hardly depends on its number of binaries). ``status`` (``(K,
    B)`` int32) and ``tables`` (``(2, group, B, row)`` of the precision's
    real type): buffers to use instead of new ones (a caller that times the
    call allocates them beforehand).
    Returns ``(hplus, hcross, status)``, ready on the current stream. Every
    batch gets its own set-up and forward: the same results as
    :func:`ops.setup` and :func:`ops.polarizations` batch by batch."""
    model = ops.model_code(approximant)
    if not (isinstance(params, torch.Tensor) and params.is_cuda and params.dtype == torch.float64
            and params.ndim == 3 and params.shape[2] == 8 and params.shape[0] > 0 and params.shape[1] > 0):
        raise ValueError("params must be a (K, B, 8) float64 CUDA tensor with K, B > 0")
    params = params.contiguous()
    K, batch = params.shape[0], params.shape[1]
    device = params.device
    real = torch.float32 if precision == _lib.FP32 else torch.float64
    complex_dtype = torch.complex64 if precision == _lib.FP32 else torch.complex128
    ops._require(freqs, "freqs", real)
    n = freqs.numel()
    if model == _lib.XHM:
        stride = _lib.XHM_STRIDE32 if precision == _lib.FP32 else _lib.XHM_STRIDE64
    else:
        stride = _lib.TABLE_STRIDE
    max_len = 0
    if offsets is not None:
        ops.check_offsets(offsets, batch, n)
        if model == _lib.XHM:
            max_len = int((offsets[1:] - offsets[:-1]).max())
    if f_min is None:
        if offsets is None:
            f_min = freqs[:1].to(torch.float64)
        else:
            f_min = freqs[offsets[:-1].clamp(max=max(n - 1, 0))].to(torch.float64)
    f_min = f_min.to(device, torch.float64).contiguous()
    if f_min.numel() not in (1, batch):
        raise ValueError("f_min must have one value or one per binary")
    if t_c is not None:
        t_c = torch.as_tensor(t_c, dtype=real, device=device).contiguous()
        if t_c.numel() != K * batch:
            raise ValueError("t_c must be (K, B)")
    ring = K if ring is None else int(ring)
    # (slot r starts at element r * slot: complex64 slots of an odd count are
    # padded by one element, so that every slot is 16-byte aligned)
    elems = batch * n if offsets is None else n
    slot = elems + (elems & 1) if precision == _lib.FP32 else elems
    shape = (ring, batch, n) if offsets is None else (ring, n)
    strides = (slot, n, 1) if offsets is None else (slot, 1)
    if out is None:
        hp, hc = (torch.as_strided(torch.empty(ring * slot, dtype=complex_dtype, device=device), shape, strides)
                  for _ in range(2))
    else:
        hp, hc = out
        for name, t in (("hplus", hp), ("hcross", hc)):
            if not isinstance(t, torch.Tensor) or t.dtype != complex_dtype or not t.is_cuda:
                raise TypeError(f"{name} must be a {complex_dtype} CUDA tensor")
            if tuple(t.shape) != shape or tuple(t.stride()) != strides:
                raise ValueError(f"{name} must be {shape} with strides {strides} (a previous call's output)")
    if group is None:
        group = max(1, min(K, SETUP_BINARIES // batch)) if f_min.numel() == 1 else 1
    group = int(group)
    if group > 1 and f_min.numel() != 1:
        raise ValueError("group > 1 needs one f_min for every binary")
    if tables is None:
        tables = torch.empty((2, group, batch, stride), dtype=real, device=device)
    elif tuple(tables.shape) != (2, group, batch, stride) or tables.dtype != real or not tables.is_contiguous():
        raise ValueError(f"tables must be a contiguous ({2}, {group}, {batch}, {stride}) {real} tensor")
    if status is None:
        status = torch.empty((K, batch), dtype=torch.int32, device=device)
    elif tuple(status.shape) != (K, batch) or status.dtype != torch.int32 or not status.is_contiguous():
        raise ValueError(f"status must be a contiguous ({K}, {batch}) int32 tensor")
    ws = None
    if model != _lib.XHM:
        ws = ops.workspace(_lib.OP_POLARIZATIONS, model, precision, batch, n, offsets is not None, device)
    own = pipeline is None
    pipe = Pipeline(device) if own else pipeline
    try:
        with torch.cuda.device(device):
            _lib.check("wfx_pipeline_run", _lib.library().wfx_pipeline_run(
                pipe.handle, model, precision, K, params.data_ptr(), batch, f_min.data_ptr(),
                0 if f_min.numel() == 1 else 1, float(amp_scale),
                float("nan") if reference_mf is None else float(reference_mf), tables.data_ptr(),
                status.data_ptr(), freqs.data_ptr(), None if offsets is None else offsets.data_ptr(), n, max_len,
                None if t_c is None else t_c.data_ptr(), hp.data_ptr(), hc.data_ptr(), ring, group,
                None if ws is None else ws.data_ptr(), 0 if ws is None else ws.numel(),
                torch.cuda.current_stream(device).cuda_stream))
    finally:
        if own:
            pipe.close()
    return hp, hc, status


def likelihood_batches(approximant: str, params: torch.Tensor, freqs: torch.Tensor, data: torch.Tensor,
                       weights: torch.Tensor, offsets: Optional[torch.Tensor] = None, *,
                       t_c: Optional[torch.Tensor] = None, f_min: Optional[torch.Tensor] = None,
                       antenna=(1.0, 0.0), scale: float = 1.0, amp_scale: float = 1e21,
                       reference_mf: Optional[float] = None, group: Optional[int] = None,
                       pipeline: Optional[Pipeline] = None, out=None, status: Optional[torch.Tensor] = None,
                       tables=None, workspace: Optional[torch.Tensor] = None):
    """The FP32 fused likelihood ``scale sum_f w |F+ h+ + Fx hx - d|^2`` and
    its ``(B, 9)`` gradient for K batches of ``params`` (``(K, B, 8)``
    float64 CUDA) in one library call (``wfx_pipeline_likelihood_run``): the
    dual-number set-ups of ``group`` batches in one launch on a further
    stream (they write the tables too), during the previous group's fused
    likelihoods on the current stream, each batch's contraction with dtable
    on a second stream beside the next batch's reverse pass. ``t_c``: ``(K, B)`` or None;
    ``freqs``, ``offsets``, ``data``, ``weights`` and ``f_min`` as
    :func:`likelihood_stream`, the same for every batch. ``group``: default
    as many batches as make up to 4096 binaries, when every binary has the
    same ``f_min``. ``out`` (``(loss (K, B), grad (K, B, 9))`` float32),
    ``status`` (``(K, B)`` int32) and ``tables`` (``((2, group, B, 72)``
    float32, ``(2, group, B, 72, 8)`` float64)) and ``workspace`` (uint8, at
    least twice ``wfx_workspace_bytes(WFX_OP_FUSED, ...)``): buffers to use
    instead of new ones (a caller that times the call allocates them
    beforehand). Returns ``(loss, grad, status)``, ready on the current
    stream: the values of :func:`ops.fused_loss_from_params` batch by
    batch."""
    model = ops.model_code(approximant)
    ops._differentiable(model)
    if not (isinstance(params, torch.Tensor) and params.is_cuda and params.dtype == torch.float64
            and params.ndim == 3 and params.shape[2] == 8 and params.shape[0] > 0 and params.shape[1] > 0):
        raise ValueError("params must be a (K, B, 8) float64 CUDA tensor with K, B > 0")
    params = params.contiguous()
    K, batch = params.shape[0], params.shape[1]
    device = params.device
    ops._require(freqs, "freqs", torch.float32)
    ops._require(data, "data", torch.complex64)
    ops._require(weights, "weights", torch.float32)
    n = freqs.numel()
    ragged = offsets is not None
    if ragged:
        ops.check_offsets(offsets, batch, n)
    data_stride = ops.check_per_frequency(data, "data", batch, n, ragged)
    weights_stride = ops.check_per_frequency(weights, "weights", batch, n, ragged)
    if f_min is None:
        if offsets is None:
            f_min = freqs[:1].to(torch.float64)
        else:
            f_min = freqs[offsets[:-1].clamp(max=max(n - 1, 0))].to(torch.float64)
    f_min = f_min.to(device, torch.float64).contiguous()
    if f_min.numel() not in (1, batch):
        raise ValueError("f_min must have one value or one per binary")
    if t_c is not None:
        t_c = torch.as_tensor(t_c, dtype=torch.float32, device=device).contiguous()
        if t_c.numel() != K * batch:
            raise ValueError("t_c must be (K, B)")
    if group is None:
        group = max(1, min(K, LIKELIHOOD_SETUP_BINARIES // batch)) if f_min.numel() == 1 else 1
    group = int(group)
    if group > 1 and f_min.numel() != 1:
        raise ValueError("group > 1 needs one f_min for every binary")
    row = _lib.TABLE_STRIDE
    if tables is None:
        tables = (torch.empty((2, group, batch, row), dtype=torch.float32, device=device),
                  torch.empty((2, group, batch, row, 8), dtype=torch.float64, device=device))
    table32, dtables = tables
    if (tuple(table32.shape) != (2, group, batch, row) or table32.dtype != torch.float32
            or not table32.is_contiguous() or tuple(dtables.shape) != (2, group, batch, row, 8)
            or dtables.dtype != torch.float64 or not dtables.is_contiguous()):
        raise ValueError(f"tables must be contiguous (2, {group}, {batch}, {row}) float32 and "
                         f"(2, {group}, {batch}, {row}, 8) float64 tensors")
    if out is None:
        out = (torch.empty((K, batch), dtype=torch.float32, device=device),
               torch.empty((K, batch, _lib.GRAD_COLUMNS), dtype=torch.float32, device=device))
    loss, grad = out
    if (tuple(loss.shape) != (K, batch) or loss.dtype != torch.float32 or not loss.is_contiguous()
            or tuple(grad.shape) != (K, batch, _lib.GRAD_COLUMNS) or grad.dtype != torch.float32
            or not grad.is_contiguous()):
        raise ValueError(f"out must be contiguous ({K}, {batch}) and ({K}, {batch}, {_lib.GRAD_COLUMNS}) float32")
    if status is None:
        status = torch.empty((K, batch), dtype=torch.int32, device=device)
    elif tuple(status.shape) != (K, batch) or status.dtype != torch.int32 or not status.is_contiguous():
        raise ValueError(f"status must be a contiguous ({K}, {batch}) int32 tensor")
    # (two halves: a batch's contraction reads one while the next batch's
    # reverse pass fills the other)
    half = int(_lib.library().wfx_workspace_bytes(_lib.OP_FUSED, model, _lib.FP32, batch, n, int(ragged)))
    if workspace is None:
        ws = torch.empty(2 * half, dtype=torch.uint8, device=device)
    else:
        ws = workspace
        if ws.dtype != torch.uint8 or not ws.is_cuda or not ws.is_contiguous() or ws.numel() < 2 * half:
            raise ValueError(f"workspace must be a contiguous uint8 CUDA tensor of at least {2 * half} bytes")
    own = pipeline is None
    pipe = Pipeline(device) if own else pipeline
    try:
        with torch.cuda.device(device):
            _lib.check("wfx_pipeline_likelihood_run", _lib.library().wfx_pipeline_likelihood_run(
                pipe.handle, model, K, params.data_ptr(), batch, f_min.data_ptr(), 0 if f_min.numel() == 1 else 1,
                float(amp_scale), float("nan") if reference_mf is None else float(reference_mf),
                table32.data_ptr(), dtables.data_ptr(), status.data_ptr(), freqs.data_ptr(),
                None if offsets is None else offsets.data_ptr(), n, None if t_c is None else t_c.data_ptr(),
                data.data_ptr(), data_stride, weights.data_ptr(), weights_stride, float(antenna[0]),
                float(antenna[1]), float(scale), loss.data_ptr(), grad.data_ptr(), group, ws.data_ptr(),
                ws.numel(), torch.cuda.current_stream(device).cuda_stream))
    finally:
        if own:
            pipe.close()
    return loss, grad, status


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
    main_handle = main.cuda_stream
    fstride = 0 if f_min.numel() == 1 else 1
    f_min_ptr = f_min.data_ptr()
    complex_dtype = torch.complex64 if precision == _lib.FP32 else torch.complex128
    n = freqs.numel()
    freqs_ptr = freqs.data_ptr()
    offsets_ptr = None if offsets is None else offsets.data_ptr()
    max_len = 0
    tables = None
    ws = None
    ws_ptr, ws_n = None, 0
    shape_of = None
    batch = None

    handle = ctypes.c_void_p()
    with torch.cuda.device(device):
        _lib.check("wfx_pipeline_create", lib.wfx_pipeline_create(ctypes.byref(handle)))

    def launch_setup(slot, params):
        """Batch ``params``'s set-up into table ``slot`` on the pipeline's
        second stream; its status, allocated on the current stream."""
        nonlocal tables, batch, shape_of, ws, ws_ptr, ws_n, max_len
        if not (isinstance(params, torch.Tensor) and params.is_cuda and params.dtype == torch.float64
                and params.ndim == 2 and params.shape[1] == 8 and params.shape[0] > 0):
            ops._require(params, "params", torch.float64)
            raise ValueError("params must be (B, 8) with B > 0")
        params = params.contiguous()
        if batch is None:
            batch = params.shape[0]
            if f_min.numel() not in (1, batch):
                raise ValueError("f_min must have one value or one per binary")
            # (allocated on the current stream, which every set-up waits for)
            tables = [torch.empty((batch, stride), dtype=real, device=device) for _ in range(2)]
            if model == _lib.XHM:
                ops._require(freqs, "freqs", real)
                if offsets is not None:
                    ops._require(offsets, "offsets", torch.int64)
                    if offsets.numel() != batch + 1:
                        raise ValueError("offsets must have B + 1 entries")
                    max_len = int((offsets[1:] - offsets[:-1]).max()) if batch else 0
            else:
                ops._grid(tables[0], freqs, offsets, None)
                # (the forwards run one after the other on the current stream)
                ws = ops.workspace(_lib.OP_POLARIZATIONS, model, precision, batch, n, offsets is not None, device)
                ws_ptr, ws_n = (None, 0) if ws is None else (ws.data_ptr(), ws.numel())
            shape_of = (batch, n) if offsets is None else (n,)
        elif params.shape[0] != batch:
            raise ValueError("every batch must have the same number of binaries")
        status = torch.empty(batch, dtype=torch.int32, device=device)
        table = tables[slot].data_ptr()
        t64, t32 = (table, None) if precision == _lib.FP64 else (None, table)
        with torch.cuda.device(device):
            _lib.check("wfx_pipeline_setup", lib.wfx_pipeline_setup(
                handle, slot, model, params.data_ptr(), batch, f_min_ptr, fstride, float(amp_scale), rmf, t64, t32,
                status.data_ptr(), main_handle))
        return params, status

    def forward(slot, t_c):
        if t_c is not None:
            t_c = torch.as_tensor(t_c, dtype=real, device=device)
            ops._require(t_c, "t_c", real)
            if t_c.numel() != batch:
                raise ValueError("t_c must have one value per binary")
        hp = torch.empty(shape_of, dtype=complex_dtype, device=device)
        hc = torch.empty(shape_of, dtype=complex_dtype, device=device)
        with torch.cuda.device(device):
            _lib.check("wfx_pipeline_forward", lib.wfx_pipeline_forward(
                handle, slot, model, precision, tables[slot].data_ptr(), freqs_ptr, offsets_ptr, batch, n, max_len,
                None if t_c is None else t_c.data_ptr(), hp.data_ptr(), hc.data_ptr(), ws_ptr, ws_n, main_handle))
        return hp, hc

    it = iter(batches)
    slot = 0
    try:
        try:
            current = _split(next(it))
        except StopIteration:
            return
        # (`held`: the batch's parameters as the set-up reads them, kept
        # until a later forward of the current stream has waited for it)
        held, status = launch_setup(0, current[0])
        while current is not None:
            try:
                following = _split(next(it))
            except StopIteration:
                following = None
            if following is not None:
                next_held, next_status = launch_setup(1 - slot, following[0])
            else:
                next_held = next_status = None
            hp, hc = forward(slot, current[1])
            yield hp, hc, status
            current, held, status = following, next_held, next_status
            slot = 1 - slot
    finally:
        # (the current stream waits for the second one before the tables and
        # the parameters it read can be freed; then the pipeline goes)
        with torch.cuda.device(device):
            lib.wfx_pipeline_join(handle, main_handle)
            lib.wfx_pipeline_destroy(handle)


def likelihood_stream(approximant: str, batches: Iterable, freqs: torch.Tensor, data: torch.Tensor,
                      weights: torch.Tensor, offsets: Optional[torch.Tensor] = None, *,
                      f_min: Optional[torch.Tensor] = None, antenna=(1.0, 0.0), scale: float = 1.0,
                      amp_scale: float = 1e21, reference_mf: Optional[float] = None) -> Iterator:
    """``(loss, grad, status)`` of each batch of ``batches``: the FP32 fused
    likelihood ``scale sum_f w |F+ h+ + Fx hx - d|^2`` and its ``(B, 9)``
    gradient, as :func:`ops.fused_loss_from_params` gives them (the same
    values), with batch k + 1's value set-up and dual-number set-up on two
    further streams while batch k's fused likelihood runs on the current
    one. Batches, ``freqs``, ``offsets`` and ``f_min`` as
    :func:`polarizations_stream` (FP32 grid); ``data`` (complex64) and
    ``weights`` (float32) per frequency, or per element of the batch's
    grid. Not IMRPhenomXHM (no fused likelihood)."""
    model = ops.model_code(approximant)
    ops._differentiable(model)
    device = freqs.device
    ops._require(freqs, "freqs", torch.float32)
    ops._require(data, "data", torch.complex64)
    ops._require(weights, "weights", torch.float32)
    if f_min is None:
        if offsets is None:
            f_min = freqs[:1].to(torch.float64)
        else:
            first = offsets[:-1].clamp(max=max(freqs.numel() - 1, 0))
            f_min = freqs[first].to(torch.float64)
    f_min = f_min.to(device, torch.float64).contiguous()
    rmf = float("nan") if reference_mf is None else float(reference_mf)
    lib = _lib.library()
    main_handle = torch.cuda.current_stream(device).cuda_stream
    fstride = 0 if f_min.numel() == 1 else 1
    n = freqs.numel()
    state = {}

    handle = ctypes.c_void_p()
    with torch.cuda.device(device):
        _lib.check("wfx_pipeline_create", lib.wfx_pipeline_create(ctypes.byref(handle)))

    def launch_setups(slot, params):
        if not (isinstance(params, torch.Tensor) and params.is_cuda and params.dtype == torch.float64
                and params.ndim == 2 and params.shape[1] == 8 and params.shape[0] > 0):
            ops._require(params, "params", torch.float64)
            raise ValueError("params must be (B, 8) with B > 0")
        params = params.contiguous()
        if not state:
            batch = params.shape[0]
            if f_min.numel() not in (1, batch):
                raise ValueError("f_min must have one value or one per binary")
            tables = [torch.empty((batch, _lib.TABLE_STRIDE), dtype=torch.float32, device=device) for _ in range(2)]
            dtables = [torch.empty((batch, _lib.TABLE_STRIDE, 8), dtype=torch.float64, device=device)
                       for _ in range(2)]
            ops._grid(tables[0], freqs, offsets, None)
            data_stride = ops.check_per_frequency(data, "data", batch, n, offsets is not None)
            weights_stride = ops.check_per_frequency(weights, "weights", batch, n, offsets is not None)
            ws = ops.workspace(_lib.OP_FUSED, model, _lib.FP32, batch, n, offsets is not None, device)
            state.update(batch=batch, tables=tables, dtables=dtables, data_stride=data_stride,
                         weights_stride=weights_stride, ws=ws)
        elif params.shape[0] != state["batch"]:
            raise ValueError("every batch must have the same number of binaries")
        batch = state["batch"]
        status = torch.empty(batch, dtype=torch.int32, device=device)
        with torch.cuda.device(device):
            _lib.check("wfx_pipeline_setup", lib.wfx_pipeline_setup(
                handle, slot, model, params.data_ptr(), batch, f_min.data_ptr(), fstride, float(amp_scale), rmf,
                None, state["tables"][slot].data_ptr(), status.data_ptr(), main_handle))
            _lib.check("wfx_pipeline_setup_jvp", lib.wfx_pipeline_setup_jvp(
                handle, slot, model, params.data_ptr(), batch, f_min.data_ptr(), fstride, float(amp_scale), rmf,
                state["dtables"][slot].data_ptr(), main_handle))
        return params, status

    def fused(slot, t_c):
        batch = state["batch"]
        if t_c is not None:
            t_c = torch.as_tensor(t_c, dtype=torch.float32, device=device)
            ops._require(t_c, "t_c", torch.float32)
            if t_c.numel() != batch:
                raise ValueError("t_c must have one value per binary")
        loss = torch.empty(batch, dtype=torch.float32, device=device)
        grad = torch.empty((batch, _lib.GRAD_COLUMNS), dtype=torch.float32, device=device)
        ws = state["ws"]
        with torch.cuda.device(device):
            _lib.check("wfx_pipeline_fused", lib.wfx_pipeline_fused(
                handle, slot, model, state["tables"][slot].data_ptr(), freqs.data_ptr(),
                None if offsets is None else offsets.data_ptr(), batch, n, None if t_c is None else t_c.data_ptr(),
                data.data_ptr(), state["data_stride"], weights.data_ptr(), state["weights_stride"],
                float(antenna[0]), float(antenna[1]), float(scale), state["dtables"][slot].data_ptr(),
                loss.data_ptr(), grad.data_ptr(), None if ws is None else ws.data_ptr(),
                0 if ws is None else ws.numel(), main_handle))
        return loss, grad

    it = iter(batches)
    slot = 0
    try:
        try:
            current = _split(next(it))
        except StopIteration:
            return
        # (`held`: the batch's parameters as the set-ups read them, kept
        # until a later fused call of the current stream has waited for them)
        held, status = launch_setups(0, current[0])
        while current is not None:
            try:
                following = _split(next(it))
            except StopIteration:
                following = None
            if following is not None:
                next_held, next_status = launch_setups(1 - slot, following[0])
            else:
                next_held = next_status = None
            loss, grad = fused(slot, current[1])
            yield loss, grad, status
            current, held, status = following, next_held, next_status
            slot = 1 - slot
    finally:
        with torch.cuda.device(device):
            lib.wfx_pipeline_join(handle, main_handle)
            lib.wfx_pipeline_destroy(handle)
