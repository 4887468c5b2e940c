"""The models as PyTorch functions on the B200 kernels: the drop-in for
``waveformx.torch.polarizations_function`` (reference
``src/waveformx/torch.py:175-183``).

``polarizations_function(approximant, options=None, **option_keywords)``
returns ``f(binary, frequencies, t_c=None) -> (hplus, hcross)``:

* ``binary`` is a :class:`~waveformx_b200.Binary` or a mapping of its
  fields (``mass_1``, ``mass_2``, ``spin_1``, ``spin_2`` required; unknown
  names raise ``TypeError``), as tensors, numbers or sequences, with an
  optional leading batch axis (``spin_*`` then ``(n, 3)``; unbatched fields
  are broadcast, differing batch sizes raise ``ValueError``);
* the precision follows the inputs: float32 if every floating-point tensor
  is float32 (the FP32 kernels with double-float phase; complex64 out),
  else float64 (the plain FP64 kernels; complex128 out);
* the output is on the device of ``frequencies`` (CPU tensors are computed
  on the current CUDA device and copied back), of shape ``(N,)``, or
  ``(n, N)`` for a batch;
* ``loss.backward()`` reaches every field that requires a gradient (the
  spins' in-plane components get zero) through the hand-written backward
  kernel, which recomputes the waveform; first derivatives only;
* ``t_c`` (s; a keyword, or a ``t_c`` entry of the mapping) multiplies the
  strain by ``exp(-2 pi i f t_c)``, with its gradient: an extension of the
  reference (``t_c = None`` reproduces it).

Like the reference's, the function makes no parameter checks: a binary LAL
refuses gives NaN.
"""

from __future__ import annotations

from typing import Any, Callable, Mapping, Optional

import numpy as np
import torch

from . import _lib, ops
from ._binary import BINARY_NAMES, Binary
from ._options import WaveformOptions, parse_options, strain_scale
from .exceptions import KernelError

__all__ = ["polarizations_function"]


def _fields(binary: Any):
    """The eight fields of a Binary or mapping, and the mapping's ``t_c``."""
    if isinstance(binary, Binary):
        return list(binary), None
    if isinstance(binary, Mapping):
        unknown = set(binary) - set(BINARY_NAMES) - {"t_c"}
        if unknown:
            raise TypeError(f"unknown fields of a Binary: {sorted(unknown)}")
        missing = [name for name in BINARY_NAMES[:4] if name not in binary]
        if missing:
            raise TypeError(f"missing fields of a Binary: {missing}")
        return [binary.get(name, Binary._field_defaults.get(name)) for name in BINARY_NAMES], binary.get("t_c")
    raise TypeError(f"binary must be a waveformx_b200.Binary or a mapping of its fields, got {type(binary).__name__}")


def _tensors(value: Any) -> list:
    if isinstance(value, torch.Tensor):
        return [value]
    if isinstance(value, (list, tuple)):
        return [x for item in value for x in _tensors(item)]
    return []


def _as_tensor(value: Any, dtype: torch.dtype, device: torch.device) -> torch.Tensor:
    if isinstance(value, torch.Tensor):
        return value.to(device=device, dtype=dtype)
    if isinstance(value, (list, tuple)) and _tensors(value):
        return torch.stack([_as_tensor(x, dtype, device) for x in value])
    return torch.as_tensor(np.asarray(value, dtype=np.float64), dtype=dtype, device=device)


def _compute_device(device: torch.device) -> torch.device:
    if device.type == "cuda":
        return device
    if not torch.cuda.is_available():
        raise KernelError("waveformx_b200 runs on a CUDA device and none is available")
    return torch.device("cuda", torch.cuda.current_device())


class _Polarizations(torch.autograd.Function):
    """``(hplus, hcross)`` of the grid, ``t_c`` and the eight fields (each
    ``(n,)`` or ``(n, 3)``, batched), with the backward kernel."""

    @staticmethod
    def forward(ctx, key, out_device, grid, t_c, *fields):
        approximant, options = key
        cdev = _compute_device(grid.device)
        real = grid.dtype
        precision = _lib.FP32 if real == torch.float32 else _lib.FP64
        f = grid.detach().to(device=cdev).contiguous()
        m1, m2, s1, s2, dist, incl, phi, f_ref = (x.detach().to(device=cdev) for x in fields)
        params = torch.stack([m1, m2, s1[..., 2], s2[..., 2], dist, incl, phi, f_ref], dim=-1)
        params = params.to(torch.float64).contiguous()
        f_min = f[:1].to(torch.float64)
        needs = any(ctx.needs_input_grad[3:])
        xhm = ops.model_code(approximant) == _lib.XHM
        ctx.key, ctx.out_device = key, out_device
        ctx.empty = None
        if params.shape[0] == 0 or f.numel() == 0:
            # (no binary or no frequency: empty outputs, as the reference's
            # vmapped function gives; nothing to launch)
            complex_dtype = torch.complex64 if precision == _lib.FP32 else torch.complex128
            ctx.empty = (params.shape[0], f.numel(), real)
            hp = torch.zeros((params.shape[0], f.numel()), dtype=complex_dtype, device=out_device)
            return hp, torch.zeros_like(hp)
        dtable = ready = None
        if needs and not xhm:
            # (the derivatives of the tables on a second stream while the
            # value set-up and the forward run; the backward waits for them)
            dtable, ready = ops.setup_jvp_async(approximant, params, f_min, amp_scale=strain_scale(options),
                                                reference_mf=options.reference_mf)
        tables = ops.setup(approximant, params, f_min, amp_scale=strain_scale(options),
                           reference_mf=options.reference_mf, precision=precision)
        tc = None if t_c is None else t_c.detach().to(device=cdev, dtype=real).contiguous()
        hp, hc = ops.polarizations(approximant, tables.table, f, None, tc)
        if (needs or ctx.needs_input_grad[2]) and xhm:
            # (IMRPhenomXHM: its backward takes the set-up's tangents itself)
            ctx.save_for_backward(params, f_min, f, tc if tc is not None else f[:0])
        elif needs or ctx.needs_input_grad[2]:
            # (the grid's derivative: from the FP64 table of the parameters)
            ctx.save_for_backward(tables.table, dtable, f, tc if tc is not None else f[:0], params, f_min)
        ctx.key, ctx.out_device, ctx.has_tc, ctx.ready, ctx.xhm = key, out_device, tc is not None, ready, xhm
        return hp.to(out_device), hc.to(out_device)

    @staticmethod
    @torch.autograd.function.once_differentiable
    def backward(ctx, g_hp, g_hc):
        approximant, options = ctx.key
        if ctx.empty is not None:
            n, n_freq, real = ctx.empty
            need = ctx.needs_input_grad
            zeros = lambda shape, i: torch.zeros(shape, dtype=real, device=ctx.out_device) if need[i] else None  # noqa: E731
            fields = [zeros((n, 3) if i in (2, 3) else (n,), 4 + i) for i in range(8)]
            return (None, None, zeros((n_freq,), 2), zeros((n,), 3), *fields)
        if ctx.xhm:
            params, f_min, f, tc = ctx.saved_tensors
            table = params
        else:
            table, dtable, f, tc, params, f_min = ctx.saved_tensors
            if ctx.ready is not None:
                torch.cuda.current_stream(table.device).wait_event(ctx.ready)
        tc = tc if ctx.has_tc else None
        complex_dtype = torch.complex64 if f.dtype == torch.float32 else torch.complex128
        shape = (table.shape[0], f.numel())

        def cot(g):
            if g is None:
                return torch.zeros(shape, dtype=complex_dtype, device=table.device)
            return g.to(device=table.device, dtype=complex_dtype).contiguous()

        # PyTorch's gradient with respect to h is dL/dRe h + i dL/dIm h: the
        # kernels' cotangent convention
        grad_grid = None
        if ctx.needs_input_grad[2]:
            table64 = ops.setup(approximant, params, f_min, amp_scale=strain_scale(options),
                                reference_mf=options.reference_mf, precision=_lib.FP64).table
            grad_grid = ops.grid_vjp(approximant, table64, f.to(torch.float64), None,
                                     None if tc is None else tc.to(torch.float64), cot(g_hp), cot(g_hc))
            grad_grid = grad_grid.to(dtype=f.dtype, device=ctx.out_device)
        if not any(ctx.needs_input_grad[3:]):
            return (None, None, grad_grid, None) + (None,) * 8
        if ctx.xhm:
            grad = ops.xhm_vjp(params, f_min, f.to(torch.float64), None, None if tc is None else tc.to(torch.float64),
                               cot(g_hp), cot(g_hc), amp_scale=strain_scale(options),
                               reference_mf=options.reference_mf).to(f.dtype)
        else:
            grad = ops.vjp(approximant, table, dtable, f, None, tc, cot(g_hp), cot(g_hc))
        grad = grad.to(ctx.out_device)
        zeros = torch.zeros_like(grad[:, 0])
        spin = lambda col: torch.stack([zeros, zeros, grad[:, col]], dim=-1)  # noqa: E731
        by_field = [grad[:, 0], grad[:, 1], spin(2), spin(3), grad[:, 4], grad[:, 5], grad[:, 6], grad[:, 7]]
        need = ctx.needs_input_grad
        out = [None, None, grad_grid, grad[:, 8] if (need[3] and ctx.has_tc) else None]
        out += [g if need[4 + i] else None for i, g in enumerate(by_field)]
        return tuple(out)


def _wrap(approximant: str, options: WaveformOptions) -> Callable:
    ops.model_code(approximant)

    def function(binary: Any, grid: Any, t_c: Optional[Any] = None):
        fields, mapped_tc = _fields(binary)
        if t_c is None:
            t_c = mapped_tc
        values = [*fields, grid] + ([t_c] if t_c is not None else [])
        tensors = [t for v in values for t in _tensors(v)]
        floats = [t for t in tensors if t.is_floating_point()]
        dtype = torch.float32 if floats and all(t.dtype == torch.float32 for t in floats) else torch.float64
        device = grid.device if isinstance(grid, torch.Tensor) else tensors[0].device if tensors else torch.device("cpu")
        fields = [_as_tensor(v, dtype, device) for v in fields]
        grid_t = _as_tensor(grid, dtype, device)
        sizes = {x.shape[0] for i, x in enumerate(fields) if x.ndim > (1 if i in (2, 3) else 0)}
        tc = None if t_c is None else _as_tensor(t_c, dtype, device)
        if tc is not None and tc.ndim > 0:
            sizes.add(tc.shape[0])
        if len(sizes) > 1:
            raise ValueError(f"the batch axes of the binary's fields differ: {sorted(sizes)}")
        batched = bool(sizes)
        n = sizes.pop() if batched else 1
        fields = [torch.broadcast_to(x, (n, 3) if i in (2, 3) else (n,)) for i, x in enumerate(fields)]
        if tc is not None:
            tc = torch.broadcast_to(tc, (n,))
        hp, hc = _Polarizations.apply((approximant, options), device, grid_t, tc, *fields)
        if not batched:
            hp, hc = hp[0], hc[0]
        return hp, hc

    function.__name__ = "polarizations"
    function.__qualname__ = f"{approximant}.polarizations"
    return function


def polarizations_function(approximant: str, options: Optional[WaveformOptions] = None,
                           **option_keywords) -> Callable:
    """The PyTorch function ``f(binary, frequencies, t_c=None) -> (hplus,
    hcross)`` of IMRPhenomXAS, IMRPhenomD or TaylorF2 on the B200 kernels
    (see the module's documentation)."""
    return _wrap(approximant, parse_options(options, option_keywords))
