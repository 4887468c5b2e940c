"""Matches between waveforms on the B200 kernels: the reference's
``waveformx.match`` (``src/waveformx/match.py:71-187``: ``inner_product``,
``match``, ``mismatch``, ``polarization_match``, ``polarization_mismatch``)
for CUDA tensors, and the same matches for a bank of templates evaluated
from their tables without writing their strain.

The waveforms are frequency series on a common uniform grid, weighted by a
power spectral density on the same grid; ``<a, b> = 4 delta_f Re sum_k a_k
conj(b_k) / S_k``, and ``z(t) = sum_k c_k e^(2 pi i f_k t)`` with ``c =
4 delta_f a conj(b) / S`` is the overlap of ``a`` with ``b`` delayed by
``t``. The match is ``|z(t)|`` (or ``Re z(t)`` without the phase
maximisation) over ``sqrt(<a, a> <b, b>)`` at the best ``t``: the largest
value on the grid of ``pad`` times as many times as frequencies (rounded to
a power of two) that an inverse FFT of ``c`` gives, refined by three Newton
steps on the exact ``z(t)``, as the reference. The overlap series and the
refinement are this library's kernels (``csrc/match.cu``; the templates'
series in ``csrc/kernels.cu``); the transform is cuFFT (``torch.fft``), or,
for complex64 series maximised over the phase with up to 16384
frequencies, this library's transform in shared memory that keeps only
each row's best grid time.

Leading axes of ``a`` and ``b`` broadcast against each other (rows); the
results are float64 tensors of the broadcast shape. complex128 inputs run
in FP64, complex64 ones keep their series in FP32 (the sums of the
refinement are FP64 either way).
"""

from __future__ import annotations

from typing import Optional, Tuple

import torch

from . import _lib, ops
from .exceptions import KernelError

__all__ = ["NEWTON_STEPS", "inner_product", "match", "mismatch", "polarization_match", "polarization_mismatch",
           "template_match", "template_mismatch", "template_polarization_match"]

#: Newton steps that refine the best time of the FFT grid (match.py:70).
NEWTON_STEPS = 3


def _grid(frequencies, device, dtype):
    f = torch.as_tensor(frequencies, device=device).to(torch.float64).contiguous()
    if f.ndim != 1 or f.numel() < 2:
        raise ValueError("frequencies must be a uniform grid of at least two values")
    return f, float(f[1] - f[0]), f.to(dtype).contiguous()


def _require_cuda(t, name):
    if not isinstance(t, torch.Tensor) or t.device.type != "cuda":
        raise KernelError(f"{name} must be a CUDA tensor: the matches run on the B200 kernels")


def inner_product(a: torch.Tensor, b: torch.Tensor, frequencies, psd) -> torch.Tensor:
    """``<a, b> = 4 delta_f Re sum a conj(b) / S`` over the last axis
    (match.py:78-81; no maximisation)."""
    _require_cuda(a, "a")
    f, delta_f, _ = _grid(frequencies, a.device, a.real.dtype)
    s = torch.as_tensor(psd, device=a.device, dtype=a.real.dtype)
    return 4 * delta_f * torch.sum((a * torch.conj(b)).real / s, dim=-1)


_SERIES: dict = {}


def _series_buffer(rows: int, n_fft: int, dtype, device) -> torch.Tensor:
    """A ``(rows, n_fft)`` buffer whose columns from ``n`` stay zero: the
    kernels write only the first ``n`` of each row, so one zeroed buffer
    per shape serves every call (the last one is kept)."""
    key = (rows, n_fft, dtype, device)
    buf = _SERIES.get(key)
    if buf is None:
        _SERIES.clear()
        buf = torch.zeros((rows, n_fft), dtype=dtype, device=device)
        _SERIES[key] = buf
    return buf


def _finish(series, f64, delta_f, norms, time, phase, pad):
    if time and phase and series.dtype == torch.complex64 and ops.grid_time_supported(f64.numel(), series.shape[1]):
        # the grid's best time by the inverse FFT in shared memory (the grid
        # never written), then the refinement from it
        t = ops.match_grid_time(series, f64.numel(), delta_f)
        return ops.match_refine(series, None, f64, delta_f, norms, time=True, phase=True, steps=NEWTON_STEPS,
                                t_start=t)
    zgrid = torch.fft.ifft(series, dim=-1, norm="forward") if time else None
    return ops.match_refine(series, zgrid, f64, delta_f, norms, time=time, phase=phase, steps=NEWTON_STEPS)


def match(a: torch.Tensor, b: torch.Tensor, frequencies, psd, *, time: bool = True, phase: bool = True,
          pad: int = 4, return_time: bool = False):
    """The match of ``a`` and ``b`` maximised over a time shift (``time``)
    and a constant phase (``phase``): match.py:129-147 on the kernels. With
    ``return_time``, also the best time (s) of each row."""
    _require_cuda(a, "a")
    _require_cuda(b, "b")
    if a.dtype != b.dtype or a.dtype not in (torch.complex64, torch.complex128):
        raise TypeError("a and b must both be complex64 or both complex128")
    f64, delta_f, f_real = _grid(frequencies, a.device, a.real.dtype)
    n = f64.numel()
    if a.shape[-1] != n or b.shape[-1] != n:
        raise ValueError("the last axis of a and b must hold one value per frequency")
    s = torch.as_tensor(psd, device=a.device, dtype=a.real.dtype).contiguous()
    shape = torch.broadcast_shapes(a.shape[:-1], b.shape[:-1])
    rows = 1
    for d in shape:
        rows *= d

    def flat(x):
        # (a one-dimensional waveform is one vector for every row)
        return x.contiguous() if x.ndim == 1 else x.expand(*shape, n).reshape(rows, n).contiguous()

    flat_a, flat_b = flat(a), flat(b)
    n_fft = ops.fft_length(n, pad)
    series = _series_buffer(rows, n_fft, a.dtype, a.device)
    norms = ops.overlap(flat_a, flat_b, s, delta_f, series)
    value, t = _finish(series, f64, delta_f, norms, time, phase, pad)
    value, t = value.reshape(shape), t.reshape(shape)
    return (value, t) if return_time else value


def mismatch(a: torch.Tensor, b: torch.Tensor, frequencies, psd, **keywords):
    """``1 - match(a, b, ...)`` (see :func:`match`)."""
    out = match(a, b, frequencies, psd, **keywords)
    if isinstance(out, tuple):
        return 1 - out[0], out[1]
    return 1 - out


def polarization_match(signal: torch.Tensor, hplus: torch.Tensor, hcross: torch.Tensor, frequencies, psd, *,
                       time: bool = True, pad: int = 4, return_time: bool = False):
    """The match of ``signal`` with ``F+ hplus + Fx hcross`` maximised over
    time and over ``F+`` and ``Fx`` (match.py:150-187 on the kernels): the
    norm of the signal's projection onto the real span of the two
    polarizations over its norm; with parallel polarizations the match with
    ``hplus`` alone. Rows as :func:`match`."""
    for name, t in (("signal", signal), ("hplus", hplus), ("hcross", hcross)):
        _require_cuda(t, name)
        if t.dtype != signal.dtype or t.dtype not in (torch.complex64, torch.complex128):
            raise TypeError("signal, hplus and hcross must all be complex64 or all complex128")
    f64, delta_f, _ = _grid(frequencies, signal.device, signal.real.dtype)
    n = f64.numel()
    s = torch.as_tensor(psd, device=signal.device, dtype=signal.real.dtype).contiguous()
    shape = torch.broadcast_shapes(signal.shape[:-1], hplus.shape[:-1], hcross.shape[:-1])
    rows = 1
    for d in shape:
        rows *= d

    def flat(x):
        return x.contiguous() if x.ndim == 1 else x.expand(*shape, n).reshape(rows, n).contiguous()

    n_fft = ops.fft_length(n, pad)
    series = _series_buffer(2 * rows, n_fft, signal.dtype, signal.device)
    norms = ops.polarization_overlap(flat(signal), flat(hplus), flat(hcross), s, delta_f, series)
    zgrid = torch.fft.ifft(series, dim=-1, norm="forward") if time else None
    value, t = ops.polarization_refine(series, zgrid, f64, delta_f, norms, time=time, steps=NEWTON_STEPS)
    value, t = value.reshape(shape), t.reshape(shape)
    return (value, t) if return_time else value


def polarization_mismatch(signal, hplus, hcross, frequencies, psd, **keywords):
    """``1 - polarization_match(...)`` (see :func:`polarization_match`)."""
    out = polarization_match(signal, hplus, hcross, frequencies, psd, **keywords)
    if isinstance(out, tuple):
        return 1 - out[0], out[1]
    return 1 - out


def template_polarization_match(approximant: str, params: torch.Tensor, frequencies, signal: torch.Tensor, psd, *,
                                t_c: Optional[torch.Tensor] = None, time: bool = True, pad: int = 4,
                                amp_scale: float = 1e21, reference_mf: Optional[float] = None
                                ) -> Tuple[torch.Tensor, torch.Tensor]:
    """:func:`polarization_match` of ``signal`` with the polarizations of a
    bank of binaries (as :func:`template_match`), without their strain in
    memory: ``(match, t)``, float64 ``(B,)``."""
    _require_cuda(params, "params")
    f64, delta_f, f32 = _grid(frequencies, params.device, torch.float32)
    n = f64.numel()
    sig = torch.as_tensor(signal, device=params.device).to(torch.complex64).contiguous()
    if sig.numel() != n:
        raise ValueError("signal must hold one value per frequency")
    s = torch.as_tensor(psd, device=params.device).to(torch.float32).contiguous()
    tables = ops.setup(approximant, params, f64[:1], amp_scale=amp_scale, reference_mf=reference_mf,
                       precision=_lib.FP32)
    n_fft = ops.fft_length(n, pad)
    series = _series_buffer(2 * params.shape[0], n_fft, torch.complex64, params.device)
    tc = None if t_c is None else torch.as_tensor(t_c, device=params.device).to(torch.float32).contiguous()
    if ops.model_code(approximant) == _lib.XHM:
        hp, hc = ops.polarizations(approximant, tables.table, f32, None, tc)
        norms = ops.polarization_overlap(sig, hp.contiguous(), hc.contiguous(), s, delta_f, series)
    else:
        norms = ops.template_polarization_overlap(approximant, tables.table, f32, sig, s, delta_f, series, t_c=tc)
    zgrid = torch.fft.ifft(series, dim=-1, norm="forward") if time else None
    return ops.polarization_refine(series, zgrid, f32.to(torch.float64), delta_f, norms, time=time,
                                   steps=NEWTON_STEPS)


def template_match(approximant: str, params: torch.Tensor, frequencies, signal: torch.Tensor, psd, *,
                   antenna=(1.0, 0.0), t_c: Optional[torch.Tensor] = None, time: bool = True, phase: bool = True,
                   pad: int = 4, amp_scale: float = 1e21, reference_mf: Optional[float] = None
                   ) -> Tuple[torch.Tensor, torch.Tensor]:
    """The matches of a bank of templates ``F+ h+ + Fx hx`` of the binaries
    ``params`` (``(B, 8)`` float64 on the device: masses, aligned spins,
    distance, inclination, phi_ref, f_ref) with ``signal`` (complex64
    ``(n,)``) on the uniform grid ``frequencies``, maximised as
    :func:`match`, without the templates' strain in memory (FP32 templates,
    FP64 set-up; IMRPhenomXHM's strain is written once, then matched):
    ``(match, t)``, float64 ``(B,)``."""
    _require_cuda(params, "params")
    f64, delta_f, f32 = _grid(frequencies, params.device, torch.float32)
    n = f64.numel()
    sig = torch.as_tensor(signal, device=params.device).to(torch.complex64).contiguous()
    if sig.numel() != n:
        raise ValueError("signal must hold one value per frequency")
    s = torch.as_tensor(psd, device=params.device).to(torch.float32).contiguous()
    tables = ops.setup(approximant, params, f64[:1], amp_scale=amp_scale, reference_mf=reference_mf,
                       precision=_lib.FP32)
    n_fft = ops.fft_length(n, pad)
    series = _series_buffer(params.shape[0], n_fft, torch.complex64, params.device)
    tc = None if t_c is None else torch.as_tensor(t_c, device=params.device).to(torch.float32).contiguous()
    if ops.model_code(approximant) == _lib.XHM:
        # (IMRPhenomXHM: its templates' strain from its kernel, then the
        # series of the given waveforms)
        hp, hc = ops.polarizations(approximant, tables.table, f32, None, tc)
        h = (float(antenna[0]) * hp + float(antenna[1]) * hc).contiguous()
        norms = ops.overlap(h, sig, s, delta_f, series)
    else:
        norms = ops.template_overlap(approximant, tables.table, f32, sig, s, delta_f, series, t_c=tc,
                                     antenna=antenna)
    # the refinement at the frequencies the templates were evaluated at
    return _finish(series, f32.to(torch.float64), delta_f, norms, time, phase, pad)


def template_mismatch(approximant: str, params: torch.Tensor, frequencies, signal: torch.Tensor, psd, **keywords):
    """``1 - template_match(...)`` and the best times."""
    value, t = template_match(approximant, params, frequencies, signal, psd, **keywords)
    return 1 - value, t
