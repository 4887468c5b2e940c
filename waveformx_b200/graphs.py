"""CUDA-graph capture of the FP32 path for fixed shapes.

A sampler evaluates the same batch shape over and over; a captured graph
replays the set-up and the frequency kernels (for a ragged batch: the work
item scan, the item map and the persistent launch) with one launch from the
host. :class:`CapturedPolarizations` (the strain) and
:class:`CapturedLikelihood` (the fused log-likelihood and its gradient, the
strain never in memory) own static input and output buffers: each call
copies the parameters in, replays, and returns the static outputs, which
the next call overwrites.
"""

from __future__ import annotations

from typing import Optional

from . import _lib, ops

__all__ = ["CapturedLikelihood", "CapturedPolarizations"]


class CapturedPolarizations:
    """``(hplus, hcross)`` of ``batch`` binaries on a fixed grid, captured.

    ``freqs``: the shared grid ``(N,)`` or, with ``offsets`` (``B + 1``
    int64), the flat grids of a ragged batch; FP32 CUDA tensors. ``t_c``:
    whether calls pass a coalescence time per binary. ``autotune``: tune the
    ragged forward on the first parameters before capturing (it
    synchronises, so it is done outside the capture)."""

    def __init__(self, approximant: str, batch: int, freqs, offsets=None, *, t_c: bool = False,
                 amp_scale: float = 1e21, reference_mf: Optional[float] = None, autotune: bool = True):
        import torch

        if freqs.dtype != torch.float32 or freqs.device.type != "cuda":
            raise TypeError("freqs must be a float32 CUDA tensor")
        self.approximant = approximant
        self.batch = int(batch)
        self.device = freqs.device
        self.freqs = freqs.contiguous()
        self.offsets = None if offsets is None else offsets.to(self.device, torch.int64).contiguous()
        if self.offsets is not None:
            # (checked here, outside any capture: the check reads them to the host)
            ops.check_offsets(self.offsets, self.batch, self.freqs.numel())
        self.amp_scale = amp_scale
        self.reference_mf = reference_mf
        self.autotune = autotune and self.offsets is not None
        self.params = torch.zeros((self.batch, 8), dtype=torch.float64, device=self.device)
        if self.offsets is None:
            self.f_min = self.freqs[:1].to(torch.float64)
        else:
            first = self.offsets[:-1].clamp(max=max(self.freqs.numel() - 1, 0))
            self.f_min = self.freqs[first].to(torch.float64)
        self.t_c = torch.zeros(self.batch, dtype=torch.float32, device=self.device) if t_c else None
        self.graph = None
        self.hp = self.hc = None
        self.status = None

    def _run(self):
        tables = ops.setup(self.approximant, self.params, self.f_min, amp_scale=self.amp_scale,
                           reference_mf=self.reference_mf, precision=_lib.FP32)
        hp, hc = ops.polarizations(self.approximant, tables.table, self.freqs, self.offsets, self.t_c)
        return hp, hc, tables

    def _capture(self):
        import torch

        side = torch.cuda.Stream(self.device)
        side.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(side):
            for _ in range(2):
                _, _, tables = self._run()
            if self.autotune:
                from .tuning import autotune_ragged

                autotune_ragged(self.approximant, tables.table, self.freqs, self.offsets, self.t_c)
        torch.cuda.current_stream(self.device).wait_stream(side)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self.hp, self.hc, tables = self._run()
            self.status = tables.status

    def __call__(self, params, t_c=None):
        """Copy ``params`` (``(batch, 8)``: masses, aligned spins, distance,
        inclination, phi_ref, f_ref) and ``t_c`` in, replay, and return the
        static ``(hplus, hcross)``."""
        import torch

        params = torch.as_tensor(params, dtype=torch.float64, device=self.device)
        if params.shape != (self.batch, 8):
            raise ValueError(f"params must be ({self.batch}, 8)")
        self.params.copy_(params)
        if self.t_c is not None:
            if t_c is None:
                raise TypeError("this capture takes t_c")
            self.t_c.copy_(torch.as_tensor(t_c, dtype=torch.float32, device=self.device))
        elif t_c is not None:
            raise TypeError("this capture was made without t_c")
        if self.graph is None:
            self._capture()
            self.params.copy_(params)
        self.graph.replay()
        return self.hp, self.hc


def _first_frequencies(freqs, offsets):
    import torch

    if offsets is None:
        return freqs[:1].to(torch.float64)
    first = offsets[:-1].clamp(max=max(freqs.numel() - 1, 0))
    return freqs[first].to(torch.float64)


class CapturedLikelihood:
    """The FP32 fused log-likelihood ``scale sum_f w |F+ h+ + Fx hx - d|^2``
    of ``batch`` binaries and its ``(batch, 9)`` gradient (the eight
    parameters and ``t_c``), captured: one replay runs the value set-up, the
    dual-number set-up on a second stream, the fused likelihood kernel and the
    contraction (``ops.fused_loss_from_params``).

    ``freqs``: the shared grid ``(N,)`` or, with ``offsets``, the flat grids
    of a ragged batch (FP32 CUDA). ``data`` (complex64) and ``weights``
    (float32): per frequency, or per element of the batch's grid; copied at
    construction (:meth:`set_data` replaces them between calls). ``t_c``:
    whether calls pass a coalescence time per binary."""

    def __init__(self, approximant: str, batch: int, freqs, data, weights, offsets=None, *, t_c: bool = False,
                 antenna=(1.0, 0.0), scale: float = 1.0, amp_scale: float = 1e21,
                 reference_mf: Optional[float] = None):
        import torch

        if freqs.dtype != torch.float32 or freqs.device.type != "cuda":
            raise TypeError("freqs must be a float32 CUDA tensor")
        ops.model_code(approximant)
        self.approximant = approximant
        self.batch = int(batch)
        self.device = freqs.device
        self.freqs = freqs.contiguous()
        self.offsets = None if offsets is None else offsets.to(self.device, torch.int64).contiguous()
        if self.offsets is not None:
            # (checked here, outside any capture: the check reads them to the host)
            ops.check_offsets(self.offsets, self.batch, self.freqs.numel())
        self.data = torch.as_tensor(data, dtype=torch.complex64, device=self.device).contiguous().clone()
        self.weights = torch.as_tensor(weights, dtype=torch.float32, device=self.device).contiguous().clone()
        self.antenna = (float(antenna[0]), float(antenna[1]))
        self.scale = float(scale)
        self.amp_scale = amp_scale
        self.reference_mf = reference_mf
        self.params = torch.zeros((self.batch, 8), dtype=torch.float64, device=self.device)
        self.f_min = _first_frequencies(self.freqs, self.offsets)
        self.t_c = torch.zeros(self.batch, dtype=torch.float32, device=self.device) if t_c else None
        self.dtable = torch.empty((self.batch, _lib.TABLE_STRIDE, 8), dtype=torch.float64, device=self.device)
        self.graph = None
        self.loss = self.grad = self.status = None

    def set_data(self, data=None, weights=None):
        """Replace the data and / or the weights (same shapes) for the next
        calls."""
        import torch

        if data is not None:
            self.data.copy_(torch.as_tensor(data, dtype=torch.complex64, device=self.device).reshape(self.data.shape))
        if weights is not None:
            self.weights.copy_(torch.as_tensor(weights, dtype=torch.float32, device=self.device)
                               .reshape(self.weights.shape))

    def _run(self):
        return ops.fused_loss_from_params(self.approximant, self.params, self.f_min, self.freqs, self.offsets,
                                          self.t_c, self.data, self.weights, antenna=self.antenna, scale=self.scale,
                                          amp_scale=self.amp_scale, reference_mf=self.reference_mf,
                                          dtable_out=self.dtable)

    def _capture(self):
        import torch

        side = torch.cuda.Stream(self.device)
        side.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(side):
            for _ in range(2):
                self._run()
        torch.cuda.current_stream(self.device).wait_stream(side)
        self.graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.graph):
            self.loss, self.grad, self.status = self._run()

    def __call__(self, params, t_c=None):
        """Copy ``params`` (``(batch, 8)``) and ``t_c`` in, replay, and
        return the static ``(loss, grad, status)``."""
        import torch

        params = torch.as_tensor(params, dtype=torch.float64, device=self.device)
        if params.shape != (self.batch, 8):
            raise ValueError(f"params must be ({self.batch}, 8)")
        self.params.copy_(params)
        if self.t_c is not None:
            if t_c is None:
                raise TypeError("this capture takes t_c")
            self.t_c.copy_(torch.as_tensor(t_c, dtype=torch.float32, device=self.device))
        elif t_c is not None:
            raise TypeError("this capture was made without t_c")
        if self.graph is None:
            self._capture()
            self.params.copy_(params)
        self.graph.replay()
        return self.loss, self.grad, self.status
