"""``wfx_fused_loss_noalloc`` (the fused likelihood with the library's static
scratch instead of a caller's workspace) against ``wfx_fused_loss``, both
called through the C ABI: two calls in a row on the shared-grid, ragged and
FP64 forms, and the refusal of a problem larger than the static scratch.

The file is named to be collected last, so that it also runs after every
other test has used the library in the same process."""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

from test_gpu_polarizations import draw_batch

pytestmark = pytest.mark.gpu

# FP32: the two entries run the same kernels on the same inputs; the loss and
# gradient agree to float32 rounding of the per-tile sums at most.
RTOL_FP32 = 1e-6
RTOL_FP64 = 1e-12


def _p(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def _problem(cuda, model, precision, ragged, batch=24, n=1500, seed=7):
    import torch

    from waveformx_b200 import _lib, ops

    rng = np.random.default_rng(seed)
    params = torch.as_tensor(draw_batch(rng, batch), device=cuda)
    approximant = "IMRPhenomXAS" if model == _lib.XAS else "IMRPhenomD"
    real = torch.float32 if precision == _lib.FP32 else torch.float64
    cplx = torch.complex64 if precision == _lib.FP32 else torch.complex128
    if ragged:
        lengths = rng.integers(n // 4, n, size=batch)
        offsets = torch.as_tensor(np.concatenate([[0], np.cumsum(lengths)]), device=cuda)
        freqs = torch.as_tensor(np.concatenate([np.geomspace(20.0, 1024.0, k) for k in lengths]), dtype=real,
                                device=cuda)
        f_min = torch.as_tensor(np.full(batch, 20.0), device=cuda)
        total = int(lengths.sum())
    else:
        offsets = None
        freqs = torch.as_tensor(np.linspace(20.0, 1024.0, n), dtype=real, device=cuda)
        f_min = torch.tensor([20.0], dtype=torch.float64, device=cuda)
        total = n
    tables = ops.setup(approximant, params, f_min, precision=precision, jvp=True)
    t_c = torch.as_tensor(rng.uniform(-0.01, 0.01, batch), dtype=real, device=cuda)
    data = torch.complex(torch.as_tensor(rng.normal(size=total), dtype=real),
                         torch.as_tensor(rng.normal(size=total), dtype=real)).to(cuda, cplx) * 1e-2
    weights = torch.as_tensor(rng.uniform(0.5, 2.0, total), dtype=real, device=cuda)
    stride = 1 if ragged else 0
    return dict(model=model, precision=precision, table=tables.table, dtable=tables.dtable, freqs=freqs,
                offsets=offsets, B=batch, n=total, t_c=t_c, data=data, data_stride=stride, weights=weights,
                weights_stride=stride, real=real)


def _call(pb, noalloc):
    import torch

    from waveformx_b200 import _lib

    lib = _lib.library()
    device = pb["table"].device
    loss = torch.full((pb["B"],), float("nan"), dtype=pb["real"], device=device)
    grad = torch.full((pb["B"], _lib.GRAD_COLUMNS), float("nan"), dtype=pb["real"], device=device)
    stream = ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)
    head = (pb["model"], pb["precision"], _p(pb["table"]), _p(pb["dtable"]), _p(pb["freqs"]), _p(pb["offsets"]),
            pb["B"], pb["n"], _p(pb["t_c"]), _p(pb["data"]), pb["data_stride"], _p(pb["weights"]),
            pb["weights_stride"], 0.6, -0.3, -0.5, _p(loss), _p(grad))
    if noalloc:
        rc = lib.wfx_fused_loss_noalloc(*head, stream)
    else:
        nbytes = int(lib.wfx_workspace_bytes(_lib.OP_FUSED, pb["model"], pb["precision"], pb["B"], pb["n"],
                                             int(pb["offsets"] is not None)))
        ws = torch.empty(max(nbytes, 1), dtype=torch.uint8, device=device)
        rc = lib.wfx_fused_loss(*head, _p(ws), nbytes, stream)
    torch.cuda.synchronize(device)
    return rc, loss.cpu().numpy().astype(np.float64), grad.cpu().numpy().astype(np.float64)


@pytest.mark.parametrize("form", ["xas_fp32_shared", "phenomd_fp32_shared", "xas_fp32_ragged", "xas_fp64_shared"])
def test_noalloc_matches_the_workspace_entry(cuda, form):
    from waveformx_b200 import _lib

    approximant, precision, layout = form.split("_")
    model = _lib.XAS if approximant == "xas" else _lib.PHENOMD
    prec = _lib.FP32 if precision == "fp32" else _lib.FP64
    pb = _problem(cuda, model, prec, layout == "ragged")
    rc, loss, grad = _call(pb, noalloc=False)
    assert rc == 0
    assert np.all(np.isfinite(loss)) and np.all(np.isfinite(grad))
    rtol = RTOL_FP32 if prec == _lib.FP32 else RTOL_FP64
    for _ in range(2):
        rc2, loss2, grad2 = _call(pb, noalloc=True)
        assert rc2 == 0, _lib.library().wfx_status_string(rc2)
        np.testing.assert_allclose(loss2, loss, rtol=rtol, atol=0)
        scale = np.max(np.abs(grad), axis=1, keepdims=True)
        np.testing.assert_allclose(grad2, grad, rtol=rtol, atol=rtol * float(scale.max()))


def test_noalloc_refuses_beyond_the_static_scratch(cuda):
    """A shared-grid FP32 problem needing more than the static scratch is
    refused before any launch (the buffers are the problem's full size all
    the same, so nothing could read past them)."""
    import torch

    from waveformx_b200 import _lib

    lib = _lib.library()
    batch, n = 40000, 3000
    need = int(lib.wfx_workspace_bytes(_lib.OP_FUSED, _lib.XAS, _lib.FP32, batch, n, 0))
    assert need > _lib.STATIC_SCRATCH_BYTES
    z = dict(device=cuda)
    table = torch.zeros((batch, _lib.TABLE_STRIDE), dtype=torch.float32, **z)
    dtable = torch.zeros((batch, _lib.TABLE_STRIDE, 8), dtype=torch.float64, **z)
    freqs = torch.linspace(20.0, 1024.0, n, dtype=torch.float32, **z)
    data = torch.zeros(n, dtype=torch.complex64, **z)
    weights = torch.ones(n, dtype=torch.float32, **z)
    loss = torch.zeros(batch, dtype=torch.float32, **z)
    grad = torch.zeros((batch, _lib.GRAD_COLUMNS), dtype=torch.float32, **z)
    stream = ctypes.c_void_p(torch.cuda.current_stream(cuda).cuda_stream)
    rc = lib.wfx_fused_loss_noalloc(_lib.XAS, _lib.FP32, _p(table), _p(dtable), _p(freqs), None, batch, n, None,
                                    _p(data), 0, _p(weights), 0, 1.0, 0.0, -0.5, _p(loss), _p(grad), stream)
    torch.cuda.synchronize(cuda)
    assert rc == _lib.ESCRATCH
    assert b"static scratch" in lib.wfx_status_string(rc)
    assert bool(torch.all(loss == 0)) and bool(torch.all(grad == 0))
