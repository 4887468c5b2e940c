"""Inconsistent ragged offsets through the C ABI: the FP32 ragged forms find
them in their first kernel and report WFX_EOFFSETS in the workspace's status
word (wfx_ragged_status), evaluate nothing and write nothing outside their
buffers; IMRPhenomXHM's and the FP64 ragged forms clamp each binary's range
to the grid. Canary regions after the workspace and the outputs must stay
unchanged. The Python layer refuses such offsets before any launch (the
reference's rows check, src/waveformx/_api.py:292-305)."""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

from test_gpu_polarizations import draw_batch

pytestmark = pytest.mark.gpu

CANARY = 4096  # bytes after each buffer that no call may touch
FILL = 0x5A


def _p(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def _guarded(nbytes, device):
    """A byte buffer of ``nbytes`` followed by CANARY bytes, all FILL."""
    import torch

    return torch.full((nbytes + CANARY,), FILL, dtype=torch.uint8, device=device)


def _setup(cuda, batch, model="IMRPhenomXAS", precision=None):
    import torch

    from waveformx_b200 import _lib, ops

    params = torch.as_tensor(draw_batch(np.random.default_rng(11), batch), device=cuda)
    precision = _lib.FP32 if precision is None else precision
    return ops.setup(model, params, torch.tensor([20.0], dtype=torch.float64, device=cuda), precision=precision,
                     jvp=model != "IMRPhenomXHM")


BAD = {
    "decreasing": lambda n: [0, n // 2, n // 4, n // 2, n],
    "overlapping": lambda n: [0, n, 0, n, n],
    "negative start": lambda n: [-8, n // 4, n // 2, 3 * n // 4, n],
    "past the end": lambda n: [0, n // 4, n // 2, 3 * n // 4, n + 4096],
    "short of the end": lambda n: [0, n // 4, n // 2, 3 * n // 4, n - 7],
}


@pytest.mark.parametrize("case", sorted(BAD))
def test_fp32_ragged_forward_reports_bad_offsets(cuda, case):
    import torch

    from waveformx_b200 import _lib

    lib = _lib.library()
    batch, n = 4, 6000
    tables = _setup(cuda, batch)
    freqs = torch.linspace(20.0, 1024.0, n, dtype=torch.float32, device=cuda)
    offsets = torch.tensor(BAD[case](n), dtype=torch.int64, device=cuda)
    need = int(lib.wfx_workspace_bytes(_lib.OP_POLARIZATIONS, _lib.XAS, _lib.FP32, batch, n, 1))
    ws = _guarded(need, cuda)
    out = [_guarded(8 * n, cuda) for _ in range(2)]
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = lib.wfx_polarizations(_lib.XAS, _lib.FP32, _p(tables.table), _p(freqs), _p(offsets), batch, n, None,
                               _p(out[0]), _p(out[1]), _p(ws), need, stream)
    assert rc == 0
    assert lib.wfx_ragged_status(_p(ws), stream) == _lib.EOFFSETS
    torch.cuda.synchronize()
    assert bool((ws[need:] == FILL).all())
    for o in out:
        assert bool((o == FILL).all())  # nothing evaluated, nothing written
    # the same workspace then serves valid offsets
    good = torch.tensor([0, n // 4, n // 2, 3 * n // 4, n], dtype=torch.int64, device=cuda)
    rc = lib.wfx_polarizations(_lib.XAS, _lib.FP32, _p(tables.table), _p(freqs), _p(good), batch, n, None,
                               _p(out[0]), _p(out[1]), _p(ws), need, stream)
    assert rc == 0 and lib.wfx_ragged_status(_p(ws), stream) == 0
    torch.cuda.synchronize()
    assert bool((ws[need:] == FILL).all())
    assert all(bool((o[8 * n:] == FILL).all()) for o in out)
    assert not bool((out[0][: 8 * n] == FILL).all())


@pytest.mark.parametrize("case", ["decreasing", "overlapping", "past the end"])
def test_fp32_ragged_fused_loss_reports_bad_offsets(cuda, case):
    import torch

    from waveformx_b200 import _lib

    lib = _lib.library()
    batch, n = 4, 6000
    tables = _setup(cuda, batch)
    freqs = torch.linspace(20.0, 1024.0, n, dtype=torch.float32, device=cuda)
    offsets = torch.tensor(BAD[case](n), dtype=torch.int64, device=cuda)
    data = torch.zeros(n, dtype=torch.complex64, device=cuda)
    weights = torch.ones(n, dtype=torch.float32, device=cuda)
    need = int(lib.wfx_workspace_bytes(_lib.OP_FUSED, _lib.XAS, _lib.FP32, batch, n, 1))
    ws = _guarded(need, cuda)
    loss = torch.zeros(batch, dtype=torch.float32, device=cuda)
    grad = torch.zeros((batch, _lib.GRAD_COLUMNS), dtype=torch.float32, device=cuda)
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = lib.wfx_fused_loss(_lib.XAS, _lib.FP32, _p(tables.table), _p(tables.dtable), _p(freqs), _p(offsets), batch,
                            n, None, _p(data), 1, _p(weights), 1, 1.0, 0.0, -0.5, _p(loss), _p(grad), _p(ws), need,
                            stream)
    assert rc == 0
    assert lib.wfx_ragged_status(_p(ws), stream) == _lib.EOFFSETS
    torch.cuda.synchronize()
    assert bool((ws[need:] == FILL).all())
    assert bool(torch.isnan(loss).all()) and bool(torch.isnan(grad).all())


def test_xhm_and_fp64_ragged_forms_clamp(cuda):
    """Offsets past the grid: each binary's range is clamped to [0, n]; the
    canaries after the outputs stay unchanged."""
    import torch

    from waveformx_b200 import _lib

    lib = _lib.library()
    batch, n = 4, 3000
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    offsets = torch.tensor(BAD["past the end"](n), dtype=torch.int64, device=cuda)
    max_len = 4096 + n // 4
    for precision, real, size in ((_lib.FP32, torch.float32, 8), (_lib.FP64, torch.float64, 16)):
        freqs = torch.linspace(20.0, 1024.0, n, dtype=real, device=cuda)
        xhm = _setup(cuda, batch, "IMRPhenomXHM", precision)
        out = [_guarded(size * n, cuda) for _ in range(2)]
        rc = lib.wfx_xhm_polarizations(precision, _p(xhm.table), _p(freqs), _p(offsets), batch, n, max_len, None,
                                       _p(out[0]), _p(out[1]), None, stream)
        assert rc == 0
        torch.cuda.synchronize()
        assert all(bool((o[size * n:] == FILL).all()) for o in out)
    freqs = torch.linspace(20.0, 1024.0, n, dtype=torch.float64, device=cuda)
    xas = _setup(cuda, batch, precision=_lib.FP64)
    out = [_guarded(16 * n, cuda) for _ in range(2)]
    rc = lib.wfx_polarizations(_lib.XAS, _lib.FP64, _p(xas.table), _p(freqs), _p(offsets), batch, n, None,
                               _p(out[0]), _p(out[1]), None, 0, stream)
    assert rc == 0
    torch.cuda.synchronize()
    assert all(bool((o[16 * n:] == FILL).all()) for o in out)


def test_python_layer_refuses_bad_offsets(cuda):
    import torch

    from waveformx_b200 import ops

    batch, n = 4, 2000
    tables = _setup(cuda, batch)
    freqs = torch.linspace(20.0, 1024.0, n, dtype=torch.float32, device=cuda)
    for case in sorted(BAD):
        offsets = torch.tensor(BAD[case](n), dtype=torch.int64, device=cuda)
        with pytest.raises(ValueError, match="offsets"):
            ops.polarizations("IMRPhenomXAS", tables.table, freqs, offsets)
    good = torch.tensor([0, 500, 1000, 1500, n], dtype=torch.int64, device=cuda)
    ops.polarizations("IMRPhenomXAS", tables.table, freqs, good)
    good[2] = 1700  # an in-place change is checked again
    with pytest.raises(ValueError, match="offsets"):
        ops.polarizations("IMRPhenomXAS", tables.table, freqs, good)
    data = torch.zeros(n - 1, dtype=torch.complex64, device=cuda)
    with pytest.raises(ValueError, match="data"):
        ops.fused_loss("IMRPhenomXAS", tables.table, tables.dtable, freqs, None, None, data,
                       torch.ones(n, dtype=torch.float32, device=cuda))
