"""CUDA-graph capture (``waveformx_b200.graphs``) and the autotuned ragged
forward: replays give the eager results bit for bit, for new parameters
each call."""

from __future__ import annotations

import numpy as np
import pytest

from test_gpu_polarizations import draw_batch

pytestmark = pytest.mark.gpu


def _ragged(rng, params):
    grids = []
    for m1, m2 in params[:, :2]:
        f_low = rng.uniform(10.0, 30.0)
        f_high = min(2048.0, 0.3 / ((m1 + m2) * 4.925490947641267e-06))
        grids.append(np.arange(f_low, f_high, 1.0 / rng.choice([4.0, 8.0])))
    return grids


@pytest.mark.parametrize("approximant", ["IMRPhenomXAS", "IMRPhenomD", "TaylorF2"])
@pytest.mark.parametrize("ragged", [False, True])
def test_replay_equals_eager(cuda, approximant, ragged):
    import torch

    from waveformx_b200 import _lib, ops
    from waveformx_b200.graphs import CapturedPolarizations

    rng = np.random.default_rng(4)
    batch = 40
    params = [draw_batch(rng, batch) for _ in range(3)]
    if ragged:
        grids = _ragged(rng, params[0])
        offsets = torch.as_tensor(np.concatenate([[0], np.cumsum([len(g) for g in grids])]), device=cuda)
        freqs = torch.as_tensor(np.concatenate(grids), dtype=torch.float32, device=cuda)
        f_min = torch.as_tensor([g[0] for g in grids], dtype=torch.float32, device=cuda).double()
    else:
        offsets = None
        freqs = torch.linspace(20.0, 1024.0, 1001, dtype=torch.float32, device=cuda)
        f_min = freqs[:1].double()
    t_c = torch.as_tensor(rng.uniform(-0.05, 0.05, batch), dtype=torch.float32, device=cuda)
    captured = CapturedPolarizations(approximant, batch, freqs, offsets, t_c=True)
    for p in params:
        hp, hc = captured(p, t_c)
        hp, hc = hp.clone(), hc.clone()
        tables = ops.setup(approximant, torch.as_tensor(p, device=cuda), f_min, precision=_lib.FP32)
        ep, ec = ops.polarizations(approximant, tables.table, freqs, offsets, t_c)
        assert torch.equal(hp, ep) and torch.equal(hc, ec)


def test_autotune_keeps_the_result(cuda):
    import torch

    from waveformx_b200 import _lib, ops, tuning

    rng = np.random.default_rng(9)
    params = draw_batch(rng, 64)
    grids = _ragged(rng, params)
    offsets = torch.as_tensor(np.concatenate([[0], np.cumsum([len(g) for g in grids])]), device=cuda)
    freqs = torch.as_tensor(np.concatenate(grids), dtype=torch.float32, device=cuda)
    f_min = torch.as_tensor([g[0] for g in grids], dtype=torch.float64, device=cuda)
    tables = ops.setup("IMRPhenomXAS", torch.as_tensor(params, device=cuda), f_min, precision=_lib.FP32)
    before = ops.polarizations("IMRPhenomXAS", tables.table, freqs, offsets)
    tile, blocks = tuning.autotune_ragged("IMRPhenomXAS", tables.table, freqs, offsets, save=False)
    assert tile in (510, 1022, 2046, 4094) and blocks in (2, 4, 8, 16)
    assert tuning.lookup("IMRPhenomXAS", 64, freqs.numel()) == (tile, blocks, True)
    after = ops.polarizations("IMRPhenomXAS", tables.table, freqs, offsets)
    for a, b in zip(before, after):
        assert torch.equal(a, b)


@pytest.mark.parametrize("approximant", ["IMRPhenomXAS", "IMRPhenomD", "TaylorF2"])
@pytest.mark.parametrize("ragged", [False, True])
def test_likelihood_replay_equals_eager(cuda, approximant, ragged):
    import torch

    from waveformx_b200 import ops
    from waveformx_b200.graphs import CapturedLikelihood

    rng = np.random.default_rng(11)
    batch = 48
    params = [draw_batch(rng, batch) for _ in range(3)]
    if ragged:
        grids = _ragged(rng, params[0])
        offsets = torch.as_tensor(np.concatenate([[0], np.cumsum([len(g) for g in grids])]), device=cuda)
        freqs = torch.as_tensor(np.concatenate(grids), dtype=torch.float32, device=cuda)
        f_min = torch.as_tensor([g[0] for g in grids], dtype=torch.float32, device=cuda).double()
        size = freqs.numel()
    else:
        offsets = None
        freqs = torch.linspace(20.0, 1024.0, 1001, dtype=torch.float32, device=cuda)
        f_min = freqs[:1].double()
        size = freqs.numel()
    data = torch.as_tensor((rng.normal(size=size) + 1j * rng.normal(size=size)) * 1e-2, dtype=torch.complex64,
                           device=cuda)
    weights = torch.as_tensor(rng.uniform(0.5, 2.0, size), dtype=torch.float32, device=cuda)
    t_c = torch.as_tensor(rng.uniform(-0.05, 0.05, batch), dtype=torch.float32, device=cuda)
    captured = CapturedLikelihood(approximant, batch, freqs, data, weights, offsets, t_c=True, antenna=(0.6, -0.3),
                                  scale=-0.5)
    for p in params:
        loss, grad, status = captured(p, t_c)
        loss, grad = loss.clone(), grad.clone()
        e_loss, e_grad, e_status = ops.fused_loss_from_params(
            approximant, torch.as_tensor(p, device=cuda), f_min, freqs, offsets, t_c, data, weights,
            antenna=(0.6, -0.3), scale=-0.5)
        assert torch.equal(loss, e_loss) and torch.equal(grad, e_grad) and torch.equal(status, e_status)
        assert torch.isfinite(loss).all() and torch.isfinite(grad).all()
    # new data between calls
    captured.set_data(data * 2.0)
    loss, grad, _ = captured(params[0], t_c)
    e_loss, e_grad, _ = ops.fused_loss_from_params(approximant, torch.as_tensor(params[0], device=cuda), f_min, freqs,
                                                    offsets, t_c, data * 2.0, weights, antenna=(0.6, -0.3),
                                                    scale=-0.5)
    assert torch.equal(loss, e_loss) and torch.equal(grad, e_grad)


def test_likelihood_capture_refusals(cuda):
    import torch

    from waveformx_b200.graphs import CapturedLikelihood

    freqs = torch.linspace(20.0, 1024.0, 101, dtype=torch.float32, device=cuda)
    data = torch.zeros(101, dtype=torch.complex64, device=cuda)
    weights = torch.ones(101, dtype=torch.float32, device=cuda)
    with pytest.raises(TypeError):
        CapturedLikelihood("IMRPhenomXAS", 4, freqs.double(), data, weights)
    captured = CapturedLikelihood("IMRPhenomXAS", 4, freqs, data, weights)
    with pytest.raises(ValueError):
        captured(np.zeros((3, 8)))
    with pytest.raises(TypeError):
        captured(draw_batch(np.random.default_rng(1), 4), t_c=torch.zeros(4, device=cuda))
