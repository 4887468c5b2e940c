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
