"""The batch pipeline (``waveformx_b200.pipeline.polarizations_stream``):
each batch's results equal the eager set-up + polarizations bit for bit,
with the set-up of the next batch on a second stream."""

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


@pytest.mark.parametrize("approximant", ["IMRPhenomXAS", "IMRPhenomD", "TaylorF2", "IMRPhenomXHM"])
@pytest.mark.parametrize("precision", ["fp32", "fp64"])
@pytest.mark.parametrize("ragged", [False, True])
def test_stream_equals_eager(cuda, approximant, precision, ragged):
    import torch

    from waveformx_b200 import _lib, ops
    from waveformx_b200.pipeline import polarizations_stream

    prec = _lib.FP32 if precision == "fp32" else _lib.FP64
    real = torch.float32 if precision == "fp32" else torch.float64
    rng = np.random.default_rng(21)
    batch = 24
    params = [torch.as_tensor(draw_batch(rng, batch), device=cuda) for _ in range(5)]
    t_cs = [torch.as_tensor(rng.uniform(-0.05, 0.05, batch), dtype=real, device=cuda) for _ in range(5)]
    if ragged:
        grids = _ragged(rng, params[0].cpu().numpy())
        offsets = torch.as_tensor(np.concatenate([[0], np.cumsum([len(g) for g in grids])]), device=cuda)
        freqs = torch.as_tensor(np.concatenate(grids), dtype=real, device=cuda)
        f_min = torch.as_tensor([g[0] for g in grids], dtype=real, device=cuda).double()
    else:
        offsets = None
        freqs = torch.linspace(20.0, 1024.0, 1001, dtype=real, device=cuda)
        f_min = freqs[:1].double()
    out = list(polarizations_stream(approximant, zip(params, t_cs), freqs, offsets, f_min=f_min, precision=prec))
    assert len(out) == len(params)
    for (hp, hc, status), p, t_c in zip(out, params, t_cs):
        tables = ops.setup(approximant, p, f_min, precision=prec)
        ep, ec = ops.polarizations(approximant, tables.table, freqs, offsets, t_c)
        assert torch.equal(hp, ep) and torch.equal(hc, ec)
        assert torch.equal(status, tables.status)


def test_stream_plain_params_and_early_exit(cuda):
    import torch

    from waveformx_b200 import _lib, ops
    from waveformx_b200.pipeline import polarizations_stream

    rng = np.random.default_rng(3)
    params = [torch.as_tensor(draw_batch(rng, 16), device=cuda) for _ in range(4)]
    freqs = torch.linspace(20.0, 512.0, 333, dtype=torch.float32, device=cuda)
    stream = polarizations_stream("IMRPhenomXAS", params, freqs)
    hp, hc, _ = next(stream)
    tables = ops.setup("IMRPhenomXAS", params[0], freqs[:1].double(), precision=_lib.FP32)
    ep, ec = ops.polarizations("IMRPhenomXAS", tables.table, freqs)
    assert torch.equal(hp, ep) and torch.equal(hc, ec)
    stream.close()
    assert list(polarizations_stream("IMRPhenomXAS", [], freqs)) == []


def test_stream_refusals(cuda):
    import torch

    from waveformx_b200.pipeline import polarizations_stream

    rng = np.random.default_rng(4)
    freqs = torch.linspace(20.0, 512.0, 101, dtype=torch.float32, device=cuda)
    batches = [torch.as_tensor(draw_batch(rng, 8), device=cuda), torch.as_tensor(draw_batch(rng, 9), device=cuda)]
    with pytest.raises(ValueError):
        list(polarizations_stream("IMRPhenomXAS", batches, freqs))
    with pytest.raises(ValueError):
        list(polarizations_stream("IMRPhenomXAS", [torch.zeros((4, 7), dtype=torch.float64, device=cuda)], freqs))
    with pytest.raises(ValueError):
        list(polarizations_stream("IMRPhenomXAS", [(batches[0], None, None)], freqs))


@pytest.mark.parametrize("approximant", ["IMRPhenomXAS", "IMRPhenomD", "TaylorF2"])
@pytest.mark.parametrize("ragged", [False, True])
def test_likelihood_stream_equals_eager(cuda, approximant, ragged):
    """The likelihood's batches through the pipeline: the same loss and
    gradient as ops.fused_loss_from_params, bit for bit."""
    import torch

    from waveformx_b200 import ops
    from waveformx_b200.pipeline import likelihood_stream

    rng = np.random.default_rng(31)
    batch = 24
    params = [torch.as_tensor(draw_batch(rng, batch), device=cuda) for _ in range(4)]
    t_cs = [torch.as_tensor(rng.uniform(-0.05, 0.05, batch), dtype=torch.float32, device=cuda) for _ in range(4)]
    if ragged:
        grids = _ragged(rng, params[0].cpu().numpy())
        offsets = torch.as_tensor(np.concatenate([[0], np.cumsum([len(g) for g in grids])]), device=cuda)
        freqs = torch.as_tensor(np.concatenate(grids), dtype=torch.float32, device=cuda)
        f_min = torch.as_tensor([g[0] for g in grids], dtype=torch.float32, device=cuda).double()
    else:
        offsets = None
        freqs = torch.linspace(20.0, 1024.0, 1001, dtype=torch.float32, device=cuda)
        f_min = freqs[:1].double()
    size = freqs.numel()
    data = torch.as_tensor((rng.normal(size=size) + 1j * rng.normal(size=size)) * 1e-2, dtype=torch.complex64,
                           device=cuda)
    weights = torch.as_tensor(rng.uniform(0.5, 2.0, size), dtype=torch.float32, device=cuda)
    out = list(likelihood_stream(approximant, zip(params, t_cs), freqs, data, weights, offsets, f_min=f_min,
                                 antenna=(0.6, -0.3), scale=-0.5))
    assert len(out) == len(params)
    for (loss, grad, status), p, t_c in zip(out, params, t_cs):
        e_loss, e_grad, e_status = ops.fused_loss_from_params(approximant, p, f_min, freqs, offsets, t_c, data, weights,
                                                              antenna=(0.6, -0.3), scale=-0.5)
        assert torch.equal(loss, e_loss) and torch.equal(grad, e_grad) and torch.equal(status, e_status)


@pytest.mark.parametrize("approximant", ["IMRPhenomXAS", "IMRPhenomD", "TaylorF2"])
@pytest.mark.parametrize("case", ["shared", "per_binary_data", "ragged"])
@pytest.mark.parametrize("group", [None, 1, 2, 5])
def test_likelihood_batches_equal_eager(cuda, approximant, case, group):
    """``likelihood_batches`` (``wfx_pipeline_likelihood_run``: K batches in
    one library call, the dual-number set-ups of a group of batches in one
    launch) gives each batch ops.fused_loss_from_params's loss, gradient and
    status bit for bit."""
    import torch

    from waveformx_b200 import ops
    from waveformx_b200.pipeline import Pipeline, likelihood_batches

    rng = np.random.default_rng(37)
    K, batch = 5, 20
    params = torch.as_tensor(np.stack([draw_batch(rng, batch) for _ in range(K)]), device=cuda)
    t_c = torch.as_tensor(rng.uniform(-0.05, 0.05, (K, batch)), dtype=torch.float32, device=cuda)
    if case == "ragged":
        grids = _ragged(rng, params[0].cpu().numpy())
        offsets = torch.as_tensor(np.concatenate([[0], np.cumsum([len(g) for g in grids])]), device=cuda)
        freqs = torch.as_tensor(np.concatenate(grids), dtype=torch.float32, device=cuda)
        f_min = torch.as_tensor([g[0] for g in grids], dtype=torch.float32, device=cuda).double()
        if group not in (None, 1):
            f_min = f_min[:1]
    else:
        offsets = None
        freqs = torch.linspace(20.0, 1024.0, 1001, dtype=torch.float32, device=cuda)
        f_min = freqs[:1].double()
    size = freqs.numel() * (batch if case == "per_binary_data" else 1)
    data = torch.as_tensor((rng.normal(size=size) + 1j * rng.normal(size=size)) * 1e-2, dtype=torch.complex64,
                           device=cuda)
    weights = torch.as_tensor(rng.uniform(0.5, 2.0, freqs.numel()), dtype=torch.float32, device=cuda)
    with Pipeline(cuda) as pipe:
        loss, grad, status = likelihood_batches(approximant, params, freqs, data, weights, offsets, t_c=t_c,
                                                f_min=f_min, antenna=(0.6, -0.3), scale=-0.5, group=group,
                                                pipeline=pipe)
        torch.cuda.synchronize()
    for k in range(K):
        e_loss, e_grad, e_status = ops.fused_loss_from_params(approximant, params[k], f_min, freqs, offsets, t_c[k],
                                                              data, weights, antenna=(0.6, -0.3), scale=-0.5)
        assert torch.equal(loss[k], e_loss) and torch.equal(grad[k], e_grad) and torch.equal(status[k], e_status), k


def test_likelihood_batches_refusals(cuda):
    import torch

    import waveformx_b200 as wb
    from waveformx_b200.pipeline import likelihood_batches

    freqs = torch.linspace(20.0, 512.0, 101, dtype=torch.float32, device=cuda)
    data = torch.zeros(101, dtype=torch.complex64, device=cuda)
    weights = torch.ones(101, dtype=torch.float32, device=cuda)
    params = torch.as_tensor(np.stack([draw_batch(np.random.default_rng(1), 4)] * 2), device=cuda)
    with pytest.raises(wb.UnsupportedError):
        likelihood_batches("IMRPhenomXHM", params, freqs, data, weights)
    with pytest.raises(ValueError):
        likelihood_batches("IMRPhenomXAS", params[0], freqs, data, weights)
    with pytest.raises(ValueError):
        likelihood_batches("IMRPhenomXAS", params, freqs, data[:100], weights)
    with pytest.raises(ValueError):
        likelihood_batches("IMRPhenomXAS", params, freqs, data, weights, t_c=torch.zeros(3, device=cuda))
    with pytest.raises(ValueError):
        likelihood_batches("IMRPhenomXAS", params, freqs, data, weights, group=2,
                           f_min=torch.full((4,), 20.0, dtype=torch.float64, device=cuda))
    with pytest.raises(ValueError):
        likelihood_batches("IMRPhenomXAS", params, freqs, data, weights,
                           workspace=torch.empty(16, dtype=torch.uint8, device=cuda))


def test_likelihood_stream_refuses_data_of_other_sizes(cuda):
    """data and weights must have one value per frequency or one per
    element of the batch's strain (no stride is guessed from other sizes)."""
    import torch

    from waveformx_b200.pipeline import likelihood_stream

    freqs = torch.linspace(20.0, 512.0, 101, dtype=torch.float32, device=cuda)
    params = torch.as_tensor(draw_batch(np.random.default_rng(2), 4), device=cuda)
    weights = torch.ones(101, dtype=torch.float32, device=cuda)
    for size in (100, 4 * 101 - 1, 3 * 101):
        data = torch.zeros(size, dtype=torch.complex64, device=cuda)
        with pytest.raises(ValueError):
            next(likelihood_stream("IMRPhenomXAS", [params], freqs, data, weights))
    data = torch.zeros(101, dtype=torch.complex64, device=cuda)
    with pytest.raises(ValueError):
        next(likelihood_stream("IMRPhenomXAS", [params], freqs, data, weights[:50]))


def test_likelihood_stream_refuses_xhm(cuda):
    import torch

    import waveformx_b200 as wb
    from waveformx_b200.pipeline import likelihood_stream

    freqs = torch.linspace(20.0, 512.0, 101, dtype=torch.float32, device=cuda)
    with pytest.raises(wb.UnsupportedError):
        next(likelihood_stream("IMRPhenomXHM", [], freqs, torch.zeros(101, dtype=torch.complex64, device=cuda),
                               torch.ones(101, dtype=torch.float32, device=cuda)))


@pytest.mark.parametrize("approximant", ["IMRPhenomXAS", "IMRPhenomD", "TaylorF2", "IMRPhenomXHM"])
@pytest.mark.parametrize("precision", ["fp32", "fp64"])
@pytest.mark.parametrize("ragged", [False, True])
@pytest.mark.parametrize("ring, group", [(None, 1), (2, None), (2, 2), (None, 4)])
def test_batches_in_one_call_equal_eager(cuda, approximant, precision, ragged, ring, group):
    """``polarizations_batches`` (``wfx_pipeline_run``: K batches queued by one
    library call) gives each batch the eager set-up + polarizations bit for
    bit, whether each batch has its own outputs or two slots alternate."""
    import torch

    from waveformx_b200 import _lib, ops
    from waveformx_b200.pipeline import Pipeline, polarizations_batches

    prec = _lib.FP32 if precision == "fp32" else _lib.FP64
    real = torch.float32 if precision == "fp32" else torch.float64
    rng = np.random.default_rng(23)
    K, batch = 5, 20
    params = torch.as_tensor(np.stack([draw_batch(rng, batch) for _ in range(K)]), device=cuda)
    t_c = torch.as_tensor(rng.uniform(-0.05, 0.05, (K, batch)), dtype=real, device=cuda)
    if ragged:
        grids = _ragged(rng, params[0].cpu().numpy())
        offsets = torch.as_tensor(np.concatenate([[0], np.cumsum([len(g) for g in grids])]), device=cuda)
        freqs = torch.as_tensor(np.concatenate(grids), dtype=real, device=cuda)
        f_min = torch.as_tensor([g[0] for g in grids], dtype=real, device=cuda).double()
    else:
        offsets = None
        freqs = torch.linspace(20.0, 1024.0, 1001, dtype=real, device=cuda)
        f_min = freqs[:1].double()
    pipe = Pipeline(cuda)
    if ragged and group != 1:
        f_min = f_min[:1].contiguous()  # (one f_min for every binary: the grouped set-ups' rule)
    hp, hc, status = polarizations_batches(approximant, params, freqs, offsets, t_c=t_c, f_min=f_min,
                                           precision=prec, ring=ring, group=group, pipeline=pipe)
    # (with two slots, the last two batches are the ones left in them)
    kept = range(K) if ring is None else range(K - 2, K)
    for k in kept:
        tables = ops.setup(approximant, params[k].contiguous(), f_min, precision=prec)
        ep, ec = ops.polarizations(approximant, tables.table, freqs, offsets, t_c[k].contiguous())
        slot = k if ring is None else k % ring
        assert torch.equal(hp[slot], ep) and torch.equal(hc[slot], ec)
    for k in range(K):
        tables = ops.setup(approximant, params[k].contiguous(), f_min, precision=prec)
        assert torch.equal(status[k], tables.status)
    pipe.close()
