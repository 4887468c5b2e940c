"""Parity at the workloads' own shapes, where the small cases of the other
tests do not reach:

* the ragged batch of 16384 binaries on their own grids: binaries drawn as
  it draws them, with durations of 16, 32 and 64 s (grid spacing 1/16 to
  1/64 Hz) and rows of up to ~131k frequencies, through the persistent
  ragged forward with its default work items and with every item length
  the autotuner chooses from, against the FP64 oracle;
* the fused likelihood at scale: 8192 frequencies on linspace(10, 2048),
  t_c uniform in [-0.1, 0.1] s, the data one injected binary plus complex
  Gaussian noise of variance eps^2 S(f) (SNR 20), the loss and its gradient
  from the parameters (the dual-number set-up overlapped with the reverse
  pass) against the plain FP64 unfused path (strain to memory, residual,
  backward), which the oracle pins.

Bars: the waveform bars of the other FP32 tests (mismatch <= 1e-6, phase
<= 1e-3 rad, amplitude <= 1e-4); loss relative 1e-4; the gradient within
the reference's FP32 bound |g32 - g64| <= 1e-2 |g64| + 1e-3 max |g64|
(its tests/test_transforms_xas.py) of the FP64 gradient.
"""

from __future__ import annotations

import numpy as np
import pytest

import oracle
from oracle.api import psd
from test_gpu_polarizations import check_fp32, draw_batch, f32

pytestmark = pytest.mark.gpu

MTSUN_SI = 4.925490947641267e-06
ITEM_LENGTHS = (510, 1022, 2046, 4094)


def long_ragged_draw(seed=31, count=12):
    """Binaries drawn as the ragged batch draws them (f_low uniform 10-30 Hz,
    f_high = min(2048 Hz, Mf = 0.3)), durations 16, 32 or 64 s: the
    ``count`` longest rows of 2048 draws plus ``count`` of the others."""
    rng = np.random.default_rng(seed)
    pool = 2048
    params = f32(draw_batch(rng, pool))
    f_low = rng.uniform(10.0, 30.0, pool)
    duration = rng.choice([16.0, 32.0, 64.0], pool)
    f_high = np.minimum(2048.0, 0.3 / ((params[:, 0] + params[:, 1]) * MTSUN_SI))
    lengths = np.floor((f_high - f_low) * duration).astype(np.int64)
    order = np.argsort(lengths)[::-1]
    pick = np.concatenate([order[:count], rng.choice(order[count:], count, replace=False)])
    grids = [f32(f_low[i] + np.arange(lengths[i]) / duration[i]) for i in pick]
    return params[pick], grids, duration[pick]


@pytest.fixture(scope="module")
def long_ragged():
    params, grids, duration = long_ragged_draw()
    refs = [oracle.polarizations("IMRPhenomXAS", params[i:i + 1], grids[i]) for i in range(len(grids))]
    return params, grids, duration, refs


def test_long_ragged_draw_covers_the_workload(long_ragged):
    _, grids, duration, _ = long_ragged
    lengths = np.array([len(g) for g in grids])
    assert lengths.max() > 120_000 and (lengths > 65_000).sum() >= 8
    assert set(duration) == {16.0, 32.0, 64.0}


@pytest.mark.parametrize("item", ("default",) + ITEM_LENGTHS)
def test_long_ragged_rows_against_the_oracle(cuda, long_ragged, item):
    import torch

    from waveformx_b200 import _lib, ops, tuning

    params, grids, _, refs = long_ragged
    lengths = [len(g) for g in grids]
    offsets = torch.as_tensor(np.concatenate([[0], np.cumsum(lengths)]), dtype=torch.int64, device=cuda)
    flat = torch.as_tensor(np.concatenate(grids), dtype=torch.float32, device=cuda)
    f_min = torch.as_tensor([g[0] for g in grids], dtype=torch.float64, device=cuda)
    batch, n = len(grids), flat.numel()
    before = tuning.lookup("IMRPhenomXAS", batch, n)
    try:
        if item != "default":
            tuning.install("IMRPhenomXAS", batch, n, item, 4)
        tables = ops.setup("IMRPhenomXAS", torch.as_tensor(params, device=cuda), f_min, precision=_lib.FP32)
        hp, hc = ops.polarizations("IMRPhenomXAS", tables.table, flat, offsets)
        torch.cuda.synchronize()
    finally:
        tuning.install("IMRPhenomXAS", batch, n, before[0], before[1])
    hp, hc = hp.cpu().numpy().astype(np.complex128), hc.cpu().numpy().astype(np.complex128)
    cuts = np.cumsum(lengths)[:-1]
    for i, (a, b) in enumerate(zip(np.split(hp, cuts), np.split(hc, cuts))):
        check_fp32(a[None], b[None], refs[i][0], refs[i][1], grids[i])


def test_long_ragged_autotuned(cuda, long_ragged):
    """The autotuner's choice on this problem gives the oracle's waveforms."""
    import torch

    from waveformx_b200 import _lib, ops, tuning

    params, grids, _, refs = long_ragged
    lengths = [len(g) for g in grids]
    offsets = torch.as_tensor(np.concatenate([[0], np.cumsum(lengths)]), dtype=torch.int64, device=cuda)
    flat = torch.as_tensor(np.concatenate(grids), dtype=torch.float32, device=cuda)
    f_min = torch.as_tensor([g[0] for g in grids], dtype=torch.float64, device=cuda)
    batch, n = len(grids), flat.numel()
    before = tuning.lookup("IMRPhenomXAS", batch, n)
    tables = ops.setup("IMRPhenomXAS", torch.as_tensor(params, device=cuda), f_min, precision=_lib.FP32)
    try:
        chosen = tuning.autotune_ragged("IMRPhenomXAS", tables.table, flat, offsets, save=False)
        assert chosen[0] in ITEM_LENGTHS
        hp, _ = ops.polarizations("IMRPhenomXAS", tables.table, flat, offsets)
        torch.cuda.synchronize()
    finally:
        tuning.install("IMRPhenomXAS", batch, n, before[0], before[1])
    hp = hp.cpu().numpy().astype(np.complex128)
    for i, a in enumerate(np.split(hp, np.cumsum(lengths)[:-1])):
        w = 1.0 / psd(grids[i])
        assert oracle.mismatch(a[None], refs[i][0], w)[0] <= 1e-6
        assert np.nanmax(oracle.phase_error(a[None], refs[i][0])) <= 1e-3


def scale_likelihood_problem(batch=48, seed=41, snr=20.0):
    """Binaries drawn as the batch draws them with t_c uniform [-0.1, 0.1] s
    on linspace(10, 2048, 8192); the data: binary 0's h+ (FP64 oracle) plus
    complex Gaussian noise of variance eps^2 S(f), eps set for an SNR of
    ``snr`` with w = 1 / S."""
    rng = np.random.default_rng(seed)
    params = f32(draw_batch(rng, batch))
    t_c = f32(rng.uniform(-0.1, 0.1, batch))
    f = f32(np.linspace(10.0, 2048.0, 8192))
    s = psd(f)
    h = oracle.polarizations("IMRPhenomXAS", params[:1], f, t_c=t_c[:1].astype(np.float64))[0][0]
    eps = np.sqrt(np.sum(np.abs(h) ** 2 / s)) / snr
    noise = eps * np.sqrt(s / 2.0) * (rng.normal(size=f.size) + 1j * rng.normal(size=f.size))
    return params, t_c, f, h + noise, 1.0 / s


def test_fused_likelihood_at_scale_against_fp64_unfused(cuda):
    import torch

    from waveformx_b200 import _lib, ops

    params, t_c, f, data, w = scale_likelihood_problem()
    batch = len(params)
    p = torch.as_tensor(params, device=cuda)
    # FP32: the fused loss and gradient from the parameters
    f32_t = torch.as_tensor(f, dtype=torch.float32, device=cuda)
    loss32, grad32, status = ops.fused_loss_from_params(
        "IMRPhenomXAS", p, f32_t[:1].double(), f32_t, None, torch.as_tensor(t_c, dtype=torch.float32, device=cuda),
        torch.as_tensor(data, dtype=torch.complex64, device=cuda),
        torch.as_tensor(w, dtype=torch.float32, device=cuda), scale=-0.5)
    assert int(status.abs().sum()) == 0
    # FP64, unfused: the strain to memory, the residual, the backward
    f64_t = torch.as_tensor(f, device=cuda)
    tc64 = torch.as_tensor(t_c.astype(np.float64), device=cuda)
    tables = ops.setup("IMRPhenomXAS", p, f64_t[:1], precision=_lib.FP64, jvp=True)
    hp, hc = ops.polarizations("IMRPhenomXAS", tables.table, f64_t, None, tc64)
    d64 = torch.as_tensor(data, device=cuda)
    w64 = torch.as_tensor(w, device=cuda)
    r = hp - d64
    loss64 = (-0.5 * (w64 * (r.real ** 2 + r.imag ** 2)).sum(-1)).cpu().numpy()
    grad64 = ops.vjp("IMRPhenomXAS", tables.table, tables.dtable, f64_t, None, tc64, (-w64 * r).contiguous(),
                     torch.zeros_like(hc)).cpu().numpy()
    # the FP64 unfused path is the oracle's
    np.testing.assert_allclose(loss64, oracle.batch_loss("IMRPhenomXAS", params, f, data, w, t_c=t_c, scale=-0.5),
                               rtol=1e-10)
    loss32 = loss32.cpu().numpy().astype(np.float64)
    grad32 = grad32.cpu().numpy().astype(np.float64)
    np.testing.assert_allclose(loss32, loss64, rtol=1e-4)
    for i in range(batch):
        bound = 1e-2 * np.abs(grad64[i]) + 1e-3 * np.max(np.abs(grad64[i]))
        assert np.all(np.abs(grad32[i] - grad64[i]) <= bound), (i, grad32[i], grad64[i])
    # the FP32 waveforms the fused kernel evaluates: mismatch <= 1e-6 per binary
    t32 = ops.setup("IMRPhenomXAS", p, f32_t[:1].double(), precision=_lib.FP32)
    h32, _ = ops.polarizations("IMRPhenomXAS", t32.table, f32_t, None,
                               torch.as_tensor(t_c, dtype=torch.float32, device=cuda))
    mm = oracle.mismatch(h32.cpu().numpy().astype(np.complex128), hp.cpu().numpy(), w)
    assert np.max(mm) <= 1e-6, np.max(mm)
