"""The backward kernel (vector-Jacobian product) and the fused likelihood
with its gradient, against central finite differences of the FP64 oracle.

Bars (the reference's gradient tests, ``tests/test_transforms_xas.py``):
* FP64: relative 1e-5 of central differences (step 1e-6 max(|x|, 1)), with
  an absolute floor of 1e-6 of the largest component;
* FP32: |g32 - g64| <= 1e-2 |g64| + 1e-3 max |g64| against the FP64 kernels.
"""

from __future__ import annotations

import numpy as np
import pytest

import oracle
from oracle.api import psd
from test_gpu_polarizations import draw_batch, f32

pytestmark = pytest.mark.gpu

MODELS = {"xas": "IMRPhenomXAS", "phenomd": "IMRPhenomD", "taylorf2": "TaylorF2"}
F = np.geomspace(20.0, 900.0, 300)


def weighted_loss(approximant, params, f, t_c, w):
    hp, hc = oracle.polarizations(approximant, params, f, t_c=t_c)
    return np.sum(w[0] * hp.real + w[1] * hp.imag + w[2] * hc.real + w[3] * hc.imag, axis=-1)


def fd_gradient(function, params, t_c):
    """Central differences (step 1e-6 max(|x|, 1)) in the 8 parameters and t_c."""
    out = np.zeros((len(params), 9))
    for k in range(9):
        x = t_c if k == 8 else params[:, k]
        h = 1e-6 * np.maximum(np.abs(x), 1.0)
        vals = []
        for sign in (1.0, -1.0):
            p, tc = params.copy(), t_c.copy()
            if k == 8:
                tc = tc + sign * h
            else:
                p[:, k] += sign * h
            vals.append(function(p, tc))
        out[:, k] = (vals[0] - vals[1]) / (2 * h)
    return out


def gpu_vjp(cuda, approximant, params, f, t_c, w, precision):
    import torch

    from waveformx_b200 import _lib, ops

    real = torch.float32 if precision == _lib.FP32 else torch.float64
    cplx = torch.complex64 if precision == _lib.FP32 else torch.complex128
    p = torch.as_tensor(params, dtype=torch.float64, device=cuda)
    freqs = torch.as_tensor(f, dtype=real, device=cuda)
    tables = ops.setup(approximant, p, freqs[:1].to(torch.float64), precision=precision, jvp=True)
    tc = torch.as_tensor(t_c, dtype=real, device=cuda)
    shape = (len(params), len(f))
    gp = torch.as_tensor(np.broadcast_to(w[0] + 1j * w[1], shape).copy(), dtype=cplx, device=cuda)
    gc = torch.as_tensor(np.broadcast_to(w[2] + 1j * w[3], shape).copy(), dtype=cplx, device=cuda)
    return ops.vjp(approximant, tables.table, tables.dtable, freqs, None, tc, gp, gc).cpu().numpy().astype(np.float64)


CASES = np.array([
    [36.0, 29.0, 0.3, -0.4, 500.0, 0.7, 1.2, 25.0],
    [50.0, 2.0, 0.9, 0.3, 300.0, 2.1, 0.3, 30.0],
    [150.0, 100.0, -0.5, 0.95, 3000.0, 0.4, 2.0, 22.0],
])


@pytest.mark.parametrize("model", MODELS)
def test_fp64_vjp_matches_fd(cuda, model):
    approximant = MODELS[model]
    w = np.random.default_rng(5).normal(size=(4, len(F)))
    t_c = np.array([0.0, 0.01, -0.02])
    grad = gpu_vjp(cuda, approximant, CASES, F, t_c, w, 0)
    fd = fd_gradient(lambda p, tc: weighted_loss(approximant, p, F, tc, w), CASES, t_c)
    for i in range(len(CASES)):
        scale = np.max(np.abs(fd[i]))
        np.testing.assert_allclose(grad[i], fd[i], rtol=1e-5, atol=1e-6 * scale)


@pytest.mark.parametrize("model", MODELS)
def test_fp32_vjp_within_bound(cuda, model):
    approximant = MODELS[model]
    w = np.random.default_rng(6).normal(size=(4, len(F)))
    params = f32(CASES)
    t_c = f32([0.0, 0.01, -0.02])
    g64 = gpu_vjp(cuda, approximant, params, f32(F), t_c, w, 0)
    g32 = gpu_vjp(cuda, approximant, params, f32(F), t_c, w, 1)
    for i in range(len(params)):
        bound = 1e-2 * np.abs(g64[i]) + 1e-3 * np.max(np.abs(g64[i]))
        assert np.all(np.abs(g32[i] - g64[i]) <= bound), (i, g32[i], g64[i])


def _fused(cuda, approximant, params, f, t_c, data, w, precision, per_binary):
    import torch

    from waveformx_b200 import _lib, ops

    real = torch.float32 if precision == _lib.FP32 else torch.float64
    cplx = torch.complex64 if precision == _lib.FP32 else torch.complex128
    p = torch.as_tensor(params, dtype=torch.float64, device=cuda)
    freqs = torch.as_tensor(f, dtype=real, device=cuda)
    tables = ops.setup(approximant, p, freqs[:1].to(torch.float64), precision=precision, jvp=True)
    tc = torch.as_tensor(t_c, dtype=real, device=cuda)
    d = torch.as_tensor(data, dtype=cplx, device=cuda)
    wt = torch.as_tensor(w, dtype=real, device=cuda)
    loss, grad = ops.fused_loss(approximant, tables.table, tables.dtable, freqs, None, tc, d, wt)
    return loss.cpu().numpy().astype(np.float64), grad.cpu().numpy().astype(np.float64)


@pytest.mark.parametrize("model", MODELS)
@pytest.mark.parametrize("per_binary", [True, False])
def test_fused_loss_and_gradient(cuda, model, per_binary):
    """L_b = sum_f w |h+_b - d_b|^2 with w = 1/S(f) and d_b the waveform at
    parameters perturbed by 1 % plus complex noise of 0.1 |h| (per binary),
    or one injected signal plus noise (shared)."""
    approximant = MODELS[model]
    rng = np.random.default_rng(9)
    params = f32(draw_batch(rng, 8))
    t_c = f32(rng.uniform(-0.01, 0.01, 8))
    f = f32(np.linspace(20.0, 1024.0, 4017))
    w = 1.0 / psd(f)
    if per_binary:
        shifted = params * (1.0 + 0.01 * rng.normal(size=params.shape))
        shifted[:, 7] = params[:, 7]
        h = oracle.polarizations(approximant, shifted, f)[0]
        data = h + 0.1 * np.abs(h) * (rng.normal(size=h.shape) + 1j * rng.normal(size=h.shape))
    else:
        h = oracle.polarizations(approximant, params[:1], f)[0][0]
        data = h + 0.05 * np.abs(h).max() * (rng.normal(size=h.shape) + 1j * rng.normal(size=h.shape))
    loss_ref = oracle.batch_loss(approximant, params, f, data, w, t_c=t_c)
    fd = oracle.loss_gradient_fd(approximant, params, f, data, w, t_c=t_c)
    for precision, rtol in ((0, 1e-10), (1, 1e-4)):
        loss, grad = _fused(cuda, approximant, params, f, t_c, data, w, precision, per_binary)
        np.testing.assert_allclose(loss, loss_ref, rtol=rtol)
        g = grad[:, [0, 1, 2, 3, 4, 5, 6, 8]]
        for i in range(len(params)):
            scale = np.max(np.abs(fd[i]))
            if precision == 0:
                np.testing.assert_allclose(g[i], fd[i], rtol=1e-5, atol=1e-6 * scale)
            else:
                assert np.all(np.abs(g[i] - fd[i]) <= 1e-2 * np.abs(fd[i]) + 1e-3 * scale), (i, g[i], fd[i])


@pytest.mark.parametrize("model", MODELS)
@pytest.mark.parametrize("ragged", [False, True])
def test_fused_loss_from_params_is_the_same(cuda, model, ragged):
    """The dual-number set-up on a second stream, overlapped with the value
    set-up and the reverse pass, then the contraction: the same bits as the
    set-up with its derivatives followed by the fused call."""
    import torch

    from waveformx_b200 import _lib, ops

    approximant = MODELS[model]
    rng = np.random.default_rng(12)
    params = f32(draw_batch(rng, 40))
    p = torch.as_tensor(params, device=cuda)
    t_c = torch.as_tensor(f32(rng.uniform(-0.01, 0.01, 40)), dtype=torch.float32, device=cuda)
    if ragged:
        lengths = rng.integers(50, 3000, 40)
        offsets = torch.as_tensor(np.concatenate([[0], np.cumsum(lengths)]), device=cuda)
        flat = np.concatenate([np.linspace(20.0, 20.0 + 0.25 * (k - 1), k) for k in lengths])
        freqs = torch.as_tensor(flat, dtype=torch.float32, device=cuda)
        f_min = torch.full((40,), 20.0, dtype=torch.float64, device=cuda)
        d = torch.as_tensor((rng.normal(size=flat.size) + 1j * rng.normal(size=flat.size)) * 1e-2,
                            dtype=torch.complex64, device=cuda)
        w = torch.as_tensor(1.0 / psd(flat), dtype=torch.float32, device=cuda)
    else:
        offsets = None
        f = np.linspace(20.0, 1024.0, 4017)
        freqs = torch.as_tensor(f, dtype=torch.float32, device=cuda)
        f_min = freqs[:1].double()
        d = torch.as_tensor((rng.normal(size=f.size) + 1j * rng.normal(size=f.size)) * 1e-2,
                            dtype=torch.complex64, device=cuda)
        w = torch.as_tensor(1.0 / psd(f), dtype=torch.float32, device=cuda)
    loss, grad, status = ops.fused_loss_from_params(approximant, p, f_min, freqs, offsets, t_c, d, w, scale=-0.5)
    tables = ops.setup(approximant, p, f_min, precision=_lib.FP32, jvp=True)
    loss2, grad2 = ops.fused_loss(approximant, tables.table, tables.dtable, freqs, offsets, t_c, d, w, scale=-0.5)
    assert torch.equal(loss, loss2) and torch.equal(grad, grad2)
    assert torch.equal(status, tables.status)
