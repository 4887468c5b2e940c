"""The PyTorch drop-in (``waveformx_b200.torch.polarizations_function``):
the behaviour of the reference's ``waveformx.torch`` (its
``tests/test_torch.py``): values against the oracle, gradients of a fixed
real function of the polarizations against central differences, inputs as
mappings, numbers and sequences, broadcasting, the batch rules and errors,
float32/float64 selection and host tensors in and out."""

from __future__ import annotations

import numpy as np
import pytest

import oracle
from conftest import compare
from test_gpu_gradients import fd_gradient, weighted_loss

pytestmark = pytest.mark.gpu

FREQUENCIES = np.geomspace(20.0, 900.0, 300)
ALIGNED = [36.0, 29.0, 0.0, 0.0, 0.3, 0.0, 0.0, -0.4, 500.0, 0.7, 1.2, 25.0]
BATCH = [ALIGNED, [50.0, 8.0, 0.0, 0.0, 0.9, 0.0, 0.0, 0.3, 300.0, 2.1, 0.3, 30.0],
         [150.0, 100.0, 0.0, 0.0, -0.5, 0.0, 0.0, 0.95, 3000.0, 0.4, 2.0, 0.0]]


def binary_of(x):
    import waveformx_b200 as wb

    return wb.Binary(x[..., 0], x[..., 1], x[..., 2:5], x[..., 5:8], x[..., 8], x[..., 9], x[..., 10], x[..., 11])


def aligned(rows):
    rows = np.atleast_2d(rows)
    return rows[:, [0, 1, 4, 7, 8, 9, 10, 11]]


@pytest.mark.parametrize("approximant", ["IMRPhenomXAS", "IMRPhenomD", "TaylorF2"])
@pytest.mark.parametrize("dtype", ["float64", "float32"])
@pytest.mark.parametrize("batched", [False, True])
def test_values_and_gradients(cuda, approximant, dtype, batched):
    import torch

    import waveformx_b200.torch as wt

    tdtype = getattr(torch, dtype)
    rows = np.asarray(BATCH if batched else ALIGNED)
    if dtype == "float32":
        rows = rows.astype(np.float32).astype(np.float64)
    grid = FREQUENCIES.astype(np.float32).astype(np.float64) if dtype == "float32" else FREQUENCIES
    f = wt.polarizations_function(approximant)
    fields = [torch.tensor(np.asarray(v), dtype=tdtype, device=cuda, requires_grad=True) for v in binary_of(rows)]
    import waveformx_b200 as wb

    hp, hc = f(wb.Binary(*fields), torch.tensor(grid, dtype=tdtype, device=cuda))
    assert hp.dtype == (torch.complex64 if dtype == "float32" else torch.complex128)
    assert hp.shape == ((3, len(grid)) if batched else (len(grid),))
    ref_p, ref_c = oracle.polarizations(approximant, aligned(rows), grid)
    if not batched:
        ref_p, ref_c = ref_p[0], ref_c[0]
    tol = 1e-10 if dtype == "float64" else 1e-4
    for a, b in ((hp, ref_p), (hc, ref_c)):
        a = a.detach().cpu().numpy()
        np.testing.assert_allclose(a, b, rtol=tol, atol=tol * np.max(np.abs(b)))
    w = np.random.default_rng(5).normal(size=(4,) + tuple(hp.shape))
    tw = torch.as_tensor(w, dtype=tdtype, device=cuda)
    loss = (tw[0] * hp.real + tw[1] * hp.imag + tw[2] * hc.real + tw[3] * hc.imag).sum()
    grads = torch.autograd.grad(loss, fields)
    params = aligned(rows)
    wl = w if batched else w[:, None, :]
    fd = fd_gradient(lambda p, tc: weighted_loss(approximant, p, grid, tc, wl), params, np.zeros(len(params)))
    # (f_ref = 0 selects the first frequency, or for TaylorF2 the reference
    # at coalescence: no derivative there)
    fd[params[:, 7] == 0, 7] = 0.0
    expected = [fd[:, 0], fd[:, 1], fd[:, 2], fd[:, 3], fd[:, 4], fd[:, 5], fd[:, 6], fd[:, 7]]
    for k, (g, e) in enumerate(zip(grads, expected)):
        g = g.detach().cpu().numpy().astype(np.float64)
        if k in (2, 3):
            assert np.all(g[..., :2] == 0)
            g = g[..., 2]
        g = np.reshape(g, np.shape(e))
        scale = np.max(np.abs(fd), axis=1)
        if k == 7:
            e = np.where(params[:, 7] == 0, g, e)
        if dtype == "float64":
            np.testing.assert_allclose(g, e, rtol=1e-5, atol=1e-6 * scale.max(), err_msg=str(k))
        else:
            assert np.all(np.abs(g - e) <= 1e-2 * np.abs(e) + 1e-3 * scale), (k, g, e)


def test_inputs(cuda):
    """Mappings, numbers, sequences of tensors and broadcast fields; the
    gradient reaches each tensor asked for; the reference's errors."""
    import torch

    import waveformx_b200 as wb
    import waveformx_b200.torch as wt

    f = wt.polarizations_function("IMRPhenomXAS")
    grid = torch.tensor(FREQUENCIES, device=cuda)
    reference = f(binary_of(torch.tensor(ALIGNED, dtype=torch.float64, device=cuda)), grid)
    chi = torch.tensor(0.3, dtype=torch.float64, device=cuda, requires_grad=True)
    binary = dict(mass_1=36.0, mass_2=29, spin_1=(0.0, 0.0, chi), spin_2=[0.0, 0.0, -0.4],
                  luminosity_distance=500.0, inclination=0.7, phi_ref=1.2, f_ref=25.0)
    hp, hc = f(binary, grid)
    assert hp.dtype == torch.complex128
    for a, b in zip((hp, hc), reference):
        torch.testing.assert_close(a, b, rtol=0, atol=0)
    (g,) = torch.autograd.grad(hp.abs().sum(), chi)
    assert torch.isfinite(g) and g != 0
    masses = torch.tensor([36.0, 40.0], dtype=torch.float64, device=cuda, requires_grad=True)
    hp, hc = f({**binary, "mass_1": masses}, grid)
    assert hp.shape == (2, len(FREQUENCIES))
    torch.testing.assert_close(hp[0].detach(), reference[0], rtol=1e-12, atol=1e-12 * float(reference[0].abs().max()))
    g_m, g_chi = torch.autograd.grad(hp.abs().sum(), (masses, chi))
    assert g_m.shape == (2,) and g_chi.shape == ()
    with pytest.raises(TypeError, match="unknown"):
        f({**binary, "mass": 1.0}, grid)
    with pytest.raises(TypeError, match="missing"):
        f({"mass_1": 1.0}, grid)
    with pytest.raises(ValueError, match="batch"):
        f({**binary, "mass_1": masses, "mass_2": torch.ones(3, device=cuda)}, grid)
    with pytest.raises(wb.UnknownApproximantError):
        wt.polarizations_function("IMRPhenomXYZ")
    with pytest.raises(wb.UnsupportedError):
        wt.polarizations_function("NRSur7dq4")
    # host tensors in, host tensors out (copied through the device)
    hp_cpu, _ = f(binary_of(torch.tensor(ALIGNED, dtype=torch.float64)), torch.tensor(FREQUENCIES))
    assert hp_cpu.device.type == "cpu"
    torch.testing.assert_close(hp_cpu, reference[0].cpu(), rtol=0, atol=0)


def test_t_c_extension(cuda):
    """t_c as a keyword or a mapping entry, with its gradient."""
    import torch

    import waveformx_b200.torch as wt

    f = wt.polarizations_function("IMRPhenomXAS")
    grid = torch.tensor(FREQUENCIES, device=cuda)
    b = binary_of(torch.tensor(ALIGNED, dtype=torch.float64, device=cuda))
    t_c = torch.tensor(0.03, dtype=torch.float64, device=cuda, requires_grad=True)
    hp, hc = f(b, grid, t_c=t_c)
    hp0, _ = f(b, grid)
    shift = torch.exp(-2j * np.pi * grid * 0.03)
    torch.testing.assert_close(hp, hp0 * shift, rtol=1e-10, atol=1e-10 * float(hp0.abs().max()))
    hp2, _ = f({**b._asdict(), "t_c": t_c}, grid)
    torch.testing.assert_close(hp2, hp, rtol=0, atol=0)
    (g,) = torch.autograd.grad(hp.real.sum(), t_c)
    eps = 1e-7
    num = (f(b, grid, t_c=0.03 + eps)[0].real.sum() - f(b, grid, t_c=0.03 - eps)[0].real.sum()) / (2 * eps)
    assert float(g) == pytest.approx(float(num), rel=1e-5)


def test_compare_metric_on_c0(cuda):
    """The single-binary workload (float64) through the torch function."""
    import torch

    import waveformx_b200 as wb
    import waveformx_b200.torch as wt
    from conftest import golden

    g = golden("xas_cases")
    p = g["single_params"][0]
    f = wt.polarizations_function("IMRPhenomXAS")
    hp, hc = f(wb.Binary(p[0], p[1], (0, 0, p[2]), (0, 0, p[3]), p[4], p[5], p[6], p[7]),
               torch.tensor(g["single_frequencies"], device=cuda))
    for a, b in ((hp, g["single_hplus"]), (hc, g["single_hcross"])):
        error, mismatch = compare(a.cpu().numpy(), b)
        assert error < 1e-10 and mismatch < 1e-14


@pytest.mark.parametrize("approximant", ["IMRPhenomXAS", "TaylorF2", "IMRPhenomXHM"])
def test_empty_inputs(cuda, approximant):
    """No binary, or no frequency: empty outputs of the batch's shape, and
    zero gradients of the fields' shapes (the reference's vmapped function
    on empty axes)."""
    import torch

    import waveformx_b200.torch as wt

    f = wt.polarizations_function(approximant)
    grid = torch.as_tensor(FREQUENCIES, device=cuda)
    empty = torch.as_tensor(np.zeros((0, 12)), device=cuda).requires_grad_(True)
    hp, hc = f(binary_of(empty), grid)
    assert tuple(hp.shape) == (0, len(FREQUENCIES)) and hp.dtype == torch.complex128
    (hp.real.sum() + hc.imag.sum()).backward()
    assert tuple(empty.grad.shape) == (0, 12)
    rows = torch.as_tensor(np.array(BATCH), device=cuda).requires_grad_(True)
    no_freq = torch.zeros(0, dtype=torch.float64, device=cuda)
    hp, hc = f(binary_of(rows), no_freq)
    assert tuple(hp.shape) == (3, 0)
    (hp.real.sum() + hc.real.sum()).backward()
    assert torch.equal(rows.grad, torch.zeros_like(rows))
    hp, hc = f(binary_of(rows[0].detach().float()), no_freq.float())
    assert tuple(hp.shape) == (0,) and hp.dtype == torch.complex64
