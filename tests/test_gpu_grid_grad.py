"""The derivative with respect to the frequency grid (the reference's
drop-in differentiates with respect to its grid for the models that allow
it, ``src/waveformx/torch.py:12-13``): ``ops.grid_vjp`` (the FP64 point on
dual-number frequencies) against fourth-order central differences of the
FP64 loss in single frequencies, and autograd through the drop-in."""

from __future__ import annotations

import numpy as np
import pytest

from test_gpu_polarizations import draw_batch

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("model", ["IMRPhenomXAS", "IMRPhenomD", "TaylorF2", "IMRPhenomXHM"])
def test_grid_gradient_against_differences(cuda, model):
    import torch

    from waveformx_b200 import _lib, ops

    params = draw_batch(np.random.default_rng(12), 3)
    grid = np.geomspace(20.0, 700.0, 301)
    p = torch.as_tensor(params, device=cuda)
    table = ops.setup(model, p, torch.as_tensor(grid[:1], device=cuda), precision=_lib.FP64).table
    rng = np.random.default_rng(13)
    a = rng.normal(size=(3, len(grid))) + 1j * rng.normal(size=(3, len(grid)))
    c = rng.normal(size=(3, len(grid))) + 1j * rng.normal(size=(3, len(grid)))
    tc = torch.as_tensor([0.0, 0.01, -0.02], dtype=torch.float64, device=cuda)

    def loss(g):
        hp, hc = ops.polarizations(model, table, torch.as_tensor(g, device=cuda), None, tc)
        return float(np.sum((np.conj(a) * hp.cpu().numpy()).real + (np.conj(c) * hc.cpu().numpy()).real))

    got = ops.grid_vjp(model, table, torch.as_tensor(grid, device=cuda), None, tc, torch.as_tensor(a, device=cuda),
                       torch.as_tensor(c, device=cuda)).cpu().numpy()
    for k in (1, 37, 150, 222, 300):
        h = 1e-7 * grid[k]

        def at(j):
            g = grid.copy()
            g[k] += j * h
            return loss(g)

        fd = (8.0 * (at(1) - at(-1)) - (at(2) - at(-2))) / (12.0 * h)
        assert abs(got[k] - fd) <= 1e-5 * abs(fd) + 1e-9 * np.max(np.abs(got)), (model, k, got[k], fd)


def test_drop_in_grid_gradient(cuda):
    """grid.requires_grad through polarizations_function: FP64 equals
    ops.grid_vjp; FP32 close to it."""
    import torch

    from waveformx_b200 import _lib, ops
    from waveformx_b200.torch import polarizations_function

    params = draw_batch(np.random.default_rng(14), 2)
    f = polarizations_function("IMRPhenomXAS")
    rng = np.random.default_rng(15)
    grid_np = np.linspace(20.0, 500.0, 400)
    a = torch.as_tensor(rng.normal(size=(2, 400)) + 1j * rng.normal(size=(2, 400)), device=cuda)
    out = {}
    for dtype in (torch.float64, torch.float32):
        grid = torch.tensor(grid_np, dtype=dtype, device=cuda, requires_grad=True)
        binary = dict(mass_1=torch.tensor(params[:, 0], dtype=dtype), mass_2=torch.tensor(params[:, 1], dtype=dtype),
                      spin_1=torch.tensor(np.stack([0 * params[:, 2], 0 * params[:, 2], params[:, 2]], -1), dtype=dtype),
                      spin_2=torch.tensor(np.stack([0 * params[:, 3], 0 * params[:, 3], params[:, 3]], -1), dtype=dtype),
                      luminosity_distance=torch.tensor(params[:, 4], dtype=dtype),
                      inclination=torch.tensor(params[:, 5], dtype=dtype), phi_ref=torch.tensor(params[:, 6], dtype=dtype),
                      f_ref=torch.tensor(params[:, 7], dtype=dtype))
        hp, hc = f(binary, grid)
        loss = (torch.conj(a.to(hp.dtype)) * hp).real.sum() + (torch.conj(a.to(hc.dtype)) * hc).real.sum()
        loss.backward()
        out[dtype] = grid.grad.double().cpu().numpy()
    p = torch.as_tensor(params, device=cuda)
    g64 = torch.as_tensor(grid_np, device=cuda)
    table = ops.setup("IMRPhenomXAS", p, g64[:1], precision=_lib.FP64).table
    ref = ops.grid_vjp("IMRPhenomXAS", table, g64, None, None, a, a).cpu().numpy()
    np.testing.assert_allclose(out[torch.float64], ref, rtol=1e-12, atol=1e-12 * np.max(np.abs(ref)))
    # (FP32 inputs: the same FP64 derivative, of the FP32-rounded parameters,
    # whose phase moves by ~1e-3 rad)
    assert np.max(np.abs(out[torch.float32] - ref)) <= 1e-2 * np.max(np.abs(ref))


def test_xhm_ragged_grid_gradient(cuda):
    """IMRPhenomXHM on a ragged grid: each binary's elements are the
    derivative of its own row, which is the one-binary shared-grid
    derivative of that binary."""
    import torch

    from waveformx_b200 import _lib, ops

    model = "IMRPhenomXHM"
    params = draw_batch(np.random.default_rng(16), 3)
    grids = [np.geomspace(20.0, 600.0, 150), np.geomspace(25.0, 800.0, 211), np.geomspace(30.0, 400.0, 97)]
    p = torch.as_tensor(params, device=cuda)
    f_min = torch.as_tensor([g[0] for g in grids], device=cuda)
    table = ops.setup(model, p, f_min, precision=_lib.FP64).table
    offsets = torch.as_tensor(np.concatenate([[0], np.cumsum([len(g) for g in grids])]), device=cuda)
    flat = torch.as_tensor(np.concatenate(grids), device=cuda)
    rng = np.random.default_rng(17)
    n = flat.numel()
    a = torch.as_tensor(rng.normal(size=n) + 1j * rng.normal(size=n), device=cuda)
    c = torch.as_tensor(rng.normal(size=n) + 1j * rng.normal(size=n), device=cuda)
    tc = torch.as_tensor([0.0, 0.02, -0.01], dtype=torch.float64, device=cuda)
    got = ops.grid_vjp(model, table, flat, offsets, tc, a, c).cpu().numpy()
    assert np.all(np.isfinite(got))
    for b in range(3):
        lo, hi = int(offsets[b]), int(offsets[b + 1])
        one = ops.grid_vjp(model, table[b:b + 1], flat[lo:hi], None, tc[b:b + 1], a[None, lo:hi],
                           c[None, lo:hi]).cpu().numpy()
        np.testing.assert_allclose(got[lo:hi], one, rtol=1e-13, atol=0.0)


def test_xhm_drop_in_grid_gradient(cuda):
    """grid.requires_grad through IMRPhenomXHM's drop-in: FP64 equals
    ops.grid_vjp of the FP64 rows, with the parameters' gradient beside it."""
    import torch

    from waveformx_b200 import _lib, ops
    from waveformx_b200.torch import polarizations_function

    params = draw_batch(np.random.default_rng(18), 2)
    f = polarizations_function("IMRPhenomXHM")
    rng = np.random.default_rng(19)
    grid_np = np.linspace(20.0, 500.0, 300)
    a = torch.as_tensor(rng.normal(size=(2, 300)) + 1j * rng.normal(size=(2, 300)), device=cuda)
    grid = torch.tensor(grid_np, dtype=torch.float64, device=cuda, requires_grad=True)
    mass_1 = torch.tensor(params[:, 0], dtype=torch.float64, requires_grad=True)
    binary = dict(mass_1=mass_1, mass_2=torch.tensor(params[:, 1]),
                  spin_1=torch.tensor(np.stack([0 * params[:, 2], 0 * params[:, 2], params[:, 2]], -1)),
                  spin_2=torch.tensor(np.stack([0 * params[:, 3], 0 * params[:, 3], params[:, 3]], -1)),
                  luminosity_distance=torch.tensor(params[:, 4]), inclination=torch.tensor(params[:, 5]),
                  phi_ref=torch.tensor(params[:, 6]), f_ref=torch.tensor(params[:, 7]))
    hp, hc = f(binary, grid)
    loss = (torch.conj(a) * hp).real.sum() + (torch.conj(a) * hc).real.sum()
    loss.backward()
    p = torch.as_tensor(params, device=cuda)
    g64 = torch.as_tensor(grid_np, device=cuda)
    table = ops.setup("IMRPhenomXHM", p, g64[:1], precision=_lib.FP64).table
    ref = ops.grid_vjp("IMRPhenomXHM", table, g64, None, None, a, a).cpu().numpy()
    np.testing.assert_allclose(grid.grad.cpu().numpy(), ref, rtol=1e-12, atol=1e-12 * np.max(np.abs(ref)))
    assert mass_1.grad is not None and torch.all(torch.isfinite(mass_1.grad))
