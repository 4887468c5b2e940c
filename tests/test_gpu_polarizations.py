"""(hplus, hcross) from the kernels against the golden vectors (FP64) and the
oracle (FP32, at the float32-rounded inputs), through the C ABI.

Bars:
* FP64 (the plain form): the reference's own bar against LAL, relative
  error < 1e-10 and mismatch < 1e-14 (its ``tests/test_xas.py:65-72``);
* FP32 with double-float phase: noise-weighted mismatch <= 1e-6 and the
  largest phase error <= 1e-3 rad against the FP64 oracle (where the
  amplitude exceeds 1e-3 of its peak), relative amplitude error <= 1e-4.
"""

from __future__ import annotations

import numpy as np
import pytest

import oracle
from conftest import compare, golden
from oracle.api import amplitude_error, psd

pytestmark = pytest.mark.gpu

MODELS = {"xas": "IMRPhenomXAS", "phenomd": "IMRPhenomD", "taylorf2": "TaylorF2"}


def gpu_polarizations(cuda, approximant, params, freqs, precision, t_c=None, reference_mf=None, amp_scale=1e21):
    """The kernels' (hplus, hcross) for a shared grid ``freqs`` (N,) or a
    list of per-binary grids (ragged)."""
    import torch

    from waveformx_b200 import _lib, ops

    real = torch.float32 if precision == _lib.FP32 else torch.float64
    p = torch.as_tensor(np.asarray(params, dtype=np.float64), device=cuda)
    if isinstance(freqs, list):
        lengths = [len(g) for g in freqs]
        offsets = torch.as_tensor(np.concatenate([[0], np.cumsum(lengths)]), dtype=torch.int64, device=cuda)
        flat = torch.as_tensor(np.concatenate(freqs), dtype=real, device=cuda)
        f_min = torch.as_tensor([g[0] for g in freqs], dtype=torch.float64, device=cuda)
    else:
        offsets = None
        flat = torch.as_tensor(np.asarray(freqs), dtype=real, device=cuda)
        f_min = flat[:1].to(torch.float64)
    tables = ops.setup(approximant, p, f_min, amp_scale=amp_scale, reference_mf=reference_mf, precision=precision)
    tc = None if t_c is None else torch.as_tensor(np.asarray(t_c), dtype=real, device=cuda)
    hp, hc = ops.polarizations(approximant, tables.table, flat, offsets, tc)
    hp, hc = hp.cpu().numpy().astype(np.complex128), hc.cpu().numpy().astype(np.complex128)
    if offsets is not None:
        cuts = np.cumsum(lengths)[:-1]
        return np.split(hp, cuts), np.split(hc, cuts)
    return hp, hc


def draw_batch(rng, n):
    """Binaries as the 4096-binary batch draws them (masses uniform 5-100
    sorted m1 >= m2, aligned spins uniform [-0.99, 0.99], distance uniform
    100-5000 Mpc, cos(inclination) uniform [-1, 1], phi_ref uniform
    [0, 2 pi), f_ref 20 Hz)."""
    m = rng.uniform(5.0, 100.0, size=(n, 2))
    chi = rng.uniform(-0.99, 0.99, size=(n, 2))
    return np.stack([m.max(1), m.min(1), chi[:, 0], chi[:, 1], rng.uniform(100.0, 5000.0, n),
                     np.arccos(rng.uniform(-1.0, 1.0, n)), rng.uniform(0.0, 2 * np.pi, n), np.full(n, 20.0)], 1)


def f32(x):
    return np.asarray(x, dtype=np.float32).astype(np.float64)


def check_fp32(hp, hc, ref_p, ref_c, f, phase_tol=1e-3, mismatch_tol=1e-6):
    w = 1.0 / psd(f)
    for a, b in ((hp, ref_p), (hc, ref_c)):
        mm = oracle.mismatch(a, b, w)
        assert np.nanmax(mm) <= mismatch_tol, np.nanmax(mm)
        assert np.nanmax(oracle.mismatch(a, b)) <= mismatch_tol
        pe = oracle.phase_error(a, b)
        assert np.nanmax(pe) <= phase_tol, np.nanmax(pe)
        assert np.nanmax(amplitude_error(a, b)) <= 1e-4


@pytest.mark.parametrize("model", MODELS)
@pytest.mark.parametrize("kind", ["cases", "random", "reference_mf", "unscaled"])
def test_fp64_matches_golden(cuda, model, kind):
    g = golden(f"{model}_{kind}")
    kwargs = {}
    if kind == "reference_mf":
        kwargs["reference_mf"] = float(g["reference_mf"])
    if kind == "unscaled":
        kwargs["amp_scale"] = 1.0
    f = g["frequencies"]
    grids = list(f) if f.ndim == 2 else f
    hp, hc = gpu_polarizations(cuda, MODELS[model], g["params"], grids, 0, **kwargs)
    for i in range(len(g["params"])):
        for a, b in ((hp[i], g["hplus"][i]), (hc[i], g["hcross"][i])):
            if np.all(np.isnan(b)):  # a binary the reference refuses
                assert np.all(np.isnan(a)), i
                continue
            error, mismatch = compare(a, b)
            assert error < 1e-10 and mismatch < 1e-14, (i, error, mismatch)


@pytest.mark.parametrize("model", MODELS)
def test_fp64_single_workload(cuda, model):
    """One binary on linspace(20, 1024, 4017), complex128."""
    g = golden(f"{model}_cases")
    hp, hc = gpu_polarizations(cuda, MODELS[model], g["single_params"], g["single_frequencies"], 0)
    for a, b in ((hp[0], g["single_hplus"]), (hc[0], g["single_hcross"])):
        error, mismatch = compare(a, b)
        assert error < 1e-10 and mismatch < 1e-14


@pytest.mark.parametrize("model", MODELS)
def test_fp32_batch_workload(cuda, model):
    """256 binaries of the batch draw on linspace(20, 1024, 4017) in FP32."""
    params = f32(draw_batch(np.random.default_rng(11), 256))
    f = np.linspace(20.0, 1024.0, 4017)
    hp, hc = gpu_polarizations(cuda, MODELS[model], params, f, 1)
    ref_p, ref_c = oracle.polarizations(MODELS[model], params, f32(f))
    check_fp32(hp, hc, ref_p, ref_c, f)


@pytest.mark.parametrize("model", MODELS)
def test_fp32_golden_cases(cuda, model):
    """The hand-picked cases (mass ratios to 25, spins to 0.995, binary
    neutron stars) on their own grids, in FP32."""
    g = golden(f"{model}_cases")
    params = f32(g["params"])
    grids = [f32(x) for x in g["frequencies"]]
    hp, hc = gpu_polarizations(cuda, MODELS[model], params, grids, 1)
    for i in range(len(params)):
        ref_p, ref_c = oracle.polarizations(MODELS[model], params[i:i + 1], grids[i])
        check_fp32(hp[i][None], hc[i][None], ref_p, ref_c, grids[i])


@pytest.mark.parametrize("model", MODELS)
def test_fp32_binary_neutron_star(cuda, model):
    """A binary neutron star from 20 Hz at 1/256 Hz (half a million
    frequencies; 10^5 rad of inspiral phase): the double-float phase keeps
    the mismatch below 1e-6 (reference ``tests/test_xas.py:90-100``)."""
    f = f32(20.0 + np.arange((2048 - 20) * 256) / 256.0)
    params = f32([[1.42, 1.27, 0.05, -0.03, 100.0, 0.5, 1.0, 0.0]])
    hp, hc = gpu_polarizations(cuda, MODELS[model], params, f, 1)
    ref_p, ref_c = oracle.polarizations(MODELS[model], params, f)
    for a, b in ((hp, ref_p), (hc, ref_c)):
        assert compare(a[0], b[0])[1] < 1e-6
        assert oracle.mismatch(a, b, 1.0 / psd(f))[0] < 1e-6


@pytest.mark.parametrize("approximant", ["IMRPhenomXAS", "TaylorF2"])
@pytest.mark.parametrize("precision", [0, 1])
def test_t_c(cuda, precision, approximant):
    """t_c multiplies the strain by exp(-2 pi i f t_c) (up to 0.1 s: 1.3e3
    rad at 2048 Hz, in double-float for FP32)."""
    rng = np.random.default_rng(5)
    params = f32(draw_batch(rng, 64))
    t_c = f32(rng.uniform(-0.1, 0.1, 64))
    f = f32(np.linspace(10.0, 2048.0, 8192))
    hp, hc = gpu_polarizations(cuda, approximant, params, f, precision, t_c=t_c)
    ref_p, ref_c = oracle.polarizations(approximant, params, f, t_c=t_c)
    if precision == 0:
        for a, b in ((hp, ref_p), (hc, ref_c)):
            for i in range(len(a)):
                error, mismatch = compare(a[i], b[i])
                assert error < 1e-10 and mismatch < 1e-14
    else:
        check_fp32(hp, hc, ref_p, ref_c, f)


@pytest.mark.parametrize("model", MODELS)
def test_fp32_ragged(cuda, model):
    """A ragged batch (per-binary uniform grids, f_low 10-30 Hz, df = 1/T,
    T in 4..64 s, to min(2048 Hz, Mf = 0.3)) in one persistent launch,
    odd offsets included."""
    rng = np.random.default_rng(21)
    n = 24
    params = f32(draw_batch(rng, n))
    grids = []
    for i in range(n):
        f_low = rng.uniform(10.0, 30.0)
        duration = rng.choice([4.0, 8.0])
        f_high = min(2048.0, 0.3 / ((params[i, 0] + params[i, 1]) * 4.925490947641267e-06))
        grids.append(f32(np.arange(f_low, f_high, 1.0 / duration)))
    grids[3] = grids[3][:1]   # a one-frequency binary
    grids[5] = grids[5][:3]
    hp, hc = gpu_polarizations(cuda, MODELS[model], params, grids, 1)
    for i in range(n):
        ref_p, ref_c = oracle.polarizations(MODELS[model], params[i:i + 1], grids[i])
        if len(grids[i]) > 8:
            check_fp32(hp[i][None], hc[i][None], ref_p, ref_c, grids[i])
        else:
            np.testing.assert_allclose(hp[i], ref_p[0], rtol=1e-4, atol=1e-4 * np.abs(ref_p).max())


@pytest.mark.parametrize("n", [1, 2, 3, 509, 510, 511, 1021])
@pytest.mark.parametrize("batch", [1, 3, 17])
def test_fp32_edge_sizes(cuda, n, batch):
    """Grid lengths around the tile sizes and odd batch counts (rows of odd
    length alternate the 16-byte alignment of their first element)."""
    params = f32(draw_batch(np.random.default_rng(n + batch), batch))
    f = f32(np.linspace(20.0, 900.0, n)) if n > 1 else f32([50.0])
    hp, hc = gpu_polarizations(cuda, "IMRPhenomXAS", params, f, 1)
    ref_p, ref_c = oracle.polarizations("IMRPhenomXAS", params, f)
    assert hp.shape == (batch, n)
    for a, b in ((hp, ref_p), (hc, ref_c)):
        np.testing.assert_allclose(a, b, rtol=0, atol=2e-4 * np.max(np.abs(b)))


def test_nan_where_lal_fails(cuda):
    g = golden("xas_nan")
    for precision in (0, 1):
        hp, hc = gpu_polarizations(cuda, "IMRPhenomXAS", g["params"], g["frequencies"], precision)
        assert np.all(np.isnan(hp)) and np.all(np.isnan(hc))


@pytest.mark.parametrize("precision", [0, 1])
def test_zero_above_the_cutoff(cuda, precision):
    """IMRPhenomXAS is exactly zero above f_cut = 0.3 / M (0.33 for
    chi_eff > 0.99), on the shared and the ragged path (the FP32 kernels
    skip those pairs), and NaN there too for a refused binary."""
    params = np.array([[90.0, 80.0, 0.2, -0.1, 400.0, 0.5, 1.0, 20.0],    # f_cut ~ 360 Hz
                       [60.0, 55.0, 0.995, 0.995, 800.0, 1.2, 0.3, 20.0],  # chi_eff > 0.99
                       [2000.0, 1.0, 0.0, 0.0, 400.0, 0.4, 0.0, 20.0]])    # refused: q = 2000
    f = f32(np.linspace(20.0, 1024.0, 1001))
    f_cut = np.array([0.3, 0.33, 0.3]) / (params[:, 0] + params[:, 1]) / 4.925490947641267e-06
    for grid in (f, [f, f[:777], f[1:]]):
        hp, hc = gpu_polarizations(cuda, "IMRPhenomXAS", params, grid, precision)
        for i in range(2):
            g = grid if not isinstance(grid, list) else grid[i]
            above = g > f_cut[i]
            assert above.any() and not above.all()
            assert np.all(hp[i][above] == 0) and np.all(hc[i][above] == 0)
            assert np.all(np.abs(hp[i][~above][:-1]) > 0)
        assert np.all(np.isnan(hp[2])) and np.all(np.isnan(hc[2]))
