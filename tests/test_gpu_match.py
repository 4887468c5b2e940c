"""The matches on the kernels (``waveformx_b200.match``): the known answers
of the reference's ``tests/test_match.py:36-94`` (the Dirichlet kernel of a
shifted flat band, a constant phase, the recovery of time and phase shifts
off the FFT grid, symmetry), rows against the oracle (``oracle/match.py``,
itself pinned to those answers), and the template bank, evaluated from its
tables without its strain, against the templates written out and matched
by the oracle.

Bars: complex128 as the reference's own (1e-12 on recovered matches,
1e-10 relative on the Dirichlet kernel); complex64 series 1e-5 absolute on
matches; the template bank (FP32 templates) 2e-5 against the oracle's match
of the same FP32 templates.
"""

from __future__ import annotations

import numpy as np
import pytest

import oracle
from oracle import match as om
from test_gpu_polarizations import draw_batch, f32

pytestmark = pytest.mark.gpu

DELTA_F = 0.25
FREQUENCIES = np.arange(80, 2049) * DELTA_F  # 20-512 Hz
PSD = (FREQUENCIES / 100.0) ** -4 + 2 + 2 * (FREQUENCIES / 100.0) ** 2


def chirp(theta=0.0):
    x = (np.pi * FREQUENCIES * (1e-4 * (1 + theta))) ** (-5 / 3)
    return FREQUENCIES ** (-7 / 6) * np.exp(-1j * (3 / 128 * x - np.pi / 4))


def shifted(h, t, phi):
    return h * np.exp(-2j * np.pi * FREQUENCIES * t + 1j * phi)


def _t(cuda, x, dtype=None):
    import torch

    return torch.as_tensor(np.asarray(x), device=cuda, dtype=dtype)


def _match(cuda, a, b, psd=PSD, **kw):
    from waveformx_b200 import match

    return match.match(_t(cuda, a), _t(cuda, b), FREQUENCIES, _t(cuda, psd), **kw).cpu().numpy()


def test_dirichlet_kernel(cuda):
    a = np.ones(len(FREQUENCIES), np.complex128)
    flat = np.ones_like(PSD)
    k = len(FREQUENCIES)
    for tau in (1e-3, 0.0123, 0.3):
        expected = abs(np.sin(np.pi * k * DELTA_F * tau) / (k * np.sin(np.pi * DELTA_F * tau)))
        np.testing.assert_allclose(_match(cuda, a, shifted(a, tau, 0.0), flat, time=False), expected, rtol=1e-10,
                                   atol=1e-14)
        assert abs(_match(cuda, a, shifted(a, tau, 0.0), flat)) == pytest.approx(1, abs=1e-12)


def test_constant_phase(cuda):
    a = chirp()
    for phi in (0.3, 2.0, -1.0):
        b = 3.0 * shifted(a, 0.0, phi)
        np.testing.assert_allclose(_match(cuda, a, b, time=False, phase=False), np.cos(phi), rtol=1e-12)
        np.testing.assert_allclose(_match(cuda, a, b, time=False), 1, atol=1e-13)


@pytest.mark.parametrize("t, phi", [(0.0, 0.0), (0.0123456, 0.7), (-0.3141, -2.5), (1.3, 3.0)])
def test_recovers_time_and_phase(cuda, t, phi):
    from waveformx_b200 import match

    a = chirp()
    m, best = match.match(_t(cuda, a), _t(cuda, shifted(a, t, phi)), FREQUENCIES, _t(cuda, PSD), return_time=True)
    assert abs(1 - float(m)) < 1e-12
    # z(t) peaks where b delayed by t lines up with a: t = -(b's delay)
    assert float(best) == pytest.approx(-t, abs=1e-9)
    if t != 0.0:
        assert 1 - _match(cuda, a, shifted(a, t, phi), time=False) > 0.1


def test_rows_against_the_oracle(cuda):
    """Rows of different waveforms and shifts, broadcast against one vector,
    with and without the phase, complex128 and complex64."""
    rng = np.random.default_rng(3)
    a = np.stack([shifted(chirp(th), t, p) for th, t, p in
                  zip(rng.uniform(-3e-3, 3e-3, 12), rng.uniform(-1, 1, 12), rng.uniform(-3, 3, 12))])
    b = chirp(1e-4)
    for phase in (True, False):
        ref = om.match(a, b, FREQUENCIES, PSD, phase=phase)
        np.testing.assert_allclose(_match(cuda, a, b, phase=phase), ref, rtol=0, atol=1e-11)
        got = _match(cuda, a.astype(np.complex64), b.astype(np.complex64), PSD.astype(np.float32), phase=phase)
        np.testing.assert_allclose(got, ref, rtol=0, atol=1e-5)
    # symmetric
    np.testing.assert_allclose(_match(cuda, b, a), om.match(a, b, FREQUENCIES, PSD), rtol=0, atol=1e-11)


@pytest.mark.parametrize("approximant", ["IMRPhenomXAS", "IMRPhenomD", "TaylorF2"])
def test_template_bank(cuda, approximant):
    """A bank of 40 templates against a signal (one of them, delayed and
    phase-shifted, plus nothing else): the fused bank against the oracle's
    match of the same FP32 templates written out, and the injected one
    recovered."""
    import torch

    from waveformx_b200 import _lib, match, ops

    rng = np.random.default_rng(8)
    params = f32(draw_batch(rng, 40))
    f = np.linspace(20.0, 1024.0, 4017)
    w = oracle.psd(f)
    p = torch.as_tensor(params, device=cuda)
    freqs = torch.as_tensor(f, dtype=torch.float32, device=cuda)
    tables = ops.setup(approximant, p, freqs[:1].double(), precision=_lib.FP32)
    hp, _ = ops.polarizations(approximant, tables.table, freqs)
    hp = hp.cpu().numpy().astype(np.complex128)
    fr = f.astype(np.float32).astype(np.float64)
    signal = (hp[7] * np.exp(-2j * np.pi * fr * 0.0217 + 0.9j)).astype(np.complex64)
    got, t = match.template_match(approximant, p, f, torch.as_tensor(signal, device=cuda), w)
    got, t = got.cpu().numpy(), t.cpu().numpy()
    ref = om.match(hp, signal.astype(np.complex128), fr, w.astype(np.float32).astype(np.float64))
    np.testing.assert_allclose(got, ref, rtol=0, atol=2e-5)
    assert got[7] == pytest.approx(1.0, abs=2e-5)
    assert t[7] == pytest.approx(-0.0217, abs=1e-5)  # (the signal is delayed by 0.0217 s)
    # the unfused path (the strain written, then matched) agrees
    unfused = match.match(torch.as_tensor(hp.astype(np.complex64), device=cuda),
                          torch.as_tensor(signal, device=cuda), f, torch.as_tensor(w, dtype=torch.float32,
                                                                                   device=cuda))
    np.testing.assert_allclose(got, unfused.cpu().numpy(), rtol=0, atol=2e-5)


def _pmatch(cuda, signal, hplus, hcross, **kw):
    from waveformx_b200 import match

    return match.polarization_match(_t(cuda, signal), _t(cuda, hplus), _t(cuda, hcross), FREQUENCIES,
                                    _t(cuda, PSD), **kw).cpu().numpy()


def test_polarizations_recovered(cuda):
    hplus = chirp()
    hcross = -1j * chirp(2e-3) * 0.8
    for fp, fx, t in ((0.3, -0.9, 0.01), (1.0, 0.0, -0.2), (0.0, 0.5, 0.0)):
        signal = shifted(fp * hplus + fx * hcross, t, 0.0)
        assert abs(1 - _pmatch(cuda, signal, hplus, hcross)) < 1e-12


def test_polarization_projection(cuda):
    hplus, hcross = chirp(), -1j * chirp(2e-3)
    noise = chirp(-5e-3) * np.exp(0.4j)

    def project(x, onto):
        return x - om.inner_product(x, onto, FREQUENCIES, PSD) / om.inner_product(onto, onto, FREQUENCIES, PSD) * onto

    e2 = project(hcross, hplus)
    orthogonal = project(project(noise, hplus), e2)
    signal = 0.4 * hplus + 0.7 * hcross + orthogonal
    inside = 0.4 * hplus + 0.7 * hcross
    expected = np.sqrt(om.inner_product(inside, inside, FREQUENCIES, PSD)
                       / om.inner_product(signal, signal, FREQUENCIES, PSD))
    np.testing.assert_allclose(_pmatch(cuda, signal, hplus, hcross, time=False), expected, rtol=1e-12)


def test_parallel_polarizations(cuda):
    a = chirp()
    np.testing.assert_allclose(_pmatch(cuda, shifted(a, 0.05, 0.0), a, 0 * a), 1, atol=1e-12)


def test_polarization_rows_against_the_oracle(cuda):
    rng = np.random.default_rng(4)
    signals = np.stack([shifted(0.6 * chirp(th) - 0.3j * chirp(th + 1e-3), t, p) for th, t, p in
                        zip(rng.uniform(-3e-3, 3e-3, 10), rng.uniform(-1, 1, 10), rng.uniform(-3, 3, 10))])
    hplus, hcross = chirp(1e-4), -1j * chirp(1.2e-3)
    ref = om.polarization_match(signals, hplus, hcross, FREQUENCIES, PSD)
    np.testing.assert_allclose(_pmatch(cuda, signals, hplus, hcross), ref, rtol=0, atol=1e-11)
    got = _pmatch(cuda, signals.astype(np.complex64), hplus.astype(np.complex64), hcross.astype(np.complex64))
    np.testing.assert_allclose(got, ref, rtol=0, atol=1e-5)


@pytest.mark.parametrize("approximant", ["IMRPhenomXAS", "TaylorF2"])
def test_template_polarization_bank(cuda, approximant):
    """The bank's polarization matches (their strain never written) against
    the oracle's on the same FP32 polarizations written out; the injected
    binary (any F+, Fx, delayed) recovered."""
    import torch

    from waveformx_b200 import _lib, match, ops

    rng = np.random.default_rng(9)
    params = f32(draw_batch(rng, 24))
    f = np.linspace(20.0, 1024.0, 4017)
    w = oracle.psd(f)
    p = torch.as_tensor(params, device=cuda)
    freqs = torch.as_tensor(f, dtype=torch.float32, device=cuda)
    tables = ops.setup(approximant, p, freqs[:1].double(), precision=_lib.FP32)
    hp, hc = ops.polarizations(approximant, tables.table, freqs)
    hp, hc = hp.cpu().numpy().astype(np.complex128), hc.cpu().numpy().astype(np.complex128)
    fr = f.astype(np.float32).astype(np.float64)
    signal = ((0.3 * hp[5] - 0.8 * hc[5]) * np.exp(-2j * np.pi * fr * 0.031)).astype(np.complex64)
    got, t = match.template_polarization_match(approximant, p, f, torch.as_tensor(signal, device=cuda), w)
    got, t = got.cpu().numpy(), t.cpu().numpy()
    ref = om.polarization_match(signal.astype(np.complex128), hp, hc, fr, w.astype(np.float32).astype(np.float64))
    np.testing.assert_allclose(got, ref, rtol=0, atol=2e-5)
    assert got[5] == pytest.approx(1.0, abs=2e-5)
    assert t[5] == pytest.approx(0.031, abs=1e-5)


@pytest.mark.parametrize("n, pad", [(1969, 4), (4017, 4), (1000, 4), (3000, 2), (5000, 2), (9000, 1)])
def test_grid_time_in_shared_memory(cuda, n, pad):
    """The grid's best time from the inverse FFT in shared memory (16384,
    8192, 4096 times; the grid never written) against the arg-max of the
    cuFFT grid, rows of a template bank's series."""
    import torch

    from waveformx_b200 import _lib, ops

    rng = np.random.default_rng(n)
    params = f32(draw_batch(rng, 64))
    f = np.linspace(20.0, 20.0 + 0.25 * (n - 1), n)
    p = torch.as_tensor(params, device=cuda)
    freqs = torch.as_tensor(f, dtype=torch.float32, device=cuda)
    tables = ops.setup("IMRPhenomXAS", p, freqs[:1].double(), precision=_lib.FP32)
    hp, _ = ops.polarizations("IMRPhenomXAS", tables.table, freqs)
    signal = (hp[3] * torch.exp(torch.tensor(-2j * np.pi * 0.0123, device=cuda) * freqs)).to(torch.complex64)
    n_fft = ops.fft_length(n, pad)
    assert ops.grid_time_supported(n, n_fft)
    series = torch.zeros((64, n_fft), dtype=torch.complex64, device=cuda)
    w = torch.as_tensor(oracle.psd(f), dtype=torch.float32, device=cuda)
    ops.template_overlap("IMRPhenomXAS", tables.table, freqs, signal, w, 0.25, series)
    t_shared = ops.match_grid_time(series, n, 0.25).cpu().numpy()
    z = torch.fft.ifft(series, dim=-1, norm="forward").abs().cpu().numpy()
    j = np.argmax(z, axis=1)
    t_cufft = j / (n_fft * 0.25)
    period = (n_fft - 1) / (n_fft * 0.25) + 1 / (n_fft * 0.25)
    t_cufft = np.where(t_cufft > period / 2, t_cufft - period, t_cufft)
    # (two FP32 transforms: a row whose two largest grid values are within
    # their rounding may pick either)
    same = t_shared == t_cufft
    zs = np.sort(z, axis=1)
    close = (zs[:, -1] - zs[:, -2]) < 1e-5 * zs[:, -1]
    assert np.all(same | close), (t_shared[~same], t_cufft[~same])


def test_template_bank_xhm(cuda):
    """template_match("IMRPhenomXHM", ...): the bank through XHM's kernel
    (its strain, then the series of given waveforms) equals match() of the
    same FP32 templates, and recovers the template that made the signal."""
    import torch

    from waveformx_b200 import _lib, ops
    from waveformx_b200 import match as wm

    rng = np.random.default_rng(21)
    params = f32(draw_batch(rng, 16))
    p = torch.as_tensor(params, device=cuda)
    f = np.linspace(20.0, 20.0 + 0.25 * 1999, 2000)
    f32_t = torch.as_tensor(f, dtype=torch.float32, device=cuda)
    w = torch.as_tensor(oracle.psd(f), dtype=torch.float32, device=cuda)
    t = ops.setup("IMRPhenomXHM", p, f32_t[:1].double(), precision=_lib.FP32)
    hp, hc = ops.polarizations("IMRPhenomXHM", t.table, f32_t)
    fp, fx = 0.6, -0.4
    h = fp * hp + fx * hc
    signal = (h[5] * torch.exp(torch.tensor(-2j * np.pi * 0.013, device=cuda) * f32_t)).to(torch.complex64)
    got, tt = wm.template_match("IMRPhenomXHM", p, f, signal, w, antenna=(fp, fx))
    ref, tref = wm.match(h.contiguous(), signal, f, w, return_time=True)
    np.testing.assert_allclose(got.cpu().numpy(), ref.cpu().numpy(), rtol=0, atol=1e-12)
    np.testing.assert_allclose(tt.cpu().numpy(), tref.cpu().numpy(), rtol=0, atol=1e-12)
    assert float(got[5]) == pytest.approx(1.0, abs=2e-5)
    assert float(tt[5]) == pytest.approx(-0.013, abs=1e-5)
    pm, _ = wm.template_polarization_match("IMRPhenomXHM", p, f, signal, w)
    assert float(pm[5]) == pytest.approx(1.0, abs=2e-5)
