"""The match oracle (``oracle/match.py``) against the known answers of the
reference's own match tests (its ``tests/test_match.py:36-94``): the white
inner product, the Dirichlet kernel of a shifted flat band, a constant phase,
the recovery of time and phase shifts off the FFT grid, and the symmetry of
the mismatch of different waveforms. These pin the oracle, which pins the
kernels (``tests/test_gpu_match.py``)."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import match as om

DELTA_F = 0.25
FREQUENCIES = np.arange(80, 2049) * DELTA_F  # 20-512 Hz
PSD = (FREQUENCIES / 100.0) ** -4 + 2 + 2 * (FREQUENCIES / 100.0) ** 2


def chirp(theta=0.0, frequencies=FREQUENCIES):
    """The reference's test signal: a stationary-phase inspiral
    ``f^(-7/6) e^(-i psi(f))`` with a chirp-mass-like parameter ``theta``."""
    x = (np.pi * frequencies * (1e-4 * (1 + theta))) ** (-5 / 3)
    return frequencies ** (-7 / 6) * np.exp(-1j * (3 / 128 * x - np.pi / 4))


def shifted(h, t, phi):
    return h * np.exp(-2j * np.pi * FREQUENCIES * t + 1j * phi)


def test_inner_product_white():
    a = chirp()
    expected = 4 * DELTA_F * np.sum(np.abs(a) ** 2)
    np.testing.assert_allclose(om.inner_product(a, a, FREQUENCIES, np.ones_like(PSD)), expected, rtol=1e-14)


def test_dirichlet_kernel():
    a = np.ones(len(FREQUENCIES), np.complex128)
    flat = np.ones_like(PSD)
    k = len(FREQUENCIES)
    for tau in (1e-3, 0.0123, 0.3):
        expected = abs(np.sin(np.pi * k * DELTA_F * tau) / (k * np.sin(np.pi * DELTA_F * tau)))
        got = om.match(a, shifted(a, tau, 0.0), FREQUENCIES, flat, time=False)
        np.testing.assert_allclose(got, expected, rtol=1e-10, atol=1e-14)
        assert abs(om.match(a, shifted(a, tau, 0.0), FREQUENCIES, flat)) == pytest.approx(1, abs=1e-12)


def test_constant_phase():
    a = chirp()
    for phi in (0.3, 2.0, -1.0):
        b = 3.0 * shifted(a, 0.0, phi)
        np.testing.assert_allclose(om.match(a, b, FREQUENCIES, PSD, time=False, phase=False), np.cos(phi),
                                   rtol=1e-12)
        np.testing.assert_allclose(om.match(a, b, FREQUENCIES, PSD, time=False), 1, atol=1e-13)


@pytest.mark.parametrize("t, phi", [(0.0, 0.0), (0.0123456, 0.7), (-0.3141, -2.5), (1.3, 3.0)])
def test_recovers_time_and_phase(t, phi):
    a = chirp()
    assert abs(om.mismatch(a, shifted(a, t, phi), FREQUENCIES, PSD)) < 1e-12
    if t != 0.0:
        assert om.mismatch(a, shifted(a, t, phi), FREQUENCIES, PSD, time=False) > 0.1


def test_different_waveforms():
    a, b = chirp(), chirp(1e-3)
    m = om.mismatch(a, b, FREQUENCIES, PSD)
    assert 1e-6 < m < 1
    np.testing.assert_allclose(m, om.mismatch(b, a, FREQUENCIES, PSD), rtol=1e-8)
    assert m < om.mismatch(a, b, FREQUENCIES, PSD, time=False)


def test_rows():
    """Rows along the leading axis: each row its own match."""
    a = np.stack([chirp(), chirp(1e-3), chirp(-2e-3)])
    b = chirp(5e-4)
    rows = om.match(a, b, FREQUENCIES, PSD)
    for i in range(3):
        np.testing.assert_allclose(rows[i], om.match(a[i], b, FREQUENCIES, PSD), rtol=1e-13)


def test_polarizations_recovered():
    """Any combination of the polarizations, delayed: a match of 1
    (reference ``tests/test_match.py:97-104``)."""
    hplus = chirp()
    hcross = -1j * chirp(2e-3) * 0.8
    for fp, fx, t in ((0.3, -0.9, 0.01), (1.0, 0.0, -0.2), (0.0, 0.5, 0.0)):
        signal = shifted(fp * hplus + fx * hcross, t, 0.0)
        assert abs(om.polarization_mismatch(signal, hplus, hcross, FREQUENCIES, PSD)) < 1e-12


def test_polarization_projection():
    """A signal with a part orthogonal to both polarizations: the norm of
    its projection over its norm (reference ``tests/test_match.py:107-121``)."""
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
    got = om.polarization_match(signal, hplus, hcross, FREQUENCIES, PSD, time=False)
    np.testing.assert_allclose(got, expected, rtol=1e-12)


def test_parallel_polarizations():
    """``hcross`` zero: the match with ``hplus`` alone, not NaN (reference
    ``tests/test_match.py:124-129``)."""
    a = chirp()
    got = om.polarization_match(shifted(a, 0.05, 0.0), a, 0 * a, FREQUENCIES, PSD)
    np.testing.assert_allclose(got, 1, atol=1e-12)
