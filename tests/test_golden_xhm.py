"""The IMRPhenomXHM golden vectors (``tests/golden/xhm_*.npz``, from the
reference's own code) checked on the CPU for what the reference states of
them, and the host side of the XHM path (no GPU):

* the polarizations are the sum of the modes with their factors
  (``models/xhm/core.py:549-556``), the factors those of the spin-weighted
  spherical harmonics (``models/xhm/reference.py:630-638``);
* the odd modes vanish for equal masses and spins (``core.py:383-389``);
* the amplitude scale is linear (``scaled_strain``);
* IMRPhenomXHM is an approximant of this path; its gradient goes through
  ``ops.xhm_vjp``, not the table-based backward or fused likelihood.
"""

from __future__ import annotations

import math

import numpy as np
import pytest

from conftest import golden

MODES = ((2, 2), (2, 1), (3, 3), (3, 2), (4, 4))
REF_HEAD = 86


def _wigner_d(ell, mp, m, beta):
    f = math.factorial
    ch, sh = math.cos(beta / 2), math.sin(beta / 2)
    pre = math.sqrt(f(ell + mp) * f(ell - mp) * f(ell + m) * f(ell - m))
    total = 0.0
    for k in range(max(0, m - mp), min(ell + m, ell - mp) + 1):
        c = (-1) ** (k - m + mp) * pre / (f(ell + m - k) * f(k) * f(ell - k - mp) * f(k - m + mp))
        total += c * ch ** (2 * ell - 2 * k + m - mp) * sh ** (2 * k - m + mp)
    return total


def _swsh(theta, ell, m):
    return math.sqrt((2 * ell + 1) / (4 * math.pi)) * _wigner_d(ell, m, 2, theta) * np.exp(1j * m * math.pi / 2)


@pytest.mark.parametrize("name", ["cases", "random", "reference_mf", "unscaled"])
def test_polarizations_are_the_sum_of_the_modes(name):
    data = golden(f"xhm_{name}")
    for b, p in enumerate(data["params"]):
        factors = data["tables"][b, REF_HEAD:REF_HEAD + 20].reshape(5, 4)
        hp = sum((factors[k, 0] + 1j * factors[k, 1]) * data["modes"][b, k] for k in range(5))
        hc = sum((factors[k, 2] + 1j * factors[k, 3]) * data["modes"][b, k] for k in range(5))
        scale = np.max(np.abs(data["hplus"][b]))
        assert np.max(np.abs(hp - data["hplus"][b])) < 1e-12 * scale
        assert np.max(np.abs(hc - data["hcross"][b])) < 1e-12 * scale
        # the factors: (Y_{l,-m} + (-1)^l conj(Y_{l,m})) / 2 and i (...) / 2
        for k, (ell, emm) in enumerate(MODES):
            sign = -1.0 if ell % 2 else 1.0
            ym, ys = _swsh(p[5], ell, -emm), np.conj(_swsh(p[5], ell, emm))
            fp, fc = 0.5 * (ym + sign * ys), 0.5j * (ym - sign * ys)
            np.testing.assert_allclose([fp.real, fp.imag, fc.real, fc.imag], factors[k], atol=1e-14)


def test_odd_modes_vanish_for_equal_binaries():
    data = golden("xhm_cases")
    equal = [b for b, p in enumerate(data["params"]) if p[0] == p[1] and p[2] == p[3]]
    assert equal
    for b in equal:
        assert np.all(data["modes"][b, 1] == 0) and np.all(data["modes"][b, 2] == 0)
        assert np.all(data["tables"][b, REF_HEAD + 22:REF_HEAD + 22 + 224] == 0)


def test_strain_scale_is_linear():
    scaled, unscaled = golden("xhm_cases"), golden("xhm_unscaled")
    for b in range(len(unscaled["params"])):
        for k in range(5):
            a, r = unscaled["modes"][b, k] * 1e21, scaled["modes"][b, k]
            assert np.max(np.abs(a - r)) <= 1e-12 * np.max(np.abs(r)), (b, k)


def test_approximant_is_forward_only():
    from waveformx_b200 import _lib, ops
    from waveformx_b200.exceptions import UnsupportedError

    assert ops.model_code("IMRPhenomXHM") == _lib.XHM == 3
    assert ops.XHM_MODES == MODES
    with pytest.raises(UnsupportedError):
        ops._differentiable(_lib.XHM)
    ops._differentiable(_lib.XAS)
