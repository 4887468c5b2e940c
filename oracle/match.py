"""Matches between waveforms in float64 NumPy: the noise-weighted inner
product and the match maximised over a time shift and a constant phase
(``src/waveformx/match.py:71-147``), vectorised over rows. Oracle only (test
infrastructure).

The reference refines the best time of its FFT grid by Newton steps whose
first and second derivatives come from ``jax.grad``; here they are the
closed forms of the same objective: with ``z(t) = sum_k c_k e^(2 pi i f_k
t)``, ``|z|^2`` has the derivatives ``2 Re(conj(z) z')`` and ``2 (|z'|^2 +
Re(conj(z) z''))``, and ``Re z`` has ``Re z'`` and ``Re z''``.
"""

from __future__ import annotations

import numpy as np

#: Newton steps that refine the best time of the FFT grid (match.py:70).
NEWTON_STEPS = 3


def _grid(frequencies):
    f = np.asarray(frequencies, dtype=np.float64)
    return f, f[1] - f[0]


def inner_product(a, b, frequencies, psd):
    """``4 delta_f Re sum a conj(b) / S`` over the last axis (match.py:78-81)."""
    _, delta_f = _grid(frequencies)
    return 4 * delta_f * np.sum((np.asarray(a) * np.conj(b)).real / np.asarray(psd), axis=-1)


def overlap(a, b, frequencies, psd):
    """``c = 4 delta_f a conj(b) / S``, the summand of ``z(t)`` (match.py:84-88)."""
    _, delta_f = _grid(frequencies)
    return 4 * delta_f * np.asarray(a) * np.conj(b) / np.asarray(psd)


def z_derivatives(c, f, t):
    """``(z, z', z'')`` at the times ``t`` (one per row)."""
    t = np.asarray(t, dtype=np.float64)[..., None]
    w = np.exp(2j * np.pi * f * t)
    k = 2j * np.pi * f
    return np.sum(c * w, -1), np.sum(c * k * w, -1), np.sum(c * k * k * w, -1)


def series(c, frequencies, pad):
    """``z`` on the times ``j / (n delta_f)`` of one period, ``n = pad``
    times the power of two above the number of frequencies (match.py:91-101)."""
    f, delta_f = _grid(frequencies)
    k = c.shape[-1]
    n = pad * (1 << (k - 1).bit_length())
    times = np.arange(n) / (n * delta_f)
    z = n * np.fft.ifft(c, n) * np.exp(2j * np.pi * f[0] * times)
    return times, z


def _objective(z, phase):
    return np.abs(z) ** 2 if phase else z.real


def refine(c, f, t, phase):
    """Newton steps towards the maximum of the objective from ``t``, each
    kept only if it does not lower the objective (match.py:104-115)."""
    t = np.asarray(t, dtype=np.float64).copy()
    for _ in range(NEWTON_STEPS):
        z0, z1, z2 = z_derivatives(c, f, t)
        if phase:
            g = 2 * (np.conj(z0) * z1).real
            h = 2 * (np.abs(z1) ** 2 + (np.conj(z0) * z2).real)
        else:
            g, h = z1.real, z2.real
        step = np.where(h < 0, g / np.where(h < 0, h, 1.0), 0.0)
        new = t - step
        keep = _objective(z_derivatives(c, f, new)[0], phase) >= _objective(z0, phase)
        t = np.where(keep, new, t)
    return t


def best_time(c, frequencies, phase, pad=4):
    """The grid's best time, wrapped to ``(-period / 2, period / 2]`` and
    refined (match.py:118-126)."""
    f, _ = _grid(frequencies)
    times, z = series(c, f, pad)
    grid = np.abs(z) if phase else z.real
    t = times[np.argmax(grid, axis=-1)]
    period = times[-1] + times[1]
    t = np.where(t > period / 2, t - period, t)
    return refine(c, f, t, phase)


def match(a, b, frequencies, psd, *, time=True, phase=True, pad=4):
    """``<a, b> / sqrt(<a, a> <b, b>)`` maximised over a time shift and a
    constant phase (match.py:129-147); rows along the leading axes."""
    f, _ = _grid(frequencies)
    norm = np.sqrt(inner_product(a, a, f, psd) * inner_product(b, b, f, psd))
    c = overlap(a, b, f, psd)
    t = best_time(c, f, phase, pad) if time else np.zeros(c.shape[:-1])
    z = z_derivatives(c, f, t)[0]
    best = np.abs(z) if phase else z.real
    return best / norm


def mismatch(a, b, frequencies, psd, **keywords):
    """``1 - match(a, b, ...)``."""
    return 1 - match(a, b, frequencies, psd, **keywords)
