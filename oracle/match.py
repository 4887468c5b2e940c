"""Matches between waveforms in float64 NumPy: the noise-weighted inner
product, the match maximised over a time shift and a constant phase, and
the polarization match (``src/waveformx/match.py:71-187``), vectorised over
rows. Oracle only (test
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


def _polarization_terms(signal, hplus, hcross, f, psd):
    """The norms, the overlap ``I`` of the normalised polarizations and the
    series of ``polarization_match`` (match.py:162-172)."""
    ss = inner_product(signal, signal, f, psd)
    pp = inner_product(hplus, hplus, f, psd)
    xx = inner_product(hcross, hcross, f, psd)
    px = inner_product(hplus, hcross, f, psd)
    with np.errstate(invalid="ignore", divide="ignore"):
        i = px / np.sqrt(pp * xx)
    degenerate = ~(1 - i ** 2 > 1e-10)
    i = np.where(degenerate, 0.0, i)
    xx = np.where(degenerate, 1.0, xx)
    cp = overlap(signal, hplus, f, psd)
    cx = overlap(signal, hcross, f, psd)
    return ss, pp, xx, i, degenerate, cp, cx


def _square(rp, rx, pp, xx, i, degenerate):
    rp, rx = rp / np.sqrt(pp), np.where(degenerate, 0.0, rx / np.sqrt(xx))
    return (rp ** 2 + rx ** 2 - 2 * rp * rx * i) / (1 - i ** 2)


def polarization_match(signal, hplus, hcross, frequencies, psd, *, time=True, pad=4):
    """The match of ``signal`` with ``F+ hplus + Fx hcross`` maximised over
    time and over ``F+`` and ``Fx`` (match.py:150-187): the norm of the
    projection of the signal onto the real span of the polarizations over
    its norm; with parallel polarizations the match with ``hplus`` alone.
    Newton steps on ``Q(t) = square(Re zp(t), Re zx(t))`` with its
    closed-form derivatives."""
    f, _ = _grid(frequencies)
    ss, pp, xx, i, degenerate, cp, cx = _polarization_terms(signal, hplus, hcross, f, psd)

    def value(t):
        return _square(z_derivatives(cp, f, t)[0].real, z_derivatives(cx, f, t)[0].real, pp, xx, i, degenerate)

    if time:
        times, sp = series(cp, f, pad)
        _, sx = series(np.where(np.asarray(degenerate)[..., None], 0.0, cx), f, pad)
        col = lambda v: np.asarray(v)[..., None]  # noqa: E731
        grid = _square(sp.real, sx.real, col(pp), col(xx), col(i), col(degenerate))
        t = times[np.argmax(grid, axis=-1)]
        period = times[-1] + times[1]
        t = np.where(t > period / 2, t - period, t)
        for _ in range(NEWTON_STEPS):
            zp = z_derivatives(cp, f, t)
            zx = z_derivatives(cx, f, t)
            sp_, sx_ = np.sqrt(pp), np.sqrt(xx)
            a, a1, a2 = (z.real / sp_ for z in zp)
            b, b1, b2 = (np.where(degenerate, 0.0, z.real / sx_) for z in zx)
            q = 1 - i ** 2
            g = (2 * a * a1 + 2 * b * b1 - 2 * i * (a1 * b + a * b1)) / q
            h = (2 * a1 * a1 + 2 * a * a2 + 2 * b1 * b1 + 2 * b * b2 - 2 * i * (a2 * b + 2 * a1 * b1 + a * b2)) / q
            new = t - np.where(h < 0, g / np.where(h < 0, h, 1.0), 0.0)
            t = np.where(value(new) >= value(t), new, t)
    else:
        t = np.zeros(np.shape(ss))
    return np.sqrt(value(t) / ss)


def polarization_mismatch(signal, hplus, hcross, frequencies, psd, **keywords):
    """``1 - polarization_match(...)``."""
    return 1 - polarization_match(signal, hplus, hcross, frequencies, psd, **keywords)
