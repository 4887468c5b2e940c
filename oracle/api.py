"""The oracle's entry points: polarizations of a batch, the per-binary loss
of the fused likelihood, central finite differences of it, and the
accuracy measures. Oracle only (test infrastructure)."""

from __future__ import annotations

import numpy as np

from . import phenomd, taylorf2, xas

MODELS = {"IMRPhenomXAS": xas, "IMRPhenomD": phenomd, "TaylorF2": taylorf2}


def table(approximant, params, f_min, amp_scale=1e21, reference_mf=None):
    """The per-binary tables (dict of arrays) of ``params`` ``(B, 8)``."""
    return MODELS[approximant].table(params, f_min, amp_scale, reference_mf)


def polarizations(approximant, params, frequencies, t_c=None, amp_scale=1e21, reference_mf=None):
    """``(hplus, hcross)`` complex128 ``(B, N)`` of the binaries ``params``
    ``(B, 8)`` at ``frequencies`` (``(N,)`` shared, or ``(B, N)``), as
    ``SimInspiralChooseFDWaveformSequence`` with the first frequency as
    ``f_min``; ``t_c`` ``(B,)`` (s) multiplies both by ``exp(-2 pi i f
    t_c)`` (the extension of the B200 path; none in the reference)."""
    params = np.atleast_2d(np.asarray(params, dtype=np.float64))
    f = np.asarray(frequencies, dtype=np.float64)
    f_min = f[..., 0]
    module = MODELS[approximant]
    tab = module.table(params, f_min, amp_scale, reference_mf)
    hp, hc = module.evaluate(tab, f)
    if t_c is not None:
        shift = np.exp(-2j * np.pi * f * np.asarray(t_c, dtype=np.float64)[:, None])
        hp, hc = hp * shift, hc * shift
    return hp, hc


def batch_loss(approximant, params, frequencies, data, weights, t_c=None, antenna=(1.0, 0.0), scale=1.0,
               amp_scale=1e21):
    """``scale * sum_f w(f) |F+ h+ + Fx hx - d(f)|^2`` per binary (float64),
    the fused likelihood's loss; ``data`` ``(N,)`` shared or ``(B, N)``."""
    hp, hc = polarizations(approximant, params, frequencies, t_c=t_c, amp_scale=amp_scale)
    h = antenna[0] * hp + antenna[1] * hc
    r = h - np.asarray(data)
    return scale * np.sum(np.asarray(weights) * (r.real ** 2 + r.imag ** 2), axis=-1)


def loss_gradient_fd(approximant, params, frequencies, data, weights, t_c=None, antenna=(1.0, 0.0), scale=1.0,
                     amp_scale=1e21, rel_step=1e-6):
    """Central finite differences of :func:`batch_loss` with respect to
    ``mass_1, mass_2, chi_1, chi_2, luminosity_distance, inclination,
    phi_ref, t_c`` (step ``rel_step * max(|x|, 1)``, as the reference's
    gradient tests): ``(B, 8)``."""
    params = np.atleast_2d(np.asarray(params, dtype=np.float64))
    b = params.shape[0]
    t_c = np.zeros(b) if t_c is None else np.asarray(t_c, dtype=np.float64)
    grad = np.zeros((b, 8))
    for k in range(8):
        x = t_c if k == 7 else params[:, k]
        step = rel_step * np.maximum(np.abs(x), 1.0)
        values = []
        for sign in (1.0, -1.0):
            p, tc = params.copy(), t_c.copy()
            if k == 7:
                tc = tc + sign * step
            else:
                p[:, k] = p[:, k] + sign * step
            values.append(batch_loss(approximant, p, frequencies, data, weights, tc, antenna, scale, amp_scale))
        grad[:, k] = (values[0] - values[1]) / (2.0 * step)
    return grad


def psd(frequencies):
    """``S(f) = (f / 20)^-4 + 2 + (f / 200)^2``, the analytic noise curve of
    the weighted mismatch and the likelihood workloads."""
    f = np.asarray(frequencies, dtype=np.float64)
    return (f / 20.0) ** -4 + 2.0 + (f / 200.0) ** 2


def mismatch(a, b, weights=None):
    """``1 - <a, b> / sqrt(<a, a> <b, b>)`` per row, ``<a, b> = Re sum w
    conj(a) b`` (the reference's definition, ``report/common.py:125-132``,
    without maximisation over time or phase)."""
    a = np.asarray(a, dtype=np.complex128)
    b = np.asarray(b, dtype=np.complex128)
    w = 1.0 if weights is None else np.asarray(weights, dtype=np.float64)
    ab = np.sum(w * (np.conj(a) * b).real, axis=-1)
    aa = np.sum(w * np.abs(a) ** 2, axis=-1)
    bb = np.sum(w * np.abs(b) ** 2, axis=-1)
    with np.errstate(invalid="ignore", divide="ignore"):
        out = 1.0 - ab / np.sqrt(aa * bb)
    return np.where((aa == 0) & (bb == 0), 0.0, out)


def phase_error(a, b, rel_floor=1e-3):
    """The largest phase difference (rad, wrapped to ``[-pi, pi]``) between
    ``a`` and ``b`` where ``|b|`` exceeds ``rel_floor`` of its row's peak
    (below it the phase of a vanishing amplitude is noise), per row."""
    a = np.asarray(a, dtype=np.complex128)
    b = np.asarray(b, dtype=np.complex128)
    mask = np.abs(b) > rel_floor * np.max(np.abs(b), axis=-1, keepdims=True)
    d = np.angle(a * np.conj(b))
    return np.max(np.where(mask, np.abs(d), 0.0), axis=-1)


def amplitude_error(a, b, rel_floor=1e-3):
    """The largest relative amplitude difference where ``|b|`` exceeds
    ``rel_floor`` of its row's peak, per row."""
    a = np.asarray(a, dtype=np.complex128)
    b = np.asarray(b, dtype=np.complex128)
    mag = np.abs(b)
    mask = mag > rel_floor * np.max(mag, axis=-1, keepdims=True)
    with np.errstate(invalid="ignore", divide="ignore"):
        r = np.abs(np.abs(a) - mag) / mag
    return np.max(np.where(mask, r, 0.0), axis=-1)
