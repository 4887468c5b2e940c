"""TaylorF2 in float64 NumPy, vectorised over binaries: the post-Newtonian
phasing (``models/taylorf2/pn.py:27-91``), the table
(``models/taylorf2/core.py:107-165``) and the waveform at the frequencies
(``core.py:168-212``). Oracle only (test infrastructure).

LAL's TaylorF2 with its defaults (3.5PN phase with every spin term, the
leading-order amplitude, no tidal terms): ``h = A f^(-7/6) exp(i phi)``,
``phi = sum_k (v_k + l_k log v) v^(k - 5)`` in ``v = (pi M f)^(1/3)``
written in powers of ``f`` in Hz. ``f_ref = 0`` is the reference at
coalescence (no reference phase).
"""

from __future__ import annotations

import numpy as np

from . import xas
from .fit_tables import CONSTANTS as K

PI = K["PI"]
MTSUN_SI = K["MTSUN_SI"]
EGAMMA = K["EGAMMA"]
LN_4 = float(np.log(4.0))
LOG_6 = -6848.0 / 21.0
# the amplitude's coefficient (core.py:86-87): A = K_AMP (m1 m2)^(1/2)
# M^(-1/6) / D, masses in solar masses and D in Mpc
K_AMP = -4.0 * K["MRSUN_SI"] * MTSUN_SI / K["MPC_SI"] * float(np.sqrt(PI / 12.0) * np.sqrt(5.0 / 32.0)) \
    * float(PI * MTSUN_SI) ** (-7.0 / 6.0)
# the phase basis but for f^(-5/3) (core.py:54): (power, power of log f)
BASIS = ((-1, 0), (-2 / 3, 0), (-1 / 3, 0), (0, 1), (0, 0), (1 / 3, 0), (1 / 3, 1), (2 / 3, 0))
INDEX = {key: i for i, key in enumerate(BASIS)}
CONST = INDEX[(0, 0)]
# their positions in the basis of models/xas/core.py:49-52
XAS_INDEX = (1, 2, 3, 4, 5, 6, 7, 8)


def spin_spin_3pn(eta, x1, x2, chi1, chi2):
    """``pn.py:48-56``."""
    phase = (32675.0 / 112.0 + 5575.0 / 18.0 * eta) * eta * chi1 * chi2
    for x, chi in ((x1, chi1), (x2, chi2)):
        phase = phase + ((47035.0 / 84.0 + 2935.0 / 6.0 * x - 120.0 * x * x)
                         + (-410825.0 / 672.0 - 1085.0 / 12.0 * x + 1255.0 / 36.0 * x * x)) * x * x * chi * chi
    return phase


def phasing(x1, x2, chi1, chi2):
    """The coefficients ``v_0 .. v_7`` of ``v^(k - 5)`` and ``l_5``, ``l_6``
    of ``v^(k - 5) log v``, with the factor ``3 / (128 eta)``
    (``pn.py:27-91``)."""
    eta = x1 * x2
    scale = 3.0 / (128.0 * eta)
    v3 = -16.0 * PI + sum(x * (25.0 + 38.0 / 3.0 * x) * chi for x, chi in ((x1, chi1), (x2, chi2)))
    v4 = 15293365.0 / 508032.0 + 27145.0 / 504.0 * eta + 3085.0 / 72.0 * eta * eta
    v4 = v4 - 395.0 / 4.0 * eta * chi1 * chi2
    for x, chi in ((x1, chi1), (x2, chi2)):
        v4 = v4 - (50.0 + 5.0 / 8.0) * x * x * chi * chi
    v5 = 5.0 / 9.0 * (7729.0 / 84.0 - 13.0 * eta) * PI
    for x, chi in ((x1, chi1), (x2, chi2)):
        v5 = v5 - chi * x * (13915.0 / 84.0 - x * (1.0 - x) * 10.0 / 3.0
                             + x * (12760.0 / 81.0 + x * (1.0 - x) * 170.0 / 9.0))
    v6 = 11583231236531.0 / 4694215680.0 - 640.0 / 3.0 * PI ** 2 - 6848.0 / 21.0 * EGAMMA
    v6 = v6 + eta * (-15737765635.0 / 3048192.0 + 2255.0 / 12.0 * PI ** 2)
    v6 = v6 + eta * eta * 76055.0 / 1728.0 - eta * eta * eta * 127825.0 / 1296.0
    v6 = v6 + LOG_6 * LN_4 + spin_spin_3pn(eta, x1, x2, chi1, chi2)
    for x, chi in ((x1, chi1), (x2, chi2)):
        v6 = v6 + PI * x * (1490.0 / 3.0 + x * 260.0) * chi
    v7 = PI * (77096675.0 / 254016.0 + 378515.0 / 1512.0 * eta - 74045.0 / 756.0 * eta * eta)
    for x, chi in ((x1, chi1), (x2, chi2)):
        v7 = v7 + chi * x * (-170978035.0 / 48384.0 + eta * 2876425.0 / 672.0 + eta * eta * 4735.0 / 144.0
                             + x * (-7189233785.0 / 1524096.0 + eta * 458555.0 / 3024.0
                                    - eta * eta * 5345.0 / 72.0))
    v = [1.0, 0.0, 55.0 * eta / 9.0 + 3715.0 / 756.0, v3, v4, v5, v6, v7]
    return [scale * c for c in v], {5: scale * 3.0 * v5, 6: scale * LOG_6}


def phase_mf(v, logs, mf, start=0):
    """``-sum_{k >= start} (v_k + l_k log u) u^(k - 5)`` at ``M f = mf``,
    ``u = (pi mf)^(1/3)`` (``core.py:95-104``)."""
    u = np.cbrt(PI * mf)
    log_u = np.log(u)
    total = 0.0
    for k in range(start, len(v)):
        if k == 1:
            continue
        total = total - (v[k] + logs[k] * log_u if k in logs else v[k]) * u ** (k - 5)
    return total


frequency_powers = xas.frequency_powers


def phase_rest(tab, fp):
    """The phase but for the leading term and the anchor (``core.py:174-181``)."""
    basis = xas.phase_basis(fp)
    col = lambda v: np.asarray(v)[..., None]  # noqa: E731
    total = col(tab["phase"][..., CONST])
    for i, k in enumerate(XAS_INDEX):
        if i != CONST:
            total = total + col(tab["phase"][..., i]) * basis[k]
    return total


def table(params, f_min=None, amp_scale=1e21, reference_mf=None):
    """The table of each binary (``core.py:107-165``); ``f_min`` is unused
    (kept for the common signature of the oracle's models)."""
    params = np.atleast_2d(np.asarray(params, dtype=np.float64))
    m1, m2, chi1, chi2, distance, inclination, phi_ref, f_ref = params.T
    total = m1 + m2
    v, logs = phasing(m1 / total, m2 / total, chi1, chi2)
    m_sec = total * MTSUN_SI
    log_pim = np.log(PI * m_sec)
    u = np.cbrt(PI * m_sec)
    u_inv = 1.0 / u
    u_pow = {-3: u_inv * u_inv * u_inv, -2: u_inv * u_inv, -1: u_inv, 0: 1.0, 1: u, 2: u * u}
    rows = [np.zeros(m1.shape)] * len(BASIS)
    for k in range(2, 8):
        a = (k - 5) / 3.0
        s = u_pow[k - 5]
        coefficient = v[k]
        if k in logs:
            coefficient = coefficient + logs[k] * log_pim / 3.0
            rows[INDEX[(a, 1)]] = -logs[k] / 3.0 * s
        rows[INDEX[(a, 0)]] = -coefficient * s
    rows = np.stack([np.broadcast_to(np.asarray(r, dtype=np.float64), m1.shape) for r in rows], -1)
    if reference_mf is None:
        invalid = np.zeros(m1.shape, dtype=bool)
        referenced = f_ref > 0.0
        f_ref_safe = np.where(referenced, f_ref, 1.0)
        rest = phase_rest(dict(phase=rows), frequency_powers(f_ref_safe[..., None]))[..., 0]
        f_ref64 = f_ref_safe
    else:
        invalid = f_ref != 0.0
        referenced = np.ones(m1.shape, dtype=bool)
        rest = phase_mf(v, logs, reference_mf, start=2)
        f_ref64 = reference_mf / (MTSUN_SI * (m1 + m2))
    rows[..., CONST] = rows[..., CONST] + (2.0 * phi_ref + PI / 4.0 - np.where(referenced, rest, 0.0))
    t0 = K["XAS_K0"] * np.cbrt(m1 + m2) / (m1 * m2)
    anchor = np.where(referenced, t0 * np.exp(-5.0 / 3.0 * np.log(f_ref64)), 0.0)
    amp = K_AMP * amp_scale * np.sqrt(m1 * m2) * np.exp(-1.0 / 6.0 * np.log(total)) / distance
    cos_i = np.cos(inclination)
    return dict(phase=rows, t0=t0, anchor=anchor, amp=amp, kp=np.where(invalid, np.nan, 0.5 * (1.0 + cos_i * cos_i)),
                kc=np.where(invalid, np.nan, -cos_i), error=invalid)


def reduce(phi):
    return phi - np.round(phi / (2.0 * np.pi)) * (2.0 * np.pi)


def amplitude_phase(tab, f):
    """The amplitude and the unreduced phase (``core.py:184-201``)."""
    fp = frequency_powers(f)
    col = lambda v: np.asarray(v)[..., None]  # noqa: E731
    phi = col(tab["t0"]) * fp[5] + phase_rest(tab, fp) - col(tab["anchor"])
    return col(tab["amp"]) * fp[4], phi


def evaluate(tab, f):
    """``(hplus, hcross)`` (``core.py:204-212``)."""
    amp, phi = amplitude_phase(tab, f)
    phi = reduce(phi)
    c, s = np.cos(phi), np.sin(phi)
    ap = np.asarray(tab["kp"])[..., None] * amp
    ac = np.asarray(tab["kc"])[..., None] * amp
    return ap * c + 1j * (ap * s), -ac * s + 1j * (ac * c)


# the order of the reference's flat table (core.py:63-70)
LAYOUT = (("phase", 8), ("big", 2), ("big_lo", 2), ("amp", 1), ("kp", 1), ("kc", 1))


def flat(tab):
    """The table in the reference's flat layout (15 values)."""
    b = np.asarray(tab["t0"]).shape
    out = []
    for name, size in LAYOUT:
        if name == "big":
            v = np.stack([tab["t0"], tab["anchor"]], -1)
        elif name == "big_lo":
            v = np.zeros(b + (2,))
        else:
            v = np.asarray(tab[name], dtype=np.float64)
        out.append(np.reshape(np.broadcast_to(v, b + v.shape[len(b):]), b + (size,)))
    return np.concatenate(out, -1)
