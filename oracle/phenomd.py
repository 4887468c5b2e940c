"""IMRPhenomD in float64 NumPy, vectorised over binaries: the coefficients
(``models/phenomd/core.py:154-274``), the table (``core.py:280-378``) and
the waveform at the frequencies (``core.py:398-485``). Oracle only (test
infrastructure)."""

from __future__ import annotations

import numpy as np

from .fit_tables import CONSTANTS as K
from .fit_tables import PHD_FDAMP, PHD_FRING
from .fits import evaluate as fit

PI = K["PI"]
MTSUN_SI = K["MTSUN_SI"]
F_PHASE_INS = 0.018
F_AMP_INS = 0.014
# the basis of the phase but for f^(-5/3) (core.py:51-56)
BASIS = ((-1, 0), (-2 / 3, 0), (-1 / 3, 0), (0, 1), (0, 0), (1 / 3, 0), (1 / 3, 1), (2 / 3, 0), (1, 0), (4 / 3, 0),
         (5 / 3, 0), (2, 0), (-3, 0), (3 / 4, 0))
INDEX = {key: i for i, key in enumerate(BASIS)}
CONST = INDEX[(0, 0)]
REGION_TERMS = (
    tuple(i for i, key in enumerate(BASIS) if key not in ((0, 0), (-3, 0), (3 / 4, 0))),
    (INDEX[(1, 0)], INDEX[(-3, 0)], INDEX[(0, 1)]),
    (INDEX[(1, 0)], INDEX[(-1, 0)], INDEX[(3 / 4, 0)]),
)


def _chebyshev(coefficients, t):
    b1 = b2 = 0.0
    for c in reversed(coefficients[1:]):
        b1, b2 = 2.0 * t * b1 - b2 + c, b1
    return t * b1 - b2 + coefficients[0]


def coefficients(x1, x2, chi1, chi2):
    """The coefficients in ``Mf`` (``core.py:154-274``)."""
    eta = x1 * x2
    delta = x1 - x2
    chi_s, chi_a = 0.5 * (chi1 + chi2), 0.5 * (chi1 - chi2)
    xi = chi_s * (1.0 - eta * 76.0 / 113.0) + delta * chi_a - 1.0
    names = ("rho1", "rho2", "rho3", "gamma1", "gamma2", "gamma3", "collocation", "alpha1", "alpha2", "alpha3",
             "alpha4", "alpha5", "beta1", "beta2", "beta3", "sigma1", "sigma2", "sigma3", "sigma4")
    ph = {n: fit("PHD_" + n.upper(), eta, xi) for n in names}
    y1, y2 = 0.5 * (1.0 + delta), 0.5 * (1.0 - delta)
    af = fit("PHD_FINAL_SPIN", eta, y1 * y1 * chi1 + y2 * y2 * chi2)
    t = 2.0 * np.cbrt(0.5 * (1.0 - af)) - 1.0
    ring, damp = _chebyshev(PHD_FRING, t), _chebyshev(PHD_FDAMP, t)
    s_e = (y1 * y1 * chi1 + y2 * y2 * chi2) / (y1 * y1 + y2 * y2)
    remnant = 1.0 - fit("PHD_RADIATED_ENERGY", eta, s_e)
    f_ring, f_damp = ring / remnant, damp / remnant
    # TaylorF2 phasing (models/taylorf2/pn.py:81-91) but for its 3PN
    # spin-spin term, plus the pseudo-PN terms
    scale = 3.0 / (128.0 * eta)
    ppn = {k: fit(f"PHD_PN_PHASE_{k}", eta, x1, x2, chi1, chi2) for k in (3, 4, 5, 6, 7)}
    v = [scale * 1.0, 0.0 * eta, scale * (55.0 * eta / 9.0 + 3715.0 / 756.0), scale * ppn[3], scale * ppn[4],
         scale * ppn[5], scale * ppn[6], scale * ppn[7], 0.0, 0.0, 0.0, 0.0]
    logs = {5: scale * 3.0 * ppn[5], 6: scale * (-6848.0 / 21.0)}
    v[5] = v[5] - PI / 4.0
    v[6] = v[6] - fit("PHD_PN_SPIN_SPIN_3", eta, x1, x2, chi1, chi2) * v[0]
    v[8] = ph["sigma1"] / eta / PI
    v[9] = ph["sigma2"] * 0.75 / eta / K["PI_POW_4_3"]
    v[10] = ph["sigma3"] * 0.6 / eta / K["PI_POW_5_3"]
    v[11] = ph["sigma4"] * 0.5 / eta / K["PI_POW_2"]
    beta = [ph["beta1"], ph["beta2"], ph["beta3"]]
    alpha = [ph[f"alpha{i}"] for i in range(1, 6)]

    def ins(mf):
        u = np.cbrt(PI * mf)
        log_u = np.log(u)
        total = sum(c * u ** (k - 5) for k, c in enumerate(v) if k != 1)
        return total + sum(c * u ** (k - 5) * log_u for k, c in logs.items())

    def dins(mf):
        u = np.cbrt(PI * mf)
        log_u = np.log(u)
        total = sum((k - 5) / 3.0 * c * u ** (k - 5) for k, c in enumerate(v) if k != 1)
        total = total + sum(c * u ** (k - 5) * ((k - 5) / 3.0 * log_u + 1.0 / 3.0) for k, c in logs.items())
        return total / mf

    def inter(mf):
        return (beta[0] * mf - beta[2] / 3.0 / mf ** 3 + beta[1] * np.log(mf)) / eta

    def dinter(mf):
        return (beta[0] + beta[2] / mf ** 4 + beta[1] / mf) / eta

    def mrd(mf):
        return (alpha[0] * mf - alpha[1] / mf + 4.0 / 3.0 * alpha[2] * mf ** 0.75
                + alpha[3] * np.arctan((mf - alpha[4] * f_ring) / f_damp)) / eta

    def dmrd(mf):
        y = (mf - alpha[4] * f_ring) / f_damp
        return (alpha[0] + alpha[1] / mf ** 2 + alpha[2] / mf ** 0.25 + alpha[3] / (f_damp * (1.0 + y * y))) / eta

    f1, f2 = F_PHASE_INS, 0.5 * f_ring
    c2_int = dins(f1) - dinter(f1)
    c1_int = ins(f1) - inter(f1) - c2_int * f1
    joined = inter(f2) + c1_int + c2_int * f2
    c2_mrd = c2_int + dinter(f2) - dmrd(f2)
    c1_mrd = joined - mrd(f2) - c2_mrd * f2
    amp_pn = [1.0 + 0.0 * eta, 0.0 * eta] + [fit(f"PHD_AMP_PN_{k}", eta, delta, chi1, chi2) for k in (2, 3, 4, 5, 6)]
    rho = amp_pn + [ph["rho1"] / K["PI_POW_7_3"], ph["rho2"] / K["PI_POW_8_3"], ph["rho3"] / K["PI_POW_3"]]
    g1, g2, g3 = ph["gamma1"], ph["gamma2"], ph["gamma3"]
    below = g2 <= 1.0
    root = np.sqrt(np.where(below, 1.0 - g2 * g2, 1.0))
    f_peak = np.abs(np.where(below, f_ring + f_damp * (root - 1.0) * g3 / g2, f_ring - f_damp * g3 / g2))
    t0 = dmrd(f_peak)

    def amp_ins(mf):
        u = np.cbrt(PI * mf)
        return sum(c * u ** k for k, c in enumerate(rho) if k != 1)

    def damp_ins(mf):
        u = np.cbrt(PI * mf)
        return sum(k / 3.0 * c * u ** k for k, c in enumerate(rho) if k > 1) / mf

    sigma = f_damp * g3

    def amp_mrd(mf):
        d = mf - f_ring
        return g1 * sigma / (d * d + sigma * sigma) * np.exp(-g2 * d / sigma)

    def damp_mrd(mf):
        d = mf - f_ring
        s2 = d * d + sigma * sigma
        return (-2.0 * d * sigma * g1 / s2 - g2 * g1) / (np.exp(g2 * d / sigma) * s2)

    # the intermediate amplitude sum_j delta_j y^j, y = Mf / f_peak
    y1 = F_AMP_INS / f_peak
    y2 = 0.5 * (1.0 + y1)
    one, zero = np.ones_like(y1), np.zeros_like(y1)
    matrix = np.stack([np.stack([one, y1, y1 ** 2, y1 ** 3, y1 ** 4], -1),
                       np.stack([one, y2, y2 ** 2, y2 ** 3, y2 ** 4], -1),
                       np.stack([one, one, one, one, one], -1),
                       np.stack([zero, one, 2.0 * y1, 3.0 * y1 ** 2, 4.0 * y1 ** 3], -1),
                       np.stack([zero, one, 2.0 * one, 3.0 * one, 4.0 * one], -1)], -2)
    values = np.stack([amp_ins(F_AMP_INS) * one, ph["collocation"], amp_mrd(f_peak), damp_ins(F_AMP_INS) * f_peak,
                       damp_mrd(f_peak) * f_peak], -1)
    delta_int = np.linalg.solve(matrix, values[..., None])[..., 0]

    def phase_mf(mf):
        """``-Psi + t0 Mf`` but for the constant, without the leading term."""
        inspiral = ins(mf) - v[0] * np.cbrt(PI * mf) ** -5
        psi = np.where(mf < f1, inspiral, np.where(mf >= f2, mrd(mf) + c1_mrd + c2_mrd * mf,
                                                   inter(mf) + c1_int + c2_int * mf))
        return -psi + t0 * mf

    return dict(v=v, l=logs, beta=beta, alpha=alpha, c_int=(c1_int, c2_int), c_mrd=(c1_mrd, c2_mrd), t0=t0,
                rho=rho, delta=delta_int, gamma=(g1, g2, g3), f_ring=f_ring, f_damp=f_damp, f_peak=f_peak,
                final_spin=af, eta=eta, phase=phase_mf)


def frequency_powers(f):
    """``core.py:398-409``."""
    f = np.asarray(f, dtype=np.float64)
    m1 = 1.0 / f
    log_f = np.log(f)
    t = np.exp(log_f / 3.0)
    t = t * (4.0 - t * t * t * m1) / 3.0
    root = np.sqrt(f)
    return f, t, m1, log_f, m1 / np.sqrt(t), root * np.sqrt(root), np.exp(-5.0 / 3.0 * log_f)


def phase_basis(fp):
    f, t, m1, log_f, _, f34, _ = fp
    t2 = t * t
    mt1 = t2 * m1
    return [m1, mt1 * mt1, mt1, log_f, None, t, t * log_f, t2, f, f * t, f * t2, f * f, m1 * m1 * m1, f34]


def phase_rest(tab, fp):
    """``core.py:426-440``."""
    f = fp[0]
    col = lambda v: np.asarray(v)[..., None]  # noqa: E731
    inspiral = f < col(tab["f_phase_ins"])
    mrd = f >= col(tab["f_phase_mrd"])
    basis = phase_basis(fp)
    sums = []
    for r, terms in enumerate(REGION_TERMS):
        total = col(tab["phase"][..., r, CONST])
        for k in terms:
            total = total + col(tab["phase"][..., r, k]) * basis[k]
        sums.append(total)
    sums[2] = sums[2] + col(tab["atan_a"]) * np.arctan(col(tab["atan_w"]) * (f - col(tab["atan_shift"])))
    return np.where(inspiral, sums[0], np.where(mrd, sums[2], sums[1])), inspiral


def table(params, f_min, amp_scale=1e21, reference_mf=None):
    """The table of each binary (``core.py:280-378``, always float64)."""
    params = np.atleast_2d(np.asarray(params, dtype=np.float64))
    m1, m2, chi1, chi2, distance, inclination, phi_ref, f_ref = params.T
    f_min = np.broadcast_to(np.asarray(f_min, dtype=np.float64), m1.shape)
    total = m1 + m2
    c = coefficients(m1 / total, m2 / total, chi1, chi2)
    eta = c["eta"]
    s = total * MTSUN_SI
    log_s = np.log(s)
    rows = np.zeros(m1.shape + (3, len(BASIS)))

    def add(r, a, log, value):
        rows[..., r, INDEX[(a, log)]] += value

    log_pis = np.log(PI * s)
    u = np.cbrt(PI * s)
    u_pow = [np.ones_like(u), u]
    for _ in range(8):
        u_pow.append(u_pow[-1] * u)
    u_inv = 1.0 / u
    u_pow_inv = {1: u_inv, 2: u_inv * u_inv, 3: u_inv * u_inv * u_inv}
    for k, coefficient in enumerate(c["v"]):
        if k < 2:
            continue
        a = (k - 5) / 3.0
        scale = u_pow[k - 5] if k >= 5 else u_pow_inv[5 - k]
        if k in c["l"]:
            coefficient = coefficient + c["l"][k] * log_pis / 3.0
            add(0, a, 1, -c["l"][k] / 3.0 * scale)
        add(0, a, 0, -coefficient * scale)
    b1, b2, b3 = c["beta"]
    add(1, 1, 0, -(b1 / eta + c["c_int"][1]) * s)
    add(1, -3, 0, b3 / (3.0 * eta) / s ** 3)
    add(1, 0, 1, -b2 / eta)
    add(1, 0, 0, -b2 / eta * log_s - c["c_int"][0])
    a1, a2, a3, a4, a5 = c["alpha"]
    add(2, 1, 0, -(a1 / eta + c["c_mrd"][1]) * s)
    add(2, -1, 0, a2 / eta / s)
    add(2, 3 / 4, 0, -4.0 / 3.0 * a3 / eta * np.sqrt(s) * np.sqrt(np.sqrt(s)))
    add(2, 0, 0, -c["c_mrd"][0])
    for r in range(3):
        add(r, 1, 0, c["t0"] * s)
    f_damp, f_ring = c["f_damp"], c["f_ring"]
    tab = dict(phase=rows, atan_a=-a4 / eta, atan_w=s / f_damp, atan_shift=a5 * f_ring / s,
               f_phase_ins=F_PHASE_INS / s, f_phase_mrd=0.5 * f_ring / s)
    if reference_mf is None:
        invalid = np.zeros(m1.shape, dtype=bool)
        f_ref = np.where(f_ref == 0.0, f_min, f_ref)
        rest, inspiral = phase_rest(tab, frequency_powers(f_ref[..., None]))
        rest, inspiral = rest[..., 0], inspiral[..., 0]
        f_ref64 = f_ref
    else:
        invalid = f_ref != 0.0
        inspiral = np.broadcast_to(reference_mf < F_PHASE_INS, m1.shape)
        rest = c["phase"](reference_mf)
        f_ref64 = reference_mf / (MTSUN_SI * (m1 + m2))
    rows[..., :, CONST] += (2.0 * phi_ref - rest)[..., None]
    t0 = K["XAS_K0"] * np.cbrt(m1 + m2) / (m1 * m2)
    anchor = np.where(inspiral, t0 * np.exp(-5.0 / 3.0 * np.log(f_ref64)), 0.0)
    prefactor = K["PHD_K_AMP"] * amp_scale * np.sqrt(m1 * m2) * np.exp(-np.log(total) / 6.0) / distance
    g1, g2, g3 = c["gamma"]
    width = g3 * f_damp
    error = (c["final_spin"] > 1.0) | invalid
    cos_i = np.cos(inclination)
    tab.update(
        t0=t0, anchor=anchor,
        amp_ins=np.stack([prefactor * x * u_pow[k] for k, x in enumerate(c["rho"])], -1),
        amp_int=prefactor[..., None] * c["delta"], amp_int_s=s / c["f_peak"], amp_rd_n=prefactor * g1 / width,
        amp_rd_gr=g2, amp_rd_s=s / width, amp_rd_shift=f_ring / s, f_amp_ins=F_AMP_INS / s,
        f_amp_mrd=c["f_peak"] / s,
        kp=np.where(error, np.nan, 0.5 * (1.0 + cos_i * cos_i)), kc=np.where(error, np.nan, -cos_i), error=error,
    )
    return tab


def reduce(phi):
    return phi - np.round(phi / (2.0 * np.pi)) * (2.0 * np.pi)


def amplitude_phase(tab, f):
    """The amplitude and the unreduced phase (``core.py:443-473``)."""
    fp = frequency_powers(f)
    f, t, _, _, m76, _, f53 = fp
    col = lambda v: np.asarray(v)[..., None]  # noqa: E731
    rest, inspiral = phase_rest(tab, fp)
    phi = np.where(inspiral, col(tab["t0"]) * f53, 0.0) + rest - col(tab["anchor"])
    poly = col(tab["amp_ins"][..., 9])
    for k in range(8, -1, -1):
        poly = poly * t + col(tab["amp_ins"][..., k])
    y = col(tab["amp_int_s"]) * f
    inter = col(tab["amp_int"][..., 4])
    for j in range(3, -1, -1):
        inter = inter * y + col(tab["amp_int"][..., j])
    u = col(tab["amp_rd_s"]) * (f - col(tab["amp_rd_shift"]))
    mrd = col(tab["amp_rd_n"]) * np.exp(-col(tab["amp_rd_gr"]) * u) / (u * u + 1.0)
    amp = np.where(f < col(tab["f_amp_ins"]), poly, np.where(f >= col(tab["f_amp_mrd"]), mrd, inter))
    return m76 * amp, phi


def evaluate(tab, f):
    """``(hplus, hcross)`` (``core.py:476-485``)."""
    amp, phi = amplitude_phase(tab, f)
    phi = reduce(phi)
    c, s = np.cos(phi), np.sin(phi)
    ap = np.asarray(tab["kp"])[..., None] * amp
    ac = np.asarray(tab["kc"])[..., None] * amp
    return ap * c + 1j * (ap * s), -ac * s + 1j * (ac * c)


LAYOUT = (("phase", 42), ("big", 2), ("big_lo", 2), ("atan_a", 1), ("atan_w", 1), ("atan_shift", 1),
          ("amp_ins", 10), ("amp_int", 5), ("amp_int_s", 1), ("amp_rd_n", 1), ("amp_rd_gr", 1), ("amp_rd_s", 1),
          ("amp_rd_shift", 1), ("f_phase_ins", 1), ("f_phase_mrd", 1), ("f_amp_ins", 1), ("f_amp_mrd", 1),
          ("kp", 1), ("kc", 1))


def flat(tab):
    """The table in the reference's flat layout (75 values)."""
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
