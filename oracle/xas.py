"""IMRPhenomXAS in float64 NumPy, vectorised over binaries: the per-binary
table (``models/xas/core.py:257-379``, with the set-up of
``models/xpnr/internals.py:38-170``, ``models/xpnr/amp22.py:26-129`` and
``models/xpnr/phase22.py:202-476``) and the waveform at the frequencies
(``models/xas/core.py:382-507``). Oracle only (test infrastructure).

Every array of a binary quantity has shape ``(B,)``; the table is a dict of
such arrays (``phase`` is ``(B, 3, 16)``).
"""

from __future__ import annotations

import numpy as np

from .fit_tables import CONSTANTS as K
from .fit_tables import XAS_FDAMP, XAS_FRING
from .fits import evaluate as fit

PI = K["PI"]
MTSUN_SI = K["MTSUN_SI"]
MRSUN_SI = K["MRSUN_SI"]
MPC_SI = K["MPC_SI"]

# the basis f^a (log f)^l of the phase (models/xas/core.py:49-52)
BASIS = ((-5 / 3, 0), (-1, 0), (-2 / 3, 0), (-1 / 3, 0), (0, 1), (0, 0), (1 / 3, 0), (1 / 3, 1), (2 / 3, 0),
         (1, 0), (1, 1), (4 / 3, 0), (5 / 3, 0), (2, 0), (-2, 0), (-3, 0))
INDEX = {key: i for i, key in enumerate(BASIS)}
CONST = INDEX[(0, 0)]
# the terms of each region: inspiral, intermediate, ringdown (core.py:409-415)
REGION_TERMS = (
    tuple(range(1, 14)),
    (INDEX[(1, 0)], INDEX[(0, 1)], INDEX[(-1, 0)], INDEX[(-2, 0)], INDEX[(-3, 0)], INDEX[(0, 0)]),
    (INDEX[(1, 0)], INDEX[(2 / 3, 0)], INDEX[(-1, 0)], INDEX[(-3, 0)], INDEX[(0, 0)]),
)


class Powers:
    """``IMRPhenomX_Initialize_Powers`` (``models/xpnr/_math.py:190-246``):
    powers of ``x`` from one cube root."""

    def __init__(self, x):
        x = np.asarray(x, dtype=np.float64)
        self.itself = x
        self.one_third = np.cbrt(x)
        self.one_sixth = np.sqrt(self.one_third)
        self.m_one = 1.0 / x
        self.log = np.log(x)
        self.two_thirds = self.one_third * self.one_third
        self.m_one_third = self.two_thirds * self.m_one
        self.m_one_sixth = self.one_sixth * self.m_one_third
        self.four_thirds = self.two_thirds * self.two_thirds
        self.five_thirds = self.four_thirds * self.one_third
        self.seven_thirds = self.four_thirds * x
        self.eight_thirds = self.seven_thirds * self.one_third
        self.m_two_thirds = self.m_one_third * self.m_one_third
        self.m_four_thirds = self.m_two_thirds * self.m_two_thirds
        self.m_five_thirds = self.m_four_thirds * self.m_one_third
        self.m_seven_thirds = self.m_four_thirds * self.m_one
        self.m_eight_thirds = self.m_seven_thirds * self.m_one_third
        self.two = x * x
        self.three = self.two * x
        self.four = self.two * self.two
        self.m_two = self.m_one * self.m_one
        self.m_three = self.m_two * self.m_one
        self.m_four = self.m_two * self.m_two
        self.seven_sixths = self.one_sixth * x
        self.m_seven_sixths = self.m_one_sixth * self.m_one


def _horner(coefficients, x):
    total = coefficients[-1]
    for c in coefficients[-2::-1]:
        total = total * x + c
    return total


def qnm(a_final):
    """``(f_ring, f_damp)`` of the (2,2) mode in units of the final mass,
    the fits in powers of ``1 - a`` (``models/xas/core.py:183-229``)."""
    u = 1.0 - a_final
    return (_horner(XAS_FRING[0], u) / _horner(XAS_FRING[1], u),
            _horner(XAS_FDAMP[0], u) / _horner(XAS_FDAMP[1], u))


def _sqrt_nonneg(x):
    return np.where(x > 0, np.sqrt(np.where(x > 0, x, 1.0)), 0.0)


def _f_isco(chif):
    """``XLALSimIMRPhenomXfISCO`` (``_generated/utilities.py:16-26``)."""
    z1 = np.cbrt(1.0 - chif * chif) * (np.cbrt(1.0 + chif) + np.cbrt(1.0 - chif)) + 1.0
    z1 = np.minimum(z1, 3.0)
    z2 = np.sqrt(3.0 * chif * chif + z1 * z1)
    sign = np.where(chif > 0.0, 1.0, np.where(chif < 0.0, -1.0, 0.0))
    r = 3.0 + z2 - sign * np.sqrt((3.0 - z1) * (3.0 + z1 + 2.0 * z2))
    root = np.sqrt(r)
    return 1.0 / (root * root * root + chif) / PI


def variables(m1_in, m2_in, chi1_in, chi2_in, f_ref, phi0, f_min, distance, amp_scale):
    """``IMRPhenomXSetWaveformVariables`` (``models/xpnr/internals.py:38-150``)
    with the QNM frequencies of ``models/xas/core.py:270-278``: a dict."""
    mass_ratio = np.where(m1_in > m2_in, m1_in / m2_in, m2_in / m1_in)
    swap = m1_in < m2_in
    m1 = np.where(swap, m2_in, m1_in)
    m2 = np.where(swap, m1_in, m2_in)
    chi1 = np.where(swap, chi2_in, chi1_in)
    chi2 = np.where(swap, chi1_in, chi2_in)
    delta = np.abs((m1 - m2) / (m1 + m2))
    eta = np.minimum(np.abs(0.25 * (1.0 - delta * delta)), 0.25)
    m_tot = m1 + m2
    m_sec = m_tot * MTSUN_SI
    # the spin combinations of the fits (_generated/utilities.py:34-63)
    delta_u = _sqrt_nonneg(-4.0 * eta + 1.0)
    mm1, mm2 = 0.5 * (1.0 + delta_u), 0.5 * (1.0 - delta_u)
    chi_eff = mm1 * chi1 + mm2 * chi2
    chi_pn_hat = (-(38.0 / 113.0 * eta) * (chi1 + chi2) + chi_eff) / (1.0 - 76.0 * eta / 113.0)
    s_tot_r = (mm1 * mm1 * chi1 + mm2 * mm2 * chi2) / (mm1 * mm1 + mm2 * mm2)
    dchi = chi1 - chi2
    f_ref = np.where(f_ref == 0.0, f_min, f_ref)
    f_cut = np.where(chi_eff > 0.99, 0.33, 0.3) / m_sec
    wf = dict(m1=m1 / m_tot, m2=m2 / m_tot, m_tot=m_tot, m_sec=m_sec, eta=eta, delta=delta, chi1=chi1, chi2=chi2,
              chi_eff=chi_eff, chi_pn_hat=chi_pn_hat, s_tot_r=s_tot_r, dchi=dchi, delta_u=delta_u, f_ref=f_ref,
              phi0=phi0, f_min=f_min, f_cut=f_cut, f_max_prime=f_cut,
              amp0=m_tot * (MRSUN_SI / MPC_SI) * (m_tot * MTSUN_SI) * amp_scale / distance,
              amp_norm=K["SQRT_TWO_THIRDS"] * np.sqrt(eta) * K["LALPI_M_ONE_SIXTH"],
              dphase0=5.0 / (128.0 * PI ** (5.0 / 3.0)))
    wf["error_mass_ratio"] = (mass_ratio > 1000.0) & (np.abs(mass_ratio - 1000.0) > 1e-12)
    wf["error_spin"] = (np.abs(chi1) > 1.0) | (np.abs(chi2) > 1.0)
    wf["m_final"] = fit("XAS_FINAL_MASS", eta, s_tot_r, dchi, delta_u)
    wf["a_final"] = fit("XAS_FINAL_SPIN", eta, s_tot_r, dchi, delta_u)
    f_ring, f_damp = qnm(wf["a_final"])
    wf["f_ring"] = f_ring / wf["m_final"]
    wf["f_damp"] = f_damp / wf["m_final"]
    wf["f_meco"] = fit("XAS_F_MECO", eta, chi_pn_hat, dchi, delta_u)
    wf["f_isco"] = _f_isco(wf["a_final"])
    wf["error"] = (wf["error_mass_ratio"] | wf["error_spin"] | (wf["m_final"] > 1.0)
                   | (np.abs(wf["a_final"]) > 1.0) | (wf["f_meco"] > wf["f_isco"]))
    return wf


def _solve(rows, values):
    """The batched linear solve of the collocation systems (``gsl`` / LAPACK
    LU with partial pivoting, ``models/xpnr/phase22.py:44-49``)."""
    matrix = np.stack([np.stack([np.broadcast_to(np.asarray(x, float), np.shape(values[0])) for x in row], -1)
                       for row in rows], -2)
    rhs = np.stack([np.asarray(v, float) for v in values], -1)
    return np.moveaxis(np.linalg.solve(matrix, rhs[..., None])[..., 0], -1, 0)


def amplitude_coefficients(wf):
    """``IMRPhenomXGetAmplitudeCoefficients`` (``models/xpnr/amp22.py:26-129``)."""
    eta, delta, chi1, chi2 = wf["eta"], wf["delta"], wf["chi1"], wf["chi2"]
    s, dchi = wf["s_tot_r"], wf["dchi"]
    f_ring, f_damp = wf["f_ring"], wf["f_damp"]
    gamma2 = fit("XAS_AMP_RD_GAMMA2", eta, s, dchi, delta)
    gamma3 = fit("XAS_AMP_RD_GAMMA3", eta, s, dchi, delta)
    # the peak of the ringdown amplitude (_generated/ringdown.py:79-81)
    below = gamma2 <= 1.0
    f_rd = np.where(below, np.abs(f_ring + f_damp * gamma3 * (_sqrt_nonneg(1.0 - gamma2 * gamma2) - 1.0) / gamma2),
                    np.abs(f_ring - f_damp * gamma3 / gamma2))
    v1_rd = fit("XAS_AMP_RD_V1", eta, s, dchi, delta)
    gamma1 = ((v1_rd / (f_damp * gamma3))
              * (f_damp * f_damp * gamma3 * gamma3 + (f_ring * f_ring + (f_rd * f_rd - 2.0 * f_rd * f_ring)))
              * np.exp(((f_rd - f_ring) * gamma2) / (f_damp * gamma3)))
    amp = dict(gamma1=gamma1, gamma2=gamma2, gamma3=gamma3, gamma_r=gamma2 / (f_damp * gamma3),
               gamma_d2=(gamma3 * f_damp) * (gamma3 * f_damp), gamma_d13=f_damp * gamma1 * gamma3,
               f_amp_rd_min=f_rd)
    f_in = wf["f_meco"] + 0.25 * (wf["f_isco"] - wf["f_meco"])
    amp["f_amp_match_in"] = f_in
    pn = [fit("XAS_AMP_PN_" + k, eta, chi1, chi2, delta)
          for k in ("TWO_THIRDS", "THREE_THIRDS", "FOUR_THIRDS", "FIVE_THIRDS", "SIX_THIRDS")]
    # the pseudo-PN coefficients rho1..3 of f^(7/3), f^(8/3), f^3 from the
    # three collocation values (the system IMRPhenomX_Inspiral_Amp_22_rho*
    # solves in closed form)
    f_col = [0.5 * f_in, 0.75 * f_in, f_in]
    v_col = [fit(k, eta, wf["chi_pn_hat"], dchi, delta) for k in ("XAS_AMP_INS_V2", "XAS_AMP_INS_V3", "XAS_AMP_INS_V4")]
    rows = [[np.cbrt(f) ** 7, np.cbrt(f) ** 8, f ** 3] for f in f_col]
    rho = _solve(rows, v_col)
    # c_k: the inspiral ansatz sum_k c_k (M f)^(k/3)
    amp["ins"] = [np.ones_like(eta), np.zeros_like(eta), *pn, rho[0], rho[1], rho[2]]

    def ins(mf):
        t = np.cbrt(mf)
        return _horner(amp["ins"], t)

    def dins(mf):
        t = np.cbrt(mf)
        return sum(k / 3.0 * c * t ** (k - 3) for k, c in enumerate(amp["ins"]) if k > 0)

    def rd(mf):
        d = mf - f_ring
        return np.exp(-d * amp["gamma_r"]) * amp["gamma_d13"] / (d * d + amp["gamma_d2"])

    def drd(mf):
        d = mf - f_ring
        dfd = f_damp * gamma3
        return (-np.exp(-gamma2 * d / dfd) * gamma1 * (f_damp * f_damp * gamma2 * gamma3 * gamma3 + d * d * gamma2
                                                       + 2.0 * f_damp * d * gamma3)
                / ((d * d + dfd * dfd) * (d * d + dfd * dfd)))

    # the intermediate amplitude: f^(7/6) / sum_j delta_j f^j, matched in
    # value at f1, f2, f4 and in derivative at f1, f4 (IntAmpVersion 104)
    f1, f4 = f_in, f_rd
    f2 = f1 + 0.5 * (f4 - f1)
    p1, p4 = Powers(f1), Powers(f4)
    a1, a4 = ins(f1), rd(f4)
    v1 = p1.seven_sixths / a1
    v4 = p4.seven_sixths / a4
    v2 = 1.0 / fit("XAS_AMP_INT_VA", eta, s, dchi, delta)
    d1 = (7.0 / 6.0) * p1.one_sixth / a1 - p1.seven_sixths * dins(f1) / (a1 * a1)
    d4 = (7.0 / 6.0) * p4.one_sixth / a4 - p4.seven_sixths * drd(f4) / (a4 * a4)
    # (solved in y = f / f4, better conditioned)
    y1, y2 = f1 / f4, f2 / f4
    one = np.ones_like(y1)
    rows = [[one, y1, y1 ** 2, y1 ** 3, y1 ** 4], [one, y2, y2 ** 2, y2 ** 3, y2 ** 4], [one, one, one, one, one],
            [0 * one, one, 2 * y1, 3 * y1 ** 2, 4 * y1 ** 3], [0 * one, one, 2 * one, 3 * one, 4 * one]]
    x = _solve(rows, [v1, v2, v4, d1 * f4, d4 * f4])
    amp["delta"] = [x[j] / f4 ** j for j in range(5)]
    return amp


def phase_coefficients(wf):
    """``IMRPhenomXGetPhaseCoefficients`` and the connection coefficients
    (``models/xpnr/phase22.py:202-436``)."""
    eta, delta, chi1, chi2 = wf["eta"], wf["delta"], wf["chi1"], wf["chi2"]
    s, dchi = wf["s_tot_r"], wf["dchi"]
    f_ring, f_damp, dphase0 = wf["f_ring"], wf["f_damp"], wf["dphase0"]
    f_im = 0.6 * (0.5 * f_ring + wf["f_isco"])
    f_in = wf["f_meco"]
    df = (f_im - f_in) * 0.03
    ph = dict(f_phase_match_in=f_in - df, f_phase_match_im=f_im + 0.5 * df)
    # ringdown: c0 + c1 f^(-1/3) + c2 f^-2 + c4 f^-4 + c_rd Lorentzian
    f_rd_min, f_rd_max = f_im, 1.25 * f_damp + f_ring
    g5 = (0.0, 0.5 - 1.0 / (2.0 * 2.0 ** 0.5), 0.5, 0.5 + 1.0 / (2.0 * 2.0 ** 0.5), 1.0)
    points = [g * (f_rd_max - f_rd_min) + f_rd_min for g in g5]
    points[3] = f_ring
    v4 = fit("XAS_PHASE_RD_V4", eta, s, dchi, delta)
    d54 = fit("XAS_PHASE_RD_D54", eta, s, dchi, delta) + v4
    d34 = fit("XAS_PHASE_RD_D34", eta, s, dchi, delta) + v4
    d24 = fit("XAS_PHASE_RD_D24", eta, s, dchi, delta) + v4
    d12 = fit("XAS_PHASE_RD_D12", eta, s, dchi, delta) + d24
    values = [d12, d24, d34, v4, d54]
    rows = []
    for f in points:
        inv = 1.0 / f
        rows.append([np.ones_like(f), np.cbrt(inv), inv * inv, (inv * inv) * (inv * inv),
                     -dphase0 / (f_damp * f_damp + (f - f_ring) * (f - f_ring))])
    c0, c1, c2, c4, c_rd = _solve(rows, values)
    c_l = -(dphase0 * c_rd)
    ph.update(c0=c0, c1=c1, c2=c2, c4=c4, c_l=c_l)
    # inspiral pseudo-PN: a0..a3 from four collocation points
    f_ins_min, f_ins_max = 0.0026, 1.020 * wf["f_meco"]
    points = [g * (f_ins_max - f_ins_min) + f_ins_min for g in (0.0, 0.25, 0.75, 1.0)]
    sp = wf["chi_pn_hat"]
    v3 = fit("XAS_PHASE_INS_V3", eta, sp, dchi, delta)
    values = [fit("XAS_PHASE_INS_D13", eta, sp, dchi, delta) + v3, fit("XAS_PHASE_INS_D23", eta, sp, dchi, delta) + v3,
              v3, fit("XAS_PHASE_INS_D43", eta, sp, dchi, delta) + v3]
    rows = [[np.ones_like(f), np.cbrt(f), np.cbrt(f) ** 2, f] for f in points]
    a0, a1, a2, a3 = _solve(rows, values)
    ph.update(a0=a0, a1=a1, a2=a2, a3=a3, sigma1=(-5.0 / 3.0) * a0, sigma2=(-5.0 / 4.0) * a1, sigma3=-a2,
              sigma4=(-5.0 / 6.0) * a3)
    # TaylorF2
    pn = {k: fit("XAS_PHASE_" + k.upper(), eta, chi1, chi2, delta)
          for k in ("phi2", "phi3", "phi4", "phi5l", "phi6", "phi6l", "phi7", "phi8", "phi8l")}
    ph.update(pn)
    ph["phi0"] = 1.0
    ph["phi_norm"] = -(3.0 * K["LALPI_M_FIVE_THIRDS"]) / 128.0
    dphi = dict(d0=1.0, d2=3.0 / 5.0 * pn["phi2"], d3=2.0 / 5.0 * pn["phi3"], d4=1.0 / 5.0 * pn["phi4"],
                d5=-3.0 / 5.0 * pn["phi5l"], d6=-(1.0 / 5.0) * pn["phi6"] - 3.0 / 5.0 * pn["phi6l"],
                d6l=-1.0 / 5.0 * pn["phi6l"], d7=-2.0 / 5.0 * pn["phi7"],
                d8=-(3.0 / 5.0) * pn["phi8"] - 3.0 / 5.0 * pn["phi8l"], d8l=-3.0 / 5.0 * pn["phi8l"])
    dphase_norm = 5.0 / (128.0 * K["LALPI_FIVE_THIRDS"])

    def ins_dphase_sum(p):
        """The bracket of the inspiral phase derivative (inspiral.py:195-211)."""
        x = (dphi["d0"] + dphi["d2"] * p.two_thirds + dphi["d3"] * p.itself + dphi["d4"] * p.four_thirds
             + dphi["d5"] * p.five_thirds + dphi["d6"] * p.two + dphi["d6l"] * p.two * p.log
             + dphi["d7"] * p.seven_thirds + dphi["d8"] * p.eight_thirds + dphi["d8l"] * p.eight_thirds * p.log)
        return x + (a0 * p.eight_thirds + a1 * p.three + a2 * p.eight_thirds * p.two_thirds
                    + a3 * p.eight_thirds * p.itself)

    def ins_dphase(p):
        """d(phase)/d(Mf) of the inspiral."""
        return ins_dphase_sum(p) * p.m_eight_thirds * dphase_norm

    def ins_phase(p):
        """The inspiral phase (inspiral.py:214-230)."""
        x = (1.0 + pn["phi2"] * p.two_thirds + pn["phi3"] * p.itself + pn["phi4"] * p.four_thirds
             + pn["phi5l"] * p.five_thirds * p.log + pn["phi6"] * p.two + pn["phi6l"] * p.two * p.log
             + pn["phi7"] * p.seven_thirds + pn["phi8"] * p.eight_thirds + pn["phi8l"] * p.eight_thirds * p.log)
        x = x + (ph["sigma1"] * p.eight_thirds + ph["sigma2"] * p.three + ph["sigma3"] * p.one_third * p.three
                 + ph["sigma4"] * p.two_thirds * p.three)
        return x * ph["phi_norm"] * p.m_five_thirds

    # the phase derivative at the end of the inspiral, the first value of
    # the intermediate collocation
    p_in = Powers(ph["f_phase_match_in"])
    dphase_in = ins_dphase_sum(p_in) * p_in.m_eight_thirds * dphase0
    # intermediate: b0 + b1 f^-1 + ... + b4 f^-4 + Lorentzian in ring-down units
    f_a, f_b = ph["f_phase_match_in"], ph["f_phase_match_im"]
    points = [g * (f_b - f_a) + f_a for g in g5]
    v2m = fit("XAS_PHASE_INT_V2M_RDV4", eta, s, dchi, delta)
    v3m = fit("XAS_PHASE_INT_V3M_RDV4", eta, s, dchi, delta)
    v2 = fit("XAS_PHASE_INT_V2", eta, s, dchi, delta)
    values = [dphase_in, 0.75 * (v2m + v4) + 0.25 * v2, v3m + v4,
              fit("XAS_PHASE_INT_D43", eta, s, dchi, delta) + v3m + v4, d12]
    rows, rhs = [], []
    for i, f in enumerate(points):
        r = f_ring / f
        lorentz = (4.0 * c_l) / ((2.0 * f_damp) * (2.0 * f_damp) + (f - f_ring) * (f - f_ring)) if i == 0 else \
            (4.0 * c_l) / ((4.0 * f_damp) * f_damp + (f - f_ring) * (f - f_ring))
        rows.append([np.ones_like(f), r, r * r, r * r * r, (r * r) * (r * r)])
        rhs.append(values[i] - lorentz)
    x = _solve(rows, rhs)
    b = [x[0], x[1] * f_ring, x[2] * f_ring * f_ring, x[3] * f_ring * f_ring * f_ring,
         x[4] * f_ring * f_ring * f_ring * f_ring]
    ph.update(b0=b[0], b1=b[1], b2=b[2], b3=b[3], b4=b[4])

    def int_dphase(f, p):
        dfr = f - f_ring
        return (b[0] + b[1] * p.m_one + b[2] * p.m_two + b[3] * p.m_three + b[4] * p.m_four
                + (4.0 * c_l) / (4.0 * f_damp * f_damp + dfr * dfr))

    def int_phase(f, p):
        return (b[0] * f + b[1] * p.log - b[2] * p.m_one - b[3] * p.m_two / 2.0 - b[4] * p.m_three / 3.0
                + (2.0 * c_l * np.arctan((f - f_ring) / (2.0 * f_damp))) / f_damp)

    def rd_dphase(f, p):
        dfr = f - f_ring
        return c0 + c1 * p.m_one_third + c2 * p.m_two + c4 * p.m_four + c_l / (f_damp * f_damp + dfr * dfr)

    def rd_phase(f, p):
        return (c0 * f + 1.5 * c1 * p.two_thirds - c2 * p.m_one - c4 / 3.0 * p.m_three
                + c_l / f_damp * np.arctan((f - f_ring) / f_damp))

    # C1, C2: continuity of the phase and its derivative
    # (IMRPhenomX_Phase_22_ConnectionCoefficients, phase22.py:266-286)
    c2_int = ins_dphase(p_in) - int_dphase(f_a, p_in)
    c1_int = -c2_int * f_a + (ins_phase(p_in) - int_phase(f_a, p_in))
    p_im = Powers(f_b)
    phi_im = c2_int * f_b + (int_phase(f_b, p_im) + c1_int)
    c2_mrd = (int_dphase(f_b, p_im) + c2_int) - rd_dphase(f_b, p_im)
    c1_mrd = -c2_mrd * f_b + (phi_im - rd_phase(f_b, p_im))
    ph.update(c2_int=c2_int, c1_int=c1_int, c2_mrd=c2_mrd, c1_mrd=c1_mrd)
    # the linear time shift (phase22.py:469-476)
    f_fit = f_ring - f_damp
    p_fit = Powers(f_fit)
    dphi_fit = np.where(f_fit < f_a, ins_dphase(p_fit),
                        np.where(f_fit >= f_b, rd_dphase(f_fit, p_fit) + c2_mrd, int_dphase(f_fit, p_fit) + c2_int))
    dphi_fit = 1.0 / eta * dphi_fit
    psi4 = fit("XAS_PSI4_TO_STRAIN", eta, s, dchi, wf["delta_u"])
    ph["linb"] = -(2.0 * PI) * (500.0 + psi4) + (fit("XAS_LINB", eta, s, dchi, delta) - dphi_fit)
    return ph


def frequency_powers(f):
    """The powers of the frequencies (``models/xas/core.py:382-392``)."""
    f = np.asarray(f, dtype=np.float64)
    m1 = 1.0 / f
    log_f = np.log(f)
    t = np.exp(log_f / 3.0)
    t = t * (4.0 - t * t * t * m1) / 3.0
    return f, t, m1, log_f, m1 / np.sqrt(t), np.exp(-5.0 / 3.0 * log_f)


def phase_basis(fp):
    """``PHASE_BASIS`` at the frequencies (``models/xas/core.py:395-403``)."""
    f, t, m1, log_f = fp[:4]
    t2 = t * t
    mt1 = t2 * m1
    mt2 = mt1 * mt1
    m2 = m1 * m1
    return [m1 * mt2, m1, mt2, mt1, log_f, None, t, t * log_f, t2, f, f * log_f, f * t, f * t2, f * f, m2, m2 * m1]


def phase_rest(tab, fp):
    """The phase but for the leading term and the anchor, and whether past
    the inspiral (``models/xas/core.py:423-442``); ``tab`` fields are
    ``(B, ...)`` and the frequencies ``(N,)`` or ``(B, N)``."""
    f = fp[0]
    col = lambda v: np.asarray(v)[..., None]  # noqa: E731
    past = f >= col(tab["f_phase_in"])
    ring = f > col(tab["f_phase_im"])
    basis = phase_basis(fp)
    sums = []
    for r, terms in enumerate(REGION_TERMS):
        total = col(tab["phase"][..., r, CONST])
        for k in terms:
            if basis[k] is not None:
                total = total + col(tab["phase"][..., r, k]) * basis[k]
        sums.append(total)
    rest = np.where(ring, sums[2], np.where(past, sums[1], sums[0]))
    a = np.where(ring, col(tab["atan_a"][..., 2]), col(tab["atan_a"][..., 1]))
    w = np.where(ring, col(tab["atan_w"][..., 2]), col(tab["atan_w"][..., 1]))
    rest = rest + np.where(past, a * np.arctan(w * (f - col(tab["shift"]))), 0.0)
    return rest, past


def table(params, f_min, amp_scale=1e21, reference_mf=None):
    """The table of each binary (``models/xas/core.py:257-379``) as a dict of
    ``(B, ...)`` arrays, with ``error`` (where LAL fails: kp, kc NaN)."""
    params = np.atleast_2d(np.asarray(params, dtype=np.float64))
    m1, m2, chi1, chi2, distance, inclination, phi_ref, f_ref = params.T
    f_min = np.broadcast_to(np.asarray(f_min, dtype=np.float64), m1.shape)
    if reference_mf is not None:
        # (models/xas/model.py:35-45)
        f_ref = np.where(f_ref == 0.0, reference_mf / (MTSUN_SI * (m1 + m2)), np.nan)
    wf = variables(m1, m2, chi1, chi2, f_ref, phi_ref, f_min, distance, amp_scale)
    amp = amplitude_coefficients(wf)
    ph = phase_coefficients(wf)
    inveta = 1.0 / wf["eta"]
    s = wf["m_sec"]
    p = Powers(s)
    s_pow = {-5 / 3: p.m_five_thirds, -1: p.m_one, -2 / 3: p.m_two_thirds, -1 / 3: p.m_one_third, 0: 1.0,
             1 / 3: p.one_third, 2 / 3: p.two_thirds, 1: s, 4 / 3: p.four_thirds, 5 / 3: p.five_thirds, 2: p.two,
             -2: p.m_two, -3: p.m_three}
    norm = inveta * ph["phi_norm"]
    regions = [
        [(norm * ph["phi2"], -1, 0), (norm * ph["phi3"], -2 / 3, 0), (norm * ph["phi4"], -1 / 3, 0),
         (norm * ph["phi5l"], 0, 1), (norm * ph["phi6"], 1 / 3, 0), (norm * ph["phi6l"], 1 / 3, 1),
         (norm * ph["phi7"], 2 / 3, 0), (norm * (ph["phi8"] + ph["sigma1"]), 1, 0), (norm * ph["phi8l"], 1, 1),
         (norm * ph["sigma2"], 4 / 3, 0), (norm * ph["sigma3"], 5 / 3, 0), (norm * ph["sigma4"], 2, 0)],
        [(inveta * (ph["b0"] + ph["c2_int"]), 1, 0), (inveta * ph["b1"], 0, 1), (-inveta * ph["b2"], -1, 0),
         (-inveta * ph["b3"] / 2.0, -2, 0), (-inveta * ph["b4"] / 3.0, -3, 0), (inveta * ph["c1_int"], 0, 0)],
        [(inveta * (ph["c0"] + ph["c2_mrd"]), 1, 0), (inveta * 1.5 * ph["c1"], 2 / 3, 0),
         (-inveta * ph["c2"], -1, 0), (-inveta * (ph["c4"] / 3.0), -3, 0), (inveta * ph["c1_mrd"], 0, 0)],
    ]
    rows = np.zeros(m1.shape + (3, len(BASIS)))
    for r, terms in enumerate(regions):
        for c, a, log in terms + [(ph["linb"], 1, 0)]:
            scaled = c * s_pow[a]
            rows[..., r, INDEX[(a, 0)]] += scaled * p.log if log else scaled
            if log:
                rows[..., r, INDEX[(a, 1)]] += scaled
    f_ring, f_damp = wf["f_ring"], wf["f_damp"]
    zero = np.zeros_like(s)
    tab = dict(
        phase=rows,
        atan_a=np.stack([zero, inveta * 2.0 * ph["c_l"] / f_damp, inveta * (ph["c_l"] / f_damp)], -1),
        atan_w=np.stack([zero, s / (2.0 * f_damp), s / f_damp], -1),
        shift=f_ring / s, f_phase_in=ph["f_phase_match_in"] / s, f_phase_im=ph["f_phase_match_im"] / s,
    )
    # the reference phase: phi(f_ref) = 2 phi0 + pi / 4 (core.py:351-358)
    fr = wf["f_ref"]
    rest, past = phase_rest(tab, frequency_powers(fr[..., None]) if fr.ndim else frequency_powers(fr))
    rest, past = rest[..., 0], past[..., 0]
    tab["phase"][..., :, CONST] += (2.0 * wf["phi0"] + PI / 4.0 - rest)[..., None]
    t0 = K["XAS_K0"] * np.cbrt(m1 + m2) / (m1 * m2)
    anchor = np.where(past, 0.0, t0 * np.exp(-5.0 / 3.0 * np.log(fr)))
    prefactor = wf["amp0"] * wf["amp_norm"]
    scale = prefactor * p.m_seven_sixths
    third = [1.0, p.one_third, p.two_thirds, s, p.four_thirds, p.five_thirds, p.two, p.two * p.one_third,
             p.two * p.two_thirds, p.three]
    s_int = [1.0, s, p.two, p.three, p.four]
    error = wf["error"]
    pfac = 0.5 * (1.0 + np.cos(inclination) ** 2)
    tab.update(
        t0=t0, anchor=anchor,
        amp_ins=np.stack([scale * c * k for c, k in zip(amp["ins"], third)], -1),
        amp_int_n=prefactor, amp_int_d=np.stack([d * k for d, k in zip(amp["delta"], s_int)], -1),
        amp_rd_n=scale * amp["gamma_d13"], amp_rd_gr=amp["gamma_r"], amp_rd_s=s, amp_rd_g=amp["gamma_d2"],
        f_amp_in=amp["f_amp_match_in"] / s, f_amp_rd=amp["f_amp_rd_min"] / s, f_cut=wf["f_max_prime"],
        kp=np.where(error, np.nan, -K["XAS_YLM"] * pfac), kc=np.where(error, np.nan, K["XAS_YLM"] * np.cos(inclination)),
        error=error,
    )
    return tab


def reduce(phi):
    """``phi`` reduced to ``[-pi, pi]`` (``models/xas/core.py:465-468``)."""
    return phi - np.round(phi / (2.0 * np.pi)) * (2.0 * np.pi)


def amplitude_phase(tab, f, anchor=True):
    """The amplitude and the unreduced phase at the frequencies ``f``
    (``(N,)`` shared, or ``(B, N)``): ``models/xas/core.py:445-493``."""
    fp = frequency_powers(f)
    f, t, m1, log_f, m76, f53 = fp
    col = lambda v: np.asarray(v)[..., None]  # noqa: E731
    rest, past = phase_rest(tab, fp)
    phi = np.where(past, 0.0, col(tab["t0"]) * f53) + rest
    if anchor:
        phi = phi - col(tab["anchor"])
    in_amp = f >= col(tab["f_amp_in"])
    rd_amp = f > col(tab["f_amp_rd"])
    poly = col(tab["amp_ins"][..., 9])
    for k in range(8, -1, -1):
        poly = poly * t + col(tab["amp_ins"][..., k])
    den = col(tab["amp_int_d"][..., 4])
    for j in range(3, -1, -1):
        den = den * f + col(tab["amp_int_d"][..., j])
    u = col(tab["amp_rd_s"]) * (f - col(tab["shift"]))
    amp_rd = col(tab["amp_rd_n"]) * m76 * np.exp(-col(tab["amp_rd_gr"]) * u) / (u * u + col(tab["amp_rd_g"]))
    amp = np.where(rd_amp, amp_rd, np.where(in_amp, col(tab["amp_int_n"]) / den, m76 * poly))
    amp = np.where(f <= col(tab["f_cut"]), amp, 0.0)
    return amp, phi


def evaluate(tab, f):
    """``(hplus, hcross)`` (``models/xas/core.py:496-507``)."""
    amp, phi = amplitude_phase(tab, f)
    phi = reduce(phi)
    c, s = np.cos(phi), np.sin(phi)
    ap = np.asarray(tab["kp"])[..., None] * amp
    ac = np.asarray(tab["kc"])[..., None] * amp
    return ap * c + 1j * (ap * s), -ac * s + 1j * (ac * c)


# the order of the reference's flat table (models/xas/core.py:68-89)
LAYOUT = (("phase", 48), ("big", 2), ("big_lo", 2), ("atan_a", 3), ("atan_w", 3), ("shift", 1), ("amp_ins", 10),
          ("amp_int_n", 1), ("amp_int_d", 5), ("amp_rd_n", 1), ("amp_rd_gr", 1), ("amp_rd_s", 1), ("amp_rd_g", 1),
          ("f_phase_in", 1), ("f_phase_im", 1), ("f_amp_in", 1), ("f_amp_rd", 1), ("f_cut", 1), ("kp", 1),
          ("kc", 1))


def flat(tab):
    """The table in the reference's flat layout (86 values), for comparing
    with its tables."""
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
