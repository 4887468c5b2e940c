// The per-binary set-up of IMRPhenomXAS in FP64: from the eight parameters
// of a binary to its table (tables.cuh, XasSlot). One thread per binary (or
// per binary and direction, with R = Dual, for the table's derivatives).
//
// The steps follow the reference's table of coefficients
// (models/xas/core.py:257-379): the waveform variables
// (models/xpnr/internals.py:38-150), the QNM frequencies re-expanded about
// a_final = 1 (core.py:183-229), the amplitude coefficients
// (models/xpnr/amp22.py:26-129), the phase coefficients with their three
// collocation solves and the C1/C2 connection (models/xpnr/phase22.py:
// 202-436), the linear time shift (phase22.py:469-476), the folding of the
// powers of M into coefficients in Hz and the phase alignment at f_ref.
#pragma once

#include "setup_common.cuh"
#include "tables.cuh"

namespace wfx {
namespace xas {

template <class R>
WFX_HDI R f_isco(const R& chif) {
  // XLALSimIMRPhenomXfISCO (_generated/utilities.py:16-26)
  R z1 = w_cbrt(1.0 - chif * chif) * (w_cbrt(1.0 + chif) + w_cbrt(1.0 - chif)) + 1.0;
  z1 = w_min(z1, 3.0);
  R z2 = w_sqrt(3.0 * chif * chif + z1 * z1);
  double sign = value(chif) > 0.0 ? 1.0 : (value(chif) < 0.0 ? -1.0 : 0.0);
  R r = 3.0 + z2 - sign * w_sqrt((3.0 - z1) * (3.0 + z1 + 2.0 * z2));
  R root = w_sqrt(r);
  return 1.0 / (root * root * root + chif) / fit::PI;
}

// The (2,2) QNM frequencies (units of the final mass) from the fits in
// powers of u = 1 - a_final.
template <class R>
WFX_HDI void qnm(const R& a_final, R& f_ring, R& f_damp) {
  const double ring_num[] = WFX_XAS_FRING_NUM;
  const double ring_den[] = WFX_XAS_FRING_DEN;
  const double damp_num[] = WFX_XAS_FDAMP_NUM;
  const double damp_den[] = WFX_XAS_FDAMP_DEN;
  R u = 1.0 - a_final;
  f_ring = horner(ring_num, fit::kXasFringNumCount, u) / horner(ring_den, fit::kXasFringDenCount, u);
  f_damp = horner(damp_num, fit::kXasFdampNumCount, u) / horner(damp_den, fit::kXasFdampDenCount, u);
}

// The phase at f of a binary's table, without its leading inspiral term:
// what the alignment at f_ref cancels (core.py:351-358). past: f is past the
// inspiral; lf = log f. (TabT: the table's scalar, R: that of f.)
template <class R, class TabT>
WFX_HDI R rest_at(const TabT* tab, const R& f, bool& past, R& lf) {
  const R mf1 = 1.0 / f;
  lf = w_log(f);
  R t = w_exp(lf / 3.0);
  t = t * (4.0 - t * t * t * mf1) / 3.0;
  past = value(f) >= value(tab[X_F_PHASE_IN]);
  const bool ring = value(f) > value(tab[X_F_PHASE_IM]);
  const R t2 = t * t, mt1 = t2 * mf1, mt2 = mt1 * mt1, m2 = mf1 * mf1;
  R rest;
  if (ring) {
    const TabT* row = tab + X_PH_RD;
    rest = row[0] + row[1] * f + row[2] * t2 + row[3] * mf1 + row[4] * (m2 * mf1);
  } else if (past) {
    const TabT* row = tab + X_PH_INT;
    rest = row[0] + row[1] * f + row[2] * lf + row[3] * mf1 + row[4] * m2 + row[5] * (m2 * mf1);
  } else {
    const TabT* row = tab + X_PH_INS;
    rest = row[4] + row[0] * mf1 + row[1] * mt2 + row[2] * mt1 + row[3] * lf + row[5] * t + row[6] * (t * lf) +
           row[7] * t2 + row[8] * f + row[9] * (f * lf) + row[10] * (f * t) + row[11] * (f * t2) + row[12] * (f * f);
  }
  if (past) {
    const int r = ring ? 1 : 0;
    rest = rest + tab[X_ATAN_A + r] * w_atan(tab[X_ATAN_W + r] * (f - tab[X_SHIFT]));
  }
  return rest;
}

// The (2,2) mode's projection on the polarizations (core.py:371-372).
template <class R>
WFX_HDI void projection(const R& inclination, R& kp, R& kc) {
  const R ci = w_cos(inclination);
  const R pfac = 0.5 * (1.0 + ci * ci);
  kp = -fit::XAS_YLM * pfac;
  kc = fit::XAS_YLM * ci;
}

// The waveform variables of a binary that the fits take
// (models/xpnr/internals.py:38-150): the masses and spins ordered so that
// m1 >= m2, and the symmetric combinations.
template <class R>
struct Vars {
  R m1, m2, chi1, chi2, delta, eta, delta_u, mm1, mm2, chi_eff, chi_pn_hat, s_tot_r, dchi;
};

template <class R>
WFX_HDI Vars<R> variables(const R* p) {
  const R m1_in = p[0], m2_in = p[1], chi1_in = p[2], chi2_in = p[3];
  const bool swap = value(m1_in) < value(m2_in);
  Vars<R> v;
  v.m1 = swap ? m2_in : m1_in;
  v.m2 = swap ? m1_in : m2_in;
  v.chi1 = swap ? chi2_in : chi1_in;
  v.chi2 = swap ? chi1_in : chi2_in;
  v.delta = w_abs((v.m1 - v.m2) / (v.m1 + v.m2));
  v.eta = w_min(w_abs(0.25 * (1.0 - v.delta * v.delta)), 0.25);
  v.delta_u = sqrt_nonneg(-4.0 * v.eta + 1.0);
  v.mm1 = 0.5 * (1.0 + v.delta_u);
  v.mm2 = 0.5 * (1.0 - v.delta_u);
  v.chi_eff = v.mm1 * v.chi1 + v.mm2 * v.chi2;
  v.chi_pn_hat = (-(38.0 / 113.0 * v.eta) * (v.chi1 + v.chi2) + v.chi_eff) / (1.0 - 76.0 * v.eta / 113.0);
  v.s_tot_r = (v.mm1 * v.mm1 * v.chi1 + v.mm2 * v.mm2 * v.chi2) / (v.mm1 * v.mm1 + v.mm2 * v.mm2);
  v.dchi = v.chi1 - v.chi2;
  return v;
}

// What the set-up of the higher modes of IMRPhenomXHM takes from that of
// the (2,2) (models/xhm/reference.py:84-95, core.py:371-376): the waveform
// variables (frequencies in units of the total mass), the (2,2) ringdown
// amplitude's gammas and the (2,2) phase coefficients (phase22.py), whose
// phase and derivative setup_xhm.cuh evaluates.
template <class R>
struct Internals {
  R eta, delta, q, chi1, chi2, chi_eff, chi_pn_hat, s_tot_r, dchi, m_sec, m_final, a_final, f_ring, f_damp, f_meco,
      amp0, amp_norm, phi0, mf_ref;
  R gamma1, gamma2, gamma3;
  R phi2, phi3, phi4, phi5l, phi6, phi6l, phi7, phi8, phi8l, sigma1, sigma2, sigma3, sigma4;
  R a0, a1, a2, a3, b0, b1, b2, b3, b4, c0, c1, c2, c4, c_l, c1_int, c2_int, c1_mrd, c2_mrd;
  R f_phase_in, f_phase_im, linb;
};

// The IMRPhenomXAS fits (ids fit::XAS_*: kFirstFit .. kFirstFit + kFitCount)
// with the variables each takes.
constexpr int kFirstFit = fit::XAS_AMP_INS_V2;
constexpr int kFitCount = fit::XAS_PHASE_PHI8L + 1 - kFirstFit;

template <class R>
WFX_HDI R fit_value(int id, const Vars<R>& v) {
  if (id == fit::XAS_FINAL_MASS || id == fit::XAS_FINAL_SPIN || id == fit::XAS_PSI4_TO_STRAIN)
    return fit4(id, v.eta, v.s_tot_r, v.dchi, v.delta_u);
  if (id == fit::XAS_F_MECO) return fit4(id, v.eta, v.chi_pn_hat, v.dchi, v.delta_u);
  if (id <= fit::XAS_PHASE_INS_D43) return fit4(id, v.eta, v.chi_pn_hat, v.dchi, v.delta);
  if (id <= fit::XAS_LINB) return fit4(id, v.eta, v.s_tot_r, v.dchi, v.delta);
  return fit4(id, v.eta, v.chi1, v.chi2, v.delta);
}

// IMRPhenomXAS table of one binary. p: mass_1, mass_2 (Msun), chi_1, chi_2,
// luminosity_distance (Mpc), inclination, phi_ref, f_ref (Hz; 0 = f_min).
// reference_mf: NaN for none, else the mass-scaled reference frequency M
// f_ref (f_ref must then be zero). Writes tab[0 .. X_USED) and returns the
// status bits; kp, kc are NaN for a refused binary.
// `fits(id)` gives the value of fit `id` for this binary (DirectFits or
// StagedFits, setup_common.cuh).
// ROLE (Role) selects the part of the table computed: the other part's
// slots are left as they are. A failed amplitude solve makes the amplitude
// slots NaN; any other refusal makes kp, kc NaN.
// `out`, when given, receives the Internals (a full set-up, ROLE kRoleAll).
template <class R, class Fits, int ROLE = kRoleAll>
WFX_HDI int32_t setup(const R* p, double f_min, double amp_scale, double reference_mf, R* tab, const Fits& fits,
                      Internals<R>* out = nullptr) {
  using fit::MTSUN_SI;
  using fit::PI;
  int32_t status = 0;
  const R m1_in = p[0], m2_in = p[1], chi1_in = p[2], chi2_in = p[3];
  const R distance = p[4], inclination = p[5], phi0 = p[6];
  R f_ref = p[7];
  if (!(value(m1_in) > 0.0) || !(value(m2_in) > 0.0) || !(value(distance) > 0.0)) status |= kStatusBadParameters;
  if (!isnan(reference_mf)) {
    // models/xas/model.py:35-45: f_ref = reference_mf / M (f_ref must be 0)
    if (value(f_ref) == 0.0) {
      f_ref = reference_mf / (MTSUN_SI * (m1_in + m2_in));
    } else {
      status |= kStatusReferenceMf;
      f_ref = R(NAN);
    }
  }
  // --- waveform variables (models/xpnr/internals.py:38-150)
  const double mass_ratio = value(m1_in) > value(m2_in) ? value(m1_in) / value(m2_in) : value(m2_in) / value(m1_in);
  const Vars<R> v = variables<R>(p);
  const R &m1 = v.m1, &m2 = v.m2, &chi1 = v.chi1, &chi2 = v.chi2, &delta = v.delta, &eta = v.eta;
  const R &delta_u = v.delta_u, &chi_eff = v.chi_eff, &chi_pn_hat = v.chi_pn_hat, &s_tot_r = v.s_tot_r;
  const R m_tot = m1 + m2;
  const R m_sec = m_tot * MTSUN_SI;
  if (value(f_ref) == 0.0) f_ref = R(f_min);
  const R f_cut = (value(chi_eff) > 0.99 ? 0.33 : 0.3) / m_sec;
  const R amp0 = m_tot * (fit::MRSUN_SI / fit::MPC_SI) * (m_tot * MTSUN_SI) * amp_scale / distance;
  const R amp_norm = fit::SQRT_TWO_THIRDS * w_sqrt(eta) * fit::LALPI_M_ONE_SIXTH;
  const double dphase0 = fit::XAS_DPHASE0;
  if (mass_ratio > 1000.0 && fabs(mass_ratio - 1000.0) > 1e-12) status |= kStatusMassRatio;
  if (fabs(value(chi1)) > 1.0 || fabs(value(chi2)) > 1.0) status |= kStatusSpin;
  const R m_final = fits(fit::XAS_FINAL_MASS);
  const R a_final = fits(fit::XAS_FINAL_SPIN);
  R f_ring, f_damp;
  qnm(a_final, f_ring, f_damp);
  f_ring = f_ring / m_final;
  f_damp = f_damp / m_final;
  const R f_meco = fits(fit::XAS_F_MECO);
  const R fisco = f_isco(a_final);
  if (value(m_final) > 1.0) status |= kStatusFinalMass;
  if (fabs(value(a_final)) > 1.0) status |= kStatusFinalSpin;
  if (value(f_meco) > value(fisco)) status |= kStatusMeco;
  if (out != nullptr) {
    out->eta = eta;
    out->delta = delta;
    out->q = value(eta) == 0.25 ? R(1.0) : (value(m1) > value(m2) ? m1 / m2 : m2 / m1);
    out->chi1 = chi1;
    out->chi2 = chi2;
    out->chi_eff = chi_eff;
    out->chi_pn_hat = chi_pn_hat;
    out->s_tot_r = s_tot_r;
    out->dchi = v.dchi;
    out->m_sec = m_sec;
    out->m_final = m_final;
    out->a_final = a_final;
    out->f_ring = f_ring;
    out->f_damp = f_damp;
    out->f_meco = f_meco;
    out->amp0 = amp0;
    out->amp_norm = amp_norm;
    out->phi0 = phi0;
    out->mf_ref = f_ref * m_sec;
  }

  if constexpr (ROLE == kRoleAll) {
#pragma unroll
    for (int k = 0; k < X_USED; ++k) tab[k] = R(0.0);
  }
  if constexpr ((ROLE & kRoleAmp) != 0) {
  // --- amplitude coefficients (models/xpnr/amp22.py:26-129)
  const R gamma2 = fits(fit::XAS_AMP_RD_GAMMA2);
  const R gamma3 = fits(fit::XAS_AMP_RD_GAMMA3);
  const R f_rd = value(gamma2) <= 1.0
                     ? w_abs(f_ring + f_damp * gamma3 * (sqrt_nonneg(1.0 - gamma2 * gamma2) - 1.0) / gamma2)
                     : w_abs(f_ring - f_damp * gamma3 / gamma2);
  const R v1_rd = fits(fit::XAS_AMP_RD_V1);
  const R gamma1 = (v1_rd / (f_damp * gamma3)) *
                   (f_damp * f_damp * gamma3 * gamma3 + (f_ring * f_ring + (f_rd * f_rd - 2.0 * f_rd * f_ring))) *
                   w_exp(((f_rd - f_ring) * gamma2) / (f_damp * gamma3));
  const R gamma_r = gamma2 / (f_damp * gamma3);
  const R gamma_d2 = (gamma3 * f_damp) * (gamma3 * f_damp);
  const R gamma_d13 = f_damp * gamma1 * gamma3;
  if (out != nullptr) {
    out->gamma1 = gamma1;
    out->gamma2 = gamma2;
    out->gamma3 = gamma3;
  }
  const R f_amp_in = f_meco + 0.25 * (fisco - f_meco);
  // the inspiral ansatz sum_k c_k (Mf)^(k/3): TaylorF2 and the pseudo-PN
  // rho1..3, solved from three collocation values
  R cins[10];
  cins[0] = R(1.0);
  cins[1] = R(0.0);
  cins[2] = fits(fit::XAS_AMP_PN_TWO_THIRDS);
  cins[3] = fits(fit::XAS_AMP_PN_THREE_THIRDS);
  cins[4] = fits(fit::XAS_AMP_PN_FOUR_THIRDS);
  cins[5] = fits(fit::XAS_AMP_PN_FIVE_THIRDS);
  cins[6] = fits(fit::XAS_AMP_PN_SIX_THIRDS);
  {
    R a[3][3], b[3];
    const double g[3] = {0.5, 0.75, 1.0};
    const int ids[3] = {fit::XAS_AMP_INS_V2, fit::XAS_AMP_INS_V3, fit::XAS_AMP_INS_V4};
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      R f = g[i] * f_amp_in;
      R c = w_cbrt(f);
      R c7 = ipow(c, 7);
      a[i][0] = c7;
      a[i][1] = c7 * c;
      a[i][2] = f * f * f;
      b[i] = fits(ids[i]);
    }
    if (!solve(a, b)) status |= kStatusSolve;
    cins[7] = b[0];
    cins[8] = b[1];
    cins[9] = b[2];
  }
  // the intermediate amplitude f^7/6 / sum_j delta_j f^j: values at f1, f2,
  // f4 and derivatives at f1, f4 (IntAmpVersion 104), solved in y = f / f4
  R amp_delta[5];
  {
    const R f1 = f_amp_in, f4 = f_rd;
    const R f2 = f1 + 0.5 * (f4 - f1);
    Powers<R> p1(f1), p4(f4);
    const R t1 = p1.one_third;
    R a1 = horner(cins, 10, t1);
    R da1(0.0);
#pragma unroll
    for (int k = 1; k < 10; ++k) da1 = da1 + (k / 3.0) * cins[k] * (k >= 3 ? ipow(t1, k - 3) : 1.0 / ipow(t1, 3 - k));
    const R d4 = f4 - f_ring;
    const R a4 = w_exp(-d4 * gamma_r) * gamma_d13 / (d4 * d4 + gamma_d2);
    const R dfd = f_damp * gamma3;
    const R da4 = -w_exp(-gamma2 * d4 / dfd) * gamma1 *
                  (f_damp * f_damp * gamma2 * gamma3 * gamma3 + d4 * d4 * gamma2 + 2.0 * f_damp * d4 * gamma3) /
                  ((d4 * d4 + dfd * dfd) * (d4 * d4 + dfd * dfd));
    const R v1 = p1.seven_sixths / a1;
    const R v4 = p4.seven_sixths / a4;
    const R v2 = 1.0 / fits(fit::XAS_AMP_INT_VA);
    const R dd1 = (7.0 / 6.0) * p1.one_sixth / a1 - p1.seven_sixths * da1 / (a1 * a1);
    const R dd4 = (7.0 / 6.0) * p4.one_sixth / a4 - p4.seven_sixths * da4 / (a4 * a4);
    const R y1 = f1 / f4, y2 = f2 / f4;
    R a[5][5] = {{R(1.0), y1, y1 * y1, y1 * y1 * y1, (y1 * y1) * (y1 * y1)},
                 {R(1.0), y2, y2 * y2, y2 * y2 * y2, (y2 * y2) * (y2 * y2)},
                 {R(1.0), R(1.0), R(1.0), R(1.0), R(1.0)},
                 {R(0.0), R(1.0), 2.0 * y1, 3.0 * (y1 * y1), 4.0 * (y1 * y1 * y1)},
                 {R(0.0), R(1.0), R(2.0), R(3.0), R(4.0)}};
    R b[5] = {v1, v2, v4, dd1 * f4, dd4 * f4};
    if (!solve(a, b)) status |= kStatusSolve;
    R scale(1.0);
#pragma unroll
    for (int j = 0; j < 5; ++j) {
      amp_delta[j] = b[j] / scale;
      scale = scale * f4;
    }
  }

  // amplitude (core.py:326-334, 365-373)
  const R prefactor = amp0 * amp_norm;
  const Powers<R> ps(m_sec);
  const R scale = prefactor * ps.m_seven_sixths;
  const R third[10] = {R(1.0),     ps.one_third, ps.two_thirds, m_sec, ps.four_thirds, ps.five_thirds, ps.two,
                       ps.two * ps.one_third, ps.two * ps.two_thirds, ps.three};
#pragma unroll
  for (int k = 0; k < 10; ++k) tab[X_AMP_INS + k] = scale * cins[k] * third[k];
  tab[X_AMP_INT_N] = prefactor;
  const R s_int[5] = {R(1.0), m_sec, ps.two, ps.three, ps.four};
#pragma unroll
  for (int j = 0; j < 5; ++j) tab[X_AMP_INT_D + j] = amp_delta[j] * s_int[j];
  tab[X_AMP_RD_N] = scale * gamma_d13;
  tab[X_AMP_RD_GR] = gamma_r;
  tab[X_AMP_RD_S] = m_sec;
  tab[X_AMP_RD_G] = gamma_d2;
  tab[X_F_AMP_IN] = f_amp_in / m_sec;
  tab[X_F_AMP_RD] = f_rd / m_sec;
  if (status & kStatusSolve) {
#pragma unroll
    for (int k = X_AMP_INS; k <= X_AMP_RD_G; ++k) tab[k] = R(NAN);
  }
  }  // amplitude

  if constexpr ((ROLE & kRolePhase) != 0) {
  // --- phase coefficients (models/xpnr/phase22.py:202-436)
  const R f_im_match = 0.6 * (0.5 * f_ring + fisco);
  const R f_in_match = f_meco;
  const R dfm = (f_im_match - f_in_match) * 0.03;
  const R f_phase_in = f_in_match - dfm;
  const R f_phase_im = f_im_match + 0.5 * dfm;
  const double half_s = 1.0 / (2.0 * sqrt(2.0));
  const double g5[5] = {0.0, 0.5 - half_s, 0.5, 0.5 + half_s, 1.0};
  // ringdown: c0 + c1 f^-1/3 + c2 f^-2 + c4 f^-4 + c_rd Lorentzian
  R c0, c1, c2, c4, c_l, v4rd, d12;
  {
    const R lo = f_im_match, hi = 1.25 * f_damp + f_ring;
    v4rd = fits(fit::XAS_PHASE_RD_V4);
    const R d54 = fits(fit::XAS_PHASE_RD_D54) + v4rd;
    const R d34 = fits(fit::XAS_PHASE_RD_D34) + v4rd;
    const R d24 = fits(fit::XAS_PHASE_RD_D24) + v4rd;
    d12 = fits(fit::XAS_PHASE_RD_D12) + d24;
    R a[5][5], b[5] = {d12, d24, d34, v4rd, d54};
#pragma unroll
    for (int i = 0; i < 5; ++i) {
      R f = i == 3 ? f_ring : g5[i] * (hi - lo) + lo;
      R inv = 1.0 / f;
      a[i][0] = R(1.0);
      a[i][1] = w_cbrt(inv);
      a[i][2] = inv * inv;
      a[i][3] = (inv * inv) * (inv * inv);
      a[i][4] = -dphase0 / (f_damp * f_damp + (f - f_ring) * (f - f_ring));
    }
    if (!solve(a, b)) status |= kStatusSolve;
    c0 = b[0];
    c1 = b[1];
    c2 = b[2];
    c4 = b[3];
    c_l = -(dphase0 * b[4]);
  }
  // inspiral pseudo-PN a0..a3 from four collocation points
  R a0, a1, a2, a3;
  {
    const double ins_min = 0.0026;
    const R ins_max = 1.020 * f_meco;
    const double g4[4] = {0.0, 0.25, 0.75, 1.0};
    const R v3 = fits(fit::XAS_PHASE_INS_V3);
    R b[4] = {fits(fit::XAS_PHASE_INS_D13) + v3,
              fits(fit::XAS_PHASE_INS_D23) + v3, v3,
              fits(fit::XAS_PHASE_INS_D43) + v3};
    R a[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      R f = g4[i] * (ins_max - ins_min) + ins_min;
      R c = w_cbrt(f);
      a[i][0] = R(1.0);
      a[i][1] = c;
      a[i][2] = c * c;
      a[i][3] = f;
    }
    if (!solve(a, b)) status |= kStatusSolve;
    a0 = b[0];
    a1 = b[1];
    a2 = b[2];
    a3 = b[3];
  }
  const R sigma1 = (-5.0 / 3.0) * a0, sigma2 = (-5.0 / 4.0) * a1, sigma3 = -a2, sigma4 = (-5.0 / 6.0) * a3;
  // TaylorF2
  const R phi2 = fits(fit::XAS_PHASE_PHI2);
  const R phi3 = fits(fit::XAS_PHASE_PHI3);
  const R phi4 = fits(fit::XAS_PHASE_PHI4);
  const R phi5l = fits(fit::XAS_PHASE_PHI5L);
  const R phi6 = fits(fit::XAS_PHASE_PHI6);
  const R phi6l = fits(fit::XAS_PHASE_PHI6L);
  const R phi7 = fits(fit::XAS_PHASE_PHI7);
  const R phi8 = fits(fit::XAS_PHASE_PHI8);
  const R phi8l = fits(fit::XAS_PHASE_PHI8L);
  const double phi_norm = -(3.0 * fit::LALPI_M_FIVE_THIRDS) / 128.0;
  const R d2 = 3.0 / 5.0 * phi2, d3 = 2.0 / 5.0 * phi3, d4 = 1.0 / 5.0 * phi4, d5 = -3.0 / 5.0 * phi5l;
  const R d6 = -(1.0 / 5.0) * phi6 - 3.0 / 5.0 * phi6l, d6l = -1.0 / 5.0 * phi6l, d7 = -2.0 / 5.0 * phi7;
  const R d8 = -(3.0 / 5.0) * phi8 - 3.0 / 5.0 * phi8l, d8l = -3.0 / 5.0 * phi8l;
  const double dphase_norm = 5.0 / (128.0 * fit::LALPI_FIVE_THIRDS);
  // the bracket of the inspiral phase derivative and the inspiral phase
  auto ins_dsum = [&](const Powers<R>& q) {
    R x = 1.0 + d2 * q.two_thirds + d3 * q.itself + d4 * q.four_thirds + d5 * q.five_thirds + d6 * q.two +
          d6l * q.two * q.log_ + d7 * q.seven_thirds + d8 * q.eight_thirds + d8l * q.eight_thirds * q.log_;
    return x + (a0 * q.eight_thirds + a1 * q.three + a2 * q.eight_thirds * q.two_thirds + a3 * q.eight_thirds * q.itself);
  };
  auto ins_dphase = [&](const Powers<R>& q) { return ins_dsum(q) * q.m_eight_thirds * dphase_norm; };
  auto ins_phase = [&](const Powers<R>& q) {
    R x = 1.0 + phi2 * q.two_thirds + phi3 * q.itself + phi4 * q.four_thirds + phi5l * q.five_thirds * q.log_ +
          phi6 * q.two + phi6l * q.two * q.log_ + phi7 * q.seven_thirds + phi8 * q.eight_thirds +
          phi8l * q.eight_thirds * q.log_;
    x = x + (sigma1 * q.eight_thirds + sigma2 * q.three + sigma3 * q.one_third * q.three +
             sigma4 * q.two_thirds * q.three);
    return x * phi_norm * q.m_five_thirds;
  };
  const Powers<R> p_in(f_phase_in);
  // intermediate: b0 + b1 r + b2 r^2 + b3 r^3 + b4 r^4 (r = f_ring / f) +
  // Lorentzian
  R b0, b1, b2, b3, b4;
  {
    const R v2m = fits(fit::XAS_PHASE_INT_V2M_RDV4);
    const R v3m = fits(fit::XAS_PHASE_INT_V3M_RDV4);
    const R v2 = fits(fit::XAS_PHASE_INT_V2);
    const R values[5] = {ins_dsum(p_in) * p_in.m_eight_thirds * dphase0, 0.75 * (v2m + v4rd) + 0.25 * v2,
                         v3m + v4rd, fits(fit::XAS_PHASE_INT_D43) + (v3m + v4rd), d12};
    R a[5][5], b[5];
#pragma unroll
    for (int i = 0; i < 5; ++i) {
      R f = g5[i] * (f_phase_im - f_phase_in) + f_phase_in;
      R r = f_ring / f;
      R lorentz = i == 0 ? (4.0 * c_l) / ((2.0 * f_damp) * (2.0 * f_damp) + (f - f_ring) * (f - f_ring))
                         : (4.0 * c_l) / ((4.0 * f_damp) * f_damp + (f - f_ring) * (f - f_ring));
      a[i][0] = R(1.0);
      a[i][1] = r;
      a[i][2] = r * r;
      a[i][3] = r * r * r;
      a[i][4] = (r * r) * (r * r);
      b[i] = values[i] - lorentz;
    }
    if (!solve(a, b)) status |= kStatusSolve;
    b0 = b[0];
    b1 = b[1] * f_ring;
    b2 = b[2] * f_ring * f_ring;
    b3 = b[3] * f_ring * f_ring * f_ring;
    b4 = b[4] * f_ring * f_ring * f_ring * f_ring;
  }
  auto int_dphase = [&](const R& f, const Powers<R>& q) {
    R dfr = f - f_ring;
    return b0 + b1 * q.m_one + b2 * q.m_two + b3 * q.m_three + b4 * q.m_four +
           (4.0 * c_l) / (4.0 * f_damp * f_damp + dfr * dfr);
  };
  auto int_phase = [&](const R& f, const Powers<R>& q) {
    return b0 * f + b1 * q.log_ - b2 * q.m_one - b3 * q.m_two / 2.0 - b4 * q.m_three / 3.0 +
           (2.0 * c_l * w_atan((f - f_ring) / (2.0 * f_damp))) / f_damp;
  };
  auto rd_dphase = [&](const R& f, const Powers<R>& q) {
    R dfr = f - f_ring;
    return c0 + c1 * q.m_one_third + c2 * q.m_two + c4 * q.m_four + c_l / (f_damp * f_damp + dfr * dfr);
  };
  auto rd_phase = [&](const R& f, const Powers<R>& q) {
    return c0 * f + 1.5 * c1 * q.two_thirds - c2 * q.m_one - c4 / 3.0 * q.m_three +
           c_l / f_damp * w_atan((f - f_ring) / f_damp);
  };
  // C1, C2 continuity (phase22.py:266-286)
  const R c2_int = ins_dphase(p_in) - int_dphase(f_phase_in, p_in);
  const R c1_int = -c2_int * f_phase_in + (ins_phase(p_in) - int_phase(f_phase_in, p_in));
  const Powers<R> p_im(f_phase_im);
  const R phi_imc = c2_int * f_phase_im + (int_phase(f_phase_im, p_im) + c1_int);
  const R c2_mrd = (int_dphase(f_phase_im, p_im) + c2_int) - rd_dphase(f_phase_im, p_im);
  const R c1_mrd = -c2_mrd * f_phase_im + (phi_imc - rd_phase(f_phase_im, p_im));
  // the linear time shift (phase22.py:469-476)
  R linb;
  {
    const R f_fit = f_ring - f_damp;
    const Powers<R> q(f_fit);
    R dphi = value(f_fit) < value(f_phase_in)
                 ? ins_dphase(q)
                 : (value(f_fit) >= value(f_phase_im) ? rd_dphase(f_fit, q) + c2_mrd : int_dphase(f_fit, q) + c2_int);
    dphi = 1.0 / eta * dphi;
    const R psi4 = fits(fit::XAS_PSI4_TO_STRAIN);
    linb = -(2.0 * PI) * (500.0 + psi4) + (fits(fit::XAS_LINB) - dphi);
  }
  if (out != nullptr) {
    out->phi2 = phi2;
    out->phi3 = phi3;
    out->phi4 = phi4;
    out->phi5l = phi5l;
    out->phi6 = phi6;
    out->phi6l = phi6l;
    out->phi7 = phi7;
    out->phi8 = phi8;
    out->phi8l = phi8l;
    out->sigma1 = sigma1;
    out->sigma2 = sigma2;
    out->sigma3 = sigma3;
    out->sigma4 = sigma4;
    out->a0 = a0;
    out->a1 = a1;
    out->a2 = a2;
    out->a3 = a3;
    out->b0 = b0;
    out->b1 = b1;
    out->b2 = b2;
    out->b3 = b3;
    out->b4 = b4;
    out->c0 = c0;
    out->c1 = c1;
    out->c2 = c2;
    out->c4 = c4;
    out->c_l = c_l;
    out->c1_int = c1_int;
    out->c2_int = c2_int;
    out->c1_mrd = c1_mrd;
    out->c2_mrd = c2_mrd;
    out->f_phase_in = f_phase_in;
    out->f_phase_im = f_phase_im;
    out->linb = linb;
  }

  // --- the table in Hz (models/xas/core.py:286-379)
  const R inveta = 1.0 / eta;
  const Powers<R> ps(m_sec);
  const R log_s = ps.log_;
  // inspiral row: c (s f)^a (log s f)^l folded; basis order of X_PH_INS
  // (f^-1, f^-2/3, f^-1/3, log f, 1, f^1/3, f^1/3 log f, f^2/3, f, f log f,
  // f^4/3, f^5/3, f^2)
  {
    R* row = tab + X_PH_INS;
    const R norm = inveta * phi_norm;
    row[0] = row[0] + norm * phi2 * ps.m_one;
    row[1] = row[1] + norm * phi3 * ps.m_two_thirds;
    row[2] = row[2] + norm * phi4 * ps.m_one_third;
    {
      R c = norm * phi5l;  // (x^0, log x)
      row[4] = row[4] + c * log_s;
      row[3] = row[3] + c;
    }
    row[5] = row[5] + norm * phi6 * ps.one_third;
    {
      R c = norm * phi6l * ps.one_third;
      row[5] = row[5] + c * log_s;
      row[6] = row[6] + c;
    }
    row[7] = row[7] + norm * phi7 * ps.two_thirds;
    row[8] = row[8] + norm * (phi8 + sigma1) * m_sec;
    {
      R c = norm * phi8l * m_sec;
      row[8] = row[8] + c * log_s;
      row[9] = row[9] + c;
    }
    row[10] = row[10] + norm * sigma2 * ps.four_thirds;
    row[11] = row[11] + norm * sigma3 * ps.five_thirds;
    row[12] = row[12] + norm * sigma4 * ps.two;
    row[8] = row[8] + linb * m_sec;
  }
  // intermediate row (1, f, log f, f^-1, f^-2, f^-3)
  {
    R* row = tab + X_PH_INT;
    row[1] = row[1] + inveta * (b0 + c2_int) * m_sec;
    {
      R c = inveta * b1;  // (x^0, log x)
      row[0] = row[0] + c * log_s;
      row[2] = row[2] + c;
    }
    row[3] = row[3] + (-inveta * b2) * ps.m_one;
    row[4] = row[4] + (-inveta * b3 / 2.0) * ps.m_two;
    row[5] = row[5] + (-inveta * b4 / 3.0) * ps.m_three;
    row[0] = row[0] + inveta * c1_int;
    row[1] = row[1] + linb * m_sec;
  }
  // ringdown row (1, f, f^2/3, f^-1, f^-3)
  {
    R* row = tab + X_PH_RD;
    row[1] = row[1] + inveta * (c0 + c2_mrd) * m_sec;
    row[2] = row[2] + inveta * 1.5 * c1 * ps.two_thirds;
    row[3] = row[3] + (-inveta * c2) * ps.m_one;
    row[4] = row[4] + (-inveta * (c4 / 3.0)) * ps.m_three;
    row[0] = row[0] + inveta * c1_mrd;
    row[1] = row[1] + linb * m_sec;
  }
  tab[X_ATAN_A + 0] = inveta * 2.0 * c_l / f_damp;
  tab[X_ATAN_A + 1] = inveta * (c_l / f_damp);
  tab[X_ATAN_W + 0] = m_sec / (2.0 * f_damp);
  tab[X_ATAN_W + 1] = m_sec / f_damp;
  tab[X_SHIFT] = f_ring / m_sec;
  tab[X_F_PHASE_IN] = f_phase_in / m_sec;
  tab[X_F_PHASE_IM] = f_phase_im / m_sec;

  // the reference phase: phi(f_ref) = 2 phi0 + pi / 4 (core.py:351-358)
  const R t0 = fit::XAS_K0 * w_cbrt(m1_in + m2_in) / (m1_in * m2_in);
  R anchor(0.0);
  {
    bool past;
    R lf;
    const R rest = rest_at<R, R>(tab, f_ref, past, lf);
    const R shift_constant = 2.0 * phi0 + PI / 4.0 - rest;
    tab[X_PH_INS + 4] = tab[X_PH_INS + 4] + shift_constant;
    tab[X_PH_INT + 0] = tab[X_PH_INT + 0] + shift_constant;
    tab[X_PH_RD + 0] = tab[X_PH_RD + 0] + shift_constant;
    if (!past) anchor = t0 * w_exp(-5.0 / 3.0 * lf);
  }
  tab[X_T0] = t0;
  tab[X_ANCHOR] = anchor;

  tab[X_F_CUT] = f_cut;
  R kp, kc;
  projection(inclination, kp, kc);
  const bool refused = status != 0;
  tab[X_KP] = refused ? R(NAN) : kp;
  tab[X_KC] = refused ? R(NAN) : kc;
  }  // phase
  return status;
}

// The same with the fits evaluated in place.
template <class R>
WFX_HDI int32_t setup(const R* p, double f_min, double amp_scale, double reference_mf, R* tab) {
  const Vars<R> v = variables<R>(p);
  return setup(p, f_min, amp_scale, reference_mf, tab, DirectFits<R, Vars<R>>{v});
}

}  // namespace xas
}  // namespace wfx
