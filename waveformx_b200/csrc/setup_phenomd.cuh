// The per-binary set-up of IMRPhenomD in FP64: from the eight parameters of
// a binary to its table (tables.cuh, PhdSlot).
//
// The steps follow the reference (models/phenomd/core.py:154-378): the
// phenomenological coefficients in (eta, chi_PN - 1), the final spin, the
// radiated energy, the QNM frequencies from Chebyshev fits in the final
// spin, the TaylorF2 phasing without its 3PN spin-spin term plus pseudo-PN
// terms, the C1/C2 connection by analytic derivatives, the time shift t0 at
// the amplitude peak, the 5 x 5 intermediate-amplitude solve in Mf/f_peak,
// and the folding into coefficients in Hz with the phase alignment at f_ref.
#pragma once

#include "setup_common.cuh"
#include "tables.cuh"

namespace wfx {
namespace phenomd {

constexpr double kFPhaseIns = 0.018;
constexpr double kFAmpIns = 0.014;

template <class R>
WFX_HDI R chebyshev(const double* c, int n, const R& t) {
  // Clenshaw's sum of sum_k c_k T_k(t)
  R b1(0.0), b2(0.0);
  for (int k = n - 1; k >= 1; --k) {
    R b0 = 2.0 * t * b1 - b2 + c[k];
    b2 = b1;
    b1 = b0;
  }
  return t * b1 - b2 + c[0];
}

// The phase at f of a binary's table, without its leading inspiral term:
// what the alignment at f_ref cancels (core.py:340-358). inspiral: f is in
// the inspiral. (TabT: the table's scalar, R: that of f.)
template <class R, class TabT>
WFX_HDI R rest_at(const TabT* tab, const R& f, bool& inspiral) {
  const R mf1 = 1.0 / f;
  const R lf = w_log(f);
  R t = w_exp(lf / 3.0);
  t = t * (4.0 - t * t * t * mf1) / 3.0;
  const R t2 = t * t, mt1 = t2 * mf1;
  const R root = w_sqrt(f);
  const R f34 = root * w_sqrt(root);
  inspiral = value(f) < value(tab[D_F_PHASE_INS]);
  const bool ring = value(f) >= value(tab[D_F_PHASE_MRD]);
  R rest;
  if (inspiral) {
    const TabT* row = tab + D_PH_INS;
    rest = row[0] + row[1] * mf1 + row[2] * (mt1 * mt1) + row[3] * mt1 + row[4] * lf + row[5] * t +
           row[6] * (t * lf) + row[7] * t2 + row[8] * f + row[9] * (f * t) + row[10] * (f * t2) + row[11] * (f * f);
  } else if (ring) {
    const TabT* row = tab + D_PH_RD;
    rest = row[0] + row[1] * f + row[2] * mf1 + row[3] * f34 +
           tab[D_ATAN_A] * w_atan(tab[D_ATAN_W] * (f - tab[D_ATAN_SHIFT]));
  } else {
    const TabT* row = tab + D_PH_INT;
    rest = row[0] + row[1] * f + row[2] * (mf1 * mf1 * mf1) + row[3] * lf;
  }
  return rest;
}

// The (2,2) mode's projection on the polarizations (core.py:376).
template <class R>
WFX_HDI void projection(const R& inclination, R& kp, R& kc) {
  const R ci = w_cos(inclination);
  kp = 0.5 * (1.0 + ci * ci);
  kc = -ci;
}

// The variables of a binary that the fits take (models/phenomd/core.py:
// 154-190).
template <class R>
struct Vars {
  R chi1, chi2, total, x1, x2, eta, delta, xi, y1, y2, spin_final_in, s_e;
};

template <class R>
WFX_HDI Vars<R> variables(const R* p) {
  const R m1 = p[0], m2 = p[1], chi1 = p[2], chi2 = p[3];
  Vars<R> v;
  v.chi1 = chi1;
  v.chi2 = chi2;
  v.total = m1 + m2;
  v.x1 = m1 / v.total;
  v.x2 = m2 / v.total;
  v.eta = v.x1 * v.x2;
  v.delta = v.x1 - v.x2;
  const R chi_s = 0.5 * (chi1 + chi2), chi_a = 0.5 * (chi1 - chi2);
  v.xi = chi_s * (1.0 - v.eta * 76.0 / 113.0) + v.delta * chi_a - 1.0;
  v.y1 = 0.5 * (1.0 + v.delta);
  v.y2 = 0.5 * (1.0 - v.delta);
  v.spin_final_in = v.y1 * v.y1 * chi1 + v.y2 * v.y2 * chi2;
  v.s_e = (v.y1 * v.y1 * chi1 + v.y2 * v.y2 * chi2) / (v.y1 * v.y1 + v.y2 * v.y2);
  return v;
}

// The IMRPhenomD fits (ids fit::PHD_*: kFirstFit .. kFirstFit + kFitCount)
// with the variables each takes.
constexpr int kFirstFit = fit::PHD_PN_PHASE_3;
constexpr int kFitCount = fit::PHD_RADIATED_ENERGY + 1 - kFirstFit;

template <class R>
WFX_HDI R fit_value(int id, const Vars<R>& v) {
  if (id <= fit::PHD_PN_SPIN_SPIN_3) return fit5(id, v.eta, v.x1, v.x2, v.chi1, v.chi2);
  if (id <= fit::PHD_AMP_PN_6) return fit4(id, v.eta, v.delta, v.chi1, v.chi2);
  if (id == fit::PHD_FINAL_SPIN) return fit2(id, v.eta, v.spin_final_in);
  if (id == fit::PHD_RADIATED_ENERGY) return fit2(id, v.eta, v.s_e);
  return fit2(id, v.eta, v.xi);
}

// IMRPhenomD table of one binary (arguments as xas::setup; `fits` as there).
template <class R, class Fits, int ROLE = kRoleAll>
WFX_HDI int32_t setup(const R* p, double f_min, double amp_scale, double reference_mf, R* tab, const Fits& fits) {
  using fit::MTSUN_SI;
  using fit::PI;
  int32_t status = 0;
  const R m1 = p[0], m2 = p[1], chi1 = p[2], chi2 = p[3];
  const R distance = p[4], inclination = p[5], phi_ref = p[6], f_ref_in = p[7];
  if (!(value(m1) > 0.0) || !(value(m2) > 0.0) || !(value(distance) > 0.0)) status |= kStatusBadParameters;
  // --- coefficients in Mf (models/phenomd/core.py:154-274)
  const Vars<R> vars = variables<R>(p);
  const R &total = vars.total, &x1 = vars.x1, &x2 = vars.x2, &eta = vars.eta, &delta = vars.delta;
  const R rho1 = fits(fit::PHD_RHO1), rho2 = fits(fit::PHD_RHO2);
  const R rho3 = fits(fit::PHD_RHO3);
  const R g1 = fits(fit::PHD_GAMMA1), g2 = fits(fit::PHD_GAMMA2);
  const R g3 = fits(fit::PHD_GAMMA3);
  const R collocation = fits(fit::PHD_COLLOCATION);
  const R al1 = fits(fit::PHD_ALPHA1), al2 = fits(fit::PHD_ALPHA2);
  const R al3 = fits(fit::PHD_ALPHA3), al4 = fits(fit::PHD_ALPHA4);
  const R al5 = fits(fit::PHD_ALPHA5);
  const R be1 = fits(fit::PHD_BETA1), be2 = fits(fit::PHD_BETA2);
  const R be3 = fits(fit::PHD_BETA3);
  const R sg1 = fits(fit::PHD_SIGMA1), sg2 = fits(fit::PHD_SIGMA2);
  const R sg3 = fits(fit::PHD_SIGMA3), sg4 = fits(fit::PHD_SIGMA4);
  const R &y1 = vars.y1, &y2 = vars.y2;
  const R af = fits(fit::PHD_FINAL_SPIN);
  if (value(af) > 1.0) status |= kStatusFinalSpin;
  const double ring_c[] = WFX_PHD_FRING;
  const double damp_c[] = WFX_PHD_FDAMP;
  const R tq = 2.0 * w_cbrt(0.5 * (1.0 - af)) - 1.0;
  const R ring = chebyshev(ring_c, fit::kPhdChebyshevCount, tq);
  const R damp = chebyshev(damp_c, fit::kPhdChebyshevCount, tq);
  const R remnant = 1.0 - fits(fit::PHD_RADIATED_ENERGY);
  const R f_ring = ring / remnant, f_damp = damp / remnant;
  const bool below = value(g2) <= 1.0;
  const R root = w_sqrt(below ? 1.0 - g2 * g2 : R(1.0));
  const R f_peak = w_abs(below ? f_ring + f_damp * (root - 1.0) * g3 / g2 : f_ring - f_damp * g3 / g2);
  if constexpr (ROLE == kRoleAll) {
#pragma unroll
    for (int k = 0; k < D_USED; ++k) tab[k] = R(0.0);
  }
  if constexpr ((ROLE & kRoleAmp) != 0) {
  // the amplitude
  R rho[10];
  rho[0] = R(1.0);
  rho[1] = R(0.0);
  rho[2] = fits(fit::PHD_AMP_PN_2);
  rho[3] = fits(fit::PHD_AMP_PN_3);
  rho[4] = fits(fit::PHD_AMP_PN_4);
  rho[5] = fits(fit::PHD_AMP_PN_5);
  rho[6] = fits(fit::PHD_AMP_PN_6);
  rho[7] = rho1 / fit::PI_POW_7_3;
  rho[8] = rho2 / fit::PI_POW_8_3;
  rho[9] = rho3 / fit::PI_POW_3;
  const R sigma = f_damp * g3;
  R delta_int[5];
  {
    const R u = w_cbrt(PI * R(kFAmpIns));
    R amp_ins(0.0), damp_ins(0.0);
    R uk(1.0);
#pragma unroll
    for (int k = 0; k < 10; ++k) {
      if (k > 0) uk = uk * u;
      if (k == 1) continue;
      amp_ins = amp_ins + rho[k] * uk;
      if (k > 1) damp_ins = damp_ins + k / 3.0 * rho[k] * uk;
    }
    damp_ins = damp_ins / kFAmpIns;
    const R d = f_peak - f_ring;
    const R amp_mrd = g1 * sigma / (d * d + sigma * sigma) * w_exp(-g2 * d / sigma);
    const R s2 = d * d + sigma * sigma;
    const R damp_mrd = (-2.0 * d * sigma * g1 / s2 - g2 * g1) / (w_exp(g2 * d / sigma) * s2);
    const R yy1 = kFAmpIns / f_peak;
    const R yy2 = 0.5 * (1.0 + yy1);
    const R yy1_2 = yy1 * yy1, yy1_3 = yy1_2 * yy1, yy2_2 = yy2 * yy2;
    R a[5][5] = {{R(1.0), yy1, yy1_2, yy1_3, yy1_2 * yy1_2},
                 {R(1.0), yy2, yy2_2, yy2_2 * yy2, yy2_2 * yy2_2},
                 {R(1.0), R(1.0), R(1.0), R(1.0), R(1.0)},
                 {R(0.0), R(1.0), 2.0 * yy1, 3.0 * yy1_2, 4.0 * yy1_3},
                 {R(0.0), R(1.0), R(2.0), R(3.0), R(4.0)}};
    R b[5] = {amp_ins, collocation, amp_mrd, damp_ins * f_peak, damp_mrd * f_peak};
    if (!solve(a, b)) status |= kStatusSolve;
#pragma unroll
    for (int j = 0; j < 5; ++j) delta_int[j] = b[j];
  }

  const R s = total * MTSUN_SI;
  const R u = w_cbrt(PI * s);
  R u_pow[10];
  u_pow[0] = R(1.0);
  u_pow[1] = u;
#pragma unroll
  for (int k = 2; k < 10; ++k) u_pow[k] = u_pow[k - 1] * u;
  // the amplitude
  const R prefactor = fit::PHD_K_AMP * amp_scale * w_sqrt(m1 * m2) * w_exp(-w_log(total) / 6.0) / distance;
#pragma unroll
  for (int k = 0; k < 10; ++k) tab[D_AMP_INS + k] = prefactor * rho[k] * u_pow[k];
#pragma unroll
  for (int j = 0; j < 5; ++j) tab[D_AMP_INT + j] = prefactor * delta_int[j];
  const R width = g3 * f_damp;
  tab[D_AMP_INT_S] = s / f_peak;
  tab[D_AMP_RD_N] = prefactor * g1 / width;
  tab[D_AMP_RD_GR] = g2;
  tab[D_AMP_RD_S] = s / width;
  tab[D_AMP_RD_SHIFT] = f_ring / s;
  tab[D_F_AMP_INS] = kFAmpIns / s;
  tab[D_F_AMP_MRD] = f_peak / s;
  if (status & kStatusSolve) {
#pragma unroll
    for (int k = D_AMP_INS; k <= D_AMP_RD_SHIFT; ++k) tab[k] = R(NAN);
  }
  }  // amplitude

  if constexpr ((ROLE & kRolePhase) != 0) {
  // TaylorF2 phasing (models/taylorf2/pn.py:81-91), minus its 3PN
  // spin-spin term, plus the pseudo-PN sigma terms
  const R scale = 3.0 / (128.0 * eta);
  R v[12];
  v[0] = scale * 1.0;
  v[1] = R(0.0);
  v[2] = scale * (55.0 * eta / 9.0 + 3715.0 / 756.0);
  v[3] = scale * fits(fit::PHD_PN_PHASE_3);
  v[4] = scale * fits(fit::PHD_PN_PHASE_4);
  const R ppn5 = fits(fit::PHD_PN_PHASE_5);
  v[5] = scale * ppn5;
  v[6] = scale * fits(fit::PHD_PN_PHASE_6);
  v[7] = scale * fits(fit::PHD_PN_PHASE_7);
  const R l5 = scale * 3.0 * ppn5;
  const R l6 = scale * (-6848.0 / 21.0);
  v[5] = v[5] - PI / 4.0;
  v[6] = v[6] - fits(fit::PHD_PN_SPIN_SPIN_3) * v[0];
  v[8] = sg1 / eta / PI;
  v[9] = sg2 * 0.75 / eta / fit::PI_POW_4_3;
  v[10] = sg3 * 0.6 / eta / fit::PI_POW_5_3;
  v[11] = sg4 * 0.5 / eta / fit::PI_POW_2;

  // u^(k - 5), k = 0 .. 11, by products of u and 1/u (the integer powers
  // of the reference's power function)
  auto u_powers = [&](const R& u, R(&up)[12]) {
    const R inv = 1.0 / u;
    up[5] = R(1.0);
    up[4] = inv;
    up[6] = u;
#pragma unroll
    for (int k = 3; k >= 0; --k) up[k] = up[k + 1] * inv;
#pragma unroll
    for (int k = 7; k < 12; ++k) up[k] = up[k - 1] * u;
  };
  auto ins = [&](const R& mf, bool leading) {
    const R u = w_cbrt(PI * mf);
    const R log_u = w_log(u);
    R up[12];
    u_powers(u, up);
    R sum(0.0);
#pragma unroll
    for (int k = 0; k < 12; ++k) {
      if (k == 1) continue;
      sum = sum + v[k] * up[k];
    }
    sum = sum + (l5 * log_u + l6 * u * log_u);
    // (without the leading term: subtracted, as the reference does)
    return leading ? sum : sum - v[0] * up[0];
  };
  auto dins = [&](const R& mf) {
    const R u = w_cbrt(PI * mf);
    const R log_u = w_log(u);
    R up[12];
    u_powers(u, up);
    R sum(0.0);
#pragma unroll
    for (int k = 0; k < 12; ++k) {
      if (k == 1) continue;
      sum = sum + (k - 5) / 3.0 * v[k] * up[k];
    }
    sum = sum + (l5 * (0.0 / 3.0 * log_u + 1.0 / 3.0) + l6 * u * (1.0 / 3.0 * log_u + 1.0 / 3.0));
    return sum / mf;
  };
  auto inter = [&](const R& mf) { return (be1 * mf - be3 / 3.0 / (mf * mf * mf) + be2 * w_log(mf)) / eta; };
  auto dinter = [&](const R& mf) { return (be1 + be3 / ((mf * mf) * (mf * mf)) + be2 / mf) / eta; };
  auto mrd = [&](const R& mf) {
    const R r4 = w_sqrt(w_sqrt(mf));
    return (al1 * mf - al2 / mf + 4.0 / 3.0 * al3 * (w_sqrt(mf) * r4) + al4 * w_atan((mf - al5 * f_ring) / f_damp)) /
           eta;
  };
  auto dmrd = [&](const R& mf) {
    const R y = (mf - al5 * f_ring) / f_damp;
    return (al1 + al2 / (mf * mf) + al3 / w_sqrt(w_sqrt(mf)) + al4 / (f_damp * (1.0 + y * y))) / eta;
  };
  const R fa = R(kFPhaseIns), fb = 0.5 * f_ring;
  const R c2_int = dins(fa) - dinter(fa);
  const R c1_int = ins(fa, true) - inter(fa) - c2_int * fa;
  const R joined = inter(fb) + c1_int + c2_int * fb;
  const R c2_mrd = c2_int + dinter(fb) - dmrd(fb);
  const R c1_mrd = joined - mrd(fb) - c2_mrd * fb;
  const R t0 = dmrd(f_peak);

  // --- the table in Hz (core.py:280-378)
  const R s = total * MTSUN_SI;
  const R log_s = w_log(s);
  const R log_pis = w_log(PI * s);
  const R u = w_cbrt(PI * s);
  R u_pow[10];
  u_pow[0] = R(1.0);
  u_pow[1] = u;
#pragma unroll
  for (int k = 2; k < 10; ++k) u_pow[k] = u_pow[k - 1] * u;
  const R u_inv = 1.0 / u;
  const R u_pow_inv[4] = {R(1.0), u_inv, u_inv * u_inv, u_inv * u_inv * u_inv};
  // the inspiral row: -v_k (pi s f)^((k-5)/3) (log terms at k = 5, 6);
  // slots of D_PH_INS for k = 2..11: f^-1, f^-2/3, f^-1/3, 1, f^1/3, f^2/3,
  // f, f^4/3, f^5/3, f^2 (log f at k = 5, f^1/3 log f at k = 6)
  {
    R* row = tab + D_PH_INS;
    const int slot[12] = {-1, -1, 1, 2, 3, 0, 5, 7, 8, 9, 10, 11};
#pragma unroll
    for (int k = 2; k < 12; ++k) {
      const R sc = k >= 5 ? u_pow[k - 5] : u_pow_inv[5 - k];
      R coefficient = v[k];
      if (k == 5 || k == 6) {
        const R l = k == 5 ? l5 : l6;
        coefficient = coefficient + l * log_pis / 3.0;
        const int log_slot = k == 5 ? 4 : 6;
        row[log_slot] = row[log_slot] + (-l / 3.0 * sc);
      }
      row[slot[k]] = row[slot[k]] + (-coefficient * sc);
    }
  }
  // intermediate (1, f, f^-3, log f)
  {
    R* row = tab + D_PH_INT;
    row[1] = row[1] + (-(be1 / eta + c2_int) * s);
    row[2] = row[2] + be3 / (3.0 * eta) / (s * s * s);
    row[3] = row[3] + (-be2 / eta);
    row[0] = row[0] + (-be2 / eta * log_s - c1_int);
  }
  // merger-ringdown (1, f, f^-1, f^3/4)
  {
    R* row = tab + D_PH_RD;
    row[1] = row[1] + (-(al1 / eta + c2_mrd) * s);
    row[2] = row[2] + al2 / eta / s;
    row[3] = row[3] + (-4.0 / 3.0 * al3 / eta * w_sqrt(s) * w_sqrt(w_sqrt(s)));
    row[0] = row[0] + (-c1_mrd);
  }
  tab[D_PH_INS + 8] = tab[D_PH_INS + 8] + t0 * s;
  tab[D_PH_INT + 1] = tab[D_PH_INT + 1] + t0 * s;
  tab[D_PH_RD + 1] = tab[D_PH_RD + 1] + t0 * s;
  tab[D_ATAN_A] = -al4 / eta;
  tab[D_ATAN_W] = s / f_damp;
  tab[D_ATAN_SHIFT] = al5 * f_ring / s;
  tab[D_F_PHASE_INS] = kFPhaseIns / s;
  tab[D_F_PHASE_MRD] = 0.5 * f_ring / s;

  // the reference phase: phi(f_ref) = 2 phi_ref (core.py:340-358)
  bool inspiral;
  R rest, f_ref64;
  if (isnan(reference_mf)) {
    const R f = value(f_ref_in) == 0.0 ? R(f_min) : f_ref_in;
    rest = rest_at<R, R>(tab, f, inspiral);
    f_ref64 = f;
  } else {
    if (value(f_ref_in) != 0.0) status |= kStatusReferenceMf;
    inspiral = reference_mf < kFPhaseIns;
    // -Psi + t0 Mf at Mf = reference_mf, without the leading term
    const R mf = R(reference_mf);
    R psi;
    if (reference_mf < value(fa)) {
      psi = ins(mf, false);
    } else if (reference_mf >= value(fb)) {
      psi = mrd(mf) + c1_mrd + c2_mrd * mf;
    } else {
      psi = inter(mf) + c1_int + c2_int * mf;
    }
    rest = -psi + t0 * mf;
    f_ref64 = reference_mf / (MTSUN_SI * (m1 + m2));
  }
  const R shift_constant = 2.0 * phi_ref - rest;
  tab[D_PH_INS + 0] = tab[D_PH_INS + 0] + shift_constant;
  tab[D_PH_INT + 0] = tab[D_PH_INT + 0] + shift_constant;
  tab[D_PH_RD + 0] = tab[D_PH_RD + 0] + shift_constant;
  const R t0_lead = fit::XAS_K0 * w_cbrt(m1 + m2) / (m1 * m2);
  tab[D_T0] = t0_lead;
  tab[D_ANCHOR] = inspiral ? t0_lead * w_exp(-5.0 / 3.0 * w_log(f_ref64)) : R(0.0);

  R kp, kc;
  projection(inclination, kp, kc);
  const bool refused = status != 0;
  tab[D_KP] = refused ? R(NAN) : kp;
  tab[D_KC] = refused ? R(NAN) : kc;
  }  // phase
  return status;
}

// The same with the fits evaluated in place.
template <class R>
WFX_HDI int32_t setup(const R* p, double f_min, double amp_scale, double reference_mf, R* tab) {
  const Vars<R> v = variables<R>(p);
  return setup(p, f_min, amp_scale, reference_mf, tab, DirectFits<R, Vars<R>>{v});
}

}  // namespace phenomd
}  // namespace wfx
