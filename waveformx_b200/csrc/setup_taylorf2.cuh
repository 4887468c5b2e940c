// The per-binary set-up of TaylorF2 in FP64: from the eight parameters of a
// binary to its table (tables.cuh, Tf2Slot).
//
// The steps follow the reference (models/taylorf2/core.py:107-165): LAL's
// 3.5PN phasing with every spin term (models/taylorf2/pn.py:27-91), folded
// into coefficients of powers of f in Hz; the reference phase
// phi(f_ref) = 2 phi_ref + pi / 4 when f_ref > 0 (f_ref = 0: the reference
// at coalescence), or at M f = reference_mf; the leading term T0 f^-5/3 and
// its value at f_ref in FP64; the amplitude A f^-7/6.
#pragma once

#include "setup_common.cuh"
#include "tables.cuh"

namespace wfx {
namespace taylorf2 {

// The amplitude's coefficient (core.py:86-87): A = kAmp (m1 m2)^(1/2)
// M^(-1/6) / D, masses in solar masses and D in Mpc; LAL's amp0
// sqrt(5 / (32 eta)) (pi M)^(-7/6), amp0 = -4 m1 m2 / D sqrt(pi / 12) in
// geometric units (the double value of
// -4 MRSUN_SI MTSUN_SI / MPC_SI sqrt(pi / 12) sqrt(5 / 32) (pi MTSUN_SI)^(-7/6)).
constexpr double kAmp = -7.806521525937898e-20;
constexpr double kLn4 = 1.3862943611198906;
constexpr double kLog6 = -6848.0 / 21.0;

// The 3PN spin-spin term (pn.py:48-56).
template <class R>
WFX_HDI R spin_spin_3pn(const R& eta, const R& x1, const R& x2, const R& chi1, const R& chi2) {
  R phase = (32675.0 / 112.0 + 5575.0 / 18.0 * eta) * eta * chi1 * chi2;
  const R x[2] = {x1, x2};
  const R chi[2] = {chi1, chi2};
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    const R& xi = x[i];
    phase = phase + ((47035.0 / 84.0 + 2935.0 / 6.0 * xi - 120.0 * xi * xi) +
                     (-410825.0 / 672.0 - 1085.0 / 12.0 * xi + 1255.0 / 36.0 * xi * xi)) *
                        xi * xi * chi[i] * chi[i];
  }
  return phase;
}

// The phasing: v[k], the coefficients of v^(k - 5), and l5, l6 those of
// v^(k - 5) log v, with the factor 3 / (128 eta) (pn.py:27-91).
template <class R>
WFX_HDI void phasing(const R& x1, const R& x2, const R& chi1, const R& chi2, R (&v)[8], R& l5, R& l6) {
  using fit::EGAMMA;
  using fit::PI;
  const R eta = x1 * x2;
  const R scale = 3.0 / (128.0 * eta);
  const R x[2] = {x1, x2};
  const R chi[2] = {chi1, chi2};
  // (the reference's sums start from the integer 0: 0 + term + term)
  R v3 = -16.0 * PI + ((R(0.0) + x[0] * (25.0 + 38.0 / 3.0 * x[0]) * chi[0]) + x[1] * (25.0 + 38.0 / 3.0 * x[1]) * chi[1]);
  R v4 = 15293365.0 / 508032.0 + 27145.0 / 504.0 * eta + 3085.0 / 72.0 * eta * eta;
  v4 = v4 - 395.0 / 4.0 * eta * chi1 * chi2;
#pragma unroll
  for (int i = 0; i < 2; ++i) v4 = v4 - (50.0 + 5.0 / 8.0) * x[i] * x[i] * chi[i] * chi[i];
  R v5 = 5.0 / 9.0 * (7729.0 / 84.0 - 13.0 * eta) * PI;
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    const R& xi = x[i];
    v5 = v5 - chi[i] * xi *
                  (13915.0 / 84.0 - xi * (1.0 - xi) * 10.0 / 3.0 + xi * (12760.0 / 81.0 + xi * (1.0 - xi) * 170.0 / 9.0));
  }
  R v6 = R(11583231236531.0 / 4694215680.0 - 640.0 / 3.0 * (PI * PI) - 6848.0 / 21.0 * EGAMMA);
  v6 = v6 + eta * (-15737765635.0 / 3048192.0 + 2255.0 / 12.0 * (PI * PI));
  v6 = v6 + eta * eta * 76055.0 / 1728.0 - eta * eta * eta * 127825.0 / 1296.0;
  v6 = v6 + kLog6 * kLn4 + spin_spin_3pn(eta, x1, x2, chi1, chi2);
#pragma unroll
  for (int i = 0; i < 2; ++i) v6 = v6 + PI * x[i] * (1490.0 / 3.0 + x[i] * 260.0) * chi[i];
  R v7 = PI * (77096675.0 / 254016.0 + 378515.0 / 1512.0 * eta - 74045.0 / 756.0 * eta * eta);
#pragma unroll
  for (int i = 0; i < 2; ++i) {
    const R& xi = x[i];
    v7 = v7 + chi[i] * xi *
                  (-170978035.0 / 48384.0 + eta * 2876425.0 / 672.0 + eta * eta * 4735.0 / 144.0 +
                   xi * (-7189233785.0 / 1524096.0 + eta * 458555.0 / 3024.0 - eta * eta * 5345.0 / 72.0));
  }
  v[0] = scale * 1.0;
  v[1] = scale * 0.0;
  v[2] = scale * (55.0 * eta / 9.0 + 3715.0 / 756.0);
  v[3] = scale * v3;
  v[4] = scale * v4;
  v[5] = scale * v5;
  v[6] = scale * v6;
  v[7] = scale * v7;
  l5 = scale * 3.0 * v5;
  l6 = scale * kLog6;
}

// The (2,2) mode's projection on the polarizations (core.py:160-164).
template <class R>
WFX_HDI void projection(const R& inclination, R& kp, R& kc) {
  const R ci = w_cos(inclination);
  kp = 0.5 * (1.0 + ci * ci);
  kc = -ci;
}

// The phase at f of a table without its leading term (core.py:174-181):
// the constant, then the terms in the order of the basis, with the powers
// of f as models/xas/core.py:382-403 forms them. (TabT: the table's scalar,
// R: that of f.)
template <class R, class TabT>
WFX_HDI R rest_at(const TabT* tab, const R& f) {
  const R mf1 = 1.0 / f;
  const R lf = w_log(f);
  R t = w_exp(lf / 3.0);
  t = t * (4.0 - t * t * t * mf1) / 3.0;
  const R t2 = t * t, mt1 = t2 * mf1, mt2 = mt1 * mt1;
  const TabT* row = tab + T_PH;
  return row[4] + row[0] * mf1 + row[1] * mt2 + row[2] * mt1 + row[3] * lf + row[5] * t + row[6] * (t * lf) +
         row[7] * t2;
}

// TaylorF2 table of one binary (arguments as xas::setup; f_min unused).
template <class R>
WFX_HDI int32_t setup(const R* p, double /*f_min*/, double amp_scale, double reference_mf, R* tab) {
  using fit::MTSUN_SI;
  using fit::PI;
  int32_t status = 0;
  const R m1 = p[0], m2 = p[1], chi1 = p[2], chi2 = p[3];
  const R distance = p[4], inclination = p[5], phi_ref = p[6], f_ref = p[7];
  if (!(value(m1) > 0.0) || !(value(m2) > 0.0) || !(value(distance) > 0.0)) status |= kStatusBadParameters;
  const R total = m1 + m2;
  R v[8], l5, l6;
  phasing<R>(m1 / total, m2 / total, chi1, chi2, v, l5, l6);
  const R m_sec = total * MTSUN_SI;
  const R log_pim = w_log(PI * m_sec);
  const R u = w_cbrt(PI * m_sec);
  const R u_inv = 1.0 / u;
  // u^(k - 5) for k = 2..7
  const R u_pow[6] = {u_inv * u_inv * u_inv, u_inv * u_inv, u_inv, R(1.0), u, u * u};
  // the slot of v^(k - 5) (and of v^(k - 5) log v) for k = 2..7
  constexpr int kSlot[8] = {-1, -1, 0, 1, 2, 4, 5, 7};
  constexpr int kLogSlot[8] = {-1, -1, -1, -1, -1, 3, 6, -1};
  R* row = tab + T_PH;
#pragma unroll
  for (int k = 2; k < 8; ++k) {
    const R s = u_pow[k - 2];
    R coefficient = v[k];
    if (kLogSlot[k] >= 0) {
      const R l = k == 5 ? l5 : l6;
      coefficient = coefficient + l * log_pim / 3.0;
      row[kLogSlot[k]] = -l / 3.0 * s;
    }
    row[kSlot[k]] = -coefficient * s;
  }

  // the reference: phi(f_ref) = 2 phi_ref + pi / 4 (core.py:142-151)
  bool referenced;
  R rest, f_ref64;
  if (isnan(reference_mf)) {
    referenced = value(f_ref) > 0.0;
    const R f = referenced ? f_ref : R(1.0);
    rest = rest_at<R, R>(tab, f);
    f_ref64 = f;
  } else {
    if (value(f_ref) != 0.0) status |= kStatusReferenceMf;
    referenced = true;
    // -sum_{k >= 2} (v_k + l_k log u) u^(k - 5) at u = (pi reference_mf)^(1/3)
    const double ur = cbrt(PI * reference_mf);
    const double log_u = log(ur);
    R total_mf(0.0);
#pragma unroll
    for (int k = 2; k < 8; ++k) {
      const R c = k == 5 ? v[k] + l5 * log_u : (k == 6 ? v[k] + l6 * log_u : v[k]);
      total_mf = total_mf - c * pow(ur, static_cast<double>(k - 5));
    }
    rest = total_mf;
    f_ref64 = reference_mf / (MTSUN_SI * (m1 + m2));
  }
  const R constant = 2.0 * phi_ref + PI / 4.0 - (referenced ? rest : R(0.0));
  row[4] = row[4] + constant;
  row[T_LIN - T_PH] = R(0.0);
  const R t0 = fit::XAS_K0 * w_cbrt(m1 + m2) / (m1 * m2);
  tab[T_T0] = t0;
  tab[T_ANCHOR] = referenced ? t0 * w_exp(-5.0 / 3.0 * w_log(f_ref64)) : R(0.0);
  tab[T_AMP] = kAmp * amp_scale * w_sqrt(m1 * m2) * w_exp(-1.0 / 6.0 * w_log(total)) / distance;
  R kp, kc;
  projection(inclination, kp, kc);
  const bool refused = status != 0;
  tab[T_KP] = refused ? R(NAN) : kp;
  tab[T_KC] = refused ? R(NAN) : kc;
  return status;
}

}  // namespace taylorf2
}  // namespace wfx
