// The per-binary set-up of IMRPhenomXHM's higher modes (2,1), (3,3), (3,2),
// (4,4) in FP64, after that of the (2,2) (setup_xas.cuh, whose Internals it
// reads): from the binary to one table per mode in the layout of the
// reference's MODE_LAYOUT (models/xhm/core.py:78-113), and the head (the
// modes' factors in the polarizations, amp0, M in seconds;
// core.py:114-122, 361-369).
//
// The steps follow models/xhm/core.py:208-353 (the mode's coefficients
// without the anchor of the (2,2), the spheroidal (3,2) ringdown, the
// alignment D with the (2,2)) over models/xhm/reference.py (LAL's
// IMRPhenomXHM 122022 in Mf: the amplitude collocations, the phase
// collocations, the rotation of the (3,2) ringdown) and
// models/xpnr/hm/{variables,inspiral,phase}.py. The phenomenological fits
// are hm_fit_code.h. Where the reference takes exact derivatives of an
// ansatz in the frequency (jax.jvp, reference.py:72-74) this code runs the
// same ansatz on Dual (first derivative) or Jet2 (first and second).
#pragma once

#include "hm_fit_code.h"
#include "setup_xas.cuh"

namespace wfx {
namespace xhm {

// ---------------------------------------------------------------------------
// Jet2: a value with its first and second derivative along one direction.

struct Jet2 {
  double v, d, dd;
  WFX_HD Jet2() : v(0.0), d(0.0), dd(0.0) {}
  WFX_HD Jet2(double value) : v(value), d(0.0), dd(0.0) {}  // NOLINT: constants promote
  WFX_HD Jet2(double value, double d1, double d2) : v(value), d(d1), dd(d2) {}
};

WFX_HD double value(const Jet2& x) { return x.v; }
WFX_HD Jet2 operator+(Jet2 a, Jet2 b) { return Jet2(a.v + b.v, a.d + b.d, a.dd + b.dd); }
WFX_HD Jet2 operator-(Jet2 a, Jet2 b) { return Jet2(a.v - b.v, a.d - b.d, a.dd - b.dd); }
WFX_HD Jet2 operator-(Jet2 a) { return Jet2(-a.v, -a.d, -a.dd); }
WFX_HD Jet2 operator*(Jet2 a, Jet2 b) {
  return Jet2(a.v * b.v, a.d * b.v + a.v * b.d, a.dd * b.v + 2.0 * a.d * b.d + a.v * b.dd);
}
// g(x) of a jet from g, g', g'' at x.v
WFX_HD Jet2 chain(const Jet2& x, double g, double g1, double g2) {
  return Jet2(g, g1 * x.d, g2 * x.d * x.d + g1 * x.dd);
}
WFX_HD Jet2 operator/(Jet2 a, Jet2 b) {
  const double r = 1.0 / b.v;
  return a * chain(b, r, -r * r, 2.0 * r * r * r);
}
WFX_HD Jet2 operator+(Jet2 a, double b) { return Jet2(a.v + b, a.d, a.dd); }
WFX_HD Jet2 operator+(double a, Jet2 b) { return Jet2(a + b.v, b.d, b.dd); }
WFX_HD Jet2 operator-(Jet2 a, double b) { return Jet2(a.v - b, a.d, a.dd); }
WFX_HD Jet2 operator-(double a, Jet2 b) { return Jet2(a - b.v, -b.d, -b.dd); }
WFX_HD Jet2 operator*(Jet2 a, double b) { return Jet2(a.v * b, a.d * b, a.dd * b); }
WFX_HD Jet2 operator*(double a, Jet2 b) { return Jet2(a * b.v, a * b.d, a * b.dd); }
WFX_HD Jet2 operator/(Jet2 a, double b) { return Jet2(a.v / b, a.d / b, a.dd / b); }
WFX_HD Jet2 operator/(double a, Jet2 b) { return Jet2(a) / b; }
WFX_HD bool operator<(Jet2 a, Jet2 b) { return a.v < b.v; }
WFX_HD bool operator>(Jet2 a, Jet2 b) { return a.v > b.v; }
WFX_HD bool operator<=(Jet2 a, Jet2 b) { return a.v <= b.v; }
WFX_HD bool operator>=(Jet2 a, Jet2 b) { return a.v >= b.v; }
WFX_HD Jet2 w_sqrt(Jet2 x) {
  const double r = sqrt(x.v);
  return chain(x, r, 0.5 / r, -0.25 / (r * x.v));
}
WFX_HD Jet2 w_cbrt(Jet2 x) {
  const double r = cbrt(x.v);
  const double g1 = r / (3.0 * x.v);
  return chain(x, r, g1, -2.0 * g1 / (3.0 * x.v));
}
WFX_HD Jet2 w_exp(Jet2 x) {
  const double e = exp(x.v);
  return chain(x, e, e, e);
}
WFX_HD Jet2 w_log(Jet2 x) { return chain(x, log(x.v), 1.0 / x.v, -1.0 / (x.v * x.v)); }
WFX_HD Jet2 w_atan(Jet2 x) {
  const double q = 1.0 / (1.0 + x.v * x.v);
  return chain(x, atan(x.v), q, -2.0 * x.v * q * q);
}
WFX_HD Jet2 w_cos(Jet2 x) { return chain(x, cos(x.v), -sin(x.v), -cos(x.v)); }
WFX_HD Jet2 w_sin(Jet2 x) { return chain(x, sin(x.v), cos(x.v), -sin(x.v)); }
WFX_HD Jet2 w_pow(Jet2 x, double p) {
  const double r = pow(x.v, p);
  return chain(x, r, p * r / x.v, p * (p - 1.0) * r / (x.v * x.v));
}

// ---------------------------------------------------------------------------
// The same derivatives in the frequency when the set-up itself runs on Dual
// (its derivative along one parameter, for the exact d table / d params):
// DualF, a Dual value with its Dual derivative in the frequency, and Jet2D,
// a Dual value with its first and second Dual derivatives. value() of
// either is the plain double.

struct DualF {
  Dual v, d;
  WFX_HD DualF() : v(0.0), d(0.0) {}
  WFX_HD DualF(double value) : v(value), d(0.0) {}  // NOLINT: constants promote
  WFX_HD DualF(const Dual& value) : v(value), d(0.0) {}  // NOLINT: set-up values promote
  WFX_HD DualF(const Dual& value, const Dual& derivative) : v(value), d(derivative) {}
};

WFX_HD double value(const DualF& x) { return x.v.v; }
WFX_HD DualF operator+(const DualF& a, const DualF& b) { return DualF(a.v + b.v, a.d + b.d); }
WFX_HD DualF operator-(const DualF& a, const DualF& b) { return DualF(a.v - b.v, a.d - b.d); }
WFX_HD DualF operator-(const DualF& a) { return DualF(-a.v, -a.d); }
WFX_HD DualF operator*(const DualF& a, const DualF& b) { return DualF(a.v * b.v, a.d * b.v + a.v * b.d); }
WFX_HD DualF operator/(const DualF& a, const DualF& b) {
  const Dual q = a.v / b.v;
  return DualF(q, (a.d - q * b.d) / b.v);
}
WFX_HD DualF operator+(const DualF& a, const Dual& b) { return DualF(a.v + b, a.d); }
WFX_HD DualF operator+(const Dual& a, const DualF& b) { return DualF(a + b.v, b.d); }
WFX_HD DualF operator-(const DualF& a, const Dual& b) { return DualF(a.v - b, a.d); }
WFX_HD DualF operator-(const Dual& a, const DualF& b) { return DualF(a - b.v, -b.d); }
WFX_HD DualF operator*(const DualF& a, const Dual& b) { return DualF(a.v * b, a.d * b); }
WFX_HD DualF operator*(const Dual& a, const DualF& b) { return DualF(a * b.v, a * b.d); }
WFX_HD DualF operator/(const DualF& a, const Dual& b) { return DualF(a.v / b, a.d / b); }
WFX_HD DualF operator/(const Dual& a, const DualF& b) { return DualF(a) / b; }
WFX_HD DualF operator+(const DualF& a, double b) { return DualF(a.v + b, a.d); }
WFX_HD DualF operator+(double a, const DualF& b) { return DualF(a + b.v, b.d); }
WFX_HD DualF operator-(const DualF& a, double b) { return DualF(a.v - b, a.d); }
WFX_HD DualF operator-(double a, const DualF& b) { return DualF(a - b.v, -b.d); }
WFX_HD DualF operator*(const DualF& a, double b) { return DualF(a.v * b, a.d * b); }
WFX_HD DualF operator*(double a, const DualF& b) { return DualF(a * b.v, a * b.d); }
WFX_HD DualF operator/(const DualF& a, double b) { return DualF(a.v / b, a.d / b); }
WFX_HD DualF operator/(double a, const DualF& b) { return DualF(a) / b; }
WFX_HD bool operator<(const DualF& a, const DualF& b) { return value(a) < value(b); }
WFX_HD bool operator>(const DualF& a, const DualF& b) { return value(a) > value(b); }
WFX_HD bool operator<=(const DualF& a, const DualF& b) { return value(a) <= value(b); }
WFX_HD bool operator>=(const DualF& a, const DualF& b) { return value(a) >= value(b); }
WFX_HD DualF w_sqrt(const DualF& x) {
  const Dual r = w_sqrt(x.v);
  return DualF(r, x.d * 0.5 / r);
}
WFX_HD DualF w_cbrt(const DualF& x) {
  const Dual r = w_cbrt(x.v);
  return DualF(r, x.d * r / (3.0 * x.v));
}
WFX_HD DualF w_exp(const DualF& x) {
  const Dual e = w_exp(x.v);
  return DualF(e, x.d * e);
}
WFX_HD DualF w_log(const DualF& x) { return DualF(w_log(x.v), x.d / x.v); }
WFX_HD DualF w_atan(const DualF& x) { return DualF(w_atan(x.v), x.d / (1.0 + x.v * x.v)); }
WFX_HD DualF w_cos(const DualF& x) { return DualF(w_cos(x.v), -w_sin(x.v) * x.d); }
WFX_HD DualF w_sin(const DualF& x) { return DualF(w_sin(x.v), w_cos(x.v) * x.d); }
WFX_HD DualF w_pow(const DualF& x, double p) {
  const Dual r = w_pow(x.v, p);
  return DualF(r, x.d * p * w_pow(x.v, p - 1.0));
}

struct Jet2D {
  Dual v, d, dd;
  WFX_HD Jet2D() : v(0.0), d(0.0), dd(0.0) {}
  WFX_HD Jet2D(double value) : v(value), d(0.0), dd(0.0) {}  // NOLINT: constants promote
  WFX_HD Jet2D(const Dual& value) : v(value), d(0.0), dd(0.0) {}  // NOLINT: set-up values promote
  WFX_HD Jet2D(const Dual& value, const Dual& d1, const Dual& d2) : v(value), d(d1), dd(d2) {}
};

WFX_HD double value(const Jet2D& x) { return x.v.v; }
WFX_HD Jet2D operator+(const Jet2D& a, const Jet2D& b) { return Jet2D(a.v + b.v, a.d + b.d, a.dd + b.dd); }
WFX_HD Jet2D operator-(const Jet2D& a, const Jet2D& b) { return Jet2D(a.v - b.v, a.d - b.d, a.dd - b.dd); }
WFX_HD Jet2D operator-(const Jet2D& a) { return Jet2D(-a.v, -a.d, -a.dd); }
WFX_HD Jet2D operator*(const Jet2D& a, const Jet2D& b) {
  return Jet2D(a.v * b.v, a.d * b.v + a.v * b.d, a.dd * b.v + 2.0 * a.d * b.d + a.v * b.dd);
}
// g(x) of a jet from g, g', g'' at x.v
WFX_HD Jet2D chain(const Jet2D& x, const Dual& g, const Dual& g1, const Dual& g2) {
  return Jet2D(g, g1 * x.d, g2 * x.d * x.d + g1 * x.dd);
}
WFX_HD Jet2D operator/(const Jet2D& a, const Jet2D& b) {
  const Dual r = 1.0 / b.v;
  return a * chain(b, r, -r * r, 2.0 * r * r * r);
}
WFX_HD Jet2D operator+(const Jet2D& a, const Dual& b) { return Jet2D(a.v + b, a.d, a.dd); }
WFX_HD Jet2D operator+(const Dual& a, const Jet2D& b) { return Jet2D(a + b.v, b.d, b.dd); }
WFX_HD Jet2D operator-(const Jet2D& a, const Dual& b) { return Jet2D(a.v - b, a.d, a.dd); }
WFX_HD Jet2D operator-(const Dual& a, const Jet2D& b) { return Jet2D(a - b.v, -b.d, -b.dd); }
WFX_HD Jet2D operator*(const Jet2D& a, const Dual& b) { return Jet2D(a.v * b, a.d * b, a.dd * b); }
WFX_HD Jet2D operator*(const Dual& a, const Jet2D& b) { return Jet2D(a * b.v, a * b.d, a * b.dd); }
WFX_HD Jet2D operator/(const Jet2D& a, const Dual& b) { return Jet2D(a.v / b, a.d / b, a.dd / b); }
WFX_HD Jet2D operator/(const Dual& a, const Jet2D& b) { return Jet2D(a) / b; }
WFX_HD Jet2D operator+(const Jet2D& a, double b) { return Jet2D(a.v + b, a.d, a.dd); }
WFX_HD Jet2D operator+(double a, const Jet2D& b) { return Jet2D(a + b.v, b.d, b.dd); }
WFX_HD Jet2D operator-(const Jet2D& a, double b) { return Jet2D(a.v - b, a.d, a.dd); }
WFX_HD Jet2D operator-(double a, const Jet2D& b) { return Jet2D(a - b.v, -b.d, -b.dd); }
WFX_HD Jet2D operator*(const Jet2D& a, double b) { return Jet2D(a.v * b, a.d * b, a.dd * b); }
WFX_HD Jet2D operator*(double a, const Jet2D& b) { return Jet2D(a * b.v, a * b.d, a * b.dd); }
WFX_HD Jet2D operator/(const Jet2D& a, double b) { return Jet2D(a.v / b, a.d / b, a.dd / b); }
WFX_HD Jet2D operator/(double a, const Jet2D& b) { return Jet2D(a) / b; }
WFX_HD bool operator<(const Jet2D& a, const Jet2D& b) { return value(a) < value(b); }
WFX_HD bool operator>(const Jet2D& a, const Jet2D& b) { return value(a) > value(b); }
WFX_HD bool operator<=(const Jet2D& a, const Jet2D& b) { return value(a) <= value(b); }
WFX_HD bool operator>=(const Jet2D& a, const Jet2D& b) { return value(a) >= value(b); }
WFX_HD Jet2D w_sqrt(const Jet2D& x) {
  const Dual r = w_sqrt(x.v);
  return chain(x, r, 0.5 / r, -0.25 / (r * x.v));
}
WFX_HD Jet2D w_cbrt(const Jet2D& x) {
  const Dual r = w_cbrt(x.v);
  const Dual g1 = r / (3.0 * x.v);
  return chain(x, r, g1, -2.0 * g1 / (3.0 * x.v));
}
WFX_HD Jet2D w_exp(const Jet2D& x) {
  const Dual e = w_exp(x.v);
  return chain(x, e, e, e);
}
WFX_HD Jet2D w_log(const Jet2D& x) { return chain(x, w_log(x.v), 1.0 / x.v, -1.0 / (x.v * x.v)); }
WFX_HD Jet2D w_atan(const Jet2D& x) {
  const Dual q = 1.0 / (1.0 + x.v * x.v);
  return chain(x, w_atan(x.v), q, -2.0 * x.v * q * q);
}
WFX_HD Jet2D w_cos(const Jet2D& x) { return chain(x, w_cos(x.v), -w_sin(x.v), -w_cos(x.v)); }
WFX_HD Jet2D w_sin(const Jet2D& x) { return chain(x, w_sin(x.v), w_cos(x.v), -w_sin(x.v)); }
WFX_HD Jet2D w_pow(const Jet2D& x, double p) {
  const Dual r = w_pow(x.v, p);
  return chain(x, r, p * r / x.v, p * (p - 1.0) * r / (x.v * x.v));
}

// tanh of a set-up scalar.
WFX_HD double w_tanh(double x) { return tanh(x); }
WFX_HD Dual w_tanh(const Dual& x) {
  const double t = tanh(x.v);
  return Dual(t, x.d * (1.0 - t * t));
}

// The derivative types of a set-up on scalar R: the first derivative in the
// frequency (F1) and the first and second (J2).
template <class R>
struct Deriv;
template <>
struct Deriv<double> {
  using F1 = Dual;
  using J2 = Jet2;
};
template <>
struct Deriv<Dual> {
  using F1 = DualF;
  using J2 = Jet2D;
};

// (the double and Dual overloads beside those of Jet2)
using wfx::value;
using wfx::w_atan;
using wfx::w_cbrt;
using wfx::w_cos;
using wfx::w_exp;
using wfx::w_log;
using wfx::w_pow;
using wfx::w_sin;
using wfx::w_sqrt;

// atan2 and hypot for double, Dual and Jet2 (the derivative types: atan2
// as the angle at the value plus atan of the turn from there, which
// vanishes at the value).
WFX_HD double w_atan2(double y, double x) { return atan2(y, x); }
WFX_HD double w_hypot(double a, double b) { return hypot(a, b); }
template <class T>
WFX_HD T w_atan2(const T& y, const T& x) {
  const double x0 = value(x), y0 = value(y);
  return T(atan2(y0, x0)) + w_atan((x0 * y - y0 * x) / (x0 * x + y0 * y));
}
template <class T>
WFX_HD T w_hypot(const T& a, const T& b) {
  return w_sqrt(a * a + b * b);
}

// ---------------------------------------------------------------------------
// The modes.

constexpr int kModes = 4;                    // (2,1), (3,3), (3,2), (4,4): LAL's modeInt 0..3
constexpr int kModeSize = 112;               // MODE_LAYOUT
constexpr int kHeadFactors = 20;             // (F+, Fx) (re, im) of (2,2), then the four
constexpr double kEtaEmr = 0.05;             // hm/variables.py:34
constexpr double kFalseZero = 1.0e-15;       // reference.py:64

// Offsets within a mode's table (MODE_LAYOUT).
enum ModeSlot : int {
  M_PHASE = 0,  // 3 x 18: inspiral, intermediate, ringdown rows over HM_BASIS
  M_SPH = 54,
  M_ATAN_A = 58,
  M_ATAN_W = 61,
  M_SHIFT = 64,
  M_F_PHASE_IN = 65,
  M_F_PHASE_IM = 66,
  M_F_AMP_IN = 67,
  M_F_AMP_IM = 68,
  M_PN_RE = 69,
  M_PN_IM = 76,
  M_PSEUDO = 83,
  M_INTER = 86,
  M_INTER_C = 94,
  M_INTER_H = 95,
  M_RD = 96,
  M_FALLOFF = 99,
  M_AUX = 102,
  M_F_AUX = 106,
  M_MIX = 107,
  M_ON = 111,
};

// HM_BASIS (core.py:64-67): f^a (log f)^l, in this order.
enum HmBasis : int {
  B_M3 = 0, B_M2, B_M4_3, B_M1, B_M2_3, B_M1_3, B_1, B_1_3, B_2_3, B_F, B_4_3, B_5_3, B_F2, B_7_3,
  B_LOG, B_1_3_LOG, B_F_LOG, B_4_3_LOG, kBasis
};

// The variables of one higher mode (hm/variables.py:100-169 for release
// 122022 with the QNM fits in 1 - a_final, reference.py:84-104).
template <class R>
struct Mode {
  int tag, ell, emm, mode_int;
  bool mixing;
  R f_ring, f_damp, f_meco_lm, chi_s, chi_a, delta_t, f_amp_rd_falloff;
  R mix[4][2];
};

template <class R>
inline WFX_HDI Mode<R> mode_struct(const xas::Internals<R>& w, int mode_int, R psi4tostrain) {
  Mode<R> hm;
  hm.mode_int = mode_int;
  hm.tag = mode_int == 0 ? 21 : (mode_int == 1 ? 33 : (mode_int == 2 ? 32 : 44));
  hm.ell = hm.tag / 10;
  hm.emm = hm.tag % 10;
  hm.mixing = hm.tag == 32;
  const R af = w.a_final;
  R fr = 0.0, fd = 0.0;
  switch (hm.tag) {
    case 21: fr = hmfit::fring21(af); fd = hmfit::fdamp21(af); break;
    case 33: fr = hmfit::fring33(af); fd = hmfit::fdamp33(af); break;
    case 32: fr = hmfit::fring32(af); fd = hmfit::fdamp32(af); break;
    default: fr = hmfit::fring44(af); fd = hmfit::fdamp44(af); break;
  }
  hm.f_ring = fr / w.m_final;
  hm.f_damp = fd / w.m_final;
  hm.f_meco_lm = w.f_meco * static_cast<double>(hm.emm) * 0.5;
  hm.chi_s = (w.chi1 + w.chi2) * 0.5;
  hm.chi_a = (w.chi1 - w.chi2) * 0.5;
  hm.delta_t = -2.0 * fit::PI * (500.0 + psi4tostrain);
  hm.f_amp_rd_falloff = 2.0 * hm.f_damp + hm.f_ring;
  for (int i = 0; i < 4; ++i) hm.mix[i][0] = hm.mix[i][1] = 0.0;
  if (hm.mixing) {
    hm.mix[0][0] = hmfit::re_l2m2lp2(af);
    hm.mix[0][1] = hmfit::im_l2m2lp2(af);
    hm.mix[1][0] = hmfit::re_l2m2lp3(af);
    hm.mix[1][1] = hmfit::im_l2m2lp3(af);
    hm.mix[2][0] = -hmfit::re_l3m2lp2(af);
    hm.mix[2][1] = -hmfit::im_l3m2lp2(af);
    hm.mix[3][0] = -hmfit::re_l3m2lp3(af);
    hm.mix[3][1] = -hmfit::im_l3m2lp3(af);
  }
  return hm;
}

// The arguments of the fits (hm_fit_code.h).
template <class R>
inline WFX_HDI hmfit::Args<R> fit_args(const xas::Internals<R>& w) {
  hmfit::Args<R> a;
  a.sq = w_sqrt(w.eta);
  a.delta = w.delta;
  a.r3 = w_sqrt(1.0 - 3.0 * w.eta);
  a.s = w.chi_pn_hat;
  a.dh = 0.5 * w.dchi;
  a.dc = w.dchi;
  a.st = w.s_tot_r;
  a.c1 = w.chi1;
  a.c2 = w.chi2;
  return a;
}

// ---------------------------------------------------------------------------
// The (2,2) phase and its derivative in Mf (phase22.py:289-326), from the
// Internals; `connected` false drops the C1/C2 connections
// (reference.py:441-443).

template <class R, class T>
inline WFX_HDI T ins_dphase22(const xas::Internals<R>& w, const Powers<T>& q) {
  const R d2 = 3.0 / 5.0 * w.phi2, d3 = 2.0 / 5.0 * w.phi3, d4 = 1.0 / 5.0 * w.phi4, d5 = -3.0 / 5.0 * w.phi5l;
  const R d6 = -(1.0 / 5.0) * w.phi6 - 3.0 / 5.0 * w.phi6l, d6l = -1.0 / 5.0 * w.phi6l, d7 = -2.0 / 5.0 * w.phi7;
  const R d8 = -(3.0 / 5.0) * w.phi8 - 3.0 / 5.0 * w.phi8l, d8l = -3.0 / 5.0 * w.phi8l;
  T x = 1.0 + d2 * q.two_thirds + d3 * q.itself + d4 * q.four_thirds + d5 * q.five_thirds + d6 * q.two +
        d6l * q.two * q.log_ + d7 * q.seven_thirds + d8 * q.eight_thirds + d8l * q.eight_thirds * q.log_;
  x = x + (w.a0 * q.eight_thirds + w.a1 * q.three + w.a2 * q.eight_thirds * q.two_thirds +
           w.a3 * q.eight_thirds * q.itself);
  return x * q.m_eight_thirds * (5.0 / (128.0 * fit::LALPI_FIVE_THIRDS));
}

template <class R, class T>
inline WFX_HDI T ins_phase22(const xas::Internals<R>& w, const Powers<T>& q) {
  const R phi_norm = -(3.0 * fit::LALPI_M_FIVE_THIRDS) / 128.0;
  T x = 1.0 + w.phi2 * q.two_thirds + w.phi3 * q.itself + w.phi4 * q.four_thirds + w.phi5l * q.five_thirds * q.log_ +
        w.phi6 * q.two + w.phi6l * q.two * q.log_ + w.phi7 * q.seven_thirds + w.phi8 * q.eight_thirds +
        w.phi8l * q.eight_thirds * q.log_;
  x = x + (w.sigma1 * q.eight_thirds + w.sigma2 * q.three + w.sigma3 * q.one_third * q.three +
           w.sigma4 * q.two_thirds * q.three);
  return x * phi_norm * q.m_five_thirds;
}

template <class R, class T>
inline WFX_HDI T dphase22(const xas::Internals<R>& w, const T& f, bool connected = true) {
  const Powers<T> q(f);
  if (value(f) < w.f_phase_in) return ins_dphase22(w, q);
  if (value(f) >= w.f_phase_im) {
    const T dfr = f - w.f_ring;
    return w.c0 + w.c1 * q.m_one_third + w.c2 * q.m_two + w.c4 * q.m_four + w.c_l / (w.f_damp * w.f_damp + dfr * dfr) +
           (connected ? w.c2_mrd : 0.0);
  }
  const T dfr = f - w.f_ring;
  return w.b0 + w.b1 * q.m_one + w.b2 * q.m_two + w.b3 * q.m_three + w.b4 * q.m_four +
         (4.0 * w.c_l) / (4.0 * w.f_damp * w.f_damp + dfr * dfr) + (connected ? w.c2_int : 0.0);
}

// The (2,2) ringdown amplitude ansatz (_generated/ringdown.py:55-61).
template <class R, class T>
inline WFX_HDI T amp22_ringdown(const xas::Internals<R>& w, const T& mf) {
  const R gamma_d13 = w.f_damp * w.gamma1 * w.gamma3;
  const R gamma_r = w.gamma2 / (w.gamma3 * w.f_damp);
  const R gamma_d2 = (w.f_damp * w.gamma3) * (w.f_damp * w.gamma3);
  const T dfr = mf - w.f_ring;
  return w_exp(-dfr * gamma_r) * gamma_d13 / (dfr * dfr + gamma_d2);
}

// The (2,2) phase at mf without its anchor from the (2,2) table in Hz
// (core.py:193-205): the table's rest plus, in the inspiral and with
// `leading`, T0 f^-5/3.
template <class R, class T>
inline WFX_HDI T rest22(const R* tab22, const T& mf, R m_sec, bool leading, bool& past) {
  const T f = mf / m_sec;
  T lf;
  T rest = xas::rest_at<T, R>(tab22, f, past, lf);
  if (leading && !past) rest = rest + tab22[X_T0] * w_exp(-5.0 / 3.0 * lf);
  return rest;
}

// ---------------------------------------------------------------------------
// The amplitude (reference.py:118-348).

template <class R>
struct Amp {
  R amp_norm, pn_dominant, f_rd_aux, f_amp_match_in, f_amp_match_im;
  R pn_re[7], pn_im[7], pn_global_factor;
  R fcut_7_3, fcut_8_3, fcut_3, ins[3];
  R rd[5], rd_aux[4];
  R inter[8], inter_center, inter_half;
  int n_inter;
};

// IMRPhenomXHM_GetPNAmplitudeCoefficients (hm/inspiral.py:45-216).
template <class R>
inline WFX_HDI void pn_amplitude(const xas::Internals<R>& w, const Mode<R>& hm, Amp<R>& amp) {
  const R chi_a = hm.chi_a, chi_s = hm.chi_s, eta = w.eta, delta = w.delta;
  const R pi = fit::PI;
  const R sqrt_5_7 = w_sqrt(5.0 / 7.0);
  const R prefactors[4] = {w_sqrt(2.0) / 3.0, 0.75 * sqrt_5_7, sqrt_5_7 / 3.0, 4.0 * w_sqrt(2.0) / 9.0 * sqrt_5_7};
  amp.pn_global_factor = w_pow(2.0 / hm.emm, -7.0 / 6.0) * prefactors[hm.mode_int];
  for (int k = 0; k < 7; ++k) amp.pn_re[k] = amp.pn_im[k] = 0.0;
  // the powers of the constant 2/m of the mode (hm/inspiral.py:30-41)
  const R base = hm.tag == 21 ? 2.0 : (hm.tag == 33 ? 2.0 / 3.0 : 0.5);
  const Powers<R> p2(base);
  if (hm.tag == 21) {
    R re = 3427.0 * chi_a;
    re = re + 3427.0 * chi_s * delta;
    re = re - 8404.0 * chi_a * eta;
    re = re - 3860.0 * chi_s * delta * eta;
    re = re - 1344.0 * delta * pi;
    R im = -(672.0 * delta);
    im = im - 672.0 * delta * w_log(16.0);
    R scale = fit::LALPI_FOUR_THIRDS * p2.four_thirds;
    amp.pn_re[4] = re / 1344.0 * scale;
    amp.pn_im[4] = im / 1344.0 * scale;
    re = 143063173.0 * chi_a;
    re = re + 143063173.0 * chi_s * delta;
    re = re - 546199608.0 * chi_a * eta;
    re = re - 169191096.0 * chi_s * delta * eta;
    re = re - 9898560.0 * delta * pi;
    re = re + 20176128.0 * delta * eta * pi;
    re = re + 61725888.0 * chi_s * delta * chi_a * chi_a;
    re = re - 81285120.0 * chi_s * delta * eta * chi_a * chi_a;
    re = re + 20575296.0 * w_pow(chi_a, 3.0);
    re = re - 81285120.0 * eta * w_pow(chi_a, 3.0);
    re = re + 61725888.0 * chi_a * chi_s * chi_s;
    re = re - 165618432.0 * chi_a * eta * chi_s * chi_s;
    re = re + 20575296.0 * delta * w_pow(chi_s, 3.0);
    re = re - 1016064.0 * delta * eta * chi_s * chi_s * chi_s;
    re = re + 128873808.0 * chi_a * eta * eta;
    re = re - 3859632.0 * chi_s * delta * eta * eta;
    im = -(1350720.0 * delta);
    im = im - 72043776.0 * delta * eta;
    im = im - 5402880.0 * delta * fit::LN_2;
    im = im - 17224704.0 * delta * eta * fit::LN_2;
    scale = fit::LALPI_TWO * p2.two;
    amp.pn_re[6] = re / 5.419008e6 * scale;
    amp.pn_im[6] = im / 5.419008e6 * scale;
    const R five = 21535920.0 * delta * eta * eta + (39626496.0 * delta * eta * chi_s * chi_s + (
        -(77982912.0 * delta * chi_s) * chi_s + (81285120.0 * delta * eta * chi_a * chi_a + (
            -(77982912.0 * delta * chi_a) * chi_a + (24385536.0 * chi_s * delta * pi + (
                24385536.0 * chi_a * pi + (-(23670792.0 * delta) * eta + (
                    432843264.0 * chi_a * chi_s * eta + (-155965824.0 * chi_a * chi_s - 964357.0 * delta)))))))));
    amp.pn_re[1] = delta * fit::LALPI_ONE_THIRD * p2.one_third;
    amp.pn_re[2] = -3.0 * (chi_s * delta + chi_a) / 2.0 * fit::LALPI_TWO_THIRDS * p2.two_thirds;
    amp.pn_re[3] = (335.0 * delta + 1404.0 * delta * eta) / 672.0 * pi * p2.itself;
    amp.pn_re[5] = five / 8.128512e6 * fit::LALPI_FIVE_THIRDS * p2.five_thirds;
  } else if (hm.tag == 33) {
    const R ln15 = w_log(1.5);
    R re = 325.0 * chi_a;
    re = re + 325.0 * chi_s * delta;
    re = re - 1120.0 * chi_a * eta;
    re = re - 80.0 * chi_s * delta * eta;
    re = re + 120.0 * delta * pi;
    R im = -(504.0 * delta);
    im = im + 720.0 * delta * ln15;
    R scale = fit::LALPI_FOUR_THIRDS * p2.four_thirds;
    amp.pn_re[4] = re / 120.0 * scale;
    amp.pn_im[4] = im / 120.0 * scale;
    re = 22007835.0 * chi_a;
    re = re + 22007835.0 * chi_s * delta;
    re = re - 80190540.0 * chi_a * eta;
    re = re - 31722300.0 * chi_s * delta * eta;
    re = re - 9193500.0 * delta * pi;
    re = re + 17826480.0 * delta * eta * pi;
    re = re - 12428640.0 * chi_a * eta * eta;
    re = re - 6078240.0 * chi_s * delta * eta * eta;
    im = 26467560.0 * delta;
    im = im - 98774368.0 * delta * eta;
    im = im - 37810800.0 * delta * ln15;
    im = im + 37558080.0 * delta * eta * ln15;
    scale = fit::LALPI_TWO * p2.two;
    amp.pn_re[6] = re / 2.17728e6 * scale;
    amp.pn_im[6] = im / 2.17728e6 * scale;
    const R five = 2966264784.0 * delta * eta * eta + (55883520.0 * delta * eta * chi_s * chi_s + (
        -(1131641280.0 * delta * chi_s) * chi_s + (4470681600.0 * delta * eta * chi_a * chi_a + (
            -(1131641280.0 * delta * chi_a) * chi_a + (-(5926068792.0 * delta) * eta + (
                9053130240.0 * chi_a * chi_s * eta + (-2263282560.0 * chi_a * chi_s - 1077664867.0 * delta)))))));
    amp.pn_re[1] = delta * fit::LALPI_ONE_THIRD * p2.one_third;
    amp.pn_re[3] = (-1945.0 * delta + 2268.0 * delta * eta) / 672.0 * pi * p2.itself;
    amp.pn_re[5] = five / 4.4706816e8 * fit::LALPI_FIVE_THIRDS * p2.five_thirds;
  } else if (hm.tag == 32) {
    R re = 0.0 - 3955.0 * chi_s;
    re = re - 3955.0 * chi_a * delta;
    re = re + 10810.0 * chi_s * eta;
    re = re + 11865.0 * chi_a * delta * eta;
    re = re - 12600.0 * chi_s * eta * eta;
    R im = 2520.0;
    im = im - 11088.0 * eta;
    const R scale = fit::LALPI_FIVE_THIRDS;
    amp.pn_re[5] = re / 840.0 * scale;
    amp.pn_im[5] = im / 840.0 * scale;
    const R six = 5907445488.0 * w_pow(eta, 3.0) + (5830513920.0 * chi_s * chi_s * eta * eta + (
        13412044800.0 * chi_a * chi_a * eta * eta + (-(13202119896.0 * eta) * eta + (
            -(11870591040.0 * eta * chi_s) * chi_s + (1131641280.0 * chi_s * chi_s + (
                -(7865605440.0 * eta * chi_a) * chi_a + (1131641280.0 * chi_a * chi_a + (
                    3576545280.0 * chi_s * eta * pi + (-(15209631360.0 * chi_a * chi_s * delta) * eta + (
                        -26069649.0 * eta + (2263282560.0 * chi_a * chi_s * delta + 824173699.0)))))))))));
    amp.pn_re[2] = (3.0 * eta - 1.0) * fit::LALPI_TWO_THIRDS;
    amp.pn_re[3] = -4.0 * chi_s * eta * pi;
    amp.pn_re[4] = (82460.0 * eta * eta + (-61625.0 * eta + 10471.0)) / 10080.0 * fit::LALPI_FOUR_THIRDS;
    amp.pn_re[6] = six / 4.4706816e8 * fit::LALPI_TWO;
  } else {
    R re = -0.0 + 565.0 * chi_s;
    re = re + 565.0 * chi_a * delta;
    re = re - 2075.0 * chi_s * eta;
    re = re - 1695.0 * chi_a * delta * eta;
    re = re + 240.0 * pi;
    re = re - 720.0 * eta * pi;
    re = re + 1140.0 * chi_s * eta * eta;
    R im = -1008.0;
    im = im + 3579.0 * eta;
    im = im + 960.0 * fit::LN_2;
    im = im - 2880.0 * eta * fit::LN_2;
    const R scale = fit::LALPI_FIVE_THIRDS * p2.five_thirds;
    amp.pn_re[5] = re / 120.0 * scale;
    amp.pn_im[5] = im / 120.0 * scale;
    const R six = -805075876080.0 * w_pow(eta, 3.0) + (-(10897286400.0 * chi_s * chi_s * eta) * eta + (
        -(871782912000.0 * chi_a * chi_a * eta) * eta + (2271682065240.0 * eta * eta + (
            224302478400.0 * eta * chi_s * chi_s + (-(73556683200.0 * chi_s) * chi_s + (
                511264353600.0 * eta * chi_a * chi_a + (-(73556683200.0 * chi_a) * chi_a + (
                    441340099200.0 * chi_a * chi_s * delta * eta + (-745140957231.0 * eta + (
                        -(147113366400.0 * chi_a * chi_s) * delta + 7888301437.0))))))))));
    amp.pn_re[2] = (-3.0 * eta + 1.0) * fit::LALPI_TWO_THIRDS * p2.two_thirds;
    amp.pn_re[4] = (-(446460.0 * eta) * eta + (641105.0 * eta - 158383.0)) / 36960.0 * fit::LALPI_FOUR_THIRDS *
                   p2.four_thirds;
    amp.pn_re[6] = six / 2.90594304e10 * fit::LALPI_TWO * p2.two;
  }
}

// The PN amplitude times pnGlobalFactor ampNorm f^-7/6 (reference.py:152-162).
template <class R, class T>
inline WFX_HDI T pn_amp_ansatz(const Powers<T>& p, const Amp<R>& amp) {
  const T terms[6] = {p.one_third, p.two_thirds, p.itself, p.four_thirds, p.five_thirds, p.two};
  T re(amp.pn_re[0]), im(amp.pn_im[0]);
  for (int k = 0; k < 6; ++k) {
    re = re + terms[k] * amp.pn_re[k + 1];
    im = im + terms[k] * amp.pn_im[k + 1];
  }
  return w_hypot(re, im) * (amp.pn_global_factor * p.m_seven_sixths * amp.amp_norm);
}

// PN plus pseudo-PN terms (reference.py:165-172).
template <class R, class T>
inline WFX_HDI T inspiral_amp_ansatz(const Powers<T>& p, const Amp<R>& amp) {
  T pseudo = p.seven_thirds / amp.fcut_7_3 * amp.ins[0] + p.eight_thirds / amp.fcut_8_3 * amp.ins[1];
  pseudo = p.three / amp.fcut_3 * amp.ins[2] + pseudo;
  return pn_amp_ansatz(p, amp) + pseudo * p.m_seven_sixths * amp.pn_dominant;
}

// The Lorentzian of the ringdown amplitude and its derivative
// (reference.py:195-214).
template <class R, class T>
inline WFX_HDI T lorentzian(const T& mf, const Mode<R>& hm, const R* rd) {
  const R fda = hm.f_damp;
  const T dfr = mf - hm.f_ring;
  const R dfd = fda * rd[2];
  return rd[0] * fda / (w_exp(rd[1] / dfd * dfr) * (dfr * dfr + dfd * dfd));
}

template <class R>
inline WFX_HDI R rd_amp_dansatz(R mf, const Mode<R>& hm, const R* rd) {
  const R fda = hm.f_damp;
  const R dfr = mf - hm.f_ring;
  const R numerator = rd[0] * (fda * fda * rd[1] * rd[2] * rd[2] + (dfr * dfr * rd[1] + 2.0 * fda * dfr * rd[2]));
  R denom = dfr * dfr + fda * fda * rd[2] * rd[2];
  denom = rd[2] * denom * denom * w_exp(dfr * rd[1] / (fda * rd[2]));
  return -numerator / denom;
}

// The ringdown amplitude ansatz: the Lorentzian, the cubic of the (3,2)
// below fRDAux, the fall-off above fAmpRDfalloff (reference.py:217-229).
template <class R, class T>
inline WFX_HDI T rd_amp_ansatz(const T& mf, const Mode<R>& hm, const Amp<R>& amp) {
  T out = value(mf) >= hm.f_amp_rd_falloff ? amp.rd[3] * w_exp(-amp.rd[4] * (mf - hm.f_amp_rd_falloff))
                                            : lorentzian(mf, hm, amp.rd);
  if (hm.mixing && value(mf) < amp.f_rd_aux) {
    const R* a = amp.rd_aux;
    out = ((a[3] * mf + a[2]) * mf + a[1]) * mf + a[0];
  }
  return out;
}

// The spheroidal ringdown phase of the (3,2) (core.py:208-234).
template <class R>
struct Spheroidal {
  R alpha0_s, alpha_l_s, alpha2_s, alpha4_s, phi0_s;
};

// The ringdown phase derivative and phase (hm/phase.py:58-82), the
// rescaled (2,2) ringdown or, for the (3,2), the spheroidal ansatz.
template <class R>
struct RdPhase {
  R alpha0, alpha2, alpha_l;
};

template <class R, class T>
inline WFX_HDI T rd_dphase(const T& ff, const Powers<T>& p, const Mode<R>& hm, const RdPhase<R>& ph, const Spheroidal<R>& sp) {
  const R frd = hm.f_ring, fda = hm.f_damp;
  const T den = fda * fda + (ff - frd) * (ff - frd);
  if (!hm.mixing) return frd * frd * ph.alpha2 * p.m_two + ph.alpha0 + (ph.alpha_l * fda) / den;
  const T d = sp.alpha2_s * p.m_two + sp.alpha0_s;
  return sp.alpha4_s * p.m_four + d + (sp.alpha_l_s * fda) / den;
}

template <class R, class T>
inline WFX_HDI T rd_phase(const T& ff, const Powers<T>& p, const Mode<R>& hm, const RdPhase<R>& ph, const Spheroidal<R>& sp) {
  const R frd = hm.f_ring, fda = hm.f_damp;
  const T arctan = w_atan((ff - frd) / fda);
  if (!hm.mixing) {
    const T phase_rd = ph.alpha0 * ff + (-(frd * frd * ph.alpha2 * p.m_one));
    return ph.alpha_l * arctan + phase_rd;
  }
  T phase_rd = sp.alpha0_s * ff + sp.phi0_s;
  phase_rd = -sp.alpha2_s * p.m_one + phase_rd;
  phase_rd = -(1.0 / 3.0 * sp.alpha4_s) * p.m_three + phase_rd;
  return sp.alpha_l_s * arctan + phase_rd;
}

// The data of the rotation of the (3,2) ringdown (core.py:250-262,
// reference.py:354-367): the (2,2) whose ringdown it recycles.
template <class R>
struct Rotation {
  const xas::Internals<R>* w;
  const R* tab22;
  const Mode<R>* hm;
  const Amp<R>* amp;
  Spheroidal<R> sp;
};

// conj(a322) h22 + conj(a323) h32_spheroidal as (re, im), the (2,2) ringdown
// ansatz rescaled by its leading order with the phase of the (2,2) without
// its anchor.
template <class R, class T>
inline WFX_HDI void rotated(const Rotation<R>& r, const T& mf, T& re, T& im) {
  const xas::Internals<R>& w = *r.w;
  const Powers<T> p(mf);
  const T a22 = amp22_ringdown(w, mf) * w.amp_norm * p.m_seven_sixths;
  bool past;
  const T phi22 = rest22(r.tab22, mf, w.m_sec, true, past);
  const T c22 = a22 * w_cos(phi22), s22 = a22 * w_sin(phi22);
  const T amplm = rd_amp_ansatz(mf, *r.hm, *r.amp);
  const RdPhase<R> none{0.0, 0.0, 0.0};
  const T philm = rd_phase(mf, p, *r.hm, none, r.sp);
  const R m2r = r.hm->mix[2][0], m2i = r.hm->mix[2][1], m3r = r.hm->mix[3][0], m3i = r.hm->mix[3][1];
  const T a_re = c22 * m2r + s22 * m2i;
  const T a_im = s22 * m2r - c22 * m2i;
  const T b_re = amplm * m3r;
  const T b_im = -(m3i * amplm);
  const T c = w_cos(philm), s = w_sin(philm);
  re = a_re + (b_re * c - b_im * s);
  im = a_im + (b_re * s + b_im * c);
}

template <int N, class R>
inline WFX_HDI bool solve_n(R (&a)[N][N], R (&b)[N]) {
  return solve<R, N>(a, b);
}

// IMRPhenomXHM_GetAmplitudeCoefficients (reference.py:337-348).
template <class R>
inline WFX_HDI bool amplitude_coefficients(const xas::Internals<R>& w, const hmfit::Args<R>& fa, const Mode<R>& hm,
                                    Rotation<R>& rot, Amp<R>& amp) {
  using F1 = typename Deriv<R>::F1;
  bool ok = true;
  amp.amp_norm = w.amp_norm;
  amp.pn_dominant = w.amp_norm * w_pow(2.0 / hm.emm, -7.0 / 6.0);
  amp.f_rd_aux = hm.mixing ? hm.f_ring - hm.f_damp : 0.0;
  // fcut of the inspiral (reference.py:118-140) and of the ringdown (:143-147)
  {
    const R emm = static_cast<double>(hm.emm), eta = w.eta, chi1 = w.chi1;
    const R fcut_emr = 1.25 * emm *
                            ((0.000316707064291237 * chi1 * chi1 + (-0.0000858396080377194 * chi1 + 0.011671068725758493)) *
                             (6.2873167352395125 * eta + 0.8447212540381764)) /
                            (-0.9977728883419751 * chi1 + 1.2857082764038923);
    const R funcs = 0.5 * w_tanh((eta - 0.0192234) / 0.004) + 0.5;
    amp.f_amp_match_in = w.q < 20.0 ? hm.f_meco_lm : funcs * hm.f_meco_lm + (1.0 - funcs) * fcut_emr;
  }
  amp.f_amp_match_im = hm.mixing ? -0.5 * w.f_damp + w.f_ring : hm.f_ring - hm.f_damp;
  pn_amplitude(w, hm, amp);
  // the inspiral: three collocation points of the pseudo-PN terms
  // (reference.py:175-190; the constant system solved here)
  {
    const R fcut = amp.f_amp_match_in;
    const Powers<R> fin(fcut);
    amp.fcut_7_3 = fin.seven_thirds;
    amp.fcut_8_3 = fin.eight_thirds;
    amp.fcut_3 = fin.three;
    const R g[3] = {0.5, 0.75, 1.0};
    R values[3];
    switch (hm.tag) {
      case 21: values[0] = hmfit::amp_21_iv1(fa); values[1] = hmfit::amp_21_iv2(fa); values[2] = hmfit::amp_21_iv3(fa); break;
      case 33: values[0] = hmfit::amp_33_iv1(fa); values[1] = hmfit::amp_33_iv2(fa); values[2] = hmfit::amp_33_iv3(fa); break;
      case 32: values[0] = hmfit::amp_32_iv1(fa); values[1] = hmfit::amp_32_iv2(fa); values[2] = hmfit::amp_32_iv3(fa); break;
      default: values[0] = hmfit::amp_44_iv1(fa); values[1] = hmfit::amp_44_iv2(fa); values[2] = hmfit::amp_44_iv3(fa); break;
    }
    R a[3][3], b[3];
    for (int i = 0; i < 3; ++i) {
      const Powers<R> fi(g[i] * fcut);
      const R pn = pn_amp_ansatz(fi, amp);
      b[i] = (w_abs(values[i]) - pn) / amp.pn_dominant / fi.m_seven_sixths;
      a[i][0] = w_pow(g[i], 7.0 / 3.0);
      a[i][1] = w_pow(g[i], 8.0 / 3.0);
      a[i][2] = w_pow(g[i], 3.0);
    }
    ok = solve_n<3>(a, b) && ok;
    amp.ins[0] = b[0];
    amp.ins[1] = b[1];
    amp.ins[2] = b[2];
  }
  // the ringdown (reference.py:232-264)
  {
    const R fdamp = hm.f_damp;
    R rd[3];
    if (hm.tag == 32) {
      rd[0] = w_abs(hmfit::amp_32_alambda(fa));
      rd[1] = hmfit::amp_32_lambda(fa);
      rd[2] = hmfit::amp_32_sigma(fa);
    } else {
      R c1, c2, c3;
      if (hm.tag == 21) {
        c1 = hmfit::amp_21_rdcp1(fa); c2 = hmfit::amp_21_rdcp2(fa); c3 = hmfit::amp_21_rdcp3(fa);
      } else if (hm.tag == 33) {
        c1 = hmfit::amp_33_rdcp1(fa); c2 = hmfit::amp_33_rdcp2(fa); c3 = hmfit::amp_33_rdcp3(fa);
      } else {
        c1 = hmfit::amp_44_rdcp1(fa); c2 = hmfit::amp_44_rdcp2(fa); c3 = hmfit::amp_44_rdcp3(fa);
      }
      c1 = w_abs(c1);
      c2 = w_abs(c2);
      c3 = w_abs(c3);
      // the vetoes
      if (c3 >= c2 * c2 / c1) c3 = 0.5 * c2 * c2 / c1;
      if (c3 > c2) c3 = 0.5 * c2;
      if (c1 < c2 && c3 > c1) c3 = c1;
      R deno = w_sqrt(c1 / c3) - c1 / c2;
      if (deno <= 0.0) deno = 1e-16;
      const R a_lambda = c1 * fdamp / deno;
      const R sigma = w_sqrt(a_lambda / (c2 * fdamp));
      rd[0] = a_lambda;
      rd[1] = 0.5 * sigma * w_log(c1 / c3);
      rd[2] = sigma;
    }
    const R falloff = hm.f_amp_rd_falloff;
    const R v = lorentzian(falloff, hm, rd);
    amp.rd[0] = rd[0];
    amp.rd[1] = rd[1];
    amp.rd[2] = rd[2];
    amp.rd[3] = v;
    amp.rd[4] = -1.0 * rd_amp_dansatz(falloff, hm, rd) / v;
    for (int j = 0; j < 4; ++j) amp.rd_aux[j] = 0.0;
    if (hm.mixing) {
      const R faux = amp.f_rd_aux, fim = amp.f_amp_match_im;
      R b[4] = {w_abs(hmfit::amp_32_rdaux1(fa)), w_abs(hmfit::amp_32_rdaux2(fa)), lorentzian(faux, hm, amp.rd),
                     rd_amp_dansatz(faux, hm, amp.rd)};
      const R freqs[3] = {fim, 0.5 * (fim + faux), faux};
      R a[4][4];
      for (int i = 0; i < 3; ++i) {
        const R f = freqs[i];
        a[i][0] = 1.0;
        a[i][1] = f;
        a[i][2] = f * f;
        a[i][3] = f * f * f;
      }
      a[3][0] = 0.0;
      a[3][1] = 1.0;
      a[3][2] = 2.0 * faux;
      a[3][3] = 3.0 * faux * faux;
      ok = solve_n<4>(a, b) && ok;
      for (int j = 0; j < 4; ++j) amp.rd_aux[j] = b[j];
    }
  }
  // the intermediate: a polynomial in u = (f - f_c) / f_h times f^-7/6
  // through equispaced collocation points (reference.py:267-322)
  {
    const int version21[6] = {1, 1, 0, 1, 0, 2};
    const int version_other[6] = {2, 1, 1, 1, 1, 2};
    const int* version = hm.tag == 21 ? version21 : version_other;
    const R f_in = amp.f_amp_match_in, f_rd = amp.f_amp_match_im;
    const R deltaf = (f_rd - f_in) / 5.0;
    const R center = 0.5 * (f_rd + f_in), half = 0.5 * (f_rd - f_in);
    amp.inter_center = center;
    amp.inter_half = half;
    const int n = hm.tag == 21 ? 5 : 8;
    amp.n_inter = n;
    const F1 ins = inspiral_amp_ansatz(Powers<F1>(F1(f_in, 1.0)), amp);
    R rd_value, rd_derivative;
    if (hm.mixing) {
      F1 re, im;
      rotated(rot, F1(f_rd, 1.0), re, im);
      const F1 h = w_hypot(re, im);
      rd_value = h.v;
      rd_derivative = h.d;
    } else {
      rd_value = rd_amp_ansatz(f_rd, hm, amp);
      rd_derivative = rd_amp_dansatz(f_rd, hm, amp.rd);
    }
    R fits_int[4];
    switch (hm.tag) {
      case 21: fits_int[0] = hmfit::amp_21_int1(fa); fits_int[1] = hmfit::amp_21_int2(fa);
               fits_int[2] = hmfit::amp_21_int3(fa); fits_int[3] = hmfit::amp_21_int4(fa); break;
      case 33: fits_int[0] = hmfit::amp_33_int1(fa); fits_int[1] = hmfit::amp_33_int2(fa);
               fits_int[2] = hmfit::amp_33_int3(fa); fits_int[3] = hmfit::amp_33_int4(fa); break;
      case 32: fits_int[0] = hmfit::amp_32_int1(fa); fits_int[1] = hmfit::amp_32_int2(fa);
               fits_int[2] = hmfit::amp_32_int3(fa); fits_int[3] = hmfit::amp_32_int4(fa); break;
      default: fits_int[0] = hmfit::amp_44_int1(fa); fits_int[1] = hmfit::amp_44_int2(fa);
               fits_int[2] = hmfit::amp_44_int3(fa); fits_int[3] = hmfit::amp_44_int4(fa); break;
    }
    R a[8][8], b[8];
    for (int i = 0; i < 8; ++i) {
      b[i] = 0.0;
      for (int j = 0; j < 8; ++j) a[i][j] = i == j ? 1.0 : 0.0;  // (unused rows of the 5-point system)
    }
    int row = 0;
    auto value_row = [&](R f) {
      const R m76 = w_pow(f, -7.0 / 6.0);
      const R u = (f - center) / half;
      R uj = 1.0;
      for (int j = 0; j < n; ++j) {
        a[row][j] = m76 * uj;
        uj = uj * u;
      }
    };
    auto derivative_row = [&](R f) {
      const R m76 = w_pow(f, -7.0 / 6.0);
      const R u = (f - center) / half;
      R uj = 1.0, ujm1 = 0.0;
      for (int j = 0; j < n; ++j) {
        a[row][j] = m76 * (-(7.0 / 6.0) / f * uj + (j ? j * ujm1 / half : 0.0));
        ujm1 = uj;
        uj = uj * u;
      }
    };
    for (int i = 0; i < 6; ++i) {
      const R f = deltaf * static_cast<double>(i) + f_in;
      const int digit = version[i];
      if (digit == 0) continue;
      if (i == 0) {
        value_row(f);
        b[row++] = ins.v;
        if (digit == 2) {
          derivative_row(f);
          b[row++] = ins.d;
        }
      } else if (i == 5) {
        value_row(f);
        b[row++] = rd_value;
        if (digit == 2) {
          derivative_row(f);
          b[row++] = rd_derivative;
        }
      } else {
        value_row(f);
        b[row++] = w_abs(fits_int[i - 1]);
      }
    }
    if (n == 5) {
      R a5[5][5], b5[5];
      for (int i = 0; i < 5; ++i) {
        b5[i] = b[i];
        for (int j = 0; j < 5; ++j) a5[i][j] = a[i][j];
      }
      ok = solve_n<5>(a5, b5) && ok;
      for (int j = 0; j < 8; ++j) amp.inter[j] = j < 5 ? b5[j] : 0.0;
    } else {
      ok = solve_n<8>(a, b) && ok;
      for (int j = 0; j < 8; ++j) amp.inter[j] = b[j];
    }
  }
  return ok;
}

// ---------------------------------------------------------------------------
// The phase (reference.py:372-560, hm/phase.py:85-113, hm/inspiral.py:331-361).

template <class R>
struct Phase {
  R phi[13], phi_l[13];
  RdPhase<R> rd;
  R c0, c1, c2, c3, c4, c_l;
  R c1_insp, c_insp, c1_rd, c_rd;
  R f_phase_match_in, f_phase_match_im;
};

template <class R, class T>
inline WFX_HDI T ins_phase_int(const T& mf, const Powers<T>& p, const Phase<R>& ph, bool leading = true) {
  const T freqs[13] = {p.m_five_thirds, p.m_four_thirds, p.m_one, p.m_two_thirds, p.m_one_third, T(1.0),
                       p.one_third, p.two_thirds, mf, p.four_thirds, p.five_thirds, p.two, p.seven_thirds};
  const T log_mf = p.log_;
  T philm(0.0);
  for (int i = leading ? 0 : 1; i < 13; ++i) philm = (ph.phi_l[i] * log_mf + ph.phi[i]) * freqs[i] + philm;
  return philm;
}

template <class R, class T>
inline WFX_HDI T ins_dphase(const T& mf, const Powers<T>& p, const Phase<R>& ph) {
  const R coeffs[13] = {-5.0 / 3.0, -4.0 / 3.0, -1.0, -2.0 / 3.0, -1.0 / 3.0, 0.0, 1.0 / 3.0, 2.0 / 3.0, 1.0,
                             4.0 / 3.0, 5.0 / 3.0, 2.0, 7.0 / 3.0};
  const T freqs[13] = {p.m_eight_thirds, p.m_seven_thirds, p.m_two, p.m_five_thirds, p.m_four_thirds, p.m_one,
                       p.m_two_thirds, p.m_one_third, T(1.0), p.one_third, p.two_thirds, mf, p.four_thirds};
  const T log_mf = p.log_;
  T d(0.0);
  for (int i = 0; i < 13; ++i) {
    const T coefficient = ph.phi_l[i] * log_mf + ph.phi[i];
    d = (coefficient * coeffs[i] + ph.phi_l[i]) * freqs[i] + d;
  }
  return d;
}

template <class R, class T>
inline WFX_HDI T int_dphase(const T& ff, const Powers<T>& p, const Mode<R>& hm, const Phase<R>& ph) {
  const R fda = hm.f_damp, frd = hm.f_ring;
  const T lor = (ph.c_l * fda) / (fda * fda + (ff - frd) * (ff - frd));
  T d = ph.c1 * p.m_one + ph.c0;
  d = ph.c2 * p.m_two + d;
  d = ph.c4 * p.m_four + d;
  if (hm.mixing) d = ph.c3 * p.m_three + d;
  return d + lor;
}

template <class R, class T>
inline WFX_HDI T int_phase(const T& ff, const Powers<T>& p, const Mode<R>& hm, const Phase<R>& ph) {
  const R fda = hm.f_damp, frd = hm.f_ring;
  T x = ph.c0 * ff + ph.c1 * p.log_;
  x = -ph.c2 * p.m_one + x;
  x = -(1.0 / 3.0 * ph.c4) * p.m_three + x;
  if (hm.mixing) x = -(0.5 * ph.c3) * p.m_two + x;
  return ph.c_l * w_atan((ff - frd) / fda) + x;
}

template <class R>
inline WFX_HDI R phase_fit(const hmfit::Args<R>& fa, int tag, int i) {
#define WFX_PF(t)                                                                                        \
  case t:                                                                                                \
    switch (i) {                                                                                         \
      case 0: return hmfit::phase_##t##_p1(fa);                                                         \
      case 1: return hmfit::phase_##t##_p2(fa);                                                         \
      case 2: return hmfit::phase_##t##_p3(fa);                                                         \
      case 3: return hmfit::phase_##t##_p4(fa);                                                         \
      case 4: return hmfit::phase_##t##_p5(fa);                                                         \
      default: return hmfit::phase_##t##_p6(fa);                                                        \
    }
  switch (tag) {
    WFX_PF(21)
    WFX_PF(33)
    WFX_PF(32)
    WFX_PF(44)
  }
#undef WFX_PF
  return NAN;
}

// IMRPhenomXHM_Insp_Phase_LambdaPN (_generated/hm_inspiral.py:26-42) or the
// extreme-mass-ratio fit.
template <class R>
inline WFX_HDI R lambda_pn(const hmfit::Args<R>& fa, R eta, int tag) {
  if (eta > 0.01) {
    const R pi = fit::PI;
    R out = 0.0;
    if (tag == 21) out = 2.0 * pi * (-2.0 * fit::LN_2 - 0.5);
    else if (tag == 33) out = 2.0 / 3.0 * pi * (6.0 * w_log(1.5) + -21.0 / 5.0);
    else if (tag == 32) out = -((2376.0 * pi * (22.0 * eta - 5.0)) / (11880.0 * eta - 3960.0));
    else out = 45045.0 * pi * (320.0 * (3.0 * eta - 1.0) * fit::LN_2 + (-1193.0 * eta + 336.0)) /
               (2.0 * (5405400.0 * eta - 1801800.0));
    return -out;
  }
  switch (tag) {
    case 21: return hmfit::phase_21_lambda(fa);
    case 33: return hmfit::phase_33_lambda(fa);
    case 32: return hmfit::phase_32_lambda(fa);
    default: return hmfit::phase_44_lambda(fa);
  }
}

// IMRPhenomXHM_PN21AmpSign (hm/phase.py:214-227).
template <class R>
inline WFX_HDI bool pn21_amp_sign(R ff, const xas::Internals<R>& w) {
  const R eta = w.eta, chi1 = w.chi1, chi2 = w.chi2;
  const R delta = w_sqrt(-4.0 * eta + 1.0);
  const R sqrt5 = w_sqrt(5.0);
  const R pi = fit::PI;
  R out = (-16.0 * delta * eta * ff * w_pow(pi, 1.5)) / (3.0 * sqrt5);
  out = out + (4.0 * w_pow(2.0, 0.3333333333333333) * (chi1 - chi2 + delta * (chi1 + chi2)) * eta *
               w_pow(ff, 1.3333333333333333) * w_pow(pi, 1.8333333333333333)) / sqrt5;
  out = out + (2.0 * w_pow(2.0, 0.6666666666666666) * eta * (306.0 * delta - 360.0 * delta * eta) *
               w_pow(ff, 1.6666666666666667) * w_pow(pi, 2.1666666666666665)) / (189.0 * sqrt5);
  return out >= 0.0;
}

template <class R>
inline WFX_HDI bool phase_coefficients(const xas::Internals<R>& w, const hmfit::Args<R>& fa, const Mode<R>& hm,
                                Rotation<R>& rot, Phase<R>& ph) {
  using J2 = typename Deriv<R>::J2;
  bool ok = true;
  const int tag = hm.tag, emm = hm.emm;
  const R eta = w.eta, eta_m1 = 1.0 / eta, fring = hm.f_ring, fdamp = hm.f_damp;
  const R fcut = (0.001 * (0.25 / eta - 1.0) + 1.0) * (emm * 1.0) * 0.5 * w.f_meco;
  const R sqrt3 = w_sqrt(3.0);
  R freqs[6];
  if (tag == 32) {
    const R f_end = -0.5 * w.f_damp + w.f_ring;
    freqs[0] = fcut;
    freqs[1] = (sqrt3 * (fcut - f_end) + 2.0 * (fcut + f_end)) / 4.0;
    freqs[2] = (3.0 * fcut + f_end) / 4.0;
    freqs[3] = (fcut + f_end) / 2.0;
    freqs[4] = f_end;
    freqs[5] = f_end;
    ph.f_phase_match_im = (eta < 0.01 && w.chi1 < 0.0) ? f_end * (-0.25 * w.chi1 + 1.2) : f_end;
  } else {
    freqs[0] = fcut;
    freqs[1] = (sqrt3 * (fcut - fring) + 2.0 * (fcut + fring)) / 4.0;
    freqs[2] = (3.0 * fcut + fring) / 4.0;
    freqs[3] = (fcut + fring) / 2.0;
    freqs[4] = (3.0 * fring + fcut) / 4.0;
    freqs[5] = (7.0 * fring + fcut) / 8.0;
    ph.f_phase_match_im = fring - fdamp;
  }
  ph.f_phase_match_in = hm.f_meco_lm;
  R values[6];
  for (int i = 0; i < 6; ++i) values[i] = phase_fit(fa, tag, i) + hm.delta_t;
  const R fcut_rd = ph.f_phase_match_im, fcut_insp = ph.f_phase_match_in;

  // the inspiral: the (2,2) coefficients rescaled (reference.py:419-436)
  {
    const R non_log[13] = {1.0, 0.0, w.phi2, w.phi3, w.phi4, 0.0, w.phi6, w.phi7, w.phi8, 0.0, 0.0, 0.0, 0.0};
    const R log_terms[13] = {0.0, 0.0, 0.0, 0.0, 0.0, w.phi5l, w.phi6l, 0.0, w.phi8l, 0.0, 0.0, 0.0, 0.0};
    const R pseudo_pn[13] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, w.sigma1, w.sigma2, w.sigma3, w.sigma4, 0.0};
    const R m_over_2 = emm * 0.5;
    const R phi_norm = -(3.0 * fit::LALPI_M_FIVE_THIRDS) / 128.0;
    const R fact = phi_norm / eta;
    const R log_m_over_2 = w_log(m_over_2);
    for (int i = 0; i < 13; ++i) {
      const R nl = non_log[i] * fact, lg = log_terms[i] * fact, ps = pseudo_pn[i] * fact;
      const R scale = w_pow(m_over_2, (8 - i) / 3.0);
      ph.phi[i] = (-lg * log_m_over_2 + (nl + ps)) * scale;
      ph.phi_l[i] = lg * scale;
    }
    ph.phi[8] = ph.phi[8] + lambda_pn(fa, eta, tag);
  }
  ph.rd = RdPhase<R>{0.0, 0.0, 0.0};
  ph.c0 = ph.c1 = ph.c2 = ph.c3 = ph.c4 = ph.c_l = 0.0;

  // the (2,1) inspiral extends into the intermediate region for high spins
  if (tag == 21) {
    const R two_over_m = 2.0 / emm;
    R v[3];
    for (int i = 0; i < 3; ++i) v[i] = 1.0 / eta * dphase22(w, two_over_m * freqs[i], false);
    const R diff12 = v[0] - v[1], diff23 = v[1] - v[2];
    if (w.s_tot_r >= 0.8) {
      const R v1 = values[2] + diff23;
      values[1] = v1;
      values[0] = v1 + diff12;
    }
  }
  auto lor = [&](R ff) { return fdamp / (fdamp * fdamp + (ff - fring) * (ff - fring)); };
  R phi0_rd, dphi0_rd;
  const Spheroidal<R>& sp = rot.sp;
  if (tag != 32) {
    bool cond_a = eta < kEtaEmr;
    if (emm == hm.ell) cond_a = cond_a || (w.s_tot_r >= 0.8);
    if (tag == 33) cond_a = cond_a || (w.s_tot_r < 0.0);
    const bool cond_b = tag == 21 ? (w.s_tot_r >= 0.8) : false;
    const int idx2 = cond_a ? 3 : 2;
    const int idx3 = cond_a ? 4 : (cond_b ? 4 : 3);
    const int chosen[5] = {0, 1, idx2, idx3, 5};
    const R wlm = emm == hm.ell ? 2.0 : emm / 3.0;
    const R alpha2_fit = hmfit::rd_phase_22_alpha2(fa), alpha_l_fit = hmfit::rd_phase_22_alpha_l(fa);
    ph.rd.alpha2 = 1.0 / (fring * fring) * wlm * alpha2_fit;
    ph.rd.alpha_l = eta_m1 * alpha_l_fit;
    const Powers<R> p_rd(fcut_rd);
    phi0_rd = rd_phase(fcut_rd, p_rd, hm, ph.rd, sp);
    dphi0_rd = rd_dphase(fcut_rd, p_rd, hm, ph.rd, sp);
    R a[5][5], b[5];
    for (int i = 0; i < 5; ++i) {
      const R ff = freqs[chosen[i]];
      const R ffm1 = 1.0 / ff, ffm2 = ffm1 * ffm1;
      a[i][0] = 1.0;
      a[i][1] = lor(ff);
      a[i][2] = ffm1;
      a[i][3] = ffm2;
      a[i][4] = ffm2 * ffm2;
      b[i] = values[chosen[i]];
    }
    ok = solve_n<5>(a, b) && ok;
    ph.c0 = b[0];
    ph.c_l = b[1];
    ph.c1 = b[2];
    ph.c2 = b[3];
    ph.c4 = b[4];
  } else {
    const J2 z0(fcut_rd, 1.0, 0.0);
    J2 re, im;
    rotated(rot, z0, re, im);
    const J2 ang = w_atan2(im, re);
    phi0_rd = ang.v;
    dphi0_rd = ang.d;
    const R d2phi0_rd = ang.dd;
    if (eta > kEtaEmr) {
      freqs[4] = fcut_rd;
      values[4] = dphi0_rd;
    }
    freqs[5] = fcut_rd;
    values[5] = d2phi0_rd;
    const R g_c = 0.5 * (1.0 / fcut_insp + 1.0 / fcut_rd);
    const R g_h = 0.5 * (1.0 / fcut_insp - 1.0 / fcut_rd);
    R a[6][6], b[6];
    for (int i = 0; i < 5; ++i) {
      const R v = (1.0 / freqs[i] - g_c) / g_h;
      a[i][0] = 1.0;
      a[i][1] = lor(freqs[i]);
      a[i][2] = v;
      a[i][3] = v * v;
      a[i][4] = v * v * v;
      a[i][5] = v * v * v * v;
      b[i] = values[i];
    }
    {
      const R ff = freqs[5];
      const R v = (1.0 / ff - g_c) / g_h;
      const R dv = -1.0 / (ff * ff * g_h);
      const R den = fdamp * fdamp + (ff - fring) * (ff - fring);
      a[5][0] = 0.0;
      a[5][1] = -2.0 * fdamp * (ff - fring) / (den * den);
      a[5][2] = dv;
      a[5][3] = 2.0 * v * dv;
      a[5][4] = 3.0 * v * v * dv;
      a[5][5] = 4.0 * v * v * v * dv;
      b[5] = values[5];
    }
    ok = solve_n<6>(a, b) && ok;
    const R quartic[5] = {b[0], b[2], b[3], b[4], b[5]};
    R p[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
    const R comb[5][5] = {{1, 0, 0, 0, 0}, {1, 1, 0, 0, 0}, {1, 2, 1, 0, 0}, {1, 3, 3, 1, 0}, {1, 4, 6, 4, 1}};
    for (int k = 0; k < 5; ++k) {
      const R scale = quartic[k] / w_pow(g_h, static_cast<double>(k));
      for (int j = 0; j <= k; ++j) p[j] = p[j] + scale * comb[k][j] * w_pow(-g_c, static_cast<double>(k - j));
    }
    ph.c0 = p[0];
    ph.c_l = b[1];
    ph.c1 = p[1];
    ph.c2 = p[2];
    ph.c4 = p[4];
    ph.c3 = p[3];
    const Powers<R> p_rd(fcut_rd);
    const R glued = ph.c0 + dphi0_rd - int_dphase(fcut_rd, p_rd, hm, ph);
    if (eta < kEtaEmr) ph.c0 = glued;
  }
  const Powers<R> p_in(fcut_insp);
  ph.c1_insp = int_dphase(fcut_insp, p_in, hm, ph) - ins_dphase(fcut_insp, p_in, ph);
  ph.c_insp = -ph.c1_insp * fcut_insp + int_phase(fcut_insp, p_in, hm, ph) - ins_phase_int(fcut_insp, p_in, ph);
  const Powers<R> p_rd(fcut_rd);
  ph.c1_rd = int_dphase(fcut_rd, p_rd, hm, ph) - dphi0_rd;
  ph.c_rd = -ph.c1_rd * fcut_rd + int_phase(fcut_rd, p_rd, hm, ph) - phi0_rd;
  return ok;
}

// The spheroidal (3,2) ringdown aligned with the (2,2) ringdown, without the
// anchor of the (2,2) in phi0_s (core.py:208-234).
template <class R>
inline WFX_HDI bool spheroidal(const xas::Internals<R>& w, const hmfit::Args<R>& fa, const R* tab22,
                        const Mode<R>& hm, Spheroidal<R>& sp) {
  const R fringlm = hm.f_ring, fdamplm = hm.f_damp;
  const R freqs[4] = {w.f_ring, -1.5 * fdamplm + fringlm, -0.5 * fdamplm + fringlm, 0.5 * fdamplm + fringlm};
  R a[4][4];
  R b[4] = {hmfit::rd_phase_32_p1(fa), hmfit::rd_phase_32_p2(fa), hmfit::rd_phase_32_p3(fa),
                  hmfit::rd_phase_32_p4(fa)};
  for (int i = 0; i < 4; ++i) {
    const R ff = freqs[i];
    const R ffm2 = 1.0 / (ff * ff);
    a[i][0] = 1.0;
    a[i][1] = fdamplm / (fdamplm * fdamplm + (ff - fringlm) * (ff - fringlm));
    a[i][2] = ffm2;
    a[i][3] = ffm2 * ffm2;
  }
  const bool ok = solve_n<4>(a, b);
  sp = Spheroidal<R>{b[0], b[1], b[2], b[3], 0.0};
  const RdPhase<R> none{0.0, 0.0, 0.0};
  {
    const R fref_rd = w.f_ring + w.f_damp;
    const Powers<R> p_ref(fref_rd);
    const R dphi22_ref = 1.0 / w.eta * dphase22(w, fref_rd) + w.linb;
    sp.alpha0_s = sp.alpha0_s + dphi22_ref + hmfit::rd_phase_32_spheroidal_time_shift(fa) -
                  rd_dphase(fref_rd, p_ref, hm, none, sp);
  }
  {
    const R fref_rd = w.f_ring;
    bool past;
    const R phi22_ref = rest22(tab22, fref_rd, w.m_sec, true, past);
    sp.phi0_s = phi22_ref - rd_phase(fref_rd, Powers<R>(fref_rd), hm, none, sp) +
                hmfit::rd_phase_32_spheroidal_phase_shift(fa);
  }
  return ok;
}

// Adds c x^a (log x)^l (x = s f) to a row over HM_BASIS (core.py:179-185).
template <class R>
struct SPowers {
  R p[14];  // s^a for the basis' exponents, in the order of HmBasis up to B_7_3
  R log_s;
};

template <class R>
inline WFX_HDI SPowers<R> s_powers(R s) {
  const Powers<R> p(s);
  SPowers<R> o;
  o.p[B_M3] = p.m_three;
  o.p[B_M2] = p.m_two;
  o.p[B_M4_3] = p.m_four_thirds;
  o.p[B_M1] = p.m_one;
  o.p[B_M2_3] = p.m_two_thirds;
  o.p[B_M1_3] = p.m_one_third;
  o.p[B_1] = 1.0;
  o.p[B_1_3] = p.one_third;
  o.p[B_2_3] = p.two_thirds;
  o.p[B_F] = s;
  o.p[B_4_3] = p.four_thirds;
  o.p[B_5_3] = p.five_thirds;
  o.p[B_F2] = p.two;
  o.p[B_7_3] = p.seven_thirds;
  o.log_s = p.log_;
  return o;
}

// b: the basis index of x^a (no log); log_index: that of x^a log x (or -1).
template <class R>
inline WFX_HDI void add_term(R* row, const SPowers<R>& sp, R c, int b, int log_index) {
  const R scaled = c * sp.p[b];
  if (log_index < 0) {
    row[b] = row[b] + scaled;
  } else {
    row[b] = row[b] + scaled * sp.log_s;
    row[log_index] = row[log_index] + scaled;
  }
}

// The table of one higher mode (core.py:237-353; MODE_LAYOUT), zero for the
// odd modes of equal masses and spins. Returns false if a collocation
// system is singular.
template <class R>
inline WFX_HDI bool mode_table(const xas::Internals<R>& w, const R* tab22, int mode_int, R* out) {
  for (int k = 0; k < kModeSize; ++k) out[k] = 0.0;
  const hmfit::Args<R> fa = fit_args(w);
  const R psi4_args[4] = {w.eta, w.s_tot_r, w.dchi, sqrt_nonneg(-4.0 * w.eta + 1.0)};
  const R psi4 = fit::fit_call(fit::XAS_PSI4_TO_STRAIN, psi4_args);
  const Mode<R> hm = mode_struct(w, mode_int, psi4);
  const bool odd = hm.tag == 21 || hm.tag == 33;
  if (odd && value(w.q) == 1.0 && value(w.chi1) == value(w.chi2)) return true;  // (core.py:383-389: zeros)
  Amp<R> amp;
  Rotation<R> rot{&w, tab22, &hm, &amp, Spheroidal<R>{0.0, 0.0, 0.0, 0.0, 0.0}};
  bool ok = true;
  if (hm.mixing) ok = spheroidal(w, fa, tab22, hm, rot.sp) && ok;
  ok = amplitude_coefficients(w, fa, hm, rot, amp) && ok;
  Phase<R> ph;
  ok = phase_coefficients(w, fa, hm, rot, ph) && ok;

  // D = deltaphi_lm + (m/2) A (core.py:270-283)
  const R s = w.m_sec;
  const R m_over_2 = hm.emm * 0.5;
  const R falign = w.eta > kEtaEmr ? 0.6 * m_over_2 * w.f_meco : m_over_2 * w.f_meco;
  R d;
  {
    bool past22;
    const R r22 = rest22(tab22, falign / m_over_2, s, false, past22);
    const R leading = ph.phi[0] * w_pow(falign, -5.0 / 3.0);
    const R phi_lm_rest = ph.c1_insp * falign + ins_phase_int(falign, Powers<R>(falign), ph, false) + ph.c_insp;
    d = (-(3.0 * (fit::PI / 4.0))) * (1.0 - m_over_2) + m_over_2 * r22 - phi_lm_rest - (past22 ? leading : 0.0);
    if (hm.tag == 21 && pn21_amp_sign(R(0.008), w)) d = d + fit::PI;
  }

  // the table (core.py:289-353)
  const SPowers<R> spw = s_powers(s);
  R* rows = out + M_PHASE;
  {
    R* row = rows;  // inspiral
    const int basis[13] = {-1, B_M4_3, B_M1, B_M2_3, B_M1_3, B_1, B_1_3, B_2_3, B_F, B_4_3, B_5_3, B_F2, B_7_3};
    for (int i = 1; i < 13; ++i) add_term(row, spw, ph.phi[i], basis[i], -1);
    add_term(row, spw, ph.phi_l[5], B_1, B_LOG);
    add_term(row, spw, ph.phi_l[6], B_1_3, B_1_3_LOG);
    add_term(row, spw, ph.phi_l[8], B_F, B_F_LOG);
    add_term(row, spw, ph.phi_l[9], B_4_3, B_4_3_LOG);
    add_term(row, spw, ph.c1_insp, B_F, -1);
    add_term(row, spw, ph.c_insp + d, B_1, -1);
  }
  {
    R* row = rows + kBasis;  // intermediate
    add_term(row, spw, ph.c0, B_F, -1);
    add_term(row, spw, ph.c1, B_1, B_LOG);
    add_term(row, spw, -ph.c2, B_M1, -1);
    add_term(row, spw, -ph.c4 / 3.0, B_M3, -1);
    add_term(row, spw, d, B_1, -1);
    if (hm.mixing) add_term(row, spw, -0.5 * ph.c3, B_M2, -1);
  }
  {
    R* row = rows + 2 * kBasis;  // ringdown
    if (hm.mixing) {
      add_term(row, spw, ph.c1_rd, B_F, -1);
      add_term(row, spw, ph.c_rd + d, B_1, -1);
    } else {
      add_term(row, spw, ph.rd.alpha0 + ph.c1_rd, B_F, -1);
      add_term(row, spw, -hm.f_ring * hm.f_ring * ph.rd.alpha2, B_M1, -1);
      add_term(row, spw, ph.c_rd + d, B_1, -1);
    }
  }
  const Powers<R> p(s);
  const R w_at = s / hm.f_damp;
  if (hm.mixing) {
    out[M_SPH + 0] = rot.sp.alpha0_s * s;
    out[M_SPH + 1] = rot.sp.phi0_s;
    out[M_SPH + 2] = -rot.sp.alpha2_s / s;
    out[M_SPH + 3] = -rot.sp.alpha4_s / 3.0 * p.m_three;
    out[M_ATAN_A + 2] = rot.sp.alpha_l_s;
    out[M_MIX + 0] = hm.mix[2][0];
    out[M_MIX + 1] = hm.mix[2][1];
    out[M_MIX + 2] = hm.mix[3][0];
    out[M_MIX + 3] = hm.mix[3][1];
  } else {
    out[M_ATAN_A + 2] = ph.rd.alpha_l;
  }
  out[M_ATAN_A + 1] = ph.c_l;
  out[M_ATAN_W + 1] = w_at;
  out[M_ATAN_W + 2] = w_at;
  out[M_SHIFT] = hm.f_ring / s;
  out[M_F_PHASE_IN] = ph.f_phase_match_in / s;
  out[M_F_PHASE_IM] = ph.f_phase_match_im / s;
  out[M_F_AMP_IN] = amp.f_amp_match_in / s;
  out[M_F_AMP_IM] = amp.f_amp_match_im / s;
  const R amp0 = w.amp0;
  const R pn_scale = amp.pn_global_factor * amp.amp_norm * p.m_seven_sixths * amp0;
  const R third[7] = {1.0, p.one_third, p.two_thirds, s, p.four_thirds, p.five_thirds, p.two};
  for (int k = 0; k < 7; ++k) {
    out[M_PN_RE + k] = amp.pn_re[k] * third[k] * pn_scale;
    out[M_PN_IM + k] = amp.pn_im[k] * third[k] * pn_scale;
  }
  const R fold = amp.pn_dominant * p.m_seven_sixths * amp0;
  out[M_PSEUDO + 0] = amp.ins[0] / amp.fcut_7_3 * p.seven_thirds * fold;
  out[M_PSEUDO + 1] = amp.ins[1] / amp.fcut_8_3 * p.eight_thirds * fold;
  out[M_PSEUDO + 2] = amp.ins[2] / amp.fcut_3 * p.three * fold;
  for (int j = 0; j < 8; ++j) out[M_INTER + j] = j < amp.n_inter ? amp.inter[j] * p.m_seven_sixths * amp0 : 0.0;
  out[M_INTER_C] = amp.inter_center / s;
  out[M_INTER_H] = s / amp.inter_half;
  const R dfd = hm.f_damp * amp.rd[2];
  out[M_RD + 0] = amp.rd[0] * hm.f_damp * amp0;
  out[M_RD + 1] = amp.rd[1] / dfd;
  out[M_RD + 2] = dfd * dfd;
  out[M_FALLOFF + 0] = amp.rd[3] * amp0;
  out[M_FALLOFF + 1] = amp.rd[4] * s;
  out[M_FALLOFF + 2] = hm.f_amp_rd_falloff / s;
  if (hm.mixing) {
    const R s_j[4] = {1.0, s, p.two, p.three};
    for (int j = 0; j < 4; ++j) out[M_AUX + j] = amp.rd_aux[j] * s_j[j] * amp0;
    out[M_F_AUX] = amp.f_rd_aux / s;
  }
  out[M_ON] = 1.0;
  return ok;
}

// ---------------------------------------------------------------------------
// The head: the factors (F+, Fx) of each mode h_{l,-m} in the polarizations
// (reference.py:630-638, _harmonics.py:17-36), amp0 and M in seconds.

// Wigner's d^l_{m' m}(beta) (the convention of LAL's XLALWignerdMatrix).
template <class R>
inline WFX_HDI R wigner_d(int ell, int mp, int m, R beta) {
  auto fact = [](int n) {
    R r = 1.0;
    for (int i = 2; i <= n; ++i) r *= i;
    return r;
  };
  const R ch = w_cos(beta / 2.0), sh = w_sin(beta / 2.0);
  const R pre = w_sqrt(fact(ell + mp) * fact(ell - mp) * fact(ell + m) * fact(ell - m));
  R total = 0.0;
  const int lo = m - mp > 0 ? m - mp : 0;
  const int hi = (ell + m) < (ell - mp) ? (ell + m) : (ell - mp);
  for (int k = lo; k <= hi; ++k) {
    const R sign = ((k - m + mp) % 2 == 0) ? 1.0 : -1.0;
    const R c = sign * pre / (fact(ell + m - k) * fact(k) * fact(ell - k - mp) * fact(k - m + mp));
    total = total + c * ipow(ch, 2 * ell - 2 * k + m - mp) * ipow(sh, 2 * k - m + mp);
  }
  return total;
}

// -2Y_lm(theta, pi/2) as (re, im).
template <class R>
inline WFX_HDI void swsh(R theta, int ell, int m, R& re, R& im) {
  const R norm = w_sqrt((2 * ell + 1) / (4.0 * fit::PI));
  const R d = norm * wigner_d(ell, m, 2, theta);
  const R x = static_cast<double>(m) * (fit::PI / 2.0);
  re = d * w_cos(x);
  im = d * w_sin(x);
}

// factors[4 k .. 4 k + 4) = Re F+, Im F+, Re Fx, Im Fx of mode k of
// (2,2), (2,1), (3,3), (3,2), (4,4).
template <class R>
inline WFX_HDI void mode_factors(R inclination, R* factors) {
  const int ells[5] = {2, 2, 3, 3, 4}, emms[5] = {2, 1, 3, 2, 4};
  for (int k = 0; k < 5; ++k) {
    const int ell = ells[k], emm = emms[k];
    const R sign = ell % 2 ? -1.0 : 1.0;
    R ymr, ymi, yr, yi;
    swsh(inclination, ell, -emm, ymr, ymi);
    swsh(inclination, ell, emm, yr, yi);
    const R ysr = yr, ysi = -yi;  // conj
    // F+ = (ym + sign ystar) / 2, Fx = i (ym - sign ystar) / 2
    factors[4 * k + 0] = 0.5 * (ymr + sign * ysr);
    factors[4 * k + 1] = 0.5 * (ymi + sign * ysi);
    const R dr = ymr - sign * ysr, di = ymi - sign * ysi;
    factors[4 * k + 2] = -0.5 * di;
    factors[4 * k + 3] = 0.5 * dr;
  }
}

}  // namespace xhm
}  // namespace wfx
