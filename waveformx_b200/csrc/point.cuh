// The waveform at one frequency for one binary's table, and its reverse-mode
// derivative with respect to the table's entries (and t_c).
//
// Two arithmetics share the code:
//  * float: FP32 throughout, with the phase's large parts carried in
//    double-float (unevaluated hi + lo pairs of floats): the leading inspiral
//    term T0 f^-5/3, the anchor A = T0 f_ref^-5/3, the time shift 2 pi f t_c,
//    and the reduction to [-pi, pi]. f^-5/3 itself comes from one Newton step
//    in double-float.
//  * double: the plain FP64 form, the same operations as the reference's
//    float64 evaluation (models/xas/core.py:382-507,
//    models/phenomd/core.py:398-485).
//
// The adjoint accumulates, for a cotangent (g+, gx) of (h+, hx) in PyTorch's
// convention (g = dL/dRe h + i dL/dIm h), sum_f dL/dT_k into acc[k] (k a
// table slot), and dL/dt_c into acc[kSlotTc]. The gradient with respect to a
// binary's parameters is then sum_k acc[k] dT_k/dtheta (kernels.cu).
#pragma once

#include <cuda_runtime.h>

#include "tables.cuh"

namespace wfx {

constexpr int kSlotTc = 60;    // acc slot of dL/dt_c
constexpr int kSlotLoss = 61;  // acc slot of the loss (fused likelihood)

// ---------------------------------------------------------------------------
// double-float arithmetic (exact sums and products of floats)

struct df {
  float hi, lo;
};

__device__ __forceinline__ df two_sum(float a, float b) {
  float s = __fadd_rn(a, b);
  float bb = __fsub_rn(s, a);
  float e = __fadd_rn(__fsub_rn(a, __fsub_rn(s, bb)), __fsub_rn(b, bb));
  return {s, e};
}
__device__ __forceinline__ df quick_two_sum(float a, float b) {
  float s = __fadd_rn(a, b);
  return {s, __fsub_rn(b, __fsub_rn(s, a))};
}
__device__ __forceinline__ df two_prod(float a, float b) {
  float p = __fmul_rn(a, b);
  return {p, __fmaf_rn(a, b, -p)};
}
__device__ __forceinline__ df df_mul(df a, df b) {
  df p = two_prod(a.hi, b.hi);
  float lo = __fmaf_rn(a.hi, b.lo, __fmaf_rn(a.lo, b.hi, p.lo));
  return quick_two_sum(p.hi, lo);
}
__device__ __forceinline__ df df_mul(df a, float b) {
  df p = two_prod(a.hi, b);
  return quick_two_sum(p.hi, __fmaf_rn(a.lo, b, p.lo));
}

// f^2/3 as a double-float from its float value t2: one Newton step on
// y^3 = f^2 with the residual in double-float.
__device__ __forceinline__ df df_pow23(float f, float t2) {
  const df f2 = two_prod(f, f);
  const df y3 = df_mul(two_prod(t2, t2), t2);
  const float r = __fsub_rn(f2.hi, y3.hi) + __fsub_rn(f2.lo, y3.lo);
  return quick_two_sum(t2, __fdividef(r, 3.0f * t2 * t2));
}

// f^3/4 as a double-float from its float value y0: one Newton step on
// y^4 = f^3.
__device__ __forceinline__ df df_pow34(float f, float y0) {
  const df f3 = df_mul(two_prod(f, f), f);
  const df y2 = two_prod(y0, y0);
  const df y4 = df_mul(y2, y2);
  const float r = __fsub_rn(f3.hi, y4.hi) + __fsub_rn(f3.lo, y4.lo);
  return quick_two_sum(y0, __fdividef(r, 4.0f * y0 * y0 * y0));
}

// 2 pi as a sum of two floats, and 1 / (2 pi)
constexpr float kTwoPiHi = 6.28318548202514648f;
constexpr float kTwoPiLo = -1.74845553e-07f;
constexpr float kInvTwoPi = 0.159154943091895336f;
constexpr double kTwoPi = 6.283185307179586;

// ---------------------------------------------------------------------------
// per-frequency powers and phase basis (shared by every binary at that
// frequency)

template <class S>
struct Freq;

template <>
struct Freq<float> {
  float f, t, m1, lf, m76;
  float t2, mt1, mt2, m2, m3, tlf, flf, ft, ft2, ff, f34;
  df y;         // f^-5/3
  float t2lo;   // f^2/3 = t2 + t2lo (double-float)
  float f34lo;  // f^3/4 = f34 + f34lo (double-float)
};

template <>
struct Freq<double> {
  double f, t, m1, lf, m76;
  double t2, mt1, mt2, m2, m3, tlf, flf, ft, ft2, ff, f34;
  double y;
};

template <class S>
__device__ __forceinline__ void basis_products(Freq<S>& q) {
  // the products of models/xas/core.py:395-403 and models/phenomd/core.py:412-418
  q.t2 = q.t * q.t;
  q.mt1 = q.t2 * q.m1;
  q.mt2 = q.mt1 * q.mt1;
  q.m2 = q.m1 * q.m1;
  q.m3 = q.m2 * q.m1;
  q.tlf = q.t * q.lf;
  q.flf = q.f * q.lf;
  q.ft = q.f * q.t;
  q.ft2 = q.f * q.t2;
  q.ff = q.f * q.f;
}

// The products of the inspiral phase basis, formed where the inspiral is
// evaluated (rather than kept with the powers: a kernel that loops over
// binaries at fixed frequencies then holds fewer values per frequency).
template <class S>
struct Basis {
  S mt1, mt2, tlf, flf, ft, ft2, ff;
};

template <class S>
__device__ __forceinline__ Basis<S> inspiral_basis(const Freq<S>& q) {
  Basis<S> x;
  x.mt1 = q.t2 * q.m1;
  x.mt2 = x.mt1 * x.mt1;
  x.tlf = q.t * q.lf;
  x.flf = q.f * q.lf;
  x.ft = q.f * q.t;
  x.ft2 = q.f * q.t2;
  x.ff = q.f * q.f;
  return x;
}

__device__ __forceinline__ Freq<float> freq_powers(float f) {
  Freq<float> q;
  q.f = f;
  q.m1 = __frcp_rn(f);
  q.lf = logf(f);
  float t = expf(q.lf * (1.0f / 3.0f));
  q.t = t * (4.0f - t * t * t * q.m1) * (1.0f / 3.0f);
  q.m76 = q.m1 * rsqrtf(q.t);
  // f^-5/3: y0 from the float exponential, then one Newton step on
  // y^3 f^5 = 1 with the residual in double-float
  float y0 = expf(-5.0f / 3.0f * q.lf);
  df f2 = two_prod(f, f);
  df f5 = df_mul(df_mul(f2, f2), f);
  df y3 = df_mul(two_prod(y0, y0), y0);
  df w = df_mul(y3, f5);
  float r = __fsub_rn(__fsub_rn(1.0f, w.hi), w.lo);
  q.y = quick_two_sum(y0, y0 * r * (1.0f / 3.0f));
  basis_products(q);
  const float root = sqrtf(f);
  q.f34 = root * sqrtf(root);
  // the ringdown's largest terms (f^2/3, f^3/4) in double-float, once per
  // frequency
  const df t23 = df_pow23(f, q.t2);
  q.t2 = t23.hi;
  q.t2lo = t23.lo;
  const df f34 = df_pow34(f, q.f34);
  q.f34 = f34.hi;
  q.f34lo = f34.lo;
  return q;
}

__device__ __forceinline__ Freq<double> freq_powers(double f) {
  // models/xas/core.py:382-392
  Freq<double> q;
  q.f = f;
  q.m1 = 1.0 / f;
  q.lf = log(f);
  double t = exp(q.lf / 3.0);
  q.t = t * (4.0 - t * t * t * q.m1) / 3.0;
  q.m76 = q.m1 / sqrt(q.t);
  q.y = exp(-5.0 / 3.0 * q.lf);
  basis_products(q);
  const double root = sqrt(f);
  q.f34 = root * sqrt(root);
  return q;
}

// ---------------------------------------------------------------------------
// arithmetic-specific pieces

// atan(x) to 2.6e-7 absolute: x P(x^2) on [0, 1], P of degree 6 minimax in
// the absolute error (Remez exchange; atan_poly.py prints the coefficients),
// and atan(x) = pi/2 - atan(1/x) beyond.
__device__ __forceinline__ float m_atan(float x) {
  const float a = fabsf(x);
  const bool inv = a > 1.0f;
  const float u = inv ? __fdividef(1.0f, a) : a;
  const float s = u * u;
  float p = 6.811792962e-03f;
  p = __fmaf_rn(p, s, -3.360421956e-02f);
  p = __fmaf_rn(p, s, 7.962366939e-02f);
  p = __fmaf_rn(p, s, -1.323334277e-01f);
  p = __fmaf_rn(p, s, 1.980781555e-01f);
  p = __fmaf_rn(p, s, -3.331736922e-01f);
  p = __fmaf_rn(p, s, 9.999961257e-01f);
  float r = u * p;
  r = inv ? 1.57079632679489662f - r : r;
  return copysignf(r, x);
}
__device__ __forceinline__ double m_atan(double x) { return atan(x); }
__device__ __forceinline__ float m_exp(float x) { return __expf(x); }
__device__ __forceinline__ double m_exp(double x) { return exp(x); }
__device__ __forceinline__ float m_div(float a, float b) { return __fdividef(a, b); }
__device__ __forceinline__ double m_div(double a, double b) { return a / b; }
__device__ __forceinline__ void m_sincos(float x, float* s, float* c) { __sincosf(x, s, c); }
__device__ __forceinline__ void m_sincos(double x, double* s, double* c) { sincos(x, s, c); }

// 2 pi t_c as a double-float.
struct TcF {
  float hi, lo;
};

__device__ __forceinline__ TcF make_tc(float t_c) {
  df p = two_prod(kTwoPiHi, t_c);
  return {p.hi, __fmaf_rn(kTwoPiLo, t_c, p.lo)};
}

// x rounded to the nearest integer (ties to even) for |x| < 2^22, by adding
// and removing 1.5 * 2^23 (two adds on the FMA pipe rather than a rounding
// instruction).
__device__ __forceinline__ float round_nearest(float x) {
  constexpr float kMagic = 12582912.0f;
  return __fsub_rn(__fadd_rn(x, kMagic), kMagic);
}

// hi + lo modulo 2 pi, as a float near [-pi, pi] (2 pi in two floats; the
// products k 2pi_hi are exact inside the FMA).
__device__ __forceinline__ float reduce_df(float hi, float lo) {
  const float k = round_nearest(hi * kInvTwoPi);
  float r = __fmaf_rn(-k, kTwoPiHi, hi);
  r = __fmaf_rn(-k, kTwoPiLo, r);
  return r + lo;
}

// A staged FP32 table made ready for the frequencies of one binary: 2 pi
// t_c folded into each region's coefficient of f (double-float, slots ls[r]
// and llo + r), and each region's constant (double-float, slots cs[r] and
// clo + r) reduced modulo 2 pi into its float slot. Once per binary.
template <int REGIONS>
__device__ __forceinline__ void prepare_f32(float* T, const int (&cs)[REGIONS], int clo, const int (&ls)[REGIONS],
                                            int llo, float t_c) {
  const TcF tc = make_tc(t_c);
#pragma unroll
  for (int r = 0; r < REGIONS; ++r) {
    const df s = two_sum(T[ls[r]], -tc.hi);
    const df out = quick_two_sum(s.hi, s.lo + T[llo + r] - tc.lo);
    T[ls[r]] = out.hi;
    T[llo + r] = out.lo;
    T[cs[r]] = reduce_df(T[cs[r]], T[clo + r]);
    T[clo + r] = 0.0f;
  }
}

// A staged FP32 table made ready for the frequencies of one binary with its
// phase in turns (phase_turns): the plain-float phase coefficients (slots
// `plain`, n_plain of them) and the double-float ones (T0 in t0/t0lo, the
// largest term past the inspiral in big/biglo when big >= 0, each region's
// coefficient of f in ls[r]/llo + r) divided by 2 pi, t_c subtracted from
// each coefficient of f, each region's constant (cs[r]/clo + r) in turns
// less its nearest integer. Once per binary.
template <int REGIONS>
__device__ __forceinline__ void prepare_turns(float* T, const int* plain, int n_plain, int t0, int t0lo, int big,
                                              int biglo, const int (&cs)[REGIONS], int clo,
                                              const int (&ls)[REGIONS], int llo, float t_c) {
  constexpr df kInvTwoPiDf{0.159154936671257019f, 6.42063824e-09f};
#pragma unroll
  for (int i = 0; i < n_plain; ++i) T[plain[i]] *= kInvTwoPi;
  const df a = df_mul(df{T[t0], T[t0lo]}, kInvTwoPiDf);
  T[t0] = a.hi;
  T[t0lo] = a.lo;
  if (big >= 0) {
    const df r = df_mul(df{T[big], T[biglo]}, kInvTwoPiDf);
    T[big] = r.hi;
    T[biglo] = r.lo;
  }
#pragma unroll
  for (int k = 0; k < REGIONS; ++k) {
    const df l = df_mul(df{T[ls[k]], T[llo + k]}, kInvTwoPiDf);
    const df s = two_sum(l.hi, -t_c);
    const df out = quick_two_sum(s.hi, s.lo + l.lo);
    T[ls[k]] = out.hi;
    T[llo + k] = out.lo;
    const df c = df_mul(df{T[cs[k]], T[clo + k]}, kInvTwoPiDf);
    T[cs[k]] = (c.hi - round_nearest(c.hi)) + c.lo;
    T[clo + k] = 0.0f;
  }
}

// The FP32 phase reduced to [-pi, pi]: C + L f + big + rest, where C is the
// region's constant (the anchor folded in, already reduced modulo 2 pi), L
// its coefficient of f (2 pi t_c folded in; double-float in slots ls/llo),
// `big` the leading inspiral term T0 f^-5/3 or the ringdown's largest term
// (double-float, zero in the intermediate region) and `rest` the other terms
// (float). Each large part is reduced modulo 2 pi on its own, then the sum.
__device__ __forceinline__ float phase_f32(const float* T, int cs, int ls, int llo, const Freq<float>& q, df big,
                                           float rest) {
  const df p = two_prod(T[ls], q.f);
  float phi = T[cs] + reduce_df(p.hi, __fmaf_rn(T[llo], q.f, p.lo));
  phi = phi + reduce_df(big.hi, big.lo);
  phi = phi + rest;
  const float k = round_nearest(phi * kInvTwoPi);
  phi = __fmaf_rn(-k, kTwoPiHi, phi);
  return __fmaf_rn(-k, kTwoPiLo, phi);
}

// The same phase with every phase coefficient of the table in turns (cycles,
// prepare_turns): each large part less its nearest integer (exact in FP32
// below 2^22 turns), the sum less its nearest integer, times 2 pi: radians
// in [-pi, pi].
__device__ __forceinline__ float phase_turns(const float* T, int cs, int ls, int llo, const Freq<float>& q, df big,
                                             float rest) {
  const df p = two_prod(T[ls], q.f);
  float phi = T[cs] + ((p.hi - round_nearest(p.hi)) + __fmaf_rn(T[llo], q.f, p.lo));
  phi = phi + ((big.hi - round_nearest(big.hi)) + big.lo);
  phi = phi + rest;
  phi = phi - round_nearest(phi);
  return phi * kTwoPiHi;
}

__device__ __forceinline__ double reduced_phase(bool inspiral, const double* T, int t0_slot, int anchor_slot,
                                                const Freq<double>& q, double rest, double tc) {
  // models/xas/core.py:445-468 (and the t_c shift)
  double phi = (inspiral ? T[t0_slot] * q.y : 0.0) + rest;
  phi = phi - T[anchor_slot];
  phi = phi - kTwoPi * q.f * tc;
  double turns = rint(phi / kTwoPi);
  return phi - turns * kTwoPi;
}

template <class S>
struct TcOf {
  using type = TcF;
};
template <>
struct TcOf<double> {
  using type = double;
};

// ---------------------------------------------------------------------------
// the state of one (binary, frequency) kept for the adjoint

template <class S>
struct Point {
  S amp, c, s;  // amplitude, cos and sin of the reduced phase
  int rp, ra;   // phase and amplitude regions
  S at, zz;     // atan(z), 1 / (1 + z^2) past the inspiral
  S a0, a1;     // amplitude aux: intermediate den (XAS); ringdown u and
                // e / (u^2 + g)
};

// ---------------------------------------------------------------------------
// IMRPhenomXAS

template <class S>
__device__ __forceinline__ void xas_regions(const S* __restrict__ T, S f, int& rp, int& ra) {
  // phase: past the inspiral where f >= f_phase_in, ringdown where
  // f > f_phase_im; amplitude likewise (models/xas/core.py:427-428, 479-480)
  rp = (f >= T[X_F_PHASE_IN]) + (f > T[X_F_PHASE_IM]);
  ra = (f >= T[X_F_AMP_IN]) + (f > T[X_F_AMP_RD]);
}

// NF frequencies q[0..NF) of one binary that share the phase region rp and
// the amplitude region ra (every table coefficient read once for them).
template <class S, int NF, int RP = -1, int RA = -1, bool TURNS = false>
__device__ __forceinline__ void xas_eval(const S* __restrict__ T, const Freq<S>* q, int rp, int ra,
                                         typename TcOf<S>::type tc, Point<S>* pt) {
  constexpr bool kF32 = sizeof(S) == 4;
  // (RP, RA >= 0: the regions are known at compile time, every branch on
  // them folds away)
  if constexpr (RP >= 0) rp = RP;
  if constexpr (RA >= 0) ra = RA;
  S rest[NF];
  df big[NF];
#pragma unroll
  for (int j = 0; j < NF; ++j) {
    pt[j].rp = rp;
    pt[j].ra = ra;
    pt[j].at = S(0);
    pt[j].zz = S(0);
    pt[j].a0 = S(0);
    pt[j].a1 = S(0);
    big[j] = df{0.0f, 0.0f};
  }
  // (FP32: the constant, the term in f and the leading or largest term
  // apart, in double-float)
  if (rp == 0) {
    const S* R = T + X_PH_INS;
#pragma unroll
    for (int j = 0; j < NF; ++j) {
      const Freq<S>& b = q[j];
      const Basis<S> x = inspiral_basis(b);
      S r = kF32 ? R[0] * b.m1 : R[4] + R[0] * b.m1;
      r = r + R[1] * x.mt2;
      r = r + R[2] * x.mt1;
      r = r + R[3] * b.lf;
      r = r + R[5] * b.t;
      r = r + R[6] * x.tlf;
      r = r + R[7] * b.t2;
      if (!kF32) r = r + R[8] * b.f;
      r = r + R[9] * x.flf;
      r = r + R[10] * x.ft;
      r = r + R[11] * x.ft2;
      r = r + R[12] * x.ff;
      rest[j] = r;
      if constexpr (kF32) big[j] = df_mul(df{T[X_T0], T[X32_T0_LO]}, b.y);
    }
  } else {
    if (rp == 1) {
      const S* R = T + X_PH_INT;
#pragma unroll
      for (int j = 0; j < NF; ++j) {
        const Freq<S>& b = q[j];
        S r = kF32 ? R[2] * b.lf : (R[0] + R[1] * b.f) + R[2] * b.lf;
        r = r + R[3] * b.m1;
        r = r + R[4] * (b.m1 * b.m1);
        r = r + R[5] * b.m3;
        rest[j] = r;
      }
    } else {
      const S* R = T + X_PH_RD;
#pragma unroll
      for (int j = 0; j < NF; ++j) {
        const Freq<S>& b = q[j];
        S r;
        if constexpr (kF32) {
          big[j] = df_mul(df{R[2], T[X32_RD_TERM_LO]}, df{b.t2, b.t2lo});
          r = R[3] * b.m1;
        } else {
          r = ((R[0] + R[1] * b.f) + R[2] * b.t2) + R[3] * b.m1;
        }
        rest[j] = r + R[4] * b.m3;
      }
    }
    const int k = rp - 1;
    const S aw = T[X_ATAN_W + k], aa = T[X_ATAN_A + k], sh = T[X_SHIFT];
#pragma unroll
    for (int j = 0; j < NF; ++j) {
      const S z = aw * (q[j].f - sh);
      pt[j].at = m_atan(z);
      pt[j].zz = m_div(S(1), S(1) + z * z);
      rest[j] = rest[j] + aa * pt[j].at;
    }
  }
  S phi[NF];
#pragma unroll
  for (int j = 0; j < NF; ++j) {
    if constexpr (kF32) {
      phi[j] = TURNS ? phase_turns(T, xas_const_slot(rp), xas_lin_slot(rp), X32_LIN_LO + rp, q[j], big[j], rest[j])
                     : phase_f32(T, xas_const_slot(rp), xas_lin_slot(rp), X32_LIN_LO + rp, q[j], big[j], rest[j]);
    } else {
      phi[j] = reduced_phase(rp == 0, T, X_T0, X_ANCHOR, q[j], rest[j], tc);
    }
  }
  S amp[NF];
  if (ra == 0) {
    const S* C = T + X_AMP_INS;
#pragma unroll
    for (int j = 0; j < NF; ++j) {
      S poly = C[9];
#pragma unroll
      for (int k = 8; k >= 0; --k) poly = poly * q[j].t + C[k];
      amp[j] = q[j].m76 * poly;
    }
  } else if (ra == 1) {
    const S* D = T + X_AMP_INT_D;
    const S n = T[X_AMP_INT_N];
#pragma unroll
    for (int j = 0; j < NF; ++j) {
      S den = D[4];
#pragma unroll
      for (int k = 3; k >= 0; --k) den = den * q[j].f + D[k];
      pt[j].a0 = den;
      amp[j] = m_div(n, den);
    }
  } else {
    const S rs = T[X_AMP_RD_S], sh = T[X_SHIFT], gr = T[X_AMP_RD_GR], g = T[X_AMP_RD_G], an = T[X_AMP_RD_N];
#pragma unroll
    for (int j = 0; j < NF; ++j) {
      const S u = rs * (q[j].f - sh);
      const S eq = m_div(m_exp(-gr * u), u * u + g);
      pt[j].a0 = u;
      pt[j].a1 = eq;
      amp[j] = an * q[j].m76 * eq;
    }
  }
  const S f_cut = T[X_F_CUT];
#pragma unroll
  for (int j = 0; j < NF; ++j) {
    pt[j].amp = q[j].f > f_cut ? S(0) : amp[j];
    m_sincos(phi[j], &pt[j].s, &pt[j].c);
  }
}

template <class S>
__device__ __forceinline__ Point<S> xas_point(const S* __restrict__ T, const Freq<S>& q,
                                              typename TcOf<S>::type tc) {
  int rp, ra;
  xas_regions(T, q.f, rp, ra);
  Point<S> pt;
  xas_eval<S, 1>(T, &q, rp, ra, tc, &pt);
  return pt;
}

// acc[k] += dL/dT_k at this frequency; (gpr, gpi, gcr, gci): the cotangent.
template <class S, class Acc>
__device__ __forceinline__ void xas_adjoint(const S* __restrict__ T, const Freq<S>& q, const Point<S>& pt, S gpr,
                                            S gpi, S gcr, S gci, Acc* acc) {
  const S A = pt.amp;
  if (A == S(0)) return;  // above the cutoff: nothing depends on the table
  const S c = pt.c, s = pt.s;
  const S kp = T[X_KP], kc = T[X_KC];
  const S ap = gpr * c + gpi * s, ac = gci * c - gcr * s;
  acc[X_KP] += A * ap;
  acc[X_KC] += A * ac;
  const S abar = kp * ap + kc * ac;
  const S pbar = A * (kp * (gpi * c - gpr * s) - kc * (gcr * c + gci * s));
  const S f = q.f, t = q.t, m1 = q.m1, lf = q.lf;
  const S t2 = q.t2, mt1 = q.mt1;
  if (pt.rp == 0) {
    const S mt2 = q.mt2;
    acc[X_PH_INS + 0] += pbar * m1;
    acc[X_PH_INS + 1] += pbar * mt2;
    acc[X_PH_INS + 2] += pbar * mt1;
    acc[X_PH_INS + 3] += pbar * lf;
    acc[X_PH_INS + 4] += pbar;
    acc[X_PH_INS + 5] += pbar * t;
    acc[X_PH_INS + 6] += pbar * (t * lf);
    acc[X_PH_INS + 7] += pbar * t2;
    acc[X_PH_INS + 8] += pbar * f;
    acc[X_PH_INS + 9] += pbar * (f * lf);
    acc[X_PH_INS + 10] += pbar * (f * t);
    acc[X_PH_INS + 11] += pbar * (f * t2);
    acc[X_PH_INS + 12] += pbar * (f * f);
    if constexpr (sizeof(S) == 4) {
      acc[X_T0] += pbar * q.y.hi;
    } else {
      acc[X_T0] += pbar * q.y;
    }
  } else {
    const S m2 = m1 * m1;
    const int r = pt.rp - 1;
    if (r == 0) {
      acc[X_PH_INT + 0] += pbar;
      acc[X_PH_INT + 1] += pbar * f;
      acc[X_PH_INT + 2] += pbar * lf;
      acc[X_PH_INT + 3] += pbar * m1;
      acc[X_PH_INT + 4] += pbar * m2;
      acc[X_PH_INT + 5] += pbar * (m2 * m1);
      const S y = f - T[X_SHIFT];
      const S g = pbar * T[X_ATAN_A] * pt.zz;
      acc[X_ATAN_A] += pbar * pt.at;
      acc[X_ATAN_W] += g * y;
      acc[X_SHIFT] -= g * T[X_ATAN_W];
    } else {
      acc[X_PH_RD + 0] += pbar;
      acc[X_PH_RD + 1] += pbar * f;
      acc[X_PH_RD + 2] += pbar * t2;
      acc[X_PH_RD + 3] += pbar * m1;
      acc[X_PH_RD + 4] += pbar * (m2 * m1);
      const S y = f - T[X_SHIFT];
      const S g = pbar * T[X_ATAN_A + 1] * pt.zz;
      acc[X_ATAN_A + 1] += pbar * pt.at;
      acc[X_ATAN_W + 1] += g * y;
      acc[X_SHIFT] -= g * T[X_ATAN_W + 1];
    }
  }
  acc[X_ANCHOR] -= pbar;
  acc[kSlotTc] -= S(kTwoPi) * f * pbar;
  if (pt.ra == 0) {
    S w = abar * q.m76;
#pragma unroll
    for (int k = 0; k < 10; ++k) {
      acc[X_AMP_INS + k] += w;
      w = w * t;
    }
  } else if (pt.ra == 1) {
    const S inv = m_div(S(1), pt.a0);
    acc[X_AMP_INT_N] += abar * inv;
    S w = -abar * A * inv;
#pragma unroll
    for (int j = 0; j < 5; ++j) {
      acc[X_AMP_INT_D + j] += w;
      w = w * f;
    }
  } else {
    const S u = pt.a0, eq = pt.a1;
    const S gA = abar * A;
    acc[X_AMP_RD_N] += abar * q.m76 * eq;
    acc[X_AMP_RD_GR] -= gA * u;
    const S qq = u * u + T[X_AMP_RD_G];
    const S ubar = gA * (-T[X_AMP_RD_GR] - m_div(S(2) * u, qq));
    acc[X_AMP_RD_S] += ubar * (f - T[X_SHIFT]);
    acc[X_SHIFT] -= ubar * T[X_AMP_RD_S];
    acc[X_AMP_RD_G] -= m_div(gA, qq);
  }
}

// ---------------------------------------------------------------------------
// IMRPhenomD

template <class S>
__device__ __forceinline__ void phd_regions(const S* __restrict__ T, S f, int& rp, int& ra) {
  // inspiral where f < f_phase_ins, merger-ringdown where f >= f_phase_mrd;
  // amplitude likewise (models/phenomd/core.py:430-431, 472)
  rp = f < T[D_F_PHASE_INS] ? 0 : (f >= T[D_F_PHASE_MRD] ? 2 : 1);
  ra = f < T[D_F_AMP_INS] ? 0 : (f >= T[D_F_AMP_MRD] ? 2 : 1);
}

template <class S, int NF, int RP = -1, int RA = -1, bool TURNS = false>
__device__ __forceinline__ void phd_eval(const S* __restrict__ T, const Freq<S>* q, int rp, int ra,
                                         typename TcOf<S>::type tc, Point<S>* pt) {
  constexpr bool kF32 = sizeof(S) == 4;
  // (RP, RA >= 0: the regions are known at compile time, every branch on
  // them folds away)
  if constexpr (RP >= 0) rp = RP;
  if constexpr (RA >= 0) ra = RA;
  S rest[NF];
  df big[NF];
#pragma unroll
  for (int j = 0; j < NF; ++j) {
    pt[j].rp = rp;
    pt[j].ra = ra;
    pt[j].at = S(0);
    pt[j].zz = S(0);
    pt[j].a0 = S(0);
    pt[j].a1 = S(0);
    big[j] = df{0.0f, 0.0f};
  }
  if (rp == 0) {
    const S* R = T + D_PH_INS;
#pragma unroll
    for (int j = 0; j < NF; ++j) {
      const Freq<S>& b = q[j];
      const Basis<S> x = inspiral_basis(b);
      S r = kF32 ? R[1] * b.m1 : R[0] + R[1] * b.m1;
      r = r + R[2] * x.mt2;
      r = r + R[3] * x.mt1;
      r = r + R[4] * b.lf;
      r = r + R[5] * b.t;
      r = r + R[6] * x.tlf;
      r = r + R[7] * b.t2;
      if (!kF32) r = r + R[8] * b.f;
      r = r + R[9] * x.ft;
      r = r + R[10] * x.ft2;
      r = r + R[11] * x.ff;
      rest[j] = r;
      if constexpr (kF32) big[j] = df_mul(df{T[D_T0], T[D32_T0_LO]}, b.y);
    }
  } else if (rp == 1) {
    const S* R = T + D_PH_INT;
#pragma unroll
    for (int j = 0; j < NF; ++j) {
      const Freq<S>& b = q[j];
      S r = kF32 ? R[2] * b.m3 : (R[0] + R[1] * b.f) + R[2] * b.m3;
      rest[j] = r + R[3] * b.lf;
    }
  } else {
    const S* R = T + D_PH_RD;
    const S aw = T[D_ATAN_W], aa = T[D_ATAN_A], sh = T[D_ATAN_SHIFT];
#pragma unroll
    for (int j = 0; j < NF; ++j) {
      const Freq<S>& b = q[j];
      S r;
      if constexpr (kF32) {
        big[j] = df_mul(df{R[3], T[D32_RD_TERM_LO]}, df{b.f34, b.f34lo});
        r = R[2] * b.m1;
      } else {
        r = ((R[0] + R[1] * b.f) + R[2] * b.m1) + R[3] * b.f34;
      }
      const S z = aw * (b.f - sh);
      pt[j].at = m_atan(z);
      pt[j].zz = m_div(S(1), S(1) + z * z);
      rest[j] = r + aa * pt[j].at;
    }
  }
  S phi[NF];
#pragma unroll
  for (int j = 0; j < NF; ++j) {
    if constexpr (kF32) {
      phi[j] = TURNS ? phase_turns(T, phd_const_slot(rp), phd_lin_slot(rp), D32_LIN_LO + rp, q[j], big[j], rest[j])
                     : phase_f32(T, phd_const_slot(rp), phd_lin_slot(rp), D32_LIN_LO + rp, q[j], big[j], rest[j]);
    } else {
      phi[j] = reduced_phase(rp == 0, T, D_T0, D_ANCHOR, q[j], rest[j], tc);
    }
  }
  S amp[NF];
  if (ra == 0) {
    const S* C = T + D_AMP_INS;
#pragma unroll
    for (int j = 0; j < NF; ++j) {
      S poly = C[9];
#pragma unroll
      for (int k = 8; k >= 0; --k) poly = poly * q[j].t + C[k];
      amp[j] = poly;
    }
  } else if (ra == 2) {
    const S rs = T[D_AMP_RD_S], sh = T[D_AMP_RD_SHIFT], gr = T[D_AMP_RD_GR], an = T[D_AMP_RD_N];
#pragma unroll
    for (int j = 0; j < NF; ++j) {
      const S u = rs * (q[j].f - sh);
      const S eq = m_div(m_exp(-gr * u), u * u + S(1));
      pt[j].a0 = u;
      pt[j].a1 = eq;
      amp[j] = an * eq;
    }
  } else {
    const S* D = T + D_AMP_INT;
    const S ys = T[D_AMP_INT_S];
#pragma unroll
    for (int j = 0; j < NF; ++j) {
      const S y = ys * q[j].f;
      S inter = D[4];
#pragma unroll
      for (int k = 3; k >= 0; --k) inter = inter * y + D[k];
      amp[j] = inter;
    }
  }
#pragma unroll
  for (int j = 0; j < NF; ++j) {
    pt[j].amp = q[j].m76 * amp[j];
    m_sincos(phi[j], &pt[j].s, &pt[j].c);
  }
}

template <class S>
__device__ __forceinline__ Point<S> phd_point(const S* __restrict__ T, const Freq<S>& q,
                                              typename TcOf<S>::type tc) {
  int rp, ra;
  phd_regions(T, q.f, rp, ra);
  Point<S> pt;
  phd_eval<S, 1>(T, &q, rp, ra, tc, &pt);
  return pt;
}

template <class S, class Acc>
__device__ __forceinline__ void phd_adjoint(const S* __restrict__ T, const Freq<S>& q, const Point<S>& pt, S gpr,
                                            S gpi, S gcr, S gci, Acc* acc) {
  const S A = pt.amp;
  const S c = pt.c, s = pt.s;
  const S kp = T[D_KP], kc = T[D_KC];
  const S ap = gpr * c + gpi * s, ac = gci * c - gcr * s;
  acc[D_KP] += A * ap;
  acc[D_KC] += A * ac;
  const S abar = kp * ap + kc * ac;
  const S pbar = A * (kp * (gpi * c - gpr * s) - kc * (gcr * c + gci * s));
  const S f = q.f, t = q.t, m1 = q.m1, lf = q.lf;
  const S t2 = q.t2, mt1 = q.mt1;
  if (pt.rp == 0) {
    acc[D_PH_INS + 0] += pbar;
    acc[D_PH_INS + 1] += pbar * m1;
    acc[D_PH_INS + 2] += pbar * (mt1 * mt1);
    acc[D_PH_INS + 3] += pbar * mt1;
    acc[D_PH_INS + 4] += pbar * lf;
    acc[D_PH_INS + 5] += pbar * t;
    acc[D_PH_INS + 6] += pbar * (t * lf);
    acc[D_PH_INS + 7] += pbar * t2;
    acc[D_PH_INS + 8] += pbar * f;
    acc[D_PH_INS + 9] += pbar * (f * t);
    acc[D_PH_INS + 10] += pbar * (f * t2);
    acc[D_PH_INS + 11] += pbar * (f * f);
    if constexpr (sizeof(S) == 4) {
      acc[D_T0] += pbar * q.y.hi;
    } else {
      acc[D_T0] += pbar * q.y;
    }
  } else if (pt.rp == 1) {
    acc[D_PH_INT + 0] += pbar;
    acc[D_PH_INT + 1] += pbar * f;
    acc[D_PH_INT + 2] += pbar * (m1 * m1 * m1);
    acc[D_PH_INT + 3] += pbar * lf;
  } else {
    acc[D_PH_RD + 0] += pbar;
    acc[D_PH_RD + 1] += pbar * f;
    acc[D_PH_RD + 2] += pbar * m1;
    acc[D_PH_RD + 3] += pbar * q.f34;
    const S y = f - T[D_ATAN_SHIFT];
    const S g = pbar * T[D_ATAN_A] * pt.zz;
    acc[D_ATAN_A] += pbar * pt.at;
    acc[D_ATAN_W] += g * y;
    acc[D_ATAN_SHIFT] -= g * T[D_ATAN_W];
  }
  acc[D_ANCHOR] -= pbar;
  acc[kSlotTc] -= S(kTwoPi) * f * pbar;
  const S am = abar * q.m76;  // d L / d (amplitude without f^-7/6)
  if (pt.ra == 0) {
    S w = am;
#pragma unroll
    for (int k = 0; k < 10; ++k) {
      acc[D_AMP_INS + k] += w;
      w = w * t;
    }
  } else if (pt.ra == 2) {
    const S u = pt.a0, eq = pt.a1;
    const S P = T[D_AMP_RD_N] * eq;
    acc[D_AMP_RD_N] += am * eq;
    acc[D_AMP_RD_GR] -= am * P * u;
    const S ubar = am * P * (-T[D_AMP_RD_GR] - m_div(S(2) * u, u * u + S(1)));
    acc[D_AMP_RD_S] += ubar * (f - T[D_AMP_RD_SHIFT]);
    acc[D_AMP_RD_SHIFT] -= ubar * T[D_AMP_RD_S];
  } else {
    const S y = T[D_AMP_INT_S] * f;
    const S* D = T + D_AMP_INT;
    S w = am;
    S dp = S(0), yk = S(1);
#pragma unroll
    for (int j = 0; j < 5; ++j) {
      acc[D_AMP_INT + j] += w;
      w = w * y;
      if (j > 0) {
        dp = dp + S(j) * D[j] * yk;
        yk = yk * y;
      }
    }
    acc[D_AMP_INT_S] += am * dp * f;
  }
}

// ---------------------------------------------------------------------------
// TaylorF2 (models/taylorf2/core.py:168-212): one region, no cutoff

template <class S>
__device__ __forceinline__ void tf2_regions(const S* __restrict__, S, int& rp, int& ra) {
  rp = 0;
  ra = 0;
}

template <class S, int NF, int RP = -1, int RA = -1, bool TURNS = false>
__device__ __forceinline__ void tf2_eval(const S* __restrict__ T, const Freq<S>* q, int, int,
                                         typename TcOf<S>::type tc, Point<S>* pt) {
  constexpr bool kF32 = sizeof(S) == 4;
  const S* R = T + T_PH;
#pragma unroll
  for (int j = 0; j < NF; ++j) {
    const Freq<S>& b = q[j];
    const Basis<S> x = inspiral_basis(b);
    pt[j].rp = 0;
    pt[j].ra = 0;
    pt[j].at = S(0);
    pt[j].zz = S(0);
    pt[j].a0 = S(0);
    pt[j].a1 = S(0);
    // the constant, then the basis f^-1, f^-2/3, f^-1/3, log f, f^1/3,
    // f^1/3 log f, f^2/3 (core.py:174-181); FP32: the constant, the term in
    // f and the leading term apart, in double-float
    S r = kF32 ? R[0] * b.m1 : R[4] + R[0] * b.m1;
    r = r + R[1] * x.mt2;
    r = r + R[2] * x.mt1;
    r = r + R[3] * b.lf;
    r = r + R[5] * b.t;
    r = r + R[6] * x.tlf;
    r = r + R[7] * b.t2;
    S phi;
    if constexpr (kF32) {
      const df big = df_mul(df{T[T_T0], T[T32_T0_LO]}, b.y);
      phi = TURNS ? phase_turns(T, T_PH + 4, T_LIN, T32_LIN_LO, b, big, r)
                  : phase_f32(T, T_PH + 4, T_LIN, T32_LIN_LO, b, big, r);
    } else {
      phi = reduced_phase(true, T, T_T0, T_ANCHOR, b, r, tc);
    }
    pt[j].amp = T[T_AMP] * b.m76;
    m_sincos(phi, &pt[j].s, &pt[j].c);
  }
}

template <class S>
__device__ __forceinline__ Point<S> tf2_point(const S* __restrict__ T, const Freq<S>& q,
                                              typename TcOf<S>::type tc) {
  Point<S> pt;
  tf2_eval<S, 1>(T, &q, 0, 0, tc, &pt);
  return pt;
}

template <class S, class Acc>
__device__ __forceinline__ void tf2_adjoint(const S* __restrict__ T, const Freq<S>& q, const Point<S>& pt, S gpr,
                                            S gpi, S gcr, S gci, Acc* acc) {
  const S A = pt.amp;
  const S c = pt.c, s = pt.s;
  const S kp = T[T_KP], kc = T[T_KC];
  const S ap = gpr * c + gpi * s, ac = gci * c - gcr * s;
  acc[T_KP] += A * ap;
  acc[T_KC] += A * ac;
  const S abar = kp * ap + kc * ac;
  const S pbar = A * (kp * (gpi * c - gpr * s) - kc * (gcr * c + gci * s));
  const S f = q.f, t = q.t, m1 = q.m1, lf = q.lf, t2 = q.t2;
  const S mt1 = t2 * m1;
  acc[T_PH + 0] += pbar * m1;
  acc[T_PH + 1] += pbar * (mt1 * mt1);
  acc[T_PH + 2] += pbar * mt1;
  acc[T_PH + 3] += pbar * lf;
  acc[T_PH + 4] += pbar;
  acc[T_PH + 5] += pbar * t;
  acc[T_PH + 6] += pbar * (t * lf);
  acc[T_PH + 7] += pbar * t2;
  if constexpr (sizeof(S) == 4) {
    acc[T_T0] += pbar * q.y.hi;
  } else {
    acc[T_T0] += pbar * q.y;
  }
  acc[T_ANCHOR] -= pbar;
  acc[kSlotTc] -= S(kTwoPi) * f * pbar;
  acc[T_AMP] += abar * q.m76;
}

}  // namespace wfx
