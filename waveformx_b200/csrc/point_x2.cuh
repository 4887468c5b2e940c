// IMRPhenomXAS's and IMRPhenomD's FP32 points at two frequencies of one
// binary in the two lanes of sm_100's packed FP32 instructions (fma.rn,
// add.rn and mul.rn .f32x2: __ffma2_rn, __fadd2_rn, __fmul2_rn; each lane
// rounds as the scalar _rn form). The operations are those of
// xas_eval / phd_eval<float, 2, RP, RA, true> (point.cuh) with their
// multiply-adds written out as fused ones, so that one instruction serves
// both frequencies; the elementary functions (atan, exp, the divisions,
// sin and cos) stay one per frequency. The forward kernel's evaluation
// where a warp's frequencies share their regions (models/xas/core.py:
// 423-507, models/phenomd/core.py:426-485).
#pragma once

#include "point.cuh"

namespace wfx {

// The powers of two frequencies (lane x: the first, y: the second) that
// the IMRPhenomXAS and IMRPhenomD evaluations read.
struct Freq2 {
  float2 f, t, m1, lf, m76, t2, t2lo, m3, yhi, ylo, f34, f34lo;
};

__device__ __forceinline__ Freq2 pack_freqs(const Freq<float>& a, const Freq<float>& b) {
  Freq2 q;
  q.f = make_float2(a.f, b.f);
  q.t = make_float2(a.t, b.t);
  q.m1 = make_float2(a.m1, b.m1);
  q.lf = make_float2(a.lf, b.lf);
  q.m76 = make_float2(a.m76, b.m76);
  q.t2 = make_float2(a.t2, b.t2);
  q.t2lo = make_float2(a.t2lo, b.t2lo);
  q.m3 = make_float2(a.m3, b.m3);
  q.yhi = make_float2(a.y.hi, b.y.hi);
  q.ylo = make_float2(a.y.lo, b.y.lo);
  q.f34 = make_float2(a.f34, b.f34);
  q.f34lo = make_float2(a.f34lo, b.f34lo);
  return q;
}

__device__ __forceinline__ float2 bc2(float x) { return make_float2(x, x); }

// A staged float table as the packed evaluation reads it: c[k] slot k's
// value in both lanes, c.s(k) the value. (Measured on 4096 x 4017 against a
// copy of the table with each value stored twice, whose 8-byte loads fill
// both lanes: that form issues more instructions and is slower, 0.0667 ms
// against 0.0616 for IMRPhenomXAS.)
struct Bcast {
  const float* T;
  __device__ __forceinline__ float2 operator[](int k) const { return bc2(T[k]); }
  __device__ __forceinline__ float s(int k) const { return T[k]; }
};

// The packed operations (sub2: the add of the negated lanes).
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __fadd2_rn(a, neg2(b)); }
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }

// round_nearest in both lanes.
__device__ __forceinline__ float2 round_nearest2(float2 x) {
  constexpr float kMagic = 12582912.0f;
  return add2(add2(x, bc2(kMagic)), bc2(-kMagic));
}

// phase_turns in both lanes (big = 0 when BIG is false).
template <bool BIG, class C>
__device__ __forceinline__ float2 phase_turns2(const C& T, int cs, int ls, int llo, const Freq2& q, float2 big_hi,
                                               float2 big_lo, float2 rest) {
  const float2 p = mul2(T[ls], q.f);
  const float2 e = fma2(T[ls], q.f, neg2(p));
  float2 phi = add2(T[cs], add2(sub2(p, round_nearest2(p)), fma2(T[llo], q.f, e)));
  if constexpr (BIG) phi = add2(phi, add2(sub2(big_hi, round_nearest2(big_hi)), big_lo));
  phi = add2(phi, rest);
  phi = sub2(phi, round_nearest2(phi));
  return mul2(phi, bc2(kTwoPiHi));
}

// The inspiral phase's products (inspiral_basis) of both lanes.
struct Basis2 {
  float2 mt1, mt2, tlf, flf, ft, ft2, ff;
};

__device__ __forceinline__ Basis2 inspiral_basis2(const Freq2& q) {
  Basis2 x;
  x.mt1 = mul2(q.t2, q.m1);
  x.mt2 = mul2(x.mt1, x.mt1);
  x.tlf = mul2(q.t, q.lf);
  x.flf = mul2(q.f, q.lf);
  x.ft = mul2(q.f, q.t);
  x.ft2 = mul2(q.f, q.t2);
  x.ff = mul2(q.f, q.f);
  return x;
}

// df_mul(df, df) of a double-float (a_hi, a_lo) common to both lanes and
// one per lane (b_hi, b_lo): two_prod, the cross terms, quick_two_sum.
__device__ __forceinline__ void df_mul2_lanes(float2 a_hi, float2 a_lo, float2 b_hi, float2 b_lo, float2& hi,
                                              float2& lo) {
  const float2 p = mul2(a_hi, b_hi);
  const float2 e = fma2(a_hi, b_hi, neg2(p));
  const float2 l = fma2(a_hi, b_lo, fma2(a_lo, b_hi, e));
  hi = add2(p, l);
  lo = sub2(l, sub2(hi, p));
}

// project() of both lanes: h+ = kp A (c, s), hx = kc A (-s, c).
__device__ __forceinline__ void project2(float2 kp, float2 kc, float2 amp, float2 phi, float4& hp, float4& hc) {
  float s0, c0, s1, c1;
  m_sincos(phi.x, &s0, &c0);
  m_sincos(phi.y, &s1, &c1);
  const float2 ap = mul2(kp, amp), ac = mul2(kc, amp);
  const float2 p0 = mul2(bc2(ap.x), make_float2(c0, s0)), p1 = mul2(bc2(ap.y), make_float2(c1, s1));
  const float2 x0 = mul2(bc2(ac.x), make_float2(-s0, c0)), x1 = mul2(bc2(ac.y), make_float2(-s1, c1));
  hp = make_float4(p0.x, p0.y, p1.x, p1.y);
  hc = make_float4(x0.x, x0.y, x1.x, x1.y);
}

// (h+, hx) of the two frequencies: lanes (x, y) of hp = (h+(f0), h+(f1))
// and hc likewise, as project() forms them. RP, RA: the regions every
// frequency of the warp's span shares; T the binary's staged table made
// ready by prepare_model (phase in turns), read through C.
template <int RP, int RA, class C>
__device__ __forceinline__ void xas_pair_x2(const C& T, const Freq2& q, float4& hp, float4& hc) {
  float2 rest, big_hi = bc2(0.0f), big_lo = bc2(0.0f);
  if constexpr (RP == 0) {
    constexpr int R = X_PH_INS;
    const Basis2 x = inspiral_basis2(q);
    float2 r = mul2(T[R + 0], q.m1);
    r = fma2(T[R + 1], x.mt2, r);
    r = fma2(T[R + 2], x.mt1, r);
    r = fma2(T[R + 3], q.lf, r);
    r = fma2(T[R + 5], q.t, r);
    r = fma2(T[R + 6], x.tlf, r);
    r = fma2(T[R + 7], q.t2, r);
    r = fma2(T[R + 9], x.flf, r);
    r = fma2(T[R + 10], x.ft, r);
    r = fma2(T[R + 11], x.ft2, r);
    r = fma2(T[R + 12], x.ff, r);
    rest = r;
    df_mul2_lanes(T[X_T0], T[X32_T0_LO], q.yhi, q.ylo, big_hi, big_lo);
  } else {
    if constexpr (RP == 1) {
      constexpr int R = X_PH_INT;
      float2 r = mul2(T[R + 2], q.lf);
      r = fma2(T[R + 3], q.m1, r);
      r = fma2(T[R + 4], mul2(q.m1, q.m1), r);
      rest = fma2(T[R + 5], q.m3, r);
    } else {
      constexpr int R = X_PH_RD;
      df_mul2_lanes(T[R + 2], T[X32_RD_TERM_LO], q.t2, q.t2lo, big_hi, big_lo);
      rest = fma2(T[R + 4], q.m3, mul2(T[R + 3], q.m1));
    }
    constexpr int k = RP - 1;
    const float2 z = mul2(T[X_ATAN_W + k], sub2(q.f, T[X_SHIFT]));
    rest = fma2(T[X_ATAN_A + k], make_float2(m_atan(z.x), m_atan(z.y)), rest);
  }
  const float2 phi = phase_turns2<RP != 1>(T, xas_const_slot(RP), xas_lin_slot(RP), X32_LIN_LO + RP, q, big_hi,
                                           big_lo, rest);
  float2 amp;
  if constexpr (RA == 0) {
    float2 poly = T[X_AMP_INS + 9];
#pragma unroll
    for (int k = 8; k >= 0; --k) poly = fma2(poly, q.t, T[X_AMP_INS + k]);
    amp = mul2(q.m76, poly);
  } else if constexpr (RA == 1) {
    float2 den = T[X_AMP_INT_D + 4];
#pragma unroll
    for (int k = 3; k >= 0; --k) den = fma2(den, q.f, T[X_AMP_INT_D + k]);
    const float n = T.s(X_AMP_INT_N);
    amp = make_float2(m_div(n, den.x), m_div(n, den.y));
  } else {
    const float2 u = mul2(T[X_AMP_RD_S], sub2(q.f, T[X_SHIFT]));
    const float2 x = mul2(T[X_AMP_RD_GR], u);  // (-gr u: the sign in the exponential)
    const float2 d = fma2(u, u, T[X_AMP_RD_G]);
    const float2 eq = make_float2(m_div(m_exp(-x.x), d.x), m_div(m_exp(-x.y), d.y));
    amp = mul2(mul2(T[X_AMP_RD_N], q.m76), eq);
  }
  const float f_cut = T.s(X_F_CUT);
  amp.x = q.f.x > f_cut ? 0.0f : amp.x;
  amp.y = q.f.y > f_cut ? 0.0f : amp.y;
  project2(T[X_KP], T[X_KC], amp, phi, hp, hc);
}

// IMRPhenomD's pair as xas_pair_x2 (the operations of
// phd_eval<float, 2, RP, RA, true>, models/phenomd/core.py:426-485).
template <int RP, int RA, class C>
__device__ __forceinline__ void phd_pair_x2(const C& T, const Freq2& q, float4& hp, float4& hc) {
  float2 rest, big_hi = bc2(0.0f), big_lo = bc2(0.0f);
  if constexpr (RP == 0) {
    constexpr int R = D_PH_INS;
    const Basis2 x = inspiral_basis2(q);
    float2 r = mul2(T[R + 1], q.m1);
    r = fma2(T[R + 2], x.mt2, r);
    r = fma2(T[R + 3], x.mt1, r);
    r = fma2(T[R + 4], q.lf, r);
    r = fma2(T[R + 5], q.t, r);
    r = fma2(T[R + 6], x.tlf, r);
    r = fma2(T[R + 7], q.t2, r);
    r = fma2(T[R + 9], x.ft, r);
    r = fma2(T[R + 10], x.ft2, r);
    r = fma2(T[R + 11], x.ff, r);
    rest = r;
    df_mul2_lanes(T[D_T0], T[D32_T0_LO], q.yhi, q.ylo, big_hi, big_lo);
  } else if constexpr (RP == 1) {
    constexpr int R = D_PH_INT;
    rest = fma2(T[R + 3], q.lf, mul2(T[R + 2], q.m3));
  } else {
    constexpr int R = D_PH_RD;
    df_mul2_lanes(T[R + 3], T[D32_RD_TERM_LO], q.f34, q.f34lo, big_hi, big_lo);
    const float2 r = mul2(T[R + 2], q.m1);
    const float2 z = mul2(T[D_ATAN_W], sub2(q.f, T[D_ATAN_SHIFT]));
    rest = fma2(T[D_ATAN_A], make_float2(m_atan(z.x), m_atan(z.y)), r);
  }
  const float2 phi = phase_turns2<RP != 1>(T, phd_const_slot(RP), phd_lin_slot(RP), D32_LIN_LO + RP, q, big_hi,
                                           big_lo, rest);
  float2 amp;
  if constexpr (RA == 0) {
    float2 poly = T[D_AMP_INS + 9];
#pragma unroll
    for (int k = 8; k >= 0; --k) poly = fma2(poly, q.t, T[D_AMP_INS + k]);
    amp = poly;
  } else if constexpr (RA == 2) {
    const float2 u = mul2(T[D_AMP_RD_S], sub2(q.f, T[D_AMP_RD_SHIFT]));
    const float2 x = mul2(T[D_AMP_RD_GR], u);  // (-gr u: the sign in the exponential)
    const float2 d = fma2(u, u, bc2(1.0f));
    const float2 eq = make_float2(m_div(m_exp(-x.x), d.x), m_div(m_exp(-x.y), d.y));
    amp = mul2(T[D_AMP_RD_N], eq);
  } else {
    const float2 y = mul2(T[D_AMP_INT_S], q.f);
    float2 inter = T[D_AMP_INT + 4];
#pragma unroll
    for (int k = 3; k >= 0; --k) inter = fma2(inter, y, T[D_AMP_INT + k]);
    amp = inter;
  }
  project2(T[D_KP], T[D_KC], mul2(q.m76, amp), phi, hp, hc);
}

}  // namespace wfx
