// The point evaluation of point.cuh in FP64 forward mode: Dual
// (scalar.cuh), a value and its derivative along one direction, for
//  * IMRPhenomXHM's gradient (xhm.cu): the table's entries carry their
//    tangent along one parameter, the frequencies none (lift);
//  * the derivative with respect to the frequency grid (kernels.cu): the
//    frequency powers carry d/df (freq_powers_dual), the table none.
// In namespace wfx, beside Dual, so that the templated point code finds
// these overloads.
#pragma once

#include <cuda_runtime.h>

#include "point.cuh"
#include "scalar.cuh"

namespace wfx {

template <>
struct Freq<Dual> {
  Dual f, t, m1, lf, m76;
  Dual t2, mt1, mt2, m2, m3, tlf, flf, ft, ft2, ff, f34;
  Dual y;
};

__device__ __forceinline__ Freq<Dual> lift(const Freq<double>& q) {
  Freq<Dual> o;
  o.f = q.f;
  o.t = q.t;
  o.m1 = q.m1;
  o.lf = q.lf;
  o.m76 = q.m76;
  o.t2 = q.t2;
  o.mt1 = q.mt1;
  o.mt2 = q.mt2;
  o.m2 = q.m2;
  o.m3 = q.m3;
  o.tlf = q.tlf;
  o.flf = q.flf;
  o.ft = q.ft;
  o.ft2 = q.ft2;
  o.ff = q.ff;
  o.f34 = q.f34;
  o.y = q.y;
  return o;
}

template <>
struct TcOf<Dual> {
  using type = double;
};

__device__ __forceinline__ Dual m_atan(const Dual& x) { return Dual(atan(x.v), x.d / (1.0 + x.v * x.v)); }
__device__ __forceinline__ Dual m_exp(const Dual& x) {
  const double e = exp(x.v);
  return Dual(e, e * x.d);
}
__device__ __forceinline__ Dual m_div(const Dual& a, const Dual& b) { return a / b; }
__device__ __forceinline__ void m_sincos(const Dual& x, Dual* s, Dual* c) {
  double sv, cv;
  sincos(x.v, &sv, &cv);
  *s = Dual(sv, cv * x.d);
  *c = Dual(cv, -sv * x.d);
}
__device__ __forceinline__ void full_sincos(const Dual& x, Dual* s, Dual* c) { m_sincos(x, s, c); }
__device__ __forceinline__ Dual m_hypot(const Dual& a, const Dual& b) {
  const double h = hypot(a.v, b.v);
  return Dual(h, h > 0.0 ? (a.v * a.d + b.v * b.d) / h : 0.0);
}
__device__ __forceinline__ Dual m_atan2(const Dual& y, const Dual& x) {
  const double r2 = x.v * x.v + y.v * y.v;
  return Dual(atan2(y.v, x.v), r2 > 0.0 ? (x.v * y.d - y.v * x.d) / r2 : 0.0);
}
// (the XAS point's FP64 phase, models/xas/core.py:445-468, in forward mode)
__device__ __forceinline__ Dual reduced_phase(bool inspiral, const Dual* T, int t0_slot, int anchor_slot,
                                              const Freq<Dual>& q, Dual rest, double tc) {
  Dual phi = (inspiral ? T[t0_slot] * q.y : Dual(0.0)) + rest;
  phi = phi - T[anchor_slot];
  phi = phi - kTwoPi * q.f * tc;
  return phi - rint(phi.v / kTwoPi) * kTwoPi;
}
// |x| (for comparisons) and the nearest integer (a constant: no derivative)
__device__ __forceinline__ float m_abs(float x) { return fabsf(x); }
__device__ __forceinline__ double m_abs(double x) { return fabs(x); }
__device__ __forceinline__ double m_abs(const Dual& x) { return fabs(x.v); }
__device__ __forceinline__ float m_round(float x) { return rintf(x); }
__device__ __forceinline__ double m_round(double x) { return rint(x); }
__device__ __forceinline__ double m_round(const Dual& x) { return rint(x.v); }

// The frequency powers of freq_powers(double) with their derivatives in f.
__device__ __forceinline__ Freq<Dual> freq_powers_dual(double f) {
  const Freq<double> q = freq_powers(f);
  const double inv = 1.0 / f;
  // d(f^a)/df = a f^a / f; the products of a power and log f by the
  // product rule
  auto pw = [&](double v, double a) { return Dual(v, a * v * inv); };
  Freq<Dual> o;
  o.f = Dual(f, 1.0);
  o.t = pw(q.t, 1.0 / 3.0);
  o.m1 = pw(q.m1, -1.0);
  o.lf = Dual(q.lf, inv);
  o.m76 = pw(q.m76, -7.0 / 6.0);
  o.t2 = pw(q.t2, 2.0 / 3.0);
  o.mt1 = pw(q.mt1, -1.0 / 3.0);
  o.mt2 = pw(q.mt2, -2.0 / 3.0);
  o.m2 = pw(q.m2, -2.0);
  o.m3 = pw(q.m3, -3.0);
  o.tlf = Dual(q.tlf, (q.t * q.lf / 3.0 + q.t) * inv);
  o.flf = Dual(q.flf, q.lf + 1.0);
  o.ft = pw(q.ft, 4.0 / 3.0);
  o.ft2 = pw(q.ft2, 5.0 / 3.0);
  o.ff = pw(q.ff, 2.0);
  o.f34 = pw(q.f34, 0.75);
  o.y = pw(q.y, -5.0 / 3.0);
  return o;
}

}  // namespace wfx
