// Scalar types of the per-binary set-up: double, and Dual (a double with one
// forward-mode derivative), with the elementary functions the set-up uses.
// The set-up templates (setup_xas.cuh, setup_phenomd.cuh) are written once
// over R in {double, Dual}: the plain set-up and its Jacobian-vector product
// along one parameter direction run the same code.
#pragma once

#include <cmath>
#include <cstdint>

#if defined(__CUDACC__)
#define WFX_HD __host__ __device__ __forceinline__
#define WFX_HDI __host__ __device__
#else
#define WFX_HD inline
#define WFX_HDI inline
#endif

namespace wfx {

struct Dual {
  double v;  // value
  double d;  // derivative along the direction being traced
  WFX_HD Dual() : v(0.0), d(0.0) {}
  WFX_HD Dual(double value) : v(value), d(0.0) {}  // NOLINT: constants promote
  WFX_HD Dual(double value, double derivative) : v(value), d(derivative) {}
};

WFX_HD double value(double x) { return x; }
WFX_HD double value(const Dual& x) { return x.v; }

WFX_HD Dual operator+(Dual a, Dual b) { return Dual(a.v + b.v, a.d + b.d); }
WFX_HD Dual operator-(Dual a, Dual b) { return Dual(a.v - b.v, a.d - b.d); }
WFX_HD Dual operator-(Dual a) { return Dual(-a.v, -a.d); }
WFX_HD Dual operator*(Dual a, Dual b) { return Dual(a.v * b.v, a.d * b.v + a.v * b.d); }
WFX_HD Dual operator/(Dual a, Dual b) {
  double q = a.v / b.v;
  return Dual(q, (a.d - q * b.d) / b.v);
}
WFX_HD Dual operator+(Dual a, double b) { return Dual(a.v + b, a.d); }
WFX_HD Dual operator+(double a, Dual b) { return Dual(a + b.v, b.d); }
WFX_HD Dual operator-(Dual a, double b) { return Dual(a.v - b, a.d); }
WFX_HD Dual operator-(double a, Dual b) { return Dual(a - b.v, -b.d); }
WFX_HD Dual operator*(Dual a, double b) { return Dual(a.v * b, a.d * b); }
WFX_HD Dual operator*(double a, Dual b) { return Dual(a * b.v, a * b.d); }
WFX_HD Dual operator/(Dual a, double b) { return Dual(a.v / b, a.d / b); }
WFX_HD Dual operator/(double a, Dual b) {
  double q = a / b.v;
  return Dual(q, -q * b.d / b.v);
}
WFX_HD Dual& operator+=(Dual& a, Dual b) { a = a + b; return a; }
WFX_HD Dual& operator-=(Dual& a, Dual b) { a = a - b; return a; }
WFX_HD Dual& operator*=(Dual& a, Dual b) { a = a * b; return a; }

// Comparisons look at values only (branches of the set-up are piecewise).
WFX_HD bool operator<(Dual a, Dual b) { return a.v < b.v; }
WFX_HD bool operator>(Dual a, Dual b) { return a.v > b.v; }
WFX_HD bool operator<=(Dual a, Dual b) { return a.v <= b.v; }
WFX_HD bool operator>=(Dual a, Dual b) { return a.v >= b.v; }

// Elementary functions, double and Dual.
WFX_HD double w_sqrt(double x) { return sqrt(x); }
WFX_HD double w_cbrt(double x) { return cbrt(x); }
WFX_HD double w_exp(double x) { return exp(x); }
WFX_HD double w_log(double x) { return log(x); }
WFX_HD double w_atan(double x) { return atan(x); }
WFX_HD double w_cos(double x) { return cos(x); }
WFX_HD double w_sin(double x) { return sin(x); }
WFX_HD double w_abs(double x) { return fabs(x); }
WFX_HD double w_pow(double x, double p) { return pow(x, p); }

WFX_HD Dual w_sqrt(Dual x) {
  double r = sqrt(x.v);
  return Dual(r, x.d * 0.5 / r);
}
WFX_HD Dual w_cbrt(Dual x) {
  double r = cbrt(x.v);
  return Dual(r, x.d * r / (3.0 * x.v));
}
WFX_HD Dual w_exp(Dual x) {
  double e = exp(x.v);
  return Dual(e, x.d * e);
}
WFX_HD Dual w_log(Dual x) { return Dual(log(x.v), x.d / x.v); }
WFX_HD Dual w_atan(Dual x) { return Dual(atan(x.v), x.d / (1.0 + x.v * x.v)); }
WFX_HD Dual w_cos(Dual x) { return Dual(cos(x.v), -sin(x.v) * x.d); }
WFX_HD Dual w_sin(Dual x) { return Dual(sin(x.v), cos(x.v) * x.d); }
WFX_HD Dual w_abs(Dual x) { return x.v < 0.0 ? -x : x; }
WFX_HD Dual w_pow(Dual x, double p) {
  double r = pow(x.v, p);
  return Dual(r, x.d * p * pow(x.v, p - 1.0));
}

// select(c, a, b): a where c, else b (jnp.where of a scalar).
template <class R>
WFX_HD R select(bool c, const R& a, const R& b) {
  return c ? a : b;
}
template <class R>
WFX_HD R w_min(const R& a, double b) {
  return value(a) < b ? a : R(b);
}
// sqrt(x) for x > 0, else 0 with a zero derivative.
template <class R>
WFX_HD R sqrt_nonneg(const R& x) {
  return value(x) > 0.0 ? w_sqrt(x) : R(0.0);
}
// x^n for a small non-negative integer n (repeated products).
template <class R>
WFX_HD R ipow(const R& x, int n) {
  R r(1.0);
  for (int i = 0; i < n; ++i) r = r * x;
  return r;
}

}  // namespace wfx
