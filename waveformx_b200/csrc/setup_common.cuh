// Pieces shared by the per-binary set-ups of IMRPhenomXAS and IMRPhenomD:
// the evaluation of the fits (fit_code.h), the powers of a number
// that the IMRPhenomX ansatzes use, Horner sums and the small dense linear
// solves of the collocation systems.
#pragma once

#include "fit_code.h"
#include "fit_tables.h"
#include "scalar.cuh"

namespace wfx {

// The fits, as straight-line nested Horner rules (fit_code.h, generated
// from the tables of fit_tables.h); `id` is a constant at every call, so the
// dispatch folds away.
template <class R>
WFX_HD R fit4(int id, const R& a, const R& b, const R& c, const R& d) {
  const R x[4] = {a, b, c, d};
  return fit::fit_call(id, x);
}
template <class R>
WFX_HD R fit2(int id, const R& a, const R& b) {
  const R x[2] = {a, b};
  return fit::fit_call(id, x);
}
template <class R>
WFX_HD R fit5(int id, const R& a, const R& b, const R& c, const R& d, const R& e) {
  const R x[5] = {a, b, c, d, e};
  return fit::fit_call(id, x);
}

// The parts of a set-up: its amplitude coefficients, its phase
// coefficients (with the alignment, f_cut and the projection), or both. The
// two parts share only the fits and the QNM frequencies, so that different
// blocks can compute them.
enum Role : int { kRoleAmp = 1, kRolePhase = 2, kRoleAll = 3 };

// Where a set-up takes its fit values from: evaluated in place from the
// binary's variables (DirectFits; fit_value of the model's namespace), or
// read from a row that other warps of the block evaluated beforehand
// (StagedFits: row[id - first]).
template <class R, class V>
struct DirectFits {
  const V& v;
  WFX_HDI R operator()(int id) const { return fit_value(id, v); }
};

template <class R>
struct StagedFits {
  const R* row;
  int first;
  WFX_HDI R operator()(int id) const { return row[id - first]; }
};

// The powers of x from one cube root, as IMRPhenomX's useful powers.
template <class R>
struct Powers {
  R itself, one_third, one_sixth, m_one, log_, two_thirds, m_one_third, m_one_sixth, four_thirds, five_thirds,
      seven_thirds, eight_thirds, m_two_thirds, m_four_thirds, m_five_thirds, m_seven_thirds, m_eight_thirds, two,
      three, four, m_two, m_three, m_four, seven_sixths, m_seven_sixths;
  WFX_HDI explicit Powers(const R& x) {
    itself = x;
    one_third = w_cbrt(x);
    one_sixth = w_sqrt(one_third);
    m_one = 1.0 / x;
    log_ = w_log(x);
    two_thirds = one_third * one_third;
    m_one_third = two_thirds * m_one;
    m_one_sixth = one_sixth * m_one_third;
    four_thirds = two_thirds * two_thirds;
    five_thirds = four_thirds * one_third;
    seven_thirds = four_thirds * x;
    eight_thirds = seven_thirds * one_third;
    m_two_thirds = m_one_third * m_one_third;
    m_four_thirds = m_two_thirds * m_two_thirds;
    m_five_thirds = m_four_thirds * m_one_third;
    m_seven_thirds = m_four_thirds * m_one;
    m_eight_thirds = m_seven_thirds * m_one_third;
    two = x * x;
    three = two * x;
    four = two * two;
    m_two = m_one * m_one;
    m_three = m_two * m_one;
    m_four = m_two * m_two;
    seven_sixths = one_sixth * x;
    m_seven_sixths = m_one_sixth * m_one;
  }
};

// sum_k c[k] x^k by Horner's rule (c lowest first).
template <class R, class C>
WFX_HD R horner(const C* c, int n, const R& x) {
  R total(c[n - 1]);
  for (int k = n - 2; k >= 0; --k) total = total * x + c[k];
  return total;
}

// Solves a x = b in place (a is N x N, row-major; the solution replaces b)
// by Gaussian elimination with partial pivoting on the values. Returns
// false if a pivot vanishes.
//
// The pivot row is brought up by compare-and-swap against each candidate in
// turn (the first row of largest magnitude wins, as with an arg-max), so
// that every index is a compile-time constant and the system stays in
// registers.
template <class R, int N>
WFX_HDI bool solve(R (&a)[N][N], R (&b)[N]) {
  bool ok = true;
#pragma unroll
  for (int col = 0; col < N; ++col) {
#pragma unroll
    for (int r = col + 1; r < N; ++r) {
      const bool larger = fabs(value(a[r][col])) > fabs(value(a[col][col]));
#pragma unroll
      for (int c = col; c < N; ++c) {
        const R top = a[col][c], other = a[r][c];
        a[col][c] = larger ? other : top;
        a[r][c] = larger ? top : other;
      }
      const R top = b[col], other = b[r];
      b[col] = larger ? other : top;
      b[r] = larger ? top : other;
    }
    ok = ok && fabs(value(a[col][col])) > 0.0;
#pragma unroll
    for (int r = col + 1; r < N; ++r) {
      const R l = a[r][col] / a[col][col];
#pragma unroll
      for (int c = col + 1; c < N; ++c) a[r][c] = a[r][c] - l * a[col][c];
      b[r] = b[r] - l * b[col];
    }
  }
#pragma unroll
  for (int r = N - 1; r >= 0; --r) {
    R s = b[r];
#pragma unroll
    for (int c = r + 1; c < N; ++c) s = s - a[r][c] * b[c];
    b[r] = s / a[r][r];
  }
  return ok;
}

// Status bits of a binary (int32, per binary): where LAL refuses it. The
// waveform of such a binary is NaN (its kp, kc are NaN).
enum Status : int32_t {
  kStatusMassRatio = 1,       // mass ratio beyond 1000 (IMRPhenomXAS)
  kStatusSpin = 2,            // an aligned spin beyond one
  kStatusFinalMass = 4,       // the fitted final mass exceeds the total
  kStatusFinalSpin = 8,       // the fitted final spin exceeds one
  kStatusMeco = 16,           // f_MECO above f_ISCO (IMRPhenomXAS)
  kStatusReferenceMf = 32,    // reference_mf given with a non-zero f_ref
  kStatusBadParameters = 64,  // non-finite or non-positive masses / distance
  kStatusSolve = 128,         // a collocation system is singular
};

}  // namespace wfx
