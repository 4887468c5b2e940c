// IMRPhenomXHM at the frequencies for sm_100a: the modes h_{l,-m} of
// (2,2), (2,1), (3,3), (3,2), (4,4) and (h+, hx) from the tables of
// wfx_xhm_setup (models/xhm/core.py:409-556), and the C-ABI entry.
//
// One block per (binary, run of frequencies), the binary's row staged in
// shared memory; one thread per frequency. The (2,2) is IMRPhenomXAS's
// point (point.cuh); each higher mode's amplitude and phase follow
// mode_rest (core.py:429-518): the phase of the region, with the (2,2)
// leading term rescaled, T0_lm f^-5/3, in the inspiral; the (3,2) ringdown
// rotates the recycled (2,2) mode with its own spheroidal ringdown.
//  * FP64: the reference's float64 evaluation;
//  * FP32: float, with each region's constant (the (2,2) anchor folded in,
//    reduced modulo 2 pi at set-up), coefficient of f and leading term in
//    double-float, as IMRPhenomXAS's FP32 phase.
// t_c multiplies every mode by exp(-2 pi i f t_c) (an extension; zero
// reproduces the reference).
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/waveformx_b200.h"
#include "dual_point.cuh"
#include "internal.h"
#include "point.cuh"
#include "setup_xhm.cuh"
#include "tables.cuh"

namespace wfx {

namespace {

constexpr int kXhmBlock = 128;
constexpr int kXhmBinariesPerBlock = 8;
constexpr int kModesOut = 5;

template <class S>
struct C2 {
  S re, im;
};

template <class S>
struct XhmRow;
// (kMinBlocks: the launch bound, blocks of 128 per SM; measured on the
// 4096 x 4017 batch: FP32 4 blocks 1.05 ms, 5 0.93, 6 0.89, 8 0.80 (64
// registers, a little spilled); FP64 4 blocks 2.45 ms, 6 2.24)
template <>
struct XhmRow<float> {
  static constexpr int kStride = kXhmStride32, kMode = kXhmModeStride32, kMinBlocks = 8;
};
template <>
struct XhmRow<double> {
  static constexpr int kStride = kXhmStride64, kMode = kXhmModeStride64, kMinBlocks = 6;
};

// FP32: atan(y / x) by the minimax atan of point.cuh (2.6e-7 absolute), moved
// to the quadrant of (x, y) (x < 0: plus or minus pi by the sign of y, signed
// zeros included); the modulus of O(1) values from the sum of squares; the
// sine and cosine of an angle reduced modulo 2 pi (2 pi in two floats) by
// the fast intrinsic. FP64: the library's functions.
__device__ __forceinline__ float m_atan2(float y, float x) {
  const float a = m_atan(__fdividef(y, x));
  return x < 0.0f ? a + copysignf(3.14159265358979323846f, y) : a;
}
__device__ __forceinline__ double m_atan2(double y, double x) { return atan2(y, x); }
__device__ __forceinline__ float m_hypot(float a, float b) { return sqrtf(__fmaf_rn(a, a, b * b)); }
__device__ __forceinline__ double m_hypot(double a, double b) { return hypot(a, b); }
__device__ __forceinline__ void full_sincos(float x, float* s, float* c) {
  const float k = rintf(x * kInvTwoPi);
  const float r = __fmaf_rn(-k, kTwoPiLo, __fmaf_rn(-k, kTwoPiHi, x));
  __sincosf(r, s, c);
}
__device__ __forceinline__ void full_sincos(double x, double* s, double* c) { sincos(x, s, c); }

// The amplitude (amp0 included, >= 0 but FALSE_ZERO) and the phase of the
// higher mode of table M (emm its m; mixing: the (3,2)) at one frequency;
// (c22, s22): the (2,2) mode without its anchor, A22 (cos, sin) of its
// phase (core.py:429-518, 524-547).
template <class S>
__device__ __forceinline__ void mode_point(const S* __restrict__ M, const S* __restrict__ H, const Freq<S>& q,
                                           int emm, bool mixing, S c22, S s22, const S* __restrict__ T22, S t0_lm,
                                           S& amp, S& phi) {
  using namespace xhm;
  constexpr bool kF32 = sizeof(S) == 4;
  const S f = q.f, t = q.t, m1 = q.m1, lf = q.lf;
  const S t2 = t * t, mt1 = t2 * m1, m2 = m1 * m1;
  const S s = H[H_S], amp0 = H[H_AMP0];
  const bool past_ins = f >= M[M_F_PHASE_IN];
  const bool rd_phase = f >= M[M_F_PHASE_IM];
  const int region = rd_phase ? 2 : (past_ins ? 1 : 0);
  const S* R = M + M_PHASE + region * kBasis;
  // the region's sum (core.py:453-460), but (FP32) its constant and its
  // coefficient of f, which go in double-float below
  S sum = kF32 ? S(0) : R[B_1] + R[B_F] * f;
  if (region == 0) {
    sum = sum + R[B_M4_3] * (m1 * mt1);
    sum = sum + R[B_M1] * m1;
    sum = sum + R[B_M2_3] * (mt1 * mt1);
    sum = sum + R[B_M1_3] * mt1;
    sum = sum + R[B_1_3] * t;
    sum = sum + R[B_2_3] * t2;
    sum = sum + R[B_4_3] * (f * t);
    sum = sum + R[B_5_3] * (f * t2);
    sum = sum + R[B_F2] * (f * f);
    sum = sum + R[B_7_3] * (f * f * t);
    sum = sum + R[B_LOG] * lf;
    sum = sum + R[B_1_3_LOG] * (t * lf);
    sum = sum + R[B_F_LOG] * (f * lf);
    sum = sum + R[B_4_3_LOG] * (f * t * lf);
  } else if (region == 1) {
    sum = sum + R[B_LOG] * lf;
    sum = sum + R[B_M1] * m1;
    sum = sum + R[B_M2] * m2;
    sum = sum + R[B_M3] * (m2 * m1);
  } else if (!mixing) {
    sum = sum + R[B_M1] * m1;
  }
  const S y = f - M[M_SHIFT];
  const bool amp_rd_region = f >= M[M_F_AMP_IM];
  // the ringdown amplitude: the Lorentzian, the fall-off, the cubic of the
  // (3,2) below f_aux; then the (3,2)'s rotation (core.py:462-497)
  S amp_rd = S(0), rest_rd = S(0);
  if (rd_phase || amp_rd_region) {
    const S u = s * y;
    S arg = M[M_RD + 1] * u;
    arg = arg < S(-30) ? S(-30) : (arg > S(30) ? S(30) : arg);
    const S lor = m_div(M[M_RD + 0], m_exp(arg) * (u * u + M[M_RD + 2]));
    const S fo2 = M[M_FALLOFF + 2];
    const S over = f - fo2;
    const S fall = M[M_FALLOFF + 0] * m_exp(-M[M_FALLOFF + 1] * (over > S(0) ? over : S(0)));
    amp_rd = f >= fo2 ? fall : lor;
    const S at_rd = M[M_ATAN_A + 2] * m_atan(M[M_ATAN_W + 2] * y);
    if (mixing) {
      const S* a = M + M_AUX;
      const S aux = ((a[3] * f + a[2]) * f + a[1]) * f + a[0];
      amp_rd = f < M[M_F_AUX] ? aux : amp_rd;
      const S phi_s = M[M_SPH + 0] * f + M[M_SPH + 1] + M[M_SPH + 2] * m1 + M[M_SPH + 3] * (m2 * m1) + at_rd;
      S sn, cn;
      full_sincos(phi_s, &sn, &cn);
      const S cs = amp_rd * cn, ss = amp_rd * sn;
      const S m2r = M[M_MIX + 0], m2i = M[M_MIX + 1], m3r = M[M_MIX + 2], m3i = M[M_MIX + 3];
      const S re = c22 * m2r + s22 * m2i + cs * m3r + ss * m3i;
      const S im = s22 * m2r - c22 * m2i + ss * m3r - cs * m3i;
      const bool nonzero = (m_abs(re) > m_abs(im) ? m_abs(re) : m_abs(im)) > 1e-37;
      amp_rd = nonzero ? m_hypot(re, im) : S(0);
      rest_rd = nonzero ? m_atan2(im, re) : S(0);
    } else {
      rest_rd = at_rd;
    }
  }
  S rest;
  if (region == 2) {
    rest = sum + rest_rd;
  } else if (region == 1) {
    rest = sum + M[M_ATAN_A + 1] * m_atan(M[M_ATAN_W + 1] * y);
  } else {
    rest = sum;
  }
  // the amplitude (core.py:500-517)
  S a;
  if (f < M[M_F_AMP_IN]) {
    S pr = M[M_PN_RE + 6], pi = M[M_PN_IM + 6];
#pragma unroll
    for (int k = 5; k >= 0; --k) {
      pr = pr * t + M[M_PN_RE + k];
      pi = pi * t + M[M_PN_IM + k];
    }
    const S t3 = t * t * t;
    const S t7 = t3 * t3 * t;
    const S pseudo = t7 * (M[M_PSEUDO + 0] + t * (M[M_PSEUDO + 1] + t * M[M_PSEUDO + 2]));
    a = q.m76 * (m_hypot(pr, pi) + pseudo);
  } else if (amp_rd_region) {
    a = amp_rd;
  } else {
    const S v = (f - M[M_INTER_C]) * M[M_INTER_H];
    S inter = M[M_INTER + 7];
#pragma unroll
    for (int j = 6; j >= 0; --j) inter = inter * v + M[M_INTER + j];
    a = q.m76 * inter;
  }
  amp = a < S(0) ? S(kFalseZero) * amp0 : a;
  // the phase: [inspiral] T0_lm f^-5/3 - (m/2) A + rest, reduced
  const S m_over_2 = S(emm) * S(0.5);
  if constexpr (kF32) {
    const int cs = M_PHASE + region * kBasis + B_1, ls = M_PHASE + region * kBasis + B_F;
    const df p = two_prod(M[ls], f);
    S ph = M[cs] + reduce_df(p.hi, __fmaf_rn(M[HM32_LIN_LO + region], f, p.lo));
    if (!past_ins) {
      const df big = df_mul(df{M[HM32_T0_HI], M[HM32_T0_LO]}, q.y);
      ph = ph + reduce_df(big.hi, big.lo);
    }
    ph = ph + rest;
    const S k = round_nearest(ph * kInvTwoPi);
    ph = __fmaf_rn(-k, kTwoPiHi, ph);
    phi = __fmaf_rn(-k, kTwoPiLo, ph);
  } else {
    S ph = !past_ins ? t0_lm * q.y : S(0);
    ph = ph - m_over_2 * T22[X_ANCHOR];
    ph = ph + rest;
    phi = ph - m_round(ph / kTwoPi) * kTwoPi;
  }
}

// e^(-2 pi i f t_c) as (cos, sin).
__device__ __forceinline__ void tc_factor(float f, float t_c, float& c, float& s) {
  const TcF tc = make_tc(t_c);
  const df p = two_prod(tc.hi, f);
  const float ph = reduce_df(p.hi, __fmaf_rn(tc.lo, f, p.lo));
  __sincosf(-ph, &s, &c);
}
__device__ __forceinline__ void tc_factor(double f, double t_c, double& c, double& s) {
  double ph = kTwoPi * f * t_c;
  ph = ph - rint(ph / kTwoPi) * kTwoPi;
  sincos(-ph, &s, &c);
}

template <class S>
__global__ void __launch_bounds__(kXhmBlock, XhmRow<S>::kMinBlocks)
    k_xhm(const S* __restrict__ table, const S* __restrict__ freqs, const int64_t* __restrict__ offsets, int64_t B,
          int64_t n, const S* __restrict__ t_c, C2<S>* __restrict__ hp, C2<S>* __restrict__ hc,
          C2<S>* __restrict__ modes) {
  constexpr bool kF32 = sizeof(S) == 4;
  constexpr int kStride = XhmRow<S>::kStride, kMode = XhmRow<S>::kMode;
  __shared__ __align__(16) S T[kStride];
  __shared__ S t0_lm[4];  // (FP64) the rescaled leading term (m/2)^(8/3) T0 of each mode
  // (a shared grid with at most one frequency a thread: each thread's
  // frequency powers, computed for the block's first binary and read back
  // for the others)
  __shared__ Freq<S> powers[kXhmBlock];
  const bool reuse = offsets == nullptr && n <= static_cast<int64_t>(gridDim.x) * blockDim.x;
  bool have_powers = false;
  for (int64_t b = blockIdx.y; b < B; b += gridDim.y) {
    __syncthreads();  // (T is rewritten)
    for (int k = threadIdx.x; k < kStride; k += blockDim.x) T[k] = table[b * kStride + k];
    if (!kF32 && threadIdx.x < 4) {
      const int m = threadIdx.x;
      const double emm = m == 0 ? 1.0 : (m == 1 ? 3.0 : (m == 2 ? 2.0 : 4.0));
      t0_lm[m] = S(pow(emm * 0.5, 8.0 / 3.0) * double(table[b * kStride + X_T0]));
    }
    __syncthreads();
    if constexpr (kF32) {
      if (threadIdx.x == 0) {
        const int cs[3] = {xas_const_slot(0), xas_const_slot(1), xas_const_slot(2)};
        const int ls[3] = {xas_lin_slot(0), xas_lin_slot(1), xas_lin_slot(2)};
        prepare_f32<3>(T, cs, X32_CONST_LO, ls, X32_LIN_LO, 0.0f);
      }
      __syncthreads();
    }
    const S tcb = t_c != nullptr ? t_c[b] : S(0);

    const S* Hd = T;
    // (a shared grid: frequencies [0, n), outputs at b n + j; ragged: the
    // binary's own [offsets[b], offsets[b + 1]) of the flat arrays, clamped
    // to [0, n]: inconsistent offsets read and write nothing out of bounds)
    const int64_t lo = offsets != nullptr ? min(max(offsets[b], int64_t(0)), n) : 0;
    const int64_t hi = offsets != nullptr ? min(max(offsets[b + 1], lo), n) : n;
    const int64_t row = offsets != nullptr ? 0 : b * n;
    for (int64_t j = lo + static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < hi;
         j += static_cast<int64_t>(gridDim.x) * blockDim.x) {
      const S f = freqs[j];
      Freq<S> q;
      if (reuse && have_powers) {
        q = powers[threadIdx.x];
      } else {
        q = freq_powers(f);
        if (reuse) {
          powers[threadIdx.x] = q;
          have_powers = true;
        }
      }
      typename TcOf<S>::type zero{};
      const Point<S> p22 = xas_point<S>(T, q, zero);
      S tcc = S(1), tcs = S(0);
      if (t_c != nullptr) tc_factor(f, tcb, tcc, tcs);
      C2<S> sp{S(0), S(0)}, sc{S(0), S(0)};
      // adds mode k (t_c applied) to the polarizations, and writes it
      auto add = [&](int k, S re, S im) {
        const S* F = Hd + H_FACTORS + 4 * k;
        const C2<S> x{re * tcc - im * tcs, im * tcc + re * tcs};
        sp.re = sp.re + (F[0] * x.re - F[1] * x.im);
        sp.im = sp.im + (F[0] * x.im + F[1] * x.re);
        sc.re = sc.re + (F[2] * x.re - F[3] * x.im);
        sc.im = sc.im + (F[2] * x.im + F[3] * x.re);
        if (modes != nullptr) modes[(b * kModesOut + k) * n + j] = x;
      };
      const S h22r = p22.amp * p22.c, h22i = p22.amp * p22.s;
      add(0, h22r, h22i);
      // the (2,2) without its anchor: the angle turned by A
      const S ca = Hd[H_COS_A], sa = Hd[H_SIN_A];
      const S c22 = h22r * ca - h22i * sa, s22 = h22i * ca + h22r * sa;
#pragma unroll 1
      for (int m = 0; m < 4; ++m) {
        const S* M = T + H_MODES + m * kMode;
        const int emm = m == 0 ? 1 : (m == 1 ? 3 : (m == 2 ? 2 : 4));
        S amp, phi;
        mode_point<S>(M, Hd, q, emm, m == 2, c22, s22, T, t0_lm[m], amp, phi);
        const S sign = (m == 0 || m == 3) ? S(1) : S(-1);  // (-1)^l
        const S a = sign * M[xhm::M_ON] * amp;
        S sn, cn;
        m_sincos(phi, &sn, &cn);
        add(m + 1, a * cn, a * sn);
      }
      hp[row + j] = sp;
      hc[row + j] = sc;
    }
  }
}

// (h+, hx) of IMRPhenomXHM on dual numbers at the powers q of one frequency,
// the modes summed as k_xhm sums them; (tcc, tcs) = e^(-2 pi i f t_c) as
// (cos, sin), double where it carries no derivative, Dual where it does.
template <class TC>
__device__ __forceinline__ void xhm_dual_sum(const Dual* T, const Dual* t0_lm, const Freq<Dual>& q, TC tcc, TC tcs,
                                             C2<Dual>& sp, C2<Dual>& sc) {
  constexpr int kMode = kXhmModeStride64;
  const Point<Dual> p22 = xas_point<Dual>(T, q, 0.0);
  sp = C2<Dual>{Dual(0.0), Dual(0.0)};
  sc = C2<Dual>{Dual(0.0), Dual(0.0)};
  auto add = [&](int k, Dual re, Dual im) {
    const Dual* F = T + H_FACTORS + 4 * k;
    const C2<Dual> x{re * tcc - im * tcs, im * tcc + re * tcs};
    sp.re = sp.re + (F[0] * x.re - F[1] * x.im);
    sp.im = sp.im + (F[0] * x.im + F[1] * x.re);
    sc.re = sc.re + (F[2] * x.re - F[3] * x.im);
    sc.im = sc.im + (F[2] * x.im + F[3] * x.re);
  };
  const Dual h22r = p22.amp * p22.c, h22i = p22.amp * p22.s;
  add(0, h22r, h22i);
  const Dual ca = T[H_COS_A], sa = T[H_SIN_A];
  const Dual c22 = h22r * ca - h22i * sa, s22 = h22i * ca + h22r * sa;
#pragma unroll 1
  for (int m = 0; m < 4; ++m) {
    const Dual* M = T + H_MODES + m * kMode;
    const int emm = m == 0 ? 1 : (m == 1 ? 3 : (m == 2 ? 2 : 4));
    Dual amp, phi;
    mode_point<Dual>(M, T, q, emm, m == 2, c22, s22, T, t0_lm[m], amp, phi);
    const double sign = (m == 0 || m == 3) ? 1.0 : -1.0;  // (-1)^l
    const Dual a = sign * M[xhm::M_ON] * amp;
    Dual sn, cn;
    m_sincos(phi, &sn, &cn);
    add(m + 1, a * cn, a * sn);
  }
}

// IMRPhenomXHM's gradient, as the reference's GPU port takes it (forward-mode
// derivatives contracted with the cotangents in a kernel,
// models/xhm/mlx/_api.py:30-46): for direction d = blockIdx.z < 8,
// grad[b][d] += sum_f Re(conj(g+) dh+ + conj(gx) dhx), dh the derivative of
// the FP64 evaluation along the table's tangent dtable[b][.][d] (the set-up's
// derivative along parameter d); the blocks of d = 0 also sum t_c's,
// dh = -2 pi i f h, from the values they evaluate (a dual number's value
// does not depend on its tangent) into grad[b][8]. grad is zeroed
// beforehand; one atomic per block, binary and sum. (Four blocks per SM:
// 35 ms for 4096 x 4017, 50 ms unbounded.)
__global__ void __launch_bounds__(kXhmBlock, 4)
    k_xhm_jvp(const double* __restrict__ table, const double* __restrict__ dtable, const double* __restrict__ freqs,
              const int64_t* __restrict__ offsets, int64_t B, int64_t n, const double* __restrict__ t_c,
              const C2<double>* __restrict__ g_p, const C2<double>* __restrict__ g_c, double* __restrict__ grad) {
  constexpr int kStride = kXhmStride64;
  // (Dual has a constructor: raw storage, every entry written before read)
  __shared__ __align__(16) double t_raw[2 * kStride];
  __shared__ __align__(16) double t0_raw[2 * 4];
  Dual* T = reinterpret_cast<Dual*>(t_raw);
  Dual* t0_lm = reinterpret_cast<Dual*>(t0_raw);
  __shared__ double red[2][kXhmBlock / 32];
  const int dir = static_cast<int>(blockIdx.z);
  for (int64_t b = blockIdx.y; b < B; b += gridDim.y) {
    __syncthreads();  // (T and red are rewritten)
    for (int k = threadIdx.x; k < kStride; k += blockDim.x) {
      const int64_t at = b * kStride + k;
      T[k] = Dual(table[at], dtable[at * 8 + dir]);
    }
    if (threadIdx.x < 4) {
      const int m = threadIdx.x;
      const double emm = m == 0 ? 1.0 : (m == 1 ? 3.0 : (m == 2 ? 2.0 : 4.0));
      const int64_t at = b * kStride + X_T0;
      t0_lm[m] = pow(emm * 0.5, 8.0 / 3.0) * Dual(table[at], dtable[at * 8 + dir]);
    }
    __syncthreads();
    const double tcb = t_c != nullptr ? t_c[b] : 0.0;
    const int64_t lo = offsets != nullptr ? min(max(offsets[b], int64_t(0)), n) : 0;
    const int64_t hi = offsets != nullptr ? min(max(offsets[b + 1], lo), n) : n;
    const int64_t row = offsets != nullptr ? 0 : b * n;
    double acc = 0.0, acc_tc = 0.0;
    for (int64_t j = lo + static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; j < hi;
         j += static_cast<int64_t>(gridDim.x) * blockDim.x) {
      const double f = freqs[j];
      const Freq<Dual> q = lift(freq_powers(f));
      double tcc = 1.0, tcs = 0.0;
      if (t_c != nullptr) tc_factor(f, tcb, tcc, tcs);
      C2<Dual> sp, sc;
      xhm_dual_sum(T, t0_lm, q, tcc, tcs, sp, sc);
      const C2<double> gp = g_p[row + j], gc = g_c[row + j];
      acc += gp.re * sp.re.d + gp.im * sp.im.d + gc.re * sc.re.d + gc.im * sc.im.d;
      if (dir == 0) {
        const double w = kTwoPi * f;  // d/dt_c of h e^(-2 pi i f t_c): (w Im h, -w Re h)
        acc_tc += gp.re * (w * sp.im.v) - gp.im * (w * sp.re.v) + gc.re * (w * sc.im.v) - gc.im * (w * sc.re.v);
      }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      acc += __shfl_xor_sync(0xffffffffu, acc, o);
      acc_tc += __shfl_xor_sync(0xffffffffu, acc_tc, o);
    }
    if ((threadIdx.x & 31) == 0) {
      red[0][threadIdx.x >> 5] = acc;
      red[1][threadIdx.x >> 5] = acc_tc;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      double total = 0.0, total_tc = 0.0;
      for (int w = 0; w < kXhmBlock / 32; ++w) {
        total += red[0][w];
        total_tc += red[1][w];
      }
      atomicAdd(&grad[b * 9 + dir], total);
      if (dir == 0) atomicAdd(&grad[b * 9 + 8], total_tc);
    }
  }
}

// IMRPhenomXHM's derivative with respect to the grid (the reference's
// drop-in differentiates its model with respect to the frequencies,
// src/waveformx/torch.py:87-91; models/xhm/model.py:40 takes the set-up's
// first frequency without a derivative): the FP64 evaluation of k_xhm_jvp
// with the table's tangents zero and the frequency's powers carrying d/df
// (freq_powers_dual), e^(-2 pi i f t_c) differentiated in f too, contracted
// with the cotangents: d[b][j] = Re(conj(g+) dh+/df + conj(gx) dhx/df).
// Blocks (run of kXhmBlock frequencies, group): on a shared grid a group is
// kXhmBinariesPerBlock consecutive binaries, whose terms each thread sums
// before one atomic per element and group into grad_f (n, zeroed
// beforehand); on a ragged grid a group is one binary, whose elements are
// its own (stored). The offsets are clamped to [0, n].
__global__ void __launch_bounds__(kXhmBlock, 4)
    k_xhm_grid_vjp(const double* __restrict__ table, const double* __restrict__ freqs,
                   const int64_t* __restrict__ offsets, int64_t B, int64_t n, const double* __restrict__ t_c,
                   const C2<double>* __restrict__ g_p, const C2<double>* __restrict__ g_c,
                   double* __restrict__ grad_f) {
  constexpr int kStride = kXhmStride64;
  // (Dual has a constructor: raw storage, every entry written before read)
  __shared__ __align__(16) double t_raw[2 * kStride];
  __shared__ __align__(16) double t0_raw[2 * 4];
  Dual* T = reinterpret_cast<Dual*>(t_raw);
  Dual* t0_lm = reinterpret_cast<Dual*>(t0_raw);
  const bool ragged = offsets != nullptr;
  const int64_t group = ragged ? 1 : kXhmBinariesPerBlock;
  const int64_t groups = (B + group - 1) / group;
  for (int64_t g = blockIdx.y; g < groups; g += gridDim.y) {
    const int64_t b0 = g * group, b1 = min(b0 + group, B);
    const int64_t lo = ragged ? min(max(offsets[b0], int64_t(0)), n) : 0;
    const int64_t hi = ragged ? min(max(offsets[b0 + 1], lo), n) : n;
    for (int64_t j0 = static_cast<int64_t>(blockIdx.x) * blockDim.x; j0 < hi - lo;
         j0 += static_cast<int64_t>(gridDim.x) * blockDim.x) {
      const int64_t j = lo + j0 + threadIdx.x;
      const bool in = j < hi;
      const double f = in ? freqs[j] : 0.0;
      double acc = 0.0;
      for (int64_t b = b0; b < b1; ++b) {
        __syncthreads();  // (T is rewritten)
        for (int k = threadIdx.x; k < kStride; k += blockDim.x) T[k] = Dual(table[b * kStride + k], 0.0);
        if (threadIdx.x < 4) {
          const int m = threadIdx.x;
          const double emm = m == 0 ? 1.0 : (m == 1 ? 3.0 : (m == 2 ? 2.0 : 4.0));
          t0_lm[m] = Dual(pow(emm * 0.5, 8.0 / 3.0) * table[b * kStride + X_T0], 0.0);
        }
        __syncthreads();
        if (!in) continue;
        const Freq<Dual> q = freq_powers_dual(f);
        // e^(-2 pi i f t_c) = (c, s) and its derivative 2 pi t_c (s, -c)
        double c = 1.0, sn = 0.0;
        const double tcb = t_c != nullptr ? t_c[b] : 0.0;
        if (t_c != nullptr) tc_factor(f, tcb, c, sn);
        const double w = kTwoPi * tcb;
        C2<Dual> sp, sc;
        xhm_dual_sum(T, t0_lm, q, Dual(c, w * sn), Dual(sn, -w * c), sp, sc);
        const int64_t e = ragged ? j : b * n + j;
        const C2<double> gp = g_p[e], gc = g_c[e];
        acc += gp.re * sp.re.d + gp.im * sp.im.d + gc.re * sc.re.d + gc.im * sc.im.d;
      }
      if (!in) continue;
      if (ragged) {
        grad_f[j] = acc;
      } else {
        atomicAdd(&grad_f[j], acc);
      }
    }
  }
}

int launched() {
  const cudaError_t err = cudaGetLastError();
  return err == cudaSuccess ? 0 : static_cast<int>(err);
}

}  // namespace

int xhm_grid_vjp(const double* table, const double* freqs, const int64_t* offsets, int64_t B, int64_t n,
                 const double* t_c, const void* cot_hp, const void* cot_hc, double* grad_f, cudaStream_t s) {
  // (a run of frequencies per block; on a ragged grid enough runs for the
  // rows' mean length, longer rows looping in their blocks)
  const int64_t span = offsets != nullptr ? (n + B - 1) / B : n;
  const int64_t runs = (span + kXhmBlock - 1) / kXhmBlock;
  const int64_t groups = offsets != nullptr ? B : (B + kXhmBinariesPerBlock - 1) / kXhmBinariesPerBlock;
  const dim3 grid(static_cast<unsigned>(runs < 1024 ? runs : 1024),
                  static_cast<unsigned>(groups < 65535 ? groups : 65535));
  k_xhm_grid_vjp<<<grid, kXhmBlock, 0, s>>>(table, freqs, offsets, B, n, t_c,
                                            static_cast<const C2<double>*>(cot_hp),
                                            static_cast<const C2<double>*>(cot_hc), grad_f);
  return launched();
}

}  // namespace wfx

using namespace wfx;

extern "C" {

int wfx_xhm_polarizations(int precision, const void* table, const void* freqs, const int64_t* offsets, int64_t B,
                          int64_t n, int64_t max_len, const void* t_c, void* hp, void* hc, void* modes,
                          wfx_stream_t stream) {
  if (table == nullptr || freqs == nullptr || hp == nullptr || hc == nullptr || B <= 0 || n <= 0) return WFX_EINVAL;
  if ((reinterpret_cast<uintptr_t>(table) & 15u) != 0) return WFX_EINVAL;
  if (offsets != nullptr && (modes != nullptr || max_len <= 0)) return WFX_EINVAL;
  const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const int64_t span = offsets != nullptr ? max_len : n;
  const int64_t runs = (span + kXhmBlock - 1) / kXhmBlock;
  // (a shared grid: kXhmBinariesPerBlock binaries a block, which share the
  // frequencies' powers; a ragged one: one binary a block)
  const int64_t rows = offsets != nullptr ? B : (B + kXhmBinariesPerBlock - 1) / kXhmBinariesPerBlock;
  const dim3 grid(static_cast<unsigned>(runs < 4096 ? runs : 4096), static_cast<unsigned>(rows < 65535 ? rows : 65535));
  if (precision == WFX_FP32) {
    k_xhm<float><<<grid, kXhmBlock, 0, s>>>(static_cast<const float*>(table), static_cast<const float*>(freqs), offsets,
                                             B, n,
                                             static_cast<const float*>(t_c), static_cast<C2<float>*>(hp),
                                             static_cast<C2<float>*>(hc), static_cast<C2<float>*>(modes));
  } else if (precision == WFX_FP64) {
    k_xhm<double><<<grid, kXhmBlock, 0, s>>>(static_cast<const double*>(table), static_cast<const double*>(freqs),
                                              offsets, B, n, static_cast<const double*>(t_c), static_cast<C2<double>*>(hp),
                                              static_cast<C2<double>*>(hc), static_cast<C2<double>*>(modes));
  } else {
    return WFX_EINVAL;
  }
  return launched();
}

int wfx_xhm_vjp(const double* table, const double* dtable, const double* freqs, const int64_t* offsets, int64_t B,
                int64_t n, int64_t max_len, const double* t_c, const void* cot_hp, const void* cot_hc, double* grad,
                wfx_stream_t stream) {
  if (table == nullptr || dtable == nullptr || freqs == nullptr || cot_hp == nullptr || cot_hc == nullptr ||
      grad == nullptr || B <= 0 || n <= 0 || (offsets != nullptr && max_len <= 0))
    return WFX_EINVAL;
  const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const cudaError_t rc = cudaMemsetAsync(grad, 0, sizeof(double) * 9 * static_cast<size_t>(B), s);
  if (rc != cudaSuccess) return static_cast<int>(rc);
  const int64_t span = offsets != nullptr ? max_len : n;
  const int64_t runs = (span + kXhmBlock - 1) / kXhmBlock;
  const dim3 grid(static_cast<unsigned>(runs < 1024 ? runs : 1024), static_cast<unsigned>(B < 65535 ? B : 65535), 8);
  k_xhm_jvp<<<grid, kXhmBlock, 0, s>>>(table, dtable, freqs, offsets, B, n, t_c, static_cast<const C2<double>*>(cot_hp),
                                       static_cast<const C2<double>*>(cot_hc), grad);
  return launched();
}

}  // extern "C"
