// The match of waveforms maximised over a time shift and a constant phase
// (src/waveformx/match.py:71-147) for sm_100a, and its C-ABI entries.
//
//  * k_overlap: c[r][k] = 4 delta_f a[r][k] conj(b[r][k]) / S[k] (the
//    summand of the overlap z(t) = sum_k c_k e^(2 pi i f_k t)) into a
//    zero-padded series, and the norms <a, a>, <b, b> of each row.
//  * (the caller's inverse FFT of the series, cuFFT, gives z on the times
//    j / (n_fft delta_f) of one period)
//  * k_match_refine: one warp per row: the best time of that grid (the
//    largest |z| or, without the phase, Re z), wrapped to (-P/2, P/2], then
//    Newton steps on the exact z(t) at the frequencies, each kept only if it
//    does not lower the objective, as the reference's _refine; in FP64.
//
// The template-bank form of k_overlap, whose templates are evaluated from
// their tables without writing the strain, is in kernels.cu
// (k_template_overlap).
#include <cuda_runtime.h>

#include <cstdint>

#include "../../include/waveformx_b200.h"

namespace wfx {
namespace {

constexpr int kMatchBlock = 256;
constexpr double kPi = 3.141592653589793;

template <class R>
struct Cplx;
template <>
struct Cplx<float> {
  using type = float2;
};
template <>
struct Cplx<double> {
  using type = double2;
};

// Sums v over the block (every thread gets the sum); `scratch` holds one
// value per warp.
__device__ __forceinline__ double block_sum(double v, double* scratch) {
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) scratch[warp] = v;
  __syncthreads();
  double total = 0.0;
#pragma unroll
  for (int w = 0; w < kMatchBlock / 32; ++w) total += scratch[w];
  return total;
}

template <class R>
__global__ void __launch_bounds__(kMatchBlock) k_overlap(const typename Cplx<R>::type* __restrict__ a,
                                                         int64_t a_stride,
                                                         const typename Cplx<R>::type* __restrict__ b,
                                                         int64_t b_stride, const R* __restrict__ psd, int64_t rows,
                                                         int64_t n, R scale, typename Cplx<R>::type* __restrict__ out,
                                                         int64_t n_fft, double* __restrict__ norms) {
  // scale = 4 delta_f (match.py:84-88)
  __shared__ double scratch[kMatchBlock / 32];
  for (int64_t r = blockIdx.x; r < rows; r += gridDim.x) {
    const auto* ar = a + r * a_stride;
    const auto* br = b + r * b_stride;
    auto* cr = out + r * n_fft;
    double aa = 0.0, bb = 0.0;
    for (int64_t k = threadIdx.x; k < n; k += kMatchBlock) {
      const auto x = ar[k], y = br[k];
      const R s = psd[k];
      // c = 4 df x conj(y) / S, in the reference's order of operations
      const R re = x.x * y.x + x.y * y.y, im = x.y * y.x - x.x * y.y;
      typename Cplx<R>::type c;
      c.x = scale * re / s;
      c.y = scale * im / s;
      cr[k] = c;
      aa += static_cast<double>((x.x * x.x + x.y * x.y) / s);
      bb += static_cast<double>((y.x * y.x + y.y * y.y) / s);
    }
    aa = block_sum(aa, scratch);
    bb = block_sum(bb, scratch);
    if (threadIdx.x == 0) {
      norms[2 * r] = static_cast<double>(scale) * aa;
      norms[2 * r + 1] = static_cast<double>(scale) * bb;
    }
  }
}

// polarization_match's series (match.py:162-172): rows 2 r and 2 r + 1 of
// `out` are 4 delta_f s conj(h+) / S and 4 delta_f s conj(hx) / S of row r,
// and norms[4 r ..] = <s, s>, <h+, h+>, <hx, hx>, <h+, hx>.
template <class R>
__global__ void __launch_bounds__(kMatchBlock) k_polarization_overlap(
    const typename Cplx<R>::type* __restrict__ sig, int64_t s_stride, const typename Cplx<R>::type* __restrict__ hp,
    int64_t p_stride, const typename Cplx<R>::type* __restrict__ hx, int64_t x_stride, const R* __restrict__ psd,
    int64_t rows, int64_t n, R scale, typename Cplx<R>::type* __restrict__ out, int64_t n_fft,
    double* __restrict__ norms) {
  __shared__ double scratch[kMatchBlock / 32];
  for (int64_t r = blockIdx.x; r < rows; r += gridDim.x) {
    const auto* sr = sig + r * s_stride;
    const auto* pr = hp + r * p_stride;
    const auto* xr = hx + r * x_stride;
    auto* cp = out + 2 * r * n_fft;
    auto* cx = cp + n_fft;
    double ss = 0.0, pp = 0.0, xx = 0.0, px = 0.0;
    for (int64_t k = threadIdx.x; k < n; k += kMatchBlock) {
      const auto a = sr[k], p = pr[k], x = xr[k];
      const R w = psd[k];
      typename Cplx<R>::type c;
      c.x = scale * (a.x * p.x + a.y * p.y) / w;
      c.y = scale * (a.y * p.x - a.x * p.y) / w;
      cp[k] = c;
      c.x = scale * (a.x * x.x + a.y * x.y) / w;
      c.y = scale * (a.y * x.x - a.x * x.y) / w;
      cx[k] = c;
      ss += static_cast<double>((a.x * a.x + a.y * a.y) / w);
      pp += static_cast<double>((p.x * p.x + p.y * p.y) / w);
      xx += static_cast<double>((x.x * x.x + x.y * x.y) / w);
      px += static_cast<double>((p.x * x.x + p.y * x.y) / w);
    }
    ss = block_sum(ss, scratch);
    pp = block_sum(pp, scratch);
    xx = block_sum(xx, scratch);
    px = block_sum(px, scratch);
    if (threadIdx.x == 0) {
      const double sc = static_cast<double>(scale);
      norms[4 * r] = sc * ss;
      norms[4 * r + 1] = sc * pp;
      norms[4 * r + 2] = sc * xx;
      norms[4 * r + 3] = sc * px;
    }
  }
}

constexpr int kRowsPerBlock = kMatchBlock / 32;  // k_match_refine: one warp per row

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
  return v;
}

// e^(2 pi i x) for x in turns (its nearest integer taken off first).
__device__ __forceinline__ void cis_turns(double x, double& c, double& s) {
  x -= rint(x);
  sincospi(2.0 * x, &s, &c);
}

// The overlap z and its first two derivatives in t at the time t, from a
// row's series c at the frequencies f: sum_k c_k (2 pi i f_k)^p e^(2 pi i
// f_k t), p = 0, 1, 2, as z[0..5] = (Re, Im) of each; every lane of the
// warp gets the sums. Lane l takes the terms k = l + 32 i, eight at a time
// (their loads issued together): the phase factor is e^(2 pi i f_k t)
// itself for the first of the eight and is advanced by the rotation
// e^(2 pi i 32 delta_f t) for the others (a uniform grid).
template <class C>
__device__ void z_derivatives(const C* __restrict__ c, const double* __restrict__ f, int64_t n, double t,
                              double delta_f, int lane, double (&z)[6]) {
  constexpr int kGroup = 8;  // terms per lane between exact phase factors (their loads issued together)
  double rc, rs;
  cis_turns(32.0 * delta_f * t, rc, rs);
  double s[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  for (int64_t k0 = lane; k0 < n; k0 += 32 * kGroup) {
    double fk[kGroup], cr[kGroup], ci[kGroup];
#pragma unroll
    for (int u = 0; u < kGroup; ++u) {
      const int64_t k = k0 + 32 * u;
      const bool in = k < n;
      fk[u] = in ? f[k] : 0.0;
      cr[u] = in ? static_cast<double>(c[k].x) : 0.0;
      ci[u] = in ? static_cast<double>(c[k].y) : 0.0;
    }
    double wc, ws;
    cis_turns(fk[0] * t, wc, ws);
#pragma unroll
    for (int u = 0; u < kGroup; ++u) {
      // (terms past n are zero)
      const double wr = cr[u] * wc - ci[u] * ws, wi = cr[u] * ws + ci[u] * wc;  // c e^(2 pi i f t)
      const double om = 2.0 * kPi * fk[u];
      s[0] += wr;
      s[1] += wi;
      s[2] -= om * wi;  // i om (wr + i wi)
      s[3] += om * wr;
      s[4] -= om * om * wr;  // (i om)^2 = -om^2
      s[5] -= om * om * wi;
      const double nc = wc * rc - ws * rs, ns = wc * rs + ws * rc;
      wc = nc;
      ws = ns;
    }
  }
#pragma unroll
  for (int j = 0; j < 6; ++j) z[j] = warp_sum(s[j]);
}

__device__ __forceinline__ double objective(const double (&z)[6], bool phase) {
  return phase ? z[0] * z[0] + z[1] * z[1] : z[0];
}

// (v, j) of the larger value, the smaller index of equal ones (the first
// maximum, as an arg-max); j < 0: none.
__device__ __forceinline__ void keep_max(double& v, int64_t& j, double ov, int64_t oj) {
  if (oj >= 0 && (j < 0 || ov > v || (ov == v && oj < j))) {
    v = ov;
    j = oj;
  }
}

template <class R>
__global__ void __launch_bounds__(kMatchBlock) k_match_refine(const typename Cplx<R>::type* __restrict__ series,
                                                              const typename Cplx<R>::type* __restrict__ zgrid,
                                                              int64_t rows, int64_t n, int64_t n_fft,
                                                              const double* __restrict__ freqs, double delta_f,
                                                              const double* __restrict__ norms, int time, int phase,
                                                              int steps, double* __restrict__ match,
                                                              double* __restrict__ t_out) {
  const int lane = threadIdx.x & 31;
  const double f0 = freqs[0];
  const double denominator = static_cast<double>(n_fft) * delta_f;
  const int64_t warps = static_cast<int64_t>(gridDim.x) * kRowsPerBlock;
  for (int64_t r = static_cast<int64_t>(blockIdx.x) * kRowsPerBlock + (threadIdx.x >> 5); r < rows; r += warps) {
    const auto* c = series + r * n_fft;
    double t = 0.0;
    if (time == 2) {
      t = t_out[r];  // (the grid's best time, from k_grid_time)
    } else if (time) {
      // the grid's best time (match.py:118-126): the first largest value;
      // without the phase the value is Re z e^(2 pi i f0 t_j), the factor
      // advanced by a fixed rotation from one of a lane's samples to the
      // next
      const auto* z = zgrid + r * n_fft;
      double rc, rs, wc, ws;
      cis_turns(f0 * (32.0 / denominator), rc, rs);
      cis_turns(f0 * (static_cast<double>(lane) / denominator), wc, ws);
      double v_max = 0.0;
      int64_t j_max = -1;
      constexpr int kGroup = 8;  // samples per lane whose loads are issued together
      for (int64_t j0 = lane; j0 < n_fft; j0 += 32 * kGroup) {
        double zr[kGroup], zi[kGroup];
#pragma unroll
        for (int u = 0; u < kGroup; ++u) {
          const int64_t j = j0 + 32 * u;
          zr[u] = j < n_fft ? static_cast<double>(z[j].x) : 0.0;
          zi[u] = j < n_fft ? static_cast<double>(z[j].y) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < kGroup; ++u) {
          const int64_t j = j0 + 32 * u;
          const double v = phase ? zr[u] * zr[u] + zi[u] * zi[u] : zr[u] * wc - zi[u] * ws;
          if (j < n_fft) keep_max(v_max, j_max, v, j);
          const double nc = wc * rc - ws * rs, ns = wc * rs + ws * rc;
          wc = nc;
          ws = ns;
        }
      }
#pragma unroll
      for (int d = 16; d > 0; d >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, v_max, d);
        const int64_t oj = __shfl_xor_sync(0xffffffffu, j_max, d);
        keep_max(v_max, j_max, ov, oj);
      }
      // times j / (n_fft delta_f); the period is times[-1] + times[1]
      t = static_cast<double>(j_max < 0 ? 0 : j_max) / denominator;
      const double period = static_cast<double>(n_fft - 1) / denominator + 1.0 / denominator;
      if (t > period / 2) t -= period;
    }
    double z[6];
    z_derivatives(c, freqs, n, t, delta_f, lane, z);
    if (time) {
      for (int s = 0; s < steps; ++s) {
        // match.py:104-115 with the closed-form derivatives
        double g, h;
        if (phase) {
          g = 2.0 * (z[0] * z[2] + z[1] * z[3]);
          h = 2.0 * (z[2] * z[2] + z[3] * z[3] + z[0] * z[4] + z[1] * z[5]);
        } else {
          g = z[2];
          h = z[4];
        }
        const double next = t - (h < 0.0 ? g / h : 0.0);
        double zn[6];
        z_derivatives(c, freqs, n, next, delta_f, lane, zn);
        if (objective(zn, phase) >= objective(z, phase)) {
          t = next;
#pragma unroll
          for (int i = 0; i < 6; ++i) z[i] = zn[i];
        }
      }
    }
    if (lane == 0) {
      const double best = phase ? sqrt(z[0] * z[0] + z[1] * z[1]) : z[0];
      match[r] = best / sqrt(norms[2 * r] * norms[2 * r + 1]);
      if (t_out != nullptr) t_out[r] = t;
    }
  }
}

// polarization_match's objective square(Re zp, Re zx) (match.py:174-176)
// of a row: the normalised polarizations' overlap i, and the scales.
struct PolarizationForm {
  double inv_p, inv_x, i, q;  // 1 / sqrt(<h+, h+>), 1 / sqrt(<hx, hx>) (0 if parallel), I, 1 - I^2
  __device__ double value(double rp, double rx) const {
    const double a = rp * inv_p, b = rx * inv_x;
    return (a * a + b * b - 2.0 * a * b * i) / q;
  }
};

__device__ __forceinline__ PolarizationForm polarization_form(const double* norms) {
  const double pp = norms[1], xx = norms[2], px = norms[3];
  double i = px / sqrt(pp * xx);
  const bool degenerate = !(1.0 - i * i > 1e-10);
  PolarizationForm form;
  form.i = degenerate ? 0.0 : i;
  form.q = 1.0 - form.i * form.i;
  form.inv_p = 1.0 / sqrt(pp);
  form.inv_x = degenerate ? 0.0 : 1.0 / sqrt(xx);
  return form;
}

template <class R>
__global__ void __launch_bounds__(kMatchBlock) k_polarization_refine(
    const typename Cplx<R>::type* __restrict__ series, const typename Cplx<R>::type* __restrict__ zgrid, int64_t rows,
    int64_t n, int64_t n_fft, const double* __restrict__ freqs, double delta_f, const double* __restrict__ norms,
    int time, int steps, double* __restrict__ match, double* __restrict__ t_out) {
  const int lane = threadIdx.x & 31;
  const double f0 = freqs[0];
  const double denominator = static_cast<double>(n_fft) * delta_f;
  const int64_t warps = static_cast<int64_t>(gridDim.x) * kRowsPerBlock;
  for (int64_t r = static_cast<int64_t>(blockIdx.x) * kRowsPerBlock + (threadIdx.x >> 5); r < rows; r += warps) {
    const auto* cp = series + 2 * r * n_fft;
    const auto* cx = cp + n_fft;
    const PolarizationForm form = polarization_form(norms + 4 * r);
    double t = 0.0;
    if (time) {
      // the first largest square(Re zp e^(2 pi i f0 t_j), Re zx ...) of the
      // grid (match.py:178-181)
      const auto* zp = zgrid + 2 * r * n_fft;
      const auto* zx = zp + n_fft;
      double rc, rs, wc, ws;
      cis_turns(f0 * (32.0 / denominator), rc, rs);
      cis_turns(f0 * (static_cast<double>(lane) / denominator), wc, ws);
      double v_max = 0.0;
      int64_t j_max = -1;
      constexpr int kGroup = 8;
      for (int64_t j0 = lane; j0 < n_fft; j0 += 32 * kGroup) {
        double pr[kGroup], pi[kGroup], xr[kGroup], xi[kGroup];
#pragma unroll
        for (int u = 0; u < kGroup; ++u) {
          const int64_t j = j0 + 32 * u;
          const bool in = j < n_fft;
          pr[u] = in ? static_cast<double>(zp[j].x) : 0.0;
          pi[u] = in ? static_cast<double>(zp[j].y) : 0.0;
          xr[u] = in ? static_cast<double>(zx[j].x) : 0.0;
          xi[u] = in ? static_cast<double>(zx[j].y) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < kGroup; ++u) {
          const int64_t j = j0 + 32 * u;
          const double v = form.value(pr[u] * wc - pi[u] * ws, xr[u] * wc - xi[u] * ws);
          if (j < n_fft) keep_max(v_max, j_max, v, j);
          const double nc = wc * rc - ws * rs, ns = wc * rs + ws * rc;
          wc = nc;
          ws = ns;
        }
      }
#pragma unroll
      for (int d = 16; d > 0; d >>= 1) {
        const double ov = __shfl_xor_sync(0xffffffffu, v_max, d);
        const int64_t oj = __shfl_xor_sync(0xffffffffu, j_max, d);
        keep_max(v_max, j_max, ov, oj);
      }
      t = static_cast<double>(j_max < 0 ? 0 : j_max) / denominator;
      const double period = static_cast<double>(n_fft - 1) / denominator + 1.0 / denominator;
      if (t > period / 2) t -= period;
    }
    double zp[6], zx[6];
    z_derivatives(cp, freqs, n, t, delta_f, lane, zp);
    z_derivatives(cx, freqs, n, t, delta_f, lane, zx);
    if (time) {
      for (int s = 0; s < steps; ++s) {
        // Newton on Q(t) = square(Re zp(t), Re zx(t)) with its closed-form
        // derivatives (match.py:104-115 on this objective)
        const double a = zp[0] * form.inv_p, a1 = zp[2] * form.inv_p, a2 = zp[4] * form.inv_p;
        const double b = zx[0] * form.inv_x, b1 = zx[2] * form.inv_x, b2 = zx[4] * form.inv_x;
        const double g = (2.0 * a * a1 + 2.0 * b * b1 - 2.0 * form.i * (a1 * b + a * b1)) / form.q;
        const double h = (2.0 * a1 * a1 + 2.0 * a * a2 + 2.0 * b1 * b1 + 2.0 * b * b2 -
                          2.0 * form.i * (a2 * b + 2.0 * a1 * b1 + a * b2)) /
                         form.q;
        const double next = t - (h < 0.0 ? g / h : 0.0);
        double np_[6], nx[6];
        z_derivatives(cp, freqs, n, next, delta_f, lane, np_);
        z_derivatives(cx, freqs, n, next, delta_f, lane, nx);
        if (form.value(np_[0], nx[0]) >= form.value(zp[0], zx[0])) {
          t = next;
#pragma unroll
          for (int i = 0; i < 6; ++i) {
            zp[i] = np_[i];
            zx[i] = nx[i];
          }
        }
      }
    }
    if (lane == 0) {
      match[r] = sqrt(form.value(zp[0], zx[0]) / norms[4 * r]);
      if (t_out != nullptr) t_out[r] = t;
    }
  }
}

// ---------------------------------------------------------------------------
// The grid's best time without the grid in memory (the match with the phase
// maximisation, FP32 series). A row's series is zero from n on, so with L
// the power of two >= max(n, 2048) and n_fft = P L, the inverse transform
// splits into P transforms of length L of which nothing reads the zeros
// (decimation in frequency):
//   z[P k + r] = sum_{m < L} (c_m e^(2 pi i r m / n_fft)) e^(2 pi i m k / L).
// One block per row runs the P transforms one after the other in shared
// memory and keeps the first largest |z_j|^2 in registers; only the best
// time is written.
//
// A length-L transform: S radix-16 passes (a thread's 16 values in
// registers, a 16-point inverse DFT as two radix-4 steps, the twiddles by
// one sincospi and products; the first pass reads the row from global
// memory), then a last radix R = L / 16^S (16, 8, 4 or 2). The outputs are
// in digit-reversed order: the group g = sum_i d_i 16^(S-1-i) of R
// consecutive positions holds k = sum_i d_i 16^i + 16^S p at its p-th.
// Shared memory holds one value of padding after every 16, which keeps
// every pass's and the last radix's accesses free of bank conflicts.

// (also the host's size of the shared buffer)
__host__ __device__ constexpr int fft_pad(int i) { return i + (i >> 4); }

constexpr int ilog2(int v) { return v <= 1 ? 0 : 1 + ilog2(v / 2); }

template <int L>
struct GridShape {
  static_assert(L == 2048 || L == 4096 || L == 8192 || L == 16384, "transform length");
  static constexpr int kPasses = (ilog2(L) - 1) / 4;    // S
  static constexpr int kLast = L >> (4 * kPasses);       // R
  static constexpr int kThreads = L / 16;                // one first-pass butterfly each
  static constexpr int kBlocksPerSM = 1024 / kThreads;   // (64 registers a thread)
  static constexpr size_t kBytes = sizeof(float2) * static_cast<size_t>(fft_pad(L - 1) + 1);
};

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }

__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }

// The 4-point inverse DFT of (a, b, c, d) in place: sum_p x_p i^(p k).
__device__ __forceinline__ void idft4(float2& a, float2& b, float2& c, float2& d) {
  const float2 s0 = cadd(a, c), d0 = csub(a, c), s1 = cadd(b, d), d1 = csub(b, d);
  a = cadd(s0, s1);
  c = csub(s0, s1);
  b = make_float2(d0.x - d1.y, d0.y + d1.x);  // d0 + i d1
  d = make_float2(d0.x + d1.y, d0.y - d1.x);  // d0 - i d1
}

// The 8-point inverse DFT in place, natural order: the 4-point transforms
// of the even and odd terms, the odd ones turned by e^(2 pi i k / 8).
__device__ __forceinline__ void idft8(float2 (&x)[8]) {
  float2 e0 = x[0], e1 = x[2], e2 = x[4], e3 = x[6], o0 = x[1], o1 = x[3], o2 = x[5], o3 = x[7];
  idft4(e0, e1, e2, e3);
  idft4(o0, o1, o2, o3);
  constexpr float kR2 = 0.707106781186547524f;
  o1 = cmul(o1, make_float2(kR2, kR2));
  o2 = make_float2(-o2.y, o2.x);
  o3 = cmul(o3, make_float2(-kR2, kR2));
  x[0] = cadd(e0, o0);
  x[4] = csub(e0, o0);
  x[1] = cadd(e1, o1);
  x[5] = csub(e1, o1);
  x[2] = cadd(e2, o2);
  x[6] = csub(e2, o2);
  x[3] = cadd(e3, o3);
  x[7] = csub(e3, o3);
}

// The 16-point inverse DFT of x: y[k1 + 4 k2] = sum_p x[p] e^(2 pi i p k / 16),
// p = r + 4 s: a 4-point transform over s, the twiddles e^(2 pi i r k1 / 16),
// a 4-point transform over r; y returned in natural order.
__device__ __forceinline__ void idft16(float2 (&x)[16]) {
#pragma unroll
  for (int r = 0; r < 4; ++r) idft4(x[r], x[r + 4], x[r + 8], x[r + 12]);
  // (x[r + 4 k1] = A[r][k1])
  constexpr float kC1 = 0.923879532511286756f, kS1 = 0.382683432365089772f, kR2 = 0.707106781186547524f;
  x[1 + 4] = cmul(x[1 + 4], make_float2(kC1, kS1));      // r 1, k1 1: e^(2 pi i / 16)
  x[1 + 8] = cmul(x[1 + 8], make_float2(kR2, kR2));      // r 1, k1 2
  x[1 + 12] = cmul(x[1 + 12], make_float2(kS1, kC1));    // r 1, k1 3
  x[2 + 4] = cmul(x[2 + 4], make_float2(kR2, kR2));      // r 2, k1 1
  x[2 + 8] = make_float2(-x[2 + 8].y, x[2 + 8].x);       // r 2, k1 2: i
  x[2 + 12] = cmul(x[2 + 12], make_float2(-kR2, kR2));   // r 2, k1 3: e^(2 pi i 6 / 16)
  x[3 + 4] = cmul(x[3 + 4], make_float2(kS1, kC1));      // r 3, k1 1: e^(2 pi i 3 / 16)
  x[3 + 8] = cmul(x[3 + 8], make_float2(-kR2, kR2));     // r 3, k1 2
  x[3 + 12] = cmul(x[3 + 12], make_float2(-kC1, -kS1));  // r 3, k1 3: e^(2 pi i 9 / 16)
#pragma unroll
  for (int k1 = 0; k1 < 4; ++k1) idft4(x[4 * k1], x[4 * k1 + 1], x[4 * k1 + 2], x[4 * k1 + 3]);
  // (x[4 k1 + k2] = y[k1 + 4 k2]): to natural order
  float2 y[16];
#pragma unroll
  for (int k1 = 0; k1 < 4; ++k1) {
#pragma unroll
    for (int k2 = 0; k2 < 4; ++k2) y[k1 + 4 * k2] = x[4 * k1 + k2];
  }
#pragma unroll
  for (int k = 0; k < 16; ++k) x[k] = y[k];
}

// Multiplies y[p] by w^p, p = 1..15, w = e^(2 pi i q / LEN).
__device__ __forceinline__ void twiddle16(float2 (&y)[16], int q, int LEN) {
  float2 w1;
  sincospif(2.0f * static_cast<float>(q) / static_cast<float>(LEN), &w1.y, &w1.x);
  float2 w = w1;
#pragma unroll
  for (int p = 1; p < 16; ++p) {
    y[p] = cmul(y[p], w);
    w = cmul(w, w1);
  }
}

// A radix-16 pass of the length-L transform over its sub-transforms of
// length LEN (LEN / 16 > 1) in place.
template <int L, int LEN>
__device__ __forceinline__ void fft_pass16(float2* X) {
  constexpr int M = LEN / 16;
  for (int u = threadIdx.x; u < L / 16; u += blockDim.x) {
    const int b = u / M, q = u % M, base = b * LEN + q;
    float2 x[16];
#pragma unroll
    for (int p = 0; p < 16; ++p) x[p] = X[fft_pad(base + p * M)];
    idft16(x);
    twiddle16(x, q, LEN);
#pragma unroll
    for (int p = 0; p < 16; ++p) X[fft_pad(base + p * M)] = x[p];
  }
}

// The radix-16 passes after the first, down to sub-transforms of length R.
template <int L, int LEN>
__device__ __forceinline__ void fft_middle_passes(float2* X) {
  if constexpr (LEN > GridShape<L>::kLast) {
    fft_pass16<L, LEN>(X);
    __syncthreads();
    fft_middle_passes<L, LEN / 16>(X);
  }
}

// The base-16 digits of g (S of them) in reverse order.
template <int S>
__device__ __forceinline__ int reverse16(int g) {
  int k = 0;
#pragma unroll
  for (int i = 0; i < S; ++i) {
    k = (k << 4) | (g & 15);
    g >>= 4;
  }
  return k;
}

__device__ __forceinline__ void keep_max_f(float& v, int& j, float ov, int oj) {
  if (oj >= 0 && (j < 0 || ov > v || (ov == v && oj < j))) {
    v = ov;
    j = oj;
  }
}

template <int L>
__global__ void __launch_bounds__(GridShape<L>::kThreads, GridShape<L>::kBlocksPerSM)
    k_grid_time(const float2* __restrict__ series, int64_t rows, int64_t n, int64_t n_fft, double delta_f,
                double* __restrict__ t_out) {
  using G = GridShape<L>;
  constexpr int M = L / 16, R = G::kLast, S = G::kPasses;
  extern __shared__ float2 X[];
  __shared__ float best_v[32];
  __shared__ int best_j[32];
  const int P = static_cast<int>(n_fft / L);
  const int q = threadIdx.x;  // (blockDim.x == M)
  for (int64_t row = blockIdx.x; row < rows; row += gridDim.x) {
    const float2* c = series + row * n_fft;
    float v_max = 0.0f;
    int j_max = -1;
    for (int r = 0; r < P; ++r) {
      {
        // the first pass: the row turned by e^(2 pi i r m / n_fft)
        float2 w, step;
        sincospif(2.0f * static_cast<float>(r * q) / static_cast<float>(n_fft), &w.y, &w.x);
        sincospif(2.0f * static_cast<float>(r * M) / static_cast<float>(n_fft), &step.y, &step.x);
        float2 x[16];
#pragma unroll
        for (int p = 0; p < 16; ++p) x[p] = (q + p * M < n) ? c[q + p * M] : make_float2(0.f, 0.f);
#pragma unroll
        for (int p = 0; p < 16; ++p) {
          x[p] = cmul(x[p], w);
          w = cmul(w, step);
        }
        idft16(x);
        twiddle16(x, q, L);
#pragma unroll
        for (int p = 0; p < 16; ++p) X[fft_pad(q + p * M)] = x[p];
      }
      __syncthreads();
      fft_middle_passes<L, L / 16>(X);
      // the last radix and the largest value
      for (int g = threadIdx.x; g < L / R; g += blockDim.x) {
        float2 x[R];
#pragma unroll
        for (int p = 0; p < R; ++p) x[p] = X[fft_pad(R * g + p)];
        if constexpr (R == 16) {
          idft16(x);
        } else if constexpr (R == 8) {
          idft8(x);
        } else if constexpr (R == 4) {
          idft4(x[0], x[1], x[2], x[3]);
        } else {
          const float2 s = cadd(x[0], x[1]), d = csub(x[0], x[1]);
          x[0] = s;
          x[1] = d;
        }
        const int kb = reverse16<S>(g);
#pragma unroll
        for (int p = 0; p < R; ++p)
          keep_max_f(v_max, j_max, x[p].x * x[p].x + x[p].y * x[p].y, P * (kb + (p << (4 * S))) + r);
      }
      __syncthreads();  // (X is rewritten by the next transform)
    }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
      const float ov = __shfl_xor_sync(0xffffffffu, v_max, d);
      const int oj = __shfl_xor_sync(0xffffffffu, j_max, d);
      keep_max_f(v_max, j_max, ov, oj);
    }
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
      best_v[warp] = v_max;
      best_j[warp] = j_max;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      float bv = best_v[0];
      int bj = best_j[0];
      for (int w = 1; w < static_cast<int>(blockDim.x / 32); ++w) keep_max_f(bv, bj, best_v[w], best_j[w]);
      const double denominator = static_cast<double>(n_fft) * delta_f;
      double t = static_cast<double>(bj < 0 ? 0 : bj) / denominator;
      const double period = static_cast<double>(n_fft - 1) / denominator + 1.0 / denominator;
      if (t > period / 2) t -= period;
      t_out[row] = t;
    }
    __syncthreads();  // (best_* are reused by the next row)
  }
}

// The transform length of k_grid_time for n frequencies on a grid of n_fft
// times: the power of two >= max(n, 2048), if at most 16384 and dividing
// n_fft; else 0 (not supported).
int64_t grid_time_length(int64_t n, int64_t n_fft) {
  int64_t L = 2048;
  while (L < n) L *= 2;
  return (L <= 16384 && n_fft % L == 0) ? L : 0;
}

template <int L>
int launch_grid_time(const float2* series, int64_t rows, int64_t n, int64_t n_fft, double delta_f, double* t,
                     cudaStream_t s) {
  using G = GridShape<L>;
  if (G::kBytes > 48 * 1024) {
    static bool configured[64] = {};
    int dev = 0;
    const cudaError_t rd = cudaGetDevice(&dev);
    if (rd != cudaSuccess) return static_cast<int>(rd);
    if (dev < 0 || dev >= 64 || !configured[dev]) {
      const cudaError_t rc = cudaFuncSetAttribute(k_grid_time<L>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                  static_cast<int>(G::kBytes));
      if (rc != cudaSuccess) return static_cast<int>(rc);
      if (dev >= 0 && dev < 64) configured[dev] = true;
    }
  }
  const int64_t grid = rows < (int64_t(1) << 20) ? rows : (int64_t(1) << 20);
  k_grid_time<L><<<static_cast<unsigned>(grid), G::kThreads, G::kBytes, s>>>(series, rows, n, n_fft, delta_f, t);
  const cudaError_t err = cudaGetLastError();
  return err == cudaSuccess ? 0 : static_cast<int>(err);
}

int launched() {
  const cudaError_t err = cudaGetLastError();
  return err == cudaSuccess ? 0 : static_cast<int>(err);
}

unsigned row_grid(int64_t rows) { return static_cast<unsigned>(rows < (int64_t(1) << 20) ? rows : (int64_t(1) << 20)); }

}  // namespace
}  // namespace wfx

using namespace wfx;

extern "C" {

int wfx_overlap(int precision, const void* a, int64_t a_stride, const void* b, int64_t b_stride, const void* psd,
                int64_t rows, int64_t n, double delta_f, void* series, int64_t n_fft, double* norms,
                wfx_stream_t stream) {
  if (a == nullptr || b == nullptr || psd == nullptr || series == nullptr || norms == nullptr || rows <= 0 ||
      n <= 0 || n_fft < n || (a_stride != 0 && a_stride != n) || (b_stride != 0 && b_stride != n))
    return WFX_EINVAL;
  const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (precision == WFX_FP64) {
    k_overlap<double><<<row_grid(rows), kMatchBlock, 0, s>>>(
        static_cast<const double2*>(a), a_stride, static_cast<const double2*>(b), b_stride,
        static_cast<const double*>(psd), rows, n, 4.0 * delta_f, static_cast<double2*>(series), n_fft, norms);
  } else if (precision == WFX_FP32) {
    k_overlap<float><<<row_grid(rows), kMatchBlock, 0, s>>>(
        static_cast<const float2*>(a), a_stride, static_cast<const float2*>(b), b_stride,
        static_cast<const float*>(psd), rows, n, static_cast<float>(4.0 * delta_f), static_cast<float2*>(series),
        n_fft, norms);
  } else {
    return WFX_EINVAL;
  }
  return launched();
}

int wfx_match_refine(int precision, const void* series, const void* zgrid, int64_t rows, int64_t n, int64_t n_fft,
                     const double* freqs, double delta_f, const double* norms, int time, int phase, int steps,
                     double* match, double* t, wfx_stream_t stream) {
  if (series == nullptr || freqs == nullptr || norms == nullptr || match == nullptr || rows <= 0 || n <= 0 ||
      n_fft < n || steps < 0 || time < 0 || time > 2 || (time == 1 && zgrid == nullptr) ||
      (time == 2 && t == nullptr) || !(delta_f > 0.0))
    return WFX_EINVAL;
  const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (precision == WFX_FP64) {
    k_match_refine<double><<<row_grid((rows + kRowsPerBlock - 1) / kRowsPerBlock), kMatchBlock, 0, s>>>(
        static_cast<const double2*>(series), static_cast<const double2*>(zgrid), rows, n, n_fft, freqs, delta_f,
        norms, time, phase, steps, match, t);
  } else if (precision == WFX_FP32) {
    k_match_refine<float><<<row_grid((rows + kRowsPerBlock - 1) / kRowsPerBlock), kMatchBlock, 0, s>>>(
        static_cast<const float2*>(series), static_cast<const float2*>(zgrid), rows, n, n_fft, freqs, delta_f, norms,
        time, phase, steps, match, t);
  } else {
    return WFX_EINVAL;
  }
  return launched();
}

int wfx_match_grid_time(const void* series, int64_t rows, int64_t n, int64_t n_fft, double delta_f, double* t,
                        wfx_stream_t stream) {
  if (series == nullptr || t == nullptr || rows <= 0 || n <= 0 || n_fft < n || !(delta_f > 0.0)) return WFX_EINVAL;
  const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const auto* c = static_cast<const float2*>(series);
  switch (grid_time_length(n, n_fft)) {
    case 2048:
      return launch_grid_time<2048>(c, rows, n, n_fft, delta_f, t, s);
    case 4096:
      return launch_grid_time<4096>(c, rows, n, n_fft, delta_f, t, s);
    case 8192:
      return launch_grid_time<8192>(c, rows, n, n_fft, delta_f, t, s);
    case 16384:
      return launch_grid_time<16384>(c, rows, n, n_fft, delta_f, t, s);
    default:
      return WFX_EINVAL;
  }
}

int wfx_polarization_overlap(int precision, const void* signal, int64_t s_stride, const void* hplus, int64_t p_stride,
                             const void* hcross, int64_t x_stride, const void* psd, int64_t rows, int64_t n,
                             double delta_f, void* series, int64_t n_fft, double* norms, wfx_stream_t stream) {
  if (signal == nullptr || hplus == nullptr || hcross == nullptr || psd == nullptr || series == nullptr ||
      norms == nullptr || rows <= 0 || n <= 0 || n_fft < n || (s_stride != 0 && s_stride != n) ||
      (p_stride != 0 && p_stride != n) || (x_stride != 0 && x_stride != n))
    return WFX_EINVAL;
  const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (precision == WFX_FP64) {
    k_polarization_overlap<double><<<row_grid(rows), kMatchBlock, 0, s>>>(
        static_cast<const double2*>(signal), s_stride, static_cast<const double2*>(hplus), p_stride,
        static_cast<const double2*>(hcross), x_stride, static_cast<const double*>(psd), rows, n, 4.0 * delta_f,
        static_cast<double2*>(series), n_fft, norms);
  } else if (precision == WFX_FP32) {
    k_polarization_overlap<float><<<row_grid(rows), kMatchBlock, 0, s>>>(
        static_cast<const float2*>(signal), s_stride, static_cast<const float2*>(hplus), p_stride,
        static_cast<const float2*>(hcross), x_stride, static_cast<const float*>(psd), rows, n,
        static_cast<float>(4.0 * delta_f), static_cast<float2*>(series), n_fft, norms);
  } else {
    return WFX_EINVAL;
  }
  return launched();
}

int wfx_polarization_refine(int precision, const void* series, const void* zgrid, int64_t rows, int64_t n,
                            int64_t n_fft, const double* freqs, double delta_f, const double* norms, int time,
                            int steps, double* match, double* t, wfx_stream_t stream) {
  if (series == nullptr || freqs == nullptr || norms == nullptr || match == nullptr || rows <= 0 || n <= 0 ||
      n_fft < n || steps < 0 || (time && zgrid == nullptr) || !(delta_f > 0.0))
    return WFX_EINVAL;
  const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const unsigned grid = row_grid((rows + kRowsPerBlock - 1) / kRowsPerBlock);
  if (precision == WFX_FP64) {
    k_polarization_refine<double><<<grid, kMatchBlock, 0, s>>>(static_cast<const double2*>(series),
                                                               static_cast<const double2*>(zgrid), rows, n, n_fft,
                                                               freqs, delta_f, norms, time, steps, match, t);
  } else if (precision == WFX_FP32) {
    k_polarization_refine<float><<<grid, kMatchBlock, 0, s>>>(static_cast<const float2*>(series),
                                                              static_cast<const float2*>(zgrid), rows, n, n_fft,
                                                              freqs, delta_f, norms, time, steps, match, t);
  } else {
    return WFX_EINVAL;
  }
  return launched();
}

}  // extern "C"
