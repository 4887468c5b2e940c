// The CUDA kernels of the aligned-spin frequency-domain path for sm_100a, and
// the C ABI of include/waveformx_b200.h.
//
// Kernels (the set-up kernels are in setup.cu):
//  * k_fwd_f32_shared: (h+, hx) on a grid shared by the batch, FP32 with
//    double-float phase. A block takes a tile of frequencies and 16
//    consecutive binaries: a warp computes the powers of its lanes' two
//    frequencies once for the 16, finds each binary's regions over its span
//    with one ballot, and each pair of outputs leaves as one 16-byte store
//    (two 8-byte stores in rows that start on an odd element).
//  * k_fwd_f32_tiles: the same for ragged batches, one persistent launch
//    over (binary, tile) work items (tile_prefix / tile_map index them).
//  * k_adj_f32: the reverse-mode pass, for cotangents (vjp) or for the fused
//    likelihood (cotangent from the data in registers: the strain never
//    reaches memory). Per-tile sums of dL/dtable go to the workspace.
//  * k_contract: per binary, the FP64 sum of its tiles' partial sums and the
//    product with dtable: the gradient in the parameters.
//  * k_fwd_f64 / k_adj_f64: the plain FP64 form, one binary per block.
#include <cuda_runtime.h>

#include <atomic>
#include <cmath>
#include <map>
#include <mutex>
#include <tuple>
#include <type_traits>
#include <cstdint>
#include <cstdio>

#include "../../include/waveformx_b200.h"
#include "dual_point.cuh"
#include "internal.h"
#include "point.cuh"
#include "point_x2.cuh"

namespace wfx {

constexpr int kBlock = 256;
constexpr int64_t kFwdTile = 2 * kBlock - 2;    // frequencies per block (shared-grid forward)
constexpr int kBinariesPerBlock = 16;          // binaries per block (shared-grid forward)
constexpr int64_t kRaggedTileMin = 2 * kBlock - 2;  // shortest work item of the ragged forward
constexpr int64_t kAdjTileMax = 8 * kBlock - 2;  // frequencies per work item (reverse mode), at most
constexpr int kGradColumns = 9;
constexpr int kDirections = 8;

// ---------------------------------------------------------------------------
// helpers of the frequency kernels

template <int MODEL, class S>
__device__ __forceinline__ Point<S> point(const S* T, const Freq<S>& q, typename TcOf<S>::type tc) {
  if constexpr (MODEL == kModelXas) {
    return xas_point<S>(T, q, tc);
  } else if constexpr (MODEL == kModelPhenomD) {
    return phd_point<S>(T, q, tc);
  } else {
    return tf2_point<S>(T, q, tc);
  }
}

template <int MODEL, class S, class Acc>
__device__ __forceinline__ void adjoint(const S* T, const Freq<S>& q, const Point<S>& pt, S gpr, S gpi, S gcr, S gci,
                                        Acc* acc) {
  if constexpr (MODEL == kModelXas) {
    xas_adjoint<S>(T, q, pt, gpr, gpi, gcr, gci, acc);
  } else if constexpr (MODEL == kModelPhenomD) {
    phd_adjoint<S>(T, q, pt, gpr, gpi, gcr, gci, acc);
  } else {
    tf2_adjoint<S>(T, q, pt, gpr, gpi, gcr, gci, acc);
  }
}

// The plain-float phase coefficients of each model's FP32 evaluation (the
// constants, the coefficients of f and the double-float terms apart).
__device__ constexpr int kXasPlainPhase[] = {
    X_PH_INS + 0,  X_PH_INS + 1, X_PH_INS + 2, X_PH_INS + 3, X_PH_INS + 5, X_PH_INS + 6, X_PH_INS + 7,
    X_PH_INS + 9,  X_PH_INS + 10, X_PH_INS + 11, X_PH_INS + 12, X_PH_INT + 2, X_PH_INT + 3, X_PH_INT + 4,
    X_PH_INT + 5,  X_PH_RD + 3,  X_PH_RD + 4,  X_ATAN_A,     X_ATAN_A + 1};
__device__ constexpr int kPhdPlainPhase[] = {
    D_PH_INS + 1, D_PH_INS + 2,  D_PH_INS + 3,  D_PH_INS + 4, D_PH_INS + 5, D_PH_INS + 6, D_PH_INS + 7,
    D_PH_INS + 9, D_PH_INS + 10, D_PH_INS + 11, D_PH_INT + 2, D_PH_INT + 3, D_PH_RD + 2,  D_ATAN_A};
__device__ constexpr int kTf2PlainPhase[] = {T_PH + 0, T_PH + 1, T_PH + 2, T_PH + 3, T_PH + 5, T_PH + 6, T_PH + 7};

// A staged FP32 table made ready for one binary's frequencies (point.cuh):
// 2 pi t_c folded in and the constants reduced modulo 2 pi (prepare_f32),
// or, with TURNS, the whole phase in turns (prepare_turns; the forward
// kernels, whose evaluation then uses phase_turns).
template <int MODEL, bool TURNS = false>
__device__ __forceinline__ void prepare_model(float* T, float t_c) {
  using L = Layout<MODEL>;
  int cs[L::kRegions], ls[L::kRegions];
#pragma unroll
  for (int r = 0; r < L::kRegions; ++r) {
    cs[r] = L::const_slot(r);
    ls[r] = L::lin_slot(r);
  }
  if constexpr (TURNS) {
    constexpr bool kXas = MODEL == kModelXas, kPhd = MODEL == kModelPhenomD;
    const int* plain = kXas ? kXasPlainPhase : (kPhd ? kPhdPlainPhase : kTf2PlainPhase);
    constexpr int n_plain = static_cast<int>(kXas ? sizeof(kXasPlainPhase) / sizeof(int)
                                                  : (kPhd ? sizeof(kPhdPlainPhase) / sizeof(int)
                                                          : sizeof(kTf2PlainPhase) / sizeof(int)));
    prepare_turns<L::kRegions>(T, plain, n_plain, L::kT0, L::kT0Lo, L::kBigTerm, L::kBigTermLo, cs, L::kConstLo, ls,
                               L::kLinLo, t_c);
  } else {
    prepare_f32<L::kRegions>(T, cs, L::kConstLo, ls, L::kLinLo, t_c);
  }
}

template <int MODEL, class S, int RP, int RA, bool TURNS = false>
__device__ __forceinline__ void eval_fixed(const S* T, const Freq<S>* q, typename TcOf<S>::type tc, Point<S>* p) {
  if constexpr (MODEL == kModelXas) {
    xas_eval<S, 2, RP, RA, TURNS>(T, q, RP, RA, tc, p);
  } else if constexpr (MODEL == kModelPhenomD) {
    phd_eval<S, 2, RP, RA, TURNS>(T, q, RP, RA, tc, p);
  } else {
    tf2_eval<S, 2, RP, RA, TURNS>(T, q, RP, RA, tc, p);
  }
}

// Two adjacent frequencies of one binary: evaluated in lockstep (each table
// coefficient read once) when they share their regions, else one by one.
// When every lane of the warp holds frequencies of the same (phase,
// amplitude) regions (all but the few warps that straddle a boundary), the
// evaluation compiled for those regions runs: no branch on them. Every lane
// of the warp must call it (a vote).
//
// SPECIALIZE = false: no vote and no specialized copies (the reverse pass,
// whose larger code is fetch-bound already).
template <int MODEL, class S, bool SPECIALIZE = true, bool TURNS = false>
__device__ __forceinline__ void point_pair(const S* T, const Freq<S>& q0, const Freq<S>& q1,
                                           typename TcOf<S>::type tc, Point<S>& p0, Point<S>& p1) {
  int rp0, ra0, rp1, ra1;
  if constexpr (MODEL == kModelXas) {
    xas_regions(T, q0.f, rp0, ra0);
    xas_regions(T, q1.f, rp1, ra1);
  } else if constexpr (MODEL == kModelPhenomD) {
    phd_regions(T, q0.f, rp0, ra0);
    phd_regions(T, q1.f, rp1, ra1);
  } else {
    tf2_regions(T, q0.f, rp0, ra0);
    tf2_regions(T, q1.f, rp1, ra1);
  }
  const int code = rp0 * 3 + ra0;
  const bool same = rp0 == rp1 && ra0 == ra1;
  const int lead = __shfl_sync(0xffffffffu, code, 0);
  const Freq<S> q[2] = {q0, q1};
  Point<S> p[2];
  if (SPECIALIZE && __all_sync(0xffffffffu, same && code == lead)) {
    switch (lead) {
      case 8:
        eval_fixed<MODEL, S, 2, 2, TURNS>(T, q, tc, p);
        break;
      case 7:
        eval_fixed<MODEL, S, 2, 1, TURNS>(T, q, tc, p);
        break;
      case 4:
        eval_fixed<MODEL, S, 1, 1, TURNS>(T, q, tc, p);
        break;
      case 3:
        eval_fixed<MODEL, S, 1, 0, TURNS>(T, q, tc, p);
        break;
      case 0:
        eval_fixed<MODEL, S, 0, 0, TURNS>(T, q, tc, p);
        break;
      default:
        if constexpr (MODEL == kModelXas) {
          xas_eval<S, 2, -1, -1, TURNS>(T, q, rp0, ra0, tc, p);
        } else if constexpr (MODEL == kModelPhenomD) {
          phd_eval<S, 2, -1, -1, TURNS>(T, q, rp0, ra0, tc, p);
        } else {
          tf2_eval<S, 2, -1, -1, TURNS>(T, q, rp0, ra0, tc, p);
        }
    }
    p0 = p[0];
    p1 = p[1];
    return;
  }
  if (same) {
    if constexpr (MODEL == kModelXas) {
      xas_eval<S, 2, -1, -1, TURNS>(T, q, rp0, ra0, tc, p);
    } else if constexpr (MODEL == kModelPhenomD) {
      phd_eval<S, 2, -1, -1, TURNS>(T, q, rp0, ra0, tc, p);
    } else {
      tf2_eval<S, 2, -1, -1, TURNS>(T, q, rp0, ra0, tc, p);
    }
    p0 = p[0];
    p1 = p[1];
  } else {
    if constexpr (MODEL == kModelXas) {
      xas_eval<S, 1, -1, -1, TURNS>(T, &q0, rp0, ra0, tc, &p0);
      xas_eval<S, 1, -1, -1, TURNS>(T, &q1, rp1, ra1, tc, &p1);
    } else if constexpr (MODEL == kModelPhenomD) {
      phd_eval<S, 1, -1, -1, TURNS>(T, &q0, rp0, ra0, tc, &p0);
      phd_eval<S, 1, -1, -1, TURNS>(T, &q1, rp1, ra1, tc, &p1);
    } else {
      tf2_eval<S, 1, -1, -1, TURNS>(T, &q0, rp0, ra0, tc, &p0);
      tf2_eval<S, 1, -1, -1, TURNS>(T, &q1, rp1, ra1, tc, &p1);
    }
  }
}

template <int MODEL>
__host__ __device__ constexpr int slot_kp() {
  return Layout<MODEL>::kKp;
}
template <int MODEL>
__host__ __device__ constexpr int slot_kc() {
  return Layout<MODEL>::kKc;
}

// The table slots whose partial sums the reverse pass produces.
template <int MODEL>
__host__ __device__ constexpr bool slot_used(int k) {
  if (k == kSlotTc || k == kSlotLoss) return true;
  if constexpr (MODEL == kModelXas) {
    return k < X_F_PHASE_IN || (k >= X_KP && k <= X_ANCHOR);
  } else if constexpr (MODEL == kModelPhenomD) {
    return k < D_F_PHASE_INS || (k >= D_KP && k <= D_ANCHOR);
  } else {
    return k < T_USED && k != T_LIN;
  }
}

// Stores the pair (e, e + 1) of complex64 outputs (e even: 16-byte aligned)
// or the one of them that is in range.
__device__ __forceinline__ void store_pair(float2* out, int64_t e, float4 v, bool v0, bool v1) {
  if (v0 && v1) {
    __stcs(reinterpret_cast<float4*>(out + e), v);
  } else if (v0) {
    out[e] = make_float2(v.x, v.y);
  } else if (v1) {
    out[e + 1] = make_float2(v.z, v.w);
  }
}

// The same pair at an address that is 8-byte aligned only: two 8-byte
// streaming stores.
__device__ __forceinline__ void store_halves(float2* out, float4 v, bool v0, bool v1) {
  if (v0) __stcs(out, make_float2(v.x, v.y));
  if (v1) __stcs(out + 1, make_float2(v.z, v.w));
}

__device__ __forceinline__ float4 load_pair(const float2* in, int64_t e, bool v0, bool v1) {
  if (v0 && v1) return __ldcs(reinterpret_cast<const float4*>(in + e));
  float4 r = make_float4(0.f, 0.f, 0.f, 0.f);
  if (v0) {
    float2 a = in[e];
    r.x = a.x;
    r.y = a.y;
  }
  if (v1) {
    float2 a = in[e + 1];
    r.z = a.x;
    r.w = a.y;
  }
  return r;
}

// A work item of the tiled kernels: binary b, its flat range [s, e) of
// outputs, and the offset from a flat index to a frequency index.
struct Item {
  int64_t b, s, e, fbase;
};

template <bool RAGGED>
__device__ __forceinline__ Item item_of(int64_t item, const int64_t* offsets, const int64_t* tile_prefix,
                                        const int32_t* tile_map, int64_t n, int64_t tile_len,
                                        int64_t tiles_per_binary) {
  Item it;
  if constexpr (RAGGED) {
    it.b = tile_map[item];
    const int64_t j = item - tile_prefix[it.b];
    // (offsets clamped to [0, n]: inconsistent ones read and write nothing
    // out of bounds)
    const int64_t rs = min(max(offsets[it.b], int64_t(0)), n);
    const int64_t re = min(max(offsets[it.b + 1], rs), n);
    it.s = rs + j * tile_len;
    it.e = min(it.s + tile_len, re);
    it.fbase = 0;
  } else {
    it.b = item / tiles_per_binary;
    const int64_t j = item - it.b * tiles_per_binary;
    const int64_t rs = it.b * n;
    it.s = rs + j * tile_len;
    it.e = min(it.s + tile_len, rs + n);
    it.fbase = rs;
  }
  return it;
}

// ---------------------------------------------------------------------------
// FP32 forward

// IMRPhenomXAS is zero above its cutoff f_cut (models/xas/core.py:493): a
// warp whose frequencies are all above it needs no evaluation (a vote: every
// lane of the warp calls this). The zeros are 0 * kp and 0 * kc, NaN for a
// refused binary as in the evaluated form.
template <int MODEL>
__device__ __forceinline__ bool all_above_cutoff(const float* T, float f0, float f1, float4& hp, float4& hc) {
  if constexpr (MODEL == kModelXas) {
    const float f_cut = T[X_F_CUT];
    if (__all_sync(0xffffffffu, f0 > f_cut && f1 > f_cut)) {
      const float zp = 0.0f * T[X_KP], zc = 0.0f * T[X_KC];
      hp = make_float4(zp, zp, zp, zp);
      hc = make_float4(zc, zc, zc, zc);
      return true;
    }
  }
  return false;
}

template <int MODEL>
__device__ __forceinline__ void project(const float* T, const Point<float>& p0, const Point<float>& p1,
                                        float4& hp, float4& hc) {
  const float kp = T[slot_kp<MODEL>()], kc = T[slot_kc<MODEL>()];
  const float ap0 = kp * p0.amp, ac0 = kc * p0.amp, ap1 = kp * p1.amp, ac1 = kc * p1.amp;
  hp = make_float4(ap0 * p0.c, ap0 * p0.s, ap1 * p1.c, ap1 * p1.s);
  hc = make_float4(-ac0 * p0.s, ac0 * p0.c, -ac1 * p1.s, ac1 * p1.c);
}

// The regions of one binary that every frequency of a warp's span [lo, hi]
// shares, from one ballot: lanes 2k and 2k + 1 test lo and hi against the
// binary's boundary k (the tests of xas_regions / phd_regions, and the XAS
// cutoff). Each test is a non-decreasing function of f, so a test that lo
// and hi pass or fail alike is passed or failed alike by every frequency in
// between: then the whole span has the regions (rp, ra). lo, hi and the
// table are the same in every lane (the result is warp-uniform).
struct SpanRegions {
  int rp, ra;
  bool uniform;    // every frequency of the span in (rp, ra)
  bool above_cut;  // XAS: every frequency of the span above f_cut
};

template <int MODEL>
__device__ __forceinline__ SpanRegions span_regions(const float* T, float lo, float hi, int lane) {
  if constexpr (MODEL == kModelTaylorF2) return SpanRegions{0, 0, true, false};  // one region, no cutoff
  constexpr bool kXas = MODEL == kModelXas;
  constexpr int kFirst = kXas ? static_cast<int>(X_F_PHASE_IN) : static_cast<int>(D_F_PHASE_INS);
  constexpr int kTests = kXas ? 5 : 4;  // XAS: f_phase_in, f_phase_im, f_amp_in, f_amp_rd, f_cut
  const int k = min(lane >> 1, kTests - 1);
  const float f = (lane & 1) ? hi : lo;
  const float bound = T[kFirst + k];
  bool pass;
  if constexpr (kXas) {
    pass = (k == 0 || k == 2) ? f >= bound : f > bound;
  } else {
    pass = (k == 0 || k == 2) ? !(f < bound) : f >= bound;
  }
  const unsigned m = __ballot_sync(0xffffffffu, pass && lane < 2 * kTests);
  SpanRegions r;
  r.uniform = ((m ^ (m >> 1)) & 0x55u) == 0u;
  const int i0 = m & 1u, i1 = (m >> 2) & 1u, i2 = (m >> 4) & 1u, i3 = (m >> 6) & 1u;
  if constexpr (kXas) {
    r.rp = i0 + i1;
    r.ra = i2 + i3;
    r.above_cut = (m >> 8) & 1u;
  } else {
    r.rp = i0 ? 1 + i1 : 0;
    r.ra = i2 ? 1 + i3 : 0;
    r.above_cut = false;
  }
  return r;
}

// span_regions of all kBinariesPerBlock binaries of a block at once (the
// same tests): lane 2j + s tests binary j's boundaries against lo (s = 0)
// or hi (s = 1), and lane 2j returns binary j's regions over [lo, hi] as
// rp | ra << 2 | uniform << 4 | above_cut << 5 (span_code reads them back
// in any lane). IMRPhenomXAS and IMRPhenomD; lo, hi as span_regions'.
template <int MODEL>
__device__ __forceinline__ int span_codes(const float (*sT)[kTableStride], float lo, float hi, int lane) {
  static_assert(2 * kBinariesPerBlock == 32, "two lanes a binary");
  constexpr bool kXas = MODEL == kModelXas;
  constexpr int kFirst = kXas ? static_cast<int>(X_F_PHASE_IN) : static_cast<int>(D_F_PHASE_INS);
  constexpr int kTests = kXas ? 5 : 4;  // XAS: f_phase_in, f_phase_im, f_amp_in, f_amp_rd, f_cut
  const float f = (lane & 1) ? hi : lo;
  const float* bound = sT[lane >> 1] + kFirst;
  unsigned bits = 0;
#pragma unroll
  for (int k = 0; k < kTests; ++k) {
    bool pass;
    if constexpr (kXas) {
      pass = (k == 0 || k == 2) ? f >= bound[k] : f > bound[k];
    } else {
      pass = (k == 0 || k == 2) ? !(f < bound[k]) : f >= bound[k];
    }
    bits |= static_cast<unsigned>(pass) << k;
  }
  // (lane 2j: bits of lo, other of hi)
  const unsigned other = __shfl_xor_sync(0xffffffffu, bits, 1);
  const int uniform = ((bits ^ other) & 0xFu) == 0u;
  const int i0 = bits & 1u, i1 = (bits >> 1) & 1u, i2 = (bits >> 2) & 1u, i3 = (bits >> 3) & 1u;
  int rp, ra, above = 0;
  if constexpr (kXas) {
    rp = i0 + i1;
    ra = i2 + i3;
    above = (bits >> 4) & 1u;
  } else {
    rp = i0 ? 1 + i1 : 0;
    ra = i2 ? 1 + i3 : 0;
  }
  return rp | (ra << 2) | (uniform << 4) | (above << 5);
}

// Binary j's regions from span_codes' result (every lane of the warp calls
// it with the same j).
__device__ __forceinline__ SpanRegions span_code(int codes, int j) {
  const int code = __shfl_sync(0xffffffffu, codes, 2 * j);
  return SpanRegions{code & 3, (code >> 2) & 3, ((code >> 4) & 1) != 0, ((code >> 5) & 1) != 0};
}

// Two adjacent frequencies of one binary whose warp span has the regions
// `sr` (every lane of the warp calls it with the same sr): the evaluation
// compiled for those regions, or, for a span that crosses a boundary, the
// regions of each lane.
template <int MODEL, bool TURNS>
__device__ __forceinline__ void span_pair(const float* T, const Freq<float>& q0, const Freq<float>& q1,
                                          const SpanRegions& sr, Point<float>& p0, Point<float>& p1) {
  if (!sr.uniform) {
    point_pair<MODEL, float, false, TURNS>(T, q0, q1, TcF{}, p0, p1);
    return;
  }
  const Freq<float> q[2] = {q0, q1};
  Point<float> p[2];
  switch (sr.rp * 3 + sr.ra) {
    case 8:
      eval_fixed<MODEL, float, 2, 2, TURNS>(T, q, TcF{}, p);
      break;
    case 7:
      eval_fixed<MODEL, float, 2, 1, TURNS>(T, q, TcF{}, p);
      break;
    case 4:
      eval_fixed<MODEL, float, 1, 1, TURNS>(T, q, TcF{}, p);
      break;
    case 3:
      eval_fixed<MODEL, float, 1, 0, TURNS>(T, q, TcF{}, p);
      break;
    case 0:
      eval_fixed<MODEL, float, 0, 0, TURNS>(T, q, TcF{}, p);
      break;
    default:
      if constexpr (MODEL == kModelXas) {
        xas_eval<float, 2, -1, -1, TURNS>(T, q, sr.rp, sr.ra, TcF{}, p);
      } else if constexpr (MODEL == kModelPhenomD) {
        phd_eval<float, 2, -1, -1, TURNS>(T, q, sr.rp, sr.ra, TcF{}, p);
      } else {
        tf2_eval<float, 2, -1, -1, TURNS>(T, q, sr.rp, sr.ra, TcF{}, p);
      }
  }
  p0 = p[0];
  p1 = p[1];
}

// The pair on the packed FP32 instructions (point_x2.cuh) for the region
// pairs the span classification meets (IMRPhenomXAS, IMRPhenomD); false
// for the others, which take span_pair. Every lane of the warp calls it
// with the same sr.
template <int MODEL, class C>
__device__ __forceinline__ bool pair_packed(const C& T, const Freq2& q, const SpanRegions& sr, float4& hp,
                                            float4& hc) {
  if constexpr (MODEL == kModelXas || MODEL == kModelPhenomD) {
    auto eval = [&](auto rp, auto ra) {
      if constexpr (MODEL == kModelXas) {
        xas_pair_x2<decltype(rp)::value, decltype(ra)::value>(T, q, hp, hc);
      } else {
        phd_pair_x2<decltype(rp)::value, decltype(ra)::value>(T, q, hp, hc);
      }
      return true;
    };
    using I0 = std::integral_constant<int, 0>;
    using I1 = std::integral_constant<int, 1>;
    using I2 = std::integral_constant<int, 2>;
    switch (sr.rp * 3 + sr.ra) {
      case 8:
        return eval(I2{}, I2{});
      case 7:
        return eval(I2{}, I1{});
      case 4:
        return eval(I1{}, I1{});
      case 3:
        return eval(I1{}, I0{});
      case 0:
        return eval(I0{}, I0{});
      default:
        return false;
    }
  }
  return false;
}

// Shared-grid forward. Block (group, tile): kFwdTile frequencies of a group
// of kBinariesPerBlock consecutive binaries, the group's tables staged once
// in shared memory. A thread takes the frequencies (m, m + 1), m even; a
// warp computes their powers once for the group and finds each binary's
// regions over its span with one ballot. A pair of outputs leaves as one
// 16-byte store in a row that starts on an even element, as two 8-byte
// stores in one that starts on an odd element (rows of odd length
// alternate).
//
// The order of the blocks (measured): the issue-bound models (XAS,
// PhenomD) run tile-major, the tiles in the order 0, T-1, 1, T-2, ...: the
// low frequencies (every binary evaluated) and the high ones (mostly zero
// above the XAS cutoff, store bound) alternate through the launch (XAS:
// its last tile last of all, fwd_tile). TaylorF2,
// whose evaluation is light and whose time is its stores, runs group-major:
// the blocks in flight then write whole rows of a few groups, contiguous
// memory, rather than one tile of every row. Tiles beyond the grid's tile
// dimension loop in the block; group0 offsets the groups of a launch.
template <int MODEL>
constexpr bool fwd_group_major() {
  return MODEL == kModelTaylorF2;
}

// The tile of a tile-major block: 0, T-1, 1, T-2, ...; for XAS the last tile
// (the highest frequencies, mostly above the cutoff: the lightest blocks)
// goes last of all and the others alternate, so that the launch ends on
// light blocks (measured on 4096 x 4017: 61.4-61.8 us against 62.8-63.0).
template <int MODEL>
__device__ __forceinline__ int64_t fwd_tile(unsigned index, unsigned count) {
  const unsigned alternating = MODEL == kModelXas && count > 2 ? count - 1 : count;
  if (index >= alternating) return index;
  return (index & 1) ? alternating - 1 - (index >> 1) : (index >> 1);
}

template <int MODEL>
__global__ void __launch_bounds__(kBlock, 4) k_fwd_f32_shared(const float* __restrict__ table,
                                                              const float* __restrict__ freqs, int64_t n, int64_t B,
                                                              int64_t group0, const float* __restrict__ t_c,
                                                              float2* __restrict__ hp, float2* __restrict__ hc) {
  constexpr bool kGroupMajor = fwd_group_major<MODEL>();
  __shared__ __align__(16) float sT[kBinariesPerBlock][kTableStride];
  const int lane = threadIdx.x & 31;
  const unsigned tile_index = kGroupMajor ? blockIdx.x : blockIdx.y;
  const unsigned tile_count = kGroupMajor ? gridDim.x : gridDim.y;
  const int64_t base = (group0 + (kGroupMajor ? blockIdx.y : blockIdx.x)) * kBinariesPerBlock;
  for (int i = threadIdx.x; i < kBinariesPerBlock * (kTableStride / 4); i += kBlock) {
    const int j = i / (kTableStride / 4), q = i % (kTableStride / 4);
    const int64_t b = base + j;
    float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
    if (b < B) v = __ldg(reinterpret_cast<const float4*>(table + b * kTableStride) + q);
    reinterpret_cast<float4*>(sT[j])[q] = v;
  }
  __syncthreads();
  if (threadIdx.x < kBinariesPerBlock) {
    const int64_t b = base + threadIdx.x;
    prepare_model<MODEL, true>(sT[threadIdx.x], (t_c != nullptr && b < B) ? t_c[b] : 0.0f);
  }
  __syncthreads();
  const int count = static_cast<int>(min(static_cast<int64_t>(kBinariesPerBlock), B - base));
  const int64_t y = fwd_tile<MODEL>(tile_index, tile_count);
  for (int64_t n0 = y * kFwdTile; n0 < n; n0 += static_cast<int64_t>(tile_count) * kFwdTile) {
    const int64_t n_end = min(n0 + kFwdTile, n);
    const int64_t m = n0 + 2 * static_cast<int64_t>(threadIdx.x);
    const bool v0 = m < n_end;
    const bool v1 = m + 1 < n_end;
    // (a lane without a frequency in the tile evaluates an in-range one and
    // stores nothing: every lane of the warp takes part in the ballots)
    const int64_t i0 = v0 ? m : n0, i1 = v1 ? m + 1 : i0;
    const Freq<float> q0 = freq_powers(freqs[i0]);
    const Freq<float> q1 = freq_powers(freqs[i1]);
    const Freq2 q2 = pack_freqs(q0, q1);
    float lo = fminf(q0.f, q1.f), hi = fmaxf(q0.f, q1.f);
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
      lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, d));
      hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, d));
    }
    // (a NaN frequency: each lane's own regions, as the one-by-one form)
    const bool nan_span = __any_sync(0xffffffffu, q0.f != q0.f || q1.f != q1.f);
    // (each binary's regions over the warp's span, classified for all the
    // block's binaries at once)
    int codes = 0;
    if constexpr (MODEL != kModelTaylorF2) codes = span_codes<MODEL>(sT, lo, hi, lane);
    float2* out_p = hp + base * n + m;
    float2* out_c = hc + base * n + m;
    // (m is even: a row's pairs are 16-byte aligned where the row's first
    // element is, b n even)
    bool aligned = ((base * n) & 1) == 0;
#pragma unroll 1
    for (int j = 0; j < count; ++j, out_p += n, out_c += n, aligned ^= (n & 1)) {
      const float* T = sT[j];
      SpanRegions sr;
      if constexpr (MODEL == kModelTaylorF2) {
        sr = span_regions<MODEL>(T, lo, hi, lane);
      } else {
        sr = span_code(codes, j);
      }
      sr.uniform = sr.uniform && !nan_span;
      float4 vp, vc;
      if (sr.above_cut && !nan_span) {
        // zero above the XAS cutoff (models/xas/core.py:493): 0 kp, 0 kc
        // (NaN for a refused binary, as the evaluated form)
        const float zp = 0.0f * T[slot_kp<MODEL>()], zc = 0.0f * T[slot_kc<MODEL>()];
        vp = make_float4(zp, zp, zp, zp);
        vc = make_float4(zc, zc, zc, zc);
      } else if (!(sr.uniform && pair_packed<MODEL>(Bcast{T}, q2, sr, vp, vc))) {
        Point<float> p0, p1;
        span_pair<MODEL, true>(T, q0, q1, sr, p0, p1);
        project<MODEL>(T, p0, p1, vp, vc);
      }
      if (aligned) {
        store_pair(out_p, 0, vp, v0, v1);
        store_pair(out_c, 0, vc, v0, v1);
      } else {
        store_halves(out_p, vp, v0, v1);
        store_halves(out_c, vc, v0, v1);
      }
    }
  }
}

// The overlap series of a bank of templates with one signal, without the
// templates' strain in memory (the match of match.py:71-147 fused with the
// waveform): for binary b of a shared grid, h_b = fp h+_b + fc hx_b in
// registers (the forward's evaluation), c[b][k] = scale h_b(f_k) conj(s_k)
// / S_k with scale = 4 delta_f, stored at series[b n_fft + k] (rows of even
// length: every pair 16-byte aligned), and <h_b, h_b> = scale sum_k
// |h_b(f_k)|^2 / S_k added into norms[2 b] (one atomic per warp and
// binary; k_template_norms zeroes it). Blocks as k_fwd_f32_shared.
//
// POLARIZATIONS: polarization_match's series instead (match.py:162-172):
// rows 2 b and 2 b + 1 of `series` are scale s conj(h+_b) / S and
// scale s conj(hx_b) / S, and norms[4 b + 1 ..] gain <h+, h+>, <hx, hx>,
// <h+, hx> (norms[4 b] = <s, s>); fp and fc unused.
template <int MODEL, bool POLARIZATIONS = false>
__global__ void __launch_bounds__(kBlock, 4) k_template_overlap(const float* __restrict__ table,
                                                                const float* __restrict__ freqs, int64_t n, int64_t B,
                                                                int64_t group0, const float* __restrict__ t_c,
                                                                float fp, float fc, const float2* __restrict__ signal,
                                                                const float* __restrict__ psd, float scale,
                                                                float2* __restrict__ series, int64_t n_fft,
                                                                double* __restrict__ norms) {
  constexpr bool kGroupMajor = fwd_group_major<MODEL>();
  __shared__ __align__(16) float sT[kBinariesPerBlock][kTableStride];
  const int lane = threadIdx.x & 31;
  const unsigned tile_index = kGroupMajor ? blockIdx.x : blockIdx.y;
  const unsigned tile_count = kGroupMajor ? gridDim.x : gridDim.y;
  const int64_t base = (group0 + (kGroupMajor ? blockIdx.y : blockIdx.x)) * kBinariesPerBlock;
  for (int i = threadIdx.x; i < kBinariesPerBlock * (kTableStride / 4); i += kBlock) {
    const int j = i / (kTableStride / 4), q = i % (kTableStride / 4);
    const int64_t b = base + j;
    float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
    if (b < B) v = __ldg(reinterpret_cast<const float4*>(table + b * kTableStride) + q);
    reinterpret_cast<float4*>(sT[j])[q] = v;
  }
  __syncthreads();
  if (threadIdx.x < kBinariesPerBlock) {
    const int64_t b = base + threadIdx.x;
    prepare_model<MODEL, true>(sT[threadIdx.x], (t_c != nullptr && b < B) ? t_c[b] : 0.0f);
  }
  __syncthreads();
  const int count = static_cast<int>(min(static_cast<int64_t>(kBinariesPerBlock), B - base));
  const int64_t y = (tile_index & 1) ? tile_count - 1 - (tile_index >> 1) : (tile_index >> 1);
  for (int64_t n0 = y * kFwdTile; n0 < n; n0 += static_cast<int64_t>(tile_count) * kFwdTile) {
    const int64_t n_end = min(n0 + kFwdTile, n);
    const int64_t m = n0 + 2 * static_cast<int64_t>(threadIdx.x);
    const bool v0 = m < n_end;
    const bool v1 = m + 1 < n_end;
    const int64_t i0 = v0 ? m : n0, i1 = v1 ? m + 1 : i0;
    const Freq<float> q0 = freq_powers(freqs[i0]);
    const Freq<float> q1 = freq_powers(freqs[i1]);
    // the signal's conjugate over the PSD, scaled (zero where out of range)
    const float2 s0 = signal[i0], s1 = signal[i1];
    const float w0 = v0 ? scale / psd[i0] : 0.0f, w1 = v1 ? scale / psd[i1] : 0.0f;
    const float4 sw = make_float4(w0 * s0.x, -w0 * s0.y, w1 * s1.x, -w1 * s1.y);
    (void)sw;
    float lo = fminf(q0.f, q1.f), hi = fmaxf(q0.f, q1.f);
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
      lo = fminf(lo, __shfl_xor_sync(0xffffffffu, lo, d));
      hi = fmaxf(hi, __shfl_xor_sync(0xffffffffu, hi, d));
    }
    const bool nan_span = __any_sync(0xffffffffu, q0.f != q0.f || q1.f != q1.f);
    // (the forward's span classification and packed pairs: the strain of
    // k_fwd_f32_shared)
    int codes = 0;
    if constexpr (MODEL != kModelTaylorF2) codes = span_codes<MODEL>(sT, lo, hi, lane);
    const Freq2 q2 = pack_freqs(q0, q1);
    float2* out = series + (POLARIZATIONS ? 2 : 1) * base * n_fft + m;
#pragma unroll 1
    for (int j = 0; j < count; ++j, out += (POLARIZATIONS ? 2 : 1) * n_fft) {
      const float* T = sT[j];
      SpanRegions sr;
      if constexpr (MODEL == kModelTaylorF2) {
        sr = span_regions<MODEL>(T, lo, hi, lane);
      } else {
        sr = span_code(codes, j);
      }
      sr.uniform = sr.uniform && !nan_span;
      float4 vp, vc;
      if (sr.above_cut && !nan_span) {
        const float zp = 0.0f * T[slot_kp<MODEL>()], zc = 0.0f * T[slot_kc<MODEL>()];
        vp = make_float4(zp, zp, zp, zp);
        vc = make_float4(zc, zc, zc, zc);
      } else if (!(sr.uniform && pair_packed<MODEL>(Bcast{T}, q2, sr, vp, vc))) {
        Point<float> p0, p1;
        span_pair<MODEL, true>(T, q0, q1, sr, p0, p1);
        project<MODEL>(T, p0, p1, vp, vc);
      }
      if constexpr (POLARIZATIONS) {
        // s conj(h) scale / S for h+ and hx
        const auto cross = [&](float4 h) {
          return make_float4(w0 * (s0.x * h.x + s0.y * h.y), w0 * (s0.y * h.x - s0.x * h.y),
                             w1 * (s1.x * h.z + s1.y * h.w), w1 * (s1.y * h.z - s1.x * h.w));
        };
        store_pair(out, 0, cross(vp), v0, v1);
        store_pair(out + n_fft, 0, cross(vc), v0, v1);
        float pp = w0 * (vp.x * vp.x + vp.y * vp.y) + w1 * (vp.z * vp.z + vp.w * vp.w);
        float xx = w0 * (vc.x * vc.x + vc.y * vc.y) + w1 * (vc.z * vc.z + vc.w * vc.w);
        float px = w0 * (vp.x * vc.x + vp.y * vc.y) + w1 * (vp.z * vc.z + vp.w * vc.w);
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) {
          pp += __shfl_xor_sync(0xffffffffu, pp, d);
          xx += __shfl_xor_sync(0xffffffffu, xx, d);
          px += __shfl_xor_sync(0xffffffffu, px, d);
        }
        if (lane == 0) {
          double* nb = norms + 4 * (base + j);
          atomicAdd(nb + 1, static_cast<double>(pp));
          atomicAdd(nb + 2, static_cast<double>(xx));
          atomicAdd(nb + 3, static_cast<double>(px));
        }
      } else {
        // h = fp h+ + fc hx; c = h conj(s) scale / S
        const float h0r = fp * vp.x + fc * vc.x, h0i = fp * vp.y + fc * vc.y;
        const float h1r = fp * vp.z + fc * vc.z, h1i = fp * vp.w + fc * vc.w;
        const float4 c = make_float4(h0r * sw.x - h0i * sw.y, h0r * sw.y + h0i * sw.x, h1r * sw.z - h1i * sw.w,
                                     h1r * sw.w + h1i * sw.z);
        store_pair(out, 0, c, v0, v1);
        float hh = w0 * (h0r * h0r + h0i * h0i) + w1 * (h1r * h1r + h1i * h1i);
#pragma unroll
        for (int d = 16; d > 0; d >>= 1) hh += __shfl_xor_sync(0xffffffffu, hh, d);
        if (lane == 0) atomicAdd(norms + 2 * (base + j), static_cast<double>(hh));
      }
    }
  }
}

// norms[stride b + ss_slot] = <s, s> = scale sum_k |s_k|^2 / S_k and the other
// stride - 1 norms of every template b zero (each block sums <s, s> itself).
__global__ void __launch_bounds__(kBlock) k_template_norms(const float2* __restrict__ signal,
                                                           const float* __restrict__ psd, int64_t n, int64_t B,
                                                           double scale, int stride, int ss_slot,
                                                           double* __restrict__ norms) {
  __shared__ double part[kBlock / 32];
  double ss = 0.0;
  for (int64_t k = threadIdx.x; k < n; k += kBlock) {
    const float2 sk = signal[k];
    ss += (static_cast<double>(sk.x) * sk.x + static_cast<double>(sk.y) * sk.y) / psd[k];
  }
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) ss += __shfl_xor_sync(0xffffffffu, ss, d);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = ss;
  __syncthreads();
  double total = 0.0;
#pragma unroll
  for (int w = 0; w < kBlock / 32; ++w) total += part[w];
  total *= scale;
  for (int64_t b = static_cast<int64_t>(blockIdx.x) * kBlock + threadIdx.x; b < B;
       b += static_cast<int64_t>(gridDim.x) * kBlock) {
    for (int k = 0; k < stride; ++k) norms[stride * b + k] = k == ss_slot ? total : 0.0;
  }
}

template <int MODEL, bool RAGGED>
__global__ void __launch_bounds__(kBlock) k_fwd_f32_tiles(const float* __restrict__ table,
                                                          const float* __restrict__ freqs,
                                                          const int64_t* __restrict__ offsets,
                                                          const int64_t* __restrict__ tile_prefix,
                                                          const int32_t* __restrict__ tile_map, int64_t n, int64_t B,
                                                          int64_t tile_len, int64_t tiles_per_binary, int64_t capacity,
                                                          const float* __restrict__ t_c, float2* __restrict__ hp,
                                                          float2* __restrict__ hc) {
  __shared__ __align__(16) float sT[kTableStride];
  // (ragged: never more items than the workspace holds, whatever tile_prefix says)
  const int64_t total = RAGGED ? min(tile_prefix[B], capacity) : B * tiles_per_binary;
  for (int64_t item = blockIdx.x; item < total; item += gridDim.x) {
    const Item it = item_of<RAGGED>(item, offsets, tile_prefix, tile_map, n, tile_len, tiles_per_binary);
    __syncthreads();
    if (threadIdx.x < kTableStride / 4) {
      reinterpret_cast<float4*>(sT)[threadIdx.x] =
          reinterpret_cast<const float4*>(table + it.b * kTableStride)[threadIdx.x];
    }
    __syncthreads();
    if (threadIdx.x == 0) prepare_model<MODEL, true>(sT, t_c != nullptr ? t_c[it.b] : 0.0f);
    __syncthreads();
    // (item-local 32-bit offsets r from s2, the even element at or below
    // the item's start; the block runs the same trip count, lanes past the
    // end evaluate the grid's first frequency and store nothing)
    const int64_t s2 = it.s & ~static_cast<int64_t>(1);
    const int lo_off = static_cast<int>(it.s - s2), hi_off = static_cast<int>(it.e - s2);
    const int npairs = (hi_off + 1) / 2;
    const float* fr = freqs + (s2 - it.fbase);
    float2* out_p = hp + s2;
    float2* out_c = hc + s2;
    for (int base = 0; base < npairs; base += kBlock) {
      const int pr = base + static_cast<int>(threadIdx.x), r = 2 * pr;
      const bool in = pr < npairs;
      const bool v0 = in && r >= lo_off && r < hi_off, v1 = in && r + 1 >= lo_off && r + 1 < hi_off;
      const float* a0 = v0 ? fr + r : (v1 ? fr + r + 1 : freqs);
      const float* a1 = v1 ? fr + r + 1 : a0;
      const float f0 = *a0, f1 = *a1;
      float4 vp, vc;
      if (!all_above_cutoff<MODEL>(sT, f0, f1, vp, vc)) {
        const Freq<float> q0 = freq_powers(f0);
        const Freq<float> q1 = freq_powers(f1);
        Point<float> p0, p1;
        point_pair<MODEL, float, true, true>(sT, q0, q1, TcF{}, p0, p1);
        project<MODEL>(sT, p0, p1, vp, vc);
      }
      store_pair(out_p, r, vp, v0, v1);
      store_pair(out_c, r, vc, v0, v1);
    }
  }
}

// ---------------------------------------------------------------------------
// ragged work items

// prefix[b] = sum over binaries < b of ceil(len_b / tile_len): one block.
// First the offsets are checked (offsets[0] >= 0, non-decreasing,
// offsets[B] == n): if they fail, *error = WFX_EOFFSETS and every prefix is
// 0 (no work item), else *error = 0. Valid offsets give at most
// n / tile_len + B items (each binary's ceil(len / tile_len) <= len /
// tile_len + 1), which carve() holds.
__global__ void k_tile_prefix(const int64_t* __restrict__ offsets, int64_t B, int64_t n, int64_t tile_len,
                              int64_t* prefix, int32_t* error) {
  __shared__ int64_t sums[1024];
  __shared__ int bad;
  const int t = threadIdx.x;
  const int64_t chunk = (B + blockDim.x - 1) / blockDim.x;
  const int64_t lo = min(B, t * chunk), hi = min(B, lo + chunk);
  if (t == 0) bad = 0;
  __syncthreads();
  bool ok = t != 0 || (offsets[0] >= 0 && offsets[B] == n);
  for (int64_t b = lo; b < hi; ++b) ok = ok && offsets[b] <= offsets[b + 1];
  if (!ok) bad = 1;
  __syncthreads();
  if (bad) {
    for (int64_t b = lo; b < hi; ++b) prefix[b] = 0;
    if (t == 0) {
      prefix[B] = 0;
      *error = WFX_EOFFSETS;
    }
    return;
  }
  if (t == 0) *error = 0;
  int64_t s = 0;
  for (int64_t b = lo; b < hi; ++b) {
    const int64_t len = offsets[b + 1] - offsets[b];
    s += (len + tile_len - 1) / tile_len;
  }
  sums[t] = s;
  __syncthreads();
  for (int d = 1; d < static_cast<int>(blockDim.x); d <<= 1) {
    int64_t v = t >= d ? sums[t - d] : 0;
    __syncthreads();
    sums[t] += v;
    __syncthreads();
  }
  int64_t run = t > 0 ? sums[t - 1] : 0;
  for (int64_t b = lo; b < hi; ++b) {
    prefix[b] = run;
    const int64_t len = offsets[b + 1] - offsets[b];
    run += (len + tile_len - 1) / tile_len;
  }
  if (t == static_cast<int>(blockDim.x) - 1) prefix[B] = sums[t];
}

// map[k] = the binary of work item k, for k below the workspace's capacity.
__global__ void k_tile_map(const int64_t* __restrict__ prefix, int64_t B, int64_t capacity, int32_t* map) {
  const int64_t b = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  if (b >= B) return;
  const int64_t end = min(prefix[b + 1], capacity);
  for (int64_t k = prefix[b]; k < end; ++k) map[k] = static_cast<int32_t>(b);
}

// ---------------------------------------------------------------------------
// FP32 reverse mode (vjp and fused likelihood)

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

struct FusedArgs {
  const void* data;
  int data_stride;
  const void* weights;
  int weights_stride;
  double fp, fc, scale;
  bool grad;
};

// The reverse pass's accumulators in compact order: the table slots it
// produces (slot_used), then nothing; kAccSlots per work item in the
// workspace.
constexpr int kAccSlots = 64;

struct AccMap {
  int slot[kAccSlots];  // table slot of compact accumulator c, or -1
  int tc, loss;         // compact indices of kSlotTc and kSlotLoss
};

template <int MODEL>
__host__ __device__ constexpr AccMap acc_map() {
  AccMap m{};
  int c = 0;
  for (int k = 0; k < kTableStride; ++k) {
    if (slot_used<MODEL>(k) && c < kAccSlots) {
      if (k == kSlotTc) m.tc = c;
      if (k == kSlotLoss) m.loss = c;
      m.slot[c++] = k;
    }
  }
  for (; c < kAccSlots; ++c) m.slot[c] = -1;
  return m;
}

template <int MODEL>
__host__ __device__ constexpr int acc_count() {
  int c = 0;
  for (int k = 0; k < kTableStride; ++k) c += slot_used<MODEL>(k) ? 1 : 0;
  return c;
}
static_assert(acc_count<kModelXas>() <= kAccSlots && acc_count<kModelPhenomD>() <= kAccSlots &&
                  acc_count<kModelTaylorF2>() <= kAccSlots,
              "the reverse pass's slots fit the compact accumulators");

// Sums v[0..63] over the lanes of a warp by recursive halving: at each step a
// lane keeps one half of its values, sends the other to its partner and adds
// the partner's; lane l ends with the sums of entries 2l and 2l + 1 (62
// shuffles for the 64 sums).
__device__ __forceinline__ float2 warp_reduce_scatter(float (&v)[kAccSlots], int lane) {
#pragma unroll
  for (int step = 0; step < 5; ++step) {
    const int half = kAccSlots >> (step + 1);
    const bool up = (lane >> (4 - step)) & 1;
#pragma unroll
    for (int i = 0; i < half; ++i) {
      const float keep = up ? v[i + half] : v[i];
      const float send = up ? v[i] : v[i + half];
      v[i] = keep + __shfl_xor_sync(0xffffffffu, send, 16 >> step);
    }
  }
  return make_float2(v[0], v[1]);
}

template <int MODEL, bool RAGGED, bool FUSED>
__global__ void __launch_bounds__(kBlock, 2) k_adj_f32(const float* __restrict__ table, const float* __restrict__ freqs,
                                                    const int64_t* __restrict__ offsets,
                                                    const int64_t* __restrict__ tile_prefix,
                                                    const int32_t* __restrict__ tile_map, int64_t n, int64_t B,
                                                    int64_t tile_len, int64_t tiles_per_binary, int64_t capacity,
                                                    const float* __restrict__ t_c, const float2* __restrict__ cot_hp,
                                                    const float2* __restrict__ cot_hc, FusedArgs fa,
                                                    float* __restrict__ partial, unsigned long long* claim) {
  // Each warp claims work items (binary, tile of frequencies) in turn from
  // the counter *claim (zero at the launch), so that warps resident early, or
  // on SMs that other kernels share, take more of them: it stages the
  // binary's table in its slice of shared memory, accumulates dL/dtable over
  // the tile in registers and leaves the warp's sums in partial[item] (no
  // block barriers).
  constexpr AccMap kMap = acc_map<MODEL>();
  __shared__ __align__(16) float sT[kBlock / 32][kTableStride];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  float* T = sT[warp];
  const float2* data = static_cast<const float2*>(fa.data);
  const float* weights = static_cast<const float*>(fa.weights);
  const float fp = static_cast<float>(fa.fp), fc = static_cast<float>(fa.fc);
  const float two_scale = static_cast<float>(2.0 * fa.scale);
  const int64_t total = RAGGED ? min(tile_prefix[B], capacity) : B * tiles_per_binary;
  const auto next = [&]() {
    unsigned long long k = 0;
    if (lane == 0) k = atomicAdd(claim, 1ull);
    return static_cast<int64_t>(__shfl_sync(0xffffffffu, k, 0));
  };
  for (int64_t item = next(); item < total; item = next()) {
    const Item it = item_of<RAGGED>(item, offsets, tile_prefix, tile_map, n, tile_len, tiles_per_binary);
    __syncwarp();
    if (lane < kTableStride / 4) {
      reinterpret_cast<float4*>(T)[lane] = __ldg(reinterpret_cast<const float4*>(table + it.b * kTableStride) + lane);
    }
    __syncwarp();
    if (lane == 0) prepare_model<MODEL>(T, t_c != nullptr ? t_c[it.b] : 0.0f);
    __syncwarp();
    float acc[kTableStride];
#pragma unroll
    for (int k = 0; k < kTableStride; ++k) acc[k] = 0.0f;
    float loss = 0.0f;
    // (item-local 32-bit offsets r from s2, the even element at or below
    // the item's start; lanes past the end evaluate the item's first
    // frequency with zero weight and cotangent: the warp runs the same trip
    // count)
    const int64_t s2 = it.s & ~static_cast<int64_t>(1);
    const int lo_off = static_cast<int>(it.s - s2), hi_off = static_cast<int>(it.e - s2);
    const int npairs = (hi_off + 1) / 2;
    const float* fr = freqs + (s2 - it.fbase);
    const float2* d_elem = data + s2;
    const float2* d_freq = data + (s2 - it.fbase);
    const float* w_elem = weights + s2;
    const float* w_freq = weights + (s2 - it.fbase);
    for (int base = 0; base < npairs; base += 32) {
      const int pr = base + lane, r = 2 * pr;
      const bool in = pr < npairs;
      const bool v0 = in && r >= lo_off && r < hi_off, v1 = in && r + 1 >= lo_off && r + 1 < hi_off;
      const int r0 = v0 ? r : (v1 ? r + 1 : lo_off), r1 = v1 ? r + 1 : r0;
      const float f0 = fr[r0], f1 = fr[r1];
      float4 vp, vc;
      const bool zero = all_above_cutoff<MODEL>(T, f0, f1, vp, vc);
      Freq<float> q0, q1;
      Point<float> p0, p1;
      if (!zero) {
        q0 = freq_powers(f0);
        q1 = freq_powers(f1);
        point_pair<MODEL, float, false>(T, q0, q1, TcF{}, p0, p1);
        if constexpr (FUSED) project<MODEL>(T, p0, p1, vp, vc);
      }
      float4 gp, gc;
      if constexpr (FUSED) {
        // r = fp h+ + fc hx - d; loss += w |r|^2; g = 2 scale w r
        float4 d;
        float w0, w1;
        if (fa.data_stride) {
          d = load_pair(d_elem, r, v0, v1);
        } else {
          const float2 a = d_freq[r0], bb = d_freq[r1];
          d = make_float4(a.x, a.y, bb.x, bb.y);
        }
        if (fa.weights_stride) {
          w0 = w_elem[r0];
          w1 = w_elem[r1];
        } else {
          w0 = w_freq[r0];
          w1 = w_freq[r1];
        }
        w0 = v0 ? w0 : 0.0f;
        w1 = v1 ? w1 : 0.0f;
        const float r0x = fp * vp.x + fc * vc.x - d.x, r0y = fp * vp.y + fc * vc.y - d.y;
        const float r1x = fp * vp.z + fc * vc.z - d.z, r1y = fp * vp.w + fc * vc.w - d.w;
        loss += w0 * (r0x * r0x + r0y * r0y) + w1 * (r1x * r1x + r1y * r1y);
        // (above the cutoff nothing depends on the table)
        if (!fa.grad || zero) continue;
        const float g0 = two_scale * w0, g1 = two_scale * w1;
        gp = make_float4(fp * g0 * r0x, fp * g0 * r0y, fp * g1 * r1x, fp * g1 * r1y);
        gc = make_float4(fc * g0 * r0x, fc * g0 * r0y, fc * g1 * r1x, fc * g1 * r1y);
      } else {
        if (zero) continue;
        gp = load_pair(cot_hp + s2, r, v0, v1);
        gc = load_pair(cot_hc + s2, r, v0, v1);
      }
      if (v0) adjoint<MODEL, float>(T, q0, p0, gp.x, gp.y, gc.x, gc.y, acc);
      if (v1) adjoint<MODEL, float>(T, q1, p1, gp.z, gp.w, gc.z, gc.w, acc);
    }
    acc[kSlotLoss] = static_cast<float>(fa.scale) * loss;
    float v[kAccSlots];
#pragma unroll
    for (int c = 0; c < kAccSlots; ++c) v[c] = kMap.slot[c] >= 0 ? acc[kMap.slot[c]] : 0.0f;
    const float2 sums = warp_reduce_scatter(v, lane);
    reinterpret_cast<float2*>(partial + item * kAccSlots)[lane] = sums;
  }
}

// The table slot of each compact accumulator, per model (-1 for none), for
// kernels that index it at run time.
template <int MODEL>
__constant__ AccMap kAccMapConst = acc_map<MODEL>();

// grad[b] = sum over b's items of partial . dtable (FP64), loss[b] likewise;
// one block of kAccSlots threads per binary: thread c sums accumulator c
// over the items (four loads in flight), multiplies it into its slot's row
// of dtable and the block adds the products of each direction (a warp
// shuffle tree, then the two warps' sums).
// Ragged: items below the workspace's capacity only; offsets that
// k_tile_prefix refused (*error != 0) give NaN loss and gradient.
template <int MODEL, class G, bool RAGGED>
__global__ void __launch_bounds__(kAccSlots) k_contract(const float* __restrict__ partial,
                                                       const int64_t* __restrict__ tile_prefix,
                                                       const int32_t* __restrict__ error, int64_t capacity,
                                                       int64_t tiles_per_binary, int64_t B,
                                                       const double* __restrict__ dtable, G* grad, G* loss) {
  static_assert(kAccSlots == 64 && kDirections == 8, "two warps, one 64-byte dtable row a thread");
  __shared__ double sw[2][kDirections];
  __shared__ double sx[2];  // the accumulators of t_c and of the loss
  const int64_t b = blockIdx.x;
  if (b >= B) return;
  const int c = threadIdx.x, lane = c & 31, warp = c >> 5;
  if (RAGGED && *error != 0) {
    if (grad != nullptr && c < kGradColumns) grad[b * kGradColumns + c] = static_cast<G>(NAN);
    if (loss != nullptr && c == kDirections + 1) loss[b] = static_cast<G>(NAN);
    return;
  }
  const int64_t i1 = RAGGED ? min(tile_prefix[b + 1], capacity) : b * tiles_per_binary + tiles_per_binary;
  const int64_t i0 = RAGGED ? min(tile_prefix[b], i1) : b * tiles_per_binary;
  double a0 = 0.0, a1 = 0.0, a2 = 0.0, a3 = 0.0;
  int64_t i = i0;
  for (; i + 4 <= i1; i += 4) {
    a0 += partial[i * kAccSlots + c];
    a1 += partial[(i + 1) * kAccSlots + c];
    a2 += partial[(i + 2) * kAccSlots + c];
    a3 += partial[(i + 3) * kAccSlots + c];
  }
  for (; i < i1; ++i) a0 += partial[i * kAccSlots + c];
  const double a = (a0 + a1) + (a2 + a3);
  const int k = kAccMapConst<MODEL>.slot[c];
  if (c == kAccMapConst<MODEL>.tc) sx[0] = a;
  if (c == kAccMapConst<MODEL>.loss) sx[1] = a;
  if (grad != nullptr && dtable != nullptr) {
    const bool use = k >= 0 && k != kSlotTc && k != kSlotLoss;
    double v[kDirections];
    if (use) {
      const double4* row = reinterpret_cast<const double4*>(dtable + (b * kTableStride + k) * kDirections);
      const double4 lo = row[0], hi = row[1];
      v[0] = a * lo.x; v[1] = a * lo.y; v[2] = a * lo.z; v[3] = a * lo.w;
      v[4] = a * hi.x; v[5] = a * hi.y; v[6] = a * hi.z; v[7] = a * hi.w;
    } else {
#pragma unroll
      for (int d = 0; d < kDirections; ++d) v[d] = 0.0;
    }
    double mine = 0.0;
#pragma unroll
    for (int d = 0; d < kDirections; ++d) {
      const double t = warp_sum(v[d]);
      mine = lane == d ? t : mine;
    }
    if (lane < kDirections) sw[warp][lane] = mine;
  }
  __syncthreads();
  if (grad != nullptr && dtable != nullptr && c < kDirections) {
    grad[b * kGradColumns + c] = static_cast<G>(sw[0][c] + sw[1][c]);
  }
  if (grad != nullptr && c == kDirections) grad[b * kGradColumns + kDirections] = static_cast<G>(sx[0]);
  if (loss != nullptr && c == kDirections + 1) loss[b] = static_cast<G>(sx[1]);
}

// ---------------------------------------------------------------------------
// FP64 plain form: one binary per block

template <int MODEL>
__global__ void __launch_bounds__(kBlock) k_fwd_f64(const double* __restrict__ table,
                                                    const double* __restrict__ freqs,
                                                    const int64_t* __restrict__ offsets, int64_t n, int64_t B,
                                                    const double* __restrict__ t_c, double2* __restrict__ hp,
                                                    double2* __restrict__ hc) {
  __shared__ double sT[kTableStride];
  for (int64_t b = blockIdx.x; b < B; b += gridDim.x) {
    __syncthreads();
    if (threadIdx.x < kTableStride) sT[threadIdx.x] = table[b * kTableStride + threadIdx.x];
    __syncthreads();
    const double tc = t_c != nullptr ? t_c[b] : 0.0;
    const int64_t rs = offsets != nullptr ? min(max(offsets[b], int64_t(0)), n) : b * n;
    const int64_t re = offsets != nullptr ? min(max(offsets[b + 1], rs), n) : rs + n;
    const int64_t fbase = offsets != nullptr ? 0 : rs;
    const double kp = sT[slot_kp<MODEL>()], kc = sT[slot_kc<MODEL>()];
    for (int64_t e = rs + threadIdx.x; e < re; e += blockDim.x) {
      const Freq<double> q = freq_powers(freqs[e - fbase]);
      const Point<double> pt = point<MODEL, double>(sT, q, tc);
      const double ap = kp * pt.amp, ac = kc * pt.amp;
      hp[e] = make_double2(ap * pt.c, ap * pt.s);
      hc[e] = make_double2(-ac * pt.s, ac * pt.c);
    }
  }
}


// d L / d f for the cotangents (g+, gx) of (h+, hx) (the derivative with
// respect to the grid of the reference's drop-in, src/waveformx/torch.py:
// 12-13, 87-91): the FP64 point evaluated on Dual frequencies
// (freq_powers_dual), contracted with the cotangents; one binary per block.
// A shared grid's grad_f (n, zeroed beforehand) sums over the binaries
// (one atomic per element and binary); a ragged one has its own element.
// As the reference's, the set-up (f_min = the first frequency) carries no
// derivative.
template <int MODEL>
__global__ void __launch_bounds__(kBlock) k_grid_vjp(const double* __restrict__ table, const double* __restrict__ freqs,
                                                     const int64_t* __restrict__ offsets, int64_t n, int64_t B,
                                                     const double* __restrict__ t_c,
                                                     const double2* __restrict__ cot_hp,
                                                     const double2* __restrict__ cot_hc, double* __restrict__ grad_f) {
  __shared__ __align__(16) double raw[2 * kTableStride];  // (Dual has a constructor: raw storage)
  Dual* sT = reinterpret_cast<Dual*>(raw);
  for (int64_t b = blockIdx.x; b < B; b += gridDim.x) {
    __syncthreads();
    if (threadIdx.x < kTableStride) sT[threadIdx.x] = Dual(table[b * kTableStride + threadIdx.x], 0.0);
    __syncthreads();
    const double tc = t_c != nullptr ? t_c[b] : 0.0;
    const int64_t rs = offsets != nullptr ? min(max(offsets[b], int64_t(0)), n) : b * n;
    const int64_t re = offsets != nullptr ? min(max(offsets[b + 1], rs), n) : rs + n;
    const int64_t fbase = offsets != nullptr ? 0 : rs;
    const double kp = sT[slot_kp<MODEL>()].v, kc = sT[slot_kc<MODEL>()].v;
    for (int64_t e = rs + threadIdx.x; e < re; e += blockDim.x) {
      const Freq<Dual> q = freq_powers_dual(freqs[e - fbase]);
      const Point<Dual> pt = point<MODEL, Dual>(sT, q, tc);
      const Dual ac = pt.amp * pt.c, as = pt.amp * pt.s;
      const double2 gp = cot_hp[e], gc = cot_hc[e];
      // h+ = kp A (c, s), hx = kc A (-s, c)
      const double d = kp * (gp.x * ac.d + gp.y * as.d) + kc * (-gc.x * as.d + gc.y * ac.d);
      if (offsets != nullptr) {
        grad_f[e] = d;
      } else {
        atomicAdd(&grad_f[e - fbase], d);
      }
    }
  }
}

template <int MODEL, bool FUSED>
__global__ void __launch_bounds__(128) k_adj_f64(const double* __restrict__ table, const double* __restrict__ freqs,
                                                 const int64_t* __restrict__ offsets, int64_t n, int64_t B,
                                                 const double* __restrict__ t_c, const double2* __restrict__ cot_hp,
                                                 const double2* __restrict__ cot_hc, FusedArgs fa,
                                                 const double* __restrict__ dtable, double* grad, double* loss_out) {
  constexpr int kAdjBlock = 128;
  __shared__ double sT[kTableStride];
  __shared__ double red[kAdjBlock / 32][kTableStride];
  __shared__ double sa[kTableStride];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const double2* data = static_cast<const double2*>(fa.data);
  const double* weights = static_cast<const double*>(fa.weights);
  for (int64_t b = blockIdx.x; b < B; b += gridDim.x) {
    __syncthreads();
    if (threadIdx.x < kTableStride) sT[threadIdx.x] = table[b * kTableStride + threadIdx.x];
    __syncthreads();
    const double tc = t_c != nullptr ? t_c[b] : 0.0;
    const int64_t rs = offsets != nullptr ? min(max(offsets[b], int64_t(0)), n) : b * n;
    const int64_t re = offsets != nullptr ? min(max(offsets[b + 1], rs), n) : rs + n;
    const int64_t fbase = offsets != nullptr ? 0 : rs;
    double acc[kTableStride];
#pragma unroll
    for (int k = 0; k < kTableStride; ++k) acc[k] = 0.0;
    double loss = 0.0;
    for (int64_t e = rs + threadIdx.x; e < re; e += kAdjBlock) {
      const Freq<double> q = freq_powers(freqs[e - fbase]);
      const Point<double> pt = point<MODEL, double>(sT, q, tc);
      double2 gp, gc;
      if constexpr (FUSED) {
        const double ap = sT[slot_kp<MODEL>()] * pt.amp, ac = sT[slot_kc<MODEL>()] * pt.amp;
        const double2 d = data[fa.data_stride ? e : e - fbase];
        const double w = weights[fa.weights_stride ? e : e - fbase];
        const double rx = fa.fp * (ap * pt.c) + fa.fc * (-ac * pt.s) - d.x;
        const double ry = fa.fp * (ap * pt.s) + fa.fc * (ac * pt.c) - d.y;
        loss += w * (rx * rx + ry * ry);
        const double g = 2.0 * fa.scale * w;
        gp = make_double2(fa.fp * g * rx, fa.fp * g * ry);
        gc = make_double2(fa.fc * g * rx, fa.fc * g * ry);
        if (!fa.grad) continue;
      } else {
        gp = cot_hp[e];
        gc = cot_hc[e];
      }
      adjoint<MODEL, double>(sT, q, pt, gp.x, gp.y, gc.x, gc.y, acc);
    }
    acc[kSlotLoss] = fa.scale * loss;
#pragma unroll
    for (int k = 0; k < kTableStride; ++k) {
      if (slot_used<MODEL>(k)) {
        const double v = warp_sum(acc[k]);
        if (lane == 0) red[warp][k] = v;
      } else if (lane == 0) {
        red[warp][k] = 0.0;
      }
    }
    __syncthreads();
    if (threadIdx.x < kTableStride) {
      double s = 0.0;
      for (int w = 0; w < kAdjBlock / 32; ++w) s += red[w][threadIdx.x];
      sa[threadIdx.x] = s;
    }
    __syncthreads();
    const int k = threadIdx.x;
    if (grad != nullptr && k < kDirections && dtable != nullptr) {
      double g = 0.0;
      for (int j = 0; j < kTableStride; ++j) g += sa[j] * dtable[(b * kTableStride + j) * kDirections + k];
      grad[b * kGradColumns + k] = g;
    }
    if (grad != nullptr && k == kDirections) grad[b * kGradColumns + kDirections] = sa[kSlotTc];
    if (loss_out != nullptr && k == kDirections + 1) loss_out[b] = sa[kSlotLoss];
  }
}

// ---------------------------------------------------------------------------
// host side

int device_sms() {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return 0;
  int sms = 0;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return 0;
  return sms;
}

// The blocks of `Kernel` (block size `threads`) that fit on the device at
// once: the grid of a persistent launch.
// (Cached per kernel and device: the query costs microseconds of host time.)
template <auto Kernel>
int64_t resident_blocks(int threads) {
  constexpr int kDevices = 64;
  static int64_t cache[kDevices] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev >= 0 && dev < kDevices && cache[dev] > 0) return cache[dev];
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, Kernel, threads, 0) != cudaSuccess || per_sm < 1)
    per_sm = 1;
  const int64_t blocks = static_cast<int64_t>(per_sm) * max(device_sms(), 1);
  if (dev >= 0 && dev < kDevices) cache[dev] = blocks;
  return blocks;
}

int launched() {
  const cudaError_t err = cudaGetLastError();
  return err == cudaSuccess ? 0 : static_cast<int>(err);
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

// The adjoint tile length of a shared grid of n frequencies: the longest
// even length that splits n into equal tiles of at most kAdjTileMax,
// kAdjTileMax / 2 or kAdjTileMax / 4 frequencies and still gives the batch
// kAdjItems work items (else the shortest). The warps claim items as they
// go, so short items balance the SMs of a small batch (1024 x 4017: 8192
// items of 504 frequencies, 68.6 us, against 2048 of 2010, 82.9 us, and
// 75.3 us with 4096 of 1006; 16384 of 252: 72.3 us), while long ones cost
// fewer stagings and reductions where items are plenty (65536 x 8192:
// 3.67 ms with tiles of 1640, 4.02 ms with 820, 4.69 ms with 410).
constexpr int64_t kAdjItems = 8192;

int64_t adj_tile_len(int64_t B, int64_t n) {
  int64_t len = 0;
  for (int64_t cap = kAdjTileMax; cap >= kAdjTileMax / 4 - 1; cap = cap / 2 - 1) {
    const int64_t tiles = (n + cap - 1) / cap;
    len = (n + tiles - 1) / tiles;
    len += len & 1;
    if (B * tiles >= kAdjItems) break;
  }
  return len;
}

struct Workspace {
  int32_t* error;  // ragged: the offsets' status word, at the start of the workspace
  int64_t* tile_prefix;
  int32_t* tile_map;
  float* partial;
  unsigned long long* claim;  // the reverse pass's next work item (zeroed before its launch)
  int64_t items;              // the work items the workspace holds
  size_t bytes;
};

size_t align256(size_t x) { return (x + 255) & ~static_cast<size_t>(255); }

// Scratch of the FP32 reverse pass (and of the ragged forward's work items).
Workspace carve(void* base, int64_t B, int64_t n, bool ragged, int64_t tile_len, bool partials) {
  Workspace w{};
  char* p = static_cast<char*>(base);
  size_t used = 0;
  int64_t items;
  if (ragged) {
    items = n / tile_len + B + 1;
    w.error = reinterpret_cast<int32_t*>(p ? p + used : nullptr);
    used += align256(sizeof(int32_t));
    w.tile_prefix = reinterpret_cast<int64_t*>(p ? p + used : nullptr);
    used += align256(sizeof(int64_t) * (B + 1));
    w.tile_map = reinterpret_cast<int32_t*>(p ? p + used : nullptr);
    used += align256(sizeof(int32_t) * items);
  } else {
    items = B * ((n + tile_len - 1) / tile_len);
  }
  if (partials) {
    w.partial = reinterpret_cast<float*>(p ? p + used : nullptr);
    used += align256(sizeof(float) * kAccSlots * items);
    w.claim = reinterpret_cast<unsigned long long*>(p ? p + used : nullptr);
    used += align256(sizeof(unsigned long long));
  }
  w.items = items;
  w.bytes = used;
  return w;
}

int build_items(const int64_t* offsets, int64_t B, int64_t n, int64_t tile_len, Workspace& w, cudaStream_t s) {
  k_tile_prefix<<<1, 1024, 0, s>>>(offsets, B, n, tile_len, w.tile_prefix, w.error);
  k_tile_map<<<static_cast<unsigned>((B + 255) / 256), 256, 0, s>>>(w.tile_prefix, B, w.items, w.tile_map);
  return launched();
}

// ---------------------------------------------------------------------------
// tuning of the ragged forward: the length of a work item and the blocks per
// SM of its persistent launch, per device, model and size class (log2 of
// the frequencies and of the binaries). Set by wfx_autotune_ragged or
// wfx_tuning; the process-wide table is guarded by a mutex.

struct RaggedConfig {
  int64_t tile_len;
  int64_t blocks_per_sm;
};
constexpr RaggedConfig kRaggedDefault{4 * kBlock - 2, 8};
constexpr int64_t kRaggedTileCandidates[] = {2 * kBlock - 2, 4 * kBlock - 2, 8 * kBlock - 2, 16 * kBlock - 2};
constexpr int64_t kRaggedBlocksCandidates[] = {2, 4, 8, 16};

using TuneKey = std::tuple<int, int, int, int>;  // device, model, log2 n, log2 B
std::mutex g_tune_mutex;
std::map<TuneKey, RaggedConfig> g_tune;

int floor_log2(int64_t x) {
  int k = 0;
  while (x > 1) {
    x >>= 1;
    ++k;
  }
  return k;
}

TuneKey tune_key(int model, int64_t B, int64_t n) {
  int dev = 0;
  cudaGetDevice(&dev);
  return TuneKey{dev, model, floor_log2(n), floor_log2(B)};
}

RaggedConfig ragged_config(int model, int64_t B, int64_t n) {
  const TuneKey key = tune_key(model, B, n);
  std::lock_guard<std::mutex> lock(g_tune_mutex);
  const auto it = g_tune.find(key);
  return it == g_tune.end() ? kRaggedDefault : it->second;
}

bool valid_config(const RaggedConfig& c) {
  return c.tile_len >= kRaggedTileMin && c.tile_len <= (int64_t(1) << 30) && c.blocks_per_sm >= 1 &&
         c.blocks_per_sm <= 64;
}

template <int MODEL>
int ragged_f32(const float* table, const float* freqs, const int64_t* offsets, int64_t B, int64_t n, const float* t_c,
               float2* hp, float2* hc, void* scratch, RaggedConfig c, cudaStream_t s) {
  // (the workspace is laid out for the shortest item: any tuned length fits)
  Workspace w = carve(scratch, B, n, true, kRaggedTileMin, false);
  if (int rc = build_items(offsets, B, n, c.tile_len, w, s)) return rc;
  const int64_t upper = n / c.tile_len + B + 1;
  const int64_t grid = min(upper, static_cast<int64_t>(max(device_sms(), 1)) * c.blocks_per_sm);
  k_fwd_f32_tiles<MODEL, true><<<static_cast<unsigned>(grid), kBlock, 0, s>>>(
      table, freqs, offsets, w.tile_prefix, w.tile_map, n, B, c.tile_len, 0, w.items, t_c, hp, hc);
  return launched();
}

template <int MODEL>
int polarizations_f32(const float* table, const float* freqs, const int64_t* offsets, int64_t B, int64_t n,
                      const float* t_c, float2* hp, float2* hc, void* scratch, cudaStream_t s) {
  if (offsets == nullptr) {
    const int64_t tiles = (n + kFwdTile - 1) / kFwdTile;
    const int64_t groups = (B + kBinariesPerBlock - 1) / kBinariesPerBlock;
    // (grid dimensions y and z hold at most 65535: more tiles loop in the
    // block, more groups take further launches)
    constexpr int64_t kMaxY = 65535;
    const int64_t per_launch = fwd_group_major<MODEL>() ? kMaxY : (int64_t(1) << 31) - 1;
    for (int64_t g0 = 0; g0 < groups; g0 += per_launch) {
      const int64_t g = min(groups - g0, per_launch);
      const unsigned t = static_cast<unsigned>(min(tiles, fwd_group_major<MODEL>() ? (int64_t(1) << 31) - 1 : kMaxY));
      const dim3 grid = fwd_group_major<MODEL>() ? dim3(t, static_cast<unsigned>(g)) : dim3(static_cast<unsigned>(g), t);
      k_fwd_f32_shared<MODEL><<<grid, kBlock, 0, s>>>(table, freqs, n, B, g0, t_c, hp, hc);
      if (int rc = launched()) return rc;
    }
    return 0;
  }
  return ragged_f32<MODEL>(table, freqs, offsets, B, n, t_c, hp, hc, scratch, ragged_config(MODEL, B, n), s);
}

// The stages of the FP32 reverse pass: the per-item sums (the reverse
// kernel), their contraction with dtable, or both in turn.
enum AdjointStage : int { kStagePartials = 1, kStageContract = 2, kStageAll = 3 };

template <int MODEL>
int adjoint_f32(bool fused, const float* table, const double* dtable, const float* freqs, const int64_t* offsets,
                int64_t B, int64_t n, const float* t_c, const float2* cot_hp, const float2* cot_hc, FusedArgs fa,
                float* loss, float* grad, void* workspace, cudaStream_t s, int stage = kStageAll) {
  const bool ragged = offsets != nullptr;
  const int64_t tile_len = ragged ? kAdjTileMax : adj_tile_len(B, n);
  Workspace w = carve(workspace, B, n, ragged, tile_len, true);
  const int64_t tpb = ragged ? 0 : (n + tile_len - 1) / tile_len;
  const int64_t upper = ragged ? n / tile_len + B + 1 : B * tpb;
  if (stage & kStagePartials) {
    if (ragged) {
      if (int rc = build_items(offsets, B, n, tile_len, w, s)) return rc;
    }
    // one warp per work item, at most the blocks that are resident at once
    const int64_t wanted = (upper + kBlock / 32 - 1) / (kBlock / 32);
    const cudaError_t zeroed = cudaMemsetAsync(w.claim, 0, sizeof(unsigned long long), s);
    if (zeroed != cudaSuccess) return static_cast<int>(zeroed);
#define WFX_ADJ(R, F)                                                                                          \
  do {                                                                                                        \
    const int64_t grid = min(wanted, resident_blocks<k_adj_f32<MODEL, R, F>>(kBlock));                        \
    k_adj_f32<MODEL, R, F><<<static_cast<unsigned>(grid > 1 ? grid : int64_t(1)), kBlock, 0, s>>>(           \
        table, freqs, offsets, w.tile_prefix, w.tile_map, n, B, tile_len, tpb, w.items, t_c, cot_hp, cot_hc,    \
        fa, w.partial, w.claim);                                                                              \
  } while (0)
    if (ragged) {
      if (fused) {
        WFX_ADJ(true, true);
      } else {
        WFX_ADJ(true, false);
      }
    } else {
      if (fused) {
        WFX_ADJ(false, true);
      } else {
        WFX_ADJ(false, false);
      }
    }
#undef WFX_ADJ
    if (int rc = launched()) return rc;
  }
  if (!(stage & kStageContract)) return 0;
  if (ragged) {
    k_contract<MODEL, float, true><<<static_cast<unsigned>(B), kAccSlots, 0, s>>>(
        w.partial, w.tile_prefix, w.error, w.items, 0, B, dtable, grad, loss);
  } else {
    k_contract<MODEL, float, false><<<static_cast<unsigned>(B), kAccSlots, 0, s>>>(
        w.partial, nullptr, nullptr, w.items, tpb, B, dtable, grad, loss);
  }
  return launched();
}

int check_model(int model) {
  return (model == kModelXas || model == kModelPhenomD || model == kModelTaylorF2) ? 0 : WFX_EINVAL;
}

// fn(std::integral_constant<int, MODEL>) for the model code `model` (one of
// check_model's), so that host code instantiates the kernels of each model
// from one call site.
template <class F>
int with_model(int model, F&& fn) {
  switch (model) {
    case kModelXas:
      return fn(std::integral_constant<int, kModelXas>{});
    case kModelPhenomD:
      return fn(std::integral_constant<int, kModelPhenomD>{});
    case kModelTaylorF2:
      return fn(std::integral_constant<int, kModelTaylorF2>{});
    default:
      return WFX_EINVAL;
  }
}

// ---------------------------------------------------------------------------
// the static scratch of wfx_fused_loss_noalloc
//
// One buffer per device, part of the module's global memory (no allocation
// at run time). Its address is looked up with the device current and cached
// with the id of the context it was looked up in: a new context on the
// device (after cudaDeviceReset, for instance) loads the module again, and
// the address is looked up again. Every byte a call uses is written by that
// call's own kernels before they read it, so nothing needs to start at zero;
// calls in flight at the same time on one device share it and race.
static __device__ __align__(256) unsigned char g_static_scratch[WFX_STATIC_SCRATCH_BYTES];

constexpr int kMaxDevices = 64;

// The current context's unique id (cuCtxGetCurrent, cuCtxGetId, reached
// through the runtime's driver entry points: the library links the runtime
// only), or 0 when there is none or the driver lacks them.
unsigned long long current_context_id() {
  using GetCurrent = int (*)(void**);
  using GetId = int (*)(void*, unsigned long long*);
  static GetCurrent get_current = nullptr;
  static GetId get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = reinterpret_cast<GetCurrent>(f);
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = reinterpret_cast<GetId>(f);
  });
  if (get_current == nullptr || get_id == nullptr) return 0;
  void* ctx = nullptr;
  unsigned long long id = 0;
  if (get_current(&ctx) != 0 || ctx == nullptr || get_id(ctx, &id) != 0) return 0;
  return id;
}

struct ScratchAddress {
  unsigned long long context;
  void* ptr;
};
std::mutex g_scratch_mutex;
ScratchAddress g_scratch_address[kMaxDevices];

int static_scratch(void** ptr) {
  int dev = -1;
  cudaError_t rc = cudaGetDevice(&dev);
  if (rc != cudaSuccess) return static_cast<int>(rc);
  if (dev < 0 || dev >= kMaxDevices) return WFX_EDEVICE;
  unsigned long long context = current_context_id();
  if (context != 0) {
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    const ScratchAddress& a = g_scratch_address[dev];
    if (a.context == context && a.ptr != nullptr) {
      *ptr = a.ptr;
      return 0;
    }
  }
  // (looked up in the current context; the lookup makes the device's primary
  // context current if none was)
  void* p = nullptr;
  rc = cudaGetSymbolAddress(&p, g_static_scratch);
  if (rc != cudaSuccess) return static_cast<int>(rc);
  context = current_context_id();
  {
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    g_scratch_address[dev] = ScratchAddress{context, p};
  }
  *ptr = p;
  return 0;
}

}  // namespace wfx

using namespace wfx;

extern "C" {

int wfx_version(void) { return 100; }

const char* wfx_status_string(int code) {
  switch (code) {
    case 0:
      return "success";
    case WFX_EINVAL:
      return "invalid argument (null pointer, non-positive size, unknown model or misaligned buffer)";
    case WFX_EOFFSETS:
      return "ragged offsets inconsistent with n (offsets[0] < 0, decreasing, or offsets[B] != n)";
    case WFX_EWORKSPACE:
      return "workspace missing or smaller than wfx_workspace_bytes()";
    case WFX_EDEVICE:
      return "no usable CUDA device";
    case WFX_ESCRATCH:
      return "problem larger than the library's static scratch (WFX_STATIC_SCRATCH_BYTES)";
    default:
      return code > 0 ? cudaGetErrorString(static_cast<cudaError_t>(code)) : "unknown error";
  }
}

int wfx_ragged_status(const void* workspace, wfx_stream_t stream) {
  if (workspace == nullptr) return WFX_EINVAL;
  const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  int32_t word = 0;
  cudaError_t rc = cudaMemcpyAsync(&word, workspace, sizeof(word), cudaMemcpyDeviceToHost, s);
  if (rc == cudaSuccess) rc = cudaStreamSynchronize(s);
  if (rc != cudaSuccess) return static_cast<int>(rc);
  return (word == 0 || word == WFX_EOFFSETS) ? word : WFX_EINVAL;
}

size_t wfx_workspace_bytes(int op, int model, int precision, int64_t B, int64_t n, int ragged) {
  if (check_model(model) || B <= 0 || n < 0) return 0;
  if (precision == WFX_FP64) return 0;
  if (op == WFX_OP_VJP || op == WFX_OP_FUSED) {
    const int64_t tile_len = ragged ? kAdjTileMax : adj_tile_len(B, n > 0 ? n : 1);
    return carve(nullptr, B, n, ragged != 0, tile_len, true).bytes;
  }
  if (op == WFX_OP_POLARIZATIONS && ragged) return carve(nullptr, B, n, true, kRaggedTileMin, false).bytes;
  return 0;
}

int wfx_grid_vjp(int model, const double* table, const double* freqs, const int64_t* offsets, int64_t B, int64_t n,
                 const double* t_c, const void* cot_hp, const void* cot_hc, double* grad_f, wfx_stream_t stream) {
  if (table == nullptr || freqs == nullptr || cot_hp == nullptr || cot_hc == nullptr || grad_f == nullptr || B <= 0 ||
      n <= 0 || (model != kModelXhm && check_model(model)))
    return WFX_EINVAL;
  const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const cudaError_t rc = cudaMemsetAsync(grad_f, 0, sizeof(double) * static_cast<size_t>(n), s);
  if (rc != cudaSuccess) return static_cast<int>(rc);
  if (model == kModelXhm) return xhm_grid_vjp(table, freqs, offsets, B, n, t_c, cot_hp, cot_hc, grad_f, s);
  const unsigned grid = static_cast<unsigned>(B < 65535 ? B : 65535);
  const auto* gp = static_cast<const double2*>(cot_hp);
  const auto* gc = static_cast<const double2*>(cot_hc);
  if (model == kModelXas) {
    k_grid_vjp<kModelXas><<<grid, kBlock, 0, s>>>(table, freqs, offsets, n, B, t_c, gp, gc, grad_f);
  } else if (model == kModelPhenomD) {
    k_grid_vjp<kModelPhenomD><<<grid, kBlock, 0, s>>>(table, freqs, offsets, n, B, t_c, gp, gc, grad_f);
  } else {
    k_grid_vjp<kModelTaylorF2><<<grid, kBlock, 0, s>>>(table, freqs, offsets, n, B, t_c, gp, gc, grad_f);
  }
  const cudaError_t err = cudaGetLastError();
  return err == cudaSuccess ? 0 : static_cast<int>(err);
}

int wfx_polarizations(int model, int precision, const void* table, const void* freqs, const int64_t* offsets,
                      int64_t B, int64_t n, const void* t_c, void* hp, void* hc, void* workspace,
                      size_t workspace_bytes, wfx_stream_t stream) {
  if (check_model(model) || table == nullptr || freqs == nullptr || hp == nullptr || hc == nullptr || B <= 0 ||
      n <= 0)
    return WFX_EINVAL;
  const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (precision == WFX_FP64) {
    const unsigned grid = static_cast<unsigned>((B < (int64_t(1) << 20) ? B : (int64_t(1) << 20)));
    return with_model(model, [&](auto m) {
      k_fwd_f64<decltype(m)::value><<<grid, kBlock, 0, s>>>(
          static_cast<const double*>(table), static_cast<const double*>(freqs), offsets, n, B,
          static_cast<const double*>(t_c), static_cast<double2*>(hp), static_cast<double2*>(hc));
      return launched();
    });
  }
  if (precision != WFX_FP32) return WFX_EINVAL;
  if (!aligned16(table) || !aligned16(hp) || !aligned16(hc)) return WFX_EINVAL;
  if (offsets != nullptr &&
      (workspace == nullptr ||
       workspace_bytes < wfx_workspace_bytes(WFX_OP_POLARIZATIONS, model, WFX_FP32, B, n, 1)))
    return WFX_EWORKSPACE;
  const auto* T = static_cast<const float*>(table);
  const auto* F = static_cast<const float*>(freqs);
  const auto* TC = static_cast<const float*>(t_c);
  auto* P = static_cast<float2*>(hp);
  auto* C = static_cast<float2*>(hc);
  return with_model(model, [&](auto m) {
    return polarizations_f32<decltype(m)::value>(T, F, offsets, B, n, TC, P, C, workspace, s);
  });
}

static int adjoint_entry(bool fused, int model, int precision, const void* table, const double* dtable,
                         const void* freqs, const int64_t* offsets, int64_t B, int64_t n, const void* t_c,
                         const void* cot_hp, const void* cot_hc, FusedArgs fa, void* loss, void* grad,
                         void* workspace, size_t workspace_bytes, wfx_stream_t stream) {
  if (check_model(model) || table == nullptr || freqs == nullptr || B <= 0 || n <= 0) return WFX_EINVAL;
  if (grad != nullptr && dtable == nullptr) return WFX_EINVAL;
  if (!fused && (cot_hp == nullptr || cot_hc == nullptr || grad == nullptr)) return WFX_EINVAL;
  if (fused && (fa.data == nullptr || fa.weights == nullptr || (loss == nullptr && grad == nullptr)))
    return WFX_EINVAL;
  const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (precision == WFX_FP64) {
    const unsigned grid = static_cast<unsigned>((B < (int64_t(1) << 20) ? B : (int64_t(1) << 20)));
    const auto* T = static_cast<const double*>(table);
    const auto* F = static_cast<const double*>(freqs);
    const auto* TC = static_cast<const double*>(t_c);
    const auto* CP = static_cast<const double2*>(cot_hp);
    const auto* CC = static_cast<const double2*>(cot_hc);
    auto* G = static_cast<double*>(grad);
    auto* L = static_cast<double*>(loss);
    return with_model(model, [&](auto m) {
      constexpr int M = decltype(m)::value;
      if (fused) {
        k_adj_f64<M, true><<<grid, 128, 0, s>>>(T, F, offsets, n, B, TC, CP, CC, fa, dtable, G, L);
      } else {
        k_adj_f64<M, false><<<grid, 128, 0, s>>>(T, F, offsets, n, B, TC, CP, CC, fa, dtable, G, L);
      }
      return launched();
    });
  }
  if (precision != WFX_FP32) return WFX_EINVAL;
  if (!aligned16(table) || (cot_hp && !aligned16(cot_hp)) || (cot_hc && !aligned16(cot_hc))) return WFX_EINVAL;
  if (fused && fa.data_stride && !aligned16(fa.data)) return WFX_EINVAL;
  if (workspace == nullptr ||
      workspace_bytes < wfx_workspace_bytes(fused ? WFX_OP_FUSED : WFX_OP_VJP, model, precision, B, n, offsets != nullptr))
    return WFX_EWORKSPACE;
  const auto* T = static_cast<const float*>(table);
  const auto* F = static_cast<const float*>(freqs);
  const auto* TC = static_cast<const float*>(t_c);
  const auto* CP = static_cast<const float2*>(cot_hp);
  const auto* CC = static_cast<const float2*>(cot_hc);
  auto* G = static_cast<float*>(grad);
  auto* L = static_cast<float*>(loss);
  return with_model(model, [&](auto m) {
    return adjoint_f32<decltype(m)::value>(fused, T, dtable, F, offsets, B, n, TC, CP, CC, fa, L, G, workspace, s);
  });
}

int wfx_vjp(int model, int precision, const void* table, const double* dtable, const void* freqs,
            const int64_t* offsets, int64_t B, int64_t n, const void* t_c, const void* cot_hp, const void* cot_hc,
            void* grad, void* workspace, size_t workspace_bytes, wfx_stream_t stream) {
  FusedArgs fa{nullptr, 0, nullptr, 0, 0.0, 0.0, 0.0, true};
  return adjoint_entry(false, model, precision, table, dtable, freqs, offsets, B, n, t_c, cot_hp, cot_hc, fa,
                       nullptr, grad, workspace, workspace_bytes, stream);
}

int wfx_fused_loss(int model, int precision, const void* table, const double* dtable, const void* freqs,
                   const int64_t* offsets, int64_t B, int64_t n, const void* t_c, const void* data,
                   int data_stride, const void* weights, int weights_stride, double fp, double fc, double scale,
                   void* loss, void* grad, void* workspace, size_t workspace_bytes, wfx_stream_t stream) {
  FusedArgs fa{data, data_stride != 0, weights, weights_stride != 0, fp, fc, scale, grad != nullptr};
  return adjoint_entry(true, model, precision, table, dtable, freqs, offsets, B, n, t_c, nullptr, nullptr, fa, loss,
                       grad, workspace, workspace_bytes, stream);
}

int wfx_fused_loss_partials(int model, const void* table, const void* freqs, const int64_t* offsets, int64_t B,
                            int64_t n, const void* t_c, const void* data, int data_stride, const void* weights,
                            int weights_stride, double fp, double fc, double scale, void* workspace,
                            size_t workspace_bytes, wfx_stream_t stream) {
  if (check_model(model) || table == nullptr || freqs == nullptr || data == nullptr || weights == nullptr || B <= 0 ||
      n <= 0)
    return WFX_EINVAL;
  if (!aligned16(table) || (data_stride && !aligned16(data))) return WFX_EINVAL;
  if (workspace == nullptr || workspace_bytes < wfx_workspace_bytes(WFX_OP_FUSED, model, WFX_FP32, B, n,
                                                                    offsets != nullptr))
    return WFX_EWORKSPACE;
  FusedArgs fa{data, data_stride != 0, weights, weights_stride != 0, fp, fc, scale, true};
  const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  return with_model(model, [&](auto m) {
    return adjoint_f32<decltype(m)::value>(true, static_cast<const float*>(table), nullptr,
                                           static_cast<const float*>(freqs), offsets, B, n,
                                           static_cast<const float*>(t_c), nullptr, nullptr, fa, nullptr, nullptr,
                                           workspace, s, kStagePartials);
  });
}

int wfx_fused_loss_contract(int model, const double* dtable, const int64_t* offsets, int64_t B, int64_t n, void* loss,
                            void* grad, void* workspace, size_t workspace_bytes, wfx_stream_t stream) {
  if (check_model(model) || B <= 0 || n <= 0 || (loss == nullptr && grad == nullptr) ||
      (grad != nullptr && dtable == nullptr))
    return WFX_EINVAL;
  if (workspace == nullptr || workspace_bytes < wfx_workspace_bytes(WFX_OP_FUSED, model, WFX_FP32, B, n,
                                                                    offsets != nullptr))
    return WFX_EWORKSPACE;
  const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  return with_model(model, [&](auto m) {
    return adjoint_f32<decltype(m)::value>(true, nullptr, dtable, nullptr, offsets, B, n, nullptr, nullptr, nullptr,
                                           FusedArgs{}, static_cast<float*>(loss), static_cast<float*>(grad),
                                           workspace, s, kStageContract);
  });
}

int wfx_autotune_ragged(int model, const void* table, const void* freqs, const int64_t* offsets, int64_t B, int64_t n,
                        const void* t_c, void* hp, void* hc, void* workspace, size_t workspace_bytes,
                        wfx_stream_t stream, int64_t* config) {
  if (check_model(model) || table == nullptr || freqs == nullptr || offsets == nullptr || hp == nullptr ||
      hc == nullptr || B <= 0 || n <= 0)
    return WFX_EINVAL;
  if (!aligned16(table) || !aligned16(hp) || !aligned16(hc)) return WFX_EINVAL;
  if (workspace == nullptr || workspace_bytes < wfx_workspace_bytes(WFX_OP_POLARIZATIONS, model, WFX_FP32, B, n, 1))
    return WFX_EWORKSPACE;
  const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const auto* T = static_cast<const float*>(table);
  const auto* F = static_cast<const float*>(freqs);
  const auto* TC = static_cast<const float*>(t_c);
  auto* P = static_cast<float2*>(hp);
  auto* C = static_cast<float2*>(hc);
  cudaEvent_t start = nullptr, stop = nullptr;
  if (cudaEventCreate(&start) != cudaSuccess || cudaEventCreate(&stop) != cudaSuccess) {
    if (start) cudaEventDestroy(start);
    return static_cast<int>(cudaGetLastError());
  }
  RaggedConfig best = kRaggedDefault;
  float best_ms = -1.0f;
  int rc = 0;
  for (const int64_t tile : kRaggedTileCandidates) {
    for (const int64_t bps : kRaggedBlocksCandidates) {
      const RaggedConfig c{tile, bps};
      float ms_min = -1.0f;
      for (int rep = 0; rep < 4 && rc == 0; ++rep) {  // one warm-up, then the best of three
        cudaEventRecord(start, s);
        rc = with_model(model, [&](auto m) {
          return ragged_f32<decltype(m)::value>(T, F, offsets, B, n, TC, P, C, workspace, c, s);
        });
        cudaEventRecord(stop, s);
        if (rc == 0) rc = static_cast<int>(cudaEventSynchronize(stop));
        float ms = 0.0f;
        if (rc == 0) rc = static_cast<int>(cudaEventElapsedTime(&ms, start, stop));
        if (rep > 0 && (ms_min < 0.0f || ms < ms_min)) ms_min = ms;
      }
      if (rc != 0) break;
      if (best_ms < 0.0f || ms_min < best_ms) {
        best_ms = ms_min;
        best = c;
      }
    }
    if (rc != 0) break;
  }
  cudaEventDestroy(start);
  cudaEventDestroy(stop);
  if (rc != 0) return rc;
  {
    const TuneKey key = tune_key(model, B, n);
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    g_tune[key] = best;
  }
  if (config != nullptr) {
    config[0] = best.tile_len;
    config[1] = best.blocks_per_sm;
  }
  return 0;
}

int wfx_tuning(int model, int64_t B, int64_t n, int64_t* config, int set) {
  if (check_model(model) || config == nullptr || B <= 0 || n <= 0) return WFX_EINVAL;
  const TuneKey key = tune_key(model, B, n);
  std::lock_guard<std::mutex> lock(g_tune_mutex);
  if (set) {
    const RaggedConfig c{config[0], config[1]};
    if (!valid_config(c)) return WFX_EINVAL;
    g_tune[key] = c;
    return 1;
  }
  const auto it = g_tune.find(key);
  const RaggedConfig c = it == g_tune.end() ? kRaggedDefault : it->second;
  config[0] = c.tile_len;
  config[1] = c.blocks_per_sm;
  return it == g_tune.end() ? 0 : 1;
}

static int template_overlap_entry(bool polarizations, int model, const float* table, const float* freqs, int64_t B,
                                  int64_t n, const float* t_c, double fp, double fc, const void* signal,
                                  const float* psd, double delta_f, void* series, int64_t n_fft, double* norms,
                                  wfx_stream_t stream) {
  if (check_model(model) || table == nullptr || freqs == nullptr || signal == nullptr || psd == nullptr ||
      series == nullptr || norms == nullptr || B <= 0 || n <= 0 || n_fft < n || (n_fft & 1) || !(delta_f > 0.0))
    return WFX_EINVAL;
  if (!aligned16(table) || !aligned16(series)) return WFX_EINVAL;
  const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const double scale = 4.0 * delta_f;
  const int64_t norm_blocks = min((B + kBlock - 1) / kBlock, static_cast<int64_t>(max(device_sms(), 1)));
  k_template_norms<<<static_cast<unsigned>(norm_blocks), kBlock, 0, s>>>(
      static_cast<const float2*>(signal), psd, n, B, scale, polarizations ? 4 : 2, polarizations ? 0 : 1, norms);
  if (int rc = launched()) return rc;
  return with_model(model, [&](auto m) {
    constexpr int M = decltype(m)::value;
    const int64_t tiles = (n + kFwdTile - 1) / kFwdTile;
    const int64_t groups = (B + kBinariesPerBlock - 1) / kBinariesPerBlock;
    constexpr int64_t kMaxY = 65535;
    const int64_t per_launch = fwd_group_major<M>() ? kMaxY : (int64_t(1) << 31) - 1;
    for (int64_t g0 = 0; g0 < groups; g0 += per_launch) {
      const int64_t g = min(groups - g0, per_launch);
      const unsigned t = static_cast<unsigned>(min(tiles, fwd_group_major<M>() ? (int64_t(1) << 31) - 1 : kMaxY));
      const dim3 grid = fwd_group_major<M>() ? dim3(t, static_cast<unsigned>(g)) : dim3(static_cast<unsigned>(g), t);
      if (polarizations) {
        k_template_overlap<M, true><<<grid, kBlock, 0, s>>>(
            table, freqs, n, B, g0, t_c, 0.0f, 0.0f, static_cast<const float2*>(signal), psd,
            static_cast<float>(scale), static_cast<float2*>(series), n_fft, norms);
      } else {
        k_template_overlap<M, false><<<grid, kBlock, 0, s>>>(
            table, freqs, n, B, g0, t_c, static_cast<float>(fp), static_cast<float>(fc),
            static_cast<const float2*>(signal), psd, static_cast<float>(scale), static_cast<float2*>(series), n_fft,
            norms);
      }
      if (int rc = launched()) return rc;
    }
    return 0;
  });
}

int wfx_template_overlap(int model, const float* table, const float* freqs, int64_t B, int64_t n, const float* t_c,
                         double fp, double fc, const void* signal, const float* psd, double delta_f, void* series,
                         int64_t n_fft, double* norms, wfx_stream_t stream) {
  return template_overlap_entry(false, model, table, freqs, B, n, t_c, fp, fc, signal, psd, delta_f, series, n_fft,
                                norms, stream);
}

int wfx_template_polarization_overlap(int model, const float* table, const float* freqs, int64_t B, int64_t n,
                                      const float* t_c, const void* signal, const float* psd, double delta_f,
                                      void* series, int64_t n_fft, double* norms, wfx_stream_t stream) {
  return template_overlap_entry(true, model, table, freqs, B, n, t_c, 0.0, 0.0, signal, psd, delta_f, series, n_fft,
                                norms, stream);
}

int wfx_fused_loss_noalloc(int model, int precision, const void* table, const double* dtable, const void* freqs,
                           const int64_t* offsets, int64_t B, int64_t n, const void* t_c, const void* data,
                           int data_stride, const void* weights, int weights_stride, double fp, double fc,
                           double scale, void* loss, void* grad, wfx_stream_t stream) {
  if (check_model(model) || B <= 0 || n <= 0) return WFX_EINVAL;
  void* scratch = nullptr;
  size_t bytes = 0;
  if (precision == WFX_FP32) {
    if (wfx_workspace_bytes(WFX_OP_FUSED, model, precision, B, n, offsets != nullptr) > WFX_STATIC_SCRATCH_BYTES)
      return WFX_ESCRATCH;
    if (int rc = static_scratch(&scratch)) return rc;
    bytes = WFX_STATIC_SCRATCH_BYTES;
  }
  return wfx_fused_loss(model, precision, table, dtable, freqs, offsets, B, n, t_c, data, data_stride, weights,
                        weights_stride, fp, fc, scale, loss, grad, scratch, bytes, stream);
}

}  // extern "C"
