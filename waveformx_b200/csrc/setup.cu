// The per-binary set-up kernels (FP64) and their C-ABI entries: the tables
// of a batch (setup_xas.cuh, setup_phenomd.cuh, setup_taylorf2.cuh), and
// with dual numbers (one
// chain per binary and parameter) dtable = d table / d params.
//  * k_setup_whole: one chain per thread, the whole set-up;
//  * k_setup_split: grid row 0 the amplitude part of each chain, row 1 the
//    phase part (they share only the fits and the QNM frequencies), each
//    writing its own slots of the table: the dual-number set-ups of
//    IMRPhenomXAS and IMRPhenomD, where it shortens the chain a block waits
//    on and spills less (measured, XAS: 72 us at 1024 binaries either way;
//    84 against 103 us at 4096, 268 against 314 at 16384, 1.01 against
//    1.28 ms at 65536; the same dtable bit for bit).
//
// This file is compiled without FMA contraction (-fmad=false): the value
// part of the dual-number set-up then rounds exactly as the plain one, so a
// waveform does not depend on whether its gradient was asked for.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "../../include/waveformx_b200.h"
#include "internal.h"
#include "setup_phenomd.cuh"
#include "setup_taylorf2.cuh"
#include "setup_xas.cuh"
#include "setup_xhm.cuh"

namespace wfx {

constexpr int kDirections = 8;      // parameters of dtable's columns
constexpr int kDualDirections = 4;  // of them traced by dual-number chains: m1, m2, chi1, chi2
constexpr int kRoleBlock = 64;           // chains per block of k_setup_split (measured: 69.8 us at 1024
                                         // XAS binaries; 72.3 with 32, 73.1 with 128, 87.4 with 256)
constexpr int kWholeBlock = 128;         // chains per block of k_setup_whole
// Blocks a SM that bound the registers of the value set-ups which run beside
// the forwards of the batch pipeline (128 registers rather than 255, a few
// spilled): a block then holds one of the forward's four block slots of an
// SM rather than two. Measured (IMRPhenomXAS, 20 batches of 4096 x 4017, two
// batches a set-up): 66.7-66.9 us a batch against 67.7-68.1; the set-up
// alone 37.4 us against 35.7 (3 blocks, 168 registers: 67.7-67.9 and 35.8).
constexpr int kBackgroundBlocks = 4;

// The parameters of chain c: binary c / directions, seeded along parameter
// c % directions for R = Dual.
template <class R>
__device__ __forceinline__ void chain_params(const double* params, int64_t c, int directions, R* p) {
  const int64_t b = c / directions;
  const int d = static_cast<int>(c % directions);
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    if constexpr (sizeof(R) == sizeof(double)) {
      p[k] = params[b * 8 + k];
    } else {
      p[k] = R(params[b * 8 + k], k == d ? 1.0 : 0.0);
    }
  }
}

template <int MODEL, int ROLE, class R, class Fits>
__device__ __forceinline__ int32_t setup_part(const R* p, double f_min, double amp_scale, double rmf, R* tab,
                                              const Fits& fits) {
  if constexpr (MODEL == kModelXas) {
    return xas::setup<R, Fits, ROLE>(p, f_min, amp_scale, rmf, tab, fits);
  } else {
    return phenomd::setup<R, Fits, ROLE>(p, f_min, amp_scale, rmf, tab, fits);
  }
}

// The amplitude part's table slots (the rest belong to the phase part).
template <int MODEL>
__device__ __forceinline__ bool amplitude_slot(int k) {
  if constexpr (MODEL == kModelXas) {
    return (k >= X_AMP_INS && k <= X_AMP_RD_G) || k == X_F_AMP_IN || k == X_F_AMP_RD;
  } else if constexpr (MODEL == kModelPhenomD) {
    return (k >= D_AMP_INS && k <= D_AMP_RD_SHIFT) || k == D_F_AMP_INS || k == D_F_AMP_MRD;
  } else {
    return k == T_AMP;
  }
}

template <int MODEL>
__device__ __forceinline__ bool owned(int role, int k) {
  const bool amp = amplitude_slot<MODEL>(k);
  return (role & kRoleAmp) ? ((role & kRolePhase) ? true : amp) : !amp;
}

// Binary b's slots of `role` from its FP64 table `tab`: FP64 as they are;
// FP32 with the phase's large parts as double-floats (tables.cuh, X32_* /
// D32_*): T0, each region's constant minus the anchor, each coefficient of
// f, the ringdown's largest term.
template <int MODEL>
__device__ __forceinline__ void write_tables(int role, const double* tab, int64_t b, double* t64, float* t32) {
  if (t64) {
#pragma unroll
    for (int k = 0; k < kTableStride; ++k) {
      if (owned<MODEL>(role, k)) t64[b * kTableStride + k] = tab[k];
    }
  }
  if (t32) {
    float out[kTableStride];
#pragma unroll
    for (int k = 0; k < kTableStride; ++k) out[k] = static_cast<float>(tab[k]);
    if (role & kRolePhase) {
      using L = Layout<MODEL>;
      out[L::kT0Lo] = static_cast<float>(tab[L::kT0] - static_cast<double>(out[L::kT0]));
#pragma unroll
      for (int r = 0; r < L::kRegions; ++r) {
        const int cs = L::const_slot(r), ls = L::lin_slot(r);
        const double c = tab[cs] - tab[L::kAnchor];
        out[cs] = static_cast<float>(c);
        out[L::kConstLo + r] = static_cast<float>(c - static_cast<double>(out[cs]));
        out[L::kLinLo + r] = static_cast<float>(tab[ls] - static_cast<double>(out[ls]));
      }
      if constexpr (L::kBigTerm >= 0) {
        out[L::kBigTermLo] = static_cast<float>(tab[L::kBigTerm] - static_cast<double>(out[L::kBigTerm]));
      }
    }
    float* row = t32 + b * kTableStride;
    if (role == kRoleAll) {
      float4* dst = reinterpret_cast<float4*>(row);
#pragma unroll
      for (int q = 0; q < kTableStride / 4; ++q)
        dst[q] = make_float4(out[4 * q], out[4 * q + 1], out[4 * q + 2], out[4 * q + 3]);
    } else {
#pragma unroll
      for (int k = 0; k < kTableStride; ++k) {
        if (owned<MODEL>(role, k)) row[k] = out[k];
      }
    }
  }
}

// The derivatives of the table along the parameters that only scale or
// shift a few slots, from the table's values (no dual-number chain): the
// distance (1 / distance in the amplitude's normalisation), the
// inclination (kp, kc), phi_ref (the phase constants) and f_ref (the phase
// constants and the anchor, through the set-up's own alignment code with a
// dual f_ref). Column j - kDualDirections of out, j = 4..7, for slot k.
template <int MODEL>
struct Tail {
  double kp, kc, constant_phi, constant_fref, anchor_fref;
};

template <int MODEL>
__device__ __forceinline__ Tail<MODEL> tail_derivatives(const double* tv, const double* p, double rmf) {
  Tail<MODEL> t{};
  Dual kp, kc;
  if constexpr (MODEL == kModelXas) {
    xas::projection(Dual(p[5], 1.0), kp, kc);
  } else if constexpr (MODEL == kModelPhenomD) {
    phenomd::projection(Dual(p[5], 1.0), kp, kc);
  } else {
    taylorf2::projection(Dual(p[5], 1.0), kp, kc);
  }
  const bool refused = isnan(tv[Layout<MODEL>::kKp]);
  t.kp = refused ? 0.0 : kp.d;
  t.kc = refused ? 0.0 : kc.d;
  t.constant_phi = (2.0 * Dual(p[6], 1.0)).d;
  // (TaylorF2: f_ref > 0 sets the reference, f_ref <= 0 none)
  if ((MODEL == kModelTaylorF2 ? p[7] > 0.0 : p[7] != 0.0) && isnan(rmf)) {
    const Dual f(p[7], 1.0);
    if constexpr (MODEL == kModelTaylorF2) {
      const Dual rest = taylorf2::rest_at<Dual, double>(tv, f);
      t.constant_fref = (Dual(0.0) - rest).d;
      t.anchor_fref = (tv[T_T0] * w_exp(-5.0 / 3.0 * w_log(f))).d;
    } else if constexpr (MODEL == kModelXas) {
      bool past;
      Dual lf;
      const Dual rest = xas::rest_at<Dual, double>(tv, f, past, lf);
      t.constant_fref = (Dual(0.0) - rest).d;
      t.anchor_fref = past ? 0.0 : (tv[X_T0] * w_exp(-5.0 / 3.0 * lf)).d;
    } else {
      bool inspiral;
      const Dual rest = phenomd::rest_at<Dual, double>(tv, f, inspiral);
      t.constant_fref = (Dual(0.0) - rest).d;
      t.anchor_fref = inspiral ? (tv[D_T0] * w_exp(-5.0 / 3.0 * w_log(f))).d : 0.0;
    }
  }
  return t;
}

template <int MODEL>
__device__ __forceinline__ bool normalisation_slot(int k) {
  if constexpr (MODEL == kModelXas) {
    return (k >= X_AMP_INS && k < X_AMP_INS + 10) || k == X_AMP_INT_N || k == X_AMP_RD_N;
  } else if constexpr (MODEL == kModelPhenomD) {
    return (k >= D_AMP_INS && k < D_AMP_INS + 10) || (k >= D_AMP_INT && k < D_AMP_INT + 5) || k == D_AMP_RD_N;
  } else {
    return k == T_AMP;
  }
}

template <int MODEL>
__device__ __forceinline__ bool constant_slot(int k) {
  if constexpr (MODEL == kModelXas) {
    return k == X_PH_INS + 4 || k == X_PH_INT || k == X_PH_RD;
  } else if constexpr (MODEL == kModelPhenomD) {
    return k == D_PH_INS || k == D_PH_INT || k == D_PH_RD;
  } else {
    return k == T_PH + 4;
  }
}

// The outputs of chain c (binary c / directions, direction c % directions)
// for the slots of `role`; the dual-number chains of direction 0 also write
// the other four directions (tail_derivatives).
template <int MODEL, class R>
__device__ __forceinline__ void write_chain(int role, const R* tab, int64_t c, int directions, const R* p,
                                            double rmf, double* t64, float* t32, double* dtable) {
  const int64_t b = c / directions;
  if constexpr (sizeof(R) == sizeof(double)) {
    write_tables<MODEL>(role, tab, b, t64, t32);
  } else {
    const int d = static_cast<int>(c % directions);
#pragma unroll
    for (int k = 0; k < kTableStride; ++k) {
      if (owned<MODEL>(role, k)) dtable[(b * kTableStride + k) * kDirections + d] = tab[k].d;
    }
    if (d == 0) {
      double v[kTableStride];
#pragma unroll
      for (int k = 0; k < kTableStride; ++k) v[k] = tab[k].v;
      write_tables<MODEL>(role, v, b, t64, t32);
      double pv[8];
#pragma unroll
      for (int k = 0; k < 8; ++k) pv[k] = p[k].v;
      const Tail<MODEL> t = tail_derivatives<MODEL>(v, pv, rmf);
      constexpr int kp_slot = Layout<MODEL>::kKp, kc_slot = Layout<MODEL>::kKc;
      constexpr int anchor_slot = Layout<MODEL>::kAnchor;
#pragma unroll 4
      for (int k = 0; k < kTableStride; ++k) {
        if (!owned<MODEL>(role, k)) continue;
        double* out = dtable + (b * kTableStride + k) * kDirections + kDualDirections;
        out[0] = normalisation_slot<MODEL>(k) && !isnan(v[k]) ? -v[k] / pv[4] : 0.0;
        out[1] = k == kp_slot ? t.kp : (k == kc_slot ? t.kc : 0.0);
        out[2] = constant_slot<MODEL>(k) ? t.constant_phi : 0.0;
        out[3] = constant_slot<MODEL>(k) ? t.constant_fref : (k == anchor_slot ? t.anchor_fref : 0.0);
      }
    }
  }
}

template <int MODEL, class R>
__global__ void __launch_bounds__(kRoleBlock) k_setup_split(const double* __restrict__ params, int64_t chains,
                                                            int directions, const double* __restrict__ f_min,
                                                            int64_t f_min_stride, double amp_scale, double rmf,
                                                            double* table64, float* table32, double* dtable,
                                                            int32_t* status) {
  const int64_t c = blockIdx.x * int64_t(kRoleBlock) + threadIdx.x;
  if (c >= chains) return;
  R p[8];
  chain_params(params, c, directions, p);
  const int64_t b = c / directions;
  R tab[kTableStride];
#pragma unroll
  for (int k = 0; k < kTableStride; ++k) tab[k] = R(0.0);
  const double fm = f_min[b * f_min_stride];
  int32_t st;
  int role;
  if constexpr (MODEL == kModelXas) {
    const xas::Vars<R> v = xas::variables<R>(p);
    const DirectFits<R, xas::Vars<R>> fits{v};
    if (blockIdx.y == 0) {
      role = kRoleAmp;
      st = setup_part<MODEL, kRoleAmp>(p, fm, amp_scale, rmf, tab, fits);
    } else {
      role = kRolePhase;
      st = setup_part<MODEL, kRolePhase>(p, fm, amp_scale, rmf, tab, fits);
    }
  } else {
    const phenomd::Vars<R> v = phenomd::variables<R>(p);
    const DirectFits<R, phenomd::Vars<R>> fits{v};
    if (blockIdx.y == 0) {
      role = kRoleAmp;
      st = setup_part<MODEL, kRoleAmp>(p, fm, amp_scale, rmf, tab, fits);
    } else {
      role = kRolePhase;
      st = setup_part<MODEL, kRolePhase>(p, fm, amp_scale, rmf, tab, fits);
    }
  }
  write_chain<MODEL, R>(role, tab, c, directions, p, rmf, table64, table32, dtable);
  if (status != nullptr && st != 0 && c % directions == 0) atomicOr(status + b, st);
}

// (MIN_BLOCKS > 1: a register bound for the set-ups that run beside the
// forwards of the batch pipeline, kBackgroundBlocks)
template <int MODEL, class R, int MIN_BLOCKS = 1>
__global__ void __launch_bounds__(kWholeBlock, MIN_BLOCKS) k_setup_whole(const double* __restrict__ params, int64_t chains,
                                                             int directions, const double* __restrict__ f_min,
                                                             int64_t f_min_stride, double amp_scale, double rmf,
                                                             double* table64, float* table32, double* dtable,
                                                             int32_t* status) {
  const int64_t c = blockIdx.x * int64_t(kWholeBlock) + threadIdx.x;
  if (c >= chains) return;
  R p[8];
  chain_params(params, c, directions, p);
  const int64_t b = c / directions;
  R tab[kTableStride];
#pragma unroll
  for (int k = 0; k < kTableStride; ++k) tab[k] = R(0.0);
  int32_t st;
  if constexpr (MODEL == kModelXas) {
    st = xas::setup<R>(p, f_min[b * f_min_stride], amp_scale, rmf, tab);
  } else if constexpr (MODEL == kModelPhenomD) {
    st = phenomd::setup<R>(p, f_min[b * f_min_stride], amp_scale, rmf, tab);
  } else {
    st = taylorf2::setup<R>(p, f_min[b * f_min_stride], amp_scale, rmf, tab);
  }
  write_chain<MODEL, R>(kRoleAll, tab, c, directions, p, rmf, table64, table32, dtable);
  if (status != nullptr && c % directions == 0) status[b] = st;
}


// IMRPhenomXHM: thread (b, part) of 5 per binary; part 0 writes the (2,2)
// table and the head of binary b, part 1 + m its higher mode m. Each
// computes the (2,2) set-up its part reads (setup_xhm.cuh). The status
// (zeroed beforehand) gathers the parts' bits.
constexpr int kXhmSetupBlock = 64;
constexpr int kXhmParts = 5;

__global__ void __launch_bounds__(kXhmSetupBlock)
    k_setup_xhm(const double* __restrict__ params, int64_t B, const double* __restrict__ f_min, int64_t f_min_stride,
                double amp_scale, double rmf, double* __restrict__ table64, float* __restrict__ table32,
                int32_t* __restrict__ status) {
  const int64_t c = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (c >= B * kXhmParts) return;
  const int64_t b = c / kXhmParts;
  const int part = static_cast<int>(c % kXhmParts);
  double p[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) p[k] = params[b * 8 + k];
  // (zeroed: the slots the FP64 (2,2) table leaves unused are written too)
  double tab[kTableStride];
#pragma unroll
  for (int k = 0; k < kTableStride; ++k) tab[k] = 0.0;
  xas::Internals<double> in;
  const xas::Vars<double> v = xas::variables<double>(p);
  const int32_t st = xas::setup(p, f_min[b * f_min_stride], amp_scale, rmf, tab,
                                DirectFits<double, xas::Vars<double>>{v}, &in);
  double* row64 = table64 != nullptr ? table64 + b * kXhmStride64 : nullptr;
  float* row32 = table32 != nullptr ? table32 + b * kXhmStride32 : nullptr;
  if (part == 0) {
    write_tables<kModelXas>(kRoleAll, tab, 0, row64, row32);
    double head[H_MODES - H_FACTORS];
    xhm::mode_factors(p[5], head);
    for (int k = 0; k < xhm::kHeadFactors; ++k) head[k] = st != 0 ? NAN : head[k];
    head[H_AMP0 - H_FACTORS] = in.amp0;
    head[H_S - H_FACTORS] = in.m_sec;
    head[H_COS_A - H_FACTORS] = cos(tab[X_ANCHOR]);
    head[H_SIN_A - H_FACTORS] = sin(tab[X_ANCHOR]);
    for (int k = 0; k < H_MODES - H_FACTORS; ++k) {
      if (row64 != nullptr) row64[H_FACTORS + k] = head[k];
      if (row32 != nullptr) row32[H_FACTORS + k] = static_cast<float>(head[k]);
    }
    if (status != nullptr && st != 0) atomicOr(&status[b], st);
    return;
  }
  const int m = part - 1;
  double out[xhm::kModeSize];
  const bool ok = xhm::mode_table(in, tab, m, out);
  if (status != nullptr && !ok) atomicOr(&status[b], static_cast<int32_t>(kStatusSolve));
  if (row64 != nullptr) {
    double* mrow = row64 + H_MODES + m * kXhmModeStride64;
    for (int k = 0; k < xhm::kModeSize; ++k) mrow[k] = out[k];
  }
  if (row32 != nullptr) {
    // FP32: the leading term (m/2)^(8/3) T0 and each region's coefficient of
    // f as double-floats, each region's constant less (m/2) A modulo 2 pi
    // (models/xhm/core.py:544-546)
    float* mrow = row32 + H_MODES + m * kXhmModeStride32;
    for (int k = 0; k < xhm::kModeSize; ++k) mrow[k] = static_cast<float>(out[k]);
    const double m_over_2 = (m == 0 ? 1 : (m == 1 ? 3 : (m == 2 ? 2 : 4))) * 0.5;
    const double t0 = pow(m_over_2, 8.0 / 3.0) * tab[X_T0];
    mrow[HM32_T0_HI] = static_cast<float>(t0);
    mrow[HM32_T0_LO] = static_cast<float>(t0 - static_cast<double>(mrow[HM32_T0_HI]));
    const double two_pi = 6.283185307179586;
    for (int r = 0; r < 3; ++r) {
      const int cs = xhm::M_PHASE + r * xhm::kBasis + xhm::B_1, ls = xhm::M_PHASE + r * xhm::kBasis + xhm::B_F;
      double cr = out[cs] - m_over_2 * tab[X_ANCHOR];
      cr = cr - two_pi * rint(cr / two_pi);
      mrow[cs] = static_cast<float>(cr);
      mrow[HM32_LIN_LO + r] = static_cast<float>(out[ls] - static_cast<double>(mrow[ls]));
    }
    for (int k = HM32_LIN_LO + 3; k < kXhmModeStride32; ++k) mrow[k] = 0.0f;
  }
}


// IMRPhenomXHM's d table / d params: thread (b, part, j) runs its part's
// set-up (as k_setup_xhm) on dual numbers seeded along parameter j and
// writes the tangents of the FP64 row's slots its part owns to
// dtable[(b * kXhmStride64 + k) * 8 + j]. f_ref = 0 stands for the first
// frequency (or reference_mf / M): its column is zero there. Where the (2,2)
// set-up failed the head's factors and their tangents are NaN.
constexpr int kXhmJvpBlock = 64;

__global__ void __launch_bounds__(kXhmJvpBlock)
    k_setup_xhm_jvp(const double* __restrict__ params, int64_t B, const double* __restrict__ f_min,
                    int64_t f_min_stride, double amp_scale, double rmf, double* __restrict__ dtable) {
  const int64_t c = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (c >= B * kXhmParts * kDirections) return;
  const int j = static_cast<int>(c % kDirections);
  const int64_t bp = c / kDirections;
  const int64_t b = bp / kXhmParts;
  const int part = static_cast<int>(bp % kXhmParts);
  Dual p[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) p[k] = Dual(params[b * 8 + k], 0.0);
  p[j].d = j == 7 && p[7].v == 0.0 ? 0.0 : 1.0;
  Dual tab[kTableStride];
  xas::Internals<Dual> in;
  const xas::Vars<Dual> v = xas::variables<Dual>(p);
  const int32_t st = xas::setup(p, f_min[b * f_min_stride], amp_scale, rmf, tab,
                                DirectFits<Dual, xas::Vars<Dual>>{v}, &in);
  double* drow = dtable + b * kXhmStride64 * kDirections + j;
  if (part == 0) {
    for (int k = 0; k < kTableStride; ++k) drow[k * kDirections] = tab[k].d;
    Dual head[H_MODES - H_FACTORS];
    xhm::mode_factors(p[5], head);
    for (int k = 0; k < xhm::kHeadFactors; ++k) head[k].d = st != 0 ? NAN : head[k].d;
    head[H_AMP0 - H_FACTORS] = in.amp0;
    head[H_S - H_FACTORS] = in.m_sec;
    head[H_COS_A - H_FACTORS] = w_cos(tab[X_ANCHOR]);
    head[H_SIN_A - H_FACTORS] = w_sin(tab[X_ANCHOR]);
    for (int k = 0; k < H_MODES - H_FACTORS; ++k) drow[(H_FACTORS + k) * kDirections] = head[k].d;
    return;
  }
  const int m = part - 1;
  Dual out[xhm::kModeSize];
  xhm::mode_table(in, tab, m, out);
  double* mrow = drow + (H_MODES + m * kXhmModeStride64) * kDirections;
  for (int k = 0; k < xhm::kModeSize; ++k) mrow[k * kDirections] = out[k].d;
}


// The phase of a binary's (2,2) mode at M f = mf (but for its constant) from
// its FP64 table: the table's rest plus, in the inspiral, T0 f^-5/3; for the
// converters between LAL's reference convention and the mass-scaled one
// (src/waveformx/_reference.py:59-80, models/taylorf2/reference.py:46-104,
// the phases of models/{xas,phenomd,taylorf2}/reference.py). mf = 0: 0 (no
// reference phase); mf < 0 or NaN: NaN.
template <int MODEL>
__device__ double table_phase(const double* tab, double m_sec, double mf) {
  if (mf == 0.0) return 0.0;
  if (!(mf > 0.0)) return NAN;
  const double f = mf / m_sec;
  if constexpr (MODEL == kModelXas) {
    bool past;
    double lf;
    const double r = xas::rest_at<double, double>(tab, f, past, lf);
    return past ? r : r + tab[X_T0] * exp(-5.0 / 3.0 * lf);
  } else if constexpr (MODEL == kModelPhenomD) {
    bool inspiral;
    const double r = phenomd::rest_at<double, double>(tab, f, inspiral);
    return inspiral ? r + tab[D_T0] * exp(-5.0 / 3.0 * log(f)) : r;
  } else {
    // (the table of phi_ref = 0 and f_ref = 0, the reference at coalescence:
    // its phase is Phi + pi / 4, models/taylorf2/core.py:142-151)
    return taylorf2::rest_at<double, double>(tab, f) + tab[T_T0] * exp(-5.0 / 3.0 * log(f)) - fit::PI / 4.0;
  }
}

template <int MODEL>
__global__ void __launch_bounds__(kWholeBlock)
    k_phase_difference(const double* __restrict__ params, int64_t B, const double* __restrict__ mf_from,
                       const double* __restrict__ mf_to, double* __restrict__ dphi) {
  const int64_t b = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  if (b >= B) return;
  double p[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) p[k] = params[b * 8 + k];
  // (the phase's constant cancels in a difference, but an mf of 0 stands
  // for no reference phase, which TaylorF2's phase at coalescence, f_ref =
  // 0 and phi_ref = 0, gives absolutely)
  p[4] = 1.0;
  p[6] = 0.0;
  p[7] = MODEL == kModelTaylorF2 ? 0.0 : 20.0;
  double tab[kTableStride];
  if constexpr (MODEL == kModelXas) {
    xas::setup<double>(p, 20.0, 1.0, NAN, tab);
  } else if constexpr (MODEL == kModelPhenomD) {
    phenomd::setup<double>(p, 20.0, 1.0, NAN, tab);
  } else {
    taylorf2::setup<double>(p, 20.0, 1.0, NAN, tab);
  }
  const double m_sec = (p[0] + p[1]) * fit::MTSUN_SI;
  dphi[b] = table_phase<MODEL>(tab, m_sec, mf_to[b]) - table_phase<MODEL>(tab, m_sec, mf_from[b]);
}


namespace {

int launched() {
  const cudaError_t err = cudaGetLastError();
  return err == cudaSuccess ? 0 : static_cast<int>(err);
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

int check_model(int model) {
  return (model == kModelXas || model == kModelPhenomD || model == kModelTaylorF2) ? 0 : WFX_EINVAL;
}

// The set-up of B binaries along `directions` (1: values, R = double;
// kDirections: dual numbers).
template <int MODEL, class R>
int launch_setup(const double* params, int64_t B, int directions, const double* f_min, int64_t f_min_stride,
                 double amp_scale, double rmf, double* table64, float* table32, double* dtable, int32_t* status,
                 cudaStream_t s, bool background = false) {
  const int64_t chains = B * directions;
  // (the dual-number set-ups of XAS and PhenomD always split; TaylorF2's
  // set-up is short: one chain per binary and direction)
  if constexpr (MODEL != kModelTaylorF2 && sizeof(R) != sizeof(double)) {
    if (status != nullptr) {
      const cudaError_t rc = cudaMemsetAsync(status, 0, sizeof(int32_t) * B, s);
      if (rc != cudaSuccess) return static_cast<int>(rc);
    }
    const unsigned grid = static_cast<unsigned>((chains + kRoleBlock - 1) / kRoleBlock);
    k_setup_split<MODEL, R><<<dim3(grid, 2), kRoleBlock, 0, s>>>(params, chains, directions, f_min, f_min_stride,
                                                                 amp_scale, rmf, table64, table32, dtable, status);
    return launched();
  } else {
    const unsigned grid = static_cast<unsigned>((chains + kWholeBlock - 1) / kWholeBlock);
    if constexpr (MODEL != kModelTaylorF2 && sizeof(R) == sizeof(double)) {
      if (background) {
        k_setup_whole<MODEL, R, kBackgroundBlocks><<<grid, kWholeBlock, 0, s>>>(
            params, chains, directions, f_min, f_min_stride, amp_scale, rmf, table64, table32, dtable, status);
        return launched();
      }
    }
    k_setup_whole<MODEL, R><<<grid, kWholeBlock, 0, s>>>(params, chains, directions, f_min, f_min_stride, amp_scale,
                                                         rmf, table64, table32, dtable, status);
    return launched();
  }
}

}  // namespace

// (internal.h; the register bound: kBackgroundBlocks)
int setup_background(int model, const double* params, int64_t B, const double* f_min, int64_t f_min_stride,
                     double amp_scale, double reference_mf, double* table64, float* table32, int32_t* status,
                     cudaStream_t s) {
  if (check_model(model) || params == nullptr || f_min == nullptr || B <= 0 || f_min_stride < 0) return WFX_EINVAL;
  if (table64 == nullptr && table32 == nullptr && status == nullptr) return WFX_EINVAL;
  if (table32 != nullptr && !aligned16(table32)) return WFX_EINVAL;
  if (model == kModelXas) {
    return launch_setup<kModelXas, double>(params, B, 1, f_min, f_min_stride, amp_scale, reference_mf, table64,
                                           table32, nullptr, status, s, true);
  }
  if (model == kModelPhenomD) {
    return launch_setup<kModelPhenomD, double>(params, B, 1, f_min, f_min_stride, amp_scale, reference_mf, table64,
                                               table32, nullptr, status, s, true);
  }
  return launch_setup<kModelTaylorF2, double>(params, B, 1, f_min, f_min_stride, amp_scale, reference_mf, table64,
                                              table32, nullptr, status, s);
}

}  // namespace wfx

using namespace wfx;

extern "C" {

int wfx_setup(int model, const double* params, int64_t B, const double* f_min, int64_t f_min_stride,
              double amp_scale, double reference_mf, double* table64, float* table32, int32_t* status,
              wfx_stream_t stream) {
  if (check_model(model) || params == nullptr || f_min == nullptr || B <= 0 || f_min_stride < 0) return WFX_EINVAL;
  if (table64 == nullptr && table32 == nullptr && status == nullptr) return WFX_EINVAL;
  if (table32 != nullptr && !aligned16(table32)) return WFX_EINVAL;
  const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (model == kModelXas) {
    return launch_setup<kModelXas, double>(params, B, 1, f_min, f_min_stride, amp_scale, reference_mf, table64,
                                           table32, nullptr, status, s);
  }
  if (model == kModelTaylorF2) {
    return launch_setup<kModelTaylorF2, double>(params, B, 1, f_min, f_min_stride, amp_scale, reference_mf, table64,
                                                table32, nullptr, status, s);
  }
  return launch_setup<kModelPhenomD, double>(params, B, 1, f_min, f_min_stride, amp_scale, reference_mf, table64,
                                             table32, nullptr, status, s);
}

int wfx_setup_jvp(int model, const double* params, int64_t B, const double* f_min, int64_t f_min_stride,
                  double amp_scale, double reference_mf, double* table64, float* table32, double* dtable,
                  int32_t* status, wfx_stream_t stream) {
  if (check_model(model) || params == nullptr || f_min == nullptr || dtable == nullptr || B <= 0 || f_min_stride < 0)
    return WFX_EINVAL;
  if (table32 != nullptr && !aligned16(table32)) return WFX_EINVAL;
  const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (model == kModelXas) {
    return launch_setup<kModelXas, Dual>(params, B, kDualDirections, f_min, f_min_stride, amp_scale, reference_mf,
                                         table64, table32, dtable, status, s);
  }
  if (model == kModelTaylorF2) {
    return launch_setup<kModelTaylorF2, Dual>(params, B, kDualDirections, f_min, f_min_stride, amp_scale,
                                              reference_mf, table64, table32, dtable, status, s);
  }
  return launch_setup<kModelPhenomD, Dual>(params, B, kDualDirections, f_min, f_min_stride, amp_scale,
                                           reference_mf, table64, table32, dtable, status, s);
}

int wfx_xhm_setup(const double* params, int64_t B, const double* f_min, int64_t f_min_stride, double amp_scale,
                  double reference_mf, double* table64, float* table32, int32_t* status, wfx_stream_t stream) {
  if (params == nullptr || f_min == nullptr || B <= 0 || f_min_stride < 0) return WFX_EINVAL;
  if (table64 == nullptr && table32 == nullptr && status == nullptr) return WFX_EINVAL;
  if (table32 != nullptr && !aligned16(table32)) return WFX_EINVAL;
  const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  if (status != nullptr) {
    const cudaError_t rc = cudaMemsetAsync(status, 0, sizeof(int32_t) * B, s);
    if (rc != cudaSuccess) return static_cast<int>(rc);
  }
  const int64_t threads = B * kXhmParts;
  const unsigned grid = static_cast<unsigned>((threads + kXhmSetupBlock - 1) / kXhmSetupBlock);
  k_setup_xhm<<<grid, kXhmSetupBlock, 0, s>>>(params, B, f_min, f_min_stride, amp_scale, reference_mf, table64,
                                              table32, status);
  return launched();
}

int wfx_xhm_setup_jvp(const double* params, int64_t B, const double* f_min, int64_t f_min_stride, double amp_scale,
                      double reference_mf, double* table64, float* table32, double* dtable, int32_t* status,
                      wfx_stream_t stream) {
  if (params == nullptr || f_min == nullptr || dtable == nullptr || B <= 0 || f_min_stride < 0) return WFX_EINVAL;
  if (table32 != nullptr && !aligned16(table32)) return WFX_EINVAL;
  if (table64 != nullptr || table32 != nullptr || status != nullptr) {
    const int rc = wfx_xhm_setup(params, B, f_min, f_min_stride, amp_scale, reference_mf, table64, table32, status,
                                 stream);
    if (rc != 0) return rc;
  }
  const int64_t threads = B * kXhmParts * kDirections;
  const unsigned grid = static_cast<unsigned>((threads + kXhmJvpBlock - 1) / kXhmJvpBlock);
  k_setup_xhm_jvp<<<grid, kXhmJvpBlock, 0, reinterpret_cast<cudaStream_t>(stream)>>>(
      params, B, f_min, f_min_stride, amp_scale, reference_mf, dtable);
  return launched();
}

int wfx_phase_difference(int model, const double* params, int64_t B, const double* mf_from, const double* mf_to,
                         double* dphi, wfx_stream_t stream) {
  if (params == nullptr || mf_from == nullptr || mf_to == nullptr || dphi == nullptr || B <= 0) return WFX_EINVAL;
  const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const unsigned grid = static_cast<unsigned>((B + kWholeBlock - 1) / kWholeBlock);
  if (model == kModelXas || model == kModelXhm) {
    k_phase_difference<kModelXas><<<grid, kWholeBlock, 0, s>>>(params, B, mf_from, mf_to, dphi);
  } else if (model == kModelPhenomD) {
    k_phase_difference<kModelPhenomD><<<grid, kWholeBlock, 0, s>>>(params, B, mf_from, mf_to, dphi);
  } else if (model == kModelTaylorF2) {
    k_phase_difference<kModelTaylorF2><<<grid, kWholeBlock, 0, s>>>(params, B, mf_from, mf_to, dphi);
  } else {
    return WFX_EINVAL;
  }
  return launched();
}

}  // extern "C"
