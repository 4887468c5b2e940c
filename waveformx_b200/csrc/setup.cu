// The per-binary set-up kernels (FP64) and their C-ABI entries: the tables
// of a batch (setup_xas.cuh, setup_phenomd.cuh, setup_taylorf2.cuh), and
// with dual numbers (one
// chain per binary and parameter) dtable = d table / d params.
//  * k_setup_whole: one chain per thread, the whole set-up;
//  * k_setup_split: grid row 0 the amplitude part of each chain, row 1 the
//    phase part (they share only the fits and the QNM frequencies), each
//    writing its own slots of the table: the dual-number set-up of up to
//    kSplitMaxBinaries binaries, where it shortens the chain a block waits
//    on.
//
// This file is compiled without FMA contraction (-fmad=false): the value
// part of the dual-number set-up then rounds exactly as the plain one, so a
// waveform does not depend on whether its gradient was asked for.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "../../include/waveformx_b200.h"
#include "setup_phenomd.cuh"
#include "setup_taylorf2.cuh"
#include "setup_xas.cuh"

namespace wfx {

constexpr int kDirections = 8;      // parameters of dtable's columns
constexpr int kDualDirections = 4;  // of them traced by dual-number chains: m1, m2, chi1, chi2
constexpr int kRoleBlock = 128;          // chains per block of k_setup_split
constexpr int kWholeBlock = 32;          // chains per block of k_setup_whole
constexpr int64_t kSplitMaxBinaries = 2048;  // dual-number set-ups split up to this batch

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

template <int MODEL, class R>
__global__ void __launch_bounds__(kWholeBlock) k_setup_whole(const double* __restrict__ params, int64_t chains,
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
                 cudaStream_t s) {
  const int64_t chains = B * directions;
  // (TaylorF2's set-up is short: one chain per binary and direction)
  if constexpr (MODEL != kModelTaylorF2) {
    if (directions > 1 && B <= kSplitMaxBinaries) {
      if (status != nullptr) {
        const cudaError_t rc = cudaMemsetAsync(status, 0, sizeof(int32_t) * B, s);
        if (rc != cudaSuccess) return static_cast<int>(rc);
      }
      const unsigned grid = static_cast<unsigned>((chains + kRoleBlock - 1) / kRoleBlock);
      k_setup_split<MODEL, R><<<dim3(grid, 2), kRoleBlock, 0, s>>>(params, chains, directions, f_min, f_min_stride,
                                                                   amp_scale, rmf, table64, table32, dtable, status);
      return launched();
    }
  }
  const unsigned grid = static_cast<unsigned>((chains + kWholeBlock - 1) / kWholeBlock);
  k_setup_whole<MODEL, R><<<grid, kWholeBlock, 0, s>>>(params, chains, directions, f_min, f_min_stride, amp_scale,
                                                       rmf, table64, table32, dtable, status);
  return launched();
}

}  // namespace

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

}  // extern "C"
