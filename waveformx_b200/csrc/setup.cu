// The per-binary set-up kernels (FP64) and their C-ABI entries:
//  * k_setup: the tables of a batch, one thread per binary (setup_xas.cuh,
//    setup_phenomd.cuh);
//  * k_setup_jvp: the same with dual numbers, one thread per binary and
//    parameter, for dtable = d table / d params.
//
// This file is compiled without FMA contraction (-fmad=false): the value
// part of the dual-number set-up then rounds exactly as the plain one, so a
// waveform does not depend on whether its gradient was asked for.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>

#include "../../include/waveformx_b200.h"
#include "setup_phenomd.cuh"
#include "setup_xas.cuh"

namespace wfx {

constexpr int kDirections = 8;
constexpr int kSetupBlock = 32;  // threads per block of the set-up kernels

template <int MODEL, class R>
__device__ __forceinline__ int32_t setup_one(const R* p, double f_min, double amp_scale, double rmf, R* tab) {
  if constexpr (MODEL == kModelXas) {
    return xas::setup<R>(p, f_min, amp_scale, rmf, tab);
  } else {
    return phenomd::setup<R>(p, f_min, amp_scale, rmf, tab);
  }
}

template <int MODEL>
__device__ __forceinline__ void write_tables(const double* tab, int64_t b, double* t64, float* t32) {
  if (t64) {
    for (int k = 0; k < kTableStride; ++k) t64[b * kTableStride + k] = tab[k];
  }
  if (t32) {
    // the phase's large parts as double-floats (tables.cuh, X32_* / D32_*):
    // T0, each region's constant minus the anchor, each coefficient of f
    float out[kTableStride];
    for (int k = 0; k < kTableStride; ++k) out[k] = static_cast<float>(tab[k]);
    const bool xas = MODEL == kModelXas;
    const int t0 = xas ? X_T0 : D_T0, anchor = xas ? X_ANCHOR : D_ANCHOR;
    const int t0_lo = xas ? X32_T0_LO : D32_T0_LO;
    const int const_lo = xas ? X32_CONST_LO : D32_CONST_LO, lin_lo = xas ? X32_LIN_LO : D32_LIN_LO;
    out[t0_lo] = static_cast<float>(tab[t0] - static_cast<double>(out[t0]));
    for (int r = 0; r < 3; ++r) {
      const int cs = xas ? xas_const_slot(r) : phd_const_slot(r);
      const int ls = xas ? xas_lin_slot(r) : phd_lin_slot(r);
      const double c = tab[cs] - tab[anchor];
      out[cs] = static_cast<float>(c);
      out[const_lo + r] = static_cast<float>(c - static_cast<double>(out[cs]));
      out[lin_lo + r] = static_cast<float>(tab[ls] - static_cast<double>(out[ls]));
    }
    const int rd = xas ? X_PH_RD + 2 : D_PH_RD + 3;
    out[xas ? X32_RD_TERM_LO : D32_RD_TERM_LO] = static_cast<float>(tab[rd] - static_cast<double>(out[rd]));
    float4* dst = reinterpret_cast<float4*>(t32 + b * kTableStride);
    for (int q = 0; q < kTableStride / 4; ++q) dst[q] = make_float4(out[4 * q], out[4 * q + 1], out[4 * q + 2], out[4 * q + 3]);
  }
}

template <int MODEL>
__global__ void k_setup(const double* __restrict__ params, int64_t B, const double* __restrict__ f_min,
                        int64_t f_min_stride, double amp_scale, double rmf, double* table64, float* table32,
                        int32_t* status) {
  const int64_t b = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  if (b >= B) return;
  double p[8];
  for (int k = 0; k < 8; ++k) p[k] = params[b * 8 + k];
  double tab[kTableStride];
  for (int k = 0; k < kTableStride; ++k) tab[k] = 0.0;
  const int32_t st = setup_one<MODEL, double>(p, f_min[b * f_min_stride], amp_scale, rmf, tab);
  write_tables<MODEL>(tab, b, table64, table32);
  if (status) status[b] = st;
}

template <int MODEL>
__global__ void k_setup_jvp(const double* __restrict__ params, int64_t B, const double* __restrict__ f_min,
                            int64_t f_min_stride, double amp_scale, double rmf, double* table64, float* table32,
                            double* dtable, int32_t* status) {
  const int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
  if (i >= B * kDirections) return;
  const int64_t b = i / kDirections;
  const int d = static_cast<int>(i % kDirections);
  Dual p[8];
  for (int k = 0; k < 8; ++k) p[k] = Dual(params[b * 8 + k], k == d ? 1.0 : 0.0);
  Dual tab[kTableStride];
  for (int k = 0; k < kTableStride; ++k) tab[k] = Dual(0.0);
  const int32_t st = setup_one<MODEL, Dual>(p, f_min[b * f_min_stride], amp_scale, rmf, tab);
  for (int k = 0; k < kTableStride; ++k) dtable[(b * kTableStride + k) * kDirections + d] = tab[k].d;
  if (d == 0) {
    double v[kTableStride];
    for (int k = 0; k < kTableStride; ++k) v[k] = tab[k].v;
    write_tables<MODEL>(v, b, table64, table32);
    if (status) status[b] = st;
  }
}


namespace {

int launched() {
  const cudaError_t err = cudaGetLastError();
  return err == cudaSuccess ? 0 : static_cast<int>(err);
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

int check_model(int model) { return (model == kModelXas || model == kModelPhenomD) ? 0 : WFX_EINVAL; }

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
  // (one warp per block: each thread's set-up is a long serial chain, so
  // the binaries are spread over as many SMs as there are warps)
  const unsigned grid = static_cast<unsigned>((B + kSetupBlock - 1) / kSetupBlock);
  if (model == kModelXas) {
    k_setup<kModelXas><<<grid, kSetupBlock, 0, s>>>(params, B, f_min, f_min_stride, amp_scale, reference_mf, table64,
                                                    table32, status);
  } else {
    k_setup<kModelPhenomD><<<grid, kSetupBlock, 0, s>>>(params, B, f_min, f_min_stride, amp_scale, reference_mf,
                                                        table64, table32, status);
  }
  return launched();
}

int wfx_setup_jvp(int model, const double* params, int64_t B, const double* f_min, int64_t f_min_stride,
                  double amp_scale, double reference_mf, double* table64, float* table32, double* dtable,
                  int32_t* status, wfx_stream_t stream) {
  if (check_model(model) || params == nullptr || f_min == nullptr || dtable == nullptr || B <= 0 || f_min_stride < 0)
    return WFX_EINVAL;
  if (table32 != nullptr && !aligned16(table32)) return WFX_EINVAL;
  const cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
  const unsigned grid = static_cast<unsigned>((B * kDirections + kSetupBlock - 1) / kSetupBlock);
  if (model == kModelXas) {
    k_setup_jvp<kModelXas><<<grid, kSetupBlock, 0, s>>>(params, B, f_min, f_min_stride, amp_scale, reference_mf,
                                                        table64, table32, dtable, status);
  } else {
    k_setup_jvp<kModelPhenomD><<<grid, kSetupBlock, 0, s>>>(params, B, f_min, f_min_stride, amp_scale, reference_mf,
                                                            table64, table32, dtable, status);
  }
  return launched();
}

}  // extern "C"
