// Functions one translation unit of the library offers another (not part of
// the C ABI).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace wfx {

// (setup.cu) wfx_setup for a set-up that runs beside other work, the batch
// pipeline's second stream: the value set-ups of IMRPhenomXAS and IMRPhenomD
// in a register-bounded form, the same results.
int setup_background(int model, const double* params, int64_t B, const double* f_min, int64_t f_min_stride,
                     double amp_scale, double reference_mf, double* table64, float* table32, int32_t* status,
                     cudaStream_t s);

// (xhm.cu) wfx_grid_vjp for IMRPhenomXHM: grad_f zeroed beforehand; the
// arguments as wfx_grid_vjp's, table a row of kXhmStride64 doubles a binary.
int xhm_grid_vjp(const double* table, const double* freqs, const int64_t* offsets, int64_t B, int64_t n,
                 const double* t_c, const void* cot_hp, const void* cot_hc, double* grad_f, cudaStream_t s);

}  // namespace wfx
