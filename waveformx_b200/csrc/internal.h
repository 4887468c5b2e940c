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

}  // namespace wfx
