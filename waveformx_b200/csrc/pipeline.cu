// The batch pipeline's launches, one C call each (waveformx_b200/pipeline.py
// drives it): per pipeline two more streams at the highest priority (the
// set-ups; the dual-number set-ups of the likelihood) and their events.
// wfx_pipeline_setup queues a batch's set-up on the second stream after
// everything queued so far on the caller's stream, then marks the batch's
// slot ready; wfx_pipeline_forward makes the caller's stream wait
// for that slot and queues the batch's forward. The set-up of batch k + 1
// then runs beside the forward of batch k. For the likelihood,
// wfx_pipeline_setup_jvp queues a batch's dual-number set-up on the third
// stream, and wfx_pipeline_fused runs the batch's fused likelihood once its
// table is ready and contracts it with dtable once that is. A pipeline
// serves one sequence of batches at a time (its events are reused).
#include <cuda_runtime.h>

#include <cstdint>
#include <new>

#include "../../include/waveformx_b200.h"
#include "internal.h"

struct wfx_pipeline {
  cudaStream_t side = nullptr;
  cudaStream_t side_jvp = nullptr;  // the dual-number set-ups of the likelihood's batches
  cudaEvent_t fork = nullptr;
  cudaEvent_t ready[2] = {nullptr, nullptr};
  cudaEvent_t ready_jvp[2] = {nullptr, nullptr};
  cudaEvent_t join = nullptr;
  // the likelihood's batches: the reverse pass of a workspace half done, the
  // contraction that read it done, and a mark of the contractions' stream
  cudaEvent_t partials_done[2] = {nullptr, nullptr};
  cudaEvent_t contracts_done[2] = {nullptr, nullptr};
  cudaEvent_t side_mark = nullptr;
};

extern "C" {

int wfx_pipeline_destroy(wfx_pipeline_t p) {
  if (p == nullptr) return 0;
  // (the second stream's last set-up completes before its handles go)
  if (p->side != nullptr) cudaStreamSynchronize(p->side);
  if (p->side_jvp != nullptr) cudaStreamSynchronize(p->side_jvp);
  if (p->fork != nullptr) cudaEventDestroy(p->fork);
  for (int i = 0; i < 2; ++i) {
    if (p->ready[i] != nullptr) cudaEventDestroy(p->ready[i]);
    if (p->ready_jvp[i] != nullptr) cudaEventDestroy(p->ready_jvp[i]);
  }
  if (p->join != nullptr) cudaEventDestroy(p->join);
  for (int i = 0; i < 2; ++i) {
    if (p->partials_done[i] != nullptr) cudaEventDestroy(p->partials_done[i]);
    if (p->contracts_done[i] != nullptr) cudaEventDestroy(p->contracts_done[i]);
  }
  if (p->side_mark != nullptr) cudaEventDestroy(p->side_mark);
  if (p->side != nullptr) cudaStreamDestroy(p->side);
  if (p->side_jvp != nullptr) cudaStreamDestroy(p->side_jvp);
  delete p;
  return 0;
}

int wfx_pipeline_create(wfx_pipeline_t* out) {
  if (out == nullptr) return WFX_EINVAL;
  *out = nullptr;
  int least = 0, greatest = 0;
  cudaError_t rc = cudaDeviceGetStreamPriorityRange(&least, &greatest);
  if (rc != cudaSuccess) return static_cast<int>(rc);
  wfx_pipeline* p = new (std::nothrow) wfx_pipeline();
  if (p == nullptr) return static_cast<int>(cudaErrorMemoryAllocation);
  rc = cudaStreamCreateWithPriority(&p->side, cudaStreamNonBlocking, greatest);
  if (rc == cudaSuccess) rc = cudaStreamCreateWithPriority(&p->side_jvp, cudaStreamNonBlocking, greatest);
  if (rc == cudaSuccess) rc = cudaEventCreateWithFlags(&p->fork, cudaEventDisableTiming);
  for (int i = 0; i < 2 && rc == cudaSuccess; ++i) {
    rc = cudaEventCreateWithFlags(&p->ready[i], cudaEventDisableTiming);
    if (rc == cudaSuccess) rc = cudaEventCreateWithFlags(&p->ready_jvp[i], cudaEventDisableTiming);
  }
  if (rc == cudaSuccess) rc = cudaEventCreateWithFlags(&p->join, cudaEventDisableTiming);
  for (int i = 0; i < 2 && rc == cudaSuccess; ++i) {
    rc = cudaEventCreateWithFlags(&p->partials_done[i], cudaEventDisableTiming);
    if (rc == cudaSuccess) rc = cudaEventCreateWithFlags(&p->contracts_done[i], cudaEventDisableTiming);
  }
  if (rc == cudaSuccess) rc = cudaEventCreateWithFlags(&p->side_mark, cudaEventDisableTiming);
  if (rc != cudaSuccess) {
    wfx_pipeline_destroy(p);
    return static_cast<int>(rc);
  }
  *out = p;
  return 0;
}

int wfx_pipeline_setup(wfx_pipeline_t p, int slot, int model, const double* params, int64_t B, const double* f_min,
                       int64_t f_min_stride, double amp_scale, double reference_mf, double* table64, float* table32,
                       int32_t* status, wfx_stream_t stream) {
  if (p == nullptr || slot < 0 || slot > 1) return WFX_EINVAL;
  const cudaStream_t caller = reinterpret_cast<cudaStream_t>(stream);
  cudaError_t rc = cudaEventRecord(p->fork, caller);
  if (rc == cudaSuccess) rc = cudaStreamWaitEvent(p->side, p->fork, 0);
  if (rc != cudaSuccess) return static_cast<int>(rc);
  const wfx_stream_t side = reinterpret_cast<wfx_stream_t>(p->side);
  const int r = model == WFX_XHM
                    ? wfx_xhm_setup(params, B, f_min, f_min_stride, amp_scale, reference_mf, table64, table32, status,
                                    side)
                    : wfx::setup_background(model, params, B, f_min, f_min_stride, amp_scale, reference_mf, table64,
                                            table32, status, p->side);
  if (r != 0) return r;
  rc = cudaEventRecord(p->ready[slot], p->side);
  return rc == cudaSuccess ? 0 : static_cast<int>(rc);
}

int wfx_pipeline_forward(wfx_pipeline_t p, int slot, int model, int precision, const void* table, const void* freqs,
                         const int64_t* offsets, int64_t B, int64_t n, int64_t max_len, const void* t_c, void* hp,
                         void* hc, void* workspace, size_t workspace_bytes, wfx_stream_t stream) {
  if (p == nullptr || slot < 0 || slot > 1) return WFX_EINVAL;
  const cudaStream_t caller = reinterpret_cast<cudaStream_t>(stream);
  const cudaError_t rc = cudaStreamWaitEvent(caller, p->ready[slot], 0);
  if (rc != cudaSuccess) return static_cast<int>(rc);
  if (model == WFX_XHM) {
    return wfx_xhm_polarizations(precision, table, freqs, offsets, B, n, max_len, t_c, hp, hc, nullptr, stream);
  }
  return wfx_polarizations(model, precision, table, freqs, offsets, B, n, t_c, hp, hc, workspace, workspace_bytes,
                           stream);
}

int wfx_pipeline_setup_jvp(wfx_pipeline_t p, int slot, int model, const double* params, int64_t B,
                           const double* f_min, int64_t f_min_stride, double amp_scale, double reference_mf,
                           double* dtable, wfx_stream_t stream) {
  if (p == nullptr || slot < 0 || slot > 1 || model == WFX_XHM) return WFX_EINVAL;
  const cudaStream_t caller = reinterpret_cast<cudaStream_t>(stream);
  cudaError_t rc = cudaEventRecord(p->fork, caller);
  if (rc == cudaSuccess) rc = cudaStreamWaitEvent(p->side_jvp, p->fork, 0);
  if (rc != cudaSuccess) return static_cast<int>(rc);
  const int r = wfx_setup_jvp(model, params, B, f_min, f_min_stride, amp_scale, reference_mf, nullptr, nullptr,
                              dtable, nullptr, reinterpret_cast<wfx_stream_t>(p->side_jvp));
  if (r != 0) return r;
  rc = cudaEventRecord(p->ready_jvp[slot], p->side_jvp);
  return rc == cudaSuccess ? 0 : static_cast<int>(rc);
}

int wfx_pipeline_fused(wfx_pipeline_t p, int slot, int model, const void* table, const void* freqs,
                       const int64_t* offsets, int64_t B, int64_t n, const void* t_c, const void* data,
                       int data_stride, const void* weights, int weights_stride, double fp, double fc, double scale,
                       const double* dtable, void* loss, void* grad, void* workspace, size_t workspace_bytes,
                       wfx_stream_t stream) {
  if (p == nullptr || slot < 0 || slot > 1) return WFX_EINVAL;
  const cudaStream_t caller = reinterpret_cast<cudaStream_t>(stream);
  cudaError_t rc = cudaStreamWaitEvent(caller, p->ready[slot], 0);
  if (rc != cudaSuccess) return static_cast<int>(rc);
  int r = wfx_fused_loss_partials(model, table, freqs, offsets, B, n, t_c, data, data_stride, weights, weights_stride,
                                  fp, fc, scale, workspace, workspace_bytes, stream);
  if (r != 0) return r;
  rc = cudaStreamWaitEvent(caller, p->ready_jvp[slot], 0);
  if (rc != cudaSuccess) return static_cast<int>(rc);
  return wfx_fused_loss_contract(model, dtable, offsets, B, n, loss, grad, workspace, workspace_bytes, stream);
}

int wfx_pipeline_run(wfx_pipeline_t p, int model, int precision, int64_t K, const double* params, int64_t B,
                     const double* f_min, int64_t f_min_stride, double amp_scale, double reference_mf, void* tables,
                     int32_t* status, const void* freqs, const int64_t* offsets, int64_t n, int64_t max_len,
                     const void* t_c, void* hp, void* hc, int64_t ring, int64_t group, void* workspace,
                     size_t workspace_bytes, wfx_stream_t stream) {
  if (p == nullptr || params == nullptr || tables == nullptr || status == nullptr || hp == nullptr ||
      hc == nullptr || K <= 0 || B <= 0 || n <= 0 || ring <= 0 || group <= 0 ||
      (precision != WFX_FP32 && precision != WFX_FP64) || (group > 1 && f_min_stride != 0))
    return WFX_EINVAL;
  // (a batch's table, outputs and t_c: their sizes in bytes; each ring slot
  // starts 16-byte aligned: complex64 slots of an odd count are padded by one
  // element)
  const bool f32 = precision == WFX_FP32;
  const int64_t xhm_stride = f32 ? WFX_XHM_STRIDE32 : WFX_XHM_STRIDE64;
  const int64_t stride = model == WFX_XHM ? xhm_stride : static_cast<int64_t>(WFX_TABLE_STRIDE);
  const int64_t table_bytes = B * stride * (f32 ? 4 : 8);
  const int64_t elems = offsets != nullptr ? n : B * n;
  const int64_t out_bytes = (f32 ? elems + (elems & 1) : elems) * (f32 ? 8 : 16);
  const int64_t tc_bytes = B * (f32 ? 4 : 8);
  char* const slots = static_cast<char*>(tables);
  // the set-up of batches [g G, g G + G) in one launch (its time hardly
  // depends on the number of binaries), into table slot g % 2
  const int64_t groups = (K + group - 1) / group;
  const auto setup = [&](int64_t g) {
    const int slot = static_cast<int>(g & 1);
    const int64_t k0 = g * group, count = (K - k0 < group ? K - k0 : group);
    void* table = slots + slot * group * table_bytes;
    return wfx_pipeline_setup(p, slot, model, params + k0 * B * 8, count * B, f_min, f_min_stride, amp_scale,
                              reference_mf, f32 ? nullptr : static_cast<double*>(table),
                              f32 ? static_cast<float*>(table) : nullptr, status + k0 * B, stream);
  };
  if (int rc = setup(0)) return rc;
  for (int64_t g = 0; g < groups; ++g) {
    // (group g + 1's set-up waits for what the caller's stream holds so far:
    // group g - 1's forwards, the last readers of its slot)
    if (g + 1 < groups) {
      if (int rc = setup(g + 1)) return rc;
    }
    const int slot = static_cast<int>(g & 1);
    for (int64_t k = g * group; k < K && k < (g + 1) * group; ++k) {
      const int64_t r = k % ring;
      const void* tc = t_c != nullptr ? static_cast<const char*>(t_c) + k * tc_bytes : nullptr;
      const char* table = slots + (slot * group + (k - g * group)) * table_bytes;
      void* out_p = static_cast<char*>(hp) + r * out_bytes;
      void* out_c = static_cast<char*>(hc) + r * out_bytes;
      // (the group's first forward makes the stream wait for the group's
      // set-up; the others follow it on the stream)
      int rc;
      if (k == g * group) {
        rc = wfx_pipeline_forward(p, slot, model, precision, table, freqs, offsets, B, n, max_len, tc, out_p, out_c,
                                  workspace, workspace_bytes, stream);
      } else if (model == WFX_XHM) {
        rc = wfx_xhm_polarizations(precision, table, freqs, offsets, B, n, max_len, tc, out_p, out_c, nullptr, stream);
      } else {
        rc = wfx_polarizations(model, precision, table, freqs, offsets, B, n, tc, out_p, out_c, workspace,
                               workspace_bytes, stream);
      }
      if (rc != 0) return rc;
    }
  }
  return wfx_pipeline_join(p, stream);
}

int wfx_pipeline_likelihood_run(wfx_pipeline_t p, int model, int64_t K, const double* params, int64_t B,
                                const double* f_min, int64_t f_min_stride, double amp_scale, double reference_mf,
                                float* tables, double* dtables, int32_t* status, const float* freqs,
                                const int64_t* offsets, int64_t n, const float* t_c, const void* data,
                                int data_stride, const void* weights, int weights_stride, double fp, double fc,
                                double scale, float* loss, float* grad, int64_t group, void* workspace,
                                size_t workspace_bytes, wfx_stream_t stream) {
  if (p == nullptr || params == nullptr || tables == nullptr || dtables == nullptr || status == nullptr ||
      loss == nullptr || grad == nullptr || K <= 0 || B <= 0 || n <= 0 || group <= 0 || model == WFX_XHM ||
      (group > 1 && f_min_stride != 0))
    return WFX_EINVAL;
  // (two halves of the workspace: batch k's partial sums in half k % 2, read
  // by its contraction on the second stream while batch k + 1's reverse pass
  // fills the other)
  const size_t half = wfx_workspace_bytes(WFX_OP_FUSED, model, WFX_FP32, B, n, offsets != nullptr);
  if (half == 0 || workspace == nullptr || workspace_bytes < 2 * half) return WFX_EWORKSPACE;
  const cudaStream_t caller = reinterpret_cast<cudaStream_t>(stream);
  const wfx_stream_t contracts = reinterpret_cast<wfx_stream_t>(p->side);
  const int64_t row = WFX_TABLE_STRIDE;
  const int64_t groups = (K + group - 1) / group;
  // the dual-number set-up of batches [g G, g G + G) into slot g % 2, after
  // what the caller's stream and the contractions' stream hold so far (group
  // g - 1's reverse passes and contractions, the last readers of that slot)
  const auto setup = [&](int64_t g) {
    const int slot = static_cast<int>(g & 1);
    const int64_t k0 = g * group, count = (K - k0 < group ? K - k0 : group);
    cudaError_t rc = cudaEventRecord(p->fork, caller);
    if (rc == cudaSuccess) rc = cudaStreamWaitEvent(p->side_jvp, p->fork, 0);
    if (rc == cudaSuccess) rc = cudaEventRecord(p->side_mark, p->side);
    if (rc == cudaSuccess) rc = cudaStreamWaitEvent(p->side_jvp, p->side_mark, 0);
    if (rc != cudaSuccess) return static_cast<int>(rc);
    const int r = wfx_setup_jvp(model, params + k0 * B * 8, count * B, f_min, f_min_stride, amp_scale, reference_mf,
                                nullptr, tables + slot * group * B * row, dtables + slot * group * B * row * 8,
                                status + k0 * B, reinterpret_cast<wfx_stream_t>(p->side_jvp));
    if (r != 0) return r;
    rc = cudaEventRecord(p->ready_jvp[slot], p->side_jvp);
    return rc == cudaSuccess ? 0 : static_cast<int>(rc);
  };
  if (int rc = setup(0)) return rc;
  for (int64_t g = 0; g < groups; ++g) {
    if (g + 1 < groups) {
      if (int rc = setup(g + 1)) return rc;
    }
    const int slot = static_cast<int>(g & 1);
    cudaError_t rc = cudaStreamWaitEvent(caller, p->ready_jvp[slot], 0);
    if (rc != cudaSuccess) return static_cast<int>(rc);
    for (int64_t k = g * group; k < K && k < (g + 1) * group; ++k) {
      const int64_t j = slot * group + (k - g * group);
      const int h = static_cast<int>(k & 1);
      char* ws = static_cast<char*>(workspace) + h * half;
      // (batch k - 2's contraction has read this half)
      if (k >= 2) rc = cudaStreamWaitEvent(caller, p->contracts_done[h], 0);
      if (rc != cudaSuccess) return static_cast<int>(rc);
      int r = wfx_fused_loss_partials(model, tables + j * B * row, freqs, offsets, B, n,
                                      t_c != nullptr ? t_c + k * B : nullptr, data, data_stride, weights,
                                      weights_stride, fp, fc, scale, ws, half, stream);
      if (r != 0) return r;
      rc = cudaEventRecord(p->partials_done[h], caller);
      if (rc == cudaSuccess) rc = cudaStreamWaitEvent(p->side, p->partials_done[h], 0);
      if (rc != cudaSuccess) return static_cast<int>(rc);
      r = wfx_fused_loss_contract(model, dtables + j * B * row * 8, offsets, B, n, loss + k * B,
                                  grad + k * B * WFX_GRAD_COLUMNS, ws, half, contracts);
      if (r != 0) return r;
      rc = cudaEventRecord(p->contracts_done[h], p->side);
      if (rc != cudaSuccess) return static_cast<int>(rc);
    }
  }
  return wfx_pipeline_join(p, stream);
}

int wfx_pipeline_join(wfx_pipeline_t p, wfx_stream_t stream) {
  if (p == nullptr) return WFX_EINVAL;
  const cudaStream_t caller = reinterpret_cast<cudaStream_t>(stream);
  cudaError_t rc = cudaEventRecord(p->join, p->side);
  if (rc == cudaSuccess) rc = cudaStreamWaitEvent(caller, p->join, 0);
  if (rc == cudaSuccess) rc = cudaEventRecord(p->join, p->side_jvp);
  if (rc == cudaSuccess) rc = cudaStreamWaitEvent(caller, p->join, 0);
  return rc == cudaSuccess ? 0 : static_cast<int>(rc);
}

}  // extern "C"
