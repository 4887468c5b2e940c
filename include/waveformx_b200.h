/*
 * waveformx-b200: the C ABI of the aligned-spin frequency-domain waveform
 * kernels (IMRPhenomXAS, IMRPhenomD, TaylorF2) for NVIDIA B200 (sm_100a).
 *
 * The reference (waveformx) has no native code: its hot path is
 * `waveformx.torch.polarizations_function` (src/waveformx/torch.py:175-183,
 * forward `_Model.forward` :100-106, backward `_Model.backward` :108-119)
 * and `waveformx.batch_polarizations` (src/waveformx/_api.py:307-360), which
 * call the models' pure JAX functions (models/xas/model.py:48-60,
 * models/phenomd/model.py:288-305, models/taylorf2/model.py:24-35) under
 * jax.jit + jax.vmap. These entry
 * points replace that evaluation and its jax.vjp; the Python layer
 * (waveformx_b200.torch, waveformx_b200.batch_polarizations) binds them
 * through ctypes with the same argument meaning and error behaviour.
 *
 * Conventions
 *  - Every pointer is a DEVICE pointer owned by the caller, unless stated.
 *    The library allocates no memory: scratch is a caller-given workspace
 *    of wfx_workspace_bytes() bytes.
 *  - Every call is stream-ordered on `stream` (a cudaStream_t; NULL is the
 *    legacy default stream) and returns immediately; calls are re-entrant.
 *  - Return value: 0 on success; a negative WFX_E* code for an invalid
 *    argument (nothing is launched); a positive CUDA error code if a launch
 *    failed. wfx_status_string() names both.
 *  - Parameters of binary b are params[8 b .. 8 b + 8): mass_1, mass_2
 *    (solar masses), chi_1, chi_2 (aligned spins), luminosity_distance
 *    (Mpc), inclination, phi_ref (rad), f_ref (Hz; 0 selects the first
 *    frequency, or for TaylorF2 the reference at coalescence), as the
 *    reference's Binary (src/waveformx/_binary.py:18-44)
 *    with the spins' z components.
 *  - Tables: one row of WFX_TABLE_STRIDE values per binary, written by
 *    wfx_setup (FP64 and/or FP32 copies) and read by every frequency kernel.
 *  - Frequency grids: `offsets == NULL` means one grid of `n` frequencies
 *    shared by every binary (outputs are B x n, row-major); otherwise binary
 *    b owns the frequencies and outputs [offsets[b], offsets[b+1]) of a
 *    flattened buffer of `n` = offsets[B] values (ragged batch).
 *  - Complex outputs are interleaved (re, im): complex64 (FP32) or
 *    complex128 (FP64).
 *  - Per-binary status (int32): 0, or the bits of WFX_STATUS_*; the
 *    waveform of a refused binary is NaN, as the reference's pure function.
 *  - t_c (s, per binary, may be NULL for zero) multiplies the strain by
 *    exp(-2 pi i f t_c): an extension, absent from the reference; t_c = 0
 *    reproduces it.
 */
#ifndef WAVEFORMX_B200_H
#define WAVEFORMX_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct CUstream_st* wfx_stream_t;

enum { WFX_XAS = 0, WFX_PHENOMD = 1, WFX_TAYLORF2 = 2, WFX_XHM = 3 };
enum { WFX_FP64 = 0, WFX_FP32 = 1 };
enum { WFX_TABLE_STRIDE = 72, WFX_GRAD_COLUMNS = 9 };
/* IMRPhenomXHM's rows (wfx_xhm_setup): 544 doubles (FP64), 576 floats (FP32). */
enum { WFX_XHM_STRIDE64 = 544, WFX_XHM_STRIDE32 = 576, WFX_XHM_MODES = 5 };

enum {
  WFX_EINVAL = -1,     /* a null pointer, a non-positive size or an unknown model */
  WFX_EOFFSETS = -2,   /* ragged offsets inconsistent with n */
  WFX_EWORKSPACE = -3, /* workspace missing or smaller than wfx_workspace_bytes() */
  WFX_EDEVICE = -4,    /* no usable CUDA device */
  WFX_ESCRATCH = -5    /* problem larger than WFX_STATIC_SCRATCH_BYTES (wfx_fused_loss_noalloc) */
};

enum {
  WFX_STATUS_MASS_RATIO = 1,    /* mass ratio beyond 1000 (IMRPhenomXAS) */
  WFX_STATUS_SPIN = 2,          /* |chi| > 1 */
  WFX_STATUS_FINAL_MASS = 4,    /* fitted final mass > total (IMRPhenomXAS) */
  WFX_STATUS_FINAL_SPIN = 8,    /* fitted final spin > 1 */
  WFX_STATUS_MECO = 16,         /* f_MECO > f_ISCO (IMRPhenomXAS) */
  WFX_STATUS_REFERENCE_MF = 32, /* reference_mf with f_ref != 0 */
  WFX_STATUS_PARAMETERS = 64,   /* non-positive masses or distance */
  WFX_STATUS_SOLVE = 128        /* a singular collocation system */
};

enum { WFX_OP_VJP = 0, WFX_OP_FUSED = 1, WFX_OP_POLARIZATIONS = 2 };

/* The library version (major * 10000 + minor * 100 + patch). */
int wfx_version(void);

/* A static description of a return code or (code > 0) a CUDA error. */
const char* wfx_status_string(int code);

/* The per-binary set-up in FP64 (the coefficient fits, the collocation
 * solves, the connection coefficients, the time shift and the phase
 * alignment at f_ref), one chain per binary. Replaces the table of
 * models/xas/core.py:257-379, models/phenomd/core.py:280-378 and
 * models/taylorf2/core.py:107-165.
 *   f_min: first frequency of each binary (f_min[b * f_min_stride]; stride 0
 *          for one value), the f_ref of f_ref = 0;
 *   amp_scale: the strain scale (1e21, or 1 with scaled_strain = False);
 *   reference_mf: NaN for none, else WaveformOptions.reference_mf;
 *   table64 (B x 72 double) and table32 (B x 72 float): either may be NULL;
 *   status (B int32): may be NULL. */
int wfx_setup(int model, const double* params, int64_t B, const double* f_min, int64_t f_min_stride,
              double amp_scale, double reference_mf, double* table64, float* table32, int32_t* status,
              wfx_stream_t stream);

/* The set-up and its forward-mode derivative along the eight parameters
 * (dual numbers, one thread per binary and parameter):
 *   dtable (B x 72 x 8 double): d table[b][k] / d params[b][j] at
 *   [(b * 72 + k) * 8 + j]. table64, table32, status as wfx_setup. */
int wfx_setup_jvp(int model, const double* params, int64_t B, const double* f_min, int64_t f_min_stride,
                  double amp_scale, double reference_mf, double* table64, float* table32, double* dtable,
                  int32_t* status, wfx_stream_t stream);

/* The set-up of IMRPhenomXHM (models/xhm/core.py:388-397 with
 * models/xhm/reference.py): the (2,2) table of IMRPhenomXAS, the factors of
 * the five modes in the polarizations, and the tables of the higher modes
 * (2,1), (3,3), (3,2), (4,4); one thread per binary and part. Arguments as
 * wfx_setup, with table64 (B x WFX_XHM_STRIDE64 double) and table32 (B x
 * WFX_XHM_STRIDE32 float, 16-byte aligned); either may be NULL. */
int wfx_xhm_setup(const double* params, int64_t B, const double* f_min, int64_t f_min_stride, double amp_scale,
                  double reference_mf, double* table64, float* table32, int32_t* status, wfx_stream_t stream);

/* IMRPhenomXHM's set-up with its forward-mode derivative along the eight
 * parameters (the tables and tangents of the reference's XHM VJP,
 * models/xhm/mlx/_api.py:42-48 and 63-69): the set-up of every part on dual
 * numbers, one thread per binary, part and parameter. dtable (B x
 * WFX_XHM_STRIDE64 x 8 double): d row64[b][k] / d params[b][j] at
 * [(b * WFX_XHM_STRIDE64 + k) * 8 + j]; zero along f_ref where it is 0 (the
 * first frequency or reference_mf / M stands for it). table64, table32 and
 * status as wfx_xhm_setup (all three NULL: the derivatives alone). */
int wfx_xhm_setup_jvp(const double* params, int64_t B, const double* f_min, int64_t f_min_stride, double amp_scale,
                      double reference_mf, double* table64, float* table32, double* dtable, int32_t* status,
                      wfx_stream_t stream);

/* IMRPhenomXHM's (hplus, hcross) (models/xhm/core.py:524-556): on a grid of
 * n frequencies shared by the B binaries (offsets NULL; B x n outputs),
 * and, where `modes` is not NULL, the modes h_{l,-m} of (2,2), (2,1),
 * (3,3), (3,2), (4,4) (B x 5 x n complex); or ragged (offsets of B + 1
 * starts into n flat frequencies and outputs, max_len the longest binary's
 * length; modes NULL). WFX_FP32: table float, freqs float, t_c float,
 * complex64 out; WFX_FP64: double, complex128. t_c (per binary, may be
 * NULL) multiplies every mode by exp(-2 pi i f t_c). */
int wfx_xhm_polarizations(int precision, const void* table, const void* freqs, const int64_t* offsets, int64_t B,
                          int64_t n, int64_t max_len, const void* t_c, void* hp, void* hc, void* modes,
                          wfx_stream_t stream);

/* The derivative with respect to the frequency grid (the reference's
 * drop-in differentiates its models with respect to the grid through
 * jax.vjp, src/waveformx/torch.py:12-13, 87-91): grad_f[k] = sum_b
 * Re(conj(g+[b][k]) dh+/df + conj(gx[b][k]) dhx/df) on a shared grid (n
 * values, zeroed here), or per element of a ragged one; the FP64 evaluation
 * of `table` (double, as wfx_setup; WFX_XHM: the FP64 rows of
 * wfx_xhm_setup) differentiated in f (the set-up's first frequency carries
 * none, as the reference's). Cotangents complex128 in the layout of
 * wfx_polarizations; t_c may be NULL. */
int wfx_grid_vjp(int model, const double* table, const double* freqs, const int64_t* offsets, int64_t B, int64_t n,
                 const double* t_c, const void* cot_hp, const void* cot_hc, double* grad_f, wfx_stream_t stream);

/* IMRPhenomXHM's gradient (the reference's jax.grad through
 * models/xhm/model.py:30-42): grad (B x 9 double, zeroed here) = d L /
 * d (mass_1, mass_2, chi_1, chi_2, luminosity_distance, inclination,
 * phi_ref, f_ref, t_c) for the cotangents cot_hp, cot_hc (complex128, dL/dRe
 * h + i dL/dIm h, the layout of wfx_xhm_polarizations) of the FP64
 * evaluation: forward-mode derivatives of the evaluation along each column
 * of dtable (B x WFX_XHM_STRIDE64 x 8 double: d table / d parameter, the
 * caller's), contracted with the cotangents. Grids as
 * wfx_xhm_polarizations. */
int wfx_xhm_vjp(const double* table, const double* dtable, const double* freqs, const int64_t* offsets, int64_t B,
                int64_t n, int64_t max_len, const double* t_c, const void* cot_hp, const void* cot_hc, double* grad,
                wfx_stream_t stream);

/* For the converters between LAL's reference convention (phi_ref at f_ref
 * in Hz) and the mass-scaled one (src/waveformx/_reference.py:59-80,
 * models/taylorf2/reference.py:46-104): dphi[b] = Phi(mf_to[b]) -
 * Phi(mf_from[b]), Phi the (2,2) phase of binary b's model at M f (but for
 * its constant; IMRPhenomXHM's that of IMRPhenomXAS), from its FP64 set-up;
 * an mf of 0 contributes 0 (no reference phase), a negative or NaN one
 * NaN. params as wfx_setup (distance and f_ref unused). */
int wfx_phase_difference(int model, const double* params, int64_t B, const double* mf_from, const double* mf_to,
                         double* dphi, wfx_stream_t stream);

/* (hplus, hcross) at the frequencies: the evaluation of
 * models/xas/core.py:496-507 / models/phenomd/core.py:476-485 behind
 * waveformx.torch's forward.
 *   WFX_FP32: table float, freqs float, t_c float, hp/hc complex64: FP32
 *     with double-float phase;
 *   WFX_FP64: table double, freqs double, t_c double, hp/hc complex128: the
 *     plain FP64 form (one binary per block).
 * The FP32 ragged form (offsets != NULL) runs one persistent launch over
 * (binary, tile) work items whose index lives in the workspace
 * (wfx_workspace_bytes(WFX_OP_POLARIZATIONS, ...)); the other forms need no
 * workspace (NULL, 0). */
int wfx_polarizations(int model, int precision, const void* table, const void* freqs, const int64_t* offsets,
                      int64_t B, int64_t n, const void* t_c, void* hp, void* hc, void* workspace,
                      size_t workspace_bytes, wfx_stream_t stream);

/* The batch pipeline (no counterpart in the reference, which evaluates one
 * call at a time): the FP64 set-up of batch k + 1 on a second stream of the
 * highest priority while batch k's forward runs on the caller's stream, two
 * table slots alternating. A pipeline (a second stream and its events, on
 * the current device) serves one sequence of batches at a time.
 *   wfx_pipeline_create / _destroy: make one / release it (destroy waits for
 *     its second stream);
 *   wfx_pipeline_setup: after everything queued on `stream` so far (the
 *     batch's parameters, the forward that last read this slot's table),
 *     the set-up of the batch (arguments as wfx_setup, or wfx_xhm_setup for
 *     WFX_XHM) on the second stream, then slot `slot` (0 or 1) is ready;
 *   wfx_pipeline_forward: `stream` waits for slot `slot`, then the batch's
 *     forward (arguments as wfx_polarizations; WFX_XHM: wfx_xhm_polarizations
 *     with max_len, no modes);
 *   wfx_pipeline_join: `stream` waits for everything queued on the second
 *     stream (before the caller frees the tables or the parameters). */
typedef struct wfx_pipeline* wfx_pipeline_t;
int wfx_pipeline_create(wfx_pipeline_t* out);
int wfx_pipeline_destroy(wfx_pipeline_t pipeline);
int wfx_pipeline_setup(wfx_pipeline_t pipeline, int slot, int model, const double* params, int64_t B,
                       const double* f_min, int64_t f_min_stride, double amp_scale, double reference_mf,
                       double* table64, float* table32, int32_t* status, wfx_stream_t stream);
int wfx_pipeline_forward(wfx_pipeline_t pipeline, int slot, int model, int precision, const void* table,
                         const void* freqs, const int64_t* offsets, int64_t B, int64_t n, int64_t max_len,
                         const void* t_c, void* hp, void* hc, void* workspace, size_t workspace_bytes,
                         wfx_stream_t stream);
int wfx_pipeline_join(wfx_pipeline_t pipeline, wfx_stream_t stream);
/* K batches through the pipeline in one call (the pairs of
 * wfx_pipeline_setup and wfx_pipeline_forward above, queued by the library,
 * then wfx_pipeline_join): batch k's parameters are params + 8 B k (K x B x 8
 * double), its t_c t_c + B k (K x B, the precision's real type; or NULL),
 * its status status + B k (K x B int32); its outputs go to ring slot k % ring
 * of hp and hc (ring slots of B x n, or n ragged, complex values each, slot r
 * starting at element r E, E that count rounded up to an even number for
 * complex64 so that every slot is 16-byte aligned; with ring < K a slot is
 * rewritten once the forward before it on `stream` has finished).
 * group: the batches set up by one launch (the set-up's time hardly depends
 * on its number of binaries: one launch for `group` batches during the
 * previous group's forwards); group > 1 needs one f_min for every binary
 * (f_min_stride 0). tables: two slots of `group` tables, 2 x group x B x the
 * model's row (WFX_TABLE_STRIDE, or IMRPhenomXHM's) of the precision's real
 * type. Other arguments as wfx_pipeline_setup and wfx_pipeline_forward. */
int wfx_pipeline_run(wfx_pipeline_t pipeline, int model, int precision, int64_t K, const double* params, int64_t B,
                     const double* f_min, int64_t f_min_stride, double amp_scale, double reference_mf, void* tables,
                     int32_t* status, const void* freqs, const int64_t* offsets, int64_t n, int64_t max_len,
                     const void* t_c, void* hp, void* hc, int64_t ring, int64_t group, void* workspace,
                     size_t workspace_bytes, wfx_stream_t stream);
/* The likelihood's batches through the same pipeline:
 *   wfx_pipeline_setup_jvp: after everything queued on `stream` so far, the
 *     batch's dual-number set-up (dtable as wfx_setup_jvp; not WFX_XHM) on a
 *     third stream, then slot `slot`'s dtable is ready;
 *   wfx_pipeline_fused: `stream` waits for slot `slot`'s table (queued by
 *     wfx_pipeline_setup), runs wfx_fused_loss_partials, waits for the
 *     slot's dtable, then wfx_fused_loss_contract (arguments as those). */
int wfx_pipeline_setup_jvp(wfx_pipeline_t pipeline, int slot, int model, const double* params, int64_t B,
                           const double* f_min, int64_t f_min_stride, double amp_scale, double reference_mf,
                           double* dtable, wfx_stream_t stream);
int wfx_pipeline_fused(wfx_pipeline_t pipeline, int slot, int model, const void* table, const void* freqs,
                       const int64_t* offsets, int64_t B, int64_t n, const void* t_c, const void* data,
                       int data_stride, const void* weights, int weights_stride, double fp, double fc, double scale,
                       const double* dtable, void* loss, void* grad, void* workspace, size_t workspace_bytes,
                       wfx_stream_t stream);
/* K likelihood batches in one call: the dual-number set-up of `group`
 * batches in one launch on the third stream (it writes their FP32 tables and
 * dtables: no separate value set-up), during the previous group's fused
 * likelihoods; each batch's wfx_fused_loss_partials on `stream`, the
 * group's first after its set-up, and its wfx_fused_loss_contract on the
 * second stream beside the next batch's. Batch k: params + 8 B k (K x B x 8
 * double), t_c + B k (K x B float, or NULL), status + B k, loss + B k (K x B
 * float), grad + 9 B k (K x B x 9 float). tables (2 x group x B x
 * WFX_TABLE_STRIDE float, 16-byte aligned) and dtables (2 x group x B x
 * WFX_TABLE_STRIDE x 8 double): two slots of `group` batches. group > 1
 * needs one f_min for every binary (f_min_stride 0). workspace: two halves
 * of wfx_workspace_bytes(WFX_OP_FUSED, model, WFX_FP32, B, n, ragged) bytes
 * (WFX_EWORKSPACE if smaller), batches alternating. freqs, offsets, data and
 * weights are shared by the batches (arguments as wfx_fused_loss_partials);
 * not WFX_XHM. Ends with wfx_pipeline_join. */
int wfx_pipeline_likelihood_run(wfx_pipeline_t pipeline, int model, int64_t K, const double* params, int64_t B,
                                const double* f_min, int64_t f_min_stride, double amp_scale, double reference_mf,
                                float* tables, double* dtables, int32_t* status, const float* freqs,
                                const int64_t* offsets, int64_t n, const float* t_c, const void* data,
                                int data_stride, const void* weights, int weights_stride, double fp, double fc,
                                double scale, float* loss, float* grad, int64_t group, void* workspace,
                                size_t workspace_bytes, wfx_stream_t stream);

/* Scratch bytes of wfx_vjp / wfx_fused_loss / wfx_polarizations (op
 * WFX_OP_*) for a problem of B binaries and n frequencies (shared grid) or n
 * flattened frequencies (ragged). Host function; 0 where none is needed
 * (the FP64 forms, the FP32 shared-grid forward).
 *
 * Ragged offsets must run from offsets[0] >= 0, non-decreasing, to
 * offsets[B] == n (the check that the reference's batch API makes on its
 * rows, src/waveformx/_api.py:292-305, and its grids,
 * src/waveformx/_results.py:31). The FP32 ragged forms check them on the
 * device, in the call's first kernel, and keep the result in the first int32
 * of the workspace: 0, or WFX_EOFFSETS, in which case no frequency is
 * evaluated (hp and hc are not written; loss and grad are NaN). The FP64 and
 * IMRPhenomXHM ragged forms clamp each binary's range to [0, n] instead. No
 * form reads or writes outside its buffers whatever the offsets hold. */
size_t wfx_workspace_bytes(int op, int model, int precision, int64_t B, int64_t n, int ragged);

/* The offsets check of the last FP32 ragged call (wfx_polarizations,
 * wfx_vjp, wfx_fused_loss, wfx_fused_loss_partials, wfx_autotune_ragged)
 * that used `workspace` on `stream`: waits for `stream`, then returns 0 or
 * WFX_EOFFSETS (a positive CUDA error if the read failed; WFX_EINVAL if the
 * workspace holds no such word). Replaces the synchronous row check of
 * src/waveformx/_api.py:292-305 for callers that hold the offsets on the
 * device only. */
int wfx_ragged_status(const void* workspace, wfx_stream_t stream);

/* The autotuner of the FP32 ragged forward (no counterpart in the
 * reference, whose ragged batches are a Python loop): times the candidate
 * work-item lengths (510, 1022, 2046, 4094 frequencies) and persistent
 * grids (2, 4, 8, 16 blocks per SM) on this problem (arguments as
 * wfx_polarizations with offsets), keeps the fastest for the current device,
 * the model and the size class (log2 n, log2 B), and writes it to config[2]
 * (item length, blocks per SM) if not NULL. Later wfx_polarizations calls of
 * that class use it; the outputs do not depend on it. Synchronises the
 * stream: call it outside any stream capture. */
int wfx_autotune_ragged(int model, const void* table, const void* freqs, const int64_t* offsets, int64_t B, int64_t n,
                        const void* t_c, void* hp, void* hc, void* workspace, size_t workspace_bytes,
                        wfx_stream_t stream, int64_t* config);

/* The tuning of the FP32 ragged forward for the size class of (B, n) on
 * the current device: set = 0 writes it to config[2] and returns 1 if tuned
 * (0 and the default otherwise); set = 1 installs config[2] (a persisted
 * result; item length >= 510, 1 to 64 blocks per SM) and returns 1. Host
 * function; the table is process-wide and guarded by a mutex. */
int wfx_tuning(int model, int64_t B, int64_t n, int64_t* config, int set);

/* The vector-Jacobian product of wfx_polarizations: for cotangents (g+, gx)
 * of (hp, hc) in PyTorch's convention (dL/dRe + i dL/dIm; complex arrays
 * like the outputs), grad[b][j] = dL/dtheta_j for theta = (mass_1, mass_2,
 * chi_1, chi_2, luminosity_distance, inclination, phi_ref, f_ref, t_c)
 * (B x WFX_GRAD_COLUMNS, float for FP32, double for FP64). Recomputes the
 * waveform (no residuals); dtable from wfx_setup_jvp. Replaces the jax.vjp
 * of src/waveformx/torch.py:87-93. */
int wfx_vjp(int model, int precision, const void* table, const double* dtable, const void* freqs,
            const int64_t* offsets, int64_t B, int64_t n, const void* t_c, const void* cot_hp, const void* cot_hc,
            void* grad, void* workspace, size_t workspace_bytes, wfx_stream_t stream);

/* The fused likelihood: loss[b] = scale * sum_f w(f) |fp hp(f) + fc hc(f) - d(f)|^2
 * and (grad != NULL, dtable != NULL) its gradient as wfx_vjp, without
 * writing the strain. data: complex (like hp), shared (data_stride 0, n
 * values) or per binary (data_stride 1, laid out like hp); weights: real,
 * shared (weights_stride 0) or per binary (weights_stride 1). loss: B values
 * (float / double). The log-likelihood of whitened Gaussian noise is
 * scale = -1/2. */
int wfx_fused_loss(int model, int precision, const void* table, const double* dtable, const void* freqs,
                   const int64_t* offsets, int64_t B, int64_t n, const void* t_c, const void* data,
                   int data_stride, const void* weights, int weights_stride, double fp, double fc, double scale,
                   void* loss, void* grad, void* workspace, size_t workspace_bytes, wfx_stream_t stream);

/* wfx_fused_loss (FP32) in two calls, so that dtable can be computed while
 * the reverse pass runs (wfx_setup_jvp with NULL tables on another stream:
 * the dual-number set-up is a latency-bound chain per binary that the
 * reverse pass, which needs only the table, does not wait for).
 *   wfx_fused_loss_partials: the reverse pass, its per-item sums left in
 *     the workspace (arguments as wfx_fused_loss, without dtable, loss and
 *     grad; the gradient's sums are always formed);
 *   wfx_fused_loss_contract: loss and grad (either may be NULL; grad needs
 *     dtable) from those sums, with the same model, offsets, B, n and
 *     workspace, untouched in between.
 * Same results as wfx_fused_loss. No counterpart in the reference (see
 * wfx_fused_loss). */
int wfx_fused_loss_partials(int model, const void* table, const void* freqs, const int64_t* offsets, int64_t B,
                            int64_t n, const void* t_c, const void* data, int data_stride, const void* weights,
                            int weights_stride, double fp, double fc, double scale, void* workspace,
                            size_t workspace_bytes, wfx_stream_t stream);
int wfx_fused_loss_contract(int model, const double* dtable, const int64_t* offsets, int64_t B, int64_t n, void* loss,
                            void* grad, void* workspace, size_t workspace_bytes, wfx_stream_t stream);

/* Matches maximised over a time shift and a constant phase (replaces the
 * match of src/waveformx/match.py:71-147: _overlap, _series, _refine,
 * _best_time, match). Three steps:
 *   1. wfx_overlap (two waveforms) or wfx_template_overlap (a bank of
 *      templates evaluated from their tables, never written to memory):
 *      the series c[r][k] = 4 delta_f a[r][k] conj(b[r][k]) / psd[k] of
 *      each row r, k < n, into `series` (rows x n_fft complex, row stride
 *      n_fft), and norms[2 r] = <a_r, a_r>, norms[2 r + 1] = <b_r, b_r>
 *      (double, <x, y> = 4 delta_f Re sum x conj(y) / psd). Columns
 *      [n, n_fft) of `series` are not written: zero them once.
 *   2. the caller's inverse FFT of each row of `series` into `zgrid`,
 *      unnormalised (zgrid[r][j] = sum_k c[r][k] e^(2 pi i k j / n_fft);
 *      cuFFT CUFFT_INVERSE), n_fft = pad x the power of two >= n (the
 *      reference's pad = 4). Skipped without the time maximisation.
 *   3. wfx_match_refine: the first largest |z| (with phase) or
 *      Re z e^(2 pi i f_0 t_j) (without) of the grid t_j = j / (n_fft
 *      delta_f), wrapped to (-P/2, P/2] (P = 1 / delta_f), then `steps`
 *      Newton steps (the reference's 3) on the exact z(t) = sum_k c_k
 *      e^(2 pi i f_k t) at the frequencies freqs (double, uniformly spaced
 *      by delta_f), each kept only if it does not lower the objective;
 *      match[r] = |z(t)| (or Re z(t)) / sqrt(norms[2 r] norms[2 r + 1]),
 *      t[r] the time (may be NULL). FP64 sums.
 * precision: WFX_FP64 (complex128 waveforms, series and zgrid, double psd)
 * or WFX_FP32 (complex64, float psd). a_stride, b_stride: n (one vector per
 * row) or 0 (one vector for every row). */
int wfx_overlap(int precision, const void* a, int64_t a_stride, const void* b, int64_t b_stride, const void* psd,
                int64_t rows, int64_t n, double delta_f, void* series, int64_t n_fft, double* norms,
                wfx_stream_t stream);

/* Step 1 for the templates h_b = fp hplus_b + fc hcross_b of B binaries
 * (FP32 tables of wfx_setup, a shared grid `freqs` of n frequencies, t_c
 * per binary or NULL) against one signal (n complex64) with psd (n
 * float): the series c[b][k] = 4 delta_f h_b(f_k) conj(signal_k) / psd_k
 * (complex64, row stride n_fft, even) and norms[2 b] = <h_b, h_b>,
 * norms[2 b + 1] = <signal, signal>, without writing the templates'
 * strain. table and series 16-byte aligned. */
int wfx_template_overlap(int model, const float* table, const float* freqs, int64_t B, int64_t n, const float* t_c,
                         double fp, double fc, const void* signal, const float* psd, double delta_f, void* series,
                         int64_t n_fft, double* norms, wfx_stream_t stream);

/* polarization_match (src/waveformx/match.py:150-187): the match of a
 * signal with F+ h+ + Fx hx maximised over time and over F+ and Fx (the
 * norm of the signal's projection onto the real span of the two
 * polarizations over its norm; with parallel polarizations the match with
 * h+ alone). The same three steps as wfx_overlap:
 *   1. wfx_polarization_overlap: rows 2 r and 2 r + 1 of `series` (2 rows x
 *      n_fft complex) are 4 delta_f s conj(h+) / psd and 4 delta_f s
 *      conj(hx) / psd of row r, norms[4 r ..] = <s, s>, <h+, h+>, <hx, hx>,
 *      <h+, hx>; strides as wfx_overlap;
 *      wfx_template_polarization_overlap: the same for the polarizations of
 *      B binaries' FP32 tables against one signal, without their strain;
 *   2. the caller's inverse FFT of the 2 rows x n_fft series;
 *   3. wfx_polarization_refine: the first largest value of the grid, then
 *      `steps` Newton steps on the exact objective; match[r], t[r]. */
int wfx_polarization_overlap(int precision, const void* signal, int64_t s_stride, const void* hplus, int64_t p_stride,
                             const void* hcross, int64_t x_stride, const void* psd, int64_t rows, int64_t n,
                             double delta_f, void* series, int64_t n_fft, double* norms, wfx_stream_t stream);
int wfx_template_polarization_overlap(int model, const float* table, const float* freqs, int64_t B, int64_t n,
                                      const float* t_c, const void* signal, const float* psd, double delta_f,
                                      void* series, int64_t n_fft, double* norms, wfx_stream_t stream);
int wfx_polarization_refine(int precision, const void* series, const void* zgrid, int64_t rows, int64_t n,
                            int64_t n_fft, const double* freqs, double delta_f, const double* norms, int time,
                            int steps, double* match, double* t, wfx_stream_t stream);

/* Step 2 and the start of step 3 without the grid in memory, for the
 * match with the phase maximisation of FP32 (complex64) series: one block
 * per row computes the row's inverse FFT in shared memory and writes only
 * t[r], the grid's best time wrapped to (-P/2, P/2]; then wfx_match_refine
 * with time = 2 starts from it. The series is zero from n on, so the
 * transform is n_fft / L transforms of length L, the power of two >=
 * max(n, 2048); supported when L <= 16384 and L divides n_fft (the
 * reference's pad of 4 and n up to 16384), else WFX_EINVAL. */
int wfx_match_grid_time(const void* series, int64_t rows, int64_t n, int64_t n_fft, double delta_f, double* t,
                        wfx_stream_t stream);

/* Step 3 (see wfx_overlap). time: 0 none, 1 from zgrid, 2 from t (the
 * times of wfx_match_grid_time, overwritten by the refined ones). */
int wfx_match_refine(int precision, const void* series, const void* zgrid, int64_t rows, int64_t n, int64_t n_fft,
                     const double* freqs, double delta_f, const double* norms, int time, int phase, int steps,
                     double* match, double* t, wfx_stream_t stream);

/* wfx_fused_loss without a workspace argument: the library allocates
 * nothing, in this call or any other. No counterpart in the reference (its
 * likelihood runs through JAX, whose allocator provides the scratch).
 *
 * For callers that cannot hand the library device memory per call: a
 * sampler's likelihood callback written in C or Fortran, or bound through a
 * plain FFI, with no caching allocator at hand, or one that evaluates the
 * likelihood every few hundred microseconds, where cudaMalloc/cudaFree
 * (which synchronise the device) would cost more than the evaluation.
 *
 * Arguments, results and errors as wfx_fused_loss. The FP32 form's scratch
 * is a buffer of WFX_STATIC_SCRATCH_BYTES per device inside the library's
 * own module: problems whose wfx_workspace_bytes(WFX_OP_FUSED, ...) exceeds
 * it are refused with WFX_ESCRATCH (about 32,000 binaries of up to 4,092
 * frequencies on a shared grid; split larger batches into several calls).
 * The FP64 form needs no scratch.
 *   - Nothing needs to start at zero: each call writes the scratch before it
 *     reads it.
 *   - The first call on each device looks up the buffer's address (with that
 *     device current), and so does the first call after the device's
 *     context changes (after cudaDeviceReset, for instance); make those calls
 *     outside any stream capture.
 *   - Ragged offsets that fail the check of wfx_workspace_bytes give NaN
 *     loss and gradient (the status word is in the library's scratch).
 *   - One buffer per device: two calls that may run at the same time on one
 *     device (different streams, or host threads without ordering) race on
 *     it. Order them on one stream, or by events. */
enum { WFX_STATIC_SCRATCH_BYTES = 16777216 };
int wfx_fused_loss_noalloc(int model, int precision, const void* table, const double* dtable, const void* freqs,
                           const int64_t* offsets, int64_t B, int64_t n, const void* t_c, const void* data,
                           int data_stride, const void* weights, int weights_stride, double fp, double fc,
                           double scale, void* loss, void* grad, wfx_stream_t stream);

#ifdef __cplusplus
}
#endif

#endif /* WAVEFORMX_B200_H */
