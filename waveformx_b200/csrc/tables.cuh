// The per-binary tables: the coefficients of a binary's waveform in powers
// of the frequency in Hz (the powers of the total mass folded in), written
// once per binary by the FP64 set-up and read by every frequency.
//
// Every model uses 72 slots (288 B as float, 576 B as double): one row of
// a (B, 72) array, staged in shared memory by the frequency kernels.
#pragma once

#if !defined(__CUDACC__)
#define __host__
#define __device__
#endif

namespace wfx {

constexpr int kTableStride = 72;

// IMRPhenomXAS.
enum XasSlot : int {
  // inspiral phase: the coefficients of f^-1, f^-2/3, f^-1/3, log f, 1,
  // f^1/3, f^1/3 log f, f^2/3, f, f log f, f^4/3, f^5/3, f^2 (the leading
  // f^-5/3 apart, in X_T0)
  X_PH_INS = 0,
  // intermediate phase: 1, f, log f, f^-1, f^-2, f^-3
  X_PH_INT = 13,
  // ringdown phase: 1, f, f^2/3, f^-1, f^-3
  X_PH_RD = 19,
  // a atan(w (f - shift)) past the inspiral: [intermediate, ringdown]
  X_ATAN_A = 24,
  X_ATAN_W = 26,
  X_SHIFT = 28,
  // inspiral amplitude f^-7/6 sum_k c_k f^(k/3), k = 0..9
  X_AMP_INS = 29,
  // intermediate amplitude n / sum_j d_j f^j, j = 0..4
  X_AMP_INT_N = 39,
  X_AMP_INT_D = 40,
  // ringdown amplitude n f^-7/6 exp(-gr u) / (u^2 + g), u = s (f - shift)
  X_AMP_RD_N = 45,
  X_AMP_RD_GR = 46,
  X_AMP_RD_S = 47,
  X_AMP_RD_G = 48,
  // region boundaries and cutoff (Hz): phase past the inspiral where
  // f >= f_phase_in, ringdown where f > f_phase_im; amplitude likewise
  // with f >= f_amp_in, f > f_amp_rd; zero above f_cut
  X_F_PHASE_IN = 49,
  X_F_PHASE_IM = 50,
  X_F_AMP_IN = 51,
  X_F_AMP_RD = 52,
  X_F_CUT = 53,
  // the polarization factors (NaN where LAL refuses the binary)
  X_KP = 54,
  X_KC = 55,
  // the leading inspiral term T0 f^-5/3 and its value A at f_ref (zero past
  // the inspiral), subtracted at every frequency
  X_T0 = 56,
  X_ANCHOR = 57,
  X_USED = 58,
  // FP32 tables only. The phase's large parts are double-floats: the float
  // slots above hold the hi parts of T0, of each region's constant (with
  // the anchor folded in: constant - A) and of its coefficient of f; these
  // hold what the floats lack (the anchor's own slot is reused)
  X32_T0_LO = 57,
  X32_CONST_LO = 58,  // inspiral, intermediate, ringdown
  X32_LIN_LO = 61,    // inspiral, intermediate, ringdown
  X32_RD_TERM_LO = 64,  // the ringdown's f^2/3 coefficient (X_PH_RD + 2)
};

// IMRPhenomD.
enum PhdSlot : int {
  // inspiral phase: 1, f^-1, f^-2/3, f^-1/3, log f, f^1/3, f^1/3 log f,
  // f^2/3, f, f^4/3, f^5/3, f^2 (the leading f^-5/3 apart, in D_T0)
  D_PH_INS = 0,
  // intermediate phase: 1, f, f^-3, log f
  D_PH_INT = 12,
  // merger-ringdown phase: 1, f, f^-1, f^3/4, plus a atan(w (f - shift))
  D_PH_RD = 16,
  D_ATAN_A = 20,
  D_ATAN_W = 21,
  D_ATAN_SHIFT = 22,
  // inspiral amplitude f^-7/6 sum_k c_k f^(k/3)
  D_AMP_INS = 23,
  // intermediate amplitude f^-7/6 sum_j d_j y^j, y = s_int f
  D_AMP_INT = 33,
  D_AMP_INT_S = 38,
  // merger-ringdown amplitude n f^-7/6 exp(-gr u) / (u^2 + 1), u = s (f - shift)
  D_AMP_RD_N = 39,
  D_AMP_RD_GR = 40,
  D_AMP_RD_S = 41,
  D_AMP_RD_SHIFT = 42,
  // boundaries (Hz): inspiral where f < f_phase_ins, merger-ringdown where
  // f >= f_phase_mrd; amplitude likewise; no cutoff
  D_F_PHASE_INS = 43,
  D_F_PHASE_MRD = 44,
  D_F_AMP_INS = 45,
  D_F_AMP_MRD = 46,
  D_KP = 47,
  D_KC = 48,
  D_T0 = 49,
  D_ANCHOR = 50,
  D_USED = 51,
  // FP32 tables only (as X32_*)
  D32_T0_LO = 50,
  D32_CONST_LO = 51,
  D32_LIN_LO = 54,
  D32_RD_TERM_LO = 57,  // the merger-ringdown's f^3/4 coefficient (D_PH_RD + 3)
};

// TaylorF2: one region, no cutoff.
enum Tf2Slot : int {
  // phase: the coefficients of f^-1, f^-2/3, f^-1/3, log f, 1, f^1/3,
  // f^1/3 log f, f^2/3 (the leading f^-5/3 apart, in T_T0)
  T_PH = 0,
  // the coefficient of f: zero in the model (the t_c extension enters it)
  T_LIN = 8,
  // the amplitude A f^-7/6
  T_AMP = 9,
  T_KP = 10,
  T_KC = 11,
  T_T0 = 12,
  T_ANCHOR = 13,
  T_USED = 14,
  // FP32 tables only (as X32_*)
  T32_T0_LO = 13,
  T32_CONST_LO = 14,
  T32_LIN_LO = 15,
};

// The slots of each phase region's constant term and coefficient of f
// (r = 0 inspiral, 1 intermediate, 2 ringdown).
__host__ __device__ constexpr int xas_const_slot(int r) { return r == 0 ? X_PH_INS + 4 : (r == 1 ? X_PH_INT : X_PH_RD); }
__host__ __device__ constexpr int xas_lin_slot(int r) { return r == 0 ? X_PH_INS + 8 : (r == 1 ? X_PH_INT : X_PH_RD) + 1; }
__host__ __device__ constexpr int phd_const_slot(int r) { return r == 0 ? D_PH_INS : (r == 1 ? D_PH_INT : D_PH_RD); }
__host__ __device__ constexpr int phd_lin_slot(int r) { return r == 0 ? D_PH_INS + 8 : (r == 1 ? D_PH_INT : D_PH_RD) + 1; }

__host__ __device__ constexpr int tf2_const_slot(int) { return T_PH + 4; }
__host__ __device__ constexpr int tf2_lin_slot(int) { return T_LIN; }

enum Model : int { kModelXas = 0, kModelPhenomD = 1, kModelTaylorF2 = 2, kModelXhm = 3 };

// IMRPhenomXHM: a row of kXhmStride64 doubles (FP64) or kXhmStride32 floats
// (FP32): the (2,2) table in slots [0, kTableStride) (XasSlot, its FP32
// form as for IMRPhenomXAS), the head, then the four higher modes (2,1),
// (3,3), (3,2), (4,4), each in the layout of the reference's MODE_LAYOUT
// (112 values; setup_xhm.cuh, ModeSlot). An FP32 mode adds the double-float
// parts of its phase: (m/2)^(8/3) T0 as hi and lo, and the lo parts of each
// region's coefficient of f; its regions' constants hold (constant - (m/2) A)
// modulo 2 pi.
enum XhmSlot : int {
  H_FACTORS = 72,  // Re F+, Im F+, Re Fx, Im Fx of (2,2), (2,1), (3,3), (3,2), (4,4)
  H_AMP0 = 92,
  H_S = 93,        // M in seconds
  H_COS_A = 94,    // cos and sin of the (2,2)'s anchor A (its phase without A
  H_SIN_A = 95,    // is the phase's angle plus A)
  H_MODES = 96,
  HM32_T0_HI = 112,  // (within an FP32 mode)
  HM32_T0_LO = 113,
  HM32_LIN_LO = 114,  // inspiral, intermediate, ringdown
};
constexpr int kXhmModeStride64 = 112;
constexpr int kXhmModeStride32 = 120;
constexpr int kXhmStride64 = H_MODES + 4 * kXhmModeStride64;  // 544
constexpr int kXhmStride32 = H_MODES + 4 * kXhmModeStride32;  // 576

// The slots that code common to the models needs: the phase regions and
// their constant and linear slots, the projection, the leading term and
// its anchor, and the FP32 double-float parts (kBigTerm: the largest term
// past the inspiral carried in double-float, -1 for none).
template <int MODEL>
struct Layout;

template <>
struct Layout<kModelXas> {
  static constexpr int kRegions = 3, kKp = X_KP, kKc = X_KC, kT0 = X_T0, kAnchor = X_ANCHOR, kT0Lo = X32_T0_LO,
                       kConstLo = X32_CONST_LO, kLinLo = X32_LIN_LO, kBigTerm = X_PH_RD + 2,
                       kBigTermLo = X32_RD_TERM_LO;
  __host__ __device__ static constexpr int const_slot(int r) { return xas_const_slot(r); }
  __host__ __device__ static constexpr int lin_slot(int r) { return xas_lin_slot(r); }
};

template <>
struct Layout<kModelPhenomD> {
  static constexpr int kRegions = 3, kKp = D_KP, kKc = D_KC, kT0 = D_T0, kAnchor = D_ANCHOR, kT0Lo = D32_T0_LO,
                       kConstLo = D32_CONST_LO, kLinLo = D32_LIN_LO, kBigTerm = D_PH_RD + 3,
                       kBigTermLo = D32_RD_TERM_LO;
  __host__ __device__ static constexpr int const_slot(int r) { return phd_const_slot(r); }
  __host__ __device__ static constexpr int lin_slot(int r) { return phd_lin_slot(r); }
};

template <>
struct Layout<kModelTaylorF2> {
  static constexpr int kRegions = 1, kKp = T_KP, kKc = T_KC, kT0 = T_T0, kAnchor = T_ANCHOR, kT0Lo = T32_T0_LO,
                       kConstLo = T32_CONST_LO, kLinLo = T32_LIN_LO, kBigTerm = -1, kBigTermLo = -1;
  __host__ __device__ static constexpr int const_slot(int r) { return tf2_const_slot(r); }
  __host__ __device__ static constexpr int lin_slot(int r) { return tf2_lin_slot(r); }
};

}  // namespace wfx
