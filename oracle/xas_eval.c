/*
 * The oracle's IMRPhenomXAS waveform at the frequencies, in plain C with
 * POSIX threads over binaries: a restatement of oracle/xas.py's frequency_powers,
 * phase_basis, phase_rest, amplitude_phase, reduce and evaluate, which
 * follow the reference's models/xas/core.py:382-507.
 *
 * TEST INFRASTRUCTURE ONLY: the tests check it against the golden vectors
 * (the reference's own tables and waveforms), and bench.py times it as the
 * CPU baseline and the reference arm. The product never links or calls it.
 *
 * Input: one row per binary of the reference's flat table (86 doubles,
 * models/xas/core.py:68-89; oracle/xas.py's LAYOUT and flat()).
 * Build: oracle/Makefile (gcc -O3 -pthread -ffp-contract=off, so that every
 * product and sum rounds as NumPy's float64 does).
 */
#include <math.h>
#include <pthread.h>
#include <stdatomic.h>
#include <stdint.h>
#include <stdlib.h>
#include <unistd.h>

/* the flat table's slots (models/xas/core.py:68-89) */
enum {
  PHASE = 0, /* 3 regions x 16 basis terms */
  T0 = 48,
  ANCHOR = 49,
  ATAN_A = 52,
  ATAN_W = 55,
  SHIFT = 58,
  AMP_INS = 59,
  AMP_INT_N = 69,
  AMP_INT_D = 70,
  AMP_RD_N = 75,
  AMP_RD_GR = 76,
  AMP_RD_S = 77,
  AMP_RD_G = 78,
  F_PHASE_IN = 79,
  F_PHASE_IM = 80,
  F_AMP_IN = 81,
  F_AMP_RD = 82,
  F_CUT = 83,
  KP = 84,
  KC = 85,
  STRIDE = 86
};
enum { CONST = 5, NBASIS = 16 };

/* the terms of each phase region (models/xas/core.py:409-415): the
 * inspiral's 1..13 (CONST among them, whose basis value is the constant
 * itself), the intermediate's f, log f, 1/f, f^-2, f^-3, 1 and the
 * ringdown's f, f^2/3, 1/f, f^-3, 1 */
static const int kInspiral[] = {1, 2, 3, 4, 6, 7, 8, 9, 10, 11, 12, 13};
static const int kIntermediate[] = {9, 4, 1, 14, 15};
static const int kRingdown[] = {9, 8, 1, 15};

typedef struct {
  double f, t, m1, lf, m76, f53;
  double basis[NBASIS];
} powers_t;

/* frequency_powers and phase_basis (models/xas/core.py:382-403) */
static void frequency_powers(double f, powers_t* p) {
  p->f = f;
  p->m1 = 1.0 / f;
  p->lf = log(f);
  const double t0 = exp(p->lf / 3.0);
  p->t = t0 * (4.0 - t0 * t0 * t0 * p->m1) / 3.0;
  p->m76 = p->m1 / sqrt(p->t);
  p->f53 = exp(-5.0 / 3.0 * p->lf);
  const double t = p->t, t2 = t * t, mt1 = t2 * p->m1, mt2 = mt1 * mt1, m2 = p->m1 * p->m1;
  double* b = p->basis;
  b[0] = p->m1 * mt2;
  b[1] = p->m1;
  b[2] = mt2;
  b[3] = mt1;
  b[4] = p->lf;
  b[5] = 1.0; /* (the constant: never multiplied) */
  b[6] = t;
  b[7] = t * p->lf;
  b[8] = t2;
  b[9] = f;
  b[10] = f * p->lf;
  b[11] = f * t;
  b[12] = f * t2;
  b[13] = f * f;
  b[14] = m2;
  b[15] = m2 * p->m1;
}

static double region_sum(const double* row, const int* terms, int count, const double* basis) {
  double total = row[CONST];
  for (int i = 0; i < count; ++i) total = total + row[terms[i]] * basis[terms[i]];
  return total;
}

/* amplitude_phase, reduce and evaluate at one frequency */
static void point(const double* T, const powers_t* p, double* hp, double* hc) {
  const double f = p->f;
  const int past = f >= T[F_PHASE_IN];
  const int ring = f > T[F_PHASE_IM];
  double rest;
  if (ring) {
    rest = region_sum(T + PHASE + 2 * NBASIS, kRingdown, 4, p->basis);
  } else if (past) {
    rest = region_sum(T + PHASE + NBASIS, kIntermediate, 5, p->basis);
  } else {
    rest = region_sum(T + PHASE, kInspiral, 12, p->basis);
  }
  if (past) {
    const double a = ring ? T[ATAN_A + 2] : T[ATAN_A + 1];
    const double w = ring ? T[ATAN_W + 2] : T[ATAN_W + 1];
    rest = rest + a * atan(w * (f - T[SHIFT]));
  } else {
    rest = rest + 0.0;
  }
  double phi = (past ? 0.0 : T[T0] * p->f53) + rest;
  phi = phi - T[ANCHOR];
  double amp;
  if (f > T[F_AMP_RD]) {
    const double u = T[AMP_RD_S] * (f - T[SHIFT]);
    amp = T[AMP_RD_N] * p->m76 * exp(-T[AMP_RD_GR] * u) / (u * u + T[AMP_RD_G]);
  } else if (f >= T[F_AMP_IN]) {
    double den = T[AMP_INT_D + 4];
    for (int j = 3; j >= 0; --j) den = den * f + T[AMP_INT_D + j];
    amp = T[AMP_INT_N] / den;
  } else {
    double poly = T[AMP_INS + 9];
    for (int k = 8; k >= 0; --k) poly = poly * p->t + T[AMP_INS + k];
    amp = p->m76 * poly;
  }
  if (!(f <= T[F_CUT])) amp = 0.0;
  const double two_pi = 2.0 * 3.141592653589793;
  phi = phi - nearbyint(phi / two_pi) * two_pi;
  const double c = cos(phi), s = sin(phi);
  const double ap = T[KP] * amp, ac = T[KC] * amp;
  hp[0] = ap * c;
  hp[1] = ap * s;
  hc[0] = -ac * s;
  hc[1] = ac * c;
}

typedef struct {
  const double* table;
  int64_t B, N, f_stride;
  const double* freqs;
  powers_t* shared;
  double *hp, *hc;
  atomic_llong next; /* the next chunk of binaries (or of frequencies, for the shared powers) */
  int stage;         /* 0: the shared powers, 1: the waveforms */
} job_t;

enum { CHUNK = 4, POWER_CHUNK = 256 };

static void* worker(void* arg) {
  job_t* job = (job_t*)arg;
  for (;;) {
    if (job->stage == 0) {
      const int64_t k0 = atomic_fetch_add(&job->next, POWER_CHUNK);
      if (k0 >= job->N) return NULL;
      const int64_t k1 = k0 + POWER_CHUNK < job->N ? k0 + POWER_CHUNK : job->N;
      for (int64_t k = k0; k < k1; ++k) frequency_powers(job->freqs[k], &job->shared[k]);
      continue;
    }
    const int64_t b0 = atomic_fetch_add(&job->next, CHUNK);
    if (b0 >= job->B) return NULL;
    const int64_t b1 = b0 + CHUNK < job->B ? b0 + CHUNK : job->B;
    for (int64_t b = b0; b < b1; ++b) {
      const double* T = job->table + b * STRIDE;
      for (int64_t k = 0; k < job->N; ++k) {
        powers_t local;
        const powers_t* p = job->shared ? &job->shared[k] : &local;
        if (!job->shared) frequency_powers(job->freqs[b * job->f_stride + k], &local);
        const int64_t e = 2 * (b * job->N + k);
        point(T, p, job->hp + e, job->hc + e);
      }
    }
  }
}

static int run(job_t* job, int threads) {
  pthread_t ids[512];
  if (threads > 512) threads = 512;
  int started = 0;
  for (int i = 1; i < threads; ++i) {
    if (pthread_create(&ids[started], NULL, worker, job) == 0) ++started;
  }
  worker(job);
  for (int i = 0; i < started; ++i) pthread_join(ids[i], NULL);
  return 0;
}

/*
 * (hplus, hcross) of B binaries: hp, hc are B x N complex128 (interleaved
 * re, im). freqs: N values shared by every binary (f_stride 0; their powers
 * computed once, as jax.vmap with the grid unbatched computes them once),
 * or one row of N per binary (f_stride N). threads: the threads to use
 * (<= 0: every online core). Returns 0, or -1 if memory ran out.
 */
int oracle_xas_evaluate(const double* table, int64_t B, const double* freqs, int64_t N, int64_t f_stride,
                        double* hp, double* hc, int threads) {
  if (threads <= 0) threads = (int)sysconf(_SC_NPROCESSORS_ONLN);
  if (threads < 1) threads = 1;
  job_t job = {table, B, N, f_stride, freqs, NULL, hp, hc, 0, 0};
  if (f_stride == 0) {
    job.shared = (powers_t*)malloc(sizeof(powers_t) * (size_t)(N > 0 ? N : 1));
    if (job.shared == NULL) return -1;
    run(&job, threads);
  }
  atomic_store(&job.next, 0);
  job.stage = 1;
  run(&job, threads);
  free(job.shared);
  return 0;
}
