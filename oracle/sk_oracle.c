/* sk_oracle.c - ORACLE (test infrastructure only): the dense-coupling (SK) chain.
 *
 * Restates, one attempt at a time, the chain the dense-coupling engine runs on fixed-point
 * couplings Jq (int32, symmetric, zero diagonal) and field hq:
 *   - sweep order: spins 0..n-1 in index order (cuda/ising_pt.cu:109-122 with every spin its own
 *     colour class, which is what drift/gpu.py:122-145 gives a complete graph);
 *   - energy change of flipping i: dE = 2 s_i F_i with F_i = sum_j J_ij s_j + h_i
 *     (drift/ising.py:63-68); here in units of 2^-shift, F exact in integers;
 *   - acceptance: flip iff s_i F_i <= D, D = floor(-ln(u) c_rung) (c = 2^shift / (2 beta) as a
 *     float), i.e. u <= exp(-beta dE), the Metropolis rule of cuda/ising_pt.cu:117-118;
 *     u = (2 (w >> 9) + 1) 2^-24, w = word ((i >> 5) & 3) of
 *     Philox4x32-10((((i >> 7) << 5) | (i & 31), t, slot, 7 << 24 | instance), seed);
 *   - -ln(u): u = m 2^e, m in (sqrt(2)/2, sqrt(2)], z = (m-1)/(m+1),
 *     ln m = 2 z (1 + z^2/3 + z^4/5 + z^6/7 + z^8/9), every operation rounded once in float;
 *   - energies: E2 = -sum_i s_i (sum_j Jq_ij s_j + 2 hq_i), exact int64 (E = E2 2^-(shift+1));
 *   - rounds: per-replica best at round ends, then the adjacent-rung exchange of
 *     drift/solvers/parallel_tempering.py:104-113 with alternating parity.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

void oracle_philox4x32_10(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4]);
double oracle_exp_neg_d(double x);

float oracle_neg_log_unit(float u) {
  uint32_t bits;
  memcpy(&bits, &u, sizeof bits);
  int e = (int)(bits >> 23) - 127;
  uint32_t mb = (bits & 0x007FFFFFu) | 0x3F800000u;
  if (mb > 0x3FB504F3u) { /* mantissa above sqrt(2): use m / 2 */
    mb -= 0x00800000u;
    e += 1;
  }
  float m;
  memcpy(&m, &mb, sizeof m);
  const float z = (m - 1.0f) / (m + 1.0f);
  const float w = z * z;
  /* 1/9, 1/7, 1/5, 1/3 rounded to float */
  float p = fmaf(w, 0x1.c71c72p-4f, 0x1.24924ap-3f);
  p = fmaf(w, p, 0x1.99999ap-3f);
  p = fmaf(w, p, 0x1.555556p-2f);
  p = fmaf(w, p, 1.0f);
  const float lnm = (z + z) * p;
  const float r = -fmaf((float)e, 0x1.62e430p-1f, lnm);
  return r > 0.0f ? r : 0.0f;
}

int32_t oracle_sk_threshold(uint32_t word, float c) {
  const float u = (float)(2u * (word >> 9) + 1u) * 0x1.0p-24f;
  const float v = oracle_neg_log_unit(u) * c;
  if (v >= 2147483648.0f) return 2147483647;
  return (int32_t)v;
}

typedef struct SkOracle {
  int32_t n, R, n_rounds, spr, init, threads;
  const int32_t* Jq;      /* [n][n] */
  const int32_t* hq;      /* [n] */
  const double* betas;    /* [R] */
  const float* scales;    /* [R] */
  double escale;          /* 2^-(shift+1) */
  uint64_t seed;
  uint32_t instance;
  int32_t reserved;
  int64_t round_offset;
  int8_t* spins;          /* [R][n] */
  int8_t* best_spins;     /* [R][n] */
  int64_t* energy;        /* [R] E2 */
  int64_t* best_energy;   /* [R] */
  int32_t* rung_of_slot;  /* [R] */
  int32_t* slot_of_rung;  /* [R] */
  int64_t* tried;         /* [R] (first R-1 used) */
  int64_t* accepted;      /* [R] */
  int64_t* best_history;  /* [n_rounds] or NULL */
} SkOracle;

static int64_t field(const SkOracle* o, const int8_t* s, int i) {
  int64_t f = o->hq[i];
  const int32_t* row = o->Jq + (size_t)i * o->n;
  for (int j = 0; j < o->n; ++j) f += (int64_t)row[j] * s[j];
  return f;
}

int64_t oracle_sk_energy(int32_t n, const int32_t* Jq, const int32_t* hq, const int8_t* s) {
  int64_t e = 0;
  for (int i = 0; i < n; ++i) {
    int64_t a = 0;
    for (int j = 0; j < n; ++j) a += (int64_t)Jq[(size_t)i * n + j] * s[j];
    e -= (int64_t)s[i] * (a + 2 * (int64_t)hq[i]);
  }
  return e;
}

/* one sweep of one slot; F holds the exact local fields of s and is kept up to date */
static int64_t sweep(const SkOracle* o, int slot, float c, uint32_t t, int8_t* s, int64_t* F) {
  const int n = o->n;
  const uint32_t key[2] = {(uint32_t)(o->seed & 0xffffffffu), (uint32_t)(o->seed >> 32)};
  int64_t de = 0;
  for (int i = 0; i < n; ++i) {
    const uint32_t ctr[4] = {((uint32_t)(i >> 7) << 5) | (uint32_t)(i & 31), t, (uint32_t)slot,
                             (7u << 24) | o->instance};
    uint32_t w[4];
    oracle_philox4x32_10(ctr, key, w);
    const int32_t D = oracle_sk_threshold(w[(i >> 5) & 3], c);
    const int64_t v = (int64_t)s[i] * F[i];
    if (v <= (int64_t)D) {
      de += 4 * v;
      const int64_t d = -2 * (int64_t)s[i]; /* s_new - s_old */
      s[i] = (int8_t)-s[i];
      for (int j = 0; j < n; ++j) F[j] += (int64_t)o->Jq[(size_t)j * n + i] * d;
    }
  }
  return de;
}

int oracle_sk_run(SkOracle* o) {
  const int n = o->n, R = o->R;
  if (n < 1 || R < 1 || o->spr < 1 || o->n_rounds < 0) return 1;
  const uint32_t key[2] = {(uint32_t)(o->seed & 0xffffffffu), (uint32_t)(o->seed >> 32)};
#ifdef _OPENMP
  if (o->threads > 0) omp_set_num_threads(o->threads);
#endif
  if (o->init) {
#pragma omp parallel for schedule(static)
    for (int slot = 0; slot < R; ++slot) {
      int8_t* s = o->spins + (size_t)slot * n;
      for (int i = 0; i < n; ++i) {
        const uint32_t ctr[4] = {(uint32_t)(i >> 2), 0u, (uint32_t)slot, (3u << 24) | o->instance};
        uint32_t w[4];
        oracle_philox4x32_10(ctr, key, w);
        s[i] = (w[i & 3] >> 31) ? (int8_t)-1 : (int8_t)1;
      }
      o->energy[slot] = oracle_sk_energy(n, o->Jq, o->hq, s);
      o->best_energy[slot] = o->energy[slot];
      memcpy(o->best_spins + (size_t)slot * n, s, (size_t)n);
      o->rung_of_slot[slot] = slot;
      o->slot_of_rung[slot] = slot;
      o->tried[slot] = 0;
      o->accepted[slot] = 0;
    }
  }
  int64_t run_best = o->best_energy[0];
  for (int r = 1; r < R; ++r)
    if (o->best_energy[r] < run_best) run_best = o->best_energy[r];
  for (int j = 0; j < o->n_rounds; ++j) {
    const int64_t round = o->round_offset + j;
#pragma omp parallel for schedule(dynamic, 1)
    for (int slot = 0; slot < R; ++slot) {
      int8_t* s = o->spins + (size_t)slot * n;
      int64_t* F = (int64_t*)malloc(sizeof(int64_t) * (size_t)n);
      for (int i = 0; i < n; ++i) F[i] = field(o, s, i);
      const float c = o->scales[o->rung_of_slot[slot]];
      int64_t d = 0;
      for (int sw = 0; sw < o->spr; ++sw) d += sweep(o, slot, c, (uint32_t)(round * o->spr + sw), s, F);
      free(F);
      o->energy[slot] += d;
      if (o->energy[slot] < o->best_energy[slot]) {
        o->best_energy[slot] = o->energy[slot];
        memcpy(o->best_spins + (size_t)slot * n, s, (size_t)n);
      }
    }
    for (int slot = 0; slot < R; ++slot)
      if (o->energy[slot] < run_best) run_best = o->energy[slot];
    if (o->best_history) o->best_history[j] = run_best;
    for (int r = (int)(round & 1); r + 1 < R; r += 2) {
      const int a = o->slot_of_rung[r], b = o->slot_of_rung[r + 1];
      const double dE = (double)(o->energy[a] - o->energy[b]) * o->escale;
      const double delta = (o->betas[r] - o->betas[r + 1]) * dE;
      int acc = delta >= 0.0;
      if (!acc) {
        const uint32_t ctr[4] = {(uint32_t)r, (uint32_t)round, (uint32_t)((uint64_t)round >> 32),
                                 (4u << 24) | o->instance};
        uint32_t w[4];
        oracle_philox4x32_10(ctr, key, w);
        const uint64_t m = ((uint64_t)(w[0] >> 5) << 26) | (uint64_t)(w[1] >> 6);
        acc = (double)m * 0x1.0p-53 < oracle_exp_neg_d(delta);
      }
      o->tried[r] += 1;
      if (acc) {
        o->accepted[r] += 1;
        o->slot_of_rung[r] = b;
        o->slot_of_rung[r + 1] = a;
        o->rung_of_slot[a] = r + 1;
        o->rung_of_slot[b] = r;
      }
    }
  }
  return 0;
}
