/* pt_oracle.c - ORACLE (test infrastructure only; never part of the product path).
 *
 * A plain-C CPU restatement of the parallel-tempering path that the CUDA engine implements, used
 * by the tests as the checker, by smoke() as the checker and by bench.py as the timed CPU
 * baseline. It is written independently of drift_b200/csrc (own Philox, own exp, own colouring,
 * spins kept in the original site numbering, CSR instead of ELL) and follows the reference:
 *
 *   - energy convention E = -1/2 s.J.s - h.s and dE_i = 2 s_i (J_i.s + h_i):
 *       drift/ising.py:50-53, 63-68
 *   - colour-ordered Metropolis sweep over CSR, local field h_i + sum_t w_t s_col(t), accept if
 *     dE <= 0 or u < p(dE, beta), incremental energy from the accepted dE:
 *       cuda/ising_pt.cu:109-122, 126-135
 *   - exchange of adjacent rungs (r, r+1) with parity = round % 2, accept if
 *     delta = (beta_r - beta_{r+1})(E_r - E_{r+1}) >= 0 or u < exp(delta), configurations (here:
 *     rung labels) swapped on accept, tried/accepted counted:
 *       drift/solvers/parallel_tempering.py:104-113
 *   - best-so-far tracking at round ends and per-round best history:
 *       drift/solvers/parallel_tempering.py:79-82, 99-102, 115
 *   - greedy colouring in index order and its stable colour order:
 *       drift/gpu.py:122-145
 *
 * The engine's own definitions that the reference leaves open (which uniform feeds which attempt,
 * the integer acceptance threshold, the fixed-point energy of the fp32 path) are restated from
 * their specification: Philox4x32-10 (Salmon et al., SC'11) under the counter layout
 *   sweep  (p>>3, t, slot, 1<<24|inst) half (p&1) of word ((p>>1)&3) = high 16 bits of u
 *   second (p, t, slot, 2<<24|inst)    low 16 bits of word 0        = low 16 bits of u
 *   init   (p>>2, 0, slot, 3<<24|inst) bit 31 of word (p&3) set     = spin -1
 *   swap   (r, round lo, round hi, 4<<24|inst) words 0,1            = 53-bit uniform
 * where p is the position of the spin in colour order and t = round * sweeps_per_round + j.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

/* ------------------------------------------------------------------------------------------ */
/* Philox4x32-10                                                                              */
/* ------------------------------------------------------------------------------------------ */
void oracle_philox4x32_10(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4]) {
  uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
  uint32_t k0 = key_in[0], k1 = key_in[1];
  for (int round = 0; round < 10; ++round) {
    if (round > 0) {
      k0 += 0x9E3779B9u;
      k1 += 0xBB67AE85u;
    }
    uint64_t p0 = (uint64_t)0xD2511F53u * c0;
    uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
    uint32_t n0 = (uint32_t)(p1 >> 32) ^ c1 ^ k0;
    uint32_t n1 = (uint32_t)p1;
    uint32_t n2 = (uint32_t)(p0 >> 32) ^ c3 ^ k1;
    uint32_t n3 = (uint32_t)p0;
    c0 = n0; c1 = n1; c2 = n2; c3 = n3;
  }
  out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

static void philox_w(uint32_t a, uint32_t b, uint32_t c, uint32_t d, uint32_t k0, uint32_t k1, uint32_t o[4]) {
  uint32_t ctr[4] = {a, b, c, d}, key[2] = {k0, k1};
  oracle_philox4x32_10(ctr, key, o);
}

/* ------------------------------------------------------------------------------------------ */
/* exp(x), x <= 0: x = n ln2 + r, e^r by its Taylor series (Horner, fused multiply-add),        */
/* result scaled by 2^n. Compiled with -ffp-contract=off so every other operation rounds once. */
/* ------------------------------------------------------------------------------------------ */
/* 1/k! as the correctly rounded double / float of the exact rational (hex literals of the rounded
 * values; 1/0! = 1/1! = 1, 1/2! = 0.5 are exact). Constant tables: the replicas call the
 * exponentials from several threads at once, so nothing here is initialised at run time. */
static const double taylor_inv_fact_d[14] = {1.0, 1.0, 0.5, 0x1.5555555555555p-3, 0x1.5555555555555p-5,
                                             0x1.1111111111111p-7, 0x1.6c16c16c16c17p-10, 0x1.a01a01a01a01ap-13,
                                             0x1.a01a01a01a01ap-16, 0x1.71de3a556c734p-19, 0x1.27e4fb7789f5cp-22,
                                             0x1.ae64567f544e4p-26, 0x1.1eed8eff8d898p-29, 0x1.6124613a86d09p-33};
static const float taylor_inv_fact_f[8] = {1.0f, 1.0f, 0.5f, 0x1.555556p-3f, 0x1.555556p-5f, 0x1.111112p-7f,
                                           0x1.6c16c2p-10f, 0x1.a01a02p-13f};

double oracle_exp_neg_d(double x) {
  if (!(x <= 0.0)) return 1.0;
  if (x < -708.0) return 0.0;
  double n = rint(x * 0x1.71547652b82fep+0);
  double r = fma(-n, 0x1.62e42p-1, x);      /* high part of ln 2 (21 significant bits) */
  r = fma(-n, 0x1.fdf473de6af28p-22, r);     /* ln 2 minus the high part               */
  double p = taylor_inv_fact_d[13];
  for (int k = 12; k >= 0; --k) p = fma(p, r, taylor_inv_fact_d[k]);
  uint64_t bits = (uint64_t)((int)n + 1023) << 52;
  double scale;
  memcpy(&scale, &bits, sizeof scale);
  return p * scale;
}

float oracle_exp_neg_f(float x) {
  if (!(x <= 0.0f)) return 1.0f;
  if (x < -87.0f) return 0.0f;
  float n = rintf(x * 0x1.715476p+0f);
  float r = fmaf(-n, 0x1.62ep-1f, x);
  r = fmaf(-n, 0x1.0bfbe8p-15f, r);
  float p = taylor_inv_fact_f[7];
  for (int k = 6; k >= 0; --k) p = fmaf(p, r, taylor_inv_fact_f[k]);
  uint32_t bits = (uint32_t)((int)n + 127) << 23;
  float scale;
  memcpy(&scale, &bits, sizeof scale);
  return p * scale;
}

/* Integer-path threshold floor(exp(-2 x beta) 2^32), saturated (the table the engine receives). */
uint32_t oracle_threshold_int(double beta, int x) {
  double e = oracle_exp_neg_d((-2.0 * beta) * (double)x);
  double v = e * 4294967296.0;
  if (v >= 4294967295.0) return 0xFFFFFFFFu;
  return (uint32_t)v;
}

static uint32_t threshold_float(float neg2beta, float x) {
  float e = oracle_exp_neg_f(neg2beta * x);
  float v = e * 4294967296.0f;
  if (v >= 4294967296.0f) return 0xFFFFFFFFu;
  return (uint32_t)v;
}

/* ------------------------------------------------------------------------------------------ */
/* Greedy colouring (drift/gpu.py:122-145)                                                     */
/* ------------------------------------------------------------------------------------------ */
int oracle_greedy_coloring(int n, const int32_t* row_ptr, const int32_t* col_idx, int32_t* color,
                           int32_t* color_ptr_out, int32_t* color_spins_out) {
  for (int i = 0; i < n; ++i) color[i] = -1;
  int kmax = 0;
  char* used = (char*)calloc((size_t)n + 2, 1);
  for (int i = 0; i < n; ++i) {
    for (int t = row_ptr[i]; t < row_ptr[i + 1]; ++t) {
      int c = color[col_idx[t]];
      if (c >= 0) used[c] = 1;
    }
    int c = 0;
    while (used[c]) ++c;
    color[i] = c;
    if (c + 1 > kmax) kmax = c + 1;
    for (int t = row_ptr[i]; t < row_ptr[i + 1]; ++t) {
      int cc = color[col_idx[t]];
      if (cc >= 0) used[cc] = 0;
    }
  }
  free(used);
  int k = n > 0 ? kmax : 1;
  if (color_ptr_out && color_spins_out) {
    /* stable argsort by colour */
    int pos = 0;
    for (int c = 0; c < k; ++c) {
      color_ptr_out[c] = pos;
      for (int i = 0; i < n; ++i)
        if (color[i] == c) color_spins_out[pos++] = i;
    }
    color_ptr_out[k] = pos;
  }
  return k;
}

/* ------------------------------------------------------------------------------------------ */
/* Parallel tempering                                                                          */
/* ------------------------------------------------------------------------------------------ */
typedef struct OracleProblem {
  int32_t n;
  const int32_t* row_ptr;
  const int32_t* col_idx;
  const float* weight;  /* fp32 couplings (the reference casts J to float32, drift/gpu.py:74) */
  const float* h;
  int32_t n_colors;
  const int32_t* color_ptr;
  const int32_t* color_spins;
  int32_t integer_path;      /* 1: integer couplings, threshold table                         */
  int32_t max_field;         /* F                                                             */
} OracleProblem;

typedef struct OracleRun {
  int32_t R, n_rounds, sweeps_per_round, threads;
  int64_t round_offset;
  uint64_t seed;
  uint32_t instance;
  const double* betas;       /* [R] by rung                                                   */
  const uint32_t* thr;       /* [R][F] integer path                                           */
  int32_t init;              /* 1: draw initial spins and energies                            */
} OracleRun;

typedef struct OracleState {  /* all per slot, spins in site order */
  int8_t* spins;             /* [R][n] */
  int64_t* energy;           /* [R] fixed point */
  int64_t* best_energy;      /* [R] */
  int8_t* best_spins;        /* [R][n] */
  int32_t* rung_of_slot;     /* [R] */
  int32_t* slot_of_rung;     /* [R] */
  int64_t* tried;            /* [R-1] */
  int64_t* accepted;         /* [R-1] */
  double* best_history;      /* [n_rounds] or NULL */
} OracleState;

static int64_t energy_fixed(const OracleProblem* P, const int8_t* s) {
  if (P->integer_path) {
    int64_t twice = 0;
    for (int i = 0; i < P->n; ++i) {
      int64_t f = 0;
      for (int t = P->row_ptr[i]; t < P->row_ptr[i + 1]; ++t) f += (int64_t)P->weight[t] * s[P->col_idx[t]];
      twice += (int64_t)s[i] * (-f - 2 * (int64_t)P->h[i]);
    }
    return twice / 2;
  }
  int64_t acc = 0;
  for (int i = 0; i < P->n; ++i) {
    float f = 0.0f;
    for (int t = P->row_ptr[i]; t < P->row_ptr[i + 1]; ++t) {
      float w = P->weight[t];
      f = f + (s[P->col_idx[t]] > 0 ? w : -w);
    }
    float term = (-0.5f * f) - P->h[i];
    if (s[i] < 0) term = -term;
    acc += llrintf(term * 4294967296.0f);
  }
  return acc;
}

/* One sweep of slot `slot` at sweep index t; returns the fixed-point energy change. */
static int64_t sweep_slot(const OracleProblem* P, const OracleRun* A, int slot, int rung, uint32_t t, int8_t* s) {
  const uint32_t k0 = (uint32_t)(A->seed & 0xffffffffu), k1 = (uint32_t)(A->seed >> 32);
  const uint32_t c_sweep = (1u << 24) | A->instance, c_second = (2u << 24) | A->instance;
  const float neg2beta = -2.0f * (float)A->betas[rung];
  int64_t dsum = 0;
  for (int c = 0; c < P->n_colors; ++c) {
    for (int p = P->color_ptr[c]; p < P->color_ptr[c + 1]; ++p) {
      const int i = P->color_spins[p];
      uint32_t thr = 0;
      int64_t dE;
      int accept;
      if (P->integer_path) {
        int64_t field = (int64_t)P->h[i];
        for (int tt = P->row_ptr[i]; tt < P->row_ptr[i + 1]; ++tt) field += (int64_t)P->weight[tt] * s[P->col_idx[tt]];
        int64_t x = (int64_t)s[i] * field;
        dE = 2 * x;
        accept = (x <= 0);
        if (!accept) thr = A->thr[(int64_t)rung * P->max_field + (x > P->max_field ? P->max_field : x) - 1];
      } else {
        float field = P->h[i];
        for (int tt = P->row_ptr[i]; tt < P->row_ptr[i + 1]; ++tt) {
          float w = P->weight[tt];
          field = field + (s[P->col_idx[tt]] > 0 ? w : -w);
        }
        float x = s[i] > 0 ? field : -field;
        dE = llrintf(x * 8589934592.0f);
        accept = !(x > 0.0f);
        if (!accept) thr = threshold_float(neg2beta, x);
      }
      if (!accept) {
        uint32_t w[4], w2[4];
        philox_w((uint32_t)(p >> 3), t, (uint32_t)slot, c_sweep, k0, k1, w);
        uint32_t word = w[(p >> 1) & 3];
        uint32_t prim = (p & 1) ? (word >> 16) : (word & 0xFFFFu);
        uint32_t u = prim << 16;
        if (prim == (thr >> 16)) {
          philox_w((uint32_t)p, t, (uint32_t)slot, c_second, k0, k1, w2);
          u |= w2[0] & 0xFFFFu;
        }
        accept = u < thr;  /* when prim != thr >> 16 the low half cannot change the outcome */
      }
      if (accept) {
        s[i] = (int8_t)-s[i];
        dsum += dE;
      }
    }
  }
  return dsum;
}

int oracle_pt_run(const OracleProblem* P, const OracleRun* A, OracleState* S) {
  const int n = P->n, R = A->R;
  const uint32_t k0 = (uint32_t)(A->seed & 0xffffffffu), k1 = (uint32_t)(A->seed >> 32);
  if (n < 1 || R < 1 || A->sweeps_per_round < 1 || A->n_rounds < 0) return 1;
#ifdef _OPENMP
  if (A->threads > 0) omp_set_num_threads(A->threads);
#endif
  if (A->init) {
#pragma omp parallel for schedule(static)
    for (int slot = 0; slot < R; ++slot) {
      int8_t* s = S->spins + (size_t)slot * n;
      for (int p = 0; p < n; ++p) {
        uint32_t w[4];
        philox_w((uint32_t)(p >> 2), 0u, (uint32_t)slot, (3u << 24) | A->instance, k0, k1, w);
        s[P->color_spins[p]] = (w[p & 3] >> 31) ? (int8_t)-1 : (int8_t)1;
      }
      S->energy[slot] = energy_fixed(P, s);
      S->best_energy[slot] = S->energy[slot];
      memcpy(S->best_spins + (size_t)slot * n, s, (size_t)n);
      S->rung_of_slot[slot] = slot;
      S->slot_of_rung[slot] = slot;
      if (slot < R - 1) {
        S->tried[slot] = 0;
        S->accepted[slot] = 0;
      }
    }
  }
  const double scale = P->integer_path ? 1.0 : 0x1.0p-32;
  int64_t run_best = S->best_energy[0];
  for (int r = 1; r < R; ++r)
    if (S->best_energy[r] < run_best) run_best = S->best_energy[r];
  for (int j = 0; j < A->n_rounds; ++j) {
    const int64_t round = A->round_offset + j;
#pragma omp parallel for schedule(dynamic, 1)
    for (int slot = 0; slot < R; ++slot) {
      int8_t* s = S->spins + (size_t)slot * n;
      const int rung = S->rung_of_slot[slot];
      int64_t d = 0;
      for (int sw = 0; sw < A->sweeps_per_round; ++sw) {
        uint32_t t = (uint32_t)(round * A->sweeps_per_round + sw);
        d += sweep_slot(P, A, slot, rung, t, s);
      }
      S->energy[slot] += d;
      if (S->energy[slot] < S->best_energy[slot]) {
        S->best_energy[slot] = S->energy[slot];
        memcpy(S->best_spins + (size_t)slot * n, s, (size_t)n);
      }
    }
    for (int slot = 0; slot < R; ++slot)
      if (S->energy[slot] < run_best) run_best = S->energy[slot];
    if (S->best_history) S->best_history[j] = (double)run_best * scale;
    /* exchange step (drift/solvers/parallel_tempering.py:106-113) */
    for (int r = (int)(round & 1); r + 1 < R; r += 2) {
      int a = S->slot_of_rung[r], b = S->slot_of_rung[r + 1];
      double dE = P->integer_path ? (double)(S->energy[a] - S->energy[b])
                                  : (double)(S->energy[a] - S->energy[b]) * 0x1.0p-32;
      double delta = (A->betas[r] - A->betas[r + 1]) * dE;
      int accept = delta >= 0.0;
      if (!accept) {
        uint32_t w[4];
        philox_w((uint32_t)r, (uint32_t)round, (uint32_t)((uint64_t)round >> 32), (4u << 24) | A->instance, k0, k1, w);
        uint64_t m = ((uint64_t)(w[0] >> 5) << 26) | (uint64_t)(w[1] >> 6);
        double u = (double)m * 0x1.0p-53;
        accept = u < oracle_exp_neg_d(delta);
      }
      S->tried[r] += 1;
      if (accept) {
        S->accepted[r] += 1;
        S->slot_of_rung[r] = b;
        S->slot_of_rung[r + 1] = a;
        S->rung_of_slot[a] = r + 1;
        S->rung_of_slot[b] = r;
      }
    }
  }
  return 0;
}

/* FP64 energy of one configuration from the CSR (drift/ising.py:50-53). */
double oracle_energy_fp64(const OracleProblem* P, const int8_t* s) {
  double E = 0.0;
  for (int i = 0; i < P->n; ++i) {
    double f = 0.0;
    for (int t = P->row_ptr[i]; t < P->row_ptr[i + 1]; ++t) f += (double)P->weight[t] * s[P->col_idx[t]];
    E += -0.5 * s[i] * f - (double)P->h[i] * s[i];
  }
  return E;
}
