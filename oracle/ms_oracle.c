/* ms_oracle.c - ORACLE (test infrastructure only): the bit-packed (multispin) lattice chain.
 *
 * Restates, one replica bit at a time and in site order, the chain the multispin kernel runs:
 * checkerboard Metropolis sweeps on a +-J cubic lattice (d = 2, 3, periodic, no field) with the
 * energy convention of drift/ising.py:50-53 and the acceptance rule of cuda/ising_pt.cu:117-118
 * (dE <= 0 accepted, else u < p(dE, beta)), exact energies recounted at each round end, per-replica
 * best tracking and the adjacent-rung exchange of drift/solvers/parallel_tempering.py:104-113.
 * Each replica bit b of word w at colour-split site q uses the full 32-bit uniform
 *   u_b = sum_{p=0..31} bit_b(plane_p) 2^(31-p),  plane_p = word (p & 3) of
 *   Philox4x32-10((q, t, (w << 8) | (p >> 2), 5 << 24 | instance), seed),
 * which the kernel evaluates bit-sliced and lazily; initial word = word 0 of
 * Philox((q, 0, w, 6 << 24 | instance), seed).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

void oracle_philox4x32_10(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4]);
double oracle_exp_neg_d(double x);

typedef struct MsOracle {
  int32_t dims, L, W;
  const uint8_t* jneg;   /* [N] colour-split order */
  const double* betas;   /* [R] */
  const uint32_t* thr;   /* [R][2d] */
  uint64_t seed;
  uint32_t instance;
  int32_t n_rounds, spr, init;
  int64_t round_offset;
  uint32_t* words;       /* [W][N] */
  uint32_t* best_words;  /* [W][N] */
  int64_t* energy;       /* [R] */
  int64_t* best_energy;  /* [R] */
  int32_t* rung_of_slot; /* [R] */
  int32_t* slot_of_rung; /* [R] */
  int64_t* tried;        /* [R-1] */
  int64_t* accepted;     /* [R-1] */
} MsOracle;

static int n_sites(const MsOracle* o) { return o->dims == 3 ? o->L * o->L * o->L : o->L * o->L; }

static int q_of(const MsOracle* o, int x, int y, int z) {
  int L = o->L, N = n_sites(o);
  x = (x + L) % L;
  y = (y + L) % L;
  z = o->dims == 3 ? (z + L) % L : 0;
  int c = (x + y + z) & 1;
  return c * (N / 2) + (x >> 1) + (L / 2) * (y + L * z);
}

static void coord_of(const MsOracle* o, int q, int* x, int* y, int* z) {
  int N = n_sites(o), half = o->L / 2;
  int c = q >= N / 2, h = q - c * (N / 2);
  int xh = h % half, rest = h / half;
  if (o->dims == 3) {
    *y = rest % o->L;
    *z = rest / o->L;
  } else {
    *y = rest;
    *z = 0;
  }
  *x = 2 * xh + ((*y + *z + c) & 1);
}

static int bit(uint32_t w, int b) { return (int)((w >> b) & 1u); }

/* unsatisfied bonds of replica bit b over every bond (positive direction of each site) */
static int64_t unsat_count(const MsOracle* o, int w, int b) {
  int N = n_sites(o);
  int64_t u = 0;
  for (int q = 0; q < N; ++q) {
    int x, y, z;
    coord_of(o, q, &x, &y, &z);
    int s = bit(o->words[(size_t)w * N + q], b);
    int nb[3] = {q_of(o, x + 1, y, z), q_of(o, x, y + 1, z), q_of(o, x, y, z + 1)};
    for (int d = 0; d < o->dims; ++d) u += s ^ bit(o->words[(size_t)w * N + nb[d]], b) ^ ((o->jneg[q] >> d) & 1);
  }
  return u;
}

static void energies(const MsOracle* o, int64_t* e) {
  int N = n_sites(o);
  for (int w = 0; w < o->W; ++w)
    for (int b = 0; b < 32; ++b) e[32 * w + b] = 2 * unsat_count(o, w, b) - (int64_t)o->dims * N;
}

int oracle_ms_run(MsOracle* o) {
  const int N = n_sites(o), R = 32 * o->W, d = o->dims, F = 2 * d;
  const uint32_t key[2] = {(uint32_t)(o->seed & 0xffffffffu), (uint32_t)(o->seed >> 32)};
  if (o->init) {
    for (int w = 0; w < o->W; ++w)
      for (int q = 0; q < N; ++q) {
        uint32_t ctr[4] = {(uint32_t)q, 0u, (uint32_t)w, (6u << 24) | o->instance}, out[4];
        oracle_philox4x32_10(ctr, key, out);
        o->words[(size_t)w * N + q] = out[0];
        o->best_words[(size_t)w * N + q] = out[0];
      }
    energies(o, o->energy);
    for (int r = 0; r < R; ++r) {
      o->best_energy[r] = o->energy[r];
      o->rung_of_slot[r] = r;
      o->slot_of_rung[r] = r;
      if (r < R - 1) o->tried[r] = o->accepted[r] = 0;
    }
  }
  for (int j = 0; j < o->n_rounds; ++j) {
    const int64_t round = o->round_offset + j;
    for (int sw = 0; sw < o->spr; ++sw) {
      const uint32_t t = (uint32_t)(round * o->spr + sw);
      for (int c = 0; c < 2; ++c)
        for (int h = 0; h < N / 2; ++h) {
          const int q = c * (N / 2) + h;
          int x, y, z;
          coord_of(o, q, &x, &y, &z);
          int nbq[6], nbd[6];
          nbq[0] = q_of(o, x + 1, y, z); nbd[0] = (o->jneg[q] >> 0) & 1;
          nbq[1] = q_of(o, x - 1, y, z); nbd[1] = (o->jneg[nbq[1]] >> 0) & 1;
          nbq[2] = q_of(o, x, y + 1, z); nbd[2] = (o->jneg[q] >> 1) & 1;
          nbq[3] = q_of(o, x, y - 1, z); nbd[3] = (o->jneg[nbq[3]] >> 1) & 1;
          nbq[4] = q_of(o, x, y, z + 1); nbd[4] = (o->jneg[q] >> 2) & 1;
          nbq[5] = q_of(o, x, y, z - 1); nbd[5] = (o->jneg[nbq[5]] >> 2) & 1;
          for (int w = 0; w < o->W; ++w) {
            uint32_t* wb = o->words + (size_t)w * N;
            uint32_t planes[32];
            for (int pc = 0; pc < 8; ++pc) {
              uint32_t ctr[4] = {(uint32_t)q, t, ((uint32_t)w << 8) | (uint32_t)pc, (5u << 24) | o->instance}, out[4];
              oracle_philox4x32_10(ctr, key, out);
              for (int i = 0; i < 4; ++i) planes[pc * 4 + i] = out[i];
            }
            uint32_t s = wb[q], nw = s;
            for (int b = 0; b < 32; ++b) {
              int k = 0;
              for (int e = 0; e < 2 * d; ++e) k += bit(s, b) ^ bit(wb[nbq[e]], b) ^ nbd[e];
              int flip;
              if (k >= d) {
                flip = 1;
              } else {
                uint32_t u = 0;
                for (int p = 0; p < 32; ++p) u |= (uint32_t)bit(planes[p], b) << (31 - p);
                const uint32_t th = o->thr[(size_t)o->rung_of_slot[32 * w + b] * F + 2 * (d - k) - 1];
                flip = u < th;
              }
              if (flip) nw ^= 1u << b;
            }
            wb[q] = nw;
          }
        }
    }
    energies(o, o->energy);
    for (int r = 0; r < R; ++r)
      if (o->energy[r] < o->best_energy[r]) {
        o->best_energy[r] = o->energy[r];
        const int w = r >> 5;
        const uint32_t m = 1u << (r & 31);
        for (int q = 0; q < N; ++q) {
          size_t i = (size_t)w * N + q;
          o->best_words[i] = (o->best_words[i] & ~m) | (o->words[i] & m);
        }
      }
    for (int r = (int)(round & 1); r + 1 < R; r += 2) {
      int a = o->slot_of_rung[r], b = o->slot_of_rung[r + 1];
      double delta = (o->betas[r] - o->betas[r + 1]) * (double)(o->energy[a] - o->energy[b]);
      int acc = delta >= 0.0;
      if (!acc) {
        uint32_t ctr[4] = {(uint32_t)r, (uint32_t)round, (uint32_t)((uint64_t)round >> 32), (4u << 24) | o->instance},
                 out[4];
        oracle_philox4x32_10(ctr, key, out);
        uint64_t m = ((uint64_t)(out[0] >> 5) << 26) | (uint64_t)(out[1] >> 6);
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
