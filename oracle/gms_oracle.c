/* gms_oracle.c - ORACLE (test infrastructure only): the bit-packed chain on a +-1 graph.
 *
 * Restates, one replica bit at a time, the chain of the graph multispin kernel: the colour-ordered
 * sweep of cuda/ising_pt.cu:109-122 over positions (colour classes in order, any order inside a
 * class), dE = 2 s_i sum_j J_ij s_j = 2 (deg - 2k) for k unsatisfied bonds (drift/ising.py:63-68),
 * accept iff deg - 2k <= 0 or u < thr[rung][deg - 2k - 1] (cuda/ising_pt.cu:117-118 with the
 * integer threshold table), exact energies E = 2U - bonds recounted at round ends, per-replica
 * best, and the adjacent-rung exchange of drift/solvers/parallel_tempering.py:104-113.
 * Replica bit b of word w uses the full 32-bit uniform u = sum_q bit_b(plane_q) 2^(31-q), plane q =
 * word (q & 3) of Philox4x32-10((p, t, (w << 8) | (q >> 2), 10 << 24 | instance), seed); the
 * initial word is word 0 of Philox((p, 0, w, 11 << 24 | instance), seed).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

void oracle_philox4x32_10(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4]);
double oracle_exp_neg_d(double x);

typedef struct GmsOracle {
  int32_t n, n_pos, k, D, W, n_rounds, spr, init;
  const int32_t* color_ptr; /* [k+1] */
  const int32_t* ell;       /* [D][n_pos] */
  const uint8_t* degree;    /* [n_pos] */
  const uint8_t* jneg;      /* [n_pos] */
  int64_t n_bonds;
  const double* betas;      /* [R] */
  const uint32_t* thr;      /* [R][D] */
  uint64_t seed;
  uint32_t instance;
  int32_t reserved;
  int64_t round_offset;
  uint32_t* words;          /* [W][n_pos] */
  uint32_t* best_words;
  int64_t* energy;          /* [R] */
  int64_t* best_energy;
  int32_t* rung_of_slot;
  int32_t* slot_of_rung;
  int64_t* tried;           /* [R] */
  int64_t* accepted;
} GmsOracle;

static int bit(uint32_t v, int b) { return (int)((v >> b) & 1u); }

static void energies(const GmsOracle* o, int64_t* e) {
  const int R = 32 * o->W;
  for (int r = 0; r < R; ++r) e[r] = 0;
  for (int w = 0; w < o->W; ++w) {
    const uint32_t* wb = o->words + (size_t)w * o->n_pos;
    for (int p = 0; p < o->n; ++p)
      for (int d = 0; d < o->degree[p]; ++d) {
        const int q = o->ell[(size_t)d * o->n_pos + p];
        if (q >= p) continue; /* each bond once */
        const uint32_t u = wb[p] ^ wb[q] ^ (((o->jneg[p] >> d) & 1u) ? ~0u : 0u);
        for (int b = 0; b < 32; ++b) e[32 * w + b] += bit(u, b);
      }
  }
  for (int r = 0; r < R; ++r) e[r] = 2 * e[r] - o->n_bonds;
}

int oracle_gms_run(GmsOracle* o) {
  const int R = 32 * o->W, D = o->D;
  const uint32_t key[2] = {(uint32_t)(o->seed & 0xffffffffu), (uint32_t)(o->seed >> 32)};
  if (o->n < 1 || o->W < 1 || o->spr < 1 || D < 1) return 1;
  if (o->init) {
    for (int w = 0; w < o->W; ++w)
      for (int p = 0; p < o->n_pos; ++p) {
        const uint32_t ctr[4] = {(uint32_t)p, 0u, (uint32_t)w, (11u << 24) | o->instance};
        uint32_t out[4];
        oracle_philox4x32_10(ctr, key, out);
        const size_t i = (size_t)w * o->n_pos + p;
        o->words[i] = p < o->n ? out[0] : 0u;
        o->best_words[i] = o->words[i];
      }
    energies(o, o->energy);
    for (int r = 0; r < R; ++r) {
      o->best_energy[r] = o->energy[r];
      o->rung_of_slot[r] = r;
      o->slot_of_rung[r] = r;
      o->tried[r] = 0;
      o->accepted[r] = 0;
    }
  }
  for (int j = 0; j < o->n_rounds; ++j) {
    const int64_t round = o->round_offset + j;
    for (int sw = 0; sw < o->spr; ++sw) {
      const uint32_t t = (uint32_t)(round * o->spr + sw);
      for (int c = 0; c < o->k; ++c)
        for (int p = o->color_ptr[c]; p < o->color_ptr[c + 1]; ++p)
          for (int w = 0; w < o->W; ++w) {
            uint32_t* wb = o->words + (size_t)w * o->n_pos;
            uint32_t planes[32];
            for (int ch = 0; ch < 8; ++ch) {
              const uint32_t ctr[4] = {(uint32_t)p, t, ((uint32_t)w << 8) | (uint32_t)ch, (10u << 24) | o->instance};
              uint32_t out[4];
              oracle_philox4x32_10(ctr, key, out);
              for (int i = 0; i < 4; ++i) planes[ch * 4 + i] = out[i];
            }
            const uint32_t s = wb[p];
            uint32_t nw = s;
            const int deg = o->degree[p];
            for (int b = 0; b < 32; ++b) {
              int k = 0;
              for (int d = 0; d < deg; ++d) {
                const int q = o->ell[(size_t)d * o->n_pos + p];
                k += bit(s, b) ^ bit(wb[q], b) ^ (int)((o->jneg[p] >> d) & 1u);
              }
              const int x = deg - 2 * k;
              int flip;
              if (x <= 0) {
                flip = 1;
              } else {
                uint32_t u = 0;
                for (int q = 0; q < 32; ++q) u |= (uint32_t)bit(planes[q], b) << (31 - q);
                flip = u < o->thr[(size_t)o->rung_of_slot[32 * w + b] * D + x - 1];
              }
              if (flip) nw ^= 1u << b;
            }
            wb[p] = nw;
          }
    }
    energies(o, o->energy);
    for (int r = 0; r < R; ++r)
      if (o->energy[r] < o->best_energy[r]) {
        o->best_energy[r] = o->energy[r];
        const int w = r >> 5;
        const uint32_t m = 1u << (r & 31);
        for (int p = 0; p < o->n_pos; ++p) {
          const size_t i = (size_t)w * o->n_pos + p;
          o->best_words[i] = (o->best_words[i] & ~m) | (o->words[i] & m);
        }
      }
    for (int r = (int)(round & 1); r + 1 < R; r += 2) {
      const int a = o->slot_of_rung[r], b = o->slot_of_rung[r + 1];
      const double delta = (o->betas[r] - o->betas[r + 1]) * (double)(o->energy[a] - o->energy[b]);
      int acc = delta >= 0.0;
      if (!acc) {
        const uint32_t ctr[4] = {(uint32_t)r, (uint32_t)round, (uint32_t)((uint64_t)round >> 32), (4u << 24) | o->instance};
        uint32_t out[4];
        oracle_philox4x32_10(ctr, key, out);
        const uint64_t m = ((uint64_t)(out[0] >> 5) << 26) | (uint64_t)(out[1] >> 6);
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
