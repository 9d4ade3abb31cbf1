// dpt_gms.cu - bit-packed (multispin) parallel tempering on any graph with +-1 couplings.
//
// 32 replicas share one 32-bit word per position (bit b of word w = replica slot 32w + b). One CTA
// owns one word for the whole launch: its words for every position, the neighbour table and the
// coupling signs sit in shared memory, so a colour phase is one pass of the CTA's threads over the
// class's positions followed by a CTA barrier - no grid barrier inside a round. For a position the
// unsatisfied-bond count k of every bit comes from bit-sliced adders over the neighbours' words; a
// flip costs dE = 2 (deg - 2k) and is always accepted when deg - 2k <= 0. The other bits compare
// their uniform with their rung's threshold bit-sliced, most significant plane first, drawing
// Philox planes only until all 32 bits are decided (the decision equals the full 32-bit compare).
//
// In a round's last sweep each position also counts, after its update, the unsatisfied bonds to
// neighbours of lower colour (positions before its class): every bond is counted once, at its
// higher-colour end, with both ends final for the round. The per-replica totals give the exact
// energies E = 2U - bonds (|E| < 2^31). The W CTAs then publish each energy with its round tag as
// one 64-bit word (a relaxed single-copy-atomic store, no fence), every CTA gathers all R with all
// its threads, and every CTA evaluates the same adjacent-rung exchange (all waits bounded by a time
// limit).
#include <climits>
#include <cstring>
#include <cuda_runtime.h>

#include "../../include/drift_pt.h"
#include "dpt_common.cuh"
#include "dpt_internal.h"

namespace dpt {
namespace {

constexpr uint32_t kTagGmsSweep = 10u, kTagGmsInit = 11u;
constexpr int kGmsThreads = 512;

struct GmsArgs {
  int n, n_pos, k, D, W, R, n_rounds, spr, ell_in_smem, max_class;
  long long round0, n_bonds;
  uint32_t k0, k1, inst;
  const int* color_ptr;
  const int* ell;
  const uint8_t* degree;
  const uint8_t* jneg;
  const double* betas;
  const uint32_t* thr;  // [R][D]
  uint32_t* words;
  uint32_t* best_words;
  long long* energy;
  long long* best_energy;
  int* rung_of_slot;
  int* slot_of_rung;
  long long* tried;
  long long* accepted;
  int* err;
  long long* pub;
  unsigned long long* tags;
  long long timeout_ns;
};

struct GmsSmem {
  size_t words, ell, deg, jn, cptr, planes, thr, rung, slot, eall, stats, cnt, misc, total;
};

__host__ __device__ inline GmsSmem gms_smem(int n_pos, int D, int k, int R, bool ell_in_smem) {
  GmsSmem L;
  size_t o = 0;
  auto al = [](size_t x) { return (x + 15) & ~(size_t)15; };
  L.words = o;  o = al(o + 4 * (size_t)n_pos);
  L.ell = o;    o = al(o + (ell_in_smem ? 4 * (size_t)D * n_pos : 0));
  L.deg = o;    o = al(o + (size_t)n_pos);
  L.jn = o;     o = al(o + (size_t)n_pos);
  L.cptr = o;   o = al(o + 4 * (size_t)(k + 1));
  L.planes = o; o = al(o + 4 * (size_t)D * 32);
  L.thr = o;    o = al(o + 4 * (size_t)R * D);
  L.rung = o;   o = al(o + 4 * (size_t)R);
  L.slot = o;   o = al(o + 4 * (size_t)R);
  L.eall = o;   o = al(o + 8 * (size_t)R);
  L.stats = o;  o = al(o + 8 * (size_t)R);
  L.cnt = o;    o = al(o + 4 * 32);
  L.misc = o;   o = al(o + 16);
  L.total = o;
  return L;
}

__device__ __forceinline__ unsigned long long gms_now() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
// one replica's energy of a round: (round + 1) << 32 | int32 energy, a single-copy-atomic word
__device__ __forceinline__ void gms_st_word(unsigned long long* p, unsigned long long v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned long long gms_ld_word(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

// bit-sliced add of one input word into the 3-bit counters (k0 + 2 k1 + 4 k2 per bit, <= 7 inputs)
__device__ __forceinline__ void add3(uint32_t u, uint32_t& k0, uint32_t& k1, uint32_t& k2) {
  const uint32_t c0 = k0 & u;
  k0 ^= u;
  const uint32_t c1 = k1 & c0;
  k1 ^= c0;
  k2 |= c1;
}

// bits whose 3-bit counter equals v
__device__ __forceinline__ uint32_t eq3(uint32_t k0, uint32_t k1, uint32_t k2, int v) {
  return ~(k0 ^ ((v & 1) ? ~0u : 0u)) & ~(k1 ^ ((v & 2) ? ~0u : 0u)) & ~(k2 ^ ((v & 4) ? ~0u : 0u));
}

// one input word into a 16-plane bit-sliced counter
__device__ __forceinline__ void add16(uint32_t v, uint32_t (&cs)[16]) {
#pragma unroll
  for (int p = 0; p < 16; ++p) {
    const uint32_t c = cs[p] & v;
    cs[p] ^= v;
    v = c;
  }
}

// 32x32 bit transpose across a warp: on return lane b holds column b (bit r = bit b of lane r's x)
__device__ __forceinline__ uint32_t bit_transpose(uint32_t x, int lane) {
  const uint32_t masks[5] = {0x0000FFFFu, 0x00FF00FFu, 0x0F0F0F0Fu, 0x33333333u, 0x55555555u};
#pragma unroll
  for (int i = 0; i < 5; ++i) {
    const int j = 16 >> i;
    const uint32_t mL = masks[i];
    const uint32_t y = __shfl_xor_sync(0xffffffffu, x, j);
    x = (lane & j) ? ((x & ~mL) | ((y & ~mL) >> j)) : ((x & mL) | ((y & mL) << j));
  }
  return x;
}

// per-bit totals of every thread's 16-plane counters, added into cnt[32]
__device__ __forceinline__ void flush_counts(uint32_t (&cs)[16], unsigned int* cnt) {
  const int lane = threadIdx.x & 31;
  unsigned int mine = 0;
#pragma unroll
  for (int p = 0; p < 16; ++p) {
    if (!__any_sync(0xffffffffu, cs[p] != 0u)) continue;
    mine += (unsigned int)__popc(bit_transpose(cs[p], lane)) << p;
    cs[p] = 0u;
  }
  if (mine) atomicAdd(cnt + lane, mine);
}

__global__ void __launch_bounds__(kGmsThreads, 1) gms_run_kernel(const GmsArgs a) {
  extern __shared__ __align__(16) unsigned char gms_raw[];
  const GmsSmem L = gms_smem(a.n_pos, a.D, a.k, a.R, a.ell_in_smem != 0);
  uint32_t* sw = reinterpret_cast<uint32_t*>(gms_raw + L.words);
  int* ell_sm = reinterpret_cast<int*>(gms_raw + L.ell);
  uint8_t* deg_sm = gms_raw + L.deg;
  uint8_t* jn_sm = gms_raw + L.jn;
  int* cptr = reinterpret_cast<int*>(gms_raw + L.cptr);
  uint32_t* planes = reinterpret_cast<uint32_t*>(gms_raw + L.planes);
  uint32_t* thr_sm = reinterpret_cast<uint32_t*>(gms_raw + L.thr);
  int* rung_sm = reinterpret_cast<int*>(gms_raw + L.rung);
  int* slot_sm = reinterpret_cast<int*>(gms_raw + L.slot);
  long long* eall = reinterpret_cast<long long*>(gms_raw + L.eall);
  int* stats = reinterpret_cast<int*>(gms_raw + L.stats);
  unsigned int* cnt = reinterpret_cast<unsigned int*>(gms_raw + L.cnt);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(gms_raw + L.misc);
  uint32_t* imp = reinterpret_cast<uint32_t*>(gms_raw + L.misc + 4);

  const int tid = threadIdx.x, B = blockDim.x;
  const int w = blockIdx.x, R = a.R, D = a.D, n_pos = a.n_pos;
  const int* ell = a.ell_in_smem ? ell_sm : a.ell;
  uint32_t* gwords = a.words + (size_t)w * n_pos;
  for (int p = tid; p < n_pos; p += B) {
    sw[p] = gwords[p];
    deg_sm[p] = (uint8_t)min((int)a.degree[p], D);
    jn_sm[p] = a.jneg[p];
  }
  if (a.ell_in_smem)
    for (int i = tid; i < D * n_pos; i += B) ell_sm[i] = a.ell[i];
  for (int i = tid; i <= a.k; i += B) cptr[i] = a.color_ptr[i];
  for (int i = tid; i < R * D; i += B) thr_sm[i] = a.thr[i];
  for (int i = tid; i < R; i += B) {
    rung_sm[i] = a.rung_of_slot[i];
    slot_sm[i] = a.slot_of_rung[i];
    stats[2 * i] = stats[2 * i + 1] = 0;
  }
  if (tid < 32) cnt[tid] = 0u;
  if (tid == 0) *abort_flag = 0;
  long long ebest = tid < 32 ? a.best_energy[32 * w + tid] : 0, ecur = tid < 32 ? a.energy[32 * w + tid] : 0;
  // planes[(x-1) * 32 + q], bit b = bit (31 - q) of the threshold for dE/2 = x at bit b's rung
  auto rebuild_planes = [&]() {
    for (int i = tid; i < D * 32; i += B) {
      const int q = i & 31, x = (i >> 5) + 1;
      uint32_t v = 0;
      for (int b = 0; b < 32; ++b) v |= ((thr_sm[rung_sm[32 * w + b] * D + x - 1] >> (31 - q)) & 1u) << b;
      planes[i] = v;
    }
  };
  __syncthreads();
  rebuild_planes();
  __syncthreads();

  const uint32_t ctag = ctr3(kTagGmsSweep, a.inst);
  const uint32_t wtag = (uint32_t)w << 8;
  uint32_t cs[16];
#pragma unroll
  for (int p = 0; p < 16; ++p) cs[p] = 0u;
  for (int j = 0; j < a.n_rounds; ++j) {
    const long long rg = a.round0 + j;
    for (int s_ = 0; s_ < a.spr; ++s_) {
      const uint32_t t = (uint32_t)(rg * a.spr + s_);
      const bool last = s_ == a.spr - 1;
      for (int c = 0; c < a.k; ++c) {
        const int lo = cptr[c], hi = cptr[c + 1];
        for (int p = lo + tid; p < hi; p += B) {
          const uint32_t s = sw[p];
          const int deg = deg_sm[p];
          const uint32_t jb = jn_sm[p];
          uint32_t u[DRIFT_PT_GMS_MAX_DEGREE];
          uint32_t k0 = 0, k1 = 0, k2 = 0;
#pragma unroll
          for (int d = 0; d < DRIFT_PT_GMS_MAX_DEGREE; ++d) {
            if (d >= D) break;
            u[d] = 0u;
            if (d < deg) {
              const int nb = ell[(size_t)d * n_pos + p];
              u[d] = s ^ sw[nb] ^ (((jb >> d) & 1u) ? ~0u : 0u);
              add3(u[d], k0, k1, k2);
            }
          }
          // bits with k < deg/2 (dE > 0) need a test against the threshold of x = deg - 2k
          uint32_t need = 0u;
          uint32_t mk[4] = {0u, 0u, 0u, 0u};
#pragma unroll
          for (int kk = 0; kk < 4; ++kk)
            if (2 * kk < deg) {
              mk[kk] = eq3(k0, k1, k2, kk);
              need |= mk[kk];
            }
          uint32_t lt = 0u, und = need;
          for (int ch = 0; ch < 8 && und; ++ch) {
            const U4 r = philox(U4{(uint32_t)p, t, wtag | (uint32_t)ch, ctag}, a.k0, a.k1);
            const uint32_t rw[4] = {r.x, r.y, r.z, r.w};
#pragma unroll
            for (int i = 0; i < 4; ++i) {
              const int q = ch * 4 + i;
              uint32_t tp = 0u;
#pragma unroll
              for (int kk = 0; kk < 4; ++kk)
                if (2 * kk < deg) tp |= mk[kk] & planes[(deg - 2 * kk - 1) * 32 + q];
              lt |= und & ~rw[i] & tp;
              und &= ~(rw[i] ^ tp);
            }
          }
          const uint32_t acc = ~need | lt;
          const uint32_t s2 = s ^ acc;
          sw[p] = s2;
          if (last) {
            // unsatisfied bonds to lower-colour neighbours, after this update
#pragma unroll
            for (int d = 0; d < DRIFT_PT_GMS_MAX_DEGREE; ++d) {
              if (d >= D) break;
              if (d < deg) {
                const int nb = ell[(size_t)d * n_pos + p];
                if (nb < lo) add16(s2 ^ sw[nb] ^ (((jb >> d) & 1u) ? ~0u : 0u), cs);
              }
            }
          }
        }
        __syncthreads();
      }
    }
    // ---- round end: exact energies, bests, publication, exchange ----
    flush_counts(cs, cnt);
    __syncthreads();
    if (tid < 32) {
      ecur = 2 * (long long)cnt[tid] - a.n_bonds;
      cnt[tid] = 0u;
      const bool better = ecur < ebest;
      if (better) ebest = ecur;
      const unsigned int mask = __ballot_sync(0xffffffffu, better);
      if (tid == 0) *imp = mask;
      unsigned long long* pw = reinterpret_cast<unsigned long long*>(a.pub) + (size_t)(rg & 1) * R;
      gms_st_word(pw + 32 * w + tid, ((unsigned long long)(uint32_t)(rg + 1) << 32) | (uint32_t)(int32_t)ecur);
    }
    __syncthreads();
    {
      const uint32_t mk = *imp;
      if (mk) {
        uint32_t* bw = a.best_words + (size_t)w * n_pos;
        for (int p = tid; p < n_pos; p += B) bw[p] = (bw[p] & ~mk) | (sw[p] & mk);
      }
    }
    {
      // gather every slot's energy of this round (W CTAs), all threads, bounded waits
      const unsigned long long* pw = reinterpret_cast<const unsigned long long*>(a.pub) + (size_t)(rg & 1) * R;
      const uint32_t tag = (uint32_t)(rg + 1);
      for (int s = tid; s < R; s += B) {
        unsigned long long v = gms_ld_word(pw + s);
        if ((uint32_t)(v >> 32) != tag) {
          const unsigned long long t0 = gms_now();
          bool bad = false;
          while ((uint32_t)((v = gms_ld_word(pw + s)) >> 32) != tag) {
            if (*abort_flag) {
              bad = true;
              break;
            }
            if (gms_now() - t0 > (unsigned long long)a.timeout_ns) {
              *abort_flag = 1;
              atomicExch(a.err, DRIFT_PT_ETIMEOUT);
              bad = true;
              break;
            }
          }
          if (bad) break;
        }
        eall[s] = (long long)(int32_t)(uint32_t)v;
      }
    }
    __syncthreads();
    if (tid < 32 && !*abort_flag) {
      // the exchange step, identical in every CTA
      const int parity = (int)(rg & 1);
      for (int rr = parity + 2 * tid; rr + 1 < R; rr += 64) {
        const int sa = slot_sm[rr], sb = slot_sm[rr + 1];
        const double dlt = d_mul(d_sub(a.betas[rr], a.betas[rr + 1]), (double)(eall[sa] - eall[sb]));
        bool acc = dlt >= 0.0;
        if (!acc) {
          const U4 u = philox(U4{(uint32_t)rr, (uint32_t)rg, (uint32_t)((unsigned long long)rg >> 32),
                                 ctr3(kTagSwap, a.inst)},
                              a.k0, a.k1);
          acc = uniform53(u.x, u.y) < exp_neg_d(dlt);
        }
        if (w == 0) {
          stats[2 * rr] += 1;
          stats[2 * rr + 1] += acc ? 1 : 0;
        }
        if (acc) {
          slot_sm[rr] = sb;
          slot_sm[rr + 1] = sa;
          rung_sm[sa] = rr + 1;
          rung_sm[sb] = rr;
        }
      }
    }
    __syncthreads();
    if (*abort_flag) break;
    rebuild_planes();
    __syncthreads();
  }
  // ---- write back ----
  for (int p = tid; p < n_pos; p += B) gwords[p] = sw[p];
  if (tid < 32) {
    a.energy[32 * w + tid] = ecur;
    a.best_energy[32 * w + tid] = ebest;
  }
  if (w == 0 && !*abort_flag) {
    for (int i = tid; i < R; i += B) {
      a.rung_of_slot[i] = rung_sm[i];
      a.slot_of_rung[i] = slot_sm[i];
    }
    for (int rr = tid; rr < R - 1; rr += B) {
      a.tried[rr] += stats[2 * rr];
      a.accepted[rr] += stats[2 * rr + 1];
    }
  }
}

// initial words, exact energies (each bond counted at its larger-position end), bests, rungs
__global__ void gms_init_kernel(const GmsArgs a) {
  const int w = blockIdx.x, n_pos = a.n_pos, tid = threadIdx.x, B = blockDim.x;
  __shared__ unsigned int cnt[32];
  if (tid < 32) cnt[tid] = 0u;
  uint32_t* gw = a.words + (size_t)w * n_pos;
  for (int p = tid; p < n_pos; p += B) {
    const U4 r = philox(U4{(uint32_t)p, 0u, (uint32_t)w, ctr3(kTagGmsInit, a.inst)}, a.k0, a.k1);
    const uint32_t v = p < a.n ? r.x : 0u;
    gw[p] = v;
    a.best_words[(size_t)w * n_pos + p] = v;
  }
  __syncthreads();
  uint32_t cs[16];
#pragma unroll
  for (int q = 0; q < 16; ++q) cs[q] = 0u;
  const int iters = (n_pos + B - 1) / B;
  for (int it = 0; it < iters; ++it) {
    const int p = it * B + tid;
    if (p < a.n) {
      const uint32_t s = gw[p];
      const int deg = a.degree[p];
      const uint32_t jb = a.jneg[p];
      for (int d = 0; d < deg; ++d) {
        const int nb = a.ell[(size_t)d * n_pos + p];
        if (nb < p) add16(s ^ gw[nb] ^ (((jb >> d) & 1u) ? ~0u : 0u), cs);
      }
    }
  }
  flush_counts(cs, cnt);
  __syncthreads();
  if (tid < 32) {
    const int slot = 32 * w + tid;
    const long long e = 2 * (long long)cnt[tid] - a.n_bonds;
    a.energy[slot] = e;
    a.best_energy[slot] = e;
    a.rung_of_slot[slot] = slot;
    a.slot_of_rung[slot] = slot;
    if (slot < a.R - 1) {
      a.tried[slot] = 0;
      a.accepted[slot] = 0;
    }
  }
}

// ---------------------------------------------------------------------------------------------
// Cluster form: a word's positions are split over a cluster of C CTAs. In every colour class c
// (positions [lo, lo + m)) CTA r owns [lo + r q, lo + min(m, (r + 1) q)), q = ceil(m / C); its
// words sit in its own shared memory in class order, and a neighbour's word is read from the
// owner's shared memory (ld.shared::cluster through an address resolved once per launch). Counters,
// thresholds and decisions are those of the one-CTA form, so both produce the same bits.
//
// The random planes do not depend on the state, and within a round neither do the thresholds: a
// position's decision depends on the state only through which of its (at most 4) positive energy
// changes each bit has. So while the deciding warps run colour phase c, the other warps of the CTA
// draw the positions of the next phase and compare their first 16 planes with the thresholds of
// every possible energy change, kGmcDraw lanes per position (one Philox block each, partial
// decisions combined in plane order by shuffles). The deciding thread then only counts unsatisfied
// bonds and selects its bits' results; bits still undecided after 16 planes continue inline. A phase
// ends with one cluster barrier (shared-memory release fence, relaxed arrive, acquiring wait).
// CTA rank 0 of each cluster sums the cluster's energy counts, publishes them as one 64-bit (round
// tag, energy) word per replica and runs the exchange; the other CTAs read its results after a
// cluster barrier.

constexpr int kGmcMaxThreads = 512;
constexpr int kGmcDraw = 4;  // Philox blocks (4 planes each) decided ahead per position, one lane each

struct GmcSmem {
  size_t words, best, addr, gpos, deg, jn, low, rng, cptr, lcp, planes, thr, rung, slot, eall, stats, cnt, rung32,
      misc, total;
};

// owned positions per CTA are at most ceil(n / C) + k (one partial share per class); a class share
// is at most ceil(max_class / C)
__host__ __device__ inline int gmc_cap(int n, int k, int C) { return (n + C - 1) / C + k; }
__host__ __device__ inline int gmc_cap_phase(int max_class, int C) { return (max_class + C - 1) / C; }

__host__ __device__ inline GmcSmem gmc_smem(int cap, int cap_ph, int D, int k, int R) {
  GmcSmem L;
  size_t o = 0;
  auto al = [](size_t x) { return (x + 15) & ~(size_t)15; };
  L.words = o;  o = al(o + 4 * (size_t)cap);
  L.best = o;   o = al(o + 4 * (size_t)cap);
  L.addr = o;   o = al(o + 4 * (size_t)D * cap);
  L.gpos = o;   o = al(o + 4 * (size_t)cap);
  L.deg = o;    o = al(o + (size_t)cap);
  L.jn = o;     o = al(o + (size_t)cap);
  L.low = o;    o = al(o + (size_t)cap);
  L.rng = o;    o = al(o + 2 * 32 * (size_t)cap_ph);
  L.cptr = o;   o = al(o + 4 * (size_t)(k + 1));
  L.lcp = o;    o = al(o + 4 * (size_t)(k + 1));
  L.planes = o; o = al(o + 4 * (size_t)D * 32);
  L.thr = o;    o = al(o + 4 * (size_t)R * D);
  L.rung = o;   o = al(o + 4 * (size_t)R);
  L.slot = o;   o = al(o + 4 * (size_t)R);
  L.eall = o;   o = al(o + 8 * (size_t)R);
  L.stats = o;  o = al(o + 8 * (size_t)R);
  L.cnt = o;    o = al(o + 4 * 32);
  L.rung32 = o; o = al(o + 4 * 32);
  L.misc = o;   o = al(o + 16);
  L.total = o;
  return L;
}

__device__ __forceinline__ uint32_t gmc_rank() {
  uint32_t r;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
  return r;
}
// full cluster barrier, release/acquire for every memory space (first and last use of the cluster)
__device__ __forceinline__ void gmc_sync_full() {
  __syncwarp();  // the .aligned barrier wants the whole warp converged
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
// arrive half of a cluster barrier that publishes this thread's shared-memory writes
__device__ __forceinline__ void gmc_arrive_smem() {
  __syncwarp();
  asm volatile("fence.release.sync_restrict::shared::cta.cluster;\n\tbarrier.cluster.arrive.relaxed.aligned;" ::: "memory");
}
__device__ __forceinline__ void gmc_wait() {
  __syncwarp();
  asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
}
__device__ __forceinline__ void gmc_sync_smem() {
  gmc_arrive_smem();
  gmc_wait();
}
__device__ __forceinline__ uint32_t gmc_saddr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ uint32_t gmc_map(uint32_t saddr, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(saddr), "r"(rank));
  return r;
}
__device__ __forceinline__ uint32_t gmc_ld(uint32_t caddr) {
  uint32_t v;
  asm volatile("ld.shared::cluster.u32 %0, [%1];" : "=r"(v) : "r"(caddr) : "memory");
  return v;
}
__device__ __forceinline__ void gmc_st_pub(unsigned long long* p, unsigned long long v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ unsigned long long gmc_ld_pub(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

// positions of class [lo, lo + m) owned by rank r
__device__ __forceinline__ int gmc_own(int m, int C, int r) {
  const int q = (m + C - 1) / C;
  return max(0, min(q, m - r * q));
}

__global__ void __launch_bounds__(kGmcMaxThreads, 1) gmc_run_kernel(const GmsArgs a, const int C) {
  extern __shared__ __align__(16) unsigned char gmc_raw[];
  const int cap = gmc_cap(a.n, a.k, C), cap_ph = gmc_cap_phase(a.max_class, C);
  const GmcSmem L = gmc_smem(cap, cap_ph, a.D, a.k, a.R);
  uint32_t* sw = reinterpret_cast<uint32_t*>(gmc_raw + L.words);
  uint32_t* bw = reinterpret_cast<uint32_t*>(gmc_raw + L.best);
  uint32_t* naddr = reinterpret_cast<uint32_t*>(gmc_raw + L.addr);  // [D][cap]
  int* gpos = reinterpret_cast<int*>(gmc_raw + L.gpos);
  uint8_t* deg_sm = gmc_raw + L.deg;
  uint8_t* jn_sm = gmc_raw + L.jn;
  uint8_t* low_sm = gmc_raw + L.low;
  uint4* pre = reinterpret_cast<uint4*>(gmc_raw + L.rng);  // [2][cap_ph][2]: accepted, undecided per change
  int* cptr = reinterpret_cast<int*>(gmc_raw + L.cptr);
  int* lcp = reinterpret_cast<int*>(gmc_raw + L.lcp);
  uint32_t* planes = reinterpret_cast<uint32_t*>(gmc_raw + L.planes);
  uint32_t* thr_sm = reinterpret_cast<uint32_t*>(gmc_raw + L.thr);
  int* rung_sm = reinterpret_cast<int*>(gmc_raw + L.rung);
  int* slot_sm = reinterpret_cast<int*>(gmc_raw + L.slot);
  long long* eall = reinterpret_cast<long long*>(gmc_raw + L.eall);
  int* stats = reinterpret_cast<int*>(gmc_raw + L.stats);
  unsigned int* cnt = reinterpret_cast<unsigned int*>(gmc_raw + L.cnt);
  int* rung32 = reinterpret_cast<int*>(gmc_raw + L.rung32);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(gmc_raw + L.misc);
  uint32_t* imp = reinterpret_cast<uint32_t*>(gmc_raw + L.misc + 4);
  int* bcast = reinterpret_cast<int*>(gmc_raw + L.misc + 8);  // [0] improved mask, [1] abort, read from rank 0

  const int tid = threadIdx.x, B = blockDim.x;
  const int rank = (int)gmc_rank(), w = blockIdx.x / C;
  const int R = a.R, D = a.D, n_pos = a.n_pos, k = a.k;
  for (int i = tid; i <= k; i += B) cptr[i] = a.color_ptr[i];
  __syncthreads();
  // the shared-memory shares are sized for classes that tile [0, n): any other colour table is rejected
  // here, by every CTA alike, before the first cluster barrier
  {
    bool ok = cptr[0] == 0 && cptr[k] == a.n;
    for (int c = 0; c < k && ok; ++c) ok = cptr[c + 1] >= cptr[c] && cptr[c + 1] - cptr[c] <= a.max_class;
    if (!ok) {
      if (tid == 0 && rank == 0) atomicExch(a.err, DRIFT_PT_EINVAL);
      return;
    }
  }
  for (int i = tid; i < R * D; i += B) thr_sm[i] = a.thr[i];
  for (int i = tid; i < R; i += B) {
    rung_sm[i] = a.rung_of_slot[i];
    slot_sm[i] = a.slot_of_rung[i];
    stats[2 * i] = stats[2 * i + 1] = 0;
  }
  if (tid < 32) {
    cnt[tid] = 0u;
    rung32[tid] = a.rung_of_slot[32 * w + tid];
  }
  if (tid == 0) {
    *abort_flag = 0;
    *imp = 0u;
    int off = 0;
    for (int c = 0; c < k; ++c) {
      lcp[c] = off;
      off += gmc_own(cptr[c + 1] - cptr[c], C, rank);
    }
    lcp[k] = off;
  }
  __syncthreads();
  // owned positions: words, degree, signs, lower-colour mask and the cluster address of every neighbour
  const uint32_t sw_base = gmc_saddr(sw);
  const uint32_t* gwords = a.words + (size_t)w * n_pos;
  const uint32_t* gbest = a.best_words + (size_t)w * n_pos;
  for (int c = 0; c < k; ++c) {
    const int lo = cptr[c], m = cptr[c + 1] - lo, q = (m + C - 1) / C;
    const int cntc = gmc_own(m, C, rank), first = lo + rank * q;
    for (int j = tid; j < cntc; j += B) {
      const int p = first + j, l = lcp[c] + j;
      gpos[l] = p;
      sw[l] = gwords[p];
      bw[l] = gbest[p];
      const int deg = min((int)a.degree[p], D);
      deg_sm[l] = (uint8_t)deg;
      jn_sm[l] = a.jneg[p];
      uint8_t low = 0;
      for (int d = 0; d < deg; ++d) {
        int nb = a.ell[(size_t)d * n_pos + p];
        if (nb < 0 || nb >= a.n) {  // not a spin: flagged, and read as the position itself
          atomicExch(a.err, DRIFT_PT_EINVAL);
          nb = p;
        }
        int c2 = 0;
        while (c2 + 1 < k && cptr[c2 + 1] <= nb) ++c2;
        const int lo2 = cptr[c2], m2 = cptr[c2 + 1] - lo2, q2 = (m2 + C - 1) / C;
        const int r2 = (nb - lo2) / q2;
        int off = 0;
        for (int c3 = 0; c3 < c2; ++c3) off += gmc_own(cptr[c3 + 1] - cptr[c3], C, r2);
        naddr[(size_t)d * cap + l] = gmc_map(sw_base + 4u * (uint32_t)(off + nb - lo2 - r2 * q2), (uint32_t)r2);
        if (nb < lo) low |= (uint8_t)(1u << d);
      }
      low_sm[l] = low;
    }
  }
  long long ebest = (rank == 0 && tid < 32) ? a.best_energy[32 * w + tid] : 0;
  long long ecur = (rank == 0 && tid < 32) ? a.energy[32 * w + tid] : 0;
  auto rebuild_planes = [&]() {
    for (int i = tid; i < D * 32; i += B) {
      const int q = i & 31, x = (i >> 5) + 1;
      uint32_t v = 0;
      for (int b = 0; b < 32; ++b) v |= ((thr_sm[rung32[b] * D + x - 1] >> (31 - q)) & 1u) << b;
      planes[i] = v;
    }
  };
  const uint32_t ctag = ctr3(kTagGmsSweep, a.inst);
  const uint32_t wtag = (uint32_t)w << 8;
  // Decisions of the first 4 kGmcDraw planes for every position of class c at sweep t, into buffer b,
  // by nd threads (d = this thread's index among them; warps stay whole). For each positive energy
  // change 2x a position can have (x = deg - 2kk, kk = unsatisfied bonds), .x..w of the first uint4
  // hold the bits already accepted and of the second the bits still undecided.
  auto draw = [&](int c, uint32_t t, int b, int d, int nd) {
    const int lo = lcp[c], m = lcp[c + 1] - lo, lane = d & 31, g = d & (kGmcDraw - 1);
    uint4* out = pre + (size_t)b * cap_ph * 2;
    const uint4* pl4 = reinterpret_cast<const uint4*>(planes);
    for (int base = d - lane; base < m * kGmcDraw; base += nd) {
      const int it = base + lane;
      const bool on = it < m * kGmcDraw;
      const int pi = on ? it / kGmcDraw : 0;
      const int deg = on ? deg_sm[lo + pi] : 0;
      const U4 r = philox(U4{(uint32_t)gpos[lo + pi], t, wtag | (uint32_t)g, ctag}, a.k0, a.k1);
      const uint32_t rw[4] = {r.x, r.y, r.z, r.w};
      uint32_t lt[4], un[4];
#pragma unroll
      for (int kk = 0; kk < 4; ++kk) {
        lt[kk] = 0u;
        un[kk] = ~0u;
        if (2 * kk < deg) {
          const uint4 pv = pl4[(deg - 2 * kk - 1) * 8 + g];
          const uint32_t tq[4] = {pv.x, pv.y, pv.z, pv.w};
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            lt[kk] |= un[kk] & ~rw[i] & tq[i];
            un[kk] &= ~(rw[i] ^ tq[i]);
          }
        }
      }
      // combine the group's blocks, earlier planes first: (lt, un) then (lt', un') gives
      // (lt | un & lt', un & un')
#pragma unroll
      for (int sft = 1; sft < kGmcDraw; sft <<= 1) {
#pragma unroll
        for (int kk = 0; kk < 4; ++kk) {
          const uint32_t ol = __shfl_xor_sync(0xffffffffu, lt[kk], sft);
          const uint32_t ou = __shfl_xor_sync(0xffffffffu, un[kk], sft);
          if (g & sft) {
            lt[kk] = ol | (ou & lt[kk]);
            un[kk] = ou & un[kk];
          } else {
            lt[kk] = lt[kk] | (un[kk] & ol);
            un[kk] = un[kk] & ou;
          }
        }
      }
      if (on && g == 0) {
        out[2 * pi] = make_uint4(lt[0], lt[1], lt[2], lt[3]);
        out[2 * pi + 1] = make_uint4(un[0], un[1], un[2], un[3]);
      }
    }
  };
  // the deciding threads [0, NC) cover the largest class share; the others draw ahead
  const int NC = min(B, (cap_ph + 31) & ~31), ND = B - NC;
  const bool split = ND >= 64;
  __syncthreads();
  rebuild_planes();
  __syncthreads();
  int buf = 0;
  if (a.n_rounds > 0) draw(0, (uint32_t)(a.round0 * a.spr), 0, tid, B);
  __syncthreads();
  gmc_sync_full();  // every CTA's words and decisions are in place before any neighbour read

  const uint32_t r0_rung = gmc_map(gmc_saddr(rung_sm), 0u);
  const uint32_t r0_bcast = gmc_map(gmc_saddr(bcast), 0u);
  uint32_t cs[16];
#pragma unroll
  for (int p = 0; p < 16; ++p) cs[p] = 0u;
  for (int j = 0; j < a.n_rounds; ++j) {
    const long long rg = a.round0 + j;
    for (int s_ = 0; s_ < a.spr; ++s_) {
      const uint32_t t = (uint32_t)(rg * a.spr + s_);
      const bool last = s_ == a.spr - 1;
      for (int c = 0; c < k; ++c) {
        const uint4* pb = pre + (size_t)buf * cap_ph * 2;
        const bool draw_next = !(last && c + 1 == k);  // the next round's first phase is drawn after the exchange
        if (!split || tid < NC) {
          for (int l = lcp[c] + tid; l < lcp[c + 1]; l += split ? NC : B) {
            const uint32_t p = (uint32_t)gpos[l];
            const uint32_t s = sw[l];
            const int deg = deg_sm[l];
            const uint32_t jb = jn_sm[l];
            uint32_t u[DRIFT_PT_GMS_MAX_DEGREE];
#pragma unroll
            for (int d = 0; d < DRIFT_PT_GMS_MAX_DEGREE; ++d)
              u[d] = d < deg ? gmc_ld(naddr[(size_t)d * cap + l]) : 0u;
            const uint4 lt4 = pb[2 * (l - lcp[c])], un4 = pb[2 * (l - lcp[c]) + 1];
            uint32_t k0 = 0, k1 = 0, k2 = 0;
#pragma unroll
            for (int d = 0; d < DRIFT_PT_GMS_MAX_DEGREE; ++d)
              if (d < deg) {
                u[d] ^= s ^ (((jb >> d) & 1u) ? ~0u : 0u);
                add3(u[d], k0, k1, k2);
              }
            uint32_t need = 0u, lt = 0u, und = 0u;
            uint32_t mk[4] = {0u, 0u, 0u, 0u};
            const uint32_t l4[4] = {lt4.x, lt4.y, lt4.z, lt4.w}, u4[4] = {un4.x, un4.y, un4.z, un4.w};
#pragma unroll
            for (int kk = 0; kk < 4; ++kk)
              if (2 * kk < deg) {
                mk[kk] = eq3(k0, k1, k2, kk);
                need |= mk[kk];
                lt |= mk[kk] & l4[kk];
                und |= mk[kk] & u4[kk];
              }
            // bits still undecided after the drawn planes continue here, plane by plane
            for (int ch = kGmcDraw; ch < 8 && und; ++ch) {
              const U4 r = philox(U4{p, t, wtag | (uint32_t)ch, ctag}, a.k0, a.k1);
              const uint32_t rw[4] = {r.x, r.y, r.z, r.w};
#pragma unroll
              for (int i = 0; i < 4; ++i) {
                const int q = ch * 4 + i;
                uint32_t tp = 0u;
#pragma unroll
                for (int kk = 0; kk < 4; ++kk)
                  if (2 * kk < deg) tp |= mk[kk] & planes[(deg - 2 * kk - 1) * 32 + q];
                lt |= und & ~rw[i] & tp;
                und &= ~(rw[i] ^ tp);
              }
            }
            const uint32_t acc = ~need | lt;
            sw[l] = s ^ acc;
            if (last) {
              // unsatisfied bonds to lower-colour neighbours after this update: u ^ acc
              const uint32_t low = low_sm[l];
#pragma unroll
              for (int d = 0; d < DRIFT_PT_GMS_MAX_DEGREE; ++d)
                if (d < deg && ((low >> d) & 1u)) add16(u[d] ^ acc, cs);
            }
          }
        }
        if (draw_next) {
          const int cn = c + 1 < k ? c + 1 : 0;
          const uint32_t tn = c + 1 < k ? t : t + 1u;
          if (!split) draw(cn, tn, buf ^ 1, tid, B);
          else if (tid >= NC) draw(cn, tn, buf ^ 1, tid - NC, ND);
        }
        gmc_sync_smem();
        buf ^= 1;
      }
    }
    // ---- round end: cluster energy counts, publication and exchange on rank 0 ----
    flush_counts(cs, cnt);
    gmc_sync_smem();
    if (rank == 0) {
      const uint32_t tag = (uint32_t)(rg + 1);
      unsigned long long* pub = reinterpret_cast<unsigned long long*>(a.pub) + (size_t)(rg & 1) * R;
      if (tid < 32) {
        unsigned int tot = 0u;
        for (int r = 0; r < C; ++r) tot += gmc_ld(gmc_map(gmc_saddr(cnt + tid), (uint32_t)r));
        ecur = 2 * (long long)tot - a.n_bonds;
        const bool better = ecur < ebest;
        if (better) ebest = ecur;
        const unsigned int mask = __ballot_sync(0xffffffffu, better);
        if (tid == 0) bcast[0] = (int)mask;
        gmc_st_pub(pub + 32 * w + tid, ((unsigned long long)tag << 32) | (uint32_t)(int32_t)ecur);
      }
      // every slot's energy of this round, gathered by all of rank 0's threads (bounded waits)
      for (int s = tid; s < R; s += B) {
        unsigned long long v = gmc_ld_pub(pub + s);
        if ((uint32_t)(v >> 32) != tag) {
          const unsigned long long t0 = gms_now();
          bool bad = false;
          while ((uint32_t)((v = gmc_ld_pub(pub + s)) >> 32) != tag) {
            if (*abort_flag) {
              bad = true;
              break;
            }
            if (gms_now() - t0 > (unsigned long long)a.timeout_ns) {
              *abort_flag = 1;
              atomicExch(a.err, DRIFT_PT_ETIMEOUT);
              bad = true;
              break;
            }
          }
          if (bad) break;
        }
        eall[s] = (long long)(int32_t)(uint32_t)v;
      }
      __syncthreads();  // rank is the same for every thread of a CTA
      if (tid < 32) {
        if (!*abort_flag) {
          const int parity = (int)(rg & 1);
          for (int rr = parity + 2 * tid; rr + 1 < R; rr += 64) {
            const int sa = slot_sm[rr], sb = slot_sm[rr + 1];
            const double dlt = d_mul(d_sub(a.betas[rr], a.betas[rr + 1]), (double)(eall[sa] - eall[sb]));
            bool acc = dlt >= 0.0;
            if (!acc) {
              const U4 uu = philox(U4{(uint32_t)rr, (uint32_t)rg, (uint32_t)((unsigned long long)rg >> 32),
                                      ctr3(kTagSwap, a.inst)},
                                   a.k0, a.k1);
              acc = uniform53(uu.x, uu.y) < exp_neg_d(dlt);
            }
            if (w == 0) {
              stats[2 * rr] += 1;
              stats[2 * rr + 1] += acc ? 1 : 0;
            }
            if (acc) {
              slot_sm[rr] = sb;
              slot_sm[rr + 1] = sa;
              rung_sm[sa] = rr + 1;
              rung_sm[sb] = rr;
            }
          }
        }
        __syncwarp();
        if (tid == 0) bcast[1] = *abort_flag ? 1 : 0;
      }
    }
    gmc_sync_smem();
    // every CTA: improved mask, abort and its word's rungs from rank 0
    if (tid < 32) {
      rung32[tid] = (int)gmc_ld(r0_rung + 4u * (uint32_t)(32 * w + tid));
      cnt[tid] = 0u;
    }
    if (tid == 0) {
      *imp = gmc_ld(r0_bcast);
      *abort_flag = (int)gmc_ld(r0_bcast + 4u);
    }
    __syncthreads();
    {
      const uint32_t mk = *imp;
      if (mk)
        for (int l = tid; l < lcp[k]; l += B) bw[l] = (bw[l] & ~mk) | (sw[l] & mk);
    }
    if (*abort_flag) break;
    rebuild_planes();
    __syncthreads();
    if (j + 1 < a.n_rounds) {
      draw(0, (uint32_t)((rg + 1) * a.spr), buf, tid, B);
      __syncthreads();
    }
  }
  // ---- write back ----
  {
    uint32_t* gw = a.words + (size_t)w * n_pos;
    uint32_t* gb = a.best_words + (size_t)w * n_pos;
    for (int l = tid; l < lcp[k]; l += B) {
      gw[gpos[l]] = sw[l];
      gb[gpos[l]] = bw[l];
    }
  }
  if (rank == 0 && tid < 32) {
    a.energy[32 * w + tid] = ecur;
    a.best_energy[32 * w + tid] = ebest;
  }
  if (w == 0 && rank == 0 && !*abort_flag) {
    for (int i = tid; i < R; i += B) {
      a.rung_of_slot[i] = rung_sm[i];
      a.slot_of_rung[i] = slot_sm[i];
    }
    for (int rr = tid; rr < R - 1; rr += B) {
      a.tried[rr] += stats[2 * rr];
      a.accepted[rr] += stats[2 * rr + 1];
    }
  }
  gmc_sync_full();  // rank 0's shared memory stays alive until every CTA has read it
}

int gms_fail(cudaError_t e, const char* what) { return set_error(DRIFT_PT_ECUDA, "%s: %s", what, cudaGetErrorString(e)); }

int gms_args(const DriftPtGmsProblem* p, const DriftPtGmsRunArgs* r, DriftPtGmsState* s, GmsArgs& a) {
  if (!p || !r || !s) return set_error(DRIFT_PT_EINVAL, "gms: null argument");
  if (p->n < 1 || p->n_pos < p->n || p->n_pos % 32 || p->n_colors < 1 || p->max_degree < 1 ||
      p->max_degree > DRIFT_PT_GMS_MAX_DEGREE || p->n_bonds < 0)
    return set_error(DRIFT_PT_EINVAL, "gms: problem sizes out of range");
  if (!p->color_ptr || !p->ell_nbr || !p->degree || !p->jneg) return set_error(DRIFT_PT_EINVAL, "gms: problem arrays missing");
  if (p->max_class < 1 || p->max_class > p->n) return set_error(DRIFT_PT_EINVAL, "gms: max_class must be in 1..n");
  if (r->n_words < 1 || r->n_words > 64) return set_error(DRIFT_PT_EINVAL, "gms: n_words must be in 1..64");
  if (p->n_bonds >= (1ll << 31)) return set_error(DRIFT_PT_EUNSUPPORTED, "gms: 2^31 or more bonds");
  if (r->instance > kMaxInstance) return set_error(DRIFT_PT_EINVAL, "gms: instance >= 2^24");
  if (!s->words || !s->best_words || !s->energy || !s->best_energy || !s->rung_of_slot || !s->slot_of_rung ||
      !s->swap_tried || !s->swap_accepted)
    return set_error(DRIFT_PT_EINVAL, "gms: state arrays missing");
  std::memset(&a, 0, sizeof a);
  a.n = p->n;
  a.n_pos = p->n_pos;
  a.k = p->n_colors;
  a.D = p->max_degree;
  a.W = r->n_words;
  a.R = 32 * r->n_words;
  a.n_rounds = r->n_rounds;
  a.spr = r->sweeps_per_round;
  a.round0 = r->round_offset;
  a.n_bonds = p->n_bonds;
  a.max_class = p->max_class;
  a.k0 = (uint32_t)(r->seed & 0xffffffffu);
  a.k1 = (uint32_t)(r->seed >> 32);
  a.inst = r->instance;
  a.color_ptr = p->color_ptr;
  a.ell = p->ell_nbr;
  a.degree = p->degree;
  a.jneg = p->jneg;
  a.betas = r->betas;
  a.thr = r->thresholds;
  a.words = s->words;
  a.best_words = s->best_words;
  a.energy = reinterpret_cast<long long*>(s->energy);
  a.best_energy = reinterpret_cast<long long*>(s->best_energy);
  a.rung_of_slot = s->rung_of_slot;
  a.slot_of_rung = s->slot_of_rung;
  a.tried = reinterpret_cast<long long*>(s->swap_tried);
  a.accepted = reinterpret_cast<long long*>(s->swap_accepted);
  a.timeout_ns = (long long)((r->timeout_s > 0 ? r->timeout_s : 10.0) * 1e9);
  return DRIFT_PT_OK;
}

int gmc_launch(GmsArgs& a, int C, int threads, int sms, int optin, unsigned char* ws, size_t need, cudaStream_t st) {
  const int cap = gmc_cap(a.n, a.k, C);
  const GmcSmem L = gmc_smem(cap, gmc_cap_phase(a.max_class, C), a.D, a.k, a.R);
  if (a.n_bonds >= (1ll << 31)) return set_error(DRIFT_PT_EUNSUPPORTED, "gms: 2^31 or more bonds");
  if (L.total > (size_t)optin)
    return set_error(DRIFT_PT_EUNSUPPORTED, "gms: a cluster of %d CTAs cannot hold %d positions", C, a.n);
  if (threads == 0) threads = kGmcMaxThreads;
  if (threads < 32 || threads > kGmcMaxThreads || threads % 32)
    return set_error(DRIFT_PT_EINVAL, "gms: threads_per_cta must be a multiple of 32 in [32, %d] with clusters",
                     kGmcMaxThreads);
  if (a.W * C > sms) return set_error(DRIFT_PT_EUNSUPPORTED, "gms: %d clusters of %d CTAs exceed the SMs", a.W, C);
  int per_sm = 0;
  int rc = prepare_kernel((const void*)gmc_run_kernel, threads, L.total, &per_sm);
  if (rc) return rc;
  if (C > 8) {
    const cudaError_t e = cudaFuncSetAttribute((const void*)gmc_run_kernel,
                                               cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (e != cudaSuccess) return gms_fail(e, "cluster size attribute");
  }
  cudaLaunchConfig_t cfg;
  std::memset(&cfg, 0, sizeof cfg);
  cfg.gridDim = dim3(a.W * C);
  cfg.blockDim = dim3(threads);
  cfg.dynamicSmemBytes = L.total;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = C;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  // the W clusters wait on one another's energies: all of them must be resident at once
  int max_clusters = 0;
  cudaError_t e = cudaOccupancyMaxActiveClusters(&max_clusters, (const void*)gmc_run_kernel, &cfg);
  if (e != cudaSuccess) return gms_fail(e, "cluster occupancy query");
  if (max_clusters < a.W)
    return set_error(DRIFT_PT_EUNSUPPORTED, "gms: only %d clusters of %d CTAs can be resident, %d needed", max_clusters,
                     C, a.W);
  e = cudaMemsetAsync(ws, 0, need, st);
  if (e != cudaSuccess) return gms_fail(e, "gms workspace reset");
  e = cudaLaunchKernelEx(&cfg, gmc_run_kernel, a, C);
  if (e != cudaSuccess) return gms_fail(e, "gmc_run_kernel launch");
  return DRIFT_PT_OK;
}

}  // namespace
}  // namespace dpt

using namespace dpt;

extern "C" int drift_pt_gms_workspace_bytes(int32_t n_words, size_t* bytes) {
  clear_error();
  if (n_words < 1 || n_words > 64 || !bytes) return set_error(DRIFT_PT_EINVAL, "gms_workspace_bytes");
  const size_t half = ((size_t)16 * 32 * n_words + 255) & ~(size_t)255;
  *bytes = 256 + 2 * half;
  return DRIFT_PT_OK;
}

extern "C" int drift_pt_gms_init(const DriftPtGmsProblem* problem, const DriftPtGmsRunArgs* args,
                                 DriftPtGmsState* state, void* stream) {
  clear_error();
  GmsArgs a;
  int rc = gms_args(problem, args, state, a);
  if (rc) return rc;
  gms_init_kernel<<<a.W, 256, 0, static_cast<cudaStream_t>(stream)>>>(a);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? DRIFT_PT_OK : gms_fail(e, "gms_init_kernel launch");
}

extern "C" int drift_pt_gms_run(const DriftPtGmsProblem* problem, const DriftPtGmsRunArgs* args, DriftPtGmsState* state,
                                void* workspace, size_t workspace_bytes, void* stream) {
  clear_error();
  GmsArgs a;
  int rc = gms_args(problem, args, state, a);
  if (rc) return rc;
  if (args->n_rounds < 0 || args->sweeps_per_round < 1 || args->round_offset < 0 || !args->betas || !args->thresholds)
    return set_error(DRIFT_PT_EINVAL, "gms: run arguments");
  size_t need = 0;
  drift_pt_gms_workspace_bytes(a.W, &need);
  if (!workspace || workspace_bytes < need) return set_error(DRIFT_PT_EINVAL, "gms: workspace too small");
  if (args->n_rounds == 0) return DRIFT_PT_OK;
  unsigned char* ws = static_cast<unsigned char*>(workspace);
  a.err = reinterpret_cast<int*>(ws + 8);
  const size_t half = ((size_t)16 * a.R + 255) & ~(size_t)255;
  a.pub = reinterpret_cast<long long*>(ws + 256);
  a.tags = reinterpret_cast<unsigned long long*>(ws + 256 + half);
  int dev = 0, optin = 0, sms = 0;
  cudaGetDevice(&dev);
  if (cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return set_error(DRIFT_PT_ECUDA, "cudaDeviceGetAttribute failed");
  GmsSmem L = gms_smem(a.n_pos, a.D, a.k, a.R, true);
  a.ell_in_smem = 1;
  if (L.total > (size_t)optin) {
    L = gms_smem(a.n_pos, a.D, a.k, a.R, false);
    a.ell_in_smem = 0;
    if (L.total > (size_t)optin)
      return set_error(DRIFT_PT_EUNSUPPORTED, "gms: %d positions do not fit one CTA's shared memory", a.n_pos);
  }
  int C = args->cluster_size;
  if (C < 0 || C > 16) return set_error(DRIFT_PT_EINVAL, "gms: cluster_size must be in 0..16");
  if (C == 0) {
    // automatic: with 16 or more words one CTA per word keeps enough SMs busy (measured on MaxCut 3-regular
    // N = 4096: 1024 replicas 202 vs 189 flips/ns with clusters of 4); with fewer words, the largest
    // cluster whose W clusters fit the SMs and whose shares stay balanced (64 replicas: 44.6 vs 16.8 flips/ns
    // with clusters of 16); a shape the device cannot hold falls through to smaller ones
    const int thr_c = args->threads_per_cta <= kGmcMaxThreads ? args->threads_per_cta : 0;
    for (int c = 16; c >= 2 && a.W < 16; c >>= 1) {
      if (a.W * c > sms || gmc_cap(a.n, a.k, c) * 2 > (a.n + c - 1) / c * 3) continue;
      rc = gmc_launch(a, c, thr_c, sms, optin, ws, need, static_cast<cudaStream_t>(stream));
      if (rc != DRIFT_PT_EUNSUPPORTED) return rc;
      clear_error();
    }
    C = 1;
  }
  if (C > 1) return gmc_launch(a, C, args->threads_per_cta, sms, optin, ws, need, static_cast<cudaStream_t>(stream));
  int threads = args->threads_per_cta;
  if (threads == 0) threads = kGmsThreads;
  if (threads < 32 || threads > kGmsThreads || threads % 32)
    return set_error(DRIFT_PT_EINVAL, "gms: threads_per_cta must be a multiple of 32 in [32, %d]", kGmsThreads);
  int per_sm = 0;
  rc = prepare_kernel((const void*)gms_run_kernel, threads, L.total, &per_sm);
  if (rc) return rc;
  if (per_sm < 1 || a.W > per_sm * sms) return set_error(DRIFT_PT_EUNSUPPORTED, "gms: %d CTAs cannot be co-resident", a.W);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemsetAsync(ws, 0, need, st);
  if (e != cudaSuccess) return gms_fail(e, "gms workspace reset");
  cudaLaunchConfig_t cfg;
  std::memset(&cfg, 0, sizeof cfg);
  cfg.gridDim = dim3(a.W);
  cfg.blockDim = dim3(threads);
  cfg.dynamicSmemBytes = L.total;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  void* kargs[] = {&a};
  e = cudaLaunchKernelExC(&cfg, (const void*)gms_run_kernel, kargs);
  if (e != cudaSuccess) return gms_fail(e, "gms_run_kernel launch");
  return DRIFT_PT_OK;
}
