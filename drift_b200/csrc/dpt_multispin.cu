// dpt_multispin.cu - bit-packed (multispin) parallel tempering on +-J cubic lattices.
//
// 32 replicas share one 32-bit word per site (bit b of word w = replica slot 32w + b). For a site
// the unsatisfied-bond count k_b of every bit is built with bit-sliced full adders from the
// neighbours' words; a flip of replica b costs dE = 4 (d - k_b) on a d-dimensional lattice and is
// always accepted when k_b >= d. The other bits compare their uniform u_b with the threshold of
// their rung, bit-sliced and most significant bit first: random bit-plane p (one Philox word) and
// threshold plane p (bit p of every bit's threshold) decide every bit where they differ, so about
// seven planes settle all 32 bits. The decision equals the full 32-bit comparison u_b < thr_b.
//
// One persistent cooperative launch per call: colour phases separated by bounded grid barriers;
// at each round end the replica energies are recomputed exactly (unsatisfied bonds counted with
// ballots), per-replica bests updated, and the adjacent-rung exchange step evaluated redundantly in
// every CTA. Sites are split by colour (q = c N/2 + h), so a phase reads and writes contiguous words.
#include <climits>
#include <cuda_runtime.h>

#include <cstring>

#include "../../include/drift_pt.h"
#include "dpt_common.cuh"
#include "dpt_internal.h"

namespace dpt {

// n / d for 32-bit n: the high 64 bits of n * m with m = floor((2^64 - 1) / d) + 1 (exact for
// every 32-bit n and d >= 2, since n * d < 2^64); d == 1 is the identity.
struct FastDiv {
  unsigned long long m;
  unsigned int d;
};

__host__ __device__ inline FastDiv make_fastdiv(unsigned int d) {
  FastDiv f;
  f.d = d;
  f.m = d > 1 ? (~0ull / d) + 1ull : 0ull;
  return f;
}

__device__ __forceinline__ unsigned int fdiv(unsigned int n, const FastDiv& f) {
  return f.d == 1 ? n : (unsigned int)__umul64hi((unsigned long long)n, f.m);
}

struct MsArgs {
  int dims, L, W, R, half, n_sites;  // half = L/2, n_sites = L^dims
  FastDiv div_half, div_L;
  const uint8_t* jneg;
  int n_rounds, spr;
  long long round0;
  uint32_t k0, k1, inst;
  const double* betas;
  const uint32_t* thr;  // [R][2*dims]
  uint32_t* words;
  uint32_t* best_words;
  long long* energy;
  long long* best_energy;
  int* rung_of_slot;
  int* slot_of_rung;
  long long* tried;
  long long* accepted;
  unsigned long long* bar;
  int* err;
  unsigned long long* ecnt;  // [2][R] unsatisfied-bond counters by round parity
  long long timeout_ns;
};

struct MsSmem {
  size_t planes, eall, rung, slot, beta, thr, ebest, cnt, imp, stats, ctl, total;
};

__host__ __device__ inline MsSmem ms_smem(int W, int R, int dims) {
  MsSmem L;
  size_t o = 0;
  auto al = [](size_t x) { return (x + 15) & ~(size_t)15; };
  L.planes = o; o = al(o + 4 * (size_t)W * dims * 32);
  L.eall = o;   o = al(o + 8 * (size_t)R);
  L.rung = o;   o = al(o + 4 * (size_t)R);
  L.slot = o;   o = al(o + 4 * (size_t)R);
  L.beta = o;   o = al(o + 8 * (size_t)R);
  L.thr = o;    o = al(o + 4 * (size_t)R * 2 * dims);
  L.ebest = o;  o = al(o + 8 * (size_t)R);
  L.cnt = o;    o = al(o + 4 * (size_t)R);
  L.imp = o;    o = al(o + 4 * (size_t)W);
  L.stats = o;  o = al(o + 8 * (size_t)(R > 1 ? R - 1 : 0));
  L.ctl = o;    o = al(o + 16);
  L.total = o;
  return L;
}

__device__ __forceinline__ unsigned long long ms_timer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ unsigned long long ms_ld_acquire(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ int ms_ld_relaxed(const int* p) {
  int v;
  asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ bool ms_grid_sync(const MsArgs& a, unsigned long long k, int* flag) {
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    atomicAdd(a.bar, 1ULL);
    const unsigned long long target = k * gridDim.x;
    const unsigned long long t0 = ms_timer();
    int abort_now = 0;
    while (ms_ld_acquire(a.bar) < target) {
      if (ms_ld_relaxed(a.err) != 0) { abort_now = 1; break; }
      if (ms_timer() - t0 > (unsigned long long)a.timeout_ns) {
        atomicExch(a.err, DRIFT_PT_ETIMEOUT);
        abort_now = 1;
        break;
      }
    }
    *flag = abort_now;
  }
  __syncthreads();
  return *flag == 0;
}

// Colour-split index of the neighbour of colour-c site (x, y, z) displaced by +-1 along `dir`.
struct Coord {
  int x, y, z;
};

__device__ __forceinline__ Coord ms_coord(const MsArgs& a, int c, int h) {
  Coord p;
  const int rest = (int)fdiv((unsigned)h, a.div_half);
  const int xh = h - rest * a.half;
  if (a.dims == 3) {
    p.z = (int)fdiv((unsigned)rest, a.div_L);
    p.y = rest - p.z * a.L;
  } else {
    p.y = rest;
    p.z = 0;
  }
  p.x = 2 * xh + ((p.y + p.z + c) & 1);
  return p;
}

__device__ __forceinline__ int ms_q(const MsArgs& a, int x, int y, int z) {
  const int c = (x + y + z) & 1;
  return c * (a.n_sites / 2) + (x >> 1) + a.half * (y + a.L * z);
}

// Bit-sliced sum of the unsatisfied-bond words: k = k0 + 2 k1 + 4 k2 per bit (up to 6 inputs).
__device__ __forceinline__ void ms_count(const uint32_t* u, int nb, uint32_t& k0, uint32_t& k1, uint32_t& k2) {
  uint32_t s1 = u[0] ^ u[1] ^ u[2];
  uint32_t c1 = (u[0] & u[1]) | (u[2] & (u[0] ^ u[1]));
  if (nb == 4) {
    // 4 inputs: (u0+u1+u2) + u3
    k0 = s1 ^ u[3];
    const uint32_t t = s1 & u[3];
    k1 = c1 ^ t;
    k2 = c1 & t;
    return;
  }
  const uint32_t s2 = u[3] ^ u[4] ^ u[5];
  const uint32_t c2 = (u[3] & u[4]) | (u[5] & (u[3] ^ u[4]));
  k0 = s1 ^ s2;
  const uint32_t t = s1 & s2;
  k1 = c1 ^ c2 ^ t;
  k2 = (c1 & c2) | (t & (c1 ^ c2));
}

__global__ void __launch_bounds__(256) ms_init_kernel(MsArgs a) {
  const long long total = (long long)a.W * a.n_sites;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const int w = (int)(i / a.n_sites), q = (int)(i - (long long)w * a.n_sites);
    const U4 r = philox(U4{(uint32_t)q, 0u, (uint32_t)w, ctr3(kTagMsInit, a.inst)}, a.k0, a.k1);
    a.words[i] = r.x;
    a.best_words[i] = r.x;
  }
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.R; i += gridDim.x * blockDim.x) {
    a.rung_of_slot[i] = i;
    a.slot_of_rung[i] = i;
    a.energy[i] = 0;
    if (i < a.R - 1) {
      a.tried[i] = 0;
      a.accepted[i] = 0;
    }
  }
}

// Unsatisfied bonds of every replica (each site's positive-direction bonds), added into cnt[R].
__device__ void ms_count_unsat(const MsArgs& a, unsigned int* cnt_sm) {
  const int lane = threadIdx.x & 31;
  const long long warps_total = (long long)gridDim.x * (blockDim.x >> 5);
  const long long gw = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int blocks_per_word = (a.n_sites + 31) / 32;
  for (long long task = gw; task < (long long)a.W * blocks_per_word; task += warps_total) {
    const int w = (int)(task / blocks_per_word);
    const int q = (int)(task - (long long)w * blocks_per_word) * 32 + lane;
    uint32_t u[3] = {0u, 0u, 0u};
    if (q < a.n_sites) {
      const int c = q >= a.n_sites / 2;
      const Coord p = ms_coord(a, c, q - c * (a.n_sites / 2));
      const uint32_t s = __ldcg(a.words + (size_t)w * a.n_sites + q);
      const uint8_t jb = a.jneg[q];
      const int xp = p.x + 1 == a.L ? 0 : p.x + 1, yp = p.y + 1 == a.L ? 0 : p.y + 1;
      u[0] = s ^ __ldcg(a.words + (size_t)w * a.n_sites + ms_q(a, xp, p.y, p.z)) ^ ((jb & 1) ? ~0u : 0u);
      u[1] = s ^ __ldcg(a.words + (size_t)w * a.n_sites + ms_q(a, p.x, yp, p.z)) ^ ((jb & 2) ? ~0u : 0u);
      if (a.dims == 3) {
        const int zp = p.z + 1 == a.L ? 0 : p.z + 1;
        u[2] = s ^ __ldcg(a.words + (size_t)w * a.n_sites + ms_q(a, p.x, p.y, zp)) ^ ((jb & 4) ? ~0u : 0u);
      }
    }
    unsigned int mine = 0;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      if (d >= a.dims) break;
#pragma unroll 4
      for (int b = 0; b < 32; ++b) {
        const unsigned int v = __ballot_sync(0xffffffffu, (u[d] >> b) & 1u);
        if (lane == b) mine += __popc(v);
      }
    }
    if (mine) atomicAdd(cnt_sm + w * 32 + lane, mine);
  }
}

__global__ void __launch_bounds__(256) ms_energy_kernel(MsArgs a) {
  extern __shared__ unsigned int ms_cnt[];
  for (int i = threadIdx.x; i < a.R; i += blockDim.x) ms_cnt[i] = 0;
  __syncthreads();
  ms_count_unsat(a, ms_cnt);
  __syncthreads();
  const long long bonds = (long long)a.dims * a.n_sites;
  for (int i = threadIdx.x; i < a.R; i += blockDim.x)
    if (ms_cnt[i]) atomicAdd(reinterpret_cast<unsigned long long*>(a.energy + i), (unsigned long long)ms_cnt[i]);
  (void)bonds;
}

__global__ void ms_energy_finalize(MsArgs a) {
  const long long bonds = (long long)a.dims * a.n_sites;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.R; i += gridDim.x * blockDim.x) {
    const long long e = 2 * a.energy[i] - bonds;  // E = -sum J s s = 2 U - bonds
    a.energy[i] = e;
    a.best_energy[i] = e;
  }
}

__global__ void __launch_bounds__(256) ms_run_kernel(const MsArgs a) {
  extern __shared__ __align__(16) unsigned char ms_smem_raw[];
  const MsSmem L = ms_smem(a.W, a.R, a.dims);
  uint32_t* planes = reinterpret_cast<uint32_t*>(ms_smem_raw + L.planes);
  long long* eall = reinterpret_cast<long long*>(ms_smem_raw + L.eall);
  int* rung_sm = reinterpret_cast<int*>(ms_smem_raw + L.rung);
  int* slot_sm = reinterpret_cast<int*>(ms_smem_raw + L.slot);
  double* beta_sm = reinterpret_cast<double*>(ms_smem_raw + L.beta);
  uint32_t* thr_sm = reinterpret_cast<uint32_t*>(ms_smem_raw + L.thr);
  long long* ebest = reinterpret_cast<long long*>(ms_smem_raw + L.ebest);
  unsigned int* cnt_sm = reinterpret_cast<unsigned int*>(ms_smem_raw + L.cnt);
  uint32_t* imp = reinterpret_cast<uint32_t*>(ms_smem_raw + L.imp);
  int* stats = reinterpret_cast<int*>(ms_smem_raw + L.stats);
  int* ctl = reinterpret_cast<int*>(ms_smem_raw + L.ctl);
  const int tid = threadIdx.x, B = blockDim.x, R = a.R, W = a.W, dims = a.dims;
  const int F = 2 * dims;
  for (int i = tid; i < R; i += B) {
    rung_sm[i] = a.rung_of_slot[i];
    slot_sm[i] = a.slot_of_rung[i];
    beta_sm[i] = a.betas[i];
    ebest[i] = a.best_energy[i];
  }
  for (int i = tid; i < R * F; i += B) thr_sm[i] = a.thr[i];
  for (int i = tid; i < R - 1; i += B) stats[2 * i] = stats[2 * i + 1] = 0;
  auto rebuild_planes = [&]() {
    // planes[(w * dims + k) * 32 + p], bit b = bit (31 - p) of thr[rung(32w + b)][x_k - 1],
    // x_k = 2 (dims - k): the threshold of class k (k unsatisfied bonds) at the bit's rung
    for (int i = tid; i < W * dims * 32; i += B) {
      const int p = i & 31, wk = i >> 5, k = wk % dims, w = wk / dims;
      const int x = 2 * (dims - k);
      uint32_t v = 0;
      for (int b = 0; b < 32; ++b) {
        const uint32_t t = thr_sm[rung_sm[32 * w + b] * F + x - 1];
        v |= ((t >> (31 - p)) & 1u) << b;
      }
      planes[i] = v;
    }
  };
  __syncthreads();
  rebuild_planes();
  __syncthreads();
  const int n2 = a.n_sites / 2;
  const int gtid = blockIdx.x * B + tid, gsz = gridDim.x * B;
  const int lane = tid & 31;
  const uint32_t cms = ctr3(kTagMsSweep, a.inst);
  unsigned long long nsync = 0;
  for (int i = tid; i < R; i += B) cnt_sm[i] = 0;
  __syncthreads();
  for (int j = 0; j < a.n_rounds; ++j) {
    const long long round = a.round0 + j;
    for (int sw = 0; sw < a.spr; ++sw) {
      const uint32_t t = (uint32_t)(round * a.spr + sw);
      for (int c = 0; c < 2; ++c) {
        // the round's last phase also counts, per replica, the unsatisfied bonds of every colour-1
        // site after its update: each bond has exactly one colour-1 end, so the sum is the total
        const bool count = (sw == a.spr - 1) && (c == 1);
        for (int w = 0; w < W; ++w) {
          uint32_t* wb = a.words + (size_t)w * a.n_sites;
          const uint32_t* pl = planes + (w * dims) * 32;
          uint32_t cs[16];
#pragma unroll
          for (int p = 0; p < 16; ++p) cs[p] = 0u;
          for (int h = gtid; h < n2; h += gsz) {
            const Coord p = ms_coord(a, c, h);
            const int q = c * n2 + h;
            const uint32_t s = __ldcg(wb + q);
            const int xp = p.x + 1 == a.L ? 0 : p.x + 1, xm = p.x == 0 ? a.L - 1 : p.x - 1;
            const int yp = p.y + 1 == a.L ? 0 : p.y + 1, ym = p.y == 0 ? a.L - 1 : p.y - 1;
            const uint8_t jb = __ldg(a.jneg + q);
            const int q_xm = ms_q(a, xm, p.y, p.z), q_ym = ms_q(a, p.x, ym, p.z);
            uint32_t u[6];
            u[0] = s ^ __ldcg(wb + ms_q(a, xp, p.y, p.z)) ^ ((jb & 1) ? ~0u : 0u);
            u[1] = s ^ __ldcg(wb + q_xm) ^ ((__ldg(a.jneg + q_xm) & 1) ? ~0u : 0u);
            u[2] = s ^ __ldcg(wb + ms_q(a, p.x, yp, p.z)) ^ ((jb & 2) ? ~0u : 0u);
            u[3] = s ^ __ldcg(wb + q_ym) ^ ((__ldg(a.jneg + q_ym) & 2) ? ~0u : 0u);
            if (dims == 3) {
              const int zp = p.z + 1 == a.L ? 0 : p.z + 1, zm = p.z == 0 ? a.L - 1 : p.z - 1;
              const int q_zm = ms_q(a, p.x, p.y, zm);
              u[4] = s ^ __ldcg(wb + ms_q(a, p.x, p.y, zp)) ^ ((jb & 4) ? ~0u : 0u);
              u[5] = s ^ __ldcg(wb + q_zm) ^ ((__ldg(a.jneg + q_zm) & 4) ? ~0u : 0u);
            }
            uint32_t k0, k1, k2;
            ms_count(u, 2 * dims, k0, k1, k2);
            // class masks: m[k] for the k < dims classes that need a test
            uint32_t m[3];
            m[0] = ~(k0 | k1 | k2);
            m[1] = k0 & ~k1 & ~k2;
            m[2] = ~k0 & k1 & ~k2;
            const uint32_t need = dims == 3 ? (m[0] | m[1] | m[2]) : (m[0] | m[1]);
            uint32_t lt = 0, und = need;
            for (int ch = 0; ch < 8 && und; ++ch) {
              const U4 r = philox(U4{(uint32_t)q, t, ((uint32_t)w << 8) | (uint32_t)ch, cms}, a.k0, a.k1);
              const uint32_t rw[4] = {r.x, r.y, r.z, r.w};
#pragma unroll
              for (int i = 0; i < 4; ++i) {
                const int pp = ch * 4 + i;
                uint32_t tp = (m[0] & pl[pp]) | (m[1] & pl[32 + pp]);
                if (dims == 3) tp |= m[2] & pl[64 + pp];
                lt |= und & ~rw[i] & tp;
                und &= ~(rw[i] ^ tp);
              }
            }
            const uint32_t acc = (~need) | lt;
            wb[q] = s ^ acc;
            if (count) {
              // unsatisfied bonds after the update: 2d - k where the bit flipped, k otherwise
              uint32_t d0, d1, d2;
              if (dims == 3) {  // 6 - k
                d0 = k0;
                d1 = ~(k1 ^ k0);
                d2 = ~(k2 ^ (k1 & k0));
              } else {  // 4 - k
                d0 = k0;
                d1 = k1 ^ k0;
                d2 = ~(k2 ^ (k1 | k0));
              }
              const uint32_t add[3] = {(acc & d0) | (~acc & k0), (acc & d1) | (~acc & k1), (acc & d2) | (~acc & k2)};
#pragma unroll
              for (int b = 0; b < 3; ++b) {
                uint32_t v = add[b];
#pragma unroll
                for (int pp = b; pp < 16; ++pp) {
                  const uint32_t tcar = cs[pp] & v;
                  cs[pp] ^= v;
                  v = tcar;
                }
              }
            }
          }
          if (count) {
            // per-replica totals: bit b of plane p summed over the warp's lanes, weight 2^p
            unsigned int mine = 0;
#pragma unroll
            for (int pp = 0; pp < 16; ++pp) {
              if (!__any_sync(0xffffffffu, cs[pp] != 0u)) continue;
#pragma unroll 8
              for (int b = 0; b < 32; ++b) {
                const unsigned int v = __ballot_sync(0xffffffffu, (cs[pp] >> b) & 1u);
                if (lane == b) mine += (unsigned int)__popc(v) << pp;
              }
            }
            if (mine) atomicAdd(cnt_sm + w * 32 + lane, mine);
          }
        }
        if (count) {
          __syncthreads();
          unsigned long long* ec = a.ecnt + (size_t)(round & 1) * R;
          for (int i = tid; i < R; i += B) {
            if (cnt_sm[i]) atomicAdd(ec + i, (unsigned long long)cnt_sm[i]);
            cnt_sm[i] = 0;
          }
        }
        if (!ms_grid_sync(a, ++nsync, ctl)) return;
      }
    }
    // ---- round end: exact energies from the unsatisfied-bond counts ----
    unsigned long long* ec = a.ecnt + (size_t)(round & 1) * R;
    const long long bonds = (long long)dims * a.n_sites;
    for (int i = tid; i < R; i += B) eall[i] = 2 * (long long)__ldcg(ec + i) - bonds;
    for (int i = tid; i < W; i += B) imp[i] = 0;
    __syncthreads();
    for (int i = tid; i < R; i += B)
      if (eall[i] < ebest[i]) {
        ebest[i] = eall[i];
        atomicOr(imp + (i >> 5), 1u << (i & 31));
      }
    if (blockIdx.x == 0)  // the other parity's counters start the next round at zero
      for (int i = tid; i < R; i += B) a.ecnt[(size_t)((round + 1) & 1) * R + i] = 0;
    __syncthreads();
    // best configurations: copy the improved replicas' bits
    for (int w = 0; w < W; ++w) {
      const uint32_t mk = imp[w];
      if (!mk) continue;
      uint32_t* bw = a.best_words + (size_t)w * a.n_sites;
      const uint32_t* cw = a.words + (size_t)w * a.n_sites;
      for (int q = gtid; q < a.n_sites; q += gsz) bw[q] = (__ldcg(bw + q) & ~mk) | (__ldcg(cw + q) & mk);
    }
    // exchange step (identical in every CTA)
    if (tid < 32) {
      const int parity = (int)(round & 1);
      for (int r = parity + 2 * tid; r + 1 < R; r += 64) {
        const int sa = slot_sm[r], sb = slot_sm[r + 1];
        const double delta = d_mul(d_sub(beta_sm[r], beta_sm[r + 1]), (double)(eall[sa] - eall[sb]));
        bool acc = delta >= 0.0;
        if (!acc) {
          const U4 u = philox(U4{(uint32_t)r, (uint32_t)round, (uint32_t)((unsigned long long)round >> 32),
                                 ctr3(kTagSwap, a.inst)}, a.k0, a.k1);
          acc = uniform53(u.x, u.y) < exp_neg_d(delta);
        }
        if (blockIdx.x == 0) {
          stats[2 * r] += 1;
          stats[2 * r + 1] += acc ? 1 : 0;
        }
        if (acc) {
          slot_sm[r] = sb;
          slot_sm[r + 1] = sa;
          rung_sm[sa] = r + 1;
          rung_sm[sb] = r;
        }
      }
    }
    __syncthreads();
    rebuild_planes();
    if (blockIdx.x == 0)
      for (int i = tid; i < R; i += B) {
        a.energy[i] = eall[i];
        a.best_energy[i] = ebest[i];
      }
    if (!ms_grid_sync(a, ++nsync, ctl)) return;
  }
  if (blockIdx.x == 0) {
    __syncthreads();
    for (int i = tid; i < R; i += B) {
      a.rung_of_slot[i] = rung_sm[i];
      a.slot_of_rung[i] = slot_sm[i];
    }
    for (int r = tid; r < R - 1; r += B) {
      a.tried[r] += stats[2 * r];
      a.accepted[r] += stats[2 * r + 1];
    }
  }
}

}  // namespace dpt

using namespace dpt;

namespace {

constexpr size_t kMsWsHeader = 256;  // barrier counter at 0, error flag at 8, counters from 256

int ms_fail(cudaError_t e, const char* what) { return set_error(DRIFT_PT_ECUDA, "%s: %s", what, cudaGetErrorString(e)); }

int ms_validate(const DriftPtLattice* lat, const DriftPtMsRunArgs* args, const DriftPtMsState* st) {
  if (!lat || !args || !st) return set_error(DRIFT_PT_EINVAL, "multispin: NULL argument");
  if ((lat->dims != 2 && lat->dims != 3) || lat->L < 4 || (lat->L & 1) || !lat->jneg)
    return set_error(DRIFT_PT_EINVAL, "multispin: dims must be 2 or 3 and L even >= 4");
  long long n = 1;
  for (int d = 0; d < lat->dims; ++d) n *= lat->L;
  if (n > (1LL << 30)) return set_error(DRIFT_PT_EUNSUPPORTED, "multispin: lattice too large");
  if (args->n_words < 1 || args->n_words > 64) return set_error(DRIFT_PT_EINVAL, "multispin: 1..64 words of 32 replicas");
  if (args->instance > kMaxInstance) return set_error(DRIFT_PT_EINVAL, "instance must be < 2^24");
  if (!args->betas || !args->thresholds) return set_error(DRIFT_PT_EINVAL, "multispin: betas and thresholds required");
  if (!st->words || !st->best_words || !st->energy || !st->best_energy || !st->rung_of_slot || !st->slot_of_rung ||
      !st->swap_tried || !st->swap_accepted)
    return set_error(DRIFT_PT_EINVAL, "multispin: state arrays missing");
  return DRIFT_PT_OK;
}

MsArgs ms_args(const DriftPtLattice* lat, const DriftPtMsRunArgs* r, DriftPtMsState* s) {
  MsArgs a;
  std::memset(&a, 0, sizeof a);
  a.dims = lat->dims;
  a.L = lat->L;
  a.W = r->n_words;
  a.R = 32 * r->n_words;
  a.half = lat->L / 2;
  a.n_sites = lat->L * lat->L * (lat->dims == 3 ? lat->L : 1);
  a.div_half = make_fastdiv((unsigned)a.half);
  a.div_L = make_fastdiv((unsigned)lat->L);
  a.jneg = lat->jneg;
  a.n_rounds = r->n_rounds;
  a.spr = r->sweeps_per_round;
  a.round0 = r->round_offset;
  a.k0 = (uint32_t)(r->seed & 0xffffffffu);
  a.k1 = (uint32_t)(r->seed >> 32);
  a.inst = r->instance;
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
  return a;
}

}  // namespace

extern "C" int drift_pt_ms_workspace_bytes(int32_t n_words, size_t* bytes) {
  clear_error();
  if (n_words < 1 || !bytes) return set_error(DRIFT_PT_EINVAL, "ms_workspace_bytes: invalid arguments");
  *bytes = kMsWsHeader + 2 * 8 * 32 * (size_t)n_words;
  return DRIFT_PT_OK;
}

extern "C" int drift_pt_ms_init(const DriftPtLattice* lat, const DriftPtMsRunArgs* args, DriftPtMsState* state,
                                void* stream) {
  clear_error();
  int rc = ms_validate(lat, args, state);
  if (rc) return rc;
  MsArgs a = ms_args(lat, args, state);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  ms_init_kernel<<<1184, 256, 0, st>>>(a);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return ms_fail(e, "ms_init_kernel");
  ms_energy_kernel<<<592, 256, sizeof(unsigned int) * a.R, st>>>(a);
  e = cudaGetLastError();
  if (e != cudaSuccess) return ms_fail(e, "ms_energy_kernel");
  ms_energy_finalize<<<(a.R + 255) / 256, 256, 0, st>>>(a);
  e = cudaGetLastError();
  if (e != cudaSuccess) return ms_fail(e, "ms_energy_finalize");
  return DRIFT_PT_OK;
}

extern "C" int drift_pt_ms_run(const DriftPtLattice* lat, const DriftPtMsRunArgs* args, DriftPtMsState* state,
                               void* workspace, size_t workspace_bytes, void* stream) {
  clear_error();
  int rc = ms_validate(lat, args, state);
  if (rc) return rc;
  if (args->n_rounds < 0 || args->sweeps_per_round < 1 || args->round_offset < 0)
    return set_error(DRIFT_PT_EINVAL, "multispin run args");
  size_t need = 0;
  drift_pt_ms_workspace_bytes(args->n_words, &need);
  if (!workspace || workspace_bytes < need) return set_error(DRIFT_PT_EINVAL, "multispin: workspace too small");
  if (args->n_rounds == 0) return DRIFT_PT_OK;
  MsArgs a = ms_args(lat, args, state);
  unsigned char* ws = static_cast<unsigned char*>(workspace);
  a.bar = reinterpret_cast<unsigned long long*>(ws);
  a.err = reinterpret_cast<int*>(ws + 8);
  a.ecnt = reinterpret_cast<unsigned long long*>(ws + kMsWsHeader);
  a.timeout_ns = (long long)((args->timeout_s > 0 ? args->timeout_s : 10.0) * 1e9);
  const MsSmem L = ms_smem(a.W, a.R, a.dims);
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return set_error(DRIFT_PT_ECUDA, "cudaDeviceGetAttribute failed");
  const int threads = 256;
  int per_sm = 0;
  rc = prepare_kernel((const void*)ms_run_kernel, threads, L.total, &per_sm);
  if (rc) return rc;
  if (per_sm < 1) return set_error(DRIFT_PT_EUNSUPPORTED, "multispin kernel does not fit an SM");
  const int want = args->ctas_per_sm > 0 ? args->ctas_per_sm : 2;  // fewer CTAs: cheaper grid barriers
  per_sm = per_sm < want ? per_sm : want;
  {
    // each thread's bit-sliced bond counter has 16 planes: its sites per word times 2d must stay below 2^16
    const long long threads_total = (long long)per_sm * sms * threads;
    const long long per_thread = (a.n_sites / 2 + threads_total - 1) / threads_total;
    if (per_thread * 2 * a.dims >= 65536) return set_error(DRIFT_PT_EUNSUPPORTED, "multispin: lattice too large for the grid");
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemsetAsync(ws, 0, need, st);
  if (e != cudaSuccess) return ms_fail(e, "workspace reset");
  cudaLaunchConfig_t cfg;
  std::memset(&cfg, 0, sizeof cfg);
  cfg.gridDim = dim3(per_sm * sms);
  cfg.blockDim = dim3(threads);
  cfg.dynamicSmemBytes = L.total;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  void* kargs[] = {&a};
  e = cudaLaunchKernelExC(&cfg, (const void*)ms_run_kernel, kargs);
  if (e != cudaSuccess) return ms_fail(e, "ms_run_kernel launch");
  return DRIFT_PT_OK;
}
