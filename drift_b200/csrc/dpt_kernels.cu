// dpt_kernels.cu - sm_100a kernels of the parallel-tempering engine.
//
// One persistent cooperative launch runs every round of a PT job (the reference launches a sweep
// kernel and a swap kernel per round from a host loop, cuda/ising_pt.cu:214-218):
//   * each CTA owns `rpc` replica slots; their int8 spins live in shared memory for the whole
//     launch, together with the coupling table when it fits (otherwise it is read through L1/L2);
//   * a sweep is one phase per colour class; within a phase every (slot, group of 8 consecutive
//     positions) item is independent, so threads take items in any order and results do not
//     depend on the launch shape;
//   * Metropolis acceptance uses counter-based Philox uniforms and, on the integer path, a
//     per-rung threshold table (no exp in the loop); energies are updated incrementally in exact
//     fixed point;
//   * after each round every CTA publishes its slots' energies, meets the others at a bounded
//     grid barrier, and all CTAs evaluate the same adjacent-rung exchange step redundantly.
#include <climits>
#include <cuda_runtime.h>

#include "../../include/drift_pt.h"
#include "dpt_common.cuh"
#include "dpt_internal.h"
#include "dpt_kernels.cuh"
#include "dpt_sweep.cuh"

namespace dpt {

__device__ __forceinline__ unsigned long long global_timer_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void st_release_u64(unsigned long long* p, unsigned long long v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ void st_relaxed_u64(unsigned long long* p, unsigned long long v) {
  asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

// Cluster form: the CTAs of one thread-block cluster hold the whole ladder. A round's energies stay
// in each CTA's shared memory; one cluster barrier (each thread's shared-memory writes released at
// cluster scope, an acquiring wait) orders them before the other CTAs read them.
__device__ __forceinline__ void cl_arrive_smem() {
  __syncwarp();  // the .aligned barrier wants the whole warp converged
  asm volatile("fence.release.sync_restrict::shared::cta.cluster;\n\tbarrier.cluster.arrive.relaxed.aligned;" ::: "memory");
}
__device__ __forceinline__ void cl_wait() {
  __syncwarp();
  asm volatile("barrier.cluster.wait.acquire.aligned;" ::: "memory");
}
__device__ __forceinline__ void cl_sync_full() {
  __syncwarp();
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}
__device__ __forceinline__ uint32_t cl_map(uint32_t saddr, uint32_t rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(saddr), "r"(rank));
  return r;
}
__device__ __forceinline__ long long cl_ld_s64(uint32_t caddr) {
  long long v;
  asm volatile("ld.shared::cluster.s64 %0, [%1];" : "=l"(v) : "r"(caddr) : "memory");
  return v;
}

// The swap test u < exp_neg_d(delta) for delta < 0, u in [0, 1). A single-precision estimate
// decides it when u lies clearly above or below: __expf's documented error is at most
// 2 + floor(1.173 |x|) ulp, with the rounding of delta to float below 2^-15.9 relative for
// |delta| <= 80, and the margin is 2^-12. Otherwise, and for u = 0, exp_neg_d decides, so the
// outcome is always that of u < exp_neg_d(delta). Below delta = -80, exp_neg_d(delta) < 2^-53, the
// smallest positive u.
__device__ __forceinline__ bool swap_accept(double u, double delta) {
  if (delta >= -80.0) {
    const double ef = (double)__expf((float)delta);
    if (u >= ef * (1.0 + 0x1p-12)) return false;
    if (u < ef * (1.0 - 0x1p-12)) return true;
  } else if (u > 0.0) {
    return false;
  }
  return u < exp_neg_d(delta);
}

// polls of a publication word between two reads of the error flag and the clock
constexpr int kPollCheck = 8;

__device__ __forceinline__ int ld_relaxed_i32(const int* p) {
  int v;
  asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// ---------------------------------------------------------------------------------------------
// One item: positions 8g .. 8g+7 of one replica slot; positions outside the colour range
// [lo, hi) are computed but never flipped. All gathers of the item are issued before the
// acceptance tests (W bounds the slice width at compile time; W = 0 walks it at run time).
// ---------------------------------------------------------------------------------------------
// kCluster: the grid is one cluster (CTA rank = blockIdx.x) and the round's energies are exchanged
// through distributed shared memory behind one cluster barrier instead of global memory.
// kUnitW > 0: the unit-regular form (every spin has kUnitW couplings of +-1, no field; one
// replica slot per CTA; P = 2 or 4 positions per item, up to kMaxUnitThreads threads): items read
// 16-bit neighbour addresses from a table staged at launch instead of gathering the sliced ELL,
// spins live as 0/1 bytes with a flipped copy, and each group's Philox block is computed once per
// sweep, a sweep ahead, into shared memory (item_unit).
// kPh: the unit-regular form's most colour phases (2 for bipartite problems, else kUnitPhases), so
// that a thread's per-phase state (item, Philox duty, neighbour-address row) takes no registers for
// phases the problem does not have.
template <bool kInt, bool kInSmem, int W, bool kExactW, bool kField, int P, bool kCluster, int kUnitW = 0,
          int kPh = kUnitPhases>
__global__ void __launch_bounds__(kUnitW > 0 ? unit_max_threads(P) : kMaxThreads, 1) pt_run_kernel(const PtKernelArgs a) {
  constexpr bool kUnit = kUnitW > 0;
  static_assert(kUnit || P == 8 || (kInt && (P == 4 || P == 1)), "positions per item");
  static_assert(!kUnit || (kInt && kInSmem && !kField && (P == 2 || P == 4)), "unit-regular form");
  constexpr int NB = kGroup / P;  // items per group
  unsigned char* smem = dpt_smem;
  const SmemLayout L = smem_layout(a.n_pos, a.rpc, a.R, a.F, a.n_colors, a.n_slices, a.n_ell, kInt, kInSmem,
                                   (int)blockDim.x, kCluster, kUnitW, kUnit ? P : 2);
  // bytes of one slot's spins in shared memory
  const uint32_t sp_stride = kUnit ? (uint32_t)unit_slot_bytes(a.n_pos) : (uint32_t)a.n_pos;
  long long* cpub = reinterpret_cast<long long*>(smem + L.cpub);
  int8_t* sp = reinterpret_cast<int8_t*>(smem + L.spins);
  long long* eacc = reinterpret_cast<long long*>(smem + L.eacc);
  long long* ecur = reinterpret_cast<long long*>(smem + L.ecur);
  long long* ebest = reinterpret_cast<long long*>(smem + L.ebest);
  int* imp = reinterpret_cast<int*>(smem + L.imp);
  long long* eall = reinterpret_cast<long long*>(smem + L.eall);
  int* rung_sm = reinterpret_cast<int*>(smem + L.rung);
  int* slot_sm = reinterpret_cast<int*>(smem + L.slot);
  double* beta_sm = reinterpret_cast<double*>(smem + L.beta);
  float* nb_sm = reinterpret_cast<float*>(smem + L.nb);
  uint32_t* thr_sm = reinterpret_cast<uint32_t*>(smem + L.thr);
  int* stats = reinterpret_cast<int*>(smem + L.stats);
  int* cptr = reinterpret_cast<int*>(smem + L.cptr);
  int* ctl = reinterpret_cast<int*>(smem + L.ctl);

  const int tid = threadIdx.x, B = blockDim.x;
  const int R = a.R, n_pos = a.n_pos;
  const int s0 = blockIdx.x * a.rpc;
  const int nloc = min(a.rpc, R - s0);

  // ---- stage state and tables ----
  if constexpr (kUnit) {
    // the storage word of each 4-position word (identity without a placement), then the spins:
    // +1 -> 0 and -1 -> 1 (the sign bit of each byte), the flipped copy, and 16 zero bytes
    uint16_t* place = reinterpret_cast<uint16_t*>(smem + L.h);
    for (int u = tid; u < n_pos / 4; u += B) place[u] = a.unit_place ? a.unit_place[u] : (uint16_t)u;
    __syncthreads();
    const uint32_t* src = reinterpret_cast<const uint32_t*>(a.spins + (size_t)s0 * n_pos);
    for (int i = tid; i < nloc * (n_pos / 4); i += B) {
      const int sl = i / (n_pos / 4), u = i - sl * (n_pos / 4);
      const uint32_t b = (src[i] >> 7) & 0x01010101u;
      unsigned char* base = smem + L.spins + (size_t)sl * sp_stride + 4 * (size_t)place[u];
      *reinterpret_cast<uint32_t*>(base) = b;
      *reinterpret_cast<uint32_t*>(base + n_pos) = b ^ 0x01010101u;
    }
    for (int i = tid; i < nloc; i += B)
      *reinterpret_cast<uint4*>(smem + L.spins + (size_t)i * sp_stride + 2 * n_pos) = make_uint4(0, 0, 0, 0);
  } else {
    const int4* src = reinterpret_cast<const int4*>(a.spins + (size_t)s0 * n_pos);
    int4* dst = reinterpret_cast<int4*>(sp);
    const int nv = nloc * n_pos / 16;
    for (int i = tid; i < nv; i += B) dst[i] = src[i];
  }
  for (int i = tid; i < nloc; i += B) {
    ecur[i] = a.energy[s0 + i];
    ebest[i] = a.best_energy[s0 + i];
    imp[i] = 0;
  }
  for (int i = tid; i < R; i += B) {
    rung_sm[i] = a.rung_of_slot[i];
    slot_sm[i] = a.slot_of_rung[i];
    beta_sm[i] = a.betas[i];
  }
  if constexpr (kUnit) {
    // decision table: entry (rung, b, k) = (x << 32) | threshold of x, x = (1 - 2b)(W - 2k)
    constexpr int row = 2 * (kUnitW + 1);
    unsigned long long* tab = reinterpret_cast<unsigned long long*>(smem + L.thr);
    for (int i = tid; i < R * row; i += B) {
      const int r = i / row, j = i - r * row, bb = j / (kUnitW + 1), kk = j - bb * (kUnitW + 1);
      const int x = (1 - 2 * bb) * (kUnitW - 2 * kk);
      const uint32_t th = x >= 1 ? a.thr[r * a.F + x - 1] : 0xFFFFFFFFu;
      tab[i] = ((unsigned long long)(uint32_t)x << 32) | th;
    }
  } else if constexpr (kInt) {
    // extended rows: entry x + F for x = -F..F; x <= 0 never reads its entry (always accepted)
    const int row = 2 * a.F + 1;
    for (int i = tid; i < R * row; i += B) {
      const int r = i / row, x = i - r * row - a.F;
      thr_sm[i] = x >= 1 ? a.thr[r * a.F + x - 1] : 0xFFFFFFFFu;
    }
  }
  for (int i = tid; i < 2 * (R - 1); i += B) stats[i] = 0;
  for (int i = tid; i <= a.n_colors; i += B) cptr[i] = a.color_ptr[i];
  Tables T;
  T.soff_o = (uint32_t)L.soff;
  T.ent_o = T.nbr_o = (uint32_t)L.nbr;
  T.wf_o = (uint32_t)L.w;
  T.h_o = (uint32_t)L.h;
  T.soff = a.slice_off;
  T.nbr = a.ell_nbr;
  T.w8 = static_cast<const int8_t*>(a.ell_w);
  T.wf = static_cast<const float*>(a.ell_w);
  T.h = a.h_pos;
  if constexpr (kUnit) {
    const uint16_t* place = reinterpret_cast<const uint16_t*>(smem + L.h);
    // neighbour-address rows, one per item of P positions: entry i W + d is the 16-bit address of
    // the byte neighbour d of position P item + i contributes, in the slot's b array (+1 coupling)
    // or b ^ 1 array (-1 coupling); padding entries (weight 0, on padding positions only) point at
    // the zero bytes behind the two arrays. The spins start at shared offset 0 (one slot per CTA),
    // so every address is below 2 n_pos + 16 <= 2^16.
    constexpr int RB = ((2 * P * kUnitW + 7) / 8) * 8;
    uint16_t* desc = reinterpret_cast<uint16_t*>(smem + L.nbr);
    const int8_t* w8 = static_cast<const int8_t*>(a.ell_w);
    const uint32_t base = (uint32_t)L.spins;
    for (int i = tid; i < kUnitW * n_pos; i += B) {
      const int p = i / kUnitW, d = i - p * kUnitW;
      const int S = p >> 8, lane = (p >> 3) & 31, q = p & 7;
      const long long e = (long long)(S * kUnitW + d) * kSlicePositions + q * 32 + lane;
      const int wt = w8[e];
      const uint32_t nq = (uint32_t)a.ell_nbr[e];
      const uint32_t at = wt == 0 ? base + 2u * (uint32_t)n_pos
                                  : base + (wt < 0 ? (uint32_t)n_pos : 0u) + 4u * place[nq >> 2] + (nq & 3u);
      desc[(size_t)(p / P) * (RB / 2) + (p % P) * kUnitW + d] = (uint16_t)at;
    }
    // the Philox blocks of the launch's first sweep (the items compute each later sweep's ahead)
    const uint32_t t0 = (uint32_t)(a.round0 * a.spr);
    uint4* ub = reinterpret_cast<uint4*>(smem + L.w + 16 * (size_t)(n_pos / kGroup) * (t0 & 1u));
    const uint32_t c_sw = ctr3(kTagSweep, a.inst);
    for (int g = tid; g < n_pos / kGroup; g += B) {
      const U4 u = philox(U4{(uint32_t)g, t0, (uint32_t)s0, c_sw}, a.k0, a.k1);
      ub[g] = make_uint4(u.x, u.y, u.z, u.w);
    }
  } else if constexpr (kInSmem) {
    int* soff_sm = reinterpret_cast<int*>(smem + L.soff);
    for (int i = tid; i <= a.n_slices; i += B) soff_sm[i] = a.slice_off[i];
    if constexpr (kInt) {
      // pack (neighbour position, int8 weight) into one word: one shared load per coupling
      uint32_t* ent_sm = reinterpret_cast<uint32_t*>(smem + L.nbr);
      const int8_t* w8 = static_cast<const int8_t*>(a.ell_w);
      for (int i = tid; i < (int)a.n_ell; i += B)
        ent_sm[i] = ((uint32_t)a.ell_nbr[i] << 8) | (uint32_t)(uint8_t)w8[i];
    } else {
      const int4* s4 = reinterpret_cast<const int4*>(a.ell_nbr);
      int4* d4 = reinterpret_cast<int4*>(smem + L.nbr);
      for (int i = tid; i < (int)(a.n_ell / 4); i += B) d4[i] = s4[i];
      const int4* w4 = reinterpret_cast<const int4*>(a.ell_w);
      int4* dw = reinterpret_cast<int4*>(smem + L.w);
      for (int i = tid; i < (int)(a.n_ell / 4); i += B) dw[i] = w4[i];
    }
    {
      const int4* s4 = reinterpret_cast<const int4*>(a.h_pos);
      int4* d4 = reinterpret_cast<int4*>(smem + L.h);
      for (int i = tid; i < n_pos / 4; i += B) d4[i] = s4[i];
    }
  }
  // Swap uniform of an exchange lane's first pair (parity + 2 lane, lanes 0..31) in round `rnd`: it
  // depends only on the pair and the round.
  auto swap_uniform = [&](long long rnd, int lane) -> double {
    const int pr = (int)(rnd & 1);
    if (pr + 2 * lane + 1 >= R) return 0.0;
    const U4 u = philox(U4{(uint32_t)(pr + 2 * lane), (uint32_t)rnd, (uint32_t)((unsigned long long)rnd >> 32),
                           ctr3(kTagSwap, a.inst)}, a.k0, a.k1);
    return uniform53(u.x, u.y);
  };
  // Unit-regular form with 3 or more warps: warp 2 draws the next round's swap uniforms while warp 0
  // runs this round's exchange, so they are ready in shared memory (by round parity) when needed.
  double* usw = reinterpret_cast<double*>(smem + L.usw);
  const bool unit_helper = kUnit && B >= 96;
  // Grid form with at most 64 slots (warp 0 polls the energies, warp 1 of CTA 0 keeps the history,
  // warp 2 draws the next swap uniforms): when the warps from 3 on have a thread for every group,
  // the Philox blocks of the next round's first sweep are computed by them while the round's
  // energies travel, instead of inside the last sweep's colour phases.
  // Compiled into the 4-phase instances only: in the 2-phase instance of 2-D EA L = 16 (24 replicas,
  // 96 threads, so never taken) its mere presence cost 7 %, while on MaxCut N = 4096 it gained 4.5 %.
  const bool unit_defer_px = kPh > 2 && unit_helper && !kCluster && gridDim.x > 1 && a.R <= 64 &&
                             B - 96 >= (a.n + kGroup - 1) / kGroup;
  if (unit_helper && (tid >> 5) == 2) usw[tid & 31] = swap_uniform(a.round0, tid & 31);
  if (tid == 0) {
    ctl[0] = 0;  // abort flag
    long long b = a.best_energy[0];
    for (int i = 1; i < R; ++i) b = min(b, a.best_energy[i]);
    reinterpret_cast<long long*>(ctl + 2)[0] = b;  // running best (CTA 0 uses it)
  }
  __syncthreads();
  if constexpr (!kInt)
    for (int i = tid; i < nloc; i += B) nb_sm[i] = -2.0f * (float)beta_sm[rung_sm[s0 + i]];
  __syncthreads();
  // unit-regular form (one slot per CTA): every thread keeps the slot's energy and best energy
  long long e_u = 0, eb_u = 0;
  if constexpr (kUnit) {
    e_u = ecur[0];
    eb_u = ebest[0];
  }

  // Thread -> slot binding: `tps` consecutive threads serve one slot for the whole launch, so each
  // thread keeps its slot's energy change in a register (no atomics in the sweep loop).
  const int tps = B / a.rpc;
  const int seg = seg_width(B, a.rpc);
  const int my_sl = tid / tps, lt = tid - my_sl * tps;
  const bool active = my_sl < nloc;
  const int my_slot = s0 + (active ? my_sl : 0);
  const uint32_t my_sp_o = (uint32_t)L.spins + (uint32_t)(active ? my_sl : 0) * sp_stride;
  const int k = a.n_colors;
  const uint32_t c_sweep = ctr3(kTagSweep, a.inst), c_second = ctr3(kTagSecond, a.inst);
  // Unit-regular form: each thread's work in each colour phase is the same every sweep, so it is
  // fixed here once: item lt of the class (item index | in-class mask << 14 | storage word of its
  // first position << 18 | 1 << 31, or 0: n_pos <= 32760 keeps the fields within 14 and 13 bits) and the
  // group whose next-sweep Philox block the thread computes (group + 1, or 0): the groups whose first
  // position lies in the class, taken by the CTA's last threads. (Moving all blocks to the phases
  // with the most idle threads instead measured slower on MaxCut N = 4096: the small phases became
  // issue-bound, while in the large phases the blocks overlap other warps' items. Spreading them
  // over every phase's threads without an item, so that no thread runs both, measured +0.2 %.) The
  // host makes the CTA wide enough for one item per thread and phase.
  // Rows of neighbour addresses of at most 16 bytes are kept in registers too (s_row).
  constexpr bool kRowReg = kUnit && unit_row_in_registers<kUnitW, P>();
  constexpr int kRB = ((2 * P * kUnitW + 7) / 8) * 8;
  uint32_t s_item[kPh], s_px[kPh];
  uint4 s_row[kPh];
#pragma unroll
  for (int c = 0; c < kPh; ++c) {
    s_item[c] = 0u;
    s_px[c] = 0u;
    s_row[c] = make_uint4(0u, 0u, 0u, 0u);
    if (kUnit && c < k) {
      const int lo = cptr[c], hi = cptr[c + 1];
      const int glo = lo >> 3, ghi = (hi + 7) >> 3;
      if (lt < (ghi - glo) * NB) {
        const uint32_t item = (uint32_t)(glo * NB + lt);
        const uint32_t msk = range_mask<P>((int)item * P, lo, hi);
        const uint32_t word = reinterpret_cast<const uint16_t*>(smem + L.h)[(item * P) >> 2];
        s_item[c] = msk ? (item | (msk << 14) | (word << 18) | 0x80000000u) : 0u;
        if constexpr (kRowReg) {
          const uint32_t row = (uint32_t)L.nbr + item * (uint32_t)kRB;
          if constexpr (kRB == 16) {
            s_row[c] = lds_u128(row);
          } else {
            const uint64_t v = lds_u64(row);
            s_row[c] = make_uint4((uint32_t)v, (uint32_t)(v >> 32), 0u, 0u);
          }
        }
      }
      const int gp = (lo + 7) / kGroup + (tps - 1 - lt);
      if (gp < (hi + 7) / kGroup) s_px[c] = (uint32_t)gp + 1u;
    }
  }
  // Grid form: publish slot s's energy of round `round` (tag round + 1) for every CTA.
  auto publish_energy = [&](long long round, int s, long long e) {
    const size_t at = (size_t)(round & 1) * R + s;
    if (a.packed) {
      // energy and round tag in one single-copy-atomic word: no ordering between two words needed
      st_relaxed_u64(reinterpret_cast<unsigned long long*>(a.pub) + at,
                     ((unsigned long long)(uint32_t)(round + 1) << 32) | (uint32_t)(int32_t)e);
    } else {
      // the energy, then (release-ordered after it) the round tag that readers poll
      __stcg(a.pub + at, e);
      st_release_u64(a.tags + at, (unsigned long long)round + 1ull);
    }
  };
  // Grid form: slot s's energy of round `round`, polled until its tag shows. Every wait is bounded
  // by the timeout; on expiry, or when another CTA has set the error flag, abort_now is set and
  // the value is not used. The clock and the error flag are read after the first unsuccessful poll
  // and then after every kPollCheck-th only: read after every poll they slowed the exchange
  // measurably (2-D EA L = 16 with 24 replicas: 3.3 against 3.65 attempts/ns).
  auto poll_energy = [&](long long round, int s, int& abort_now) -> long long {
    const size_t at = (size_t)(round & 1) * R + s;
    const unsigned long long want = (unsigned long long)round + 1ull;
    if (a.packed) {
      const unsigned long long* pw = reinterpret_cast<const unsigned long long*>(a.pub) + at;
      const uint32_t tag = (uint32_t)want;
      unsigned long long v = ld_relaxed_u64(pw);
      if ((uint32_t)(v >> 32) != tag) {
        const unsigned long long t0 = global_timer_ns();
        for (int it = 1; (uint32_t)((v = ld_relaxed_u64(pw)) >> 32) != tag; ++it) {
          if (it != 1 && it % kPollCheck != 0) continue;
          if (ld_relaxed_i32(a.err) != 0) { abort_now = 1; break; }
          if (global_timer_ns() - t0 > (unsigned long long)a.timeout_ns) {
            atomicExch(a.err, DRIFT_PT_ETIMEOUT);
            abort_now = 1;
            break;
          }
        }
      }
      return (long long)(int32_t)(uint32_t)v;
    }
    if (ld_acquire_u64(a.tags + at) < want) {
      const unsigned long long t0 = global_timer_ns();
      for (int it = 1; ld_acquire_u64(a.tags + at) < want; ++it) {
        if (it != 1 && it % kPollCheck != 0) continue;
        if (ld_relaxed_i32(a.err) != 0) { abort_now = 1; break; }
        if (global_timer_ns() - t0 > (unsigned long long)a.timeout_ns) {
          atomicExch(a.err, DRIFT_PT_ETIMEOUT);
          abort_now = 1;
          break;
        }
      }
    }
    return abort_now ? 0ll : __ldcg(a.pub + at);
  };
  // The decision of pair (r, r + 1) of round `round` between slots sa (rung r) and sb (rung r + 1)
  // with energy difference de = E(sa) - E(sb) and dbeta = beta_r - beta_{r+1}; u_first is the
  // uniform of the lane's first pair.
  auto decide_pair = [&](long long round, int r, int sa, int sb, long long de, double dbeta, double u_first) {
    const double ded = kInt ? (double)de : d_mul((double)de, kFloatEnergyScale);
    const double delta = d_mul(dbeta, ded);
    bool acc = delta >= 0.0;
    if (!acc) {
      double u = u_first;  // the first pair of the lane (r < 64)
      if (r >= 64) {
        const U4 w = philox(U4{(uint32_t)r, (uint32_t)round, (uint32_t)((unsigned long long)round >> 32),
                               ctr3(kTagSwap, a.inst)}, a.k0, a.k1);
        u = uniform53(w.x, w.y);
      }
      acc = swap_accept(u, delta);
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
  };
  // The exchange lane `tid` (< 32) of round `round`: its pairs parity + 2 tid, + 64, ...
  // `energy(slot)` reads a slot's energy of this round.
  auto exchange_lane = [&](long long round, double u_first, auto&& energy) {
    for (int r = (int)(round & 1) + 2 * tid; r + 1 < R; r += 64) {
      const int sa = slot_sm[r], sb = slot_sm[r + 1];
      decide_pair(round, r, sa, sb, energy(sa) - energy(sb), d_sub(beta_sm[r], beta_sm[r + 1]), u_first);
    }
  };
  // Grid form: the energies of slots sa and sb (none when sb < 0) of round `round`, both polled at
  // once (bounded as poll_energy).
  auto poll_pair = [&](long long round, int sa, int sb, long long& ea, long long& eb, int& abort_now) {
    if (!a.packed) {
      ea = poll_energy(round, sa, abort_now);
      eb = (abort_now || sb < 0) ? 0ll : poll_energy(round, sb, abort_now);
      return;
    }
    const unsigned long long* base = reinterpret_cast<const unsigned long long*>(a.pub) + (size_t)(round & 1) * R;
    const uint32_t tag = (uint32_t)(round + 1);
    unsigned long long va = ld_relaxed_u64(base + sa);
    unsigned long long vb = sb >= 0 ? ld_relaxed_u64(base + sb) : (unsigned long long)tag << 32;
    if ((uint32_t)(va >> 32) != tag || (uint32_t)(vb >> 32) != tag) {
      const unsigned long long t0 = global_timer_ns();
      for (int it = 1;; ++it) {
        const bool need_a = (uint32_t)(va >> 32) != tag, need_b = (uint32_t)(vb >> 32) != tag;
        if (!need_a && !need_b) break;
        if (need_a) va = ld_relaxed_u64(base + sa);
        if (need_b) vb = ld_relaxed_u64(base + sb);  // sb >= 0 here
        if (it != 1 && it % kPollCheck != 0) continue;
        if (ld_relaxed_i32(a.err) != 0) { abort_now = 1; break; }
        if (global_timer_ns() - t0 > (unsigned long long)a.timeout_ns) {
          atomicExch(a.err, DRIFT_PT_ETIMEOUT);
          abort_now = 1;
          break;
        }
      }
    }
    ea = (long long)(int32_t)(uint32_t)va;
    eb = (long long)(int32_t)(uint32_t)vb;
  };
  // the running best energy after round j (CTA 0, one whole warp)
  // (history_from takes each lane's minimum over the energies it read)
  auto history_from = [&](int j, long long m) {
    for (int off = 16; off > 0; off >>= 1) m = min(m, __shfl_xor_sync(0xffffffffu, m, off));
    if ((tid & 31) == 0) {
      long long* rb = reinterpret_cast<long long*>(ctl + 2);
      rb[0] = min(rb[0], m);
      a.best_hist[j] = kInt ? (double)rb[0] : d_mul((double)rb[0], kFloatEnergyScale);
    }
  };
  auto best_history = [&](int j, auto&& energy) {
    long long m = LLONG_MAX;
    for (int i = tid & 31; i < R; i += 32) m = min(m, (long long)energy(i));
    history_from(j, m);
  };
  for (int j = 0; j < a.n_rounds; ++j) {
    const long long round = a.round0 + j;
    long long dacc = 0;
    int dacc_u = 0;  // unit-regular form: |change| <= 2 W P per phase, spr <= 2^23 keeps it in 32 bits
    const uint32_t thr_o = kUnit ? (uint32_t)L.thr + 16u * (uint32_t)(rung_sm[my_slot] * (kUnitW + 1))
                           : kInt ? (uint32_t)L.thr + 4u * (uint32_t)(rung_sm[my_slot] * (2 * a.F + 1) + a.F) : 0u;
    // unit-regular form: the rung's thresholds of the positive x = W - 2j, entries (b = 0, k = j) of
    // its decision-table row, in registers for the round
    UnitThr uthr{};
    if constexpr (kUnit) {
#pragma unroll
      for (int jj = 0; jj < (kUnitW + 1) / 2; ++jj) uthr.t[jj] = lds_u32(thr_o + 8u * (uint32_t)jj);
    }
    const float neg2beta = kInt ? 0.0f : nb_sm[active ? my_sl : 0];
    // the class bounds never change during the launch: each phase reads the next phase's before
    // its barrier, so no shared load starts the phase after it
    int lo_n = cptr[0], hi_n = cptr[1];
    for (int sw = 0; sw < a.spr; ++sw) {
      const uint32_t t = (uint32_t)(round * a.spr + sw);
      if constexpr (kUnit) {
        // the static schedule: at most one item and one next-sweep Philox block per thread and phase.
        // The phase loop stays unrolled: a rolled loop (each phase's state picked by selects) ran
        // MaxCut N = 4096 at 79 against 112 attempts/ns.
        const uint32_t ng = (uint32_t)(n_pos / kGroup);
        const uint32_t ubuf = (uint32_t)L.w + 16u * ng * (t & 1u), unext = (uint32_t)L.w + 16u * ng * ((t + 1u) & 1u);
#pragma unroll
        for (int c = 0; c < kPh; ++c) {
          if (c < k) {
            if (s_px[c] && !(unit_defer_px && sw == a.spr - 1))
              unit_next_block(s_px[c] - 1u, t, (uint32_t)my_slot, unext, c_sweep, a.k0, a.k1);
            if (s_item[c] >> 31) {
              const uint32_t item = s_item[c] & 0x3FFFu;
              const uint32_t own_o = my_sp_o + 4u * ((s_item[c] >> 18) & 0x1FFFu) + ((item * P) & 3u);
              dacc_u += item_unit<kUnitW, P>(item, (s_item[c] >> 14) & 0xFu, t, (uint32_t)my_slot, own_o,
                                           own_o + (uint32_t)n_pos, (uint32_t)L.nbr, s_row[c], ubuf, uthr,
                                           c_second, a.k0, a.k1);
            }
            __syncthreads();
          }
        }
      } else {
        for (int c = 0; c < k; ++c) {
          const int lo = lo_n, hi = hi_n;
          {
            const int cn = c + 1 < k ? c + 1 : 0;
            lo_n = cptr[cn];
            hi_n = cptr[cn + 1];
          }
          const int glo = lo >> 3, ghi = (hi + 7) >> 3;
          {
            // item v -> (group, sub-block): 32 consecutive items are 32 consecutive groups (coalesced
            // coupling reads), the NB sub-blocks of those groups follow as the next 32-item runs
            const int span = ((ghi - glo + 31) >> 5) * 32 * NB;
            if (active) {
              for (int v = lt; v < span; v += tps) {
                const int b = (v >> 5) & (NB - 1);
                const int g = glo + (v / (32 * NB)) * 32 + (v & 31);
                if (g >= ghi) continue;
                if constexpr (kInt)
                  dacc += group_int<W, kExactW, kInSmem, kField, P>(g, b, lo, hi, t, (uint32_t)my_slot, my_sp_o, T,
                                                                    thr_o, c_sweep, c_second, a.k0, a.k1);
                else
                  dacc += group_f32<W, kExactW, kInSmem, kField>(g, lo, hi, t, (uint32_t)my_slot, my_sp_o, T,
                                                                 neg2beta, c_sweep, c_second, a.k0, a.k1);
              }
            }
          }
          __syncthreads();
        }
      }
    }
    // ---- round end ----
    if constexpr (kUnit) {
      // One slot per CTA. Each warp adds its threads' energy changes as two 32-bit sums, of the low
      // 16 bits and of the rest, so no sum can overflow; after one barrier every thread adds the
      // warps' sums itself and holds the slot's new energy. Integer sums: any order, the same bits.
      // (Storing the warps' sums before the last colour phase's barrier instead, to save this
      // barrier, measured slower: MaxCut N = 4096 111.6 -> 107.8, 2-D EA L = 16 3.88 -> 3.60.)
      const int lane = tid & 31, wid = tid >> 5;
      double u_first = 0.0;
      if (!unit_helper && tid < 32) u_first = swap_uniform(round, tid);
      {
        const int lo = __reduce_add_sync(0xffffffffu, dacc_u & 0xFFFF);
        const int hi = __reduce_add_sync(0xffffffffu, dacc_u >> 16);
        if (lane == 0) reinterpret_cast<int2*>(eacc)[wid] = make_int2(lo, hi);
      }
      __syncthreads();
      {
        const int2 pw = lane < (B >> 5) ? reinterpret_cast<const int2*>(eacc)[lane] : make_int2(0, 0);
        const int lo = __reduce_add_sync(0xffffffffu, pw.x), hi = __reduce_add_sync(0xffffffffu, pw.y);
        e_u += (long long)hi * 65536 + lo;
      }
      const bool improved = e_u < eb_u;
      if (improved) eb_u = e_u;
      if (tid == 0) {
        ecur[0] = e_u;
        ebest[0] = eb_u;
        if constexpr (kCluster) cpub[(round & 1) * a.rpc] = e_u;
        else if (gridDim.x > 1) publish_energy(round, s0, e_u);
        else eall[0] = e_u;
      }
      if (improved) {
        // the spins of the new best, from the 0/1 bytes in storage order (b -> 1 - 2b: 0 -> 0x01,
        // 1 -> 0xFF); the spins change again only after the round's last barrier
        const uint16_t* place = reinterpret_cast<const uint16_t*>(smem + L.h);
        uint32_t* dst = reinterpret_cast<uint32_t*>(a.best_spins + (size_t)s0 * n_pos);
        for (int i = tid; i < n_pos / 4; i += B)
          dst[i] = (*reinterpret_cast<const uint32_t*>(sp + 4 * (size_t)place[i]) * 0xFEu) ^ 0x01010101u;
      }
      if (unit_helper && tid < 32) u_first = usw[(j & 1) * 32 + tid];
      if constexpr (kCluster) {
        // one cluster barrier publishes this round's energies; the exchange and history warps read
        // them from their owners' shared memory
        cl_arrive_smem();
        cl_wait();
        const uint32_t cbase = (uint32_t)__cvta_generic_to_shared(cpub + (round & 1) * a.rpc);
        auto cl_energy = [&](int sl) {
          const int o = sl / a.rpc;
          return cl_ld_s64(cl_map(cbase + 8u * (uint32_t)(sl - o * a.rpc), (uint32_t)o));
        };
        if (tid < 32) exchange_lane(round, u_first, cl_energy);
        if (blockIdx.x == 0 && a.best_hist && wid == (B > 32 ? 1 : 0)) best_history(j, cl_energy);
      } else {
        // With at most 64 slots and 3 or more warps, warp 0 polls every slot's energy (lane l slots
        // l and l + 32, coalesced), hands each pair's lane its two energies by shuffles and decides
        // the pairs: no gather into shared memory and no barrier of the whole CTA. In CTA 0, warp 1
        // polls them as well for the best-energy history. Other shapes gather through shared memory.
        const bool direct = gridDim.x > 1 && R <= 64 && unit_helper;
        if (direct) {
          if (wid == 0) {
            const int r = (int)(round & 1) + 2 * lane;
            const bool has = r + 1 < R;
            const int sa = has ? slot_sm[r] : 0, sb = has ? slot_sm[r + 1] : 0;
            // read before polling: the polls' memory clobbers keep the compiler from moving it later
            const double dbeta = has ? d_sub(beta_sm[r], beta_sm[r + 1]) : 0.0;
            int abort_now = 0;
            long long e0 = 0, e1 = 0;
            poll_pair(round, lane < R ? lane : 0, lane + 32 < R ? lane + 32 : -1, e0, e1, abort_now);
            // an abort leaves the permutation of the last whole round
            if (__any_sync(0xffffffffu, abort_now)) {
              if (lane == 0) ctl[0] = 1;
            } else {
              const long long a0 = __shfl_sync(0xffffffffu, e0, sa & 31), a1 = __shfl_sync(0xffffffffu, e1, sa & 31);
              const long long b0 = __shfl_sync(0xffffffffu, e0, sb & 31), b1 = __shfl_sync(0xffffffffu, e1, sb & 31);
              if (has) decide_pair(round, r, sa, sb, (sa < 32 ? a0 : a1) - (sb < 32 ? b0 : b1), dbeta, u_first);
            }
          } else if (wid == 1 && blockIdx.x == 0 && a.best_hist) {
            int abort_now = 0;
            long long e0 = 0, e1 = 0;
            poll_pair(round, lane < R ? lane : 0, lane + 32 < R ? lane + 32 : -1, e0, e1, abort_now);
            if (!__any_sync(0xffffffffu, abort_now))
              history_from(j, min(lane < R ? e0 : LLONG_MAX, lane + 32 < R ? e1 : LLONG_MAX));
          }
        } else {
          if (gridDim.x > 1) {
            int abort_now = 0;
            for (int s = tid; s < R && !abort_now; s += B) {
              const long long e = poll_energy(round, s, abort_now);
              if (!abort_now) eall[s] = e;
            }
            if (abort_now) ctl[0] = 1;
          }
          __syncthreads();
          if (!ctl[0]) {
            if (tid < 32) exchange_lane(round, u_first, [&](int s) { return eall[s]; });
            if (blockIdx.x == 0 && a.best_hist && wid == (B > 32 ? 1 : 0)) best_history(j, [&](int s) { return eall[s]; });
          }
        }
      }
      if (unit_helper && wid == 2) usw[((j + 1) & 1) * 32 + lane] = swap_uniform(round + 1, lane);
      if (unit_defer_px && tid >= 96 && tid - 96 < (a.n + kGroup - 1) / kGroup) {
        // the next round's first sweep t + 1 = (round + 1) spr: its blocks, from this round's last sweep t
        const uint32_t tl = (uint32_t)(round * a.spr + a.spr - 1);
        const uint32_t ng = (uint32_t)(n_pos / kGroup);
        unit_next_block((uint32_t)(tid - 96), tl, (uint32_t)my_slot,
                        (uint32_t)L.w + 16u * ng * ((tl + 1u) & 1u), c_sweep, a.k0, a.k1);
      }
      __syncthreads();
      if (ctl[0]) break;
    } else {
      // The exchange lanes draw the swap uniform of their first pair now: its latency hides behind
      // the energy reduction.
      double u_first = 0.0;
      if (tid < 32) u_first = swap_uniform(round, tid);
      // reduce the energy change of each slot over its threads
      for (int off = seg >> 1; off > 0; off >>= 1) dacc += __shfl_xor_sync(0xffffffffu, dacc, off);
      if (lt % seg == 0) eacc[tid / seg] = dacc;
      __syncthreads();
      // a slot's nseg <= 32 partial sums are added by one warp (shuffles, not a serial chain of
      // shared loads); slots are spread over the warps. Integer sums: any order gives the same bits.
      const int nseg = tps / seg;
      for (int i = tid >> 5; i < nloc; i += B >> 5) {
        const int ln = tid & 31;
        long long part = ln < nseg ? eacc[i * nseg + ln] : 0ll;
        for (int off = 16; off > 0; off >>= 1) part += __shfl_xor_sync(0xffffffffu, part, off);
        if (ln == 0) {
          const long long e = ecur[i] + part;
          ecur[i] = e;
          imp[i] = (e < ebest[i]) ? 1 : 0;
          if (e < ebest[i]) ebest[i] = e;
          if constexpr (kCluster) cpub[(round & 1) * a.rpc + i] = e;
          else if (gridDim.x > 1) publish_energy(round, s0 + i, e);
        }
      }
      if constexpr (kCluster) {
        // one cluster barrier publishes this round's energies to the other CTAs and, being a
        // barrier of every thread of the cluster, orders this CTA's own round-end writes for all
        // its threads
        cl_arrive_smem();
        cl_wait();
      } else {
        __syncthreads();
      }
      {
        // copy the spins of every slot that reached a new best, all slots in one pass
        const int chunks = n_pos / 16;
        const int4* src = reinterpret_cast<const int4*>(sp);
        int4* dst = reinterpret_cast<int4*>(a.best_spins + (size_t)s0 * n_pos);
        for (int i = tid; i < nloc * chunks; i += B)
          if (imp[i / chunks]) dst[i] = src[i];
      }
      // cluster form: a slot's energy of this round, read from its owner's shared memory
      const uint32_t cbase = kCluster ? (uint32_t)__cvta_generic_to_shared(cpub + (round & 1) * a.rpc) : 0u;
      auto cl_energy = [&](int sl) {
        const int o = sl / a.rpc;
        return cl_ld_s64(cl_map(cbase + 8u * (uint32_t)(sl - o * a.rpc), (uint32_t)o));
      };
      if constexpr (kCluster) {
        // nothing to gather: the exchange and history warps read the energies they use directly
      } else if (gridDim.x > 1) {
        // gather every slot's energy of this round: the only grid-wide synchronisation of the round
        int abort_now = 0;
        for (int s = tid; s < R && !abort_now; s += B) {
          const long long e = poll_energy(round, s, abort_now);
          if (!abort_now) eall[s] = e;
        }
        if (abort_now) ctl[0] = 1;
        __syncthreads();
        if (ctl[0]) break;
      } else {
        for (int i = tid; i < R; i += B) eall[i] = ecur[i];
        __syncthreads();
      }
      // ---- exchange step: identical in every CTA (disjoint pairs, one lane per pair) ----
      if (tid < 32) {
        if constexpr (kCluster) exchange_lane(round, u_first, cl_energy);
        else exchange_lane(round, u_first, [&](int s) { return eall[s]; });
      }
      // best-energy history (CTA 0): warp 1 while warp 0 runs the exchange, or warp 0 after it
      if (blockIdx.x == 0 && a.best_hist && (tid >> 5) == (B > 32 ? 1 : 0)) {
        if constexpr (kCluster) best_history(j, cl_energy);
        else best_history(j, [&](int s) { return eall[s]; });
      }
      __syncthreads();
      if constexpr (!kInt) {
        for (int i = tid; i < nloc; i += B) nb_sm[i] = -2.0f * (float)beta_sm[rung_sm[s0 + i]];
        __syncthreads();
      }
    }
  }

  // ---- write back ----
  // cluster form: no CTA leaves while another may still read its last round's energies
  if constexpr (kCluster) cl_sync_full();
  __syncthreads();
  if constexpr (kUnit) {
    const uint16_t* place = reinterpret_cast<const uint16_t*>(smem + L.h);
    const int words = n_pos / 4;
    uint32_t* dst = reinterpret_cast<uint32_t*>(a.spins + (size_t)s0 * n_pos);
    for (int i = tid; i < nloc * words; i += B) {
      const int sl = i / words;
      const uint32_t v =
          *reinterpret_cast<const uint32_t*>(sp + (size_t)sl * sp_stride + 4 * (size_t)place[i - sl * words]);
      dst[i] = (v * 0xFEu) ^ 0x01010101u;
    }
  } else {
    const int4* src = reinterpret_cast<const int4*>(sp);
    int4* dst = reinterpret_cast<int4*>(a.spins + (size_t)s0 * n_pos);
    const int nv = nloc * n_pos / 16;
    for (int i = tid; i < nv; i += B) dst[i] = src[i];
  }
  for (int i = tid; i < nloc; i += B) {
    a.energy[s0 + i] = ecur[i];
    a.best_energy[s0 + i] = ebest[i];
  }
  if (blockIdx.x == 0) {
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

// ---------------------------------------------------------------------------------------------
// Initialisation
// ---------------------------------------------------------------------------------------------
__global__ void init_spins_kernel(int n, int n_pos, int R, uint32_t inst, uint32_t k0, uint32_t k1,
                                  int8_t* spins, int8_t* best_spins) {
  const int g = blockIdx.x * blockDim.x + threadIdx.x;
  const int slot = blockIdx.y;
  if (g * kGroup >= n_pos || slot >= R) return;
  uint64_t s8 = 0;
#pragma unroll
  for (int half = 0; half < 2; ++half) {
    const int p0 = g * kGroup + half * 4;
    const U4 u = philox(U4{(uint32_t)(p0 >> 2), 0u, (uint32_t)slot, ctr3(kTagInit, inst)}, k0, k1);
    const uint32_t w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int p = p0 + q;
      const uint8_t v = (p < n && (w[q] >> 31)) ? 0xFFu : 0x01u;
      s8 |= (uint64_t)v << (8 * (half * 4 + q));
    }
  }
  const size_t off = (size_t)slot * n_pos + (size_t)g * kGroup;
  *reinterpret_cast<uint64_t*>(spins + off) = s8;
  *reinterpret_cast<uint64_t*>(best_spins + off) = s8;
}

// Energy of every slot from its spins, in the engine's fixed point, with an order-independent
// int64 reduction (the integer path accumulates 2E, halved by the finalize kernel).
template <bool kInt>
__global__ void energy_fixed_kernel(PtKernelArgs a) {
  const int S = blockIdx.x, slot = blockIdx.y;
  const int lane = threadIdx.x & 31, q = threadIdx.x >> 5;  // 256 threads = one slice
  const int p = S * kSlicePositions + lane * kGroup + q;
  const int8_t* sp = a.spins + (size_t)slot * a.n_pos;
  const int w0 = a.slice_off[S], width = a.slice_off[S + 1] - w0;
  const long long base = (long long)w0 * kSlicePositions + lane;
  long long v = 0;
  if (p < a.n) {
    const int si = sp[p];
    if constexpr (kInt) {
      const int8_t* w = static_cast<const int8_t*>(a.ell_w);
      int f = 0;
      for (int d = 0; d < width; ++d) {
        const long long e = base + (long long)(d * kGroup + q) * 32;
        f += (int)w[e] * (int)sp[a.ell_nbr[e]];
      }
      const int hh = static_cast<const int*>(a.h_pos)[(long long)S * kSlicePositions + q * 32 + lane];
      v = (long long)si * (long long)(-f - 2 * hh);
    } else {
      const float* w = static_cast<const float*>(a.ell_w);
      float f = 0.0f;
      for (int d = 0; d < width; ++d) {
        const long long e = base + (long long)(d * kGroup + q) * 32;
        f = f_add(f, sp[a.ell_nbr[e]] > 0 ? w[e] : -w[e]);
      }
      const float hh = static_cast<const float*>(a.h_pos)[(long long)S * kSlicePositions + q * 32 + lane];
      float term = f_sub(f_mul(-0.5f, f), hh);
      if (si < 0) term = -term;
      v = f_to_ll_rn(f_mul(term, kFloatEnergyQuant));
    }
  }
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  __shared__ long long red[8];
  if (lane == 0) red[q] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    long long s = 0;
    for (int i = 0; i < 8; ++i) s += red[i];
    if (s != 0) atomicAdd(reinterpret_cast<unsigned long long*>(a.energy + slot), (unsigned long long)s);
  }
}

__global__ void init_finalize_kernel(int R, int halve, long long* energy, long long* best_energy,
                                     int* rung_of_slot, int* slot_of_rung, long long* tried,
                                     long long* accepted) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < R; i += gridDim.x * blockDim.x) {
    if (halve) energy[i] /= 2;  // exact: 2E is even for integer couplings
    best_energy[i] = energy[i];
    rung_of_slot[i] = i;
    slot_of_rung[i] = i;
    if (i < R - 1) {
      tried[i] = 0;
      accepted[i] = 0;
    }
  }
}

// FP64 recompute: E = sum_p s_p (-1/2 sum_j J s_j - h_p), weights and field widened to double.
template <bool kInt>
__global__ void energy_fp64_kernel(PtKernelArgs a, const int8_t* spins, double* out) {
  const int S = blockIdx.x, slot = blockIdx.y;
  const int lane = threadIdx.x & 31, q = threadIdx.x >> 5;
  const int p = S * kSlicePositions + lane * kGroup + q;
  const int8_t* sp = spins + (size_t)slot * a.n_pos;
  const int w0 = a.slice_off[S], width = a.slice_off[S + 1] - w0;
  const long long base = (long long)w0 * kSlicePositions + lane;
  double v = 0.0;
  if (p < a.n) {
    double f = 0.0, hh;
    for (int d = 0; d < width; ++d) {
      const long long e = base + (long long)(d * kGroup + q) * 32;
      const double wt = kInt ? (double)static_cast<const int8_t*>(a.ell_w)[e] : (double)static_cast<const float*>(a.ell_w)[e];
      f += wt * (double)sp[a.ell_nbr[e]];
    }
    const long long hi = (long long)S * kSlicePositions + q * 32 + lane;
    hh = kInt ? (double)static_cast<const int*>(a.h_pos)[hi] : (double)static_cast<const float*>(a.h_pos)[hi];
    v = (double)sp[p] * (-0.5 * f - hh);
  }
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  __shared__ double red[8];
  if (lane == 0) red[q] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int i = 0; i < 8; ++i) s += red[i];
    atomicAdd(out + slot, s);
  }
}

// ---------------------------------------------------------------------------------------------
// Launch helpers (called from the C ABI in dpt_capi.cu)
// ---------------------------------------------------------------------------------------------
cudaError_t launch_init(const PtKernelArgs& a, int integer_path, cudaStream_t st) {
  dim3 grid((a.n_pos / kGroup + 127) / 128, a.R);
  init_spins_kernel<<<grid, 128, 0, st>>>(a.n, a.n_pos, a.R, a.inst, a.k0, a.k1, a.spins, a.best_spins);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  e = cudaMemsetAsync(a.energy, 0, sizeof(long long) * a.R, st);
  if (e != cudaSuccess) return e;
  dim3 g2(a.n_slices, a.R);
  if (integer_path) energy_fixed_kernel<true><<<g2, 256, 0, st>>>(a);
  else energy_fixed_kernel<false><<<g2, 256, 0, st>>>(a);
  e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  init_finalize_kernel<<<(a.R + 255) / 256, 256, 0, st>>>(a.R, integer_path, a.energy, a.best_energy, a.rung_of_slot,
                                                         a.slot_of_rung, a.tried, a.accepted);
  return cudaGetLastError();
}

cudaError_t launch_energy_fp64(const PtKernelArgs& a, int integer_path, const int8_t* spins, int R, double* out,
                               cudaStream_t st) {
  cudaError_t e = cudaMemsetAsync(out, 0, sizeof(double) * R, st);
  if (e != cudaSuccess) return e;
  dim3 g2(a.n_slices, R);
  if (integer_path) energy_fp64_kernel<true><<<g2, 256, 0, st>>>(a, spins, out);
  else energy_fp64_kernel<false><<<g2, 256, 0, st>>>(a, spins, out);
  return cudaGetLastError();
}

template <bool kInt, bool kInSmem, bool kField, int P, bool kCl>
static const void* pick_w(int max_w, int min_w) {
  // uniform slice widths 3, 4 and 6 (regular graphs and lattices) get an exact-width gather;
  // otherwise widths up to 8 a predicated one, and wider slices a run-time loop
  if constexpr (kInSmem) {
    if (min_w == max_w && max_w == 3) return (const void*)pt_run_kernel<kInt, kInSmem, 3, true, kField, P, kCl>;
    if (min_w == max_w && max_w == 4) return (const void*)pt_run_kernel<kInt, kInSmem, 4, true, kField, P, kCl>;
    if (min_w == max_w && max_w == 6) return (const void*)pt_run_kernel<kInt, kInSmem, 6, true, kField, P, kCl>;
  }
  if (max_w >= 1 && max_w <= 8) return (const void*)pt_run_kernel<kInt, kInSmem, 8, false, kField, P, kCl>;
  return (const void*)pt_run_kernel<kInt, kInSmem, 0, false, kField, P, kCl>;
}

template <bool kInt, bool kInSmem, bool kField, bool kCl>
static const void* pick_p(int max_w, int min_w, int p) {
  if constexpr (kInt) {
    if (p == 4) return pick_w<kInt, kInSmem, kField, 4, kCl>(max_w, min_w);
    // one position per item: small problems only (coupling table in shared memory)
    if constexpr (kInSmem)
      if (p == 1) return pick_w<kInt, kInSmem, kField, 1, kCl>(max_w, min_w);
    if (p == 1) return nullptr;
  }
  return pick_w<kInt, kInSmem, kField, 8, kCl>(max_w, min_w);
}

template <bool kCl, int P, int kPh>
static const void* pick_unit(int w) {
  switch (w) {
    case 2: return (const void*)pt_run_kernel<true, true, 2, true, false, P, kCl, 2, kPh>;
    case 3: return (const void*)pt_run_kernel<true, true, 3, true, false, P, kCl, 3, kPh>;
    case 4: return (const void*)pt_run_kernel<true, true, 4, true, false, P, kCl, 4, kPh>;
    case 6: return (const void*)pt_run_kernel<true, true, 6, true, false, P, kCl, 6, kPh>;
    default: return nullptr;
  }
}

template <bool kCl, int P>
static const void* pick_unit_phases(int w, int phases) {
  return phases <= 2 ? pick_unit<kCl, P, 2>(w) : pick_unit<kCl, P, kUnitPhases>(w);
}

bool unit_width_supported(int w) { return w == 2 || w == 3 || w == 4 || w == 6; }

// The cluster form exists with the coupling table in shared memory only (small problems, where the
// round end is a large share of the round).
const void* run_kernel_ptr(int integer_path, int in_smem, int max_width, int min_width, int has_field,
                           int positions_per_item, int cluster, int unit) {
  if (unit) {
    if (!integer_path || has_field || max_width != min_width) return nullptr;
    if (positions_per_item == 2)
      return cluster ? pick_unit_phases<true, 2>(max_width, unit) : pick_unit_phases<false, 2>(max_width, unit);
    if (positions_per_item == 4)
      return cluster ? pick_unit_phases<true, 4>(max_width, unit) : pick_unit_phases<false, 4>(max_width, unit);
    return nullptr;
  }
  const int p = positions_per_item, w = max_width, m = min_width;
  if (cluster) {
    if (!in_smem) return nullptr;
    if (integer_path)
      return has_field ? pick_p<true, true, true, true>(w, m, p) : pick_p<true, true, false, true>(w, m, p);
    return has_field ? pick_p<false, true, true, true>(w, m, p) : pick_p<false, true, false, true>(w, m, p);
  }
  if (integer_path) {
    if (in_smem) return has_field ? pick_p<true, true, true, false>(w, m, p) : pick_p<true, true, false, false>(w, m, p);
    return has_field ? pick_p<true, false, true, false>(w, m, p) : pick_p<true, false, false, false>(w, m, p);
  }
  if (in_smem) return has_field ? pick_p<false, true, true, false>(w, m, p) : pick_p<false, true, false, false>(w, m, p);
  return has_field ? pick_p<false, false, true, false>(w, m, p) : pick_p<false, false, false, false>(w, m, p);
}

}  // namespace dpt
