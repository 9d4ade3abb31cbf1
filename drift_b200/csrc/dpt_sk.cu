// dpt_sk.cu - dense couplings (SK type): sequential-order Metropolis sweeps with exact integer
// local fields, updated on the tensor cores (tcgen05.mma kind::i8, accumulators in tensor memory).
//
// One persistent cooperative launch runs every round. A CTA owns G <= 12 replica slots and has
// three kinds of warps:
//   * resolvers (one per slot) run the sequential chain 32 spins at a time, lane l holding spin
//     32B + l. All 32 tentative decisions of a block are evaluated at once; the first accepted one
//     (ballot + find-first-set) is applied, the later spins' fields are corrected from the block's
//     32 x 32 diagonal couplings, and the scan resumes after it. Each pass resolves at least one
//     attempt and a block where nothing flips takes one pass;
//   * the producer streams the coupling table (one entry per block: 3 int8 limb tiles per 128
//     rows plus the int32 diagonal block) into a 3-deep shared-memory ring with cp.async.bulk, and
//     after each block issues 3 x n_tiles MMAs F^T[rows][slots] += Jq[rows][block] delta[block][slots];
//   * four loaders (one per tensor-memory lane quarter) read back the fields of the block about
//     to be resolved (tcgen05.ld) and stage them in shared memory.
// Pipelining: the fields staged for block j contain every spin change up to block j-2; the
// resolvers add block j-1's changes themselves from its couplings, which are still in the ring.
// The accumulators come in two sets (MMAs of even / odd blocks), so a loader reads one set while
// the MMA of the next block writes the other, and the MMA of block j-1 overlaps the resolution of
// block j. Every wait is on an mbarrier with a time limit; a timeout raises a CTA-wide abort
// flag, and every role drains its outstanding tensor-core work before the CTA releases its
// tensor memory.
#include <climits>
#include <cstring>
#include <cuda_runtime.h>

#include "../../include/drift_pt.h"
#include "dpt_common.cuh"
#include "dpt_internal.h"
#include "dpt_sk.h"

// Profiling build only (-DDPT_SK_STAMPS, `python -m drift_b200.build --sk-stamps`): clock64 stamps of
// CTA 0 at each hand-off of a block (resolver 0 picks up block j, resolver 0 publishes its delta,
// the producer sees all deltas, the loaders' reads of the set are done, the MMAs are committed, a
// loader sees block j-2's MMAs, a loader releases block j's stage), read back by drift_pt_sk_stamps
// (drift_b200/sk_stamps.py). The product build compiles the stamps to nothing.
#ifdef DPT_SK_STAMPS
namespace dpt {
__device__ unsigned long long g_sk_stamp[8][4096];
}
#define SK_STAMP(e, j)                                                        \
  do {                                                                        \
    if (blockIdx.x == 0 && (j) < 4096) ::dpt::g_sk_stamp[e][j] = clock64(); \
  } while (0)
extern "C" DRIFT_PT_API int drift_pt_sk_stamps(unsigned long long* out) {
  return cudaMemcpyFromSymbol(out, dpt::g_sk_stamp, sizeof(dpt::g_sk_stamp)) == cudaSuccess ? 0 : DRIFT_PT_ECUDA;
}
#else
#define SK_STAMP(e, j) \
  do {                 \
  } while (0)
#endif

namespace dpt {
namespace {

using namespace sk;

constexpr int kRing = 3;             // coupling-table ring entries
constexpr int kScanMin = 8;          // tentative accepts from which a block is walked in full
constexpr int kSkThreads = 32 * (kMaxG + 5);  // 12 resolvers, 4 loaders, 1 producer
// Instruction descriptor: kind::i8, D int32 (bits 4-5 = 2), A and B signed int8 (bits 7-9 and
// 10-12 = 1), both K-major, N = 16 (bits 17-22 = N >> 3), M = 128 (bits 24-28 = M >> 4).
constexpr uint32_t kIdesc = (2u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(kCols >> 3) << 17) |
                            ((uint32_t)(kTile >> 4) << 24);

// barrier slots
enum : int {
  kBarSlabFull = 0,   // [kRing] coupling entry landed (producer arrive + tx bytes)
  kBarSlabFree = 3,   // [kRing] resolvers are done with the entry (Gc arrivals)
  kBarDelta = 6,      // [4] delta operand of a block written (Gc arrivals)
  kBarMma = 10,       // [4] MMAs of a block complete (tcgen05.commit)
  kBarRead = 14,      // [4] both loader reads of an accumulator set done before the next MMA (2)
  kBarInitMma = 18,   // [kRing] initial product, entry consumed
  kBarInitReady = 21, // initial spin operand written (Gc)
  kBarInitDone = 22,  // initial product and zeroed second set complete
  kBarEnergy = 23,    // initial energies summed (4 loaders)
  kBarXchg = 24,      // exchange of the round decided (1)
  kBarFinal = 25,     // all MMAs drained
  kNumBars = 26
};

struct SkArgs {
  int n, nt, nb, R, G, spr, n_rounds, n_steps;
  long long round0;
  uint32_t k0, k1, inst, tmem_cols;
  double escale;
  const unsigned char* layout;
  unsigned int entry;
  const int* hq;
  const float* scales;
  const double* betas;
  int8_t* spins;
  int8_t* best_spins;
  long long* energy;
  long long* best_energy;
  int* rung_of_slot;
  int* slot_of_rung;
  long long* tried;
  long long* accepted;
  long long* best_hist;
  int* err;
  long long* pub;
  unsigned long long* tags;
  long long timeout_ns;
};

struct SkSmem {
  unsigned ring, delta, fields, thr, rung, slot, eall, stats, einit, bars, misc, total;
};

__host__ __device__ inline unsigned up128(unsigned x) { return (x + 127u) & ~127u; }

__host__ __device__ inline SkSmem sk_smem(int n, int G, int R) {
  SkSmem L;
  unsigned o = 0;
  L.ring = o;
  o += up128((unsigned)(kRing * entry_bytes(n)));
  L.delta = o;
  o += 4 * kOpBytes;
  L.fields = o;  // staged fields [4][G][32] int32, before the pipeline starts the initial spin operand
  const unsigned fb = (unsigned)(4 * G * kBlock * 4), ib = (unsigned)(n_blocks(n) * kOpBytes);
  o += up128(fb > ib ? fb : ib);
  L.thr = o;  // acceptance thresholds of the staged blocks [4][G][32] int32
  o += up128(fb);
  L.rung = o;
  o += up128(4u * R);
  L.slot = o;
  o += up128(4u * R);
  L.eall = o;
  o += up128(8u * R);
  L.stats = o;
  o += up128(8u * R);
  L.einit = o;
  o += 8 * kMaxG;
  L.bars = o;
  o += 8 * kNumBars;
  L.misc = o;  // tensor-memory address, abort flag, 4 stage tags
  o += 32;
  L.total = up128(o);
  return L;
}

// ------------------------------------------------------------------------------------------------
// PTX wrappers
// ------------------------------------------------------------------------------------------------
__device__ __forceinline__ unsigned long long sk_now() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}
__device__ __forceinline__ uint32_t sk_smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint32_t bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}
__device__ __forceinline__ void mbar_arrive_tx(uint32_t bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_test(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ bool mbar_probe(uint32_t bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(bar), "r"(parity)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ void bulk_load(uint32_t dst, const void* src, uint32_t bytes, uint32_t bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void tc_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// Shared-memory matrix descriptor: start >> 4, leading offset 128 B, stride offset 256 B, the
// sm_100 descriptor version (bits 46-47 = 1), no swizzle.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)(128u >> 4) << 16) | ((uint64_t)(256u >> 4) << 32) |
         ((uint64_t)1 << 46);
}
__device__ __forceinline__ void mma_i8(uint32_t d_tmem, uint64_t adesc, uint64_t bdesc, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}" ::"r"(d_tmem),
      "l"(adesc), "l"(bdesc), "r"(kIdesc), "r"(accumulate), "r"(0u)
      : "memory");
}
__device__ __forceinline__ void mma_commit(uint32_t bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(bar) : "memory");
}
// Three 32-lane x 16-column loads (the three limb accumulators) and the wait for them, in one
// statement so no use of the registers can be scheduled before the wait.
__device__ __forceinline__ void tmem_ld3(uint32_t a0, uint32_t a1, uint32_t a2, uint32_t (&x)[3][16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%48];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%49];\n\t"
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%32,%33,%34,%35,%36,%37,%38,%39,%40,%41,%42,%43,%44,%45,%46,%47}, [%50];\n\t"
      "tcgen05.wait::ld.sync.aligned;"
      : "=r"(x[0][0]), "=r"(x[0][1]), "=r"(x[0][2]), "=r"(x[0][3]), "=r"(x[0][4]), "=r"(x[0][5]), "=r"(x[0][6]),
        "=r"(x[0][7]), "=r"(x[0][8]), "=r"(x[0][9]), "=r"(x[0][10]), "=r"(x[0][11]), "=r"(x[0][12]), "=r"(x[0][13]),
        "=r"(x[0][14]), "=r"(x[0][15]), "=r"(x[1][0]), "=r"(x[1][1]), "=r"(x[1][2]), "=r"(x[1][3]), "=r"(x[1][4]),
        "=r"(x[1][5]), "=r"(x[1][6]), "=r"(x[1][7]), "=r"(x[1][8]), "=r"(x[1][9]), "=r"(x[1][10]), "=r"(x[1][11]),
        "=r"(x[1][12]), "=r"(x[1][13]), "=r"(x[1][14]), "=r"(x[1][15]), "=r"(x[2][0]), "=r"(x[2][1]), "=r"(x[2][2]),
        "=r"(x[2][3]), "=r"(x[2][4]), "=r"(x[2][5]), "=r"(x[2][6]), "=r"(x[2][7]), "=r"(x[2][8]), "=r"(x[2][9]),
        "=r"(x[2][10]), "=r"(x[2][11]), "=r"(x[2][12]), "=r"(x[2][13]), "=r"(x[2][14]), "=r"(x[2][15])
      : "r"(a0), "r"(a1), "r"(a2)
      : "memory");
}

// ------------------------------------------------------------------------------------------------
// Bounded waits. `abort` is the CTA's shared flag; a timeout raises it and the global error.
// ------------------------------------------------------------------------------------------------
struct Ctl {
  volatile int* abort;
  int* err;
  long long timeout_ns;
};

// one thread
__device__ bool wait1(uint32_t bar, uint32_t parity, const Ctl& c) {
  if (mbar_probe(bar, parity)) return true;
  const unsigned long long t0 = sk_now();
  while (true) {
    if (mbar_test(bar, parity)) return true;
    if (*c.abort) return false;
    if (sk_now() - t0 > (unsigned long long)c.timeout_ns) {
      *c.abort = 1;
      atomicExch(c.err, DRIFT_PT_ETIMEOUT);
      return false;
    }
  }
}

// a whole warp: every lane observes the completed phase itself; the outcome is warp-uniform
__device__ bool wait_warp(uint32_t bar, uint32_t parity, const Ctl& c) {
  if (__all_sync(0xffffffffu, mbar_probe(bar, parity))) return true;  // usually already complete
  unsigned long long t0 = 0;
  for (int it = 0;; ++it) {
    const bool ok = mbar_test(bar, parity);
    if (__all_sync(0xffffffffu, ok)) return true;
    int stop = 0;
    if ((threadIdx.x & 31) == 0) {
      if (*c.abort) {
        stop = 1;
      } else {
        const unsigned long long now = sk_now();
        if (it == 0) {
          t0 = now;
        } else if (now - t0 > (unsigned long long)c.timeout_ns) {
          *c.abort = 1;
          atomicExch(c.err, DRIFT_PT_ETIMEOUT);
          stop = 1;
        }
      }
    }
    if (__shfl_sync(0xffffffffu, stop, 0)) return false;
  }
}

__device__ __forceinline__ unsigned long long ld_acquire(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_release(unsigned long long* p, unsigned long long v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ void st_release_cta(int* p, int v) {
  asm volatile("st.release.cta.shared::cta.s32 [%0], %1;" ::"r"(sk_smem_addr(p)), "r"(v) : "memory");
}
__device__ __forceinline__ int ld_acquire_cta(const int* p) {
  int v;
  asm volatile("ld.acquire.cta.shared::cta.s32 %0, [%1];" : "=r"(v) : "r"(sk_smem_addr(p)) : "memory");
  return v;
}
// a whole warp waits until a stage tag reaches `want` (every lane acquires it itself)
__device__ bool wait_stage(const int* tag, int want, const Ctl& c) {
  if (__all_sync(0xffffffffu, ld_acquire_cta(tag) >= want)) return true;
  unsigned long long t0 = 0;
  for (int it = 0;; ++it) {
    if (__all_sync(0xffffffffu, ld_acquire_cta(tag) >= want)) return true;
    int stop = 0;
    if ((threadIdx.x & 31) == 0) {
      if (*c.abort) {
        stop = 1;
      } else {
        const unsigned long long now = sk_now();
        if (it == 0) {
          t0 = now;
        } else if (now - t0 > (unsigned long long)c.timeout_ns) {
          *c.abort = 1;
          atomicExch(c.err, DRIFT_PT_ETIMEOUT);
          stop = 1;
        }
      }
    }
    if (__shfl_sync(0xffffffffu, stop, 0)) return false;
  }
}

__device__ __forceinline__ long long warp_sum64(long long v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// tensor-memory column of accumulator (set, tile, limb)
__device__ __forceinline__ uint32_t acc_col(int set, int tile, int limb, int nt) {
  return (uint32_t)(((set * nt + tile) * kLimbs + limb) * kCols);
}

// limb accumulators -> field contribution, exact mod 2^32 (every staged sum is a true field < 2^30)
__device__ __forceinline__ uint32_t combine(uint32_t a0, uint32_t a1, uint32_t a2) { return a0 + (a1 << 8) + (a2 << 16); }

// ------------------------------------------------------------------------------------------------
// The persistent kernel
// ------------------------------------------------------------------------------------------------
__global__ void __launch_bounds__(kSkThreads, 1) sk_run_kernel(const SkArgs a) {
  extern __shared__ __align__(1024) unsigned char sk_raw[];
  constexpr uint32_t kFull = 0xffffffffu;
  const SkSmem L = sk_smem(a.n, a.G, a.R);
  unsigned char* ring = sk_raw + L.ring;
  int8_t* delta = reinterpret_cast<int8_t*>(sk_raw + L.delta);
  int32_t* fields = reinterpret_cast<int32_t*>(sk_raw + L.fields);
  int8_t* init_op = reinterpret_cast<int8_t*>(sk_raw + L.fields);
  int32_t* thr = reinterpret_cast<int32_t*>(sk_raw + L.thr);
  int* rung_sm = reinterpret_cast<int*>(sk_raw + L.rung);
  int* slot_sm = reinterpret_cast<int*>(sk_raw + L.slot);
  long long* eall = reinterpret_cast<long long*>(sk_raw + L.eall);
  int* stats = reinterpret_cast<int*>(sk_raw + L.stats);
  unsigned long long* einit = reinterpret_cast<unsigned long long*>(sk_raw + L.einit);
  const uint32_t bars = sk_smem_addr(sk_raw + L.bars);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(sk_raw + L.misc);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(sk_raw + L.misc + 4);
  int* stage = reinterpret_cast<int*>(sk_raw + L.misc + 16);  // stage[j & 3] = j + 1 once block j is staged
  auto bar = [&](int i) { return bars + 8u * (uint32_t)i; };

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int n = a.n, nt = a.nt, nb = a.nb, R = a.R, G = a.G;
  const int gpad = (G + 3) & ~3;
  const int loader0 = gpad, producer = gpad + 4;
  const int slot0 = blockIdx.x * G;
  const int Gc = min(G, R - slot0);
  const unsigned EB = a.entry;
  const Ctl ctl{abort_flag, a.err, a.timeout_ns};
  const uint32_t tbase = (uint32_t)((unsigned long long)a.round0 * (unsigned long long)a.spr);

  // ---- set-up ----
  if (tid == 0) {
    for (int i = 0; i < kRing; ++i) {
      mbar_init(bar(kBarSlabFull + i), 1);
      mbar_init(bar(kBarSlabFree + i), (uint32_t)Gc);
      mbar_init(bar(kBarInitMma + i), 1);
    }
    for (int i = 0; i < 4; ++i) {
      mbar_init(bar(kBarDelta + i), (uint32_t)Gc);
      mbar_init(bar(kBarMma + i), 1);
      mbar_init(bar(kBarRead + i), 2);
    }
    mbar_init(bar(kBarInitReady), (uint32_t)Gc);
    mbar_init(bar(kBarInitDone), 1);
    mbar_init(bar(kBarEnergy), 4);
    mbar_init(bar(kBarXchg), 1);
    mbar_init(bar(kBarFinal), 1);
    *abort_flag = 0;
    for (int i = 0; i < 4; ++i) stage[i] = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  for (int i = tid; i < 4 * kOpBytes / 4; i += blockDim.x) reinterpret_cast<int*>(delta)[i] = 0;
  {
    const int words = (int)(L.thr - L.fields) / 4;
    for (int i = tid; i < words; i += blockDim.x) fields[i] = 0;
  }
  for (int i = tid; i < R; i += blockDim.x) {
    rung_sm[i] = a.rung_of_slot[i];
    slot_sm[i] = a.slot_of_rung[i];
    stats[2 * i] = 0;
    stats[2 * i + 1] = 0;
  }
  if (tid < kMaxG) einit[tid] = 0ull;
  fence_async_smem();
  if (warp == producer) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(sk_smem_addr(tmem_slot)),
                 "r"(a.tmem_cols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_before();
  __syncthreads();
  tc_after();
  const uint32_t tmem = *reinterpret_cast<volatile uint32_t*>(tmem_slot);
  const uint32_t ring_a = sk_smem_addr(ring), delta_a = sk_smem_addr(delta), init_a = sk_smem_addr(init_op);

  if (warp < Gc) {
    // =========================== resolver: slot slot0 + warp ===========================
    const int r = warp, slot = slot0 + r;
    uint32_t sbits = 0;  // bit B: spin 32B + lane is -1
    for (int B = 0; B < nb; ++B) {
      const int i = kBlock * B + lane;
      const int8_t s = i < n ? a.spins[(size_t)slot * n + i] : (int8_t)1;
      if (s < 0) sbits |= 1u << B;
      init_op[B * kOpBytes + core_offset(r, lane)] = s;
    }
    fence_async_smem();
    __syncwarp();
    if (lane == 0) mbar_arrive(bar(kBarInitReady));
    long long e2 = 0, best = a.best_energy[slot], epart = 0;
    if (wait_warp(bar(kBarEnergy), 0, ctl)) {
      e2 = (long long)einit[r];
      uint32_t pmask = 0, psign = 0;
      int B = 0, tl = 0;
      for (int j = 0; j < a.n_steps; ++j) {
        // block j staged: fields complete up to block j-2, thresholds, coupling entry in the ring
        if (!wait_stage(stage + (j & 3), j + 1, ctl)) break;
        if (r == 0 && lane == 0) SK_STAMP(0, j);
        int32_t F = fields[((j & 3) * G + r) * kBlock + lane];
        const int32_t D = thr[((j & 3) * G + r) * kBlock + lane];
        const int32_t* dg = reinterpret_cast<const int32_t*>(ring + (size_t)(j % kRing) * EB +
                                                             (size_t)nt * kLimbs * kTileBytes);
        if (pmask) {
          // block j-1's changes, from the previous-block couplings of this entry
          const int32_t* pv = dg + kBlock * kBlock;
          int32_t c0 = 0, c1 = 0, c2 = 0, c3 = 0;
#pragma unroll
          for (int f = 0; f < kBlock; f += 4) {
            const uint32_t m4 = pmask >> f, s4 = psign >> f;
            c0 += ((m4 & 1u) ? ((s4 & 1u) ? 2 : -2) : 0) * pv[f * kBlock + lane];
            c1 += ((m4 & 2u) ? ((s4 & 2u) ? 2 : -2) : 0) * pv[(f + 1) * kBlock + lane];
            c2 += ((m4 & 4u) ? ((s4 & 4u) ? 2 : -2) : 0) * pv[(f + 2) * kBlock + lane];
            c3 += ((m4 & 8u) ? ((s4 & 8u) ? 2 : -2) : 0) * pv[(f + 3) * kBlock + lane];
          }
          F += (c0 + c1) + (c2 + c3);
        }
        // ---- resolve the block ----
        const uint32_t sb = __ballot_sync(kFull, (sbits >> B) & 1u);  // old spins, 1 = -1
        const int32_t sp = ((sbits >> B) & 1u) ? -1 : 1;               // a lane is done once it flips
        int32_t v = sp * F;
        uint32_t fl = 0;
        const uint32_t tent = __ballot_sync(kFull, v <= D);
        if (__popc(tent) >= kScanMin) {
          // busy block: walk all 32 positions in order; lane l holds the change of its v caused
          // by a flip of each position f, so the only thing on the chain is one vote per position
          int32_t dv[kBlock];
#pragma unroll
          for (int f = 0; f < kBlock; ++f) dv[f] = sp * (((sb >> f) & 1u) ? 2 : -2) * dg[f * kBlock + lane];
          int32_t vme = 0;  // this lane's v when its own position is tested
#pragma unroll
          for (int f = 0; f < kBlock; ++f) {
            const uint32_t bit = __ballot_sync(kFull, v <= D) & (1u << f);
            vme = lane == f ? v : vme;
            fl |= bit;
            v += bit ? dv[f] : 0;  // a decided lane's v is never read again
          }
          epart += ((fl >> lane) & 1u) ? 4LL * vme : 0LL;
        } else {
          // sparse block: jump to the first accepted position, apply it, rescan after it
          uint32_t acc = tent;
          while (acc) {
            const int f = __ffs(acc) - 1;
            fl |= 1u << f;
            const uint32_t live = ~((2u << f) - 1u);
            const int32_t w = ((sb >> f) & 1u) ? 2 : -2;
            const int32_t Jlf = dg[f * kBlock + lane];  // zero for lane f
            const bool me = lane == f;
            epart += me ? 4LL * v : 0LL;
            v = me ? -v : v + sp * w * Jlf;
            acc = __ballot_sync(kFull, v <= D) & live;
          }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive(bar(kBarSlabFree + j % kRing));  // done with this entry
        sbits ^= ((fl >> lane) & 1u) << B;
        delta[(j & 3) * kOpBytes + core_offset(r, lane)] =
            ((fl >> lane) & 1u) ? (((sb >> lane) & 1u) ? (int8_t)2 : (int8_t)-2) : (int8_t)0;
        fence_async_smem();
        __syncwarp();
        if (lane == 0) mbar_arrive(bar(kBarDelta + (j & 3)));
        if (r == 0 && lane == 0) SK_STAMP(1, j);
        pmask = fl;
        psign = sb;
        // ---- round end: best, then publish the energy for the exchange ----
        if (B == nb - 1 && (tl + 1) % a.spr == 0) {
          e2 += warp_sum64(epart);
          epart = 0;
          const long long rg = a.round0 + tl / a.spr;
          if (e2 < best) {
            best = e2;
            for (int B2 = 0; B2 < nb; ++B2) {
              const int i2 = kBlock * B2 + lane;
              if (i2 < n) a.best_spins[(size_t)slot * n + i2] = ((sbits >> B2) & 1u) ? (int8_t)-1 : (int8_t)1;
            }
          }
          if (lane == 0) {
            const size_t at = (size_t)(rg & 1) * R + slot;
            __stcg(a.pub + at, e2);
            st_release(a.tags + at, (unsigned long long)rg + 1ull);
          }
        }
        if (++B == nb) {
          B = 0;
          ++tl;
        }
      }
    }
    // ---- write back ----
    for (int B2 = 0; B2 < nb; ++B2) {
      const int i2 = kBlock * B2 + lane;
      if (i2 < n) a.spins[(size_t)slot * n + i2] = ((sbits >> B2) & 1u) ? (int8_t)-1 : (int8_t)1;
    }
    e2 += warp_sum64(epart);
    if (lane == 0) {
      a.energy[slot] = e2;
      a.best_energy[slot] = best;
    }
  } else if (warp >= loader0 && warp < loader0 + 4) {
    // ====================== loader: tensor-memory lane quarter q ======================
    // Loader q stages the blocks j with j % 4 == q: their fields (tcgen05.ld of both accumulator
    // sets) and their acceptance thresholds (its Philox word is always word q). Loader 0 also runs
    // the exchange step that ends each round, which every CTA evaluates identically.
    const int q = warp - loader0;  // == warp & 3
    const uint32_t lane_base = tmem + ((uint32_t)(32 * q) << 16);
    long long run_best = LLONG_MAX;
    if (q == 0 && blockIdx.x == 0) {
      for (int s = lane; s < R; s += 32) run_best = min(run_best, a.best_energy[s]);
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) run_best = min(run_best, __shfl_xor_sync(kFull, run_best, o));
    }
    // exchange step of round rl (parallel_tempering.py:104-113): gather every slot's published
    // energy, then one lane per disjoint pair
    auto exchange = [&](int rl) -> bool {
      const long long rg = a.round0 + rl;
      const unsigned long long want = (unsigned long long)rg + 1ull;
      int bad = 0;
      for (int s = lane; s < R && !bad; s += 32) {
        const size_t at = (size_t)(rg & 1) * R + s;
        if (ld_acquire(a.tags + at) < want) {
          const unsigned long long t0 = sk_now();
          while (ld_acquire(a.tags + at) < want) {
            if (*abort_flag) {
              bad = 1;
              break;
            }
            if (sk_now() - t0 > (unsigned long long)a.timeout_ns) {
              *abort_flag = 1;
              atomicExch(a.err, DRIFT_PT_ETIMEOUT);
              bad = 1;
              break;
            }
          }
        }
        if (!bad) eall[s] = __ldcg(a.pub + at);
      }
      if (__any_sync(kFull, bad)) return false;
      __syncwarp();
      const int parity = (int)(rg & 1);
      for (int rr = parity + 2 * lane; rr + 1 < R; rr += 64) {
        const int sa = slot_sm[rr], sbb = slot_sm[rr + 1];
        const double ded = d_mul((double)(eall[sa] - eall[sbb]), a.escale);
        const double dlt = d_mul(d_sub(a.betas[rr], a.betas[rr + 1]), ded);
        bool acc = dlt >= 0.0;
        if (!acc) {
          const U4 u = philox(U4{(uint32_t)rr, (uint32_t)rg, (uint32_t)((unsigned long long)rg >> 32),
                                 ctr3(kTagSwap, a.inst)},
                              a.k0, a.k1);
          acc = uniform53(u.x, u.y) < exp_neg_d(dlt);
        }
        if (blockIdx.x == 0) {
          stats[2 * rr] += 1;
          stats[2 * rr + 1] += acc ? 1 : 0;
        }
        if (acc) {
          slot_sm[rr] = sbb;
          slot_sm[rr + 1] = sa;
          rung_sm[sa] = rr + 1;
          rung_sm[sbb] = rr;
        }
      }
      if (blockIdx.x == 0 && a.best_hist) {
        long long m = LLONG_MAX;
        for (int s = lane; s < R; s += 32) m = min(m, eall[s]);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) m = min(m, __shfl_xor_sync(kFull, m, o));
        run_best = min(run_best, m);
        if (lane == 0) a.best_hist[rl] = run_best;
      }
      __syncwarp();
      if (lane == 0) mbar_arrive(bar(kBarXchg));
      return true;
    };
    bool ok = wait_warp(bar(kBarInitReady), 0, ctl) && wait_warp(bar(kBarInitDone), 0, ctl);
    if (ok) {
      tc_after();
      // initial energies from the initial product (set 0; set 1 is zero)
      for (int t = 0; t < nt; ++t) {
        uint32_t x[3][16];
        tmem_ld3(lane_base + acc_col(0, t, 0, nt), lane_base + acc_col(0, t, 1, nt), lane_base + acc_col(0, t, 2, nt), x);
        const int m = kTile * t + 32 * q + lane;
        const long long h2 = m < n ? 2LL * a.hq[m] : 0LL;
#pragma unroll
        for (int c = 0; c < kMaxG; ++c) {
          if (c >= Gc) break;
          long long ep = 0;
          if (m < n) {
            const int32_t A = (int32_t)combine(x[0][c], x[1][c], x[2][c]);
            const long long s = init_op[(m >> 5) * kOpBytes + core_offset(c, m & 31)];
            ep = -s * ((long long)A + h2);
          }
          ep = warp_sum64(ep);
          if (lane == 0) atomicAdd(&einit[c], (unsigned long long)ep);
        }
      }
      tc_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(bar(kBarEnergy));
      // the staged-field buffers overlap the initial spin operand: every loader is past it first
      ok = wait_warp(bar(kBarEnergy), 0, ctl);
    }
    int round_seen = 0;
    const int steps_per_round = a.spr * nb;
    for (int j = q; ok && j < a.n_steps; j += 4) {
      const int B = j % nb, t = B >> 2, tl = j / nb, rl = j / steps_per_round;
      const int m = kBlock * B + lane;
      const int32_t hv = m < n ? a.hq[m] : 0;
      uint32_t* fb = reinterpret_cast<uint32_t*>(fields) + (size_t)(j & 3) * G * kBlock + lane;
      // first read: the set of block j-1's parity, complete up to block j-3
      if (j >= 3 && !wait_warp(bar(kBarMma + ((j - 3) & 3)), (uint32_t)((j - 3) >> 2) & 1u, ctl)) break;
      if (lane == 0) SK_STAMP(7, j);
      tc_after();
      {
        const int set = (j - 1) & 1;
        uint32_t x[3][16];
        tmem_ld3(lane_base + acc_col(set, t, 0, nt), lane_base + acc_col(set, t, 1, nt),
                 lane_base + acc_col(set, t, 2, nt), x);
#pragma unroll
        for (int c = 0; c < kMaxG; ++c)
          if (c < Gc) fb[c * kBlock] = combine(x[0][c], x[1][c], x[2][c]) + (uint32_t)hv;
      }
      tc_before();
      __syncwarp();
      if (lane == 0 && j >= 1) mbar_arrive(bar(kBarRead + ((j - 1) & 3)));
      // thresholds: word q of Philox(((B >> 2) << 5) | lane, t, slot); the words do not depend on
      // the rungs, so they are drawn before a new round's exchange is waited for
      uint32_t wq[kMaxG];
#pragma unroll
      for (int c = 0; c < kMaxG; ++c) {
        if (c >= Gc) break;
        const U4 u = philox(U4{(uint32_t)(((B >> 2) << 5) | lane), tbase + (uint32_t)tl, (uint32_t)(slot0 + c),
                               ctr3(kTagSkSweep, a.inst)},
                            a.k0, a.k1);
        wq[c] = q == 0 ? u.x : q == 1 ? u.y : q == 2 ? u.z : u.w;
      }
      if (rl > round_seen) {  // a new round: its rungs are those after the previous round's exchange
        if (q == 0 ? !exchange(rl - 1) : !wait_warp(bar(kBarXchg), (uint32_t)(rl - 1) & 1u, ctl)) break;
        round_seen = rl;
      }
#pragma unroll
      for (int c = 0; c < kMaxG; ++c) {
        if (c >= Gc) break;
        thr[((j & 3) * G + c) * kBlock + lane] = m < n ? sk_threshold(wq[c], a.scales[rung_sm[slot0 + c]]) : -1;
      }
      // second read: the set of block j's parity, complete up to block j-2
      if (j >= 2 && !wait_warp(bar(kBarMma + ((j - 2) & 3)), (uint32_t)((j - 2) >> 2) & 1u, ctl)) break;
      if (lane == 0) SK_STAMP(5, j);
      tc_after();
      {
        const int set = j & 1;
        uint32_t x[3][16];
        tmem_ld3(lane_base + acc_col(set, t, 0, nt), lane_base + acc_col(set, t, 1, nt),
                 lane_base + acc_col(set, t, 2, nt), x);
#pragma unroll
        for (int c = 0; c < kMaxG; ++c)
          if (c < Gc) fb[c * kBlock] += combine(x[0][c], x[1][c], x[2][c]);
      }
      tc_before();
      __syncwarp();
      if (lane == 0) mbar_arrive(bar(kBarRead + (j & 3)));
      {
        // coupling entry of block j: loads into ring slot b are counted from the initial product
        const int b = j % kRing;
        const int n_init = (nb - b + kRing - 1) / kRing;
        if (!wait_warp(bar(kBarSlabFull + b), (uint32_t)(n_init + j / kRing) & 1u, ctl)) break;
      }
      __syncwarp();
      if (lane == 0) SK_STAMP(6, j);
      if (lane == 0) st_release_cta(stage + (j & 3), j + 1);
    }
    // the exchange that ends the last round
    if (ok && q == 0 && !*abort_flag) exchange(a.n_rounds - 1);
  } else if (warp == producer) {
    // =========================== producer: coupling ring and MMAs ===========================
    if (lane == 0) {
      uint32_t nload[kRing] = {0u, 0u, 0u};
      const int n_steps = a.n_steps;
      auto load = [&](int blk, int b) {
        mbar_arrive_tx(bar(kBarSlabFull + b), EB);
        bulk_load(ring_a + (uint32_t)b * EB, a.layout + (size_t)blk * EB, EB, bar(kBarSlabFull + b));
        ++nload[b];
      };
      auto wait_full = [&](int b) { return wait1(bar(kBarSlabFull + b), (nload[b] - 1u) & 1u, ctl); };
      auto issue = [&](int set, int b, uint32_t b_op, uint32_t accumulate) {
        for (int t = 0; t < nt; ++t)
          for (int k = 0; k < kLimbs; ++k)
            mma_i8(tmem + acc_col(set, t, k, nt),
                   smem_desc(ring_a + (uint32_t)b * EB + (uint32_t)((t * kLimbs + k) * kTileBytes)), smem_desc(b_op),
                   accumulate);
      };
      bool ok = wait1(bar(kBarInitReady), 0, ctl);
      // initial product: set 0 = Jq s over all blocks
      for (int blk = 0; ok && blk < nb; ++blk) {
        const int b = blk % kRing;
        if (blk >= kRing && !wait1(bar(kBarInitMma + b), (uint32_t)(blk / kRing - 1) & 1u, ctl)) { ok = false; break; }
        load(blk, b);
        if (!wait_full(b)) { ok = false; break; }
        tc_after();
        issue(0, b, init_a + (uint32_t)(blk * kOpBytes), blk > 0 ? 1u : 0u);
        mma_commit(bar(kBarInitMma + b));
      }
      if (ok) {
        // set 1 = 0 (product with the all-zero delta buffer 0)
        issue(1, (nb - 1) % kRing, delta_a, 0u);
        mma_commit(bar(kBarInitDone));
        ok = wait1(bar(kBarInitDone), 0, ctl);
      }
      if (ok) {
        load(0, 0);
        if (n_steps > 1) load(1 % nb, 1);
        for (int i = 0; i < n_steps; ++i) {
          if (i + 2 < n_steps) {
            const int b = (i + 2) % kRing;  // held block i-1
            if (i >= 1) {
              if (!wait1(bar(kBarSlabFree + b), (uint32_t)((i - 1) / kRing) & 1u, ctl)) break;
              if (i - 1 <= n_steps - 3 && !wait1(bar(kBarMma + ((i - 1) & 3)), (uint32_t)((i - 1) >> 2) & 1u, ctl))
                break;
            }
            load((i + 2) % nb, b);
          }
          if (i <= n_steps - 3) {  // the last two blocks' products are never read
            if (!wait1(bar(kBarDelta + (i & 3)), (uint32_t)(i >> 2) & 1u, ctl)) break;
            SK_STAMP(2, i);
            if (!wait1(bar(kBarRead + (i & 3)), (uint32_t)(i >> 2) & 1u, ctl)) break;
            SK_STAMP(3, i);
            if (!wait_full(i % kRing)) break;
            tc_after();
            issue(i & 1, i % kRing, delta_a + (uint32_t)((i & 3) * kOpBytes), 1u);
            mma_commit(bar(kBarMma + (i & 3)));
            SK_STAMP(4, i);
          }
        }
      }
      // drain every MMA issued by this thread before tensor memory is released
      mma_commit(bar(kBarFinal));
      const unsigned long long t0 = sk_now();
      while (!mbar_test(bar(kBarFinal), 0)) {
        if (sk_now() - t0 > (unsigned long long)a.timeout_ns) {
          atomicExch(a.err, DRIFT_PT_ETIMEOUT);
          break;
        }
      }
    }
    __syncwarp();
  }

  // ---- teardown ----
  tc_before();
  __syncthreads();
  if (warp == producer) {
    tc_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(a.tmem_cols) : "memory");
  }
  if (blockIdx.x == 0 && !*abort_flag) {
    for (int i = tid; i < R; i += blockDim.x) {
      a.rung_of_slot[i] = rung_sm[i];
      a.slot_of_rung[i] = slot_sm[i];
    }
    for (int rr = tid; rr < R - 1; rr += blockDim.x) {
      a.tried[rr] += stats[2 * rr];
      a.accepted[rr] += stats[2 * rr + 1];
    }
  }
}

// ------------------------------------------------------------------------------------------------
// Initialisation and exact energies
// ------------------------------------------------------------------------------------------------
__device__ long long block_sum64(long long v, long long* red) {
  v = warp_sum64(v);
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31, nw = blockDim.x >> 5;
  if (l == 0) red[w] = v;
  __syncthreads();
  long long t = 0;
  if (w == 0) {
    t = l < nw ? red[l] : 0;
    t = warp_sum64(t);
  }
  __syncthreads();
  return t;
}

__device__ long long energy_of(int n, const int* Jq, const int* hq, const int8_t* s_sm, long long* red) {
  long long e = 0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    long long A = 0;
    const int* row = Jq + (size_t)i * n;
    for (int j = 0; j < n; ++j) A += (long long)row[j] * s_sm[j];
    e -= (long long)s_sm[i] * (A + 2LL * hq[i]);
  }
  return block_sum64(e, red);
}

__global__ void sk_init_kernel(int n, int R, uint32_t inst, uint32_t k0, uint32_t k1, const int* Jq, const int* hq,
                               int8_t* spins, int8_t* best_spins, long long* energy, long long* best_energy,
                               int* rung_of_slot, int* slot_of_rung, long long* tried, long long* accepted) {
  __shared__ int8_t s_sm[kMaxN];
  __shared__ long long red[32];
  const int slot = blockIdx.x;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const U4 u = philox(U4{(uint32_t)(i >> 2), 0u, (uint32_t)slot, ctr3(kTagInit, inst)}, k0, k1);
    const uint32_t w = (i & 3) == 0 ? u.x : (i & 3) == 1 ? u.y : (i & 3) == 2 ? u.z : u.w;
    const int8_t s = (w >> 31) ? (int8_t)-1 : (int8_t)1;
    s_sm[i] = s;
    spins[(size_t)slot * n + i] = s;
    best_spins[(size_t)slot * n + i] = s;
  }
  __syncthreads();
  const long long e = energy_of(n, Jq, hq, s_sm, red);
  if (threadIdx.x == 0) {
    energy[slot] = e;
    best_energy[slot] = e;
    rung_of_slot[slot] = slot;
    slot_of_rung[slot] = slot;
    if (slot < R - 1) {
      tried[slot] = 0;
      accepted[slot] = 0;
    }
  }
}

__global__ void sk_energy_kernel(int n, const int* Jq, const int* hq, const int8_t* spins, long long* out) {
  __shared__ int8_t s_sm[kMaxN];
  __shared__ long long red[32];
  const int slot = blockIdx.x;
  for (int i = threadIdx.x; i < n; i += blockDim.x) s_sm[i] = spins[(size_t)slot * n + i];
  __syncthreads();
  const long long e = energy_of(n, Jq, hq, s_sm, red);
  if (threadIdx.x == 0) out[slot] = e;
}

int sk_fail(cudaError_t e, const char* what) {
  return set_error(DRIFT_PT_ECUDA, "%s: %s", what, cudaGetErrorString(e));
}

int sk_validate(const DriftPtSkProblem* p, const DriftPtSkRunArgs* args, const DriftPtSkState* st) {
  if (!p || !args || !st) return set_error(DRIFT_PT_EINVAL, "sk: null argument");
  if (p->n < 1 || p->n > kMaxN) return set_error(DRIFT_PT_EINVAL, "sk: n must be in 1..%d", kMaxN);
  if (p->shift < -60 || p->shift > 60) return set_error(DRIFT_PT_EINVAL, "sk: shift out of range");
  if (!p->Jq || !p->hq || !p->layout) return set_error(DRIFT_PT_EINVAL, "sk: null problem array");
  const int R = args->n_replicas;
  if (R < 2 || R > kMaxR) return set_error(DRIFT_PT_EINVAL, "sk: n_replicas must be in 2..%d", kMaxR);
  if (args->replicas_per_cta < 0 || args->replicas_per_cta > kMaxG)
    return set_error(DRIFT_PT_EINVAL, "sk: replicas_per_cta must be in 0..%d", kMaxG);
  if (args->instance > kMaxInstance) return set_error(DRIFT_PT_EINVAL, "sk: instance >= 2^24");
  if (!st->spins || !st->best_spins || !st->energy || !st->best_energy || !st->rung_of_slot || !st->slot_of_rung ||
      !st->swap_tried || !st->swap_accepted)
    return set_error(DRIFT_PT_EINVAL, "sk: null state array");
  return DRIFT_PT_OK;
}

}  // namespace
}  // namespace dpt

using namespace dpt;

extern "C" int drift_pt_sk_workspace_bytes(int32_t n_replicas, size_t* bytes) {
  clear_error();
  if (n_replicas < 1 || n_replicas > sk::kMaxR || !bytes) return set_error(DRIFT_PT_EINVAL, "sk_workspace_bytes");
  const size_t half = ((size_t)16 * n_replicas + 255) & ~(size_t)255;
  *bytes = 256 + 2 * half;
  return DRIFT_PT_OK;
}

extern "C" int drift_pt_sk_init(const DriftPtSkProblem* problem, const DriftPtSkRunArgs* args, DriftPtSkState* state,
                                void* stream) {
  clear_error();
  int rc = sk_validate(problem, args, state);
  if (rc) return rc;
  const int R = args->n_replicas;
  sk_init_kernel<<<R, 256, 0, static_cast<cudaStream_t>(stream)>>>(
      problem->n, R, args->instance, (uint32_t)(args->seed & 0xffffffffu), (uint32_t)(args->seed >> 32), problem->Jq,
      problem->hq, state->spins, state->best_spins, reinterpret_cast<long long*>(state->energy),
      reinterpret_cast<long long*>(state->best_energy), state->rung_of_slot, state->slot_of_rung,
      reinterpret_cast<long long*>(state->swap_tried), reinterpret_cast<long long*>(state->swap_accepted));
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? DRIFT_PT_OK : sk_fail(e, "sk_init_kernel launch");
}

extern "C" int drift_pt_sk_energy(const DriftPtSkProblem* problem, int32_t n_replicas, const int8_t* spins,
                                  int64_t* energy, void* stream) {
  clear_error();
  if (!problem || problem->n < 1 || problem->n > sk::kMaxN || !problem->Jq || !problem->hq || !spins || !energy ||
      n_replicas < 1)
    return set_error(DRIFT_PT_EINVAL, "sk_energy: bad arguments");
  sk_energy_kernel<<<n_replicas, 256, 0, static_cast<cudaStream_t>(stream)>>>(
      problem->n, problem->Jq, problem->hq, spins, reinterpret_cast<long long*>(energy));
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? DRIFT_PT_OK : sk_fail(e, "sk_energy_kernel launch");
}

extern "C" int drift_pt_sk_run(const DriftPtSkProblem* problem, const DriftPtSkRunArgs* args, DriftPtSkState* state,
                               void* workspace, size_t workspace_bytes, void* stream) {
  clear_error();
  int rc = sk_validate(problem, args, state);
  if (rc) return rc;
  if (args->n_rounds < 0 || args->sweeps_per_round < 1 || args->round_offset < 0)
    return set_error(DRIFT_PT_EINVAL, "sk: run arguments");
  if (!args->betas || !args->scales) return set_error(DRIFT_PT_EINVAL, "sk: null betas / scales");
  const int R = args->n_replicas, n = problem->n;
  size_t need = 0;
  drift_pt_sk_workspace_bytes(R, &need);
  if (!workspace || workspace_bytes < need) return set_error(DRIFT_PT_EINVAL, "sk: workspace too small");
  if (args->n_rounds == 0) return DRIFT_PT_OK;
  const long long steps = (long long)args->n_rounds * args->sweeps_per_round * sk::n_blocks(n);
  if (steps >= (1LL << 31)) return set_error(DRIFT_PT_EINVAL, "sk: too many sweeps in one call");
  int dev = 0, sms = 0;
  cudaGetDevice(&dev);
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return set_error(DRIFT_PT_ECUDA, "cudaDeviceGetAttribute failed");
  int G = args->replicas_per_cta;
  if (G == 0) {
    G = (R + sms - 1) / sms;
    if (G < 1) G = 1;
  }
  const int grid = (R + G - 1) / G;
  const int gpad = (G + 3) & ~3;
  const int threads = 32 * (gpad + 5);
  const SkSmem L = sk_smem(n, G, R);
  int per_sm = 0;
  rc = prepare_kernel((const void*)sk_run_kernel, threads, L.total, &per_sm);
  if (rc) return rc;
  if (per_sm < 1) return set_error(DRIFT_PT_EUNSUPPORTED, "sk: kernel does not fit an SM");
  if (grid > sms) return set_error(DRIFT_PT_EUNSUPPORTED, "sk: %d CTAs exceed the %d SMs; raise replicas_per_cta", grid, sms);

  SkArgs a;
  std::memset(&a, 0, sizeof a);
  a.n = n;
  a.nt = sk::n_tiles(n);
  a.nb = sk::n_blocks(n);
  a.R = R;
  a.G = G;
  a.spr = args->sweeps_per_round;
  a.n_rounds = args->n_rounds;
  a.n_steps = (int)steps;
  a.round0 = args->round_offset;
  a.k0 = (uint32_t)(args->seed & 0xffffffffu);
  a.k1 = (uint32_t)(args->seed >> 32);
  a.inst = args->instance;
  {
    const int cols = 2 * a.nt * sk::kLimbs * sk::kCols;
    uint32_t c = 32;
    while ((int)c < cols) c <<= 1;
    a.tmem_cols = c;
  }
  a.escale = std::ldexp(1.0, -(problem->shift + 1));
  a.layout = static_cast<const unsigned char*>(problem->layout);
  a.entry = (unsigned)sk::entry_bytes(n);
  a.hq = problem->hq;
  a.scales = args->scales;
  a.betas = args->betas;
  a.spins = state->spins;
  a.best_spins = state->best_spins;
  a.energy = reinterpret_cast<long long*>(state->energy);
  a.best_energy = reinterpret_cast<long long*>(state->best_energy);
  a.rung_of_slot = state->rung_of_slot;
  a.slot_of_rung = state->slot_of_rung;
  a.tried = reinterpret_cast<long long*>(state->swap_tried);
  a.accepted = reinterpret_cast<long long*>(state->swap_accepted);
  a.best_hist = reinterpret_cast<long long*>(state->best_history);
  unsigned char* ws = static_cast<unsigned char*>(workspace);
  a.err = reinterpret_cast<int*>(ws + 8);
  const size_t half = ((size_t)16 * R + 255) & ~(size_t)255;
  a.pub = reinterpret_cast<long long*>(ws + 256);
  a.tags = reinterpret_cast<unsigned long long*>(ws + 256 + half);
  a.timeout_ns = (long long)((args->timeout_s > 0 ? args->timeout_s : 10.0) * 1e9);

  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemsetAsync(ws, 0, need, st);
  if (e != cudaSuccess) return sk_fail(e, "sk workspace reset");
  cudaLaunchConfig_t cfg;
  std::memset(&cfg, 0, sizeof cfg);
  cfg.gridDim = dim3(grid);
  cfg.blockDim = dim3(threads);
  cfg.dynamicSmemBytes = L.total;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeCooperative;
  attr[0].val.cooperative = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  void* kargs[] = {&a};
  e = cudaLaunchKernelExC(&cfg, (const void*)sk_run_kernel, kargs);
  if (e != cudaSuccess) return sk_fail(e, "sk_run_kernel launch");
  return DRIFT_PT_OK;
}
