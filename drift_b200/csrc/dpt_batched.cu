// dpt_batched.cu - many independent PT instances of uneven size in one persistent launch.
//
// Each round: CTAs pull work items (replicas [first, first+count) of one instance) from a queue
// ordered largest first, stage the item's spins in shared memory, run the round's colour-phase
// sweeps with the same item update as the single-ladder kernel (dpt_sweep.cuh), write spins and
// energies back; a bounded grid barrier; one warp per instance runs that instance's exchange step;
// a second barrier. Instance k with stream id s_k is, bit for bit, the chain a single-instance run
// with instance = s_k produces: the uniforms are keyed by (stream, local slot, position, sweep).
#include <climits>
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cstring>
#include <numeric>
#include <vector>

#include "../../include/drift_pt.h"
#include "dpt_common.cuh"
#include "dpt_internal.h"
#include "dpt_kernels.cuh"
#include "dpt_sweep.cuh"

namespace dpt {

struct BatchArgs {
  int n_instances, F_max, max_colors, max_item_bytes;
  const DriftPtInstanceDesc* desc;
  const int* color_ptr;
  const int* slice_off;
  const int* ell_nbr;
  const void* ell_w;
  const void* h_pos;
  const double* betas;
  const uint32_t* thr;
  int n_rounds, spr;
  long long round0;
  uint32_t k0, k1;
  const int* items;
  int n_items, max_tile, tps;
  int8_t* spins;
  long long* energy;
  long long* best_energy;
  int8_t* best_spins;
  int* rung_of_slot;
  int* slot_of_rung;
  long long* tried;
  long long* accepted;
  unsigned long long* bar;  // grid barrier counter
  unsigned long long* ctr;  // work-queue counter
  int* err;
  long long timeout_ns;
};

struct BatchSmem {
  size_t spins, eacc, ecur, ebest, imp, nb, thr, cptr, ctl, total;
};

__host__ __device__ inline BatchSmem batch_smem(int max_tile, int max_item_bytes, int threads, int tps, int F_max,
                                                int max_colors, bool integer_path) {
  BatchSmem L;
  size_t o = 0;
  const int seg = tps < 32 ? tps : 32;
  L.spins = o; o = align16(o + (size_t)max_item_bytes);
  L.eacc = o;  o = align16(o + 8 * (size_t)(threads / seg));
  L.ecur = o;  o = align16(o + 8 * (size_t)max_tile);
  L.ebest = o; o = align16(o + 8 * (size_t)max_tile);
  L.imp = o;   o = align16(o + 4 * (size_t)max_tile);
  L.nb = o;    o = align16(o + 4 * (size_t)max_tile);
  L.thr = o;   o = align16(o + (integer_path ? 4 * (size_t)max_tile * (2 * F_max + 1) : 0));
  L.cptr = o;  o = align16(o + 4 * (size_t)(max_colors + 1));
  L.ctl = o;   o = align16(o + 16);
  L.total = o;
  return L;
}

__device__ __forceinline__ unsigned long long b_timer() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ unsigned long long b_ld_acquire(const unsigned long long* p) {
  unsigned long long v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ int b_ld_relaxed(const int* p) {
  int v;
  asm volatile("ld.relaxed.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

// Bounded grid barrier number `k` (1-based) of this launch; returns false if it gave up.
__device__ bool batch_grid_sync(const BatchArgs& a, unsigned long long k, int* ctl_abort) {
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    atomicAdd(a.bar, 1ULL);
    const unsigned long long target = k * gridDim.x;
    int abort_now = 0;
    // the error flag and the clock are read after the first unsuccessful poll and then after every
    // 8th only (read after every poll they lengthen each poll)
    if (b_ld_acquire(a.bar) < target) {
      const unsigned long long t0 = b_timer();
      for (int it = 1; b_ld_acquire(a.bar) < target; ++it) {
        if (it != 1 && it % 8 != 0) continue;
        if (b_ld_relaxed(a.err) != 0) { abort_now = 1; break; }
        if (b_timer() - t0 > (unsigned long long)a.timeout_ns) {
          atomicExch(a.err, DRIFT_PT_ETIMEOUT);
          abort_now = 1;
          break;
        }
      }
    }
    *ctl_abort = abort_now;
  }
  __syncthreads();
  return *ctl_abort == 0;
}

template <bool kInt, int W, bool kExactW, bool kField, int P>
__global__ void __launch_bounds__(kMaxThreads, 1) pt_batched_kernel(const BatchArgs a) {
  unsigned char* smem = dpt_smem;
  const int B = blockDim.x, tid = threadIdx.x;
  const BatchSmem L = batch_smem(a.max_tile, a.max_item_bytes, B, a.tps, a.F_max, a.max_colors, kInt);
  long long* eacc = reinterpret_cast<long long*>(smem + L.eacc);
  long long* ecur = reinterpret_cast<long long*>(smem + L.ecur);
  long long* ebest = reinterpret_cast<long long*>(smem + L.ebest);
  int* imp = reinterpret_cast<int*>(smem + L.imp);
  float* nb_sm = reinterpret_cast<float*>(smem + L.nb);
  uint32_t* thr_sm = reinterpret_cast<uint32_t*>(smem + L.thr);
  int* cptr = reinterpret_cast<int*>(smem + L.cptr);
  int* ctl = reinterpret_cast<int*>(smem + L.ctl);
  constexpr int NB = kGroup / P;
  const int tps = a.tps, seg = tps < 32 ? tps : 32;
  const int my_sl = tid / tps, lt = tid - my_sl * tps;
  const int row = 2 * a.F_max + 1;
  unsigned long long nsync = 0;

  for (int j = 0; j < a.n_rounds; ++j) {
    const long long round = a.round0 + j;
    const unsigned long long qbase = (unsigned long long)j * (unsigned long long)(a.n_items + gridDim.x);
    for (;;) {
      __syncthreads();
      if (tid == 0) ctl[0] = (int)min((unsigned long long)INT_MAX, atomicAdd(a.ctr, 1ULL) - qbase);
      __syncthreads();
      const int it = ctl[0];
      if (it >= a.n_items) break;
      const int inst = a.items[3 * it], first = a.items[3 * it + 1], cnt = a.items[3 * it + 2];
      const DriftPtInstanceDesc D = a.desc[inst];
      const int n_pos = D.n_pos;
      const long long gs0 = D.slot0 + first;  // global slot of local slot `first`
      // ---- stage the item (L1 is bypassed: other CTAs wrote these in earlier rounds) ----
      {
        const int4* src = reinterpret_cast<const int4*>(a.spins + D.spin0 + (long long)first * n_pos);
        int4* dst = reinterpret_cast<int4*>(smem + L.spins);
        for (int i = tid; i < cnt * n_pos / 16; i += B) dst[i] = __ldcg(src + i);
      }
      for (int s = tid; s < cnt; s += B) {
        ecur[s] = __ldcg(a.energy + gs0 + s);
        ebest[s] = __ldcg(a.best_energy + gs0 + s);
        const int rung = __ldcg(a.rung_of_slot + gs0 + s);
        if constexpr (!kInt) nb_sm[s] = -2.0f * (float)a.betas[D.slot0 + rung];
        imp[s] = rung;  // temporarily: the rung, for the threshold rows below
      }
      for (int i = tid; i <= D.n_colors; i += B) cptr[i] = a.color_ptr[D.color_ptr + i];
      __syncthreads();
      if constexpr (kInt) {
        for (int i = tid; i < cnt * row; i += B) {
          const int s = i / row, x = i - s * row - a.F_max;
          uint32_t v = 0xFFFFFFFFu;
          if (x >= 1) v = (x <= D.max_field) ? a.thr[D.thr + (long long)imp[s] * D.max_field + x - 1] : 0u;
          thr_sm[i] = v;
        }
      }
      __syncthreads();
      Tables T;
      T.soff_o = T.ent_o = T.nbr_o = T.wf_o = T.h_o = 0;
      T.soff = a.slice_off + D.slice_off;
      T.nbr = a.ell_nbr + D.ell;
      T.w8 = static_cast<const int8_t*>(a.ell_w) + D.ell;
      T.wf = static_cast<const float*>(a.ell_w) + D.ell;
      T.h = kInt ? (const void*)(static_cast<const int*>(a.h_pos) + D.pos)
                 : (const void*)(static_cast<const float*>(a.h_pos) + D.pos);
      const bool active = my_sl < cnt;
      const int sl = active ? my_sl : 0;
      const uint32_t slot = (uint32_t)(first + sl);  // local slot: keys the uniforms
      const uint32_t sp_o = (uint32_t)L.spins + (uint32_t)sl * (uint32_t)n_pos;
      const uint32_t thr_o = (uint32_t)L.thr + 4u * (uint32_t)(sl * row + a.F_max);
      const float neg2beta = kInt ? 0.0f : nb_sm[sl];
      const uint32_t c_sweep = ctr3(kTagSweep, (uint32_t)D.stream_id);
      const uint32_t c_second = ctr3(kTagSecond, (uint32_t)D.stream_id);
      long long dacc = 0;
      for (int sw = 0; sw < a.spr; ++sw) {
        const uint32_t t = (uint32_t)(round * a.spr + sw);
        for (int c = 0; c < D.n_colors; ++c) {
          const int lo = cptr[c], hi = cptr[c + 1];
          const int glo = lo >> 3, ghi = (hi + 7) >> 3;
          const int span = ((ghi - glo + 31) >> 5) * 32 * NB;
          if (active) {
            for (int v = lt; v < span; v += tps) {
              const int b = (v >> 5) & (NB - 1);
              const int g = glo + (v / (32 * NB)) * 32 + (v & 31);
              if (g >= ghi) continue;
              if constexpr (kInt)
                dacc += group_int<W, kExactW, false, kField, P>(g, b, lo, hi, t, slot, sp_o, T, thr_o, c_sweep,
                                                                c_second, a.k0, a.k1);
              else
                dacc += group_f32<W, kExactW, false, kField>(g, lo, hi, t, slot, sp_o, T, neg2beta, c_sweep,
                                                             c_second, a.k0, a.k1);
            }
          }
          __syncthreads();
        }
      }
      // ---- item end: per-slot energy change, best, write back ----
      for (int off = seg >> 1; off > 0; off >>= 1) dacc += __shfl_xor_sync(0xffffffffu, dacc, off);
      if (lt % seg == 0) eacc[tid / seg] = dacc;
      __syncthreads();
      for (int s = tid; s < cnt; s += B) {
        long long e = ecur[s];
        const int nseg = tps / seg;
        for (int q = 0; q < nseg; ++q) e += eacc[s * nseg + q];
        a.energy[gs0 + s] = e;
        const int better = e < ebest[s];
        imp[s] = better;
        if (better) a.best_energy[gs0 + s] = e;
      }
      __syncthreads();
      {
        const int chunks = n_pos / 16;
        const int4* src = reinterpret_cast<const int4*>(smem + L.spins);
        int4* dst = reinterpret_cast<int4*>(a.spins + D.spin0 + (long long)first * n_pos);
        int4* bdst = reinterpret_cast<int4*>(a.best_spins + D.spin0 + (long long)first * n_pos);
        for (int i = tid; i < cnt * chunks; i += B) {
          const int4 v = src[i];
          dst[i] = v;
          if (imp[i / chunks]) bdst[i] = v;
        }
      }
    }
    if (!batch_grid_sync(a, ++nsync, ctl + 1)) break;
    // ---- exchange: one warp per instance, one lane per rung pair ----
    {
      const int warps = B >> 5, lane = tid & 31;
      const int parity = (int)(round & 1);
      for (int inst = blockIdx.x * warps + (tid >> 5); inst < a.n_instances; inst += gridDim.x * warps) {
        const DriftPtInstanceDesc D = a.desc[inst];
        const long long b0 = D.slot0;
        const int R = D.n_replicas;
        for (int r = parity + 2 * lane; r + 1 < R; r += 64) {
          const int sa = __ldcg(a.slot_of_rung + b0 + r), sb = __ldcg(a.slot_of_rung + b0 + r + 1);
          const long long de = __ldcg(a.energy + b0 + sa) - __ldcg(a.energy + b0 + sb);
          const double ded = kInt ? (double)de : d_mul((double)de, kFloatEnergyScale);
          const double delta = d_mul(d_sub(a.betas[b0 + r], a.betas[b0 + r + 1]), ded);
          bool acc = delta >= 0.0;
          if (!acc) {
            const U4 u = philox(U4{(uint32_t)r, (uint32_t)round, (uint32_t)((unsigned long long)round >> 32),
                                   ctr3(kTagSwap, (uint32_t)D.stream_id)}, a.k0, a.k1);
            acc = uniform53(u.x, u.y) < exp_neg_d(delta);
          }
          a.tried[b0 + r] = __ldcg(a.tried + b0 + r) + 1;
          if (acc) {
            a.accepted[b0 + r] = __ldcg(a.accepted + b0 + r) + 1;
            a.slot_of_rung[b0 + r] = sb;
            a.slot_of_rung[b0 + r + 1] = sa;
            a.rung_of_slot[b0 + sa] = r + 1;
            a.rung_of_slot[b0 + sb] = r;
          }
        }
      }
    }
    if (!batch_grid_sync(a, ++nsync, ctl + 1)) break;
  }
}

template <bool kInt, bool kField, int P>
static const void* batch_pick_w(int max_w, int min_w) {
  if constexpr (kInt) {
    if (min_w == max_w && max_w == 3) return (const void*)pt_batched_kernel<kInt, 3, true, kField, P>;
    if (min_w == max_w && max_w == 6) return (const void*)pt_batched_kernel<kInt, 6, true, kField, P>;
  }
  if (min_w == max_w && max_w == 4) return (const void*)pt_batched_kernel<kInt, 4, true, kField, P>;
  if (max_w >= 1 && max_w <= 8) return (const void*)pt_batched_kernel<kInt, 8, false, kField, P>;
  return (const void*)pt_batched_kernel<kInt, 0, false, kField, P>;
}

static const void* batch_kernel_ptr(int integer_path, int max_w, int min_w, int has_field, int P) {
  if (integer_path) {
    if (P == 4) return has_field ? batch_pick_w<true, true, 4>(max_w, min_w) : batch_pick_w<true, false, 4>(max_w, min_w);
    return has_field ? batch_pick_w<true, true, 8>(max_w, min_w) : batch_pick_w<true, false, 8>(max_w, min_w);
  }
  return has_field ? batch_pick_w<false, true, 8>(max_w, min_w) : batch_pick_w<false, false, 8>(max_w, min_w);
}

}  // namespace dpt

using namespace dpt;

namespace {

constexpr size_t kBatchWsHeader = 256;  // barrier counter at 0, queue counter at 8, error flag at 16

int b_fail(cudaError_t e, const char* what) { return set_error(DRIFT_PT_ECUDA, "%s: %s", what, cudaGetErrorString(e)); }

int validate_batch(const DriftPtBatchProblem* p) {
  if (!p) return set_error(DRIFT_PT_EINVAL, "batch problem is NULL");
  if (p->n_instances < 1 || p->total_slots < 1 || !p->desc || !p->color_ptr || !p->slice_off || !p->h_pos ||
      !p->betas || (p->integer_path && (!p->thresholds || p->max_field < 1)))
    return set_error(DRIFT_PT_EINVAL, "batch problem: missing arrays or sizes");
  if (p->max_n_pos < kSlicePositions || p->max_n_pos % kSlicePositions || p->max_colors < 1)
    return set_error(DRIFT_PT_EINVAL, "batch problem: max_n_pos / max_colors");
  return DRIFT_PT_OK;
}

}  // namespace

// Items: each instance split into tiles of at most max_tile replicas whose spins fit the budget;
// ordered by work (n_pos x count) descending, ties by instance then first slot.
extern "C" int drift_pt_batch_items(int32_t n_instances, const int32_t* n_pos, const int32_t* n_replicas,
                                    int32_t max_tile, int64_t smem_budget, int32_t* items, int32_t* n_items) {
  clear_error();
  if (n_instances < 1 || !n_pos || !n_replicas || max_tile < 1 || smem_budget < 1 || !n_items)
    return set_error(DRIFT_PT_EINVAL, "batch_items: invalid arguments");
  std::vector<std::array<int32_t, 3>> v;
  for (int32_t k = 0; k < n_instances; ++k) {
    if (n_pos[k] < 1 || n_replicas[k] < 1) return set_error(DRIFT_PT_EINVAL, "batch_items: instance %d", k);
    int64_t fit = smem_budget / n_pos[k];
    if (fit < 1) return set_error(DRIFT_PT_EUNSUPPORTED, "instance %d (%d positions) does not fit the budget", k, n_pos[k]);
    const int32_t tile = (int32_t)std::min<int64_t>({(int64_t)max_tile, (int64_t)n_replicas[k], fit});
    for (int32_t f = 0; f < n_replicas[k]; f += tile) v.push_back({k, f, std::min(tile, n_replicas[k] - f)});
  }
  std::stable_sort(v.begin(), v.end(), [&](const std::array<int32_t, 3>& x, const std::array<int32_t, 3>& y) {
    return (int64_t)n_pos[x[0]] * x[2] > (int64_t)n_pos[y[0]] * y[2];
  });
  if (items) {
    if (*n_items < (int32_t)v.size()) return set_error(DRIFT_PT_EINVAL, "batch_items: items array holds %d, need %zu", *n_items, v.size());
    for (size_t i = 0; i < v.size(); ++i)
      for (int q = 0; q < 3; ++q) items[3 * i + q] = v[i][q];
  }
  *n_items = (int32_t)v.size();
  return DRIFT_PT_OK;
}

extern "C" int drift_pt_batch_workspace_bytes(const DriftPtBatchProblem* prob, size_t* bytes) {
  clear_error();
  if (!bytes) return set_error(DRIFT_PT_EINVAL, "bytes is NULL");
  *bytes = kBatchWsHeader;
  (void)prob;
  return DRIFT_PT_OK;
}

extern "C" int drift_pt_batch_init(const DriftPtBatchProblem* prob, const DriftPtBatchRunArgs* args,
                                   DriftPtDeviceState* state, void* stream) {
  clear_error();
  int rc = validate_batch(prob);
  if (rc) return rc;
  if (!args || !state || !state->spins || !state->energy || !state->best_energy || !state->best_spins ||
      !state->rung_of_slot || !state->slot_of_rung || !state->swap_tried || !state->swap_accepted)
    return set_error(DRIFT_PT_EINVAL, "batch init: state arrays missing");
  // the per-instance views are the single-instance init on offset pointers
  std::vector<DriftPtInstanceDesc> desc(prob->n_instances);
  cudaError_t e = cudaMemcpy(desc.data(), prob->desc, sizeof(DriftPtInstanceDesc) * desc.size(), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return b_fail(e, "batch init: descriptor download");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  for (const DriftPtInstanceDesc& D : desc) {
    PtKernelArgs a;
    std::memset(&a, 0, sizeof a);
    a.n = D.n;
    a.n_pos = D.n_pos;
    a.n_slices = D.n_slices;
    a.n_colors = D.n_colors;
    a.slice_off = prob->slice_off + D.slice_off;
    a.ell_nbr = prob->ell_nbr + D.ell;
    a.ell_w = prob->integer_path ? (const void*)(static_cast<const int8_t*>(prob->ell_w) + D.ell)
                                 : (const void*)(static_cast<const float*>(prob->ell_w) + D.ell);
    a.h_pos = prob->integer_path ? (const void*)(static_cast<const int*>(prob->h_pos) + D.pos)
                                 : (const void*)(static_cast<const float*>(prob->h_pos) + D.pos);
    a.R = D.n_replicas;
    a.inst = (uint32_t)D.stream_id;
    a.k0 = (uint32_t)(args->seed & 0xffffffffu);
    a.k1 = (uint32_t)(args->seed >> 32);
    a.spins = state->spins + D.spin0;
    a.best_spins = state->best_spins + D.spin0;
    a.energy = reinterpret_cast<long long*>(state->energy) + D.slot0;
    a.best_energy = reinterpret_cast<long long*>(state->best_energy) + D.slot0;
    a.rung_of_slot = state->rung_of_slot + D.slot0;
    a.slot_of_rung = state->slot_of_rung + D.slot0;
    a.tried = reinterpret_cast<long long*>(state->swap_tried) + D.slot0;
    a.accepted = reinterpret_cast<long long*>(state->swap_accepted) + D.slot0;
    e = launch_init(a, prob->integer_path, st);
    if (e != cudaSuccess) return b_fail(e, "batch init launch");
  }
  return DRIFT_PT_OK;
}

extern "C" int drift_pt_batch_run(const DriftPtBatchProblem* prob, const DriftPtBatchRunArgs* args,
                                  DriftPtDeviceState* state, void* workspace, size_t workspace_bytes, void* stream) {
  clear_error();
  int rc = validate_batch(prob);
  if (rc) return rc;
  if (!args || args->n_rounds < 0 || args->sweeps_per_round < 1 || args->round_offset < 0 || !args->items ||
      args->n_items < 1 || args->max_tile < 1)
    return set_error(DRIFT_PT_EINVAL, "batch run args");
  if (!state || !state->spins || !state->energy || !state->best_energy || !state->best_spins ||
      !state->rung_of_slot || !state->slot_of_rung || !state->swap_tried || !state->swap_accepted)
    return set_error(DRIFT_PT_EINVAL, "batch run: state arrays missing");
  if (!workspace || workspace_bytes < kBatchWsHeader) return set_error(DRIFT_PT_EINVAL, "batch run: workspace too small");
  if (args->n_rounds == 0) return DRIFT_PT_OK;
  int P = args->positions_per_item;
  if (P != 0 && P != 4 && P != 8) return set_error(DRIFT_PT_EINVAL, "positions_per_item must be 0, 4 or 8");
  if (!prob->integer_path) P = 8;
  else if (P == 0) P = 4;
  const int tps = args->threads_per_slot;
  const bool tps_ok = tps >= 1 && (tps % 32 == 0 || (tps < 32 && (tps & (tps - 1)) == 0));
  const int threads = args->max_tile * tps;
  if (!tps_ok || threads < 32 || threads > kMaxThreads || threads % 32)
    return set_error(DRIFT_PT_EINVAL, "max_tile * threads_per_slot must be a multiple of 32 in [32, %d] (got %d x %d)",
                     kMaxThreads, args->max_tile, tps);
  int dev = 0, sms = 0, optin = 0;
  cudaGetDevice(&dev);
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
    return set_error(DRIFT_PT_ECUDA, "cudaDeviceGetAttribute failed");
  if (args->max_item_bytes < kSlicePositions || args->max_item_bytes % kSlicePositions)
    return set_error(DRIFT_PT_EINVAL, "max_item_bytes must be the largest count * n_pos of the items");
  const BatchSmem L = batch_smem(args->max_tile, args->max_item_bytes, threads, tps, prob->max_field, prob->max_colors,
                                 prob->integer_path != 0);
  if (L.total > (size_t)optin) return set_error(DRIFT_PT_EUNSUPPORTED, "batch item state (%zu B) exceeds shared memory", L.total);
  const void* fn = batch_kernel_ptr(prob->integer_path, prob->max_width, prob->min_width, prob->has_field, P);
  int per_sm = 0;
  rc = prepare_kernel(fn, threads, L.total, &per_sm);
  if (rc) return rc;
  cudaError_t e = cudaSuccess;
  if (per_sm < 1) return set_error(DRIFT_PT_EUNSUPPORTED, "batch kernel does not fit an SM");
  if (args->ctas_per_sm > 0) per_sm = std::min(per_sm, args->ctas_per_sm);
  const int grid = per_sm * sms;
  BatchArgs a;
  std::memset(&a, 0, sizeof a);
  a.n_instances = prob->n_instances;
  a.F_max = prob->integer_path ? prob->max_field : 0;
  a.max_colors = prob->max_colors;
  a.max_item_bytes = args->max_item_bytes;
  a.desc = prob->desc;
  a.color_ptr = prob->color_ptr;
  a.slice_off = prob->slice_off;
  a.ell_nbr = prob->ell_nbr;
  a.ell_w = prob->ell_w;
  a.h_pos = prob->h_pos;
  a.betas = prob->betas;
  a.thr = prob->thresholds;
  a.n_rounds = args->n_rounds;
  a.spr = args->sweeps_per_round;
  a.round0 = args->round_offset;
  a.k0 = (uint32_t)(args->seed & 0xffffffffu);
  a.k1 = (uint32_t)(args->seed >> 32);
  a.items = args->items;
  a.n_items = args->n_items;
  a.max_tile = args->max_tile;
  a.tps = tps;
  a.spins = state->spins;
  a.energy = reinterpret_cast<long long*>(state->energy);
  a.best_energy = reinterpret_cast<long long*>(state->best_energy);
  a.best_spins = state->best_spins;
  a.rung_of_slot = state->rung_of_slot;
  a.slot_of_rung = state->slot_of_rung;
  a.tried = reinterpret_cast<long long*>(state->swap_tried);
  a.accepted = reinterpret_cast<long long*>(state->swap_accepted);
  unsigned char* ws = static_cast<unsigned char*>(workspace);
  a.bar = reinterpret_cast<unsigned long long*>(ws);
  a.ctr = reinterpret_cast<unsigned long long*>(ws + 8);
  a.err = reinterpret_cast<int*>(ws + 16);
  a.timeout_ns = (long long)((args->timeout_s > 0 ? args->timeout_s : 10.0) * 1e9);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  e = cudaMemsetAsync(ws, 0, kBatchWsHeader, st);
  if (e != cudaSuccess) return b_fail(e, "workspace reset");
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
  e = cudaLaunchKernelExC(&cfg, fn, kargs);
  if (e != cudaSuccess) return b_fail(e, "pt_batched_kernel launch");
  return DRIFT_PT_OK;
}
