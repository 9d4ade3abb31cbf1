// dpt_capi.cu - device layer and host convenience entry points of the C ABI (include/drift_pt.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <tuple>
#include <mutex>
#include <utility>
#include <vector>

#include "../../include/drift_pt.h"
#include "dpt_common.cuh"
#include "dpt_internal.h"
#include "dpt_kernels.cuh"

namespace dpt {

int prepare_kernel(const void* fn, int threads, size_t smem, int* per_sm) {
  struct Key {
    const void* fn;
    int dev, threads;
    size_t smem;
    bool operator<(const Key& o) const {
      if (fn != o.fn) return fn < o.fn;
      if (dev != o.dev) return dev < o.dev;
      if (threads != o.threads) return threads < o.threads;
      return smem < o.smem;
    }
  };
  static std::mutex mu;
  static std::map<Key, int> occ;
  static std::map<std::pair<const void*, int>, size_t> smem_set;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lock(mu);
  const Key key{fn, dev, threads, smem};
  auto it = occ.find(key);
  if (it != occ.end()) {
    *per_sm = it->second;
    return DRIFT_PT_OK;
  }
  size_t& cur = smem_set[std::make_pair(fn, dev)];
  if (cur < smem) {
    cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return set_error(DRIFT_PT_ECUDA, "cudaFuncSetAttribute: %s", cudaGetErrorString(e));
    cur = smem;
  }
  int n = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, fn, threads, smem);
  if (e != cudaSuccess) return set_error(DRIFT_PT_ECUDA, "occupancy query: %s", cudaGetErrorString(e));
  occ[key] = n;
  *per_sm = n;
  return DRIFT_PT_OK;
}

}  // namespace dpt

using namespace dpt;

namespace {

// Workspace: 256-byte header (error flag, i32, at 8), then [2][R] int64 published energies and
// [2][R] uint64 round tags; all of it is cleared at the start of every launch.
constexpr size_t kWsHeader = 256;

struct DeviceInfo {
  int sm_count = 0;
  int max_smem_optin = 0;
};

int device_info(DeviceInfo* di) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return set_error(DRIFT_PT_ECUDA, "cudaGetDevice failed");
  if (cudaDeviceGetAttribute(&di->sm_count, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
      cudaDeviceGetAttribute(&di->max_smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess)
    return set_error(DRIFT_PT_ECUDA, "cudaDeviceGetAttribute failed");
  return DRIFT_PT_OK;
}

int cuda_fail(cudaError_t e, const char* what) {
  return set_error(DRIFT_PT_ECUDA, "%s: %s", what, cudaGetErrorString(e));
}

int validate_problem(const DriftPtDeviceProblem* p) {
  if (!p) return set_error(DRIFT_PT_EINVAL, "problem is NULL");
  if (p->n < 1 || p->n_pos < p->n || p->n_pos % kSlicePositions || p->n_slices * kSlicePositions != p->n_pos)
    return set_error(DRIFT_PT_EINVAL, "inconsistent problem sizes (n=%d, n_pos=%d, n_slices=%d)", p->n, p->n_pos, p->n_slices);
  if (p->n_colors < 1 || p->max_class < 1 || p->n_ell < 0 || p->n_ell % kSlicePositions)
    return set_error(DRIFT_PT_EINVAL, "inconsistent colouring / ELL sizes");
  if (!p->color_ptr || !p->slice_off || !p->h_pos || (p->n_ell > 0 && (!p->ell_nbr || !p->ell_w)))
    return set_error(DRIFT_PT_EINVAL, "problem arrays missing");
  if (p->integer_path && p->max_field < 1) return set_error(DRIFT_PT_EINVAL, "integer path needs max_field >= 1");
  return DRIFT_PT_OK;
}

int validate_state(const DriftPtDeviceState* s, int R) {
  if (!s || !s->spins || !s->energy || !s->best_energy || !s->best_spins || !s->rung_of_slot || !s->slot_of_rung ||
      (R > 1 && (!s->swap_tried || !s->swap_accepted)))
    return set_error(DRIFT_PT_EINVAL, "state arrays missing");
  return DRIFT_PT_OK;
}

PtKernelArgs make_args(const DriftPtDeviceProblem* p, const DriftPtRunArgs* r, DriftPtDeviceState* s) {
  PtKernelArgs a;
  std::memset(&a, 0, sizeof a);
  a.n = p->n;
  a.n_pos = p->n_pos;
  a.n_slices = p->n_slices;
  a.n_colors = p->n_colors;
  a.F = p->integer_path ? p->max_field : 0;
  a.n_ell = p->n_ell;
  a.color_ptr = p->color_ptr;
  a.slice_off = p->slice_off;
  a.ell_nbr = p->ell_nbr;
  a.ell_w = p->ell_w;
  a.h_pos = p->h_pos;
  a.unit_place = p->unit_place;
  a.R = r->n_replicas;
  a.spr = r->sweeps_per_round;
  a.n_rounds = r->n_rounds;
  a.round0 = r->round_offset;
  a.k0 = (uint32_t)(r->seed & 0xffffffffu);
  a.k1 = (uint32_t)(r->seed >> 32);
  a.inst = r->instance;
  a.betas = r->betas;
  a.thr = r->thresholds;
  a.spins = s->spins;
  a.energy = reinterpret_cast<long long*>(s->energy);
  a.best_energy = reinterpret_cast<long long*>(s->best_energy);
  a.best_spins = s->best_spins;
  a.rung_of_slot = s->rung_of_slot;
  a.slot_of_rung = s->slot_of_rung;
  a.tried = reinterpret_cast<long long*>(s->swap_tried);
  a.accepted = reinterpret_cast<long long*>(s->swap_accepted);
  a.best_hist = s->best_history;
  return a;
}

}  // namespace

extern "C" int drift_pt_workspace_bytes(int32_t n_replicas, size_t* bytes) {
  clear_error();
  if (n_replicas < 1 || !bytes) return set_error(DRIFT_PT_EINVAL, "workspace_bytes: invalid arguments");
  *bytes = kWsHeader + 2 * ((2 * sizeof(long long) * (size_t)n_replicas + 255) & ~(size_t)255);
  return DRIFT_PT_OK;
}

extern "C" int drift_pt_init(const DriftPtDeviceProblem* prob, const DriftPtRunArgs* args,
                             DriftPtDeviceState* state, void* stream) {
  clear_error();
  int rc = validate_problem(prob);
  if (rc) return rc;
  if (!args || args->n_replicas < 1) return set_error(DRIFT_PT_EINVAL, "n_replicas must be >= 1");
  if (args->instance > kMaxInstance) return set_error(DRIFT_PT_EINVAL, "instance must be < 2^24");
  rc = validate_state(state, args->n_replicas);
  if (rc) return rc;
  PtKernelArgs a = make_args(prob, args, state);
  cudaError_t e = launch_init(a, prob->integer_path, static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return cuda_fail(e, "drift_pt_init launch");
  return DRIFT_PT_OK;
}

namespace {

struct LaunchPlan {
  int rpc, threads, in_smem, grid, p;
  int cluster;  // > 0: the grid is one cluster of this many CTAs
  int unit;     // > 0: the unit-regular item form, compiled for this many colour phases at most
  size_t smem;
};

constexpr int kMaxCluster = 16;

// Can `C` CTAs of `threads` threads and `smem` bytes run as one cluster on this device? The answer
// is cached per kernel, device and shape (the occupancy query costs more than a small run).
int cluster_fits(const void* fn, int C, int threads, size_t smem, bool* ok) {
  *ok = false;
  int dev = 0;
  cudaGetDevice(&dev);
  static std::mutex mu;
  static std::map<std::tuple<const void*, int, int, int, size_t>, bool> known;
  std::lock_guard<std::mutex> lock(mu);
  const auto key = std::make_tuple(fn, dev, C, threads, smem);
  const auto it = known.find(key);
  if (it != known.end()) {
    *ok = it->second;
    return DRIFT_PT_OK;
  }
  if (C > 8) {
    const cudaError_t e = cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
    if (e != cudaSuccess) return cuda_fail(e, "cluster size attribute");
  }
  cudaLaunchConfig_t cfg;
  std::memset(&cfg, 0, sizeof cfg);
  cfg.gridDim = dim3(C);
  cfg.blockDim = dim3(threads);
  cfg.dynamicSmemBytes = smem;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = C;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  int n = 0;
  const cudaError_t e = cudaOccupancyMaxActiveClusters(&n, fn, &cfg);
  if (e != cudaSuccess) return cuda_fail(e, "cluster occupancy query");
  *ok = n >= 1;
  known[key] = *ok;
  return DRIFT_PT_OK;
}

int plan_launch(const DriftPtDeviceProblem* p, const DriftPtRunArgs* r, LaunchPlan* lp) {
  DeviceInfo di;
  int rc = device_info(&di);
  if (rc) return rc;
  const int R = r->n_replicas;
  const int ip = p->integer_path;
  auto total = [&](int rpc, bool ell, int threads, bool cluster = false) {
    return smem_layout(p->n_pos, rpc, R, p->max_field, p->n_colors, p->n_slices, p->n_ell, ip != 0, ell, threads,
                       cluster)
        .total;
  };
  // positions per item (8, 4 or 1; the fp32 path always uses 8); 0 = chosen below
  const int P_user = r->positions_per_item;
  if (P_user != 0 && P_user != 8 && P_user != 4 && P_user != 2 && P_user != 1)
    return set_error(DRIFT_PT_EINVAL, "positions_per_item must be 0, 1, 2, 4 or 8");
  // threads per slot: one per item of the largest colour class (32-group runs times 8/P
  // sub-blocks), as a power of two below 32 or a multiple of 32, with rpc * tps a multiple of 32
  // and at most kMaxThreads (0 = none)
  auto want_of = [&](int P_) { return ((p->max_class / kGroup + 2 + 31) / 32) * 32 * (kGroup / P_); };
  auto pick_tps = [&](int rpc, int P_) -> int {
    const int want = want_of(P_);
    int tps = 1;
    while (tps < 32 && tps < want) tps *= 2;
    if (tps >= 32) tps = ((want + 31) / 32) * 32;
    while (rpc * tps > kMaxThreads && tps > 1) tps = tps > 32 ? tps - 32 : tps / 2;
    while ((rpc * tps) % 32 != 0) {
      tps = tps < 32 ? tps * 2 : tps + 32;
      if (rpc * tps > kMaxThreads) return 0;
    }
    return rpc * tps <= kMaxThreads ? tps : 0;
  };
  // one pass over each colour class: the slot gets a thread for every item of the largest class
  auto one_pass = [&](int rpc, int P_) {
    const int want = want_of(P_);
    int full = 1;
    while (full < 32 && full < want) full *= 2;
    if (full >= 32) full = ((want + 31) / 32) * 32;
    return pick_tps(rpc, P_) == full;
  };
  auto shape_ok = [&](int rpc_, int threads_) {
    const int tps = threads_ / rpc_;
    const bool pow2 = tps > 0 && (tps & (tps - 1)) == 0;
    return threads_ >= 32 && threads_ <= kMaxThreads && threads_ % 32 == 0 && threads_ % rpc_ == 0 &&
           (tps % 32 == 0 || (tps < 32 && pow2));
  };
  const int mode = r->round_sync;
  if (mode < 0 || mode > 2) return set_error(DRIFT_PT_EINVAL, "round_sync must be 0 (auto), 1 (grid) or 2 (cluster)");
  lp->cluster = 0;
  lp->unit = 0;

  // ---- the unit-regular form: one replica slot per CTA, 2 or 4 positions per item, neighbour addresses
  // and the decision table staged in shared memory (problems whose spins all have W couplings of
  // +-1 and no field) ----
  const int form = r->item_form;
  if (form < 0 || form > 2) return set_error(DRIFT_PT_EINVAL, "item_form must be 0 (auto), 1 (gather) or 2 (unit)");
  const bool unit_ok = ip && p->unit_regular && !p->has_field && p->max_width == p->min_width &&
                       p->max_field == p->max_width && unit_width_supported(p->max_width) &&
                       r->replicas_per_cta <= 1 && (P_user == 0 || P_user == 2 || P_user == 4) &&
                       p->n_colors <= kUnitPhases && 2 * (long long)p->n_pos + 16 <= 65536 &&
                       r->sweeps_per_round <= (1 << 23) &&
                       (p->max_class + 14) / kGroup * 2 <= kMaxUnitThreads;
  if (form == 2 && !unit_ok)
    return set_error(DRIFT_PT_EUNSUPPORTED,
                     "item_form 2 needs a unit-regular problem (every spin with the same number, 2, 3, 4 or 6, of "
                     "+-1 couplings, no field, at most 32760 positions, at most 4 colour classes of at most 4080 "
                     "spins), at most 2^23 sweeps per round, one replica per CTA and 2 or 4 positions per item");
  if (P_user == 2 && (!unit_ok || form == 1))
    return set_error(DRIFT_PT_EINVAL, "positions_per_item 2 exists in the unit-regular form only");
  if (unit_ok && form != 1) {
    const int W = p->max_width;
    // items of the largest colour class: a class of m positions touches at most (m + 14) / 8 groups
    auto items_of = [&](int P_) { return ((p->max_class + 14) / kGroup) * (kGroup / P_); };
    const int PU = P_user ? P_user : unit_auto_positions(p->max_class);
    const int uph = p->n_colors <= 2 ? 2 : kUnitPhases;  // the instance compiled for these phases
    auto total_u = [&](int threads_, bool cl) {
      return smem_layout(p->n_pos, 1, R, p->max_field, p->n_colors, p->n_slices, p->n_ell, true, true, threads_, cl,
                         W, PU)
          .total;
    };
    // one item per thread and colour phase (the kernel's static schedule)
    const int threads = r->threads_per_cta > 0 ? r->threads_per_cta : ((items_of(PU) + 31) / 32) * 32;
    if (threads >= items_of(PU) && threads <= unit_max_threads(PU) && threads % 32 == 0) {
      if (mode != 1 && R >= 2 && R <= kMaxCluster && total_u(threads, true) <= (size_t)di.max_smem_optin) {
        const void* fn = run_kernel_ptr(ip, 1, W, W, 0, PU, 1, uph);
        const size_t smem = total_u(threads, true);
        int per_sm = 0;
        bool ok = false;
        rc = prepare_kernel(fn, threads, smem, &per_sm);
        if (rc) return rc;
        rc = cluster_fits(fn, R, threads, smem, &ok);
        if (rc) return rc;
        if (ok) {
          *lp = LaunchPlan{1, threads, 1, R, PU, R, uph, smem};
          return DRIFT_PT_OK;
        }
      }
      if (mode != 2 && total_u(threads, false) <= (size_t)di.max_smem_optin) {
        const void* fn = run_kernel_ptr(ip, 1, W, W, 0, PU, 0, uph);
        const size_t smem = total_u(threads, false);
        int per_sm = 0;
        rc = prepare_kernel(fn, threads, smem, &per_sm);
        if (rc) return rc;
        if ((long long)per_sm * di.sm_count >= R) {
          // Chosen over every form of the gather: on B200 it ran 2-D EA L = 16 with 24 replicas and a
          // swap after every sweep at 3.4 attempts/ns against 2.6 for the gather's cluster form.
          *lp = LaunchPlan{1, threads, 1, R, PU, 0, uph, smem};
          return DRIFT_PT_OK;
        }
      }
    }
    if (form == 2)
      return set_error(DRIFT_PT_EUNSUPPORTED, "item_form 2: no launch shape with one replica per CTA fits (%d replicas, "
                       "%d positions, round_sync %d)", R, p->n_pos, mode);
  }
  // ---- the cluster form: the ladder in one cluster of at most 16 CTAs, coupling table in shared
  // memory; a round's energies cross through distributed shared memory behind one barrier ----
  auto try_cluster = [&](int P_, bool require_one_pass, bool* done) -> int {
    *done = false;
    if (R < 2) return DRIFT_PT_OK;
    int rc_c = r->replicas_per_cta;
    if (rc_c <= 0) {
      rc_c = 1;
      while ((R + rc_c - 1) / rc_c > kMaxCluster) rc_c *= 2;
    }
    rc_c = std::min(rc_c, R);
    const int C = (R + rc_c - 1) / rc_c;
    int thr_c = r->threads_per_cta;
    bool ok = C >= 2 && C <= kMaxCluster;
    if (ok && thr_c <= 0) {
      ok = pick_tps(rc_c, P_) > 0 && (!require_one_pass || one_pass(rc_c, P_));
      thr_c = rc_c * pick_tps(rc_c, P_);
    }
    ok = ok && shape_ok(rc_c, thr_c) && total(rc_c, true, thr_c, true) <= (size_t)di.max_smem_optin;
    if (!ok) return DRIFT_PT_OK;
    const void* fn = run_kernel_ptr(ip, 1, p->max_width, p->min_width, p->has_field, P_, 1);
    if (!fn) return DRIFT_PT_OK;
    const size_t smem = total(rc_c, true, thr_c, true);
    int per_sm = 0;
    int rc2 = prepare_kernel(fn, thr_c, smem, &per_sm);
    if (rc2) return rc2;
    rc2 = cluster_fits(fn, C, thr_c, smem, &ok);
    if (rc2 || !ok) return rc2;
    lp->rpc = rc_c;
    lp->p = P_;
    lp->threads = thr_c;
    lp->in_smem = 1;
    lp->grid = C;
    lp->cluster = C;
    lp->smem = smem;
    *done = true;
    return DRIFT_PT_OK;
  };

  // ---- the grid form: any ladder; CTAs meet at a bounded barrier in global memory ----
  auto plan_grid = [&](int P_) -> int {
    int rpc = r->replicas_per_cta;
    if (rpc <= 0) {
      // One replica per CTA, as many CTAs as SMs allow. Measured on B200 from 24 to 576 spins,
      // 16-64 replicas and 1-5 sweeps per round, this beats keeping every replica in one CTA
      // (which needs no grid barrier) by 1.3x to 13x: the grid barrier costs less than running
      // the replicas one after another on one SM.
      rpc = 1;
      while (rpc < R && (R + rpc - 1) / rpc > di.sm_count) rpc *= 2;
      rpc = std::min(rpc, R);
      while (rpc > 1 && pick_tps(rpc, P_) == 0) rpc /= 2;
    }
    rpc = std::min(rpc, R);
    if ((R + rpc - 1) / rpc > 65535) return set_error(DRIFT_PT_EUNSUPPORTED, "too many CTAs");
    int threads = r->threads_per_cta;
    if (threads <= 0) {
      const int tps = pick_tps(rpc, P_);
      if (tps == 0) return set_error(DRIFT_PT_EUNSUPPORTED, "no launch shape for %d replicas per CTA", rpc);
      threads = rpc * tps;
    }
    if (!shape_ok(rpc, threads))
      return set_error(DRIFT_PT_EINVAL,
                       "threads_per_cta (%d) must be a multiple of 32 in [32, 512] and of replicas_per_cta (%d), "
                       "with threads/replica a power of two below 32 or a multiple of 32", threads, rpc);
    if (total(rpc, false, threads) > (size_t)di.max_smem_optin)
      return set_error(DRIFT_PT_EUNSUPPORTED, "replica state of %d x %d positions exceeds shared memory (%d B)", rpc,
                       p->n_pos, di.max_smem_optin);
    const bool in_smem = total(rpc, true, threads) <= (size_t)di.max_smem_optin;
    lp->rpc = rpc;
    lp->p = P_;
    lp->threads = threads;
    lp->in_smem = in_smem ? 1 : 0;
    lp->grid = (R + rpc - 1) / rpc;
    lp->smem = total(rpc, in_smem, threads);
    const void* fn = run_kernel_ptr(ip, lp->in_smem, p->max_width, p->min_width, p->has_field, lp->p);
    if (!fn)
      return set_error(DRIFT_PT_EUNSUPPORTED, "one position per item needs the coupling table in shared memory");
    int per_sm = 0;
    const int rc2 = prepare_kernel(fn, threads, lp->smem, &per_sm);
    if (rc2) return rc2;
    if ((long long)per_sm * di.sm_count < lp->grid)
      return set_error(DRIFT_PT_EUNSUPPORTED,
                       "%d CTAs of %d threads / %zu B shared memory cannot be co-resident (%d per SM x %d SMs)",
                       lp->grid, threads, lp->smem, per_sm, di.sm_count);
    return DRIFT_PT_OK;
  };

  bool done = false;
  if (!ip || P_user != 0 || r->replicas_per_cta > 0 || r->threads_per_cta > 0 || mode != 0) {
    // the caller fixed part of the shape: the integer path defaults to 4 positions per item
    const int P = !ip ? 8 : (P_user ? P_user : 4);
    if (mode != 1) {
      rc = try_cluster(P, mode == 0, &done);
      if (rc || done) return rc;
      if (mode == 2)
        return set_error(DRIFT_PT_EUNSUPPORTED, "round_sync = 2: the ladder does not fit one cluster of at most %d "
                         "CTAs with its coupling table in shared memory", kMaxCluster);
    }
    return plan_grid(P);
  }
  // Automatic shape on the integer path, from measurements on B200 (2-D EA L = 8, 16, 32 with 16-24
  // replicas and G(n, p) n = 400 with 32, 1-4 sweeps per round):
  //  * one position per item (the gather chain of a quarter of the positions) wins with one
  //    replica per CTA when a class takes one pass, and loses with two replicas per CTA;
  //  * the cluster form's round end is ~0.35 us shorter than the grid form's, a position per item
  //    saves ~0.1 us per colour phase: with 16 replicas or fewer both are had at once; otherwise
  //    the cluster (4 positions per item, 2+ replicas per CTA) wins below 4 colour phases per round
  //    and one replica per CTA with a position per item from 4 phases on;
  //  * 4 positions per item elsewhere (the largest classes, many replicas).
  const bool p1_alone = one_pass(1, 1) && total(1, true, pick_tps(1, 1)) <= (size_t)di.max_smem_optin;
  const long long phases = (long long)r->sweeps_per_round * p->n_colors;
  if (p1_alone && R <= kMaxCluster) {
    rc = try_cluster(1, true, &done);
    if (rc || done) return rc;
  }
  if (p1_alone && R <= di.sm_count && phases >= 4) return plan_grid(1);
  rc = try_cluster(4, true, &done);
  if (rc || done) return rc;
  return plan_grid(p1_alone && R <= di.sm_count ? 1 : 4);
}

}  // namespace

extern "C" int drift_pt_run(const DriftPtDeviceProblem* prob, const DriftPtRunArgs* args,
                            DriftPtDeviceState* state, void* workspace, size_t workspace_bytes, void* stream) {
  clear_error();
  int rc = validate_problem(prob);
  if (rc) return rc;
  if (!args || args->n_replicas < 1 || args->n_rounds < 0 || args->sweeps_per_round < 1 || args->round_offset < 0)
    return set_error(DRIFT_PT_EINVAL, "run args: need n_replicas >= 1, n_rounds >= 0, sweeps_per_round >= 1");
  if (args->instance > kMaxInstance) return set_error(DRIFT_PT_EINVAL, "instance must be < 2^24");
  if (!args->betas || (prob->integer_path && !args->thresholds))
    return set_error(DRIFT_PT_EINVAL, "run args: betas (and thresholds on the integer path) are required");
  rc = validate_state(state, args->n_replicas);
  if (rc) return rc;
  size_t need = 0;
  drift_pt_workspace_bytes(args->n_replicas, &need);
  if (!workspace || workspace_bytes < need)
    return set_error(DRIFT_PT_EINVAL, "workspace of %zu bytes is smaller than the %zu required", workspace_bytes, need);
  if (args->n_rounds == 0) return DRIFT_PT_OK;
  LaunchPlan lp;
  rc = plan_launch(prob, args, &lp);
  if (rc) return rc;
  PtKernelArgs a = make_args(prob, args, state);
  a.rpc = lp.rpc;
  unsigned char* ws = static_cast<unsigned char*>(workspace);
  const size_t half = (2 * sizeof(long long) * (size_t)args->n_replicas + 255) & ~(size_t)255;
  a.err = reinterpret_cast<int*>(ws + 8);
  a.pub = reinterpret_cast<long long*>(ws + kWsHeader);
  a.tags = reinterpret_cast<unsigned long long*>(ws + kWsHeader + half);
  // integer energies obey |E| <= n F: below 2^31 they travel with their round tag in one word
  a.packed = prob->integer_path && (long long)prob->n * prob->max_field < (1ll << 31) ? 1 : 0;
  const double to = args->timeout_s > 0 ? args->timeout_s : 10.0;
  a.timeout_ns = (long long)(to * 1e9);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaError_t e = cudaMemsetAsync(ws, 0, need, st);
  if (e != cudaSuccess) return cuda_fail(e, "workspace reset");
  cudaLaunchConfig_t cfg;
  std::memset(&cfg, 0, sizeof cfg);
  cfg.gridDim = dim3(lp.grid);
  cfg.blockDim = dim3(lp.threads);
  cfg.dynamicSmemBytes = lp.smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  if (lp.cluster > 0) {
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = lp.cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
  } else {
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
  }
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  void* kargs[] = {&a};
  e = cudaLaunchKernelExC(&cfg, run_kernel_ptr(prob->integer_path, lp.in_smem, prob->max_width, prob->min_width,
                                                prob->has_field, lp.p, lp.cluster > 0 ? 1 : 0, lp.unit),
                          kargs);
  if (e != cudaSuccess) return cuda_fail(e, "pt_run_kernel launch");
  return DRIFT_PT_OK;
}

extern "C" int drift_pt_check(void* workspace, void* stream) {
  clear_error();
  if (!workspace) return set_error(DRIFT_PT_EINVAL, "workspace is NULL");
  cudaError_t e = cudaStreamSynchronize(static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return cuda_fail(e, "stream synchronize");
  int flag = 0;
  e = cudaMemcpy(&flag, static_cast<unsigned char*>(workspace) + 8, sizeof flag, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(e, "error flag read");
  if (flag) return set_error(DRIFT_PT_ETIMEOUT, "a bounded in-kernel wait timed out (flag %d); the state is incomplete", flag);
  return DRIFT_PT_OK;
}

extern "C" int drift_pt_energy_fp64(const DriftPtDeviceProblem* prob, const int8_t* spins, int32_t n_replicas,
                                    double* out, void* stream) {
  clear_error();
  int rc = validate_problem(prob);
  if (rc) return rc;
  if (!spins || !out || n_replicas < 1) return set_error(DRIFT_PT_EINVAL, "energy_fp64: invalid arguments");
  DriftPtRunArgs r;
  std::memset(&r, 0, sizeof r);
  r.n_replicas = n_replicas;
  DriftPtDeviceState s;
  std::memset(&s, 0, sizeof s);
  PtKernelArgs a = make_args(prob, &r, &s);
  cudaError_t e = launch_energy_fp64(a, prob->integer_path, spins, n_replicas, out, static_cast<cudaStream_t>(stream));
  if (e != cudaSuccess) return cuda_fail(e, "energy_fp64 launch");
  return DRIFT_PT_OK;
}

// ---------------------------------------------------------------------------------------------
// drift_pt_solve: host buffers in, host results out.
// ---------------------------------------------------------------------------------------------
namespace {

// The device arena of drift_pt_solve, kept per thread and device across calls and grown when a call
// needs more: a solve then allocates and frees no device memory when an earlier one on the same
// thread was as large, and makes fewer driver calls (each a chance to wait on the driver's lock
// while another process queries the GPU). Every array a solve reads is written by it first
// (upload, initialisation), so nothing carries over from one call to the next.
// drift_pt_solve_release frees it.
struct SolveArena {
  int dev = -1;
  void* base = nullptr;
  size_t cap = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  void release() {
    if (base) cudaFree(base);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    base = nullptr;
    ev0 = ev1 = nullptr;
    cap = 0;
    dev = -1;
  }
  ~SolveArena() { release(); }
};

SolveArena& thread_arena() {
  static thread_local SolveArena a;
  return a;
}

int solve_arena(size_t bytes, SolveArena** out) {
  SolveArena& a = thread_arena();
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return set_error(DRIFT_PT_ECUDA, "cudaGetDevice failed");
  if (a.dev != dev) a.release();
  if (a.cap < bytes) {
    if (a.base) cudaFree(a.base);
    a.base = nullptr;
    a.cap = 0;
    const cudaError_t e = cudaMalloc(&a.base, bytes);
    if (e != cudaSuccess) {
      a.base = nullptr;
      return set_error(DRIFT_PT_ENOMEM, "cudaMalloc of %zu bytes failed: %s", bytes, cudaGetErrorString(e));
    }
    a.cap = bytes;
  }
  if (!a.ev0 && (cudaEventCreate(&a.ev0) != cudaSuccess || cudaEventCreate(&a.ev1) != cudaSuccess))
    return set_error(DRIFT_PT_ECUDA, "solve: cudaEventCreate failed");
  a.dev = dev;
  *out = &a;
  return DRIFT_PT_OK;
}

size_t bump(size_t& off, size_t bytes) {
  size_t o = off;
  off = (off + bytes + 255) & ~(size_t)255;
  return o;
}

}  // namespace

extern "C" int drift_pt_solve_release(void) {
  clear_error();
  thread_arena().release();
  return DRIFT_PT_OK;
}

extern "C" int drift_pt_solve(const DriftPtCsr* csr, const DriftPtSolveArgs* args, DriftPtSolveResult* out) {
  clear_error();
  if (!args || !out || !out->best_s) return set_error(DRIFT_PT_EINVAL, "solve: args/out/best_s required");
  const int R = args->n_replicas;
  if (R < 1 || args->n_rounds < 0 || args->sweeps_per_round < 1)
    return set_error(DRIFT_PT_EINVAL, "solve: need n_replicas >= 1, n_rounds >= 0, sweeps_per_round >= 1");
  DriftPtLayoutInfo info;
  int rc = drift_pt_layout_query(csr, &info);
  if (rc) return rc;
  const int ip = info.integer_couplings;
  // ---- ladder (drift/solvers/parallel_tempering.py:29-36,72-73) ----
  std::vector<double> betas((size_t)R);
  if (args->betas) {
    for (int r = 0; r < R; ++r) betas[r] = args->betas[r];
  } else {
    if (!(args->T_min > 0.0) || !(args->T_max > 0.0)) return set_error(DRIFT_PT_EINVAL, "solve: T_min and T_max must be > 0");
    for (int r = 0; r < R; ++r) {
      double T = (R == 1) ? args->T_min : args->T_min * std::pow(args->T_max / args->T_min, (double)r / (R - 1));
      betas[r] = 1.0 / std::max(T, 1e-12);
    }
  }
  std::vector<uint32_t> thr;
  if (ip) {
    thr.resize((size_t)R * info.max_field);
    rc = drift_pt_thresholds(R, betas.data(), info.max_field, thr.data());
    if (rc) return rc;
  }
  // ---- host layout ----
  std::vector<int32_t> color_ptr(info.n_colors + 1), slice_off(info.n_slices + 1), ell_nbr(info.n_ell),
      site_of_pos(info.n_pos), pos_of_site(info.n);
  std::vector<unsigned char> ell_w((size_t)info.n_ell * (ip ? 1 : 4)), h_pos((size_t)info.n_pos * 4);
  DriftPtLayout lay{color_ptr.data(), slice_off.data(), ell_nbr.data(), ell_w.data(), h_pos.data(), site_of_pos.data(),
                    pos_of_site.data()};
  rc = drift_pt_layout_fill(csr, ip, &lay);
  if (rc) return rc;
  int max_class = 1;
  for (int c = 0; c < info.n_colors; ++c) max_class = std::max(max_class, color_ptr[c + 1] - color_ptr[c]);
  // the unit-regular form's storage order of spin bytes
  std::vector<uint16_t> place;
  if (ip && info.unit_regular) {
    place.resize((size_t)info.n_pos / 4);
    rc = drift_pt_unit_placement(csr, 0, place.data());
    if (rc) return rc;
  }
  // ---- device arena: the inputs first (one upload), then the results read back together, then
  // the device-only state; the arena is kept per thread and device across calls ----
  size_t ws_bytes = 0;
  drift_pt_workspace_bytes(R, &ws_bytes);
  size_t off = 0;
  const size_t o_cp = bump(off, color_ptr.size() * 4), o_so = bump(off, slice_off.size() * 4),
               o_nb = bump(off, ell_nbr.size() * 4), o_w = bump(off, ell_w.size()), o_h = bump(off, h_pos.size()),
               o_beta = bump(off, (size_t)R * 8), o_thr = bump(off, thr.size() * 4), o_pl = bump(off, place.size() * 2);
  const size_t up_bytes = off;
  const size_t o_be = bump(off, (size_t)R * 8), o_e = bump(off, (size_t)R * 8), o_sr = bump(off, (size_t)R * 4),
               o_tr = bump(off, (size_t)R * 8), o_ac = bump(off, (size_t)R * 8);
  const size_t res_bytes = off - o_be;
  const size_t o_bh = bump(off, (size_t)std::max(1, args->n_rounds) * 8), o_sp = bump(off, (size_t)R * info.n_pos),
               o_bsp = bump(off, (size_t)R * info.n_pos), o_rs = bump(off, (size_t)R * 4), o_ws = bump(off, ws_bytes);
  SolveArena* arena = nullptr;
  rc = solve_arena(off, &arena);
  if (rc) return rc;
  unsigned char* d = static_cast<unsigned char*>(arena->base);
  cudaError_t e;
  {
    std::vector<unsigned char> stage(up_bytes);
    auto put = [&](size_t o, const void* src, size_t bytes) {
      if (bytes) std::memcpy(stage.data() + o, src, bytes);
    };
    put(o_cp, color_ptr.data(), color_ptr.size() * 4);
    put(o_so, slice_off.data(), slice_off.size() * 4);
    put(o_nb, ell_nbr.data(), ell_nbr.size() * 4);
    put(o_w, ell_w.data(), ell_w.size());
    put(o_h, h_pos.data(), h_pos.size());
    put(o_beta, betas.data(), (size_t)R * 8);
    put(o_thr, thr.data(), thr.size() * 4);
    put(o_pl, place.data(), place.size() * 2);
    if ((e = cudaMemcpy(d, stage.data(), up_bytes, cudaMemcpyHostToDevice)) != cudaSuccess)
      return cuda_fail(e, "solve: upload");
  }
  DriftPtDeviceProblem prob;
  std::memset(&prob, 0, sizeof prob);
  prob.n = info.n;
  prob.n_pos = info.n_pos;
  prob.n_slices = info.n_slices;
  prob.n_colors = info.n_colors;
  prob.integer_path = ip;
  prob.max_field = info.max_field;
  prob.max_width = info.max_degree;
  prob.min_width = info.min_width;
  prob.unit_regular = ip ? info.unit_regular : 0;
  prob.max_class = max_class;
  prob.has_field = info.has_field;
  prob.n_ell = info.n_ell;
  prob.color_ptr = reinterpret_cast<const int32_t*>(d + o_cp);
  prob.slice_off = reinterpret_cast<const int32_t*>(d + o_so);
  prob.ell_nbr = reinterpret_cast<const int32_t*>(d + o_nb);
  prob.ell_w = d + o_w;
  prob.h_pos = d + o_h;
  prob.unit_place = place.empty() ? nullptr : reinterpret_cast<const uint16_t*>(d + o_pl);
  DriftPtDeviceState st;
  st.spins = reinterpret_cast<int8_t*>(d + o_sp);
  st.best_spins = reinterpret_cast<int8_t*>(d + o_bsp);
  st.energy = reinterpret_cast<int64_t*>(d + o_e);
  st.best_energy = reinterpret_cast<int64_t*>(d + o_be);
  st.rung_of_slot = reinterpret_cast<int32_t*>(d + o_rs);
  st.slot_of_rung = reinterpret_cast<int32_t*>(d + o_sr);
  st.swap_tried = reinterpret_cast<int64_t*>(d + o_tr);
  st.swap_accepted = reinterpret_cast<int64_t*>(d + o_ac);
  st.best_history = reinterpret_cast<double*>(d + o_bh);
  DriftPtRunArgs ra;
  std::memset(&ra, 0, sizeof ra);
  ra.n_replicas = R;
  ra.n_rounds = args->n_rounds;
  ra.sweeps_per_round = args->sweeps_per_round;
  ra.seed = args->seed;
  ra.betas = reinterpret_cast<const double*>(d + o_beta);
  ra.thresholds = ip ? reinterpret_cast<const uint32_t*>(d + o_thr) : nullptr;
  rc = drift_pt_init(&prob, &ra, &st, nullptr);
  if (rc) return rc;
  cudaEventRecord(arena->ev0, nullptr);
  rc = drift_pt_run(&prob, &ra, &st, d + o_ws, ws_bytes, nullptr);
  cudaEventRecord(arena->ev1, nullptr);
  if (rc == DRIFT_PT_OK) rc = drift_pt_check(d + o_ws, nullptr);
  float ms = 0.0f;
  cudaEventElapsedTime(&ms, arena->ev0, arena->ev1);
  if (rc) return rc;
  // ---- results: energies, bests, permutation and swap counts in one copy ----
  std::vector<unsigned char> res(res_bytes);
  if ((e = cudaMemcpy(res.data(), d + o_be, res_bytes, cudaMemcpyDeviceToHost)) != cudaSuccess)
    return cuda_fail(e, "solve: download");
  const long long* be = reinterpret_cast<const long long*>(res.data());
  const long long* en = reinterpret_cast<const long long*>(res.data() + (o_e - o_be));
  const int32_t* slot_of_rung = reinterpret_cast<const int32_t*>(res.data() + (o_sr - o_be));
  const long long* tried = reinterpret_cast<const long long*>(res.data() + (o_tr - o_be));
  const long long* acc = reinterpret_cast<const long long*>(res.data() + (o_ac - o_be));
  int best = 0;
  for (int r = 1; r < R; ++r)
    if (be[r] < be[best]) best = r;
  std::vector<int8_t> bs(info.n_pos);
  if ((e = cudaMemcpy(bs.data(), d + o_bsp + (size_t)best * info.n_pos, info.n_pos, cudaMemcpyDeviceToHost)) != cudaSuccess)
    return cuda_fail(e, "solve: download best");
  for (int p = 0; p < info.n; ++p) out->best_s[site_of_pos[p]] = (float)bs[p];
  // best_E in FP64 from the configuration itself (E = -1/2 s.J.s - h.s, drift/ising.py:50-53)
  double E = 0.0;
  for (int i = 0; i < info.n; ++i) {
    double f = 0.0;
    for (int t = csr->row_ptr[i]; t < csr->row_ptr[i + 1]; ++t) f += (double)csr->weight[t] * out->best_s[csr->col_idx[t]];
    E += -0.5 * out->best_s[i] * f - (double)csr->h[i] * out->best_s[i];
  }
  out->best_E = E;
  out->seconds = ms * 1e-3;
  out->throughput = out->seconds > 0 ? (double)R * args->n_rounds * args->sweeps_per_round * info.n / out->seconds : 0.0;
  long long tt = 0, ta = 0;
  for (int r = 0; r + 1 < R; ++r) {
    tt += tried[r];
    ta += acc[r];
  }
  out->swap_rate = tt ? (double)ta / (double)tt : 0.0;
  if (out->swap_tried)
    for (int r = 0; r + 1 < R; ++r) out->swap_tried[r] = tried[r];
  if (out->swap_accepted)
    for (int r = 0; r + 1 < R; ++r) out->swap_accepted[r] = acc[r];
  if (out->rung_energy)
    for (int r = 0; r < R; ++r) out->rung_energy[r] = ip ? (double)en[slot_of_rung[r]] : (double)en[slot_of_rung[r]] * kFloatEnergyScale;
  if (out->rung_spins) {
    std::vector<int8_t> sp((size_t)R * info.n_pos);
    if ((e = cudaMemcpy(sp.data(), d + o_sp, sp.size(), cudaMemcpyDeviceToHost)) != cudaSuccess)
      return cuda_fail(e, "solve: download spins");
    for (int r = 0; r < R; ++r)
      for (int p = 0; p < info.n; ++p)
        out->rung_spins[(size_t)r * info.n + site_of_pos[p]] = sp[(size_t)slot_of_rung[r] * info.n_pos + p];
  }
  if (out->best_history && args->n_rounds > 0)
    if ((e = cudaMemcpy(out->best_history, d + o_bh, (size_t)args->n_rounds * 8, cudaMemcpyDeviceToHost)) != cudaSuccess)
      return cuda_fail(e, "solve: download history");
  return DRIFT_PT_OK;
}
