// dpt_batch_mh.cu - whole-configuration proposals on a batch of instances (integer path).
//
// Two steps serve a proposal network per instance (the batched twin of drift_pt_made_mh):
//   * batch_gather_kernel copies the configuration at (instance, rung) from the batch state (slot
//     order, position order) into a caller buffer in the instance's original site order, the order a
//     network models;
//   * batch_mh_kernel takes a proposal x' (site order) for (instance, rung), recomputes its energy
//     exactly from the instance's layout (the same sums as the initial-energy kernel), and accepts it
//     with min(1, exp(-beta (E' - E)) q(x) / q(x')), the log-ratio in double. An accepted proposal
//     replaces the slot's spins and energy, and its best when lower.
// Both are one CTA per request; requests name distinct (instance, rung) pairs within a call.
#include <cuda_runtime.h>

#include "../../include/drift_pt.h"
#include "dpt_common.cuh"
#include "dpt_internal.h"

namespace dpt {
namespace {

constexpr uint32_t kTagBatchMh = 12u;
constexpr int kMhThreads = 256;

struct MhArgs {
  const DriftPtInstanceDesc* desc;
  int n_instances, count, max_n_pos;
  const int32_t* slice_off;
  const int32_t* ell_nbr;
  const int8_t* ell_w;
  const int32_t* h_pos;
  const double* betas;
  const int32_t* inst;
  const int32_t* rung;
  const int64_t* site_off;
  const int32_t* pos_of_site;
  const int64_t* prop_off;
  const int8_t* prop;
  const float* lq_prop;
  const float* lq_cur;
  int8_t* scratch;
  int8_t* spins;
  long long* energy;
  int8_t* best_spins;
  long long* best_energy;
  const int32_t* slot_of_rung;
  long long* prop_energy;
  long long* tried;
  long long* accepted;
  int32_t* err;
  uint32_t k0, k1;
  long long round;
};

// request j -> instance descriptor and local slot, or false (flagged) when out of range
__device__ __forceinline__ bool mh_target(const DriftPtInstanceDesc* desc, int n_instances, const int32_t* inst,
                                          const int32_t* rung, const int32_t* slot_of_rung, int j, int32_t* err,
                                          DriftPtInstanceDesc& D, int& r, int& slot) {
  const int k = inst[j];
  if (k < 0 || k >= n_instances) {
    if (threadIdx.x == 0) atomicExch(err, DRIFT_PT_EINVAL);
    return false;
  }
  D = desc[k];
  r = rung[j];
  if (r < 0 || r >= D.n_replicas) {
    if (threadIdx.x == 0) atomicExch(err, DRIFT_PT_EINVAL);
    return false;
  }
  slot = slot_of_rung[D.slot0 + r];
  return slot >= 0 && slot < D.n_replicas;
}

__global__ void __launch_bounds__(kMhThreads) batch_gather_kernel(
    const DriftPtInstanceDesc* desc, int n_instances, const int32_t* inst, const int32_t* rung,
    const int32_t* slot_of_rung, const int8_t* spins, const int64_t* site_off, const int32_t* pos_of_site,
    const int64_t* out_off, const int64_t* out_step, long long rep, int8_t* out, int32_t* err) {
  const int j = blockIdx.x;
  DriftPtInstanceDesc D;
  int r, slot;
  if (!mh_target(desc, n_instances, inst, rung, slot_of_rung, j, err, D, r, slot)) return;
  const int8_t* sp = spins + D.spin0 + (size_t)slot * D.n_pos;
  const int32_t* pos = pos_of_site + site_off[inst[j]];
  int8_t* o = out + out_off[j] + (out_step ? rep * out_step[j] : 0);
  for (int i = threadIdx.x; i < D.n; i += blockDim.x) o[i] = sp[pos[i]];
}

__global__ void __launch_bounds__(kMhThreads) batch_mh_kernel(const MhArgs a) {
  const int j = blockIdx.x;
  DriftPtInstanceDesc D;
  int r, slot;
  if (!mh_target(a.desc, a.n_instances, a.inst, a.rung, a.slot_of_rung, j, a.err, D, r, slot)) return;
  const int n = D.n;
  const int32_t* pos = a.pos_of_site + a.site_off[a.inst[j]];
  const int8_t* xs = a.prop + a.prop_off[j];
  int8_t* sc = a.scratch + (size_t)j * a.max_n_pos;
  for (int i = threadIdx.x; i < n; i += blockDim.x) sc[pos[i]] = xs[i];
  __syncthreads();
  // 2E' = sum_p s_p (-f_p - 2 h_p) over the instance's sliced ELL (position p = 256 S + 8 lane + q)
  const int32_t* so = a.slice_off + D.slice_off;
  const int32_t* nbr = a.ell_nbr + D.ell;
  const int8_t* wt = a.ell_w + D.ell;
  const int32_t* hp = a.h_pos + D.pos;
  long long v = 0;
  for (int p = threadIdx.x; p < n; p += blockDim.x) {
    const int S = p / kSlicePositions, rem = p - S * kSlicePositions, lane = rem / kGroup, q = rem - lane * kGroup;
    const int w0 = so[S], width = so[S + 1] - w0;
    const long long base = (long long)w0 * kSlicePositions + lane;
    int f = 0;
    for (int d = 0; d < width; ++d) {
      const long long e = base + (long long)(d * kGroup + q) * 32;
      f += (int)wt[e] * (int)sc[nbr[e]];
    }
    v += (long long)sc[p] * (long long)(-f - 2 * hp[(long long)S * kSlicePositions + q * 32 + lane]);
  }
#pragma unroll
  for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
  __shared__ long long red[kMhThreads / 32];
  __shared__ int acc_sm;
  __shared__ long long ep_sm;
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    long long e2 = 0;
    for (int i = 0; i < (int)(blockDim.x >> 5); ++i) e2 += red[i];
    const long long ep = e2 / 2;  // exact: 2E is even for integer couplings
    const size_t gs = (size_t)D.slot0 + slot;
    // log A = -beta (E' - E) + log q(x) - log q(x'), in double; E exact
    const double la = d_add(d_mul(-a.betas[D.slot0 + r], (double)(ep - a.energy[gs])),
                            d_sub((double)a.lq_cur[j], (double)a.lq_prop[j]));
    bool acc = la >= 0.0;
    if (!acc) {
      const U4 u = philox(U4{(uint32_t)r, (uint32_t)a.round, (uint32_t)((unsigned long long)a.round >> 32),
                             ctr3(kTagBatchMh, (uint32_t)D.stream_id)},
                          a.k0, a.k1);
      acc = uniform53(u.x, u.y) < exp_neg_d(la);
    }
    if (a.prop_energy) a.prop_energy[j] = ep;
    a.tried[j] += 1;
    if (acc) a.accepted[j] += 1;
    acc_sm = acc ? 1 : 0;
    ep_sm = ep;
  }
  __syncthreads();
  if (!acc_sm) return;
  const size_t gs = (size_t)D.slot0 + slot;
  const bool better = ep_sm < a.best_energy[gs];
  int8_t* sp = a.spins + D.spin0 + (size_t)slot * D.n_pos;
  int8_t* bp = a.best_spins + D.spin0 + (size_t)slot * D.n_pos;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const int8_t s = xs[i];
    sp[pos[i]] = s;
    if (better) bp[pos[i]] = s;
  }
  if (threadIdx.x == 0) {
    a.energy[gs] = ep_sm;
    if (better) a.best_energy[gs] = ep_sm;
  }
}

int mh_fail(const char* what) {
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? DRIFT_PT_OK : set_error(DRIFT_PT_ECUDA, "%s: %s", what, cudaGetErrorString(e));
}

int mh_check_problem(const DriftPtBatchProblem* p, const DriftPtDeviceState* s) {
  if (!p || !s) return set_error(DRIFT_PT_EINVAL, "batch proposals: null problem or state");
  if (p->n_instances < 1 || !p->desc || !p->slice_off || !p->ell_nbr || !p->ell_w || !p->h_pos || !p->betas ||
      p->max_n_pos < 1)
    return set_error(DRIFT_PT_EINVAL, "batch proposals: problem arrays missing");
  if (!p->integer_path) return set_error(DRIFT_PT_EUNSUPPORTED, "batch proposals: integer couplings only");
  if (!s->spins || !s->energy || !s->best_spins || !s->best_energy || !s->slot_of_rung)
    return set_error(DRIFT_PT_EINVAL, "batch proposals: state arrays missing");
  return DRIFT_PT_OK;
}

}  // namespace
}  // namespace dpt

using namespace dpt;

extern "C" int drift_pt_batch_gather(const DriftPtBatchProblem* prob, const DriftPtDeviceState* state, int32_t count,
                                     const int32_t* instance, const int32_t* rung, const int64_t* site_off,
                                     const int32_t* pos_of_site, const int64_t* out_off, const int64_t* out_step,
                                     int64_t rep, int8_t* out, int32_t* error_flag, void* stream) {
  clear_error();
  int rc = mh_check_problem(prob, state);
  if (rc) return rc;
  if (count < 0 || (count > 0 && (!instance || !rung || !site_off || !pos_of_site || !out_off || !out || !error_flag)))
    return set_error(DRIFT_PT_EINVAL, "batch_gather: bad arguments");
  if (count == 0) return DRIFT_PT_OK;
  batch_gather_kernel<<<count, kMhThreads, 0, static_cast<cudaStream_t>(stream)>>>(
      prob->desc, prob->n_instances, instance, rung, state->slot_of_rung, state->spins, site_off, pos_of_site, out_off,
      out_step, (long long)rep, out, error_flag);
  return mh_fail("batch_gather_kernel");
}

extern "C" int drift_pt_batch_mh(const DriftPtBatchProblem* prob, DriftPtDeviceState* state, uint64_t seed,
                                 int32_t count, const int32_t* instance, const int32_t* rung, const int64_t* site_off,
                                 const int32_t* pos_of_site, const int64_t* prop_off, const int8_t* proposals,
                                 const float* logq_prop, const float* logq_cur, int64_t round, int8_t* scratch,
                                 int64_t* prop_energy, int64_t* prop_tried, int64_t* prop_accepted,
                                 int32_t* error_flag, void* stream) {
  clear_error();
  int rc = mh_check_problem(prob, state);
  if (rc) return rc;
  if (count < 0 || round < 0 ||
      (count > 0 && (!instance || !rung || !site_off || !pos_of_site || !prop_off || !proposals || !logq_prop ||
                     !logq_cur || !scratch || !prop_tried || !prop_accepted || !error_flag)))
    return set_error(DRIFT_PT_EINVAL, "batch_mh: bad arguments");
  if (count == 0) return DRIFT_PT_OK;
  MhArgs a;
  a.desc = prob->desc;
  a.n_instances = prob->n_instances;
  a.count = count;
  a.max_n_pos = prob->max_n_pos;
  a.slice_off = prob->slice_off;
  a.ell_nbr = prob->ell_nbr;
  a.ell_w = static_cast<const int8_t*>(prob->ell_w);
  a.h_pos = static_cast<const int32_t*>(prob->h_pos);
  a.betas = prob->betas;
  a.inst = instance;
  a.rung = rung;
  a.site_off = site_off;
  a.pos_of_site = pos_of_site;
  a.prop_off = prop_off;
  a.prop = proposals;
  a.lq_prop = logq_prop;
  a.lq_cur = logq_cur;
  a.scratch = scratch;
  a.spins = state->spins;
  a.energy = reinterpret_cast<long long*>(state->energy);
  a.best_spins = state->best_spins;
  a.best_energy = reinterpret_cast<long long*>(state->best_energy);
  a.slot_of_rung = state->slot_of_rung;
  a.prop_energy = reinterpret_cast<long long*>(prop_energy);
  a.tried = reinterpret_cast<long long*>(prop_tried);
  a.accepted = reinterpret_cast<long long*>(prop_accepted);
  a.err = error_flag;
  a.k0 = (uint32_t)(seed & 0xffffffffu);
  a.k1 = (uint32_t)(seed >> 32);
  a.round = (long long)round;
  batch_mh_kernel<<<count, kMhThreads, 0, static_cast<cudaStream_t>(stream)>>>(a);
  return mh_fail("batch_mh_kernel");
}
