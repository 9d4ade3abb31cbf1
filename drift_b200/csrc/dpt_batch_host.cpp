// dpt_batch_host.cpp - host layout of a whole batch of instances in two calls.
//
// The batched layer reads one concatenation of every instance's layout (colour ranges, slice
// offsets, ELL neighbours and weights, fields, position maps) plus a descriptor per instance with
// the offsets into it. Building that from Python one instance at a time costs more than the device
// run for batches of hundreds of instances; here the query sizes everything at once and the fill
// writes each instance's layout straight into the concatenated arrays, instances split over the
// host's threads.
#include <algorithm>
#include <string>
#include <thread>
#include <vector>

#include "../../include/drift_pt.h"
#include "dpt_internal.h"

namespace {

// runs f(k) for k in [0, count) on up to hardware_concurrency threads; returns the first failing
// status and its message (errors are thread-local, so they are carried back to the caller's thread)
template <class F>
int for_instances(int32_t count, F f, std::string* msg) {
  const int T = std::max(1, std::min<int>((int)std::thread::hardware_concurrency(), (count + 15) / 16));
  std::vector<int> rc((size_t)T, DRIFT_PT_OK);
  std::vector<std::string> why((size_t)T);
  auto work = [&](int t) {
    for (int32_t k = t; k < count; k += T) {
      const int r = f(k);
      if (r != DRIFT_PT_OK) {
        rc[(size_t)t] = r;
        why[(size_t)t] = std::string("instance ") + std::to_string(k) + ": " + drift_pt_last_error();
        return;
      }
    }
  };
  if (T == 1) {
    work(0);
  } else {
    std::vector<std::thread> pool;
    for (int t = 0; t < T; ++t) pool.emplace_back(work, t);
    for (auto& th : pool) th.join();
  }
  for (int t = 0; t < T; ++t)
    if (rc[(size_t)t] != DRIFT_PT_OK) {
      *msg = why[(size_t)t];
      return rc[(size_t)t];
    }
  return DRIFT_PT_OK;
}

}  // namespace

using namespace dpt;

extern "C" int drift_pt_batch_layout_query(int32_t n_instances, const DriftPtCsr* csrs, DriftPtLayoutInfo* infos,
                                           DriftPtBatchSizes* sizes) {
  clear_error();
  if (n_instances < 1 || !csrs || !infos || !sizes) return set_error(DRIFT_PT_EINVAL, "batch_layout_query: bad arguments");
  std::string msg;
  const int rc = for_instances(n_instances, [&](int32_t k) { return drift_pt_layout_query(csrs + k, infos + k); }, &msg);
  if (rc) return set_error(rc, "batch_layout_query: %s", msg.c_str());
  DriftPtBatchSizes s = {};
  s.all_integer = 1;
  for (int32_t k = 0; k < n_instances; ++k) {
    const DriftPtLayoutInfo& I = infos[k];
    s.color_ptr += I.n_colors + 1;
    s.slice_off += I.n_slices + 1;
    s.ell += I.n_ell;
    s.pos += I.n_pos;
    s.sites += I.n;
    s.all_integer &= I.integer_couplings ? 1 : 0;
  }
  *sizes = s;
  return DRIFT_PT_OK;
}

extern "C" int drift_pt_batch_layout_fill(int32_t n_instances, const DriftPtCsr* csrs, const DriftPtLayoutInfo* infos,
                                          int32_t integer_path, const int32_t* n_replicas, const int32_t* stream_ids,
                                          const double* betas, DriftPtInstanceDesc* desc, uint32_t* thresholds,
                                          DriftPtBatchLayout* out) {
  clear_error();
  if (n_instances < 1 || !csrs || !infos || !n_replicas || !stream_ids || !desc || !out || !out->color_ptr ||
      !out->slice_off || !out->ell_nbr || !out->ell_w || !out->h_pos || !out->site_of_pos || !out->pos_of_site ||
      (integer_path && (!betas || !thresholds)))
    return set_error(DRIFT_PT_EINVAL, "batch_layout_fill: bad arguments");
  // offsets of every instance (the descriptor) from the sizes, in instance order
  int64_t cp = 0, so = 0, ell = 0, pos = 0, site = 0, slot = 0, spin = 0, thr = 0;
  std::vector<int64_t> site0((size_t)n_instances);
  for (int32_t k = 0; k < n_instances; ++k) {
    const DriftPtLayoutInfo& I = infos[k];
    const int32_t R = n_replicas[k];
    if (R < 1) return set_error(DRIFT_PT_EINVAL, "batch_layout_fill: instance %d has no replicas", k);
    if (stream_ids[k] < 0 || stream_ids[k] >= (1 << 24))
      return set_error(DRIFT_PT_EINVAL, "batch_layout_fill: stream id of instance %d outside [0, 2^24)", k);
    if (integer_path && !I.integer_couplings)
      return set_error(DRIFT_PT_EINVAL, "batch_layout_fill: instance %d has non-integer couplings", k);
    DriftPtInstanceDesc& d = desc[k];
    d.n = I.n;
    d.n_pos = I.n_pos;
    d.n_slices = I.n_slices;
    d.n_colors = I.n_colors;
    d.n_replicas = R;
    d.max_field = integer_path ? I.max_field : 0;
    d.stream_id = stream_ids[k];
    d.reserved = 0;
    d.color_ptr = cp;
    d.slice_off = so;
    d.ell = ell;
    d.pos = pos;
    d.slot0 = slot;
    d.spin0 = spin;
    d.thr = thr;
    site0[(size_t)k] = site;
    cp += I.n_colors + 1;
    so += I.n_slices + 1;
    ell += I.n_ell;
    pos += I.n_pos;
    site += I.n;
    slot += R;
    spin += (int64_t)R * I.n_pos;
    if (integer_path) thr += (int64_t)R * I.max_field;
  }
  int8_t* w8 = static_cast<int8_t*>(out->ell_w);
  float* wf = static_cast<float*>(out->ell_w);
  int32_t* h32 = static_cast<int32_t*>(out->h_pos);
  float* hf = static_cast<float*>(out->h_pos);
  std::string msg;
  const int rc = for_instances(
      n_instances,
      [&](int32_t k) {
        const DriftPtInstanceDesc& d = desc[k];
        DriftPtLayout lay;
        lay.color_ptr = out->color_ptr + d.color_ptr;
        lay.slice_off = out->slice_off + d.slice_off;
        lay.ell_nbr = out->ell_nbr + d.ell;
        lay.ell_w = integer_path ? static_cast<void*>(w8 + d.ell) : static_cast<void*>(wf + d.ell);
        lay.h_pos = integer_path ? static_cast<void*>(h32 + d.pos) : static_cast<void*>(hf + d.pos);
        lay.site_of_pos = out->site_of_pos + d.pos;
        lay.pos_of_site = out->pos_of_site + site0[(size_t)k];
        int r = drift_pt_layout_fill(csrs + k, integer_path, &lay);
        if (r == DRIFT_PT_OK && integer_path)
          r = drift_pt_thresholds(d.n_replicas, betas + d.slot0, d.max_field, thresholds + d.thr);
        return r;
      },
      &msg);
  if (rc) return set_error(rc, "batch_layout_fill: %s", msg.c_str());
  return DRIFT_PT_OK;
}
