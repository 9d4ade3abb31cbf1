// dpt_unit_host.cpp - the storage order of the unit-regular form's spin bytes in shared memory.
//
// In the unit-regular form a warp's neighbour gather is one byte load per lane from 32 scattered
// positions. Shared memory serves a load in as many passes (wavefronts) as the largest number of
// distinct 4-byte words any of its 32 banks is asked for, so on a random graph each gather costs
// about 3.3 passes. The chain does not depend on where a position's byte is stored, only on
// positions, so the bytes can be laid out to spread each gather over the banks. Here the unit of
// storage is the 4-byte word of positions 4u .. 4u + 3; word u is stored at word_slot[u], whose bank
// is word_slot[u] % 32. The gathers are known in advance: the kernel's schedule gives every item a
// fixed warp and every load a fixed index. A greedy pass places the words with the most gathers
// first, each in the bank with free room where it adds least to the loads of the gathers it takes
// part in. On MaxCut N = 4096 this lowers the passes of a sweep's gathers by about a quarter.
#include <algorithm>
#include <cstdint>
#include <numeric>
#include <vector>

#include "../../include/drift_pt.h"
#include "dpt_internal.h"

using namespace dpt;

extern "C" int drift_pt_unit_placement(const DriftPtCsr* csr, int32_t positions_per_item, uint16_t* word_slot) {
  clear_error();
  DriftPtLayoutInfo info;
  int rc = drift_pt_layout_query(csr, &info);
  if (rc) return rc;
  if (!word_slot) return set_error(DRIFT_PT_EINVAL, "unit_placement: word_slot is NULL");
  if (!info.unit_regular) return set_error(DRIFT_PT_EUNSUPPORTED, "unit_placement: the problem is not unit-regular");
  const int n = csr->n, n_pos = info.n_pos, W = info.max_degree, k = csr->n_colors;
  int max_class = 0;
  for (int c = 0; c < k; ++c) max_class = std::max(max_class, csr->color_ptr[c + 1] - csr->color_ptr[c]);
  int P = positions_per_item;
  if (P == 0) P = unit_auto_positions(max_class);
  if (P != 2 && P != 4) return set_error(DRIFT_PT_EINVAL, "unit_placement: positions_per_item must be 0, 2 or 4");
  const int units = n_pos / 4;
  if (units > 65536) return set_error(DRIFT_PT_EUNSUPPORTED, "unit_placement: too many positions");
  std::vector<int> pos_of_site(n);
  for (int p = 0; p < n; ++p) pos_of_site[csr->color_spins[p]] = p;
  // the gathers (and each warp's own-word accesses) as sets of words: (phase, warp, load index)
  const int NB = kGroup / P, K = P * W + 1, kWarps = kMaxUnitThreads / 32;
  std::vector<std::vector<int>> sets((size_t)std::max(k, 1) * kWarps * K);
  for (int c = 0; c < k; ++c) {
    const int lo = csr->color_ptr[c], hi = csr->color_ptr[c + 1];
    const int glo = lo >> 3, ghi = (hi + 7) >> 3;
    for (int lt = 0; lt < (ghi - glo) * NB; ++lt) {
      const int item = glo * NB + lt, w = lt >> 5;
      if (w >= kWarps) break;
      sets[((size_t)c * kWarps + w) * K + P * W].push_back(item * P / 4);
      for (int i = 0; i < P; ++i) {
        const int p = item * P + i;
        if (p >= n) continue;
        const int s = csr->color_spins[p];
        for (int d = 0; d < W && csr->row_ptr[s] + d < csr->row_ptr[s + 1]; ++d)
          sets[((size_t)c * kWarps + w) * K + i * W + d].push_back(pos_of_site[csr->col_idx[csr->row_ptr[s] + d]] / 4);
      }
    }
  }
  std::vector<std::vector<int>> memb(units);
  for (size_t si = 0; si < sets.size(); ++si) {
    auto& v = sets[si];
    std::sort(v.begin(), v.end());
    v.erase(std::unique(v.begin(), v.end()), v.end());
    for (int u : v) memb[u].push_back((int)si);
  }
  std::vector<int> order(units);
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return memb[a].size() > memb[b].size(); });
  std::vector<int> load(sets.size() * 32, 0), cap(32, units / 32), filled(32, 0);
  for (int u : order) {
    long long best_score = -1;
    int best = -1;
    for (int b = 0; b < 32; ++b) {
      if (cap[b] == 0) continue;
      long long sc = 0;
      for (int si : memb[u]) sc += load[(size_t)si * 32 + b];
      if (best < 0 || sc < best_score) {
        best = b;
        best_score = sc;
      }
    }
    --cap[best];
    for (int si : memb[u]) ++load[(size_t)si * 32 + best];
    word_slot[u] = (uint16_t)(filled[best]++ * 32 + best);
  }
  return DRIFT_PT_OK;
}
