// dpt_host.cpp - host half of the C ABI: colouring, device layout, Metropolis thresholds, errors.
//
// The reference does this preprocessing in Python on every call (drift/gpu.py:66-81 and the
// pure-Python greedy colouring of drift/gpu.py:122-145). Here it is O(nnz) C++ behind the ABI.
#include <algorithm>
#include <cstdarg>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/drift_pt.h"
#include "dpt_common.cuh"
#include "dpt_internal.h"

namespace dpt {

static thread_local std::string g_last_error;

int set_error(int code, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  g_last_error = buf;
  return code;
}

void clear_error() { g_last_error.clear(); }

}  // namespace dpt

using namespace dpt;

extern "C" const char* drift_pt_last_error(void) { return g_last_error.c_str(); }

extern "C" const char* drift_pt_version(void) { return "drift-b200-pt 0.1.0 sm_100a"; }

// Greedy colouring in index order (drift/gpu.py:130-141): spin i takes the smallest colour not
// used by a neighbour that already has one (neighbours j < i in index order, but any coloured
// neighbour counts, exactly as the reference's `color[col_idx[t]] >= 0` test).
extern "C" int drift_pt_greedy_coloring(int32_t n, const int32_t* row_ptr, const int32_t* col_idx,
                                        int32_t* color, int32_t* n_colors) {
  clear_error();
  if (n < 0 || (n > 0 && (!row_ptr || !color)) || !n_colors)
    return set_error(DRIFT_PT_EINVAL, "greedy_coloring: invalid arguments");
  int32_t maxdeg = 0;
  for (int32_t i = 0; i < n; ++i) {
    int32_t d = row_ptr[i + 1] - row_ptr[i];
    if (d < 0) return set_error(DRIFT_PT_EINVAL, "greedy_coloring: row_ptr not monotone at %d", i);
    maxdeg = std::max(maxdeg, d);
  }
  for (int32_t i = 0; i < n; ++i) color[i] = -1;
  // stamp[c] == i+1 marks colour c as used by a neighbour of spin i
  std::vector<int32_t> stamp((size_t)maxdeg + 2, 0);
  int32_t k = 0;
  for (int32_t i = 0; i < n; ++i) {
    for (int32_t t = row_ptr[i]; t < row_ptr[i + 1]; ++t) {
      int32_t j = col_idx[t];
      if (j < 0 || j >= n) return set_error(DRIFT_PT_EINVAL, "greedy_coloring: col_idx out of range");
      int32_t c = color[j];
      if (c >= 0 && c <= maxdeg) stamp[c] = i + 1;
    }
    int32_t c = 0;
    while (stamp[c] == i + 1) ++c;
    color[i] = c;
    k = std::max(k, c + 1);
  }
  *n_colors = (n > 0) ? k : 1;  // the reference reports k = 1 for an empty model
  return DRIFT_PT_OK;
}

// Stable counting sort of spins by colour (drift/gpu.py:142-144).
extern "C" int drift_pt_color_order(int32_t n, const int32_t* color, int32_t n_colors,
                                    int32_t* color_ptr, int32_t* color_spins) {
  clear_error();
  if (n < 0 || n_colors < 1 || !color_ptr || (n > 0 && (!color || !color_spins)))
    return set_error(DRIFT_PT_EINVAL, "color_order: invalid arguments");
  std::vector<int32_t> cnt((size_t)n_colors + 1, 0);
  for (int32_t i = 0; i < n; ++i) {
    if (color[i] < 0 || color[i] >= n_colors) return set_error(DRIFT_PT_EINVAL, "color_order: colour out of range");
    cnt[color[i] + 1]++;
  }
  for (int32_t c = 0; c < n_colors; ++c) cnt[c + 1] += cnt[c];
  for (int32_t c = 0; c <= n_colors; ++c) color_ptr[c] = cnt[c];
  for (int32_t i = 0; i < n; ++i) color_spins[cnt[color[i]]++] = i;
  return DRIFT_PT_OK;
}

namespace {

bool is_int_in(float v, float lim) { return std::nearbyint(v) == v && std::fabs(v) <= lim; }

}  // namespace

namespace dpt {

int validate_csr(const DriftPtCsr* c) {
  if (!c) return set_error(DRIFT_PT_EINVAL, "csr is NULL");
  if (c->n < 1) return set_error(DRIFT_PT_EINVAL, "n must be >= 1 (got %d)", c->n);
  if (c->n > (1 << 30)) return set_error(DRIFT_PT_EUNSUPPORTED, "n too large");
  if (!c->row_ptr || !c->h || !c->color_ptr || !c->color_spins)
    return set_error(DRIFT_PT_EINVAL, "csr arrays missing");
  if (c->nnz < 0 || (c->nnz > 0 && (!c->col_idx || !c->weight)))
    return set_error(DRIFT_PT_EINVAL, "csr entries missing");
  if (c->row_ptr[0] != 0 || c->row_ptr[c->n] != c->nnz)
    return set_error(DRIFT_PT_EINVAL, "row_ptr[0] must be 0 and row_ptr[n] == nnz");
  for (int32_t i = 0; i < c->n; ++i)
    if (c->row_ptr[i + 1] < c->row_ptr[i]) return set_error(DRIFT_PT_EINVAL, "row_ptr not monotone");
  for (int64_t t = 0; t < c->nnz; ++t)
    if (c->col_idx[t] < 0 || c->col_idx[t] >= c->n) return set_error(DRIFT_PT_EINVAL, "col_idx out of range");
  int32_t k = c->n_colors;
  if (k < 1 || c->color_ptr[0] != 0 || c->color_ptr[k] != c->n)
    return set_error(DRIFT_PT_EINVAL, "color_ptr must run from 0 to n");
  std::vector<int32_t> col((size_t)c->n, -1);
  for (int32_t cc = 0; cc < k; ++cc) {
    if (c->color_ptr[cc + 1] < c->color_ptr[cc]) return set_error(DRIFT_PT_EINVAL, "color_ptr not monotone");
    for (int32_t p = c->color_ptr[cc]; p < c->color_ptr[cc + 1]; ++p) {
      int32_t i = c->color_spins[p];
      if (i < 0 || i >= c->n || col[i] != -1) return set_error(DRIFT_PT_EINVAL, "color_spins is not a permutation");
      col[i] = cc;
    }
  }
  // The independence invariant that makes flipping a colour class in parallel exact
  // (cuda/ising_pt.cu:12-13): no coupling inside a colour class.
  for (int32_t i = 0; i < c->n; ++i)
    for (int32_t t = c->row_ptr[i]; t < c->row_ptr[i + 1]; ++t) {
      int32_t j = c->col_idx[t];
      if (j == i && c->weight[t] != 0.0f) return set_error(DRIFT_PT_EINVAL, "non-zero diagonal coupling at %d", i);
      if (j != i && col[j] == col[i] && c->weight[t] != 0.0f)
        return set_error(DRIFT_PT_EINVAL, "invalid colouring: spins %d and %d are coupled and share colour %d", i, j, col[i]);
    }
  return DRIFT_PT_OK;
}

}  // namespace dpt

extern "C" int drift_pt_layout_query(const DriftPtCsr* csr, DriftPtLayoutInfo* info) {
  clear_error();
  int rc = validate_csr(csr);
  if (rc) return rc;
  if (!info) return set_error(DRIFT_PT_EINVAL, "info is NULL");
  const int32_t n = csr->n;
  info->n = n;
  info->n_pos = ((n + kSlicePositions - 1) / kSlicePositions) * kSlicePositions;
  info->n_slices = info->n_pos / kSlicePositions;
  info->n_colors = csr->n_colors;
  int64_t widths = 0;
  int32_t maxdeg = 0, minw = 1 << 30;
  for (int32_t s = 0; s < info->n_slices; ++s) {
    int32_t w = 0;
    for (int32_t p = s * kSlicePositions; p < std::min(n, (s + 1) * kSlicePositions); ++p) {
      int32_t i = csr->color_spins[p];
      w = std::max(w, csr->row_ptr[i + 1] - csr->row_ptr[i]);
    }
    widths += w;
    maxdeg = std::max(maxdeg, w);
    minw = std::min(minw, w);
  }
  info->n_ell = widths * kSlicePositions;
  info->max_degree = maxdeg;
  info->min_width = minw;
  bool integer = true;
  int64_t F = 0;
  for (int32_t i = 0; i < n && integer; ++i) {
    if (!is_int_in(csr->h[i], 1048576.0f)) { integer = false; break; }
    int64_t f = (int64_t)std::fabs(csr->h[i]);
    for (int32_t t = csr->row_ptr[i]; t < csr->row_ptr[i + 1]; ++t) {
      if (!is_int_in(csr->weight[t], 127.0f)) { integer = false; break; }
      f += (int64_t)std::fabs(csr->weight[t]);
    }
    F = std::max(F, f);
  }
  if (integer && F > (1 << 24)) integer = false;
  info->has_field = 0;
  for (int32_t i = 0; i < n; ++i)
    if (csr->h[i] != 0.0f) {
      info->has_field = 1;
      break;
    }
  info->integer_couplings = integer ? 1 : 0;
  info->max_field = integer ? (int32_t)std::max<int64_t>(F, 1) : 0;
  // unit-regular: every spin has exactly max_degree couplings, each +1 or -1, and no field
  bool unit = integer && !info->has_field && maxdeg >= 1;
  for (int32_t i = 0; i < n && unit; ++i) {
    if (csr->row_ptr[i + 1] - csr->row_ptr[i] != maxdeg) unit = false;
    for (int32_t t = csr->row_ptr[i]; t < csr->row_ptr[i + 1] && unit; ++t)
      if (std::fabs(csr->weight[t]) != 1.0f) unit = false;
  }
  info->unit_regular = unit ? 1 : 0;
  return DRIFT_PT_OK;
}

extern "C" int drift_pt_layout_fill(const DriftPtCsr* csr, int32_t integer_path, DriftPtLayout* out) {
  DriftPtLayoutInfo info;
  int rc = drift_pt_layout_query(csr, &info);
  if (rc) return rc;
  if (!out || !out->color_ptr || !out->slice_off || !out->h_pos || !out->site_of_pos || !out->pos_of_site ||
      (info.n_ell > 0 && (!out->ell_nbr || !out->ell_w)))
    return set_error(DRIFT_PT_EINVAL, "layout_fill: output arrays missing");
  if (integer_path && !info.integer_couplings)
    return set_error(DRIFT_PT_EINVAL, "layout_fill: integer path requested for non-integer couplings");
  const int32_t n = csr->n, n_pos = info.n_pos;
  for (int32_t c = 0; c <= csr->n_colors; ++c) out->color_ptr[c] = csr->color_ptr[c];
  for (int32_t p = 0; p < n_pos; ++p) out->site_of_pos[p] = (p < n) ? csr->color_spins[p] : -1;
  for (int32_t p = 0; p < n; ++p) out->pos_of_site[csr->color_spins[p]] = p;
  int8_t* w8 = static_cast<int8_t*>(out->ell_w);
  float* wf = static_cast<float*>(out->ell_w);
  int32_t* h32 = static_cast<int32_t*>(out->h_pos);
  float* hf = static_cast<float*>(out->h_pos);
  int64_t off = 0;
  out->slice_off[0] = 0;
  for (int32_t s = 0; s < info.n_slices; ++s) {
    int32_t w = 0;
    for (int32_t p = s * kSlicePositions; p < std::min(n, (s + 1) * kSlicePositions); ++p) {
      int32_t i = csr->color_spins[p];
      w = std::max(w, csr->row_ptr[i + 1] - csr->row_ptr[i]);
    }
    for (int32_t lane = 0; lane < 32; ++lane)
      for (int32_t q = 0; q < 8; ++q) {
        int32_t p = s * kSlicePositions + lane * 8 + q;
        int32_t i = (p < n) ? csr->color_spins[p] : -1;
        int64_t hidx = (int64_t)s * kSlicePositions + q * 32 + lane;
        if (integer_path) h32[hidx] = (i >= 0) ? (int32_t)csr->h[i] : 0;
        else hf[hidx] = (i >= 0) ? csr->h[i] : 0.0f;
        int32_t deg = (i >= 0) ? csr->row_ptr[i + 1] - csr->row_ptr[i] : 0;
        for (int32_t d = 0; d < w; ++d) {
          int64_t e = off * kSlicePositions + (int64_t)(d * 8 + q) * 32 + lane;
          int32_t nb = p;  // padding: self with weight 0
          float wt = 0.0f;
          if (d < deg) {
            int64_t t = csr->row_ptr[i] + d;
            nb = out->pos_of_site[csr->col_idx[t]];
            wt = csr->weight[t];
          }
          out->ell_nbr[e] = nb;
          if (integer_path) w8[e] = (int8_t)wt;
          else wf[e] = wt;
        }
      }
    off += w;
    out->slice_off[s + 1] = (int32_t)off;
  }
  return DRIFT_PT_OK;
}

extern "C" int drift_pt_thresholds(int32_t n_rungs, const double* betas, int32_t max_field, uint32_t* thr) {
  clear_error();
  if (n_rungs < 1 || max_field < 1 || !betas || !thr) return set_error(DRIFT_PT_EINVAL, "thresholds: invalid arguments");
  for (int32_t r = 0; r < n_rungs; ++r) {
    if (!(betas[r] >= 0.0) || !std::isfinite(betas[r])) return set_error(DRIFT_PT_EINVAL, "beta[%d] must be finite and >= 0", r);
    for (int32_t x = 1; x <= max_field; ++x) thr[(int64_t)r * max_field + x - 1] = threshold_int(betas[r], x);
  }
  return DRIFT_PT_OK;
}
