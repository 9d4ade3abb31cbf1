// dpt_gms_host.cpp - host side of the graph multispin layer: the position order, neighbour table
// and coupling signs of a +-1 graph.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <vector>

#include "../../include/drift_pt.h"
#include "dpt_internal.h"

using namespace dpt;

namespace {

int gms_check(const DriftPtCsr* c, int32_t* max_degree) {
  int rc = validate_csr(c);
  if (rc) return rc;
  int32_t dmax = 0;
  for (int32_t i = 0; i < c->n; ++i) {
    if (c->h[i] != 0.0f) return set_error(DRIFT_PT_EUNSUPPORTED, "graph multispin: h[%d] != 0 (no field)", i);
    int32_t deg = 0;
    for (int32_t t = c->row_ptr[i]; t < c->row_ptr[i + 1]; ++t) {
      if (c->col_idx[t] == i) continue;
      if (c->weight[t] != 1.0f && c->weight[t] != -1.0f)
        return set_error(DRIFT_PT_EUNSUPPORTED, "graph multispin: couplings must be +-1 (J[%d][%d] = %g)", i,
                         c->col_idx[t], (double)c->weight[t]);
      ++deg;
    }
    if (deg > DRIFT_PT_GMS_MAX_DEGREE)
      return set_error(DRIFT_PT_EUNSUPPORTED, "graph multispin: degree %d of spin %d exceeds %d", deg, i,
                       DRIFT_PT_GMS_MAX_DEGREE);
    if (deg > dmax) dmax = deg;
  }
  *max_degree = dmax < 1 ? 1 : dmax;
  return DRIFT_PT_OK;
}

}  // namespace

extern "C" int drift_pt_gms_layout_query(const DriftPtCsr* csr, DriftPtGmsLayoutInfo* info) {
  clear_error();
  if (!info) return set_error(DRIFT_PT_EINVAL, "gms_layout_query: info is NULL");
  int32_t dmax = 0;
  int rc = gms_check(csr, &dmax);
  if (rc) return rc;
  info->n = csr->n;
  info->n_pos = (csr->n + 31) & ~31;
  info->n_colors = csr->n_colors;
  info->max_degree = dmax;
  int64_t nnz = 0;
  for (int32_t i = 0; i < csr->n; ++i)
    for (int32_t t = csr->row_ptr[i]; t < csr->row_ptr[i + 1]; ++t) nnz += csr->col_idx[t] != i;
  info->n_bonds = nnz / 2;
  info->max_class = 0;
  info->reserved = 0;
  for (int32_t c = 0; c < csr->n_colors; ++c)
    info->max_class = std::max(info->max_class, csr->color_ptr[c + 1] - csr->color_ptr[c]);
  return DRIFT_PT_OK;
}

// Position p holds spin color_spins[p]; ell_nbr[d][p] is the position of its d-th neighbour in
// CSR order; padding positions (p >= n) have degree 0.
extern "C" int drift_pt_gms_layout_fill(const DriftPtCsr* csr, DriftPtGmsLayout* out) {
  clear_error();
  DriftPtGmsLayoutInfo info;
  int rc = drift_pt_gms_layout_query(csr, &info);
  if (rc) return rc;
  if (!out || !out->color_ptr || !out->ell_nbr || !out->degree || !out->jneg || !out->pos_of_site ||
      !out->site_of_pos)
    return set_error(DRIFT_PT_EINVAL, "gms_layout_fill: output arrays missing");
  const int32_t n = info.n, n_pos = info.n_pos, D = info.max_degree;
  for (int32_t c = 0; c <= csr->n_colors; ++c) out->color_ptr[c] = csr->color_ptr[c];
  for (int32_t p = 0; p < n_pos; ++p) out->site_of_pos[p] = p < n ? csr->color_spins[p] : -1;
  for (int32_t p = 0; p < n; ++p) out->pos_of_site[csr->color_spins[p]] = p;
  std::memset(out->ell_nbr, 0, sizeof(int32_t) * (size_t)D * n_pos);
  std::memset(out->degree, 0, (size_t)n_pos);
  std::memset(out->jneg, 0, (size_t)n_pos);
  for (int32_t p = 0; p < n; ++p) {
    const int32_t i = out->site_of_pos[p];
    int d = 0;
    for (int32_t t = csr->row_ptr[i]; t < csr->row_ptr[i + 1]; ++t) {
      const int32_t j = csr->col_idx[t];
      if (j == i) continue;
      out->ell_nbr[(size_t)d * n_pos + p] = out->pos_of_site[j];
      if (csr->weight[t] < 0.0f) out->jneg[p] |= (uint8_t)(1u << d);
      ++d;
    }
    out->degree[p] = (uint8_t)d;
  }
  return DRIFT_PT_OK;
}
