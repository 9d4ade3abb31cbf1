// dpt_sk_host.cpp - host side of the dense-coupling (SK) layer: fixed-point quantisation of the
// couplings, the device coupling table, and the per-rung acceptance scales.
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>

#include "../../include/drift_pt.h"
#include "dpt_internal.h"
#include "dpt_sk.h"

using namespace dpt;

// The model enters as IsingModel's dense J (drift/ising.py:31-42: symmetric, zero diagonal) and
// h. The chain runs on Jq = rint(J 2^shift), hq = rint(h 2^shift): shift is the largest power of
// two for which every coupling fits three int8 limbs and every local field stays below 2^30
// (so s_i F_i, the thresholds and all partial sums are exact int32).
extern "C" int drift_pt_sk_quantize(int32_t n, const double* J, const double* h, int32_t* Jq, int32_t* hq,
                                    int32_t* shift) {
  clear_error();
  if (n < 1 || n > sk::kMaxN) return set_error(DRIFT_PT_EINVAL, "sk: n must be in 1..%d", sk::kMaxN);
  if (!J || !Jq || !hq || !shift) return set_error(DRIFT_PT_EINVAL, "sk_quantize: null pointer");
  double maxabs = 0.0, maxrow = 0.0;
  for (int i = 0; i < n; ++i) {
    const double hi = h ? h[i] : 0.0;
    if (!std::isfinite(hi)) return set_error(DRIFT_PT_EINVAL, "sk_quantize: h[%d] is not finite", i);
    double row = std::fabs(hi);
    for (int j = 0; j < n; ++j) {
      const double v = J[(size_t)i * n + j];
      if (!std::isfinite(v)) return set_error(DRIFT_PT_EINVAL, "sk_quantize: J[%d][%d] is not finite", i, j);
      if (i == j && v != 0.0) return set_error(DRIFT_PT_EINVAL, "sk_quantize: nonzero diagonal J[%d][%d]", i, i);
      if (v != J[(size_t)j * n + i])
        return set_error(DRIFT_PT_EINVAL, "sk_quantize: J is not symmetric at (%d, %d)", i, j);
      row += std::fabs(v);
      if (std::fabs(v) > maxabs) maxabs = std::fabs(v);
    }
    if (row > maxrow) maxrow = row;
  }
  int s = 0;
  if (maxrow > 0.0) {
    auto fits = [&](int sh) {
      return std::ldexp(maxabs, sh) <= (double)sk::kMaxCoupling &&
             std::ldexp(maxrow, sh) + (double)n <= (double)sk::kMaxField;
    };
    s = 60;
    while (s > -60 && !fits(s)) --s;
    if (!fits(s)) return set_error(DRIFT_PT_EINVAL, "sk_quantize: couplings out of range");
  }
  for (int i = 0; i < n; ++i) {
    int64_t row = 0;
    for (int j = 0; j < n; ++j) {
      const double v = std::rint(std::ldexp(J[(size_t)i * n + j], s));
      Jq[(size_t)i * n + j] = (int32_t)v;
      row += (int64_t)std::llabs((long long)v);
    }
    const double hv = h ? std::rint(std::ldexp(h[i], s)) : 0.0;
    hq[i] = (int32_t)hv;
    row += (int64_t)std::llabs((long long)hv);
    if (row >= (int64_t)sk::kMaxField) return set_error(DRIFT_PT_EINVAL, "sk_quantize: field bound violated");
  }
  *shift = s;
  return DRIFT_PT_OK;
}

extern "C" int drift_pt_sk_layout_bytes(int32_t n, size_t* bytes) {
  clear_error();
  if (n < 1 || n > sk::kMaxN || !bytes) return set_error(DRIFT_PT_EINVAL, "sk_layout_bytes: bad arguments");
  *bytes = (size_t)sk::n_blocks(n) * sk::entry_bytes(n);
  return DRIFT_PT_OK;
}

// Entry of block B (spins 32B .. 32B+31): for tile t = 0..n_tiles-1 and limb k = 0..2 a 128 x 32
// int8 operand holding limb k of Jq[128t + row][32B + col] (zero outside n) at
// core_offset(row, col); then Jq[32B + f][32B + l] as int32 at [f][l]; then
// Jq[32 prev(B) + f][32B + l] as int32 at [f][l], prev(B) = (B - 1) mod n_blocks.
extern "C" int drift_pt_sk_layout_fill(int32_t n, const int32_t* Jq, void* layout) {
  clear_error();
  if (n < 1 || n > sk::kMaxN || !Jq || !layout) return set_error(DRIFT_PT_EINVAL, "sk_layout_fill: bad arguments");
  for (size_t i = 0; i < (size_t)n * n; ++i)
    if (Jq[i] > sk::kMaxCoupling || Jq[i] < -sk::kMaxCoupling)
      return set_error(DRIFT_PT_EINVAL, "sk_layout_fill: coupling %zu out of the 24-bit range", i);
  for (int i = 0; i < n; ++i)
    if (Jq[(size_t)i * n + i] != 0) return set_error(DRIFT_PT_EINVAL, "sk_layout_fill: nonzero diagonal");
  const int nt = sk::n_tiles(n), nb = sk::n_blocks(n);
  const size_t eb = sk::entry_bytes(n);
  unsigned char* out = static_cast<unsigned char*>(layout);
  std::memset(out, 0, (size_t)nb * eb);
  for (int B = 0; B < nb; ++B) {
    unsigned char* e = out + (size_t)B * eb;
    for (int m = 0; m < nt * sk::kTile; ++m) {
      const int t = m / sk::kTile, row = m % sk::kTile;
      for (int k = 0; k < sk::kBlock; ++k) {
        const int col = sk::kBlock * B + k;
        const int32_t v = (m < n && col < n) ? Jq[(size_t)m * n + col] : 0;
        int8_t d[3];
        sk::limbs(v, d);
        for (int l = 0; l < sk::kLimbs; ++l)
          e[(size_t)(t * sk::kLimbs + l) * sk::kTileBytes + sk::core_offset(row, k)] = (unsigned char)d[l];
      }
    }
    int32_t* dg = reinterpret_cast<int32_t*>(e + (size_t)nt * sk::kLimbs * sk::kTileBytes);
    int32_t* pv = dg + sk::kBlock * sk::kBlock;
    const int Bp = (B + nb - 1) % nb;
    for (int f = 0; f < sk::kBlock; ++f)
      for (int l = 0; l < sk::kBlock; ++l) {
        const int r = sk::kBlock * B + f, c = sk::kBlock * B + l, rp = sk::kBlock * Bp + f;
        dg[f * sk::kBlock + l] = (r < n && c < n) ? Jq[(size_t)r * n + c] : 0;
        pv[f * sk::kBlock + l] = (rp < n && c < n) ? Jq[(size_t)rp * n + c] : 0;
      }
  }
  return DRIFT_PT_OK;
}

extern "C" int drift_pt_sk_scales(int32_t n_replicas, const double* betas, int32_t shift, float* scales) {
  clear_error();
  if (n_replicas < 1 || !betas || !scales || shift < -60 || shift > 60)
    return set_error(DRIFT_PT_EINVAL, "sk_scales: bad arguments");
  for (int r = 0; r < n_replicas; ++r) {
    if (!(betas[r] > 0.0) || !std::isfinite(betas[r]))
      return set_error(DRIFT_PT_EINVAL, "sk_scales: beta[%d] must be > 0", r);
    scales[r] = (float)(std::ldexp(1.0, shift) / (2.0 * betas[r]));
  }
  return DRIFT_PT_OK;
}
