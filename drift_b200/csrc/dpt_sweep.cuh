// dpt_sweep.cuh - the colour-phase item update shared by the single-ladder and batched kernels.
//
// One item is P consecutive positions (P = 8 or 4) of one replica: gather the local fields from
// the sliced-ELL coupling table, draw the item's Philox block, apply the Metropolis test with the
// 16+16-bit lazy uniforms, flip in shared memory and return the exact energy change.
#pragma once
#include <cstdint>

#include "dpt_common.cuh"
#include "dpt_internal.h"

namespace dpt {

// Shared memory is addressed through 32-bit byte offsets into the one dynamic shared array, so
// every access compiles to a shared load/store with 32-bit address arithmetic.
extern __shared__ __align__(16) unsigned char dpt_smem[];

__device__ __forceinline__ uint32_t lds_u32(uint32_t off) { return *reinterpret_cast<const uint32_t*>(dpt_smem + off); }
__device__ __forceinline__ int lds_s32(uint32_t off) { return *reinterpret_cast<const int*>(dpt_smem + off); }
__device__ __forceinline__ float lds_f32(uint32_t off) { return *reinterpret_cast<const float*>(dpt_smem + off); }
__device__ __forceinline__ int lds_s8(uint32_t off) { return (int)*reinterpret_cast<const int8_t*>(dpt_smem + off); }
__device__ __forceinline__ uint32_t lds_u8(uint32_t off) { return (uint32_t)*reinterpret_cast<const uint8_t*>(dpt_smem + off); }
__device__ __forceinline__ uint64_t lds_u64(uint32_t off) { return *reinterpret_cast<const uint64_t*>(dpt_smem + off); }
__device__ __forceinline__ uint4 lds_u128(uint32_t off) { return *reinterpret_cast<const uint4*>(dpt_smem + off); }
__device__ __forceinline__ void sts_u64(uint32_t off, uint64_t v) { *reinterpret_cast<uint64_t*>(dpt_smem + off) = v; }

struct Tables {
  // byte offsets in shared memory (tables staged in shared memory)
  uint32_t soff_o, ent_o, nbr_o, wf_o, h_o;
  // global pointers (tables read through L1/L2)
  const int* soff;
  const int* nbr;
  const int8_t* w8;
  const float* wf;
  const void* h;
};

template <bool kInSmem>
__device__ __forceinline__ int slice_off(const Tables& T, int S) {
  if constexpr (kInSmem) return lds_s32(T.soff_o + 4u * (uint32_t)S);
  else return __ldg(T.soff + S);
}

// P positions per item: sub-block b of group g covers positions 8g + P*b .. 8g + P*b + P-1. Every
// item computes the group's whole Philox block and uses its own halves of it.
template <int P> struct SpinWord;
template <> struct SpinWord<8> { using T = uint64_t; };
template <> struct SpinWord<4> { using T = uint32_t; };
template <> struct SpinWord<1> { using T = uint8_t; };

// Bits i of the result: position 8g + q0 + i lies in the colour range [lo, hi).
template <int P>
__device__ __forceinline__ uint32_t range_mask(int p0, int lo, int hi) {
  const int a = min(max(lo - p0, 0), P), e = min(max(hi - p0, 0), P);
  return ((1u << e) - 1u) & ~((1u << a) - 1u);
}

// Gather of the local fields of one item. W > 0 with kExactW: every slice has exactly W entries
// per position (so slice S starts at entry block S * W), and all 2 * W * P shared loads are
// independent and issued before any use. W > 0 without kExactW: W bounds the width, loads beyond it
// are predicated off. W == 0: run-time loop. An integer-path entry is (neighbour position << 8) |
// (uint8) weight: the spin's address is one shift-and-add of it.
template <int W, bool kExactW, bool kInSmem, bool kField, int P>
__device__ __forceinline__ void gather_int(int field[P], int S, int lane, int q0, uint32_t sp_o, const Tables& T) {
  const int w0 = kExactW ? S * W : slice_off<kInSmem>(T, S);
  const int width = kExactW ? W : slice_off<kInSmem>(T, S + 1) - w0;
  const uint32_t base = (uint32_t)w0 * kSlicePositions + lane;
#pragma unroll
  for (int i = 0; i < P; ++i) {
    const uint32_t hi_e = (uint32_t)(S * kSlicePositions + (q0 + i) * 32 + lane);
    if constexpr (!kField) field[i] = 0;
    else if constexpr (kInSmem) field[i] = lds_s32(T.h_o + 4u * hi_e);
    else field[i] = __ldg(static_cast<const int*>(T.h) + hi_e);
  }
  if constexpr (W > 0) {
    uint32_t ev[W][P];
#pragma unroll
    for (int d = 0; d < W; ++d)
#pragma unroll
      for (int i = 0; i < P; ++i) {
        const uint32_t e = base + (uint32_t)d * kSlicePositions + (uint32_t)(q0 + i) * 32;
        if (kExactW || d < width) {
          if constexpr (kInSmem) ev[d][i] = lds_u32(T.ent_o + 4u * e);
          else ev[d][i] = ((uint32_t)__ldg(T.nbr + e) << 8) | (uint32_t)(uint8_t)__ldg(T.w8 + e);
        } else {
          ev[d][i] = 0u;  // neighbour 0 with weight 0
        }
      }
    int sv[W][P];
#pragma unroll
    for (int d = 0; d < W; ++d)
#pragma unroll
      for (int i = 0; i < P; ++i) sv[d][i] = lds_s8(sp_o + (ev[d][i] >> 8));
#pragma unroll
    for (int d = 0; d < W; ++d)
#pragma unroll
      for (int i = 0; i < P; ++i) field[i] += (int)(int8_t)(uint8_t)ev[d][i] * sv[d][i];
  } else {
    for (int d = 0; d < width; ++d) {
      uint32_t ev[P];
#pragma unroll
      for (int i = 0; i < P; ++i) {
        const uint32_t e = base + (uint32_t)d * kSlicePositions + (uint32_t)(q0 + i) * 32;
        if constexpr (kInSmem) ev[i] = lds_u32(T.ent_o + 4u * e);
        else ev[i] = ((uint32_t)__ldg(T.nbr + e) << 8) | (uint32_t)(uint8_t)__ldg(T.w8 + e);
      }
#pragma unroll
      for (int i = 0; i < P; ++i) field[i] += (int)(int8_t)(uint8_t)ev[i] * lds_s8(sp_o + (ev[i] >> 8));
    }
  }
}

// sp_o: byte offset of the slot's spins; thr_o: byte offset of entry x = 0 of its rung's
// extended threshold row (entries x = -F..F; x <= 0 is accepted before the lookup).
template <int W, bool kExactW, bool kInSmem, bool kField, int P>
__device__ __forceinline__ int group_int(int g, int b, int lo, int hi, uint32_t t, uint32_t slot, uint32_t sp_o,
                                         const Tables& T, uint32_t thr_o, uint32_t c_sweep, uint32_t c_second,
                                         uint32_t k0, uint32_t k1) {
  using SW = typename SpinWord<P>::T;
  const int q0 = P * b;
  const int S = g >> 5, lane = g & 31;
  int field[P];
  gather_int<W, kExactW, kInSmem, kField, P>(field, S, lane, q0, sp_o, T);
  const U4 rnd = philox(U4{(uint32_t)g, t, slot, c_sweep}, k0, k1);
  const uint32_t words[4] = {rnd.x, rnd.y, rnd.z, rnd.w};
  const uint32_t own_o = sp_o + (uint32_t)(g * kGroup + q0);
  uint64_t s8 = (uint64_t)*reinterpret_cast<const SW*>(dpt_smem + own_o);
  const uint32_t inmask = range_mask<P>(g * kGroup + q0, lo, hi);
  // decisions of the item's positions as bit masks: accepted on the first 16 bits, and tied on
  // them (then the second 16 bits decide); one branch per item for the rare ties, and the spin
  // word updated once at the end
  uint32_t flips = 0u, ties = 0u;
  int dacc = 0;
#pragma unroll
  for (int i = 0; i < P; ++i) {
    const int q = q0 + i;
    const int si = (int)(int8_t)(uint8_t)(s8 >> (8 * i));
    const int x = si * field[i];
    const uint32_t thr = lds_u32(thr_o + 4u * (uint32_t)x);
    // the 16-bit uniform of position q of the group: half q & 1 of word q >> 1
    uint32_t word, sh;
    if constexpr (P == 8) {
      word = words[i >> 1];
      sh = (uint32_t)(i & 1) * 16u;
    } else if constexpr (P == 4) {
      word = b ? words[2 + (i >> 1)] : words[i >> 1];
      sh = (uint32_t)(i & 1) * 16u;
    } else {
      word = (q & 4) ? ((q & 2) ? words[3] : words[2]) : ((q & 2) ? words[1] : words[0]);
      sh = (uint32_t)(q & 1) * 16u;
    }
    const uint32_t prim = (word >> sh) & 0xFFFFu;
    const uint32_t th = thr >> 16;
    const bool in = (inmask >> i) & 1u;
    const bool acc = in & ((x <= 0) | (prim < th));
    flips |= (uint32_t)acc << i;
    ties |= (uint32_t)(in & (x > 0) & (prim == th)) << i;
    dacc += acc ? 2 * x : 0;
  }
  if (ties) {  // the first 16 bits tie: the second half of the uniform decides
#pragma unroll
    for (int i = 0; i < P; ++i)
      if ((ties >> i) & 1u) {
        const int x = (int)(int8_t)(uint8_t)(s8 >> (8 * i)) * field[i];
        const uint32_t thr = lds_u32(thr_o + 4u * (uint32_t)x);
        const U4 r2 = philox(U4{(uint32_t)(g * kGroup + q0 + i), t, slot, c_second}, k0, k1);
        if ((r2.x & 0xFFFFu) < (thr & 0xFFFFu)) {
          flips |= 1u << i;
          dacc += 2 * x;
        }
      }
  }
  // bit i of 4 flip bits -> byte i: the four shifted copies (by 0, 7, 14, 21) do not overlap, so the
  // product has no carries; then 0x01 <-> 0xFF (+1 <-> -1) in every flipped byte
  if constexpr (P == 8) {
    const uint32_t lo = ((flips & 15u) * 0x00204081u) & 0x01010101u;
    const uint32_t hi = ((flips >> 4) * 0x00204081u) & 0x01010101u;
    s8 ^= (((uint64_t)hi << 32) | lo) * 0xFEull;
  } else if constexpr (P == 4) {
    s8 ^= (uint64_t)(((flips * 0x00204081u) & 0x01010101u) * 0xFEu);
  } else {
    s8 ^= (uint64_t)(flips * 0xFEu);
  }
  *reinterpret_cast<SW*>(dpt_smem + own_o) = (SW)s8;
  return dacc;
}

__device__ __forceinline__ uint32_t lds_u16(uint32_t off) { return (uint32_t)*reinterpret_cast<const uint16_t*>(dpt_smem + off); }
__device__ __forceinline__ void sts_u16(uint32_t off, uint32_t v) { *reinterpret_cast<uint16_t*>(dpt_smem + off) = (uint16_t)v; }
__device__ __forceinline__ void sts_u32(uint32_t off, uint32_t v) { *reinterpret_cast<uint32_t*>(dpt_smem + off) = v; }
__device__ __forceinline__ void sts_u128(uint32_t off, uint4 v) { *reinterpret_cast<uint4*>(dpt_smem + off) = v; }

// The thresholds of a slot's rung for the positive energy changes x = W - 2j, j < (W + 1) / 2
// (x <= 0 is always accepted), held in registers for the round.
struct UnitThr {
  uint32_t t[3];
};

// One item of the unit-regular form: positions 8g + P j .. 8g + P j + P - 1 (P = 2 or 4) of one
// replica slot, on a problem whose spins all have W couplings of +-1 and no field.
//  * The slot's spins are bytes b (0 for +1, 1 for -1) and their flipped copy b ^ 1, at the addresses
//    the neighbour-address rows and own_o / own_nb_o give.
//  * The item's row of the neighbour-address table (desc_o, unit_row_bytes(P, W) bytes per item)
//    holds, for each position i and coupling d, the 16-bit shared address of the byte that neighbour
//    contributes: its b for a +1 coupling, its b ^ 1 for a -1 coupling. So J s_nb = 1 - 2 byte and
//    the position's field is W - 2k, k the sum of its W bytes.
//  * The position's x = (1 - 2b)(W - 2k) (= s_i field_i, half the flip's energy change) is computed
//    from b and k; for x > 0 its threshold comes from thr (registers, no shared-memory lookup).
//  * The uniforms come from the group's Philox block of this sweep, read from ubuf_o (16 bytes per
//    group); the caller computes the next sweep's blocks separately (unit_next_block).
// The Metropolis test, the uniforms and the energy change are those of group_int, so every form
// runs the same chain bit for bit.
// The item is given by its index (item = g NI + j, NI = 8 / P items per group) and the mask of its
// positions that lie in the phase's colour class.
// own_o / own_nb_o: the shared addresses of the item's P bytes in the b and b ^ 1 arrays (the
// storage order of words may differ from the position order; a word keeps its 4 positions in order).
// kRowReg: rows of at most 16 bytes (P W <= 8) come in registers (rowv, loaded once per launch:
// an item's row never changes), which takes one dependent shared load off every item's chain.
template <int W, int P>
constexpr bool unit_row_in_registers() {
  return ((2 * P * W + 7) / 8) * 8 <= 16;
}

template <int W, int P>
__device__ __forceinline__ int item_unit(uint32_t item, uint32_t inmask, uint32_t t, uint32_t slot, uint32_t own_o,
                                         uint32_t own_nb_o, uint32_t desc_o, uint4 rowv, uint32_t ubuf_o,
                                         const UnitThr& thr, uint32_t c_second, uint32_t k0, uint32_t k1) {
  static_assert(P == 2 || P == 4, "positions per item");
  constexpr int NI = kGroup / P;
  constexpr int RB = ((2 * P * W + 7) / 8) * 8;  // unit_row_bytes(P, W)
  const uint32_t g = item / NI, j = item % NI;
  const int p0 = (int)(item * P);
  uint32_t a16[RB / 2];
  {
    const uint32_t row = desc_o + item * RB;
    uint32_t w32[RB / 4];
    if constexpr (unit_row_in_registers<W, P>()) {
      const uint32_t rv[4] = {rowv.x, rowv.y, rowv.z, rowv.w};
#pragma unroll
      for (int c = 0; c < RB / 4; ++c) w32[c] = rv[c];
    } else if constexpr (RB % 16 == 0) {
#pragma unroll
      for (int c = 0; c < RB / 16; ++c) {
        const uint4 v = lds_u128(row + 16u * c);
        w32[4 * c] = v.x; w32[4 * c + 1] = v.y; w32[4 * c + 2] = v.z; w32[4 * c + 3] = v.w;
      }
    } else {
#pragma unroll
      for (int c = 0; c < RB / 8; ++c) {
        const uint64_t v = lds_u64(row + 8u * c);
        w32[2 * c] = (uint32_t)v;
        w32[2 * c + 1] = (uint32_t)(v >> 32);
      }
    }
#pragma unroll
    for (int c = 0; c < RB / 4; ++c) {
      a16[2 * c] = w32[c] & 0xFFFFu;
      a16[2 * c + 1] = w32[c] >> 16;
    }
  }
  uint32_t nbv[P * W];
#pragma unroll
  for (int k = 0; k < P * W; ++k) nbv[k] = lds_u8(a16[k]);
  uint32_t own = P == 2 ? lds_u16(own_o) : lds_u32(own_o);
  uint32_t words[P / 2];
  if constexpr (P == 2) {
    words[0] = lds_u32(ubuf_o + 16u * (uint32_t)g + 4u * (uint32_t)j);
  } else {
    const uint64_t w2 = lds_u64(ubuf_o + 16u * (uint32_t)g + 8u * (uint32_t)j);
    words[0] = (uint32_t)w2;
    words[1] = (uint32_t)(w2 >> 32);
  }
  uint32_t flips = 0u, ties = 0u;
  int dacc = 0;
  uint32_t kk[P];
#pragma unroll
  for (int i = 0; i < P; ++i) {
    uint32_t k = 0;
#pragma unroll
    for (int d = 0; d < W; ++d) k += nbv[i * W + d];
    kk[i] = k;
  }
  // x = (1 - 2b)(W - 2k); for x > 0 its threshold is thr.t[(W - x) / 2]
  int xs[P];
  uint32_t ths[P];
#pragma unroll
  for (int i = 0; i < P; ++i) {
    const uint32_t b = (own >> (8 * i)) & 1u;
    const int v = W - 2 * (int)kk[i];
    const int x = b ? -v : v;
    const int jx = (W - x) >> 1;
    uint32_t th32 = thr.t[0];
    if constexpr (W > 2) th32 = jx == 1 ? thr.t[1] : th32;
    if constexpr (W > 4) th32 = jx == 2 ? thr.t[2] : th32;
    xs[i] = x;
    ths[i] = th32;
    // position q = P j + i of the group: half q & 1 (= i & 1) of word q >> 1
    const uint32_t prim = (words[i >> 1] >> ((i & 1) * 16)) & 0xFFFFu;
    const uint32_t th = th32 >> 16;
    const bool in = (inmask >> i) & 1u;
    const bool acc = in & ((x <= 0) | (prim < th));
    flips |= (uint32_t)acc << i;
    ties |= (uint32_t)(in & (x > 0) & (prim == th)) << i;
    dacc += acc ? 2 * x : 0;
  }
  if (ties) {  // the first 16 bits tie: the second half of the uniform decides
#pragma unroll
    for (int i = 0; i < P; ++i)
      if ((ties >> i) & 1u) {
        const U4 r2 = philox(U4{(uint32_t)(p0 + i), t, slot, c_second}, k0, k1);
        if ((r2.x & 0xFFFFu) < (ths[i] & 0xFFFFu)) {
          flips |= 1u << i;
          dacc += 2 * xs[i];
        }
      }
  }
  if (flips) {
    // bit i of the flips -> bit 0 of byte i (see group_int), then b and b ^ 1 stored
    own ^= ((flips * 0x00204081u) & 0x01010101u);
    if constexpr (P == 2) {
      sts_u16(own_o, own);
      sts_u16(own_nb_o, own ^ 0x0101u);
    } else {
      sts_u32(own_o, own);
      sts_u32(own_nb_o, own ^ 0x01010101u);
    }
  }
  return dacc;
}

// The Philox block of group g for sweep t + 1 (computed during sweep t into unext_o).
__device__ __forceinline__ void unit_next_block(uint32_t g, uint32_t t, uint32_t slot, uint32_t unext_o,
                                                uint32_t c_sweep, uint32_t k0, uint32_t k1) {
  const U4 nx = philox(U4{g, t + 1u, slot, c_sweep}, k0, k1);
  sts_u128(unext_o + 16u * g, make_uint4(nx.x, nx.y, nx.z, nx.w));
}

template <int W, bool kExactW, bool kInSmem, bool kField>
__device__ __forceinline__ void gather_f32(float field[kGroup], int S, int lane, uint32_t sp_o, const Tables& T) {
  const int w0 = kExactW ? S * W : slice_off<kInSmem>(T, S);
  const int width = kExactW ? W : slice_off<kInSmem>(T, S + 1) - w0;
  const uint32_t base = (uint32_t)w0 * kSlicePositions + lane;
#pragma unroll
  for (int q = 0; q < kGroup; ++q) {
    const uint32_t hi_e = (uint32_t)(S * kSlicePositions + q * 32 + lane);
    if constexpr (!kField) field[q] = 0.0f;
    else if constexpr (kInSmem) field[q] = lds_f32(T.h_o + 4u * hi_e);
    else field[q] = __ldg(static_cast<const float*>(T.h) + hi_e);
  }
  // the sum runs over d in order (the fp32 rounding sequence is part of the definition)
  auto step = [&](int d) {
    int nb[kGroup];
    float wt[kGroup];
#pragma unroll
    for (int q = 0; q < kGroup; ++q) {
      const uint32_t e = base + (uint32_t)d * kSlicePositions + q * 32;
      if constexpr (kInSmem) {
        nb[q] = lds_s32(T.nbr_o + 4u * e);
        wt[q] = lds_f32(T.wf_o + 4u * e);
      } else {
        nb[q] = __ldg(T.nbr + e);
        wt[q] = __ldg(T.wf + e);
      }
    }
#pragma unroll
    for (int q = 0; q < kGroup; ++q) field[q] = f_add(field[q], lds_s8(sp_o + (uint32_t)nb[q]) > 0 ? wt[q] : -wt[q]);
  };
  if constexpr (W > 0) {
#pragma unroll
    for (int d = 0; d < W; ++d)
      if (kExactW || d < width) step(d);
  } else {
    for (int d = 0; d < width; ++d) step(d);
  }
}

template <int W, bool kExactW, bool kInSmem, bool kField>
__device__ __forceinline__ long long group_f32(int g, int lo, int hi, uint32_t t, uint32_t slot, uint32_t sp_o,
                                               const Tables& T, float neg2beta, uint32_t c_sweep,
                                               uint32_t c_second, uint32_t k0, uint32_t k1) {
  const int S = g >> 5, lane = g & 31;
  float field[kGroup];
  gather_f32<W, kExactW, kInSmem, kField>(field, S, lane, sp_o, T);
  const U4 rnd = philox(U4{(uint32_t)g, t, slot, c_sweep}, k0, k1);
  const uint32_t words[4] = {rnd.x, rnd.y, rnd.z, rnd.w};
  const uint32_t own_o = sp_o + (uint32_t)(g * kGroup);
  uint64_t s8 = *reinterpret_cast<const uint64_t*>(dpt_smem + own_o);
  const uint32_t inmask = range_mask<kGroup>(g * kGroup, lo, hi);
  long long dacc = 0;
#pragma unroll
  for (int q = 0; q < kGroup; ++q) {
    const int si = (int)(int8_t)(uint8_t)(s8 >> (8 * q));
    const float x = si > 0 ? field[q] : -field[q];
    const bool in = (inmask >> q) & 1u;
    const bool pos = x > 0.0f;
    const uint32_t thr = threshold_f(neg2beta, pos ? x : 0.0f);
    const uint32_t prim = (words[q >> 1] >> ((q & 1) * 16)) & 0xFFFFu;
    const uint32_t th = thr >> 16;
    bool acc = (!pos) | (prim < th);
    if (in & pos & (prim == th)) {
      const U4 r2 = philox(U4{(uint32_t)(g * kGroup + q), t, slot, c_second}, k0, k1);
      acc = (r2.x & 0xFFFFu) < (thr & 0xFFFFu);
    }
    acc = acc & in;
    s8 ^= acc ? ((uint64_t)0xFEu << (8 * q)) : 0ull;
    dacc += acc ? f_to_ll_rn(f_mul(x, 2.0f * kFloatEnergyQuant)) : 0ll;
  }
  *reinterpret_cast<uint64_t*>(dpt_smem + own_o) = s8;
  return dacc;
}

}  // namespace dpt
