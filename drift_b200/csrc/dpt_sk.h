// dpt_sk.h - geometry of the dense-coupling (SK) engine, shared by the host layout code and the
// sm_100a kernel (not public ABI).
//
// Spins are processed in blocks of 32 (one per lane). The local-field update after a block is the
// product F^T[rows][replicas] += Jq[rows][block] * delta[block][replicas], issued as
// tcgen05.mma kind::i8 with M = 128 rows per tile, N = 16 replica columns, K = 32 spins, int32
// accumulators in tensor memory. The 24-bit couplings enter as three int8 limbs, each its own
// accumulator; delta is the spin change s_new - s_old in {-2, 0, 2}.
//
// Operand layout in shared memory (K-major, no swizzle): a tile of `rows` x 32 int8 is a grid of
// 8-row x 16-byte core matrices; row r, byte k lives at
//   (r >> 3) * 256 + (k >> 4) * 128 + (r & 7) * 16 + (k & 15),
// i.e. leading-dimension offset 128 bytes (the two 16-byte K halves) and stride-dimension offset
// 256 bytes (consecutive 8-row groups).
#pragma once
#include <stddef.h>
#include <stdint.h>

#if defined(__CUDACC__)
#define DPT_SK_HD __host__ __device__ inline
#else
#define DPT_SK_HD inline
#endif

namespace dpt {
namespace sk {

constexpr int kBlock = 32;                       // spins per block
constexpr int kTile = 128;                       // MMA M
constexpr int kLimbs = 3;                        // int8 limbs of a 24-bit coupling
constexpr int kCols = 16;                        // MMA N (replica columns of one CTA)
constexpr int kTileBytes = kTile * kBlock;       // 4096: one tile of one limb
constexpr int kDiagBytes = kBlock * kBlock * 4;  // int32 diagonal block
constexpr int kOpBytes = kCols * kBlock;         // 512: one delta / spin operand
constexpr int kMaxN = 512;
constexpr int kMaxR = 512;
constexpr int kMaxG = 12;                        // replicas per CTA (12 resolver + 5 other warps: 96 registers)
constexpr int32_t kMaxCoupling = (1 << 23) - (1 << 16);
constexpr int32_t kMaxField = 1 << 30;

DPT_SK_HD int core_offset(int row, int k) { return (row >> 3) * 256 + (k >> 4) * 128 + (row & 7) * 16 + (k & 15); }

// n spins -> n_tiles 128-row tiles, n_blocks = 4 n_tiles blocks (padding spins never flip).
DPT_SK_HD int n_tiles(int n) { return (n + kTile - 1) / kTile; }
DPT_SK_HD int n_blocks(int n) { return 4 * n_tiles(n); }
// One block's entry in the device coupling table: n_tiles * 3 limb tiles, then two int32 32 x 32
// blocks: the diagonal block [f][l] = Jq[32B + f][32B + l] and the previous-block couplings
// [f][l] = Jq[32 prev(B) + f][32B + l], prev(B) = (B - 1) mod n_blocks (the sweep order wraps).
DPT_SK_HD size_t entry_bytes(int n) { return (size_t)n_tiles(n) * kLimbs * kTileBytes + 2 * kDiagBytes; }

// Balanced base-256 digits of |v| < 2^23 - 2^16: v = d0 + 256 d1 + 65536 d2, d in [-128, 127].
DPT_SK_HD void limbs(int32_t v, int8_t d[3]) {
  const int32_t d0 = ((v + 128) & 255) - 128;
  const int32_t v1 = (v - d0) / 256;
  const int32_t d1 = ((v1 + 128) & 255) - 128;
  const int32_t d2 = (v1 - d1) / 256;
  d[0] = (int8_t)d0;
  d[1] = (int8_t)d1;
  d[2] = (int8_t)d2;
}

}  // namespace sk
}  // namespace dpt
