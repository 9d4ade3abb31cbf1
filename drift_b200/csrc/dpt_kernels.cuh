// dpt_kernels.cuh - kernel argument block and shared-memory plan of the PT kernels.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace dpt {

struct PtKernelArgs {
  // problem, position space
  int n, n_pos, n_slices, n_colors, F;
  long long n_ell;
  const int* color_ptr;
  const int* slice_off;
  const int* ell_nbr;
  const void* ell_w;
  const void* h_pos;
  const uint16_t* unit_place;  // unit-regular form: storage word of each 4-position word, or NULL
  // ladder and run
  int R, rpc, spr, n_rounds;
  long long round0;
  uint32_t k0, k1, inst;
  const double* betas;
  const uint32_t* thr;
  // state
  int8_t* spins;
  long long* energy;
  long long* best_energy;
  int8_t* best_spins;
  int* rung_of_slot;
  int* slot_of_rung;
  long long* tried;
  long long* accepted;
  double* best_hist;
  // workspace
  int* err;
  long long* pub;                // [2][R] energies published per round parity
  unsigned long long* tags;      // [2][R] round + 1 once the matching energy is visible
  int packed;                    // 1: pub holds (round + 1) << 32 | int32 energy words, tags unused
  long long timeout_ns;
};

struct SmemLayout {
  size_t spins, eacc, ecur, ebest, imp, eall, rung, slot, beta, nb, thr, stats, cptr, ctl;
  size_t soff, nbr, w, h, cpub, usw, total;
};

__host__ __device__ inline size_t align16(size_t x) { return (x + 15) & ~(size_t)15; }

// Byte offsets of every shared-memory array; the host sizes the launch with the same function.
// Threads are bound to replica slots: `threads / rpc` threads per slot (a power of two below 32 or
// a multiple of 32, so shuffle segments never straddle two slots). `eacc` holds one partial energy
// change per shuffle segment. `cpub` (cluster form only) holds the slots' energies of the last two
// rounds, read by the other CTAs of the cluster through distributed shared memory.
__host__ __device__ inline int seg_width(int threads, int rpc) {
  const int tps = threads / rpc;
  return tps < 32 ? tps : 32;
}

// Unit-regular form (unit_w = W > 0, unit_p = P positions per item): a slot's spins are two byte
// arrays, b (0 for +1, 1 for -1) and b ^ 1, followed by 16 zero bytes, at the start of shared memory
// (so every spin byte has a 16-bit address); the coupling table is replaced by one row per item of
// P * W 16-bit neighbour addresses (unit_row_bytes), the threshold rows by the decision table of
// 2 (W + 1) 64-bit entries per rung, and the Philox blocks of the current and the next sweep are
// kept per group (2 x 16 bytes per group). `usw` holds the swap uniforms of the exchange lanes' first
// pairs for two rounds (by round parity), drawn a round ahead.
__host__ __device__ inline size_t unit_slot_bytes(int n_pos) { return 2 * (size_t)n_pos + 16; }
__host__ __device__ inline int unit_row_bytes(int P, int W) { return ((2 * P * W + 7) / 8) * 8; }

__host__ __device__ inline SmemLayout smem_layout(int n_pos, int rpc, int R, int F, int n_colors, int n_slices,
                                                  long long n_ell, bool integer_path, bool ell_in_smem,
                                                  int threads, bool cluster = false, int unit_w = 0,
                                                  int unit_p = 2) {
  SmemLayout L;
  size_t o = 0;
  L.spins = o; o = align16(o + (size_t)rpc * (unit_w ? unit_slot_bytes(n_pos) : (size_t)n_pos));
  L.eacc = o;  o = align16(o + 8 * (size_t)(threads / seg_width(threads, rpc)));
  L.ecur = o;  o = align16(o + 8 * (size_t)rpc);
  L.ebest = o; o = align16(o + 8 * (size_t)rpc);
  L.imp = o;   o = align16(o + 4 * (size_t)rpc);
  L.eall = o;  o = align16(o + 8 * (size_t)R);
  L.rung = o;  o = align16(o + 4 * (size_t)R);
  L.slot = o;  o = align16(o + 4 * (size_t)R);
  L.beta = o;  o = align16(o + 8 * (size_t)R);
  L.nb = o;    o = align16(o + 4 * (size_t)rpc);
  if (unit_w) {
    L.thr = o; o = align16(o + 8 * (size_t)R * 2 * (unit_w + 1));  // (threshold, x) per (rung, spin, count)
  } else {
    L.thr = o; o = align16(o + (integer_path ? 4 * (size_t)R * (2 * F + 1) : 0));  // rows for x = -F..F
  }
  L.stats = o; o = align16(o + 8 * (size_t)(R > 1 ? R - 1 : 0));
  L.cptr = o;  o = align16(o + 4 * (size_t)(n_colors + 1));
  L.ctl = o;   o = align16(o + 16);
  L.soff = L.nbr = L.w = L.h = o;
  if (unit_w) {
    // neighbour addresses: (n_pos / P) item rows; Philox blocks: [2][n_pos / 8] x 16 bytes
    L.nbr = o; o = align16(o + (size_t)(n_pos / unit_p) * unit_row_bytes(unit_p, unit_w));
    L.w = o;   o = align16(o + 2 * 16 * (size_t)(n_pos / 8));
    L.h = o;   o = align16(o + 2 * (size_t)(n_pos / 4));  // storage word of each 4-position word
  } else if (ell_in_smem) {
    L.soff = o; o = align16(o + 4 * (size_t)(n_slices + 1));
    L.nbr = o;  o = align16(o + 4 * (size_t)n_ell);  // integer path: packed neighbour | weight << 24
    L.w = o;    o = align16(o + (integer_path ? 0 : 4) * (size_t)n_ell);
    L.h = o;    o = align16(o + 4 * (size_t)n_pos);
  }
  L.cpub = o;   o = align16(o + (cluster ? 16 * (size_t)rpc : 0));
  L.usw = o;    o = align16(o + (unit_w ? 2 * 32 * sizeof(double) : 0));
  L.total = o;
  return L;
}

cudaError_t launch_init(const PtKernelArgs& a, int integer_path, cudaStream_t st);
cudaError_t launch_energy_fp64(const PtKernelArgs& a, int integer_path, const int8_t* spins, int R, double* out,
                               cudaStream_t st);
// unit > 0: the unit-regular form with positions_per_item = 2 or 4, compiled for `unit` colour phases
// at most (2 or kUnitPhases; any value up to 2 picks the 2-phase instance)
const void* run_kernel_ptr(int integer_path, int in_smem, int max_width, int min_width, int has_field,
                           int positions_per_item, int cluster = 0, int unit = 0);
// widths the unit-regular form is compiled for
bool unit_width_supported(int w);

}  // namespace dpt
