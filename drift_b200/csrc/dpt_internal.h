// dpt_internal.h - declarations shared by the translation units of libdrift_pt (not public ABI).
#pragma once
#include <cstdarg>
#include <cstdint>

struct DriftPtCsr;

namespace dpt {

// Sliced-ELL geometry: a thread owns a group of 8 consecutive positions, a warp 32 groups,
// so one slice of the coupling table covers 256 positions.
constexpr int kGroup = 8;
constexpr int kSlicePositions = 256;
// Largest CTA of the sweep kernel: 512 threads leave 128 registers per thread for the gathers.
constexpr int kMaxThreads = 512;
// Largest CTA of the unit-regular form: 832 threads with 2 positions per item (72 registers per
// thread), 1024 with 4 (64 registers).
constexpr int kMaxUnitThreads = 1024;
constexpr int unit_max_threads(int P) { return P == 2 ? 832 : 1024; }
// The form's choice of positions per item for a largest colour class of `max_class` spins: 2 while
// one item per thread fits the 2-position CTA (a class touches at most (max_class + 14) / 8 groups).
constexpr int unit_auto_positions(int max_class) { return (max_class + 14) / kGroup * 4 <= 832 ? 2 : 4; }
// Colour classes the unit-regular form schedules statically (per class, a thread's item, Philox
// duty and row of neighbour addresses in registers).
constexpr int kUnitPhases = 4;

int set_error(int code, const char* fmt, ...);
void clear_error();

// Raises the kernel's dynamic shared-memory limit to `smem` (if needed) and returns how many CTAs
// of `threads` threads fit an SM. Results are cached per (kernel, threads, smem), so repeated
// launches (and launches inside a stream capture) make no further attribute or occupancy calls.
int prepare_kernel(const void* fn, int threads, size_t smem, int* per_sm);

// Checks a CSR problem and its colouring (ranges, permutation, no coupling inside a colour class);
// sets the error message and returns its status on failure.
int validate_csr(const DriftPtCsr* csr);

}  // namespace dpt
