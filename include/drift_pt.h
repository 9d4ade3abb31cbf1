/* drift_pt.h - C ABI of the B200 parallel-tempering (replica-exchange Metropolis) engine.
 *
 * This library replaces the process boundary of DRiFT's GPU path: drift/gpu.py:83-103 writes a
 * problem.bin, runs the cuda/ising_pt executable as a subprocess and parses result.bin and its
 * stderr. Here the same inputs (CSR couplings, field, greedy colouring, ladder, rounds, sweeps,
 * seed) cross a plain C ABI instead: no file, no process, no torch types. Every function returns
 * an int status (DRIFT_PT_OK = 0) instead of exiting (cuda/ising_pt.cu:30-38); the message of the
 * last failure on the calling thread is available from drift_pt_last_error().
 *
 * Two layers:
 *   - host helpers (colouring, layout, thresholds) and drift_pt_solve(): host buffers in and out,
 *     the whole problem.bin -> result.bin contract in one call (it allocates device memory);
 *   - the device layer (drift_pt_init / drift_pt_run / drift_pt_energy_fp64): every pointer is
 *     device memory owned by the caller, the call is asynchronous on the given CUDA stream and
 *     allocates nothing. Scratch space is a caller-provided workspace of
 *     drift_pt_workspace_bytes() bytes.
 *
 * Streams are passed as void* (a cudaStream_t; NULL = legacy default stream).
 */
#ifndef DRIFT_PT_H
#define DRIFT_PT_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define DRIFT_PT_API __attribute__((visibility("default")))
#else
#define DRIFT_PT_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define DRIFT_PT_OK 0
#define DRIFT_PT_EINVAL 1       /* invalid argument (sizes, pointers, colouring, ladder)        */
#define DRIFT_PT_ECUDA 2        /* a CUDA runtime call failed                                   */
#define DRIFT_PT_ETIMEOUT 3     /* a bounded wait inside a kernel gave up (error flag was set)  */
#define DRIFT_PT_ENOMEM 4       /* device allocation failed (drift_pt_solve only)               */
#define DRIFT_PT_EUNSUPPORTED 5 /* problem does not fit the engine's limits                     */

/* Version string of the library, e.g. "drift-b200-pt 0.1.0 sm_100a". */
DRIFT_PT_API const char* drift_pt_version(void);

/* Message of the last failed call on this thread ("" if none). */
DRIFT_PT_API const char* drift_pt_last_error(void);

/* ---------------------------------------------------------------------------------------------
 * Problem description in the reference's own terms (drift/gpu.py:66-81): CSR of the symmetric,
 * zero-diagonal coupling matrix J (rows grouped, columns ascending within a row as np.nonzero
 * yields them), fp32 weights and field, and a colouring given as color_ptr[k+1] / color_spins[n]
 * (spin ids grouped by colour, ascending within a colour: the stable argsort of gpu.py:142-144).
 * ------------------------------------------------------------------------------------------- */
typedef struct DriftPtCsr {
  int32_t n;                  /* number of spins                                            */
  int64_t nnz;                /* directed CSR entries (2 x edges)                           */
  const int32_t* row_ptr;     /* [n+1]                                                      */
  const int32_t* col_idx;     /* [nnz]                                                      */
  const float* weight;        /* [nnz] J_ij                                                 */
  const float* h;             /* [n]   h_i                                                  */
  int32_t n_colors;           /* k                                                          */
  const int32_t* color_ptr;   /* [k+1]                                                      */
  const int32_t* color_spins; /* [n]                                                        */
} DriftPtCsr;

/* Greedy colouring in index order, smallest colour unused by an already-coloured neighbour.
 * Replaces drift/gpu.py:122-141 (_greedy_coloring). color[n] receives each spin's colour. */
DRIFT_PT_API int drift_pt_greedy_coloring(int32_t n, const int32_t* row_ptr, const int32_t* col_idx,
                             int32_t* color, int32_t* n_colors);

/* color_ptr[k+1] and color_spins[n] from color[n]: the stable argsort of drift/gpu.py:142-144. */
DRIFT_PT_API int drift_pt_color_order(int32_t n, const int32_t* color, int32_t n_colors, int32_t* color_ptr,
                         int32_t* color_spins);

/* ---------------------------------------------------------------------------------------------
 * Device layout. Spins are renumbered into "positions": colour classes are contiguous position
 * ranges in color_spins order. Couplings are stored as a sliced ELL: a slice is 256 positions
 * (32 groups of 8 consecutive positions); its entries are laid out [d][q][lane] where
 * position = 256*slice + 8*lane + q and d < width(slice) = max degree in the slice. Padded
 * entries have weight 0. Neighbours keep the CSR (ascending original column) order. Field h is
 * stored in the same [q][lane] order per slice (width 1).
 * No counterpart in the reference (its kernel walks the CSR directly, cuda/ising_pt.cu:111-115).
 * ------------------------------------------------------------------------------------------- */
typedef struct DriftPtLayoutInfo {
  int32_t n;                 /* spins                                                       */
  int32_t n_pos;             /* positions, n rounded up to a multiple of 256                */
  int32_t n_slices;          /* n_pos / 256                                                 */
  int32_t n_colors;          /* k                                                           */
  int64_t n_ell;             /* ELL entries = 256 * sum of slice widths                     */
  int32_t max_degree;        /* largest row length                                          */
  int32_t integer_couplings; /* 1 if every J_ij is an integer in [-127,127] and every h_i an
                                integer in [-2^20, 2^20]                                    */
  int32_t max_field;         /* F = max_i (sum_j |J_ij| + |h_i|) on the integer path        */
  int32_t has_field;         /* 1 if some h_i != 0                                          */
  int32_t min_width;         /* smallest slice width (== max_degree: uniform, e.g. lattices) */
  int32_t unit_regular;      /* 1 if every spin has max_degree couplings, every coupling is
                                +1 or -1 and there is no field (MaxCut on regular graphs,
                                +-J lattices): such problems can run the unit-regular sweep
                                (item_form 2 of the run args)                               */
} DriftPtLayoutInfo;

DRIFT_PT_API int drift_pt_layout_query(const DriftPtCsr* csr, DriftPtLayoutInfo* info);

typedef struct DriftPtLayout { /* caller-allocated arrays, sized from DriftPtLayoutInfo */
  int32_t* color_ptr;        /* [k+1] position offsets of the colour classes                */
  int32_t* slice_off;        /* [n_slices+1] offsets in units of 256 entries                */
  int32_t* ell_nbr;          /* [n_ell] neighbour positions                                 */
  void* ell_w;               /* [n_ell] int8 (integer path) or float                        */
  void* h_pos;               /* [n_pos] int32 (integer path) or float, [q][lane] per slice  */
  int32_t* site_of_pos;      /* [n_pos] original spin id, -1 for padding                    */
  int32_t* pos_of_site;      /* [n]                                                         */
} DriftPtLayout;

DRIFT_PT_API int drift_pt_layout_fill(const DriftPtCsr* csr, int32_t integer_path, DriftPtLayout* out);

/* Storage order of the unit-regular form's spin bytes in shared memory: word_slot[n_pos / 4]
 * receives, for the 4-byte word of positions 4u .. 4u+3, the shared-memory word it is stored in
 * (a permutation of 0 .. n_pos/4 - 1), chosen so that the neighbour gathers of the form's items
 * (positions_per_item 2 or 4; 0 = the form's own choice) fall on few banks at a time. Pass it as
 * DriftPtDeviceProblem.unit_place; any permutation gives the same chain bit for bit, only the
 * shared-memory conflicts differ. Host function; DRIFT_PT_EUNSUPPORTED if the problem is not
 * unit-regular. No counterpart in the reference. */
DRIFT_PT_API int drift_pt_unit_placement(const DriftPtCsr* csr, int32_t positions_per_item, uint16_t* word_slot);

/* Metropolis thresholds of the integer path, thr[r*F + x-1] = floor(exp(-2 x beta_r) 2^32)
 * (saturated at 2^32-1) for x = 1..F. Host function. Replaces the per-attempt expf of
 * cuda/ising_pt.cu:118. */
DRIFT_PT_API int drift_pt_thresholds(int32_t n_rungs, const double* betas, int32_t max_field, uint32_t* thr);

/* ---------------------------------------------------------------------------------------------
 * Device layer. All pointers below are device memory.
 * ------------------------------------------------------------------------------------------- */
typedef struct DriftPtDeviceProblem {
  int32_t n, n_pos, n_slices, n_colors;
  int32_t integer_path;      /* 1: int8 weights, int32 field, threshold table; 0: fp32      */
  int32_t max_field;         /* F (integer path)                                            */
  int32_t max_width;         /* largest slice width                                         */
  int32_t max_class;         /* size of the largest colour class                            */
  int32_t has_field;         /* 0 if every h_i == 0 (the field is then never read)          */
  int32_t min_width;         /* smallest slice width; the layout's values of max_field,
                                max_width, min_width and unit_regular must be passed unchanged */
  int32_t unit_regular;      /* DriftPtLayoutInfo.unit_regular (0 is always allowed)        */
  int64_t n_ell;
  const int32_t* color_ptr;
  const int32_t* slice_off;
  const int32_t* ell_nbr;
  const void* ell_w;
  const void* h_pos;
  const uint16_t* unit_place;  /* [n_pos/4] from drift_pt_unit_placement, or NULL (positions in order);
                                  used by the unit-regular form only                            */
} DriftPtDeviceProblem;

/* Replica state, indexed by replica *slot*. Slots keep their configuration; replica exchange
 * permutes which rung (beta) each slot holds (rung_of_slot / slot_of_rung). This is the same
 * Markov chain as swapping configurations between fixed rungs
 * (drift/solvers/parallel_tempering.py:104-113). */
typedef struct DriftPtDeviceState {
  int8_t* spins;             /* [R][n_pos] +-1, position order                              */
  int64_t* energy;           /* [R] fixed point (scale 1 integer path, 2^-32 float path)    */
  int64_t* best_energy;      /* [R] lowest energy each slot has held at a round end         */
  int8_t* best_spins;        /* [R][n_pos]                                                  */
  int32_t* rung_of_slot;     /* [R]                                                         */
  int32_t* slot_of_rung;     /* [R]                                                         */
  int64_t* swap_tried;       /* [R-1] per rung pair (r, r+1), cumulative                    */
  int64_t* swap_accepted;    /* [R-1]                                                       */
  double* best_history;      /* [n_rounds of a run] best energy so far after each round, or NULL */
} DriftPtDeviceState;

typedef struct DriftPtRunArgs {
  int32_t n_replicas;        /* R (rungs = slots)                                           */
  int32_t n_rounds;          /* rounds in this call                                         */
  int32_t sweeps_per_round;  /* Metropolis sweeps between exchange steps                    */
  int32_t round_sync;        /* how the CTAs meet at each round end: 0 = auto, 1 = grid
                                (bounded barrier in global memory, any ladder), 2 = one
                                thread-block cluster of at most 16 CTAs (energies through
                                distributed shared memory; ladders that fit, coupling table in
                                shared memory). The results do not depend on it.            */
  int64_t round_offset;      /* index of the first round (resume); sweeps are numbered
                                round * sweeps_per_round + j                                */
  uint64_t seed;
  uint32_t instance;         /* stream id (< 2^24), distinct per independent chain set      */
  int32_t replicas_per_cta;  /* 0 = auto (autotuner)                                        */
  int32_t threads_per_cta;   /* 0 = auto; at most 512                                       */
  int32_t positions_per_item;/* 8, 4 or 1 spins per thread and phase (4 and 1: integer path;
                                1: coupling table in shared memory); 0 = auto               */
  int32_t item_form;         /* how an item reads its neighbours: 0 = auto, 1 = the sliced
                                ELL gather (any problem), 2 = the unit-regular sweep (problems
                                with unit_regular set, one replica per CTA, 8 positions per
                                item: neighbour addresses precomputed in shared memory, spins
                                as 0/1 bytes with a sign-flipped copy, the decision looked up
                                by (spin, unsatisfied-bond count)). Results do not depend on it. */
  const double* betas;       /* [R] inverse temperature of each rung                        */
  const uint32_t* thresholds;/* [R][F] integer path (from drift_pt_thresholds), else NULL   */
  double timeout_s;          /* bound on any in-kernel wait (0 = 10 s)                      */
} DriftPtRunArgs;

/* Bytes of device workspace drift_pt_run needs for R replicas. */
DRIFT_PT_API int drift_pt_workspace_bytes(int32_t n_replicas, size_t* bytes);

/* Random initial spins (Philox, seed/instance of args), their energies, best = initial,
 * identity rung assignment, zeroed swap counters. Asynchronous. */
DRIFT_PT_API int drift_pt_init(const DriftPtDeviceProblem* prob, const DriftPtRunArgs* args,
                  DriftPtDeviceState* state, void* stream);

/* Runs args->n_rounds rounds of (sweeps_per_round colour-ordered Metropolis sweeps on every
 * replica, then one exchange step over adjacent rungs with parity = round & 1). Replaces the
 * host loop of cuda/ising_pt.cu:214-218 with one persistent launch. Asynchronous; the
 * workspace must not be shared with a concurrent call. Call drift_pt_check() to learn whether
 * a bounded wait timed out. */
DRIFT_PT_API int drift_pt_run(const DriftPtDeviceProblem* prob, const DriftPtRunArgs* args,
                 DriftPtDeviceState* state, void* workspace, size_t workspace_bytes, void* stream);

/* drift_pt_run for callers that cannot allocate device memory (a framework already holds the
 * device's memory in its own pool, a real-time loop may not call cudaMalloc after start-up, or a
 * foreign-language binding only receives pointers to buffers others own). It takes no workspace:
 * the scratch lives in an array built into the library, DRIFT_PT_NOALLOC_MAX_REPLICAS replicas
 * at most (about 128 KiB, held on every GPU that loads the library until the process exits); more
 * replicas return DRIFT_PT_EUNSUPPORTED. The caller still passes the problem, the state and the
 * ladder. Nothing is allocated: no cudaMalloc, no cudaFree, no allocating library call.
 * The first call on a device looks up the array's device address (cudaGetSymbolAddress) while
 * that device is current; make that first call before any stream capture. All calls in the
 * process share the one array: calls that overlap on the GPU (other streams, other threads) race
 * on it and must be serialised by the caller. Call drift_pt_noalloc_check() to learn whether a
 * bounded in-kernel wait timed out. No counterpart in the reference. */
#define DRIFT_PT_NOALLOC_MAX_REPLICAS 4096
DRIFT_PT_API int drift_pt_run_noalloc(const DriftPtDeviceProblem* prob, const DriftPtRunArgs* args,
                                      DriftPtDeviceState* state, void* stream);

/* drift_pt_check for drift_pt_run_noalloc: synchronises the stream and returns DRIFT_PT_ETIMEOUT
 * if the built-in scratch array's error flag is set (the last run's bounded wait gave up and its
 * state is incomplete). Reads the flag with a synchronous copy from the array; allocates nothing.
 * No counterpart in the reference. */
DRIFT_PT_API int drift_pt_noalloc_check(void* stream);

/* Synchronises the stream and returns DRIFT_PT_ETIMEOUT if the workspace's error flag is set. */
DRIFT_PT_API int drift_pt_check(void* workspace, void* stream);

/* Full recompute of every slot's energy in FP64 from its spins (the check on the incremental
 * bookkeeping; cuda/ising_pt.cu:59-68 computes it at init only). out[R] in the model's units. */
DRIFT_PT_API int drift_pt_energy_fp64(const DriftPtDeviceProblem* prob, const int8_t* spins, int32_t n_replicas,
                         double* out, void* stream);

/* ---------------------------------------------------------------------------------------------
 * Batched layer: many independent instances (each its own couplings, colouring, size, ladder and
 * replica count) advanced together by one persistent launch per call. No counterpart in the
 * reference (its engine runs one instance per process, drift/gpu.py:97). Instance k is the same
 * chain as a single-instance run with instance = desc[k].stream_id, so batching never changes
 * results. All pointers are device memory. The per-instance layout arrays are the single-instance
 * layout arrays concatenated; desc[k] holds the offsets.
 * ------------------------------------------------------------------------------------------- */
typedef struct DriftPtInstanceDesc {
  int32_t n, n_pos, n_slices, n_colors;
  int32_t n_replicas;        /* R_k                                                         */
  int32_t max_field;         /* F_k (integer path)                                          */
  int32_t stream_id;         /* Philox stream of the instance (< 2^24)                      */
  int32_t reserved;
  int64_t color_ptr;         /* element offset of the instance's color_ptr[k+1]             */
  int64_t slice_off;         /* element offset of its slice_off[n_slices+1]                 */
  int64_t ell;               /* element offset of its ELL entries (slice_off is relative)   */
  int64_t pos;               /* element offset of its h_pos[n_pos]                          */
  int64_t slot0;             /* first replica slot of the instance in the batch             */
  int64_t spin0;             /* byte offset of its spins [R_k][n_pos] in the spin arrays     */
  int64_t thr;               /* element offset of its thresholds [R_k][F_k] (integer path)  */
} DriftPtInstanceDesc;

typedef struct DriftPtBatchProblem {
  int32_t n_instances;
  int32_t integer_path;      /* the same path for every instance of a batch                 */
  int32_t has_field;         /* 1 if any instance has a non-zero field                      */
  int32_t max_width;         /* largest slice width over the batch                          */
  int32_t min_width;         /* smallest slice width over the batch                         */
  int32_t max_field;         /* largest F_k                                                 */
  int32_t max_n_pos;         /* largest n_pos                                               */
  int32_t max_colors;        /* largest colour count                                        */
  int64_t total_slots;       /* sum of R_k                                                  */
  const DriftPtInstanceDesc* desc; /* [n_instances]                                         */
  const int32_t* color_ptr;
  const int32_t* slice_off;
  const int32_t* ell_nbr;
  const void* ell_w;
  const void* h_pos;
  const double* betas;       /* [total_slots]: beta of rung r of instance k at slot0_k + r  */
  const uint32_t* thresholds;/* integer path: [R_k][F_k] per instance at desc.thr           */
} DriftPtBatchProblem;

/* Layout of a whole batch in two calls (the per-instance layout query/fill of every instance, with
 * the descriptor offsets and the threshold tables): drift_pt_batch_layout_query sizes the
 * concatenated arrays and returns each instance's DriftPtLayoutInfo; drift_pt_batch_layout_fill
 * writes instance k's layout at its offsets (desc[k]) and, on the integer path, its thresholds
 * [R_k][F_k] from betas (concatenated, R_k per instance). Instances are split over the host's
 * threads. Replaces the per-instance host loop of a batch (drift/gpu.py:69-81 once per instance). */
typedef struct DriftPtBatchSizes {
  int64_t color_ptr, slice_off, ell, pos, sites; /* element counts of the concatenated arrays    */
  int32_t all_integer;       /* 1 if every instance has integer couplings                    */
  int32_t reserved;
} DriftPtBatchSizes;

typedef struct DriftPtBatchLayout { /* caller-allocated, sized from DriftPtBatchSizes */
  int32_t* color_ptr;        /* [color_ptr]                                                  */
  int32_t* slice_off;        /* [slice_off]                                                  */
  int32_t* ell_nbr;          /* [ell]                                                        */
  void* ell_w;               /* [ell] int8 (integer path) or float                           */
  void* h_pos;               /* [pos] int32 (integer path) or float                          */
  int32_t* site_of_pos;      /* [pos]                                                        */
  int32_t* pos_of_site;      /* [sites]: instance k's at the sum of the earlier instances' n  */
} DriftPtBatchLayout;

DRIFT_PT_API int drift_pt_batch_layout_query(int32_t n_instances, const DriftPtCsr* csrs, DriftPtLayoutInfo* infos,
                                             DriftPtBatchSizes* sizes);
DRIFT_PT_API int drift_pt_batch_layout_fill(int32_t n_instances, const DriftPtCsr* csrs, const DriftPtLayoutInfo* infos,
                                            int32_t integer_path, const int32_t* n_replicas, const int32_t* stream_ids,
                                            const double* betas, DriftPtInstanceDesc* desc, uint32_t* thresholds,
                                            DriftPtBatchLayout* out);

/* Work items: one item = replicas [first, first + count) of one instance, processed by one CTA
 * for a round. items[3*i] = instance, items[3*i+1] = first local slot, items[3*i+2] = count.
 * Order them largest first for load balance (drift_pt_batch_items does). */
DRIFT_PT_API int drift_pt_batch_items(int32_t n_instances, const int32_t* n_pos, const int32_t* n_replicas,
                                      int32_t max_tile, int64_t smem_budget, int32_t* items, int32_t* n_items);

typedef struct DriftPtBatchRunArgs {
  int32_t n_rounds, sweeps_per_round;
  int64_t round_offset;
  uint64_t seed;
  const int32_t* items;      /* device [n_items][3]                                         */
  int32_t n_items;
  int32_t max_tile;          /* largest item count                                          */
  int32_t threads_per_slot;  /* threads bound to each slot of an item: 1..32 power of two or
                                a multiple of 32; max_tile * threads_per_slot <= 512        */
  int32_t ctas_per_sm;       /* 0 = as many as fit                                          */
  int32_t positions_per_item;/* 8 or 4 (integer path), 0 = auto                             */
  int32_t max_item_bytes;    /* largest count * n_pos over the items (spins staged per item) */
  double timeout_s;
} DriftPtBatchRunArgs;

/* Initial spins/energies of every instance (as drift_pt_init with instance = stream_id). The
 * state arrays are the single-instance arrays of all instances concatenated (spins at spin0,
 * per-slot arrays at slot0; swap_tried/accepted have one entry per slot, R_k - 1 used). */
DRIFT_PT_API int drift_pt_batch_init(const DriftPtBatchProblem* prob, const DriftPtBatchRunArgs* args,
                                     DriftPtDeviceState* state, void* stream);
DRIFT_PT_API int drift_pt_batch_workspace_bytes(const DriftPtBatchProblem* prob, size_t* bytes);
/* n_rounds rounds of every instance: each round, CTAs take items from a queue and run the
 * sweeps; a grid barrier; one warp per instance runs its exchange step; a grid barrier. */
DRIFT_PT_API int drift_pt_batch_run(const DriftPtBatchProblem* prob, const DriftPtBatchRunArgs* args,
                                    DriftPtDeviceState* state, void* workspace, size_t workspace_bytes,
                                    void* stream);

/* ---------------------------------------------------------------------------------------------
 * Multispin layer: +-J cubic lattices (d = 2 or 3, even side L, periodic, no field) with 32
 * replicas packed per 32-bit word. No counterpart in the reference: its engine stores one float
 * per spin per replica and a CSR of J (cuda/ising_pt.cu:47-52,190-191), and a 3-D L = 64 lattice
 * cannot even be built as its dense IsingModel (drift/ising.py:32).
 *   Sites are split by checkerboard colour c = (x + y + z) & 1: q = c * N/2 + (x >> 1)
 *   + (L/2) * (y + L * z). Spin words [W][N]: bit b of word w at q is replica slot 32 w + b,
 *   1 = spin -1. jneg[q] bit d (d = 0: +x, 1: +y, 2: +z) is set when J(site, site + e_d) = -1.
 *   Thresholds: [R][2d] from drift_pt_thresholds(R, betas, 2d, ...) (a flip with k unsatisfied
 *   bonds has dE = 4 (d - k); k >= d is always accepted).
 * ------------------------------------------------------------------------------------------- */
typedef struct DriftPtLattice {
  int32_t dims, L;
  const uint8_t* jneg;       /* device [N]                                                  */
} DriftPtLattice;

typedef struct DriftPtMsState { /* device arrays; R = 32 * n_words */
  uint32_t* words;           /* [W][N]                                                      */
  uint32_t* best_words;      /* [W][N]: bit b holds replica b's lowest-energy configuration  */
  int64_t* energy;           /* [R] exact, E = -sum_bonds J s s                             */
  int64_t* best_energy;      /* [R]                                                         */
  int32_t* rung_of_slot;     /* [R]                                                         */
  int32_t* slot_of_rung;     /* [R]                                                         */
  int64_t* swap_tried;       /* [R-1]                                                       */
  int64_t* swap_accepted;    /* [R-1]                                                       */
} DriftPtMsState;

typedef struct DriftPtMsRunArgs {
  int32_t n_words;           /* W (replicas R = 32 W), 1..64                                */
  int32_t n_rounds, sweeps_per_round;
  int32_t ctas_per_sm;       /* 0 = 2                                                       */
  int64_t round_offset;
  uint64_t seed;
  uint32_t instance;
  int32_t reserved;
  const double* betas;       /* [R] device                                                  */
  const uint32_t* thresholds;/* [R][2d] device                                              */
  double timeout_s;
} DriftPtMsRunArgs;

DRIFT_PT_API int drift_pt_ms_workspace_bytes(int32_t n_words, size_t* bytes);
/* Random initial words (Philox), exact energies, best = initial, identity rungs. */
DRIFT_PT_API int drift_pt_ms_init(const DriftPtLattice* lat, const DriftPtMsRunArgs* args, DriftPtMsState* state,
                                  void* stream);
/* n_rounds rounds of (sweeps_per_round checkerboard sweeps of all replicas, exact energy
 * recount, per-replica best update, adjacent-rung exchange). One persistent launch. */
DRIFT_PT_API int drift_pt_ms_run(const DriftPtLattice* lat, const DriftPtMsRunArgs* args, DriftPtMsState* state,
                                 void* workspace, size_t workspace_bytes, void* stream);

/* ---------------------------------------------------------------------------------------------
 * Graph multispin layer: +-1 couplings on any graph (max degree <= 7, no field), 32 replicas per
 * 32-bit word, one CTA (or a cluster of 2..16 CTAs) per word. No counterpart in the reference (its engine stores one float per
 * spin per replica, cuda/ising_pt.cu:190-191); the chain is the sparse layer's colour-ordered sweep
 * with a different uniform per attempt:
 *   positions: the colour order of drift_pt_color_order (class c = positions color_ptr[c] ..);
 *   bit b of word w at position p = replica slot 32w + b, 1 = spin -1;
 *   ell_nbr[d][p] (d < degree[p]): neighbour positions; jneg[p] bit d set when that bond's J = -1;
 *   a flip with k unsatisfied bonds has dE = 2 (deg - 2k); accepted when deg - 2k <= 0, else
 *   when u < thr[rung][deg - 2k - 1] (drift_pt_thresholds with max_field = max degree), u the
 *   32-bit number whose bit 31-q is bit b of plane q, plane q = word (q & 3) of
 *   Philox((p, t, (w << 8) | (q >> 2), 10 << 24 | instance), seed);
 *   initial word = word 0 of Philox((p, 0, w, 11 << 24 | instance), seed);
 *   energies exact: E = 2 U - bonds, U = unsatisfied bonds.
 * ------------------------------------------------------------------------------------------- */
#define DRIFT_PT_GMS_MAX_DEGREE 7

typedef struct DriftPtGmsProblem { /* device arrays */
  int32_t n, n_pos, n_colors, max_degree;
  int64_t n_bonds;
  int32_t max_class;         /* size of the largest colour class                              */
  int32_t reserved;
  const int32_t* color_ptr;  /* [k+1] position ranges of the colour classes                  */
  const int32_t* ell_nbr;    /* [max_degree][n_pos]                                           */
  const uint8_t* degree;     /* [n_pos] (0 for padding)                                       */
  const uint8_t* jneg;       /* [n_pos]                                                       */
} DriftPtGmsProblem;

typedef struct DriftPtGmsLayoutInfo {
  int32_t n, n_pos, n_colors, max_degree;
  int64_t n_bonds;
  int32_t max_class;         /* size of the largest colour class                              */
  int32_t reserved;
} DriftPtGmsLayoutInfo;

typedef struct DriftPtGmsLayout { /* caller-allocated host arrays sized from the info */
  int32_t* color_ptr;        /* [k+1]                                                         */
  int32_t* ell_nbr;          /* [max_degree][n_pos]                                           */
  uint8_t* degree;           /* [n_pos]                                                       */
  uint8_t* jneg;             /* [n_pos]                                                       */
  int32_t* pos_of_site;      /* [n]                                                           */
  int32_t* site_of_pos;      /* [n_pos] (-1 for padding)                                      */
} DriftPtGmsLayout;

typedef struct DriftPtGmsState { /* device arrays; R = 32 * n_words */
  uint32_t* words;           /* [W][n_pos]                                                    */
  uint32_t* best_words;      /* [W][n_pos]                                                    */
  int64_t* energy;           /* [R]                                                           */
  int64_t* best_energy;      /* [R]                                                           */
  int32_t* rung_of_slot;     /* [R]                                                           */
  int32_t* slot_of_rung;     /* [R]                                                           */
  int64_t* swap_tried;       /* [R-1]                                                         */
  int64_t* swap_accepted;    /* [R-1]                                                         */
} DriftPtGmsState;

typedef struct DriftPtGmsRunArgs {
  int32_t n_words;           /* W: replicas R = 32 W                                          */
  int32_t n_rounds, sweeps_per_round;
  int32_t threads_per_cta;   /* 0 = automatic                                                 */
  int64_t round_offset;
  uint64_t seed;
  uint32_t instance;
  int32_t cluster_size;      /* CTAs per word: 1 = one CTA holds the word; 2..16 = a cluster   */
                             /* splits it (shared-memory neighbour reads); 0 = automatic       */
  const double* betas;       /* [R] device                                                    */
  const uint32_t* thresholds;/* [R][max_degree] device, drift_pt_thresholds                   */
  double timeout_s;
} DriftPtGmsRunArgs;

/* Host: check that every coupling is +-1 and h = 0, and size the layout (colour order of `csr`). */
DRIFT_PT_API int drift_pt_gms_layout_query(const DriftPtCsr* csr, DriftPtGmsLayoutInfo* info);
DRIFT_PT_API int drift_pt_gms_layout_fill(const DriftPtCsr* csr, DriftPtGmsLayout* out);
DRIFT_PT_API int drift_pt_gms_workspace_bytes(int32_t n_words, size_t* bytes);
/* Random initial words, exact energies, best = initial, identity rungs, zero counts. */
DRIFT_PT_API int drift_pt_gms_init(const DriftPtGmsProblem* problem, const DriftPtGmsRunArgs* args,
                                   DriftPtGmsState* state, void* stream);
/* n_rounds rounds in one persistent launch; the state lives in shared memory for the whole launch.
 * cluster_size 1: one CTA per word; 2..16: the word's positions split over a cluster (neighbour words
 * read from the owning CTA's shared memory; same bits as cluster_size 1); 0: 1 from 16 words up, else
 * the largest cluster the GPU holds resident for all words. Shapes that cannot be co-resident are
 * refused with DRIFT_PT_EUNSUPPORTED. Bit-identical to any other cluster_size and to a split of the
 * rounds over several calls (round_offset). */
DRIFT_PT_API int drift_pt_gms_run(const DriftPtGmsProblem* problem, const DriftPtGmsRunArgs* args,
                                  DriftPtGmsState* state, void* workspace, size_t workspace_bytes, void* stream);

/* ---------------------------------------------------------------------------------------------
 * Dense layer: fully connected couplings (Sherrington-Kirkpatrick type), n <= 512, R <= 512.
 * The reference runs such models through the same CSR kernel as sparse ones
 * (cuda/ising_pt.cu:109-122): every spin is its own colour class and each attempt walks n - 1
 * neighbours. Here the chain keeps every replica's local fields F = J s + h exact in integer
 * fixed point and updates them on the tensor cores.
 *   Couplings: Jq = rint(J 2^shift), hq = rint(h 2^shift) (int32), shift chosen by
 *   drift_pt_sk_quantize so that |Jq| < 2^23 - 2^16 and every |F| < 2^30.
 *   Sweep: spins 0..n-1 in order; spin i flips iff s_i F_i <= D, D = floor(-ln(u) scale[rung])
 *   with scale[rung] = float(2^shift / (2 beta_rung)) (drift_pt_sk_scales) and u from word
 *   ((i >> 5) & 3) of Philox(((i >> 7) << 5 | (i & 31), t, slot, 7 << 24 | instance)).
 *   Energies are exact int64 in units of 2^-(shift+1): E2 = -sum_i s_i (sum_j Jq_ij s_j + 2 hq_i).
 *   Rounds, best tracking and the adjacent-rung exchange are those of drift_pt_run (the exchange
 *   uses E = E2 2^-(shift+1)).
 * Device coupling table: drift_pt_sk_layout_fill writes, for every block of 32 spins, the 24-bit
 * couplings of those 32 columns as three int8 limbs (Jq = d0 + 2^8 d1 + 2^16 d2, each in
 * [-128, 127]) in the tensor cores' shared-memory operand layout, followed by two 32 x 32 int32
 * blocks: the diagonal block and the couplings to the previous block of the sweep.
 * ------------------------------------------------------------------------------------------- */
#define DRIFT_PT_SK_MAX_N 512
#define DRIFT_PT_SK_MAX_R 512

typedef struct DriftPtSkProblem {
  int32_t n;
  int32_t shift;
  const int32_t* Jq;         /* device [n][n] symmetric, zero diagonal                       */
  const int32_t* hq;         /* device [n]                                                   */
  const void* layout;        /* device, drift_pt_sk_layout_bytes(n) bytes                    */
} DriftPtSkProblem;

typedef struct DriftPtSkState { /* device arrays */
  int8_t* spins;             /* [R][n] +-1, natural spin order                               */
  int8_t* best_spins;        /* [R][n]                                                       */
  int64_t* energy;           /* [R] E2 (units 2^-(shift+1))                                  */
  int64_t* best_energy;      /* [R]                                                          */
  int32_t* rung_of_slot;     /* [R]                                                          */
  int32_t* slot_of_rung;     /* [R]                                                          */
  int64_t* swap_tried;       /* [R-1]                                                        */
  int64_t* swap_accepted;    /* [R-1]                                                        */
  int64_t* best_history;     /* [n_rounds] or NULL: lowest E2 seen up to each round          */
} DriftPtSkState;

typedef struct DriftPtSkRunArgs {
  int32_t n_replicas;
  int32_t n_rounds, sweeps_per_round;
  int32_t replicas_per_cta;  /* 1..12; 0 = automatic                                        */
  int64_t round_offset;
  uint64_t seed;
  uint32_t instance;
  int32_t reserved;
  const double* betas;       /* [R] device                                                   */
  const float* scales;       /* [R] device, drift_pt_sk_scales                               */
  double timeout_s;
} DriftPtSkRunArgs;

/* Host: choose shift and quantise (J [n][n] symmetric with zero diagonal, h [n] or NULL). */
DRIFT_PT_API int drift_pt_sk_quantize(int32_t n, const double* J, const double* h, int32_t* Jq, int32_t* hq,
                                      int32_t* shift);
DRIFT_PT_API int drift_pt_sk_layout_bytes(int32_t n, size_t* bytes);
DRIFT_PT_API int drift_pt_sk_layout_fill(int32_t n, const int32_t* Jq, void* layout);
/* Host: scale[r] = float(2^shift / (2 betas[r])). */
DRIFT_PT_API int drift_pt_sk_scales(int32_t n_replicas, const double* betas, int32_t shift, float* scales);
DRIFT_PT_API int drift_pt_sk_workspace_bytes(int32_t n_replicas, size_t* bytes);
/* Random initial spins (the Philox init of drift_pt_init, in natural order), exact energies,
 * best = initial, identity rungs, zero exchange counts. */
DRIFT_PT_API int drift_pt_sk_init(const DriftPtSkProblem* problem, const DriftPtSkRunArgs* args,
                                  DriftPtSkState* state, void* stream);
/* n_rounds rounds in one persistent launch. */
DRIFT_PT_API int drift_pt_sk_run(const DriftPtSkProblem* problem, const DriftPtSkRunArgs* args,
                                 DriftPtSkState* state, void* workspace, size_t workspace_bytes, void* stream);
/* Exact E2 of R configurations [R][n] (check). */
DRIFT_PT_API int drift_pt_sk_energy(const DriftPtSkProblem* problem, int32_t n_replicas, const int8_t* spins,
                                    int64_t* energy, void* stream);

/* ---------------------------------------------------------------------------------------------
 * Tensor-core GEMM for the proposal network (no counterpart in the reference, which has no
 * learned component): C[m][n] = epi(sum_k A[m][k] B[n][k]) with A [M][lda] and B [N][ldb] bf16,
 * K contiguous, FP32 accumulation in tensor memory. epi: + bias[n] (optional), then ReLU (act = 1)
 * or, when relu_ref is given, a multiply by (relu_ref[m][n] > 0) (relu_ref [M][ldc] bf16); the
 * result is stored to out_f32 and / or out_bf16 ([M][ldc]). K, lda, ldb multiples of 8; A and B
 * 16-byte aligned. error_flag (device int, may be NULL) is set to DRIFT_PT_ETIMEOUT if a bounded
 * wait inside the kernel gives up.
 * ------------------------------------------------------------------------------------------- */
typedef struct DriftPtGemm {
  int32_t M, N, K, lda, ldb, ldc, act, reserved;
  const void* A;             /* bf16 [M][lda]                                                */
  const void* B;             /* bf16 [N][ldb]                                                */
  const float* bias;         /* [N] or NULL                                                  */
  const void* relu_ref;      /* bf16 [M][ldc] or NULL                                        */
  float* out_f32;            /* [M][ldc] or NULL                                             */
  void* out_bf16;            /* bf16 [M][ldc] or NULL                                        */
} DriftPtGemm;

DRIFT_PT_API int drift_pt_gemm_bf16(const DriftPtGemm* gemm, int32_t* error_flag, void* stream);

/* ---------------------------------------------------------------------------------------------
 * Proposal network (no counterpart in the reference): a masked autoregressive MLP over n spins,
 * q(x) = prod_i sigma(x_i l_i(x_<i)), l = W3 relu(W2 relu(W1 x + b1) + b2) + b3, with the masks of
 * unit degrees (input i: degree i+1; hidden degrees 1..n-1; W1[k][i] kept iff m1(k) >= i+1,
 * W2[k'][k] iff m2(k') >= m1(k), W3[i][k'] iff i+1 > m2(k')). Training kernels (element-wise parts;
 * the products are drift_pt_gemm_bf16):
 * ------------------------------------------------------------------------------------------- */
/* logq[b] = sum_i log sigma(x_i l_i); dlogits = -scale x sigma(-x l) (bf16, may be NULL). */
DRIFT_PT_API int drift_pt_made_loss(int32_t batch, int32_t n, const float* logits, const int8_t* x, float* logq,
                                    void* dlogits_bf16, float scale, void* stream);
DRIFT_PT_API int drift_pt_made_spins_to_bf16(int64_t count, const int8_t* x, void* out_bf16, void* stream);
DRIFT_PT_API int drift_pt_transpose_bf16(int32_t rows, int32_t cols, const void* in, void* out, void* stream);
DRIFT_PT_API int drift_pt_colsum_bf16(int32_t rows, int32_t cols, const void* in, float* out, void* stream);
/* Adam (bias-corrected, step >= 1) on a [rows][cols] fp32 tensor; entries with mask 0 are held at 0.
 * With w_bf16 / wt_bf16 it also writes the bf16 copy and its transpose. */
DRIFT_PT_API int drift_pt_adam(int32_t rows, int32_t cols, float* w, const float* g, float* m, float* v,
                               const uint8_t* mask, float lr, float beta1, float beta2, float eps, int32_t step,
                               void* w_bf16, void* wt_bf16, void* stream);

typedef struct DriftPtMadeNet { /* device arrays */
  int32_t n, h1, h2;
  int32_t max_units_per_degree; /* <= 4                                                        */
  const void* w1t;           /* bf16 [n][h1]  (W1 transposed, masked)                        */
  const void* w2t;           /* bf16 [h1][h2]                                                */
  const void* w3t;           /* bf16 [h2][n]                                                 */
  const float* b1;           /* [h1]                                                         */
  const float* b2;           /* [h2]                                                         */
  const float* b3;           /* [n]                                                          */
  const int32_t* ord1;       /* [h1] first-layer units sorted by degree                      */
  const int32_t* off1;       /* [n+1] units of degree d at ord1[off1[d-1] .. off1[d])         */
  const int32_t* ord2;       /* [h2]                                                         */
  const int32_t* off2;       /* [n+1]                                                        */
} DriftPtMadeNet;

/* mode 0: draw count configurations x [count][n] (+-1) from q with Philox(i, sample, stream_id,
 * 8 << 24; seed) and return log q of each; mode 1: log q of the given x. Both walk the spins in
 * order and accumulate every sum in one fixed order, so the log q of a drawn x equals its
 * mode-1 value exactly. No counterpart in the reference (it has no learned component). */
DRIFT_PT_API int drift_pt_made_sample(const DriftPtMadeNet* net, int32_t count, int32_t mode, int8_t* x,
                                      float* logq, uint64_t seed, uint32_t stream_id, void* stream);

/* Exact Metropolis-Hastings step for whole-configuration proposals on the dense layer's state:
 * slot s (if active[s], or all when active is NULL) takes proposal x' with probability
 * min(1, exp(-beta_rung (E' - E)) q(x) / q(x')), log of the ratio in double from the exact int64
 * energies (units 2^-(shift+1)) and the fp32 log q values; uniform from
 * Philox(slot, round lo, round hi, 9 << 24 | instance; seed). Counts per rung in prop_tried /
 * prop_accepted [R]; an accepted proposal below the slot's best also becomes its best. */
/* Conditional proposals: for each of the count configurations in x [count][n], keep spins
 * 0 .. keep-1 and draw spins keep .. n-1 from q's conditionals given them (uniforms as in mode 0);
 * x is overwritten with the result and logq receives its full log q, bit-identical to mode 1 on the
 * result. A Metropolis-Hastings test with this proposal uses q(x) / q(x') exactly like an
 * independent draw, because the kept spins' factors of q cancel. No counterpart in the reference. */
DRIFT_PT_API int drift_pt_made_sample_suffix(const DriftPtMadeNet* net, int32_t count, int32_t keep, int8_t* x,
                                             float* logq, uint64_t seed, uint32_t stream_id, void* stream);

DRIFT_PT_API int drift_pt_made_mh(const DriftPtSkProblem* problem, const DriftPtSkRunArgs* args, DriftPtSkState* state,
                                  const int8_t* proposals, const int64_t* prop_energy, const float* logq_prop,
                                  const float* logq_cur, const uint8_t* active, int64_t* prop_tried,
                                  int64_t* prop_accepted, int64_t round, void* stream);

/* Several proposal networks in one launch (a batch of instances with one network each). The group
 * table (drift_pt_made_group_bytes(n_nets) bytes of device memory, opaque) is filled once, synchronously,
 * from the networks, their sample counts, their output buffers x[g] ([counts[g]][n_g] int8, site
 * order) and logq[g] ([counts[g]] fp32), and a mode (0: draw, 1: evaluate the given x). Each
 * drift_pt_made_group_run then runs network g exactly as drift_pt_made_sample would with
 * stream_id[g] + stream_add, on blocks (., g) of one launch; max_* bound every network's sizes.
 * No counterpart in the reference (learned proposals are this engine's own). */
DRIFT_PT_API int drift_pt_made_group_bytes(int32_t n_nets, size_t* bytes);
DRIFT_PT_API int drift_pt_made_group_fill(int32_t n_nets, const DriftPtMadeNet* nets, const int32_t* counts,
                                          int32_t mode, int8_t* const* x, float* const* logq, uint64_t seed,
                                          const uint32_t* stream_id, void* table);
DRIFT_PT_API int drift_pt_made_group_run(const void* table, int32_t n_nets, int32_t max_count, int32_t max_n,
                                         int32_t max_h1, int32_t max_h2, uint32_t stream_add, void* stream);

/* ---------------------------------------------------------------------------------------------
 * Whole-configuration proposals on a batch (integer path). Request j names rung rung[j] of
 * instance instance[j]; requests of one call name distinct (instance, rung) pairs. Site i of
 * instance k is position pos_of_site[site_off[k] + i] of its layout (the DriftPtLayout
 * pos_of_site arrays of the batch's instances, concatenated).
 * ------------------------------------------------------------------------------------------- */
/* Copy the configuration at each requested rung, in site order, to out + out_off[j] +
 * rep * out_step[j] (out_step may be NULL). */
DRIFT_PT_API int drift_pt_batch_gather(const DriftPtBatchProblem* prob, const DriftPtDeviceState* state, int32_t count,
                                       const int32_t* instance, const int32_t* rung, const int64_t* site_off,
                                       const int32_t* pos_of_site, const int64_t* out_off, const int64_t* out_step,
                                       int64_t rep, int8_t* out, int32_t* error_flag, void* stream);
/* Exact Metropolis-Hastings step for independent proposals x'_j (site order, at proposals +
 * prop_off[j]): the energy E' is recomputed exactly from the instance's layout, and x'_j replaces
 * the configuration at (instance, rung) with probability min(1, exp(-beta (E' - E)) q(x) / q(x')),
 * the log of the ratio in double from the exact energies and the fp32 log q values, the uniform
 * from Philox((rung, round lo, round hi, 12 << 24 | stream id of the instance); seed). An accepted
 * proposal below the slot's best also becomes its best. prop_tried / prop_accepted [count] are
 * incremented per request; prop_energy [count] (may be NULL) receives E'. scratch: count *
 * max_n_pos bytes. Out-of-range requests set *error_flag = DRIFT_PT_EINVAL and are skipped. No
 * counterpart in the reference (the exact MH test for learned proposals is this engine's own). */
DRIFT_PT_API int drift_pt_batch_mh(const DriftPtBatchProblem* prob, DriftPtDeviceState* state, uint64_t seed,
                                   int32_t count, const int32_t* instance, const int32_t* rung, const int64_t* site_off,
                                   const int32_t* pos_of_site, const int64_t* prop_off, const int8_t* proposals,
                                   const float* logq_prop, const float* logq_cur, int64_t round, int8_t* scratch,
                                   int64_t* prop_energy, int64_t* prop_tried, int64_t* prop_accepted,
                                   int32_t* error_flag, void* stream);

/* ---------------------------------------------------------------------------------------------
 * Host convenience: one call from host buffers to host results (the problem.bin -> result.bin
 * contract of cuda/ising_pt.cu:159-243 and drift/gpu.py:83-114). Allocates and frees device
 * memory internally; synchronous.
 * ------------------------------------------------------------------------------------------- */
typedef struct DriftPtSolveArgs {
  int32_t n_replicas;
  int32_t n_rounds;
  int32_t sweeps_per_round;
  int32_t reserved0;
  uint64_t seed;
  double T_min, T_max;       /* geometric ladder (drift/solvers/parallel_tempering.py:29-36) */
  const double* betas;       /* optional explicit ladder [R] (host), overrides T_min/T_max  */
} DriftPtSolveArgs;

typedef struct DriftPtSolveResult { /* caller-allocated host buffers; optional ones may be NULL */
  double best_E;
  double seconds;            /* device time of the round loop                               */
  double throughput;         /* attempts per second = R * n_rounds * sweeps * n / seconds   */
  double swap_rate;          /* accepted / tried over all exchange attempts                 */
  float* best_s;             /* [n] +-1 of the lowest-energy configuration seen             */
  int8_t* rung_spins;        /* [R][n] optional: final configuration at each rung           */
  double* rung_energy;       /* [R] optional: final energy at each rung                     */
  int64_t* swap_tried;       /* [R-1] optional                                              */
  int64_t* swap_accepted;    /* [R-1] optional                                              */
  double* best_history;      /* [n_rounds] optional                                         */
} DriftPtSolveResult;

DRIFT_PT_API int drift_pt_solve(const DriftPtCsr* csr, const DriftPtSolveArgs* args, DriftPtSolveResult* out);

/* Frees the device arena drift_pt_solve keeps on the calling thread between calls (it is grown as
 * calls need and otherwise freed when the thread exits). No counterpart in the reference, whose
 * subprocess boundary frees everything with the process. */
DRIFT_PT_API int drift_pt_solve_release(void);

#ifdef __cplusplus
}
#endif
#endif /* DRIFT_PT_H */
