/*
 * nbl_b200.h -- C-ABI of the B200 neighbour-list engine.
 *
 * The engine is a drop-in for the device path of matscipy-neighbours'
 * `neighbour_list(quantities, positions, cell, pbc, cutoff)`.  Every entry
 * point takes plain pointers and sizes, returns an nbl_status and never aborts
 * the process; on failure a thread-local message is available from
 * nbl_last_error().  No torch (or other framework) type appears here.
 *
 * Reference interfaces replaced (paths inside the reference project):
 *   - NeighbourListRequest           src/libneighbours/neighbour_list_gpu.hh:49-65
 *       -> nbl_request
 *   - neighbour_list_gpu_device()    src/libneighbours/neighbour_list_gpu.hh:95-96
 *       -> nbl_neighbour_list_device() (and the two-phase nbl_count/nbl_fill)
 *   - neighbour_count_gpu_device()   src/libneighbours/neighbour_list_gpu.hh:101-102
 *       -> nbl_count + nbl_counts
 *   - neighbour_list_gpu() (host in, host out)
 *                                    src/libneighbours/neighbour_list_gpu.hh:28-34
 *       -> nbl_count + nbl_fill_host (host positions, host outputs)
 *   - error_t / has_error / error_string
 *                                    src/libneighbours/types.hh:32-34,
 *                                    src/libneighbours/error.hh:27-33
 *       -> nbl_status + nbl_last_error()
 *   - Quantity flags                 src/libneighbours/types.hh:38-44
 *       -> NBL_QUANTITY_* (same bit values)
 *   - _has_gpu / _device_type        language_bindings/python/module.c:104-113
 *       -> nbl_has_gpu() / nbl_device_type()
 *
 * Output contract (identical to the reference CPU path, neighbour_list.cc:
 * 40-95): pairs sorted by i, and within one i in the reference's traversal
 * order; D (npairs x 3, row-major) satisfies D == r[j] - r[i] + S @ cell;
 * d = |D| correctly rounded; i, j, S are int32; D, d are float64.
 */
#ifndef NBL_B200_H
#define NBL_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define NBL_API __attribute__((visibility("default")))
#else
#define NBL_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum nbl_status {
    NBL_SUCCESS = 0,
    NBL_ERROR_INVALID_ARGUMENT = 1, /* bad sizes / pointers / flags          */
    NBL_ERROR_ZERO_VOLUME = 2,      /* "Zero cell volume." (cell_list.cc:161) */
    NBL_ERROR_RANGE = 3,            /* non-finite position, or an atom more
                                       than 2^29 cells outside the box        */
    NBL_ERROR_OUT_OF_MEMORY = 4,
    NBL_ERROR_CUDA = 5,             /* a CUDA runtime error (message says which) */
    NBL_ERROR_CAPACITY = 6,         /* output capacity smaller than the pair
                                       count (batched / graph path); retry     */
    NBL_ERROR_NO_DEVICE = 7,
    NBL_ERROR_INTERNAL = 8          /* a device-side bound was hit (never
                                       expected; reported instead of hanging)  */
} nbl_status;

/* Quantity bits, same values as matscipy::Quantity (types.hh:38-44). */
#define NBL_QUANTITY_FIRST 1   /* i */
#define NBL_QUANTITY_SECOND 2  /* j */
#define NBL_QUANTITY_DISTVEC 4 /* D */
#define NBL_QUANTITY_ABSDIST 8 /* d */
#define NBL_QUANTITY_SHIFT 16  /* S */

/* Cell grid layout.  All produce identical output; they differ in memory
   layout and lookup only (the reference's CellOrder Linear/Morton,
   cell_list.hh:25, and its dense/sparse backends, cell_list.cc:184-203). */
typedef enum nbl_grid {
    NBL_GRID_AUTO = 0,   /* dense, or hashed when the grid is far larger than
                            the atom count (the reference's own rule)      */
    NBL_GRID_DENSE = 1,  /* dense table, cells in linear (z-major) order   */
    NBL_GRID_MORTON = 2, /* dense table, atoms laid out in Morton order    */
    NBL_GRID_HASHED = 3  /* hashed compact table of occupied cells only    */
} nbl_grid;

/* Candidate-test precision.  Both give the reference's exact pair set and
   bit-identical D and d; FP32_FILTER rejects most candidates in FP32 and
   re-tests only those inside a rigorous guard band of the cutoff in FP64. */
typedef enum nbl_precision {
    NBL_PRECISION_FP32_FILTER = 0,
    NBL_PRECISION_FP64 = 1
} nbl_precision;

/* One system.  Mirrors NeighbourListRequest (neighbour_list_gpu.hh:49-65).
   Geometry arrays are host memory.  `pbc` entries are 0/1 bytes. */
typedef struct nbl_request {
    int quantities;                    /* NBL_QUANTITY_* bits                 */
    const double *cell_origin;         /* [3]                                 */
    const double *cell;                /* [9] row-major, rows = lattice vectors */
    const double *inv_cell;            /* [9] inv(cell.T): inv_cell . r = frac */
    const uint8_t *pbc;                /* [3]                                 */
    int64_t nat;
    const double *positions;           /* [3*nat] row-major                   */
    int positions_on_device;           /* 1: device pointer, used in place    */
    double cutoff;                     /* binning / global cutoff             */
    const double *per_atom_cutoff;     /* [nat] radii (pair cutoff = sum) or NULL */
    const double *per_type_cutoff_sq;  /* [ncutoffs^2] host, squared, or NULL */
    int32_t ncutoffs;
    const int32_t *types;              /* [nat] or NULL                       */
    int aux_on_device;                 /* per_atom_cutoff / types on device   */
    int grid;                          /* nbl_grid                            */
    int precision;                     /* nbl_precision                       */
    int device_id;                     /* -1: current device                  */
} nbl_request;

/* Output buffers for one fill.  NULL skips a quantity.  Device pointers for
   nbl_fill, host pointers for nbl_fill_host.  Each must hold npairs entries
   (distvec and shift 3*npairs). */
typedef struct nbl_outputs {
    int32_t *first;
    int32_t *second;
    double *distvec;
    double *absdist;
    int32_t *shift;
} nbl_outputs;

/* Opaque state: device workspace reused across calls, plus the result of the
   last count phase.  A plan belongs to one device; calls on one plan must not
   overlap (use one plan per host thread). */
typedef struct nbl_plan nbl_plan;

NBL_API nbl_status nbl_plan_create(int device_id, nbl_plan **plan);
NBL_API nbl_status nbl_plan_destroy(nbl_plan *plan);
/* Releases the plan's device workspace (it is re-grown on the next call). */
NBL_API nbl_status nbl_plan_trim(nbl_plan *plan);

/* Row split: later nbl_count / nbl_fill calls on this plan produce only the
   rows i with lo <= i < hi (original atom indices; every atom stays a
   candidate j).  The pair count and the output are then exactly the slice
   [offsets[lo], offsets[hi]) of the full list, so ranks that each take one
   contiguous range reproduce the full list by concatenation.  hi < 0 means
   "to the end"; lo = 0, hi = -1 restores the full list.  The range takes
   effect at the next nbl_count, and a fill always uses its count's range, so
   it may be reset between the two.  No reference
   counterpart: the reference builds one list per process
   (src/libneighbours/neighbour_list.cc:99-204). */
NBL_API nbl_status nbl_set_atom_range(nbl_plan *plan, int64_t lo, int64_t hi);

/* Launch configuration of the plan's pair passes: CTAs per SM of the count
   and fill grids (0: two full waves of the kernel's resident CTAs, the
   default) and atoms per sweep in the FP32 count (2 or 4; 0 keeps 4).  Takes
   effect at the next nbl_count.  A tuning knob with no effect on results.  No
   reference counterpart (the reference's core is serial per cell,
   src/libneighbours/neighbour_list.cc:99-204). */
NBL_API nbl_status nbl_plan_set_launch(nbl_plan *plan, int count_ctas_per_sm, int count_group,
                                       int fill_ctas_per_sm);

/* The full launch configuration of the pair passes (what the batch
   autotuner chooses; a single call uses the defaults unless set here).  Every
   value gives bit-identical output.  Zero fields mean the default.
     count_ctas_per_sm, fill_ctas_per_sm  grid of each pass (0: two waves of
                                          its resident CTAs), <= 64
     count_strided, fill_strided          work items by a fixed warp stride
                                          (1) instead of by atomic ticket (0)
     count_warps, fill_warps              block size: 2, 4 or 8 warps
                                          (64, 128 or 256 threads; default
                                          4 for the count, 8 for the fill)
     count_group                          atoms per FP32 sweep: 2 or 4 (4)
     count_large_staging                  candidates staged per count warp:
                                          0 = 384 (FP32) / 192 (FP64),
                                          1 = 768 / 384
     atoms_per_item                       cell-occupancy tile: atoms of one
                                          cell per work item, 1..32; 0 = by
                                          the atom count: 4 up to 4,096
                                          atoms, 8 up to 16,384, 16 up to
                                          65,536, else 32
     cells_per_item                       home cells one work item may join
                                          along x when their atoms fit one
                                          tile: 0 = chosen on the device from
                                          the mean cell occupancy (sparse
                                          grids join up to 8), 1 = one cell
                                          per item, 2..8 = at most that many
                                          (dense grid and FP32 filter only)
     one_launch_atoms                     systems of up to this many atoms
                                          (one system, dense grid of at most
                                          16,384 cells) run the whole count
                                          phase as one launch (one CTA up to
                                          128 atoms, else a thread-block
                                          cluster of up to 8 CTAs):
                                          0 = the default, -1 = never, 1..2048
     thread_per_atom                      pair passes with one thread per atom
                                          instead of one warp per work item:
                                          0 = where the occupied cells hold
                                          fewer than two atoms on average
                                          (known after a first count of the
                                          same sizes; before it, fewer atoms
                                          than cells), -1 =
                                          never, 1 = always (systems with a
                                          visit table: at most 2^20 visited
                                          offsets in all); the force sink
                                          always uses work items
   No reference counterpart (the reference has no tuner). */
typedef struct nbl_launch_config {
    int count_ctas_per_sm;
    int fill_ctas_per_sm;
    int count_strided;
    int fill_strided;
    int count_warps;
    int fill_warps;
    int count_group;
    int count_large_staging;
    int atoms_per_item;
    int cells_per_item;
    int one_launch_atoms;
    int thread_per_atom;
} nbl_launch_config;

NBL_API nbl_status nbl_plan_set_launch_config(nbl_plan *plan, const nbl_launch_config *cfg);
NBL_API nbl_status nbl_plan_get_launch_config(nbl_plan *plan, nbl_launch_config *cfg);

/* Count phase: bins the atoms, counts every atom's neighbours and scans the
   counts into row offsets.  Host positions are copied in on `stream`.
   Synchronises `stream` to return the pair count. */
NBL_API nbl_status nbl_count(nbl_plan *plan, const nbl_request *req, void *stream,
                     int64_t *npairs);

/* Fill phase for the last nbl_count: writes the requested quantities into
   caller-allocated device buffers, asynchronously on `stream`. */
NBL_API nbl_status nbl_fill(nbl_plan *plan, const nbl_outputs *out, void *stream);

/* Fill into HOST buffers: fills device scratch owned by the plan and copies
   each requested quantity back; returns after the copies complete. */
NBL_API nbl_status nbl_fill_host(nbl_plan *plan, const nbl_outputs *host_out,
                         void *stream);

/* Synchronises `stream` and reports any error the device flagged during the
   last count/fill (capacity overflow, internal bound); NBL_SUCCESS if none. */
NBL_API nbl_status nbl_check(nbl_plan *plan, void *stream);

/* Per-atom neighbour counts (coordination numbers, original atom order) of
   the last nbl_count, into a device int32[nat] buffer, on `stream`.
   (neighbour_count_gpu_device, neighbour_list_gpu.hh:101-102.) */
NBL_API nbl_status nbl_counts(nbl_plan *plan, int32_t *counts, void *stream);

/* Dense fixed-capacity neighbour matrix of the last nbl_count
   (neighbour_matrix_gpu_device, neighbour_list_gpu.hh:112-123): row a of the
   device buffers idx [nat*K] int32 and dist [nat*K*3] float64 holds atom a's
   first min(count[a], K) neighbours (j and D) in the reference's row order;
   unused slots are 0; count [nat] int32 holds the full degree.  *overflow
   (host int) is set to 1 when some atom has more than K neighbours.
   Synchronises `stream`. */
NBL_API nbl_status nbl_fill_matrix(nbl_plan *plan, int32_t max_neighbours,
                                   int32_t *idx, double *dist, int32_t *count,
                                   int *overflow, void *stream);

/* Row offsets (exclusive prefix of the counts, int64[nat+1], device) of the
   last nbl_count, on `stream`: row i of the pair list is [off[i], off[i+1]). */
NBL_API nbl_status nbl_row_offsets(nbl_plan *plan, int64_t *offsets, void *stream);

/* One-shot device entry (neighbour_list_gpu_device): the library allocates
   the outputs with stream-ordered allocation on `stream`; release them with
   nbl_device_result_free on a stream ordered after their last use. */
typedef struct nbl_device_result {
    int64_t npairs;
    int32_t *first;
    int32_t *second;
    double *distvec;
    double *absdist;
    int32_t *shift;
    int device_id;
} nbl_device_result;

NBL_API nbl_status nbl_neighbour_list_device(const nbl_request *req, void *stream,
                                     nbl_device_result *result);
NBL_API nbl_status nbl_device_result_free(nbl_device_result *result, void *stream);

/* ---- batches: many independent systems, one launch sequence --------------
   (Build-only form with no reference counterpart: the reference handles one
   system per call, neighbour_list_gpu.hh:95-96.)  Each system has its own
   cell, pbc and cutoff; atoms are concatenated system after system.  Outputs
   are concatenated too: the pairs of system s are [sys_offsets[s],
   sys_offsets[s+1]) and their i, j are indices within system s. */
typedef struct nbl_system {
    const double *cell_origin;  /* [3] host */
    const double *cell;         /* [9] host, rows = lattice vectors */
    const double *inv_cell;     /* [9] host */
    const uint8_t *pbc;         /* [3] host */
    int64_t nat;
    double cutoff;              /* binning / global cutoff (per-atom: max 2r) */
} nbl_system;

typedef struct nbl_batch_request {
    int quantities;
    int32_t nsys;
    const nbl_system *systems;          /* host [nsys] */
    const double *positions;            /* [3*N] concatenated */
    int positions_on_device;            /* 0: copied once into the batch */
    const double *per_atom_cutoff;      /* [N] concatenated, or NULL */
    const int32_t *types;               /* [N] or NULL */
    const double *per_type_cutoff_sq;   /* [ncutoffs^2] host, shared, or NULL */
    int32_t ncutoffs;
    int aux_on_device;
    int grid;                           /* nbl_grid */
    int precision;                      /* nbl_precision */
    int autotune;                       /* 1: time launch configurations at set-up */
} nbl_batch_request;

typedef struct nbl_batch_outputs {
    int32_t *first;
    int32_t *second;
    double *distvec;
    double *absdist;
    int32_t *shift;
    int64_t *sys_offsets;               /* [nsys+1] pair offset of each system */
    int64_t capacity;                   /* pairs the output buffers hold */
    double *positions;                  /* device positions the batch reads */
} nbl_batch_outputs;

typedef struct nbl_batch nbl_batch;

NBL_API nbl_status nbl_batch_create(int device_id, nbl_batch **batch);
NBL_API nbl_status nbl_batch_destroy(nbl_batch *batch);
/* Plans every system, uploads the tables once and allocates device outputs for
   `capacity` pairs (<= 0: the exact count plus 25 % headroom).  Synchronous. */
NBL_API nbl_status nbl_batch_setup(nbl_batch *batch, const nbl_batch_request *req,
                                   int64_t capacity);
/* Enqueues the whole build on `stream` (NULL: the batch's own stream): no host
   synchronisation and no allocation, so it can be captured in a CUDA graph. */
NBL_API nbl_status nbl_batch_run(nbl_batch *batch, void *stream);
/* Captures nbl_batch_run into a CUDA graph (stream must not be the legacy
   default stream; NULL uses the batch's own stream). */
NBL_API nbl_status nbl_batch_capture(nbl_batch *batch, void *stream);
/* Replays the captured graph: one launch for the whole batch. */
NBL_API nbl_status nbl_batch_launch(nbl_batch *batch, void *stream);
/* Synchronises `stream`, returns the total pair count; NBL_ERROR_CAPACITY when
   it exceeds the capacity (outputs then hold only the pairs that fit). */
NBL_API nbl_status nbl_batch_finish(nbl_batch *batch, void *stream, int64_t *npairs);
NBL_API nbl_status nbl_batch_get_outputs(nbl_batch *batch, nbl_batch_outputs *out);
/* The launch configuration in use (chosen by the autotuner when enabled). */
NBL_API nbl_status nbl_batch_get_config(nbl_batch *batch, int *count_mult,
                                        int *count_group, int *fill_mult);
/* Whether the count and fill passes hand work items out by atomic ticket (1)
   or by a fixed warp stride (0), as the autotuner chose. */
NBL_API nbl_status nbl_batch_get_tickets(nbl_batch *batch, int *count_tickets,
                                         int *fill_tickets);
/* Everything the autotuner chose (nbl_launch_config above), and the median
   device times (ms) of the count phase and of the fill with that choice, as
   the autotuner measured them (0 when it did not run). */
NBL_API nbl_status nbl_batch_get_launch_config(nbl_batch *batch, nbl_launch_config *cfg,
                                               float *count_ms, float *fill_ms);

/* ---- backward: gradients through the pair list -------------------------
   (Build-only form with no reference counterpart.)  For a fixed pair list of
   one system, D = r_j - r_i + sum_m c_m cell[m] with c_m = S_m on periodic
   axes and 0 on non-periodic ones, and d = |D|.  Given dL/dD and/or dL/dd,
   writes dL/dpositions [nat*3] and dL/dcell [9] (row-major, cell rows =
   lattice vectors).  All pointers are device pointers except pbc.  With
   deterministic != 0 the result is bit-reproducible (the j-side is reduced
   after a stable sort by j instead of with atomics). */
typedef struct nbl_backward_args {
    int64_t npairs;
    int64_t nat;
    const int32_t *first;          /* [npairs], sorted (as the fill writes it) */
    const int32_t *second;         /* [npairs] */
    const int32_t *shift;          /* [3*npairs] */
    const double *distvec;         /* [3*npairs] (needed with grad_absdist) */
    const double *absdist;         /* [npairs]   (needed with grad_absdist) */
    const double *grad_distvec;    /* [3*npairs] or NULL */
    const double *grad_absdist;    /* [npairs] or NULL */
    const int64_t *row_offsets;    /* [nat+1] (nbl_row_offsets) or NULL */
    const uint8_t *pbc;            /* [3] host */
    double *grad_positions;        /* [3*nat] out */
    double *grad_cell;             /* [9] out */
    int deterministic;
} nbl_backward_args;

NBL_API nbl_status nbl_backward(const nbl_backward_args *args, void *stream);

/* ---- fused consumer: Lennard-Jones forces without a pair list ------------ */

/* Forces and energy of a truncated Lennard-Jones pair potential over the
   request's neighbour pairs, U = 4 eps ((sigma/r)^12 - (sigma/r)^6) for
   r < cutoff, computed inside the fill pass: no pair is written.  forces
   (device, 3 * nat doubles, original atom order) receives F_i = -dU/dr_i
   summed over the pairs of row i; *energy (device, one double) receives
   sum over pairs of U / 2 per directed pair, i.e. each unordered pair once.
   Asynchronous on `stream` (no host synchronisation): call nbl_check to see
   input errors.  The same pair set as nbl_count/nbl_fill, so the forces are
   those of the reference's pair list (lj_langevin_gpu.cu:59-74, the
   reference's example, with eps = sigma = 1 and atomics instead of row sums).
   The request's quantities are ignored. */
NBL_API nbl_status nbl_lj_forces(nbl_plan *plan, const nbl_request *req, double epsilon,
                                 double sigma, double *forces, double *energy,
                                 void *stream);

/* ---- list reuse across steps (Verlet list) ------------------------------- */

/* *out (device, one double) = max over the n atoms of |positions - reference|
   (device, n x 3 each), for the skin test of a reused list.  Asynchronous.
   No reference counterpart: the reference's MD example rebuilds its list
   every step (examples/lj_langevin/lj_langevin_gpu.cu:171-179). */
NBL_API nbl_status nbl_max_displacement(int64_t n, const double *positions,
                                        const double *reference, double *out, void *stream);

/* Refreshes a stored list (first, second, shift: device, built with a larger
   cutoff) at the current device positions: D = r_j - r_i + sum over periodic
   axes of S_m cell[m] (cell: host row-major 3x3, rows are lattice vectors;
   pbc: host[3]), d = |D|, and keeps the pairs with d < cutoff, in the stored
   order, into `out` (device; NULL members are skipped).  Sets *nkept
   (synchronises `stream`); NBL_ERROR_CAPACITY if `capacity` is too small;
   out == NULL only counts.  With capacity >= npairs the pairs are written
   before the one synchronisation (a single call per step).  No reference
   counterpart (see above). */
NBL_API nbl_status nbl_verlet_refresh(int64_t npairs, const int32_t *first,
                                      const int32_t *second, const int32_t *shift,
                                      const double *positions, const double *cell,
                                      const uint8_t *pbc, double cutoff,
                                      const nbl_outputs *out, int64_t capacity,
                                      int64_t *nkept, void *stream);

/* ---- CSR helpers of a pair list, on the device --------------------------- */

/* Row starts of an i-sorted pair list (all pointers device memory):
   seed[k], k in [0, n], is the first pair of atom k; -1 before the first atom
   with pairs, npairs after the last; an empty row gets the next row's start.
   Asynchronous on `stream`.  Replaces first_neighbours()
   (src/libneighbours/first_neighbours.cc:15-38). */
NBL_API nbl_status nbl_first_neighbours(int64_t n, int64_t npairs, const int32_t *first,
                                        int32_t *seed, void *stream);

/* Triplets of pairs sharing a first atom, from row starts first_i[nfirst]
   (device memory): for each row, every ordered (ij, ik), ij != ik, ij major;
   with absdist (device, may be NULL) only pairs with absdist < cutoff take
   part.  Sets *ntriplets (synchronises `stream`); writes ij/ik (device,
   `capacity` entries) when both are given, NBL_ERROR_CAPACITY if they are too
   short.  Call with ij = ik = NULL to size the outputs.  Replaces
   triplet_list() (src/libneighbours/triplet_list.cc:15-34). */
NBL_API nbl_status nbl_triplet_list(int64_t nfirst, const int32_t *first_i,
                                    const double *absdist, double cutoff, int32_t *ij,
                                    int32_t *ik, int64_t capacity, int64_t *ntriplets,
                                    void *stream);

/* Allocation-free variant of nbl_count + nbl_fill, for callers that cannot
   allocate device memory at call time (an MD loop that forbids allocation
   after start-up, a host whose pool allocator has reserved the device
   memory).  No counterpart in the reference.  All scratch lives in one static
   8 MiB __device__ array inside the library, held by every GPU that loads it
   until exit; at most NBL_NOALLOC_MAX_ATOMS atoms.  Inputs as in nbl_request
   (positions device or host); `out` holds caller-allocated DEVICE buffers of
   `capacity` pairs.  Sets *npairs and returns NBL_ERROR_CAPACITY (writing
   nothing) when npairs > capacity.  Synchronises `stream`: on return the
   outputs are written and the scratch is free again.  Calls overlapping on
   the GPU race on the shared scratch: serialise them.  The first call on a
   device resolves the scratch address (device must be current), caches it for
   the life of the process (one primary context per device is assumed: not
   valid across cudaDeviceReset) and should come before any stream capture. */
#define NBL_NOALLOC_MAX_ATOMS 32768
NBL_API nbl_status nbl_neighbour_list_noalloc(const nbl_request *req,
                                              const nbl_outputs *out,
                                              int64_t capacity, int64_t *npairs,
                                              void *stream);

/* Test hooks: failures made on the host, so that the error paths can be
   exercised without faulting a GPU.  No counterpart in the reference, whose
   device errors abort the process (src/libneighbours/device.hh:68-74).
     NBL_INJECT_ALLOC_FAILURES  the next `value` growths of a plan's device
                                workspace fail as if the device were out of
                                memory (nbl_count returns
                                NBL_ERROR_OUT_OF_MEMORY and keeps nothing);
     NBL_INJECT_HASH_CAPACITY   hashed grids get `value` slots (rounded up to a
                                power of two) instead of 2N+1 rounded up; 0
                                restores the default.  With fewer slots than
                                occupied cells the bounded probe gives up and
                                the count returns NBL_ERROR_INTERNAL.
   Process-wide; not for production use. */
#define NBL_INJECT_ALLOC_FAILURES 1
#define NBL_INJECT_HASH_CAPACITY 2
NBL_API nbl_status nbl_debug_inject(int what, int64_t value);

/* Last error message of the calling thread ("" if none). */
NBL_API const char *nbl_last_error(void);

/* Number of CUDA kernels this library launched from the calling thread since
   the last reset (reset when `reset` is non-zero). */
NBL_API long long nbl_launch_count(int reset);

/* 1 if a CUDA device is visible, else 0 (module.c:104-113 `_has_gpu`). */
NBL_API int nbl_has_gpu(void);
/* DLPack device type of the outputs: 2 (kDLCUDA). */
NBL_API int nbl_device_type(void);
/* Library version string. */
NBL_API const char *nbl_version(void);

#ifdef __cplusplus
}
#endif

#endif /* NBL_B200_H */
