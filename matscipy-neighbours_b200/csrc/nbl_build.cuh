// nbl_build.cuh -- argument blocks and launchers of the pair kernels.
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

#include "nbl_internal.cuh"

namespace nbl {

constexpr int kModeCount = 0;
constexpr int kModeFill = 1;

struct BinArgs {
    const SysDev *sys;
    const int64_t *sys_atom_base;
    int nsys;
    int grid;
    const double *positions;  // [3*natoms], concatenated systems
    int64_t natoms;
    uint32_t *keys;
    int32_t *vals;
    unsigned long long *hkey;
    unsigned long long hmask;
    int *err;
};

struct GatherArgs {
    const SysDev *sys;
    const int64_t *sys_atom_base;
    int nsys;
    int grid;
    const double *positions;
    const double *per_atom;   // [natoms] or null
    const int32_t *types;     // [natoms] or null
    int64_t natoms;
    const uint32_t *keys;     // sorted
    const int32_t *vals;      // sorted: global atom index
    int2 *table;
    double4 *pos64;
    float4 *pos32;
    int4 *aux;
    float *amax;              // [nsys], zeroed
    HomeCell *home;
    int *n_home;              // zeroed
};

struct TraverseArgs {
    const SysDev *sys;
    const VisitDev *visit;    // per-system visit tables (systems with visit_base >= 0)
    const HomeCell *home;
    const int *n_home;
    const WorkItem *items;    // work items: (home cell, tile of its sorted atoms)
    const int *n_items;
    int grid;
    const int2 *table;
    const unsigned long long *hkey;
    unsigned long long hmask;
    const double4 *pos64;
    const float4 *pos32;
    const int4 *aux;
    const float *amax;
    const float *pt32;        // per-type squared cutoffs, FP32
    const double *pt64;       // per-type squared cutoffs, FP64
    int64_t natoms;           // atoms of the batch (offsets[natoms] = pair total)
    int32_t *counts;          // COUNT: per global atom
    const int64_t *offsets;   // FILL: row starts per global atom (+1)
    int32_t *first;
    int32_t *second;
    double *distvec;
    double *absdist;
    int32_t *shift;
    int64_t capacity;
    // Dense-matrix sink (neighbour_matrix): when mat_k > 0 the fill pass writes
    // row (global atom index) a, slot s < mat_k of mat_idx / mat_dist instead
    // of the pair list, and mat_count[a] = row length.
    // Hit-mask pool: the count pass stores one 32-bit word per (atom,
    // 32-candidate chunk) for each (work item, segment batch) it can fit
    // (home_mask[item * kMaskBatches + batch] = first word, -1 if none); the
    // fill pass then reads the words instead of repeating the distance
    // sweep.  mask_pool == nullptr disables it.
    uint32_t *mask_pool;
    unsigned long long *mask_cursor;
    long long mask_cap;
    long long *home_mask;     // per (work item, segment batch < kMaskBatches)
    int32_t mat_k;
    int32_t *mat_idx;
    double *mat_dist;
    int32_t *mat_count;
    int *mat_overflow;
    // Force sink (lj_force != nullptr): instead of writing pairs, the fill
    // pass sums Lennard-Jones forces per atom i into lj_force[3 * atom] and
    // its energy share (1/2 U per pair of its row) into lj_energy[atom];
    // every in-range atom is written once.
    double *lj_force;
    double *lj_energy;
    double lj_eps4, lj_eps24, lj_sig2;
    int *err;
    // Rows produced: only atoms whose global index lies in [i_lo, i_hi) act
    // as i; every atom stays a candidate j.  Rows outside keep count 0.
    long long i_lo;
    long long i_hi;
    // Work-item ticket (one int, zeroed by launch_traverse before each pass):
    // each warp claims its next item with one atomic, so warps that drew
    // cheap items take more.  NULL: a fixed warp stride over the items.
    int *item_next;
    // Atoms per work item (the cell-occupancy tile, <= 32): the items were
    // cut by k_tiles with the same value.
    int itile;
    // Nonzero: *item_next is already zero (the count phase's init kernel
    // cleared it), so the launch skips its reset.
    int ticket_ready;
    // Nonzero: k_tiles may have joined home cells into runs (WorkItem::run),
    // so the pair passes use the instantiations that take them.
    int runs;
    // Nonzero: the pair passes run one thread per sorted atom
    // (nbl_trav_atoms.cu) instead of one warp per work item; no work items
    // or hit words are built.  Needs the sorted cell keys, the systems'
    // atom bases and the visit tables.
    int atoms;
    const uint32_t *skeys;          // sorted cell keys (the sort's output)
    const int64_t *sys_atom_base;   // first atom of each system
    int nsys;
};

// Launch shape of one pair pass: warps per CTA (2, 4 or 8, i.e. 64, 128 or
// 256 threads), candidates staged per warp in the count (cand 0: 384 FP32 /
// 192 FP64 positions, cand 1: 768 / 384), atoms swept together per pass in
// the FP32 count (2 or 4).  A tuning choice with no effect on results.
struct TravShape {
    int warps = 4;
    int cand = 0;
    int group = 4;
};
// The fill's default shape: 8-warp CTAs (two per SM with 128 registers a
// thread, which the fill uses without spilling).
inline TravShape default_fill_shape() {
    TravShape s;
    s.warps = 8;
    return s;
}

cudaError_t launch_bin(const BinArgs &a, cudaStream_t st);
cudaError_t launch_gather(const GatherArgs &a, cudaStream_t st);
// Segment batches per work item with hit words in the mask pool (a batch is
// up to 32 visited cells: 27 for the usual 3x3x3 stencil, up to 125 for
// boxes smaller than the cutoff); home_mask holds kMaskBatches entries per
// work item.
constexpr int kMaskBatches = 4;


// Sum of n per-atom energies in a fixed order into *out (one double);
// scratch holds at least n / 2048 + n / 2048^2 + 2 doubles.
cudaError_t launch_lj_energy(const double *atom_e, int64_t n, double *scratch, double *out,
                             cudaStream_t st);

// The whole count phase of one small system in one CTA (nbl_small.cu): init,
// bin, a stable sort in shared memory, gather, work items, the count pass and
// the row offsets, leaving the same buffers as the multi-kernel sequence.
// Dense grid, one system, 1..kSmallMaxAtoms atoms (by default systems of up
// to kSmallDefaultAtoms take it), at most kSmallMaxCells cells, every row.
constexpr int kSmallMaxAtoms = 2048;
constexpr int kSmallDefaultAtoms = 128;
constexpr int kSmallTile = 8;  // atoms per work item on this path at most
constexpr int64_t kSmallMaxCells = 16384;
struct SmallCountArgs {
    BinArgs bin;          // keys / vals: sorted in place
    GatherArgs gather;    // keys / vals: the same arrays
    TraverseArgs trav;    // the count pass (and, unchanged, the fill after it)
    int64_t ncells;       // cell-table entries to clear
    int *small;           // the 8-int flag block
    int *items_count;     // == trav.n_items
    int64_t *offsets;     // [natoms + 1]
};
constexpr int kSmallMaxCtas = 8;  // a portable thread-block cluster
// ctas: 1 (one CTA) or a thread-block cluster of up to kSmallMaxCtas CTAs.
cudaError_t launch_count_small(bool fp32, int kind, const SmallCountArgs &a, int ctas,
                               cudaStream_t st);

// Start of a count phase in one launch: zero the 8-int flag block, the cell
// table (ntable int2) and the per-system maxima, mark every hash slot empty
// (hkey != NULL), and fill the systems' visit tables (visit != NULL).
cudaError_t launch_init(const SysDev *sys, int nsys, VisitDev *visit, int *small, int2 *table,
                        int64_t ntable, float *amax, unsigned long long *hkey, int num_sms,
                        cudaStream_t st);
// Work items: each occupied cell cut into tiles of `itile` (<= 32) atoms, or
// runs of up to `max_run` occupied cells along x (0: chosen from the mean
// occupancy; 1: no runs; runs need the dense grid and are only taken where
// every direction scans one cell each way).
cudaError_t launch_tiles(const HomeCell *home, const int *n_home, const int2 *table,
                         const SysDev *sys, WorkItem *items, int *n_items, int64_t natoms,
                         int num_sms, int itile, int max_run, cudaStream_t st);
cudaError_t launch_traverse(int mode, bool fp32, int kind, const TraverseArgs &a,
                            int grid, cudaStream_t st, const TravShape &shape = TravShape());
// CTAs of the pair pass (mode, precision, cutoff kind, shape, force sink)
// resident per SM on the current device: the grid of one full wave is this
// times the SM count.  0 on error.
int traverse_blocks_per_sm(int mode, bool fp32, int kind, const TravShape &shape = TravShape(),
                           bool lj = false, bool runs = false);
// Candidates one count warp stages per sweep for a shape.
constexpr int count_candidates(bool fp32, int cand) {
    return (fp32 ? 384 : 192) * (cand != 0 ? 2 : 1);
}
// Whether `shape` is one of the compiled launch shapes of the pass.
bool traverse_shape_ok(int mode, bool fp32, const TravShape &shape);

// Per precision and pass (nbl_trav_*.cu): launch / resident CTAs per SM.
cudaError_t launch_count_fp32(int kind, const TraverseArgs &a, int grid, cudaStream_t st,
                              const TravShape &shape);
cudaError_t launch_count_fp64(int kind, const TraverseArgs &a, int grid, cudaStream_t st,
                              const TravShape &shape);
cudaError_t launch_fill_fp32(int kind, const TraverseArgs &a, int grid, cudaStream_t st,
                             const TravShape &shape);
cudaError_t launch_fill_fp64(int kind, const TraverseArgs &a, int grid, cudaStream_t st,
                             const TravShape &shape);
int occupancy_count_fp32(int kind, const TravShape &shape);
// The FP32 instantiations that also take runs of home cells (TraverseArgs::runs).
cudaError_t launch_count_fp32_runs(int kind, const TraverseArgs &a, int grid, cudaStream_t st,
                                   const TravShape &shape);
cudaError_t launch_fill_fp32_runs(int kind, const TraverseArgs &a, int grid, cudaStream_t st,
                                  const TravShape &shape);
int occupancy_count_fp32_runs(int kind, const TravShape &shape);
int occupancy_fill_fp32_runs(int kind, const TravShape &shape, bool lj);
int occupancy_count_fp64(int kind, const TravShape &shape);
// The thread-per-atom passes (TraverseArgs::atoms, nbl_trav_atoms.cu): one
// thread per sorted atom walks its visited cells in the reference's order
// with the exact FP64 test; the grid covers the atoms.  No force sink.
cudaError_t launch_count_atoms(int kind, const TraverseArgs &a, cudaStream_t st);
cudaError_t launch_fill_atoms(int kind, const TraverseArgs &a, cudaStream_t st);
int occupancy_fill_fp32(int kind, const TravShape &shape, bool lj);
int occupancy_fill_fp64(int kind, const TravShape &shape, bool lj);

}  // namespace nbl
