// nbl_plan.hh -- host-side state of the engine (plans, batches, workspace).
#pragma once

#include <cstdint>
#include <cstring>
#include <vector>

#include <cuda_runtime.h>
#include <nvtx3/nvToolsExt.h>

#include "nbl_b200.h"
#include "nbl_build.cuh"
#include "nbl_internal.cuh"

namespace nbl {

// A batch of independent systems planned on the host.
struct Batch {
    std::vector<SysDev> sys;
    std::vector<int64_t> ncells;
    std::vector<double> pt64;      // concatenated per-type squared cutoffs
    int64_t natoms = 0;
    const double *positions = nullptr;
    bool pos_on_device = false;
    const double *per_atom = nullptr;
    const int32_t *types = nullptr;
    bool aux_on_device = false;
    int grid = kGridDense;         // resolved kGrid*
    int64_t table_size = 1;
    int key_bits = 0;
    bool fp32 = true;
    int quantities = 0;
};

// Device buffers of one call, carved out of the workspace.
struct Bufs {
    double *pos = nullptr;
    double *per_atom = nullptr;
    int32_t *types = nullptr;
    SysDev *sys = nullptr;
    VisitDev *visit = nullptr;     // per-system visit tables (nullptr: none)
    int64_t *sys_atom_base = nullptr;
    double *pt64 = nullptr;
    float *pt32 = nullptr;
    uint32_t *keys = nullptr, *keys2 = nullptr;
    int32_t *vals = nullptr, *vals2 = nullptr;
    int32_t *hist = nullptr, *hist_scan = nullptr, *scan32 = nullptr;
    int64_t *scan64 = nullptr;
    int2 *table = nullptr;
    unsigned long long *hkey = nullptr;
    double4 *pos64 = nullptr;
    float4 *pos32 = nullptr;
    int4 *aux = nullptr;
    float *amax = nullptr;
    HomeCell *home = nullptr;
    int32_t *counts = nullptr;
    int64_t *offsets = nullptr;
    int *small = nullptr;  // [0] occupied cells, [1] error bits, [2] matrix
                           // overflow, [3] work items, [4..5] mask-pool cursor
                           // (u64), [6] work-item ticket of the pair passes;
                           // placed right after offsets[N], so one copy of
                           // 32 bytes from offsets + N returns the pair count
                           // and the first six flags
    // The small host tables (systems, their atom bases, per-type cutoffs in
    // FP64 and FP32) lie at these byte offsets from `sys`, one contiguous
    // block of tab_bytes, so that they go up in one copy.
    size_t tab_sab = 0, tab_pt64 = 0, tab_pt32 = 0, tab_bytes = 0;
    uint32_t *mask_pool = nullptr;
    long long mask_cap = 0;
    long long *home_mask = nullptr;
    WorkItem *items = nullptr;
    double *lj_part = nullptr;     // force sink: per-atom energies, then block sums
};

struct Workspace {
    void *base = nullptr;
    size_t bytes = 0;
    void *out_base = nullptr;  // device output scratch of nbl_fill_host
    size_t out_bytes = 0;
    void release();
};

// Full waves of resident CTAs in the default grid of a pair pass.
constexpr int kAutoWaves = 2;

// Everything that shapes the count phase's launches on a plan: when two
// consecutive single calls have the same key, the second captures the count
// phase into a CUDA graph and later ones replay it (compared bytewise; the
// constructor zeroes the padding).
struct CountKey {
    const void *ws_base, *pos, *per_atom, *types;
    int64_t natoms, table_size, mask_cap, pt_size, i_lo, i_hi;
    int32_t nsys, grid, key_bits, fp32, kind, itile, max_run, nvisit_tab;
    int32_t count_mult, count_warps, count_cand, count_group, count_tickets, atoms;
    CountKey() { std::memset(this, 0, sizeof(*this)); }
    bool operator==(const CountKey &o) const { return std::memcmp(this, &o, sizeof(*this)) == 0; }
};

struct Plan {
    int device = 0;
    int num_sms = 148;
    Workspace ws;
    Bufs bufs;
    TraverseArgs targs{};
    int trav_grid = 0;        // count-pass grid (CTAs)
    int fill_grid = 0;        // fill-pass grid (CTAs)
    // Launch configuration (set by the autotuner for batches, or by
    // nbl_plan_set_launch / nbl_plan_set_launch_config): CTAs per SM of the
    // count and fill passes (0: a whole number of waves of resident CTAs),
    // each pass's launch shape (warps per CTA, staged candidates, atoms per
    // sweep) and the atoms per work item (cell-occupancy tile).
    int count_mult = 0;
    int fill_mult = 0;
    TravShape count_shape;
    TravShape fill_shape = default_fill_shape();
    int itile = 32;
    // Tile chosen per call from the atom count (launch config atoms_per_item
    // 0); itile is then the tile of large systems.
    bool itile_auto = true;
    // Home cells per work item at most (0: chosen on the device from the
    // cells' mean occupancy; 1: one cell per item).  Runs of several cells
    // are only built on the dense grid with the FP32 filter.
    int max_run = 0;
    // Systems of up to this many atoms (at most kSmallMaxAtoms) take the
    // one-CTA count phase; 0: never.
    int small_atoms = kSmallDefaultAtoms;
    // Pair passes with one thread per atom (nbl_trav_atoms.cu): 0 = where the
    // occupied cells hold fewer than two atoms on average, -1 = never, 1 =
    // always (where the systems have visit tables).  no_atoms turns them off
    // for one count (the force sink needs the work items).
    int atom_threads = 0;
    bool no_atoms = false;
    // Occupied cells counted by the last synchronised count, with the atom
    // count and table size it ran on (steers the default choice above).
    int64_t occ_natoms = -1, occ_table = -1, occ_cells = 0;
    // Work items by atomic ticket (else a fixed warp stride) in each pass.
    bool count_tickets = true;
    bool fill_tickets = true;
    int64_t mask_hint = 0;    // mask-pool words the last count asked for
    // Row range of nbl_set_atom_range (global atom indices, [lo, hi)).
    int64_t i_lo = 0;
    int64_t i_hi = INT64_MAX;
    int64_t batch_natoms = 0;
    int batch_nsys = 0;
    bool batch_fp32 = true;
    int batch_kind = kCutScalar;
    int batch_grid = kGridDense;
    bool have_count = false;
    int64_t npairs = 0;
    int quantities = 0;
    int64_t *host_small = nullptr;  // pinned: [0] pair count, [1] flags
    void *host_stage = nullptr;     // pinned staging of the small host tables
    size_t host_stage_bytes = 0;
    void *host_out = nullptr;       // pinned landing area of small host fills
    size_t host_out_bytes = 0;
    cudaEvent_t stage_done = nullptr;
    bool stage_in_flight = false;
    // Count-phase graph of the single-call path (see CountKey).
    CountKey last_key, graph_key;
    bool have_last_key = false;
    bool graphs_off = false;        // capture failed once: direct launches only
    cudaStream_t capture_stream = nullptr;
    cudaGraphExec_t count_graph = nullptr;
    long long graph_launches = 0;   // kernels in the graph (launch accounting)
    TraverseArgs graph_targs{};     // host state the capture left behind
    int graph_trav_grid = 0, graph_kind = 0;
};

// Drops the plan's count-phase graph (its pointers refer to the workspace).
void drop_count_graph(Plan &p);

// An NVTX range over one host-side stage (bin, sort, gather, count, scan,
// fill): profilers show the stages of a call by name and can filter their
// kernels by it.  Costs a few nanoseconds when no tool is attached.
struct StageRange {
    explicit StageRange(const char *name) { nvtxRangePushA(name); }
    ~StageRange() { nvtxRangePop(); }
    StageRange(const StageRange &) = delete;
    StageRange &operator=(const StageRange &) = delete;
};

// Stream-ordered scratch pool of device `dev` that keeps its memory between
// calls (cudaMallocFromPoolAsync / cudaFreeAsync on it).
cudaError_t scratch_pool(int dev, cudaMemPool_t *pool);

nbl_status set_error(nbl_status st, const char *fmt, ...);
nbl_status cuda_status(cudaError_t e, const char *where);
nbl_status plan_system(const double origin[3], const double cell[9],
                       const double inv_cell[9], const uint8_t pbc[3], double cutoff,
                       SysDev &S, int64_t &ncells);
nbl_status finish_batch(Batch &b, int grid_req);
nbl_status upload_batch(Plan &p, const Batch &b, cudaStream_t st);
nbl_status enqueue_count(Plan &p, const Batch &b, cudaStream_t st);
nbl_status run_count(Plan &p, const Batch &b, cudaStream_t st, bool sync);
nbl_status run_fill(Plan &p, const nbl_outputs &o, int64_t capacity, cudaStream_t st);
// The device flags of the last count / fill as a status (copy: read them
// first, synchronising st).
nbl_status read_flags(Plan &p, cudaStream_t st, bool copy = true);
void launch_config_of(const Plan &p, nbl_launch_config *cfg);

}  // namespace nbl
