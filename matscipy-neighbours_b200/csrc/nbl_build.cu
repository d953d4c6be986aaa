// nbl_build.cu -- the neighbour-list kernels for sm_100a.
//
// Pipeline (one launch sequence per batch of systems, all on one stream; the
// per-atom and per-cell bodies of the first stages are in nbl_stages.cuh):
//   k_init      flag block, cell table, per-system maxima, hash slots, and the
//               visited cell offsets' vectors (reference order) per system
//   k_bin       per atom: raw cell (reference arithmetic), fold, cell key;
//               hashed grid: insert the cell into the open-addressing table
//   radix sort  (nbl_sort.cu) stable by cell key -> cell-sorted atom order
//   k_gather    per sorted atom: bin-relative position (FP64, reference
//               arithmetic), its FP32 copy, image indices, cell slices,
//               occupied-cell work list
//   k_tiles     occupied cells -> work items (home cell x i-tile of <= 32
//               atoms, or runs of sparse cells along x)
//   k_count     per work item: neighbour counts per atom, hit words
//   scan        (nbl_sort.cu) counts -> row offsets, total pair count
//   k_fill      per work item: writes i, j, D, d, S (or feeds a force sink)
// A small system's count phase (init to scan) can instead be one launch
// (nbl_small.cu).
//
// The traversal reproduces neighbour_visit.hh:51-120 exactly: the same
// visited offsets in the same z/y/x order, the same cell slices in ascending
// atom order, the same FP64 operations (no FMA contraction: every FP64 op is an
// explicit __d*_rn intrinsic), so the output is the reference CPU output,
// including the order of pairs within a row.
//
// Work decomposition (instead of the reference's thread-per-atom loop): one
// warp per work item, the item's visited neighbour cells ("segments") one per
// lane, their atoms ("candidates") staged in shared memory; the count sweeps
// them 32 at a time against the tile's atoms (FP32 filter with an FP64 guard
// band, or plain FP64; __ballot_sync + __popc), and the fill turns the hit
// words into 32 pairs per round so that the FP64 epilogue and the stores run
// with full warps and near-contiguous addresses (details in nbl_traverse.cuh).
#include <algorithm>
#include <atomic>
#include <climits>
#include <cstdint>
#include <type_traits>

#include <cuda_runtime.h>

#include "nbl_build.cuh"
#include "nbl_internal.cuh"
#include "nbl_stages.cuh"

namespace nbl {

// ---------------------------------------------------------------------------
// k_bin
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
k_bin(BinArgs a) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < a.natoms) bin_one(a, t);
}

// ---------------------------------------------------------------------------
// k_gather
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
k_gather(GatherArgs a) {
    gather_one(a, (int64_t)blockIdx.x * blockDim.x + threadIdx.x);
}

// ---------------------------------------------------------------------------
// k_tiles: work items = (occupied cell, i-tile of `itile` <= 32 atoms), or
// runs of consecutive occupied cells along x
// ---------------------------------------------------------------------------
// Splitting large cells keeps one warp from holding a whole big cell (a
// small periodic system often is one cell) while the rest of the GPU idles.
// Sparse grids (few atoms per cell) instead pack the occupied cells of each
// aligned block of `R` cells along x into one item when their atoms fit one
// tile: the run's neighbour cells are then visited once for up to R home
// cells.  R = max_run, or (max_run == 0) chosen from the mean occupancy:
// 1 (no runs) at 6 or more atoms per occupied cell, else about itile / (2 x
// occupancy), at most kMaxRun.  Runs need the dense grid (the run's atoms are
// contiguous in sorted order) and a +-1 cell scan in every direction.
__global__ void __launch_bounds__(256)
k_tiles(const HomeCell *__restrict__ home, const int *__restrict__ n_home,
        const int2 *__restrict__ table, const SysDev *__restrict__ sys,
        WorkItem *__restrict__ items, int *__restrict__ n_items, int64_t natoms, int itile,
        int max_run) {
    const int nh = *n_home;
    const int R = tiles_run_length(nh, natoms, itile, max_run);
    for (int base = blockIdx.x * blockDim.x; base < nh; base += gridDim.x * blockDim.x)
        tiles_one(home, table, sys, items, n_items, itile, R, base + threadIdx.x, nh);
}

cudaError_t launch_tiles(const HomeCell *home, const int *n_home, const int2 *table,
                         const SysDev *sys, WorkItem *items, int *n_items, int64_t natoms,
                         int num_sms, int itile, int max_run, cudaStream_t st) {
    if (natoms <= 0) return cudaSuccess;
    if (itile < 1 || itile > 32 || max_run < 0) return cudaErrorInvalidValue;
    const int64_t blocks = std::min<int64_t>((natoms + 255) / 256, (int64_t)num_sms * 4);
    k_tiles<<<(unsigned)blocks, 256, 0, st>>>(home, n_home, table, sys, items, n_items, natoms,
                                              itile, max_run);
    count_launch();
    return cudaGetLastError();
}


// Start of a count phase: block s < nsys also fills system s's visit table
// (its visited offsets in the traversal's z/y/x order, neighbour_visit.hh:
// 63-84); every thread clears its share of the flags, the cell table (and
// the hash slots) and the per-system maxima.
__global__ void __launch_bounds__(256)
k_init(const SysDev *__restrict__ sys, int nsys, VisitDev *__restrict__ visit,
       int *__restrict__ small, int2 *__restrict__ table, int64_t ntable,
       float *__restrict__ amax, unsigned long long *__restrict__ hkey) {
    if (visit != nullptr && (int)blockIdx.x < nsys)
        visit_fill(sys[blockIdx.x], visit, threadIdx.x, blockDim.x);
    const int64_t t0 = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t step = (int64_t)gridDim.x * blockDim.x;
    if (t0 < 8) small[t0] = 0;
    for (int64_t i = t0; i < ntable; i += step) {
        table[i] = make_int2(0, 0);
        if (hkey != nullptr) hkey[i] = kHashEmpty;
    }
    for (int64_t i = t0; i < nsys; i += step) amax[i] = 0.f;
}

cudaError_t launch_init(const SysDev *sys, int nsys, VisitDev *visit, int *small, int2 *table,
                        int64_t ntable, float *amax, unsigned long long *hkey, int num_sms,
                        cudaStream_t st) {
    const int64_t work = std::max<int64_t>(ntable, nsys);
    int64_t blocks = std::min<int64_t>((work + 255) / 256, (int64_t)num_sms * 8);
    blocks = std::max<int64_t>(blocks, visit != nullptr ? nsys : 1);
    blocks = std::max<int64_t>(blocks, 1);
    k_init<<<(unsigned)blocks, 256, 0, st>>>(sys, nsys, visit, small, table, ntable, amax, hkey);
    count_launch();
    return cudaGetLastError();
}


// Fixed-order sum of n values: block b sums values [2048 b, 2048 b + 2048)
// (thread t: 8 consecutive values, then a fixed tree) into part2[b]; one
// block then sums the block sums the same way.  The same bits every run.
__global__ void __launch_bounds__(256) k_sum_fixed(const double *__restrict__ v, int64_t n,
                                                   double *__restrict__ out) {
    __shared__ double s[256];
    const int64_t b0 = (int64_t)blockIdx.x * 2048 + (int64_t)threadIdx.x * 8;
    double t = 0.0;
#pragma unroll
    for (int k = 0; k < 8; k++)
        if (b0 + k < n) t += v[b0 + k];
    s[threadIdx.x] = t;
    __syncthreads();
    for (int h = 128; h > 0; h >>= 1) {
        if ((int)threadIdx.x < h) s[threadIdx.x] += s[threadIdx.x + h];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[blockIdx.x] = s[0];
}

cudaError_t launch_lj_energy(const double *atom_e, int64_t n, double *scratch, double *out,
                             cudaStream_t st) {
    const int64_t nb = (n + 2047) / 2048;
    if (nb <= 1) {
        k_sum_fixed<<<1, 256, 0, st>>>(atom_e, n, out);
        count_launch();
        return cudaGetLastError();
    }
    k_sum_fixed<<<(unsigned)nb, 256, 0, st>>>(atom_e, n, scratch);
    count_launch();
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    return launch_lj_energy(scratch, nb, scratch + nb, out, st);
}

cudaError_t launch_bin(const BinArgs &a, cudaStream_t st) {
    if (a.natoms <= 0) return cudaSuccess;
    const unsigned grid = (unsigned)((a.natoms + 255) / 256);
    k_bin<<<grid, 256, 0, st>>>(a);
    count_launch();
    return cudaGetLastError();
}

cudaError_t launch_gather(const GatherArgs &a, cudaStream_t st) {
    if (a.natoms <= 0) return cudaSuccess;
    const unsigned grid = (unsigned)((a.natoms + 255) / 256);
    k_gather<<<grid, 256, 0, st>>>(a);
    count_launch();
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// pair-pass dispatch (kernels: nbl_traverse.cuh, instantiated in nbl_trav_*.cu)
// ---------------------------------------------------------------------------

bool traverse_shape_ok(int mode, bool fp32, const TravShape &s) {
    if (s.warps != 2 && s.warps != 4 && s.warps != 8) return false;
    if (mode != kModeCount) return true;
    return (s.cand == 0 || s.cand == 1) && (!fp32 || s.group == 2 || s.group == 4);
}

int traverse_blocks_per_sm(int mode, bool fp32, int kind, const TravShape &shape, bool lj,
                           bool runs) {
    // cached per device, pass, precision, kind, shape and run instantiation
    constexpr int kDev = 16;
    static std::atomic<int> cache[kDev][2][2][3][3][2][2][2][2];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kDev) {
        cudaGetLastError();
        dev = -1;
    }
    const int mi = mode == kModeCount ? 0 : 1, fi = fp32 ? 1 : 0;
    const int ki = kind == kCutPerAtom ? 1 : (kind == kCutPerType ? 2 : 0), li = lj ? 1 : 0;
    const int wi = shape.warps == 2 ? 0 : (shape.warps == 8 ? 2 : 1);
    const int ci = shape.cand != 0 ? 1 : 0;
    const int gi = shape.group == 2 ? 0 : 1;
    runs = runs && fp32;  // runs are only built for the FP32 filter
    const int ri = runs ? 1 : 0;
    if (dev >= 0) {
        const int c = cache[dev][mi][fi][ki][wi][ci][gi][li][ri].load(std::memory_order_relaxed);
        if (c > 0) return c;
    }
    int n = 0;
    if (mode == kModeCount)
        n = !fp32 ? occupancy_count_fp64(kind, shape)
                  : (runs ? occupancy_count_fp32_runs(kind, shape)
                          : occupancy_count_fp32(kind, shape));
    else
        n = !fp32 ? occupancy_fill_fp64(kind, shape, lj)
                  : (runs ? occupancy_fill_fp32_runs(kind, shape, lj)
                          : occupancy_fill_fp32(kind, shape, lj));
    if (dev >= 0 && n > 0)
        cache[dev][mi][fi][ki][wi][ci][gi][li][ri].store(n, std::memory_order_relaxed);
    return n;
}

cudaError_t launch_traverse(int mode, bool fp32, int kind, const TraverseArgs &a,
                            int grid, cudaStream_t st, const TravShape &shape) {
    if (grid <= 0) return cudaSuccess;
    if (!traverse_shape_ok(mode, fp32, shape)) return cudaErrorInvalidValue;
    if (a.atoms) {  // one thread per atom; precision does not apply (exact FP64)
        if (a.lj_force != nullptr) return cudaErrorInvalidValue;
        return mode == kModeCount ? launch_count_atoms(kind, a, st)
                                  : launch_fill_atoms(kind, a, st);
    }
    if (!fp32) {
        return mode == kModeCount ? launch_count_fp64(kind, a, grid, st, shape)
                                  : launch_fill_fp64(kind, a, grid, st, shape);
    }
    if (a.runs)  // the items may be runs of several home cells
        return mode == kModeCount ? launch_count_fp32_runs(kind, a, grid, st, shape)
                                  : launch_fill_fp32_runs(kind, a, grid, st, shape);
    return mode == kModeCount ? launch_count_fp32(kind, a, grid, st, shape)
                              : launch_fill_fp32(kind, a, grid, st, shape);
}

}  // namespace nbl
