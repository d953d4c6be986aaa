// nbl_build.cu -- the neighbour-list kernels for sm_100a.
//
// Pipeline (one launch sequence per batch of systems, all on one stream):
//   k_bin       per atom: raw cell (reference arithmetic), fold, cell key;
//               hashed grid: insert the cell into the open-addressing table
//   radix sort  (nbl_sort.cu) stable by cell key -> cell-sorted atom order
//   k_gather    per sorted atom: bin-relative position (FP64, reference
//               arithmetic), its FP32 copy, image indices, cell slices,
//               occupied-cell work list
//   k_tiles     occupied cells -> work items (home cell x i-tile of <= 32 atoms)
//   k_visit     per system: the visited cell offsets' vectors (reference order)
//   k_count     per work item: neighbour counts per atom, hit words
//   scan        (nbl_sort.cu) counts -> row offsets, total pair count
//   k_fill      per work item: writes i, j, D, d, S (or feeds a force sink)
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

namespace nbl {

namespace {

__device__ __forceinline__ int sys_of(const int64_t *__restrict__ bases, int nsys,
                                      int64_t a) {
    int lo = 0, hi = nsys - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (bases[mid] <= a)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

// Open-addressing insert; returns the slot.  At most cap probes.
__device__ __forceinline__ uint32_t hash_insert(unsigned long long *hkey,
                                                unsigned long long mask,
                                                unsigned long long key, int *err) {
    unsigned long long h = mix64(key) & mask;
    for (unsigned long long p = 0; p <= mask; p++) {
        unsigned long long cur = *((volatile unsigned long long *)&hkey[h]);
        if (cur == key) return (uint32_t)h;
        if (cur == kHashEmpty) {
            unsigned long long prev = atomicCAS(&hkey[h], kHashEmpty, key);
            if (prev == kHashEmpty || prev == key) return (uint32_t)h;
        }
        h = (h + 1) & mask;
    }
    atomicOr(err, kErrInternal);
    return 0;
}

}  // namespace

// ---------------------------------------------------------------------------
// k_bin
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
k_bin(BinArgs a) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= a.natoms) return;
    const int s = a.nsys > 1 ? sys_of(a.sys_atom_base, a.nsys, t) : 0;
    const SysDev &S = a.sys[s];
    double r[3] = {a.positions[3 * t + 0], a.positions[3 * t + 1],
                   a.positions[3 * t + 2]};
    int32_t raw[3];
    if (!raw_cell_of(S, r, raw)) atomicOr(a.err, kErrRange);
    int32_t c[3];
#pragma unroll
    for (int k = 0; k < 3; k++)
        c[k] = S.pbc[k] ? wrap_cell(raw[k], S.n[k]) : trunc_cell(raw[k], S.n[k]);
    const int64_t lin = (int64_t)c[0] + (int64_t)S.n[0] *
                                            ((int64_t)c[1] + (int64_t)S.n[1] * c[2]);
    uint32_t key;
    if (a.grid == kGridHashed) {
        const unsigned long long ck =
            ((unsigned long long)s << kHashSysShift) | (unsigned long long)lin;
        key = hash_insert(a.hkey, a.hmask, ck, a.err);
    } else if (a.grid == kGridMorton) {
        key = (uint32_t)(S.key_base + morton3(c[0], c[1], c[2]));
    } else {
        key = (uint32_t)(S.key_base + lin);
    }
    a.keys[t] = key;
    a.vals[t] = (int32_t)t;
}

// ---------------------------------------------------------------------------
// k_gather
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(256)
k_gather(GatherArgs a) {
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = s < a.natoms;
    const unsigned full = 0xffffffffu;
    bool start = false;
    int sysid = 0;
    uint32_t tidx = 0;
    int32_t c[3] = {0, 0, 0};
    float amax = 0.f;
    if (valid) {
        const int32_t at = a.vals[s];
        sysid = a.nsys > 1 ? sys_of(a.sys_atom_base, a.nsys, at) : 0;
        const SysDev &S = a.sys[sysid];
        const double r[3] = {a.positions[3 * (int64_t)at + 0],
                             a.positions[3 * (int64_t)at + 1],
                             a.positions[3 * (int64_t)at + 2]};
        int32_t raw[3];
        raw_cell_of(S, r, raw);  // range errors were flagged by k_bin
        int32_t rc[3], q[3];
#pragma unroll
        for (int k = 0; k < 3; k++) {
            if (S.pbc[k]) {
                c[k] = wrap_cell(raw[k], S.n[k]);
                rc[k] = raw[k];
                q[k] = floor_div(raw[k], S.n[k]);
            } else {
                c[k] = trunc_cell(raw[k], S.n[k]);
                rc[k] = c[k];
                q[k] = (raw[k] - c[k]) / S.n[k];  // C truncating division
            }
        }
        // neighbour_list.cc:157-159: ((r - r1 b1) - r2 b2) - r3 b3
        double rel[3];
#pragma unroll
        for (int k = 0; k < 3; k++) {
            double v = dsub(r[k], dmul((double)rc[0], S.bin[0][k]));
            v = dsub(v, dmul((double)rc[1], S.bin[1][k]));
            v = dsub(v, dmul((double)rc[2], S.bin[2][k]));
            rel[k] = v;
        }
        double w64 = 0.0;
        float w32 = 0.f;
        if (S.cutoff_kind == kCutPerAtom) {
            w64 = a.per_atom[at];
            w32 = __double2float_rn(w64);
        } else if (S.cutoff_kind == kCutPerType) {
            w32 = __int_as_float(a.types[at]);
        }
        a.pos64[s] = make_double4(rel[0], rel[1], rel[2], w64);
        a.pos32[s] = make_float4(__double2float_rn(rel[0]), __double2float_rn(rel[1]),
                                 __double2float_rn(rel[2]), w32);
        a.aux[s] = make_int4(at, q[0], q[1], q[2]);
        amax = __double2float_ru(fmax(fabs(rel[0]), fmax(fabs(rel[1]), fabs(rel[2]))));

        const uint32_t key = a.keys[s];
        const int64_t lin = (int64_t)c[0] +
                            (int64_t)S.n[0] * ((int64_t)c[1] + (int64_t)S.n[1] * c[2]);
        tidx = (a.grid == kGridMorton) ? (uint32_t)(S.cell_base + lin) : key;
        start = (s == 0) || (a.keys[s - 1] != key);
        const bool end = (s == a.natoms - 1) || (a.keys[s + 1] != key);
        if (start) a.table[tidx].x = (int32_t)s;
        if (end) a.table[tidx].y = (int32_t)(s + 1);
    }
    // Per-system max |rel| (non-negative floats order like their bit patterns):
    // one atomic per warp when the warp lies inside one system, else per lane.
    {
        const int lane = threadIdx.x & 31;
        const int s0 = __shfl_sync(full, sysid, 0);
        const bool uni = __all_sync(full, !valid || sysid == s0);
        const unsigned bits = valid ? (unsigned)__float_as_int(amax) : 0u;
        if (uni) {
            const unsigned mx = __reduce_max_sync(full, bits);
            const unsigned anyv = __ballot_sync(full, valid);
            if (lane == 0 && anyv) atomicMax(reinterpret_cast<unsigned *>(a.amax) + s0, mx);
        } else if (valid) {
            atomicMax(reinterpret_cast<unsigned *>(a.amax) + sysid, bits);
        }
    }
    // Occupied-cell work list (warp-aggregated append).
    const unsigned m = __ballot_sync(full, start);
    if (m) {
        const int lane = threadIdx.x & 31;
        int base = 0;
        if (lane == __ffs(m) - 1) base = atomicAdd(a.n_home, __popc(m));
        base = __shfl_sync(full, base, __ffs(m) - 1);
        if (start) {
            HomeCell h;
            h.tidx = (int32_t)tidx;
            h.sys = sysid;
            h.c[0] = c[0];
            h.c[1] = c[1];
            h.c[2] = c[2];
            h.pad = 0;
            a.home[base + __popc(m & lanemask_lt())] = h;
        }
    }
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
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const int nh = *n_home;
    int R = max_run;
    if (R == 0) {
        const float occ = (float)natoms / (float)max(nh, 1);
        R = occ >= 6.f ? 1 : min(kMaxRun, max(1, (int)((float)itile / (2.f * occ))));
    }
    R = min(R, kMaxRun);
    for (int base = blockIdx.x * blockDim.x; base < nh; base += gridDim.x * blockDim.x) {
        const int h = base + threadIdx.x;
        int2 hs = make_int2(0, 0);
        HomeCell hc{};
        if (h < nh) {
            hc = home[h];
            hs = table[hc.tidx];
        }
        int nt = (hs.y - hs.x + itile - 1) / itile;
        int run = 1, run_atoms = 0;
        if (R > 1 && h < nh) {
            const SysDev &S = sys[hc.sys];
            if (S.nscan[0] == 1 && S.nscan[1] == 1 && S.nscan[2] == 1) {
                const int x = hc.c[0];
                const int xb = (x / R) * R, xe = min(xb + R, S.n[0]);
                int total = 0, first = -1, last = -1;
                for (int xc = xb; xc < xe; xc++) {
                    const int2 sl = table[hc.tidx + (xc - x)];
                    const int n = sl.y - sl.x;
                    if (n > 0) {
                        total += n;
                        if (first < 0) first = xc;
                        last = xc;
                    }
                }
                if (total <= itile && first != last) {  // two or more occupied cells
                    nt = (x == first) ? 1 : 0;
                    run = last - first + 1;
                    run_atoms = total;
                }
            }
        }
        int incl = nt;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int o = __shfl_up_sync(full, incl, d);
            if (lane >= d) incl += o;
        }
        const int tot = __shfl_sync(full, incl, 31);
        int first = 0;
        if (lane == 0 && tot > 0) first = atomicAdd(n_items, tot);
        first = __shfl_sync(full, first, 0) + incl - nt;
        for (int t = 0; t < nt; t++) {
            WorkItem w;
            w.c[0] = hc.c[0];
            w.c[1] = hc.c[1];
            w.c[2] = hc.c[2];
            w.sys = hc.sys;
            w.ib = hs.x + itile * t;
            w.nt = run > 1 ? run_atoms : min(itile, hs.y - w.ib);
            w.tidx = hc.tidx;
            w.run = run;
            items[first + t] = w;
        }
    }
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


// One block per system with a visit table: its visited offsets in the
// traversal's z/y/x order (neighbour_visit.hh:63-84).
__global__ void k_visit(const SysDev *__restrict__ sys, VisitDev *__restrict__ visit) {
    const SysDev &S = sys[blockIdx.x];
    if (S.visit_base < 0) return;
    const int nx = S.nscan[0], ny = S.nscan[1], nz = S.nscan[2];
    const int wx = 2 * nx + 1, wy = 2 * ny + 1;
    for (int v = threadIdx.x; v < S.nvisit; v += blockDim.x) {
        const int xr = v % wx, rest = v / wx;
        const int yr = rest % wy, zr = rest / wy;
        const int d[3] = {xr - nx, yr - ny, zr - nz};
        double o[3];
        visit_offset(S, d, o);
        VisitDev e;
#pragma unroll
        for (int k = 0; k < 3; k++) {
            e.off[k] = o[k];
            e.off32[k] = __double2float_rn(o[k]);
            e.d[k] = d[k];
        }
        visit[S.visit_base + v] = e;
    }
}

__global__ void __launch_bounds__(256)
k_init(const SysDev *__restrict__ sys, int nsys, VisitDev *__restrict__ visit,
       int *__restrict__ small, int2 *__restrict__ table, int64_t ntable,
       float *__restrict__ amax, unsigned long long *__restrict__ hkey) {
    if (visit != nullptr && (int)blockIdx.x < nsys) {
        const SysDev &S = sys[blockIdx.x];
        if (S.visit_base >= 0) {
            const int nx = S.nscan[0], ny = S.nscan[1], nz = S.nscan[2];
            const int wx = 2 * nx + 1, wy = 2 * ny + 1;
            for (int v = threadIdx.x; v < S.nvisit; v += blockDim.x) {
                const int xr = v % wx, rest = v / wx;
                const int yr = rest % wy, zr = rest / wy;
                const int d[3] = {xr - nx, yr - ny, zr - nz};
                double o[3];
                visit_offset(S, d, o);
                VisitDev e;
#pragma unroll
                for (int k = 0; k < 3; k++) {
                    e.off[k] = o[k];
                    e.off32[k] = __double2float_rn(o[k]);
                    e.d[k] = d[k];
                }
                visit[S.visit_base + v] = e;
            }
        }
    }
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

cudaError_t launch_visit(const SysDev *sys, int nsys, VisitDev *visit, cudaStream_t st) {
    if (nsys <= 0 || visit == nullptr) return cudaSuccess;
    k_visit<<<nsys, 64, 0, st>>>(sys, visit);
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
