// nbl_api.cu -- host side of the engine: request validation, bit-exact grid
// planning, workspace management and the C-ABI of include/nbl_b200.h.
//
// Host arithmetic that feeds the kernels (cell widths, cells per direction,
// bin vectors, scan ranges, cutoff^2) follows the reference's operation order
// (src/libneighbours/cell_list.cc:153-182, neighbour_list.cc:169-192) and is
// compiled without FP contraction, so the device sees the same doubles the
// reference CPU core computes.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <limits>
#include <mutex>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "nbl_b200.h"
#include "nbl_build.cuh"
#include "nbl_internal.cuh"
#include "nbl_plan.hh"
#include "nbl_sort.cuh"

namespace nbl {

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
static thread_local std::string g_last_error;

nbl_status set_error(nbl_status st, const char *fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return st;
}

static void clear_error() { g_last_error.clear(); }

static thread_local long long g_launches = 0;
void count_launch(int n) { g_launches += n; }

nbl_status cuda_status(cudaError_t e, const char *where) {
    if (e == cudaSuccess) return NBL_SUCCESS;
    if (e == cudaErrorMemoryAllocation)
        return set_error(NBL_ERROR_OUT_OF_MEMORY, "%s: out of device memory", where);
    return set_error(NBL_ERROR_CUDA, "%s: %s", where, cudaGetErrorString(e));
}

#define NBL_CUDA(call, where)                                  \
    do {                                                       \
        cudaError_t e_ = (call);                               \
        if (e_ != cudaSuccess) return cuda_status(e_, where);  \
    } while (0)

// ---------------------------------------------------------------------------
// geometry (cell_list.cc:153-182 and neighbour_list.cc:169-192)
// ---------------------------------------------------------------------------

// static_cast<int>(double) as x86-64 executes it: out of range or NaN gives
// INT32_MIN (cvttsd2si).  The reference relies on it for very small cutoffs
// (len/cutoff beyond 2^31 gives n = max(INT32_MIN, 1) = 1).
static int32_t x86_to_i32(double v) {
    if (!(v > -2147483649.0 && v < 2147483648.0)) return INT32_MIN;
    return (int32_t)v;
}

static void cross3(const double *a, const double *b, double *c) {
    c[0] = a[1] * b[2] - a[2] * b[1];
    c[1] = a[2] * b[0] - a[0] * b[2];
    c[2] = a[0] * b[1] - a[1] * b[0];
}

static double norm3(const double *a) {
    return std::sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
}

nbl_status plan_system(const double origin[3], const double cell[9],
                       const double inv_cell[9], const uint8_t pbc[3],
                       double cutoff, SysDev &S, int64_t &ncells) {
    std::memset(&S, 0, sizeof(S));
    if (!std::isfinite(cutoff))
        return set_error(NBL_ERROR_INVALID_ARGUMENT, "cutoff must be finite");
    const double *c1 = &cell[0], *c2 = &cell[3], *c3 = &cell[6];
    double nrm1[3], nrm2[3], nrm3[3];
    cross3(c2, c3, nrm1);
    cross3(c3, c1, nrm2);
    cross3(c1, c2, nrm3);
    const double volume =
        std::fabs(c3[0] * nrm3[0] + c3[1] * nrm3[1] + c3[2] * nrm3[2]);
    if (volume < 1e-12) return set_error(NBL_ERROR_ZERO_VOLUME, "Zero cell volume.");
    double len[3];
    len[0] = volume / norm3(nrm1);
    len[1] = volume / norm3(nrm2);
    len[2] = volume / norm3(nrm3);
    for (int k = 0; k < 3; k++) {
        const int32_t n = x86_to_i32(std::floor(len[k] / cutoff));
        S.n[k] = std::max(n, 1);
    }
    for (int k = 0; k < 3; k++) {
        S.bin[0][k] = c1[k] / S.n[0];
        S.bin[1][k] = c2[k] / S.n[1];
        S.bin[2][k] = c3[k] / S.n[2];
        S.origin[k] = origin[k];
        S.pbc[k] = pbc[k] ? 1 : 0;
    }
    for (int k = 0; k < 9; k++) S.inv[k] = inv_cell[k];
    int64_t nvisit = 1;
    for (int k = 0; k < 3; k++) {
        const double s = cutoff * S.n[k] / len[k];
        const double cs = std::ceil(s);
        if (!(cs < 1e6))
            return set_error(NBL_ERROR_INVALID_ARGUMENT,
                             "cutoff spans more than 10^6 periodic images of the cell");
        S.nscan[k] = (int32_t)cs;
        nvisit *= (S.nscan[k] < 0) ? 0 : (2 * (int64_t)S.nscan[k] + 1);
    }
    if (nvisit > (int64_t(1) << 24))
        return set_error(NBL_ERROR_INVALID_ARGUMENT,
                         "cutoff spans more than 2^24 neighbour cells per cell");
    S.nvisit = (int32_t)nvisit;
    S.visit_base = -1;
    S.cutoff = cutoff;
    S.cutoff_sq = cutoff * cutoff;
    double off_max = 0.0;
    for (int k = 0; k < 3; k++) {
        const double bmax = std::max(std::fabs(S.bin[k][0]),
                                     std::max(std::fabs(S.bin[k][1]), std::fabs(S.bin[k][2])));
        off_max += std::max(S.nscan[k], 0) * bmax;
    }
    S.off_max = off_max * (1.0 + 1e-12);
    ncells = (int64_t)S.n[0] * S.n[1] * S.n[2];
    return NBL_SUCCESS;
}

static int bits_for(uint64_t maxval) {
    int b = 0;
    while (b < 64 && (maxval >> b) != 0) b++;
    return b;
}

// ---------------------------------------------------------------------------
// workspace
// ---------------------------------------------------------------------------

struct Layout {
    size_t total = 0;
    size_t add(size_t bytes) {
        size_t off = total;
        total += (bytes + 255) & ~size_t(255);
        return off;
    }
};

void Workspace::release() {
    if (base) cudaFree(base);
    base = nullptr;
    bytes = 0;
    if (out_base) cudaFree(out_base);
    out_base = nullptr;
    out_bytes = 0;
}

// Host-side failure injection (nbl_debug_inject): workspace growths that are
// made to fail, and a forced hashed-table size.
static std::atomic<int64_t> g_inject_alloc_failures{0};
static std::atomic<int64_t> g_inject_hash_capacity{0};

static nbl_status ensure(void *&ptr, size_t &have, size_t need, const char *what) {
    if (need <= have) return NBL_SUCCESS;
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    have = 0;
    for (int64_t n = g_inject_alloc_failures.load(); n > 0;
         n = g_inject_alloc_failures.load()) {
        if (g_inject_alloc_failures.compare_exchange_weak(n, n - 1))
            return set_error(NBL_ERROR_OUT_OF_MEMORY,
                             "%s: cannot allocate %zu bytes (injected failure)", what, need);
    }
    size_t grow = need + need / 4;
    cudaError_t e = cudaMalloc(&ptr, grow);
    if (e != cudaSuccess) {
        cudaGetLastError();
        e = cudaMalloc(&ptr, need);
        grow = need;
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        ptr = nullptr;
        return set_error(NBL_ERROR_OUT_OF_MEMORY, "%s: cannot allocate %zu bytes", what,
                         need);
    }
    have = grow;
    return NBL_SUCCESS;
}

// Visit tables for all systems when their entries are few (the usual case:
// 27 per system); with more, the pair kernels compute offsets per item.
constexpr int64_t kVisitCap = int64_t(1) << 20;
static int64_t visit_entries(const Batch &b) {
    int64_t n = 0;
    for (const SysDev &S : b.sys) n += S.nvisit;
    return n <= kVisitCap ? n : 0;
}

// Mask-pool words: per system, atoms x (chunks of a full candidate list +
// one partial chunk per segment batch), with the candidates of an atom
// estimated as visited cells x atoms per cell; or the demand of the last
// count on this plan if that was larger.  Items that do not fit are
// recomputed by the fill, so this only steers speed.
static int64_t mask_words(const Plan &p, const Batch &b) {
    double est = 0.0;
    for (size_t s2 = 0; s2 < b.sys.size(); s2++) {
        const SysDev &S = b.sys[s2];
        const double per_cell = (double)S.nat / (double)std::max<int64_t>(b.ncells[s2], 1);
        const double nv = (double)S.nvisit;
        est += (double)S.nat * (std::ceil(nv * per_cell / 32.0) + std::ceil(nv / 32.0));
    }
    double w = std::max(1.25 * est, 1.1 * (double)p.mask_hint);
    w = std::min(std::max(w, (double)(int64_t(1) << 20)), (double)(int64_t(1) << 29));
    return (int64_t)w;
}

// Carve the per-call buffers out of the plan's workspace.
static nbl_status layout_workspace(Plan &p, const Batch &b) {
    const int64_t N = b.natoms;
    const int64_t nsys = (int64_t)b.sys.size();
    const int64_t hist = radix_hist_elems(std::max<int64_t>(N, 1));
    Layout L;
    Bufs &B = p.bufs;
    size_t o_pos = b.pos_on_device ? 0 : L.add(sizeof(double) * 3 * N);
    size_t o_pa = (b.per_atom && !b.aux_on_device) ? L.add(sizeof(double) * N) : 0;
    size_t o_ty = (b.types && !b.aux_on_device) ? L.add(sizeof(int32_t) * N) : 0;
    // the small host tables, contiguous (one upload)
    size_t o_sys = L.add(sizeof(SysDev) * nsys);
    size_t o_sab = L.add(sizeof(int64_t) * nsys);
    size_t o_pt64 = L.add(sizeof(double) * std::max<size_t>(b.pt64.size(), 1));
    size_t o_pt32 = L.add(sizeof(float) * std::max<size_t>(b.pt64.size(), 1));
    const size_t tab_end = L.total;
    const int64_t nvis = visit_entries(b);
    size_t o_vis = nvis ? L.add(sizeof(VisitDev) * nvis) : 0;
    size_t o_keys = L.add(sizeof(uint32_t) * N);
    size_t o_vals = L.add(sizeof(int32_t) * N);
    size_t o_keys2 = L.add(sizeof(uint32_t) * N);
    size_t o_vals2 = L.add(sizeof(int32_t) * N);
    size_t o_hist = L.add(sizeof(int32_t) * hist);
    size_t o_hscan = L.add(sizeof(int32_t) * hist);
    size_t o_sscr32 = L.add(sizeof(int32_t) * scan_scratch_elems(hist));
    size_t o_sscr64 = L.add(sizeof(int64_t) * scan_scratch_elems(N + 1));
    size_t o_table = L.add(sizeof(int2) * b.table_size);
    size_t o_hkey = b.grid == kGridHashed ? L.add(sizeof(unsigned long long) * b.table_size) : 0;
    size_t o_pos64 = L.add(sizeof(double4) * N);
    size_t o_pos32 = L.add(sizeof(float4) * N);
    size_t o_aux = L.add(sizeof(int4) * N);
    size_t o_amax = L.add(sizeof(float) * nsys);
    size_t o_home = L.add(sizeof(HomeCell) * N);
    size_t o_cnt = L.add(sizeof(int32_t) * (N + 1));
    // row offsets, then the 8-int flag block right after offsets[N]
    size_t o_off = L.add(sizeof(int64_t) * (N + 1) + sizeof(int) * 8);
    const int64_t mask_cap = mask_words(p, b);
    size_t o_mask = L.add(sizeof(uint32_t) * mask_cap);
    size_t o_hmask = L.add(sizeof(long long) * std::max<int64_t>(N, 1) * kMaskBatches);
    size_t o_items = L.add(sizeof(WorkItem) * std::max<int64_t>(N, 1));
    size_t o_ljp = L.add(sizeof(double) * (size_t)(std::max<int64_t>(N, 1) + N / 1024 + 64));
    nbl_status st = ensure(p.ws.base, p.ws.bytes, L.total, "workspace");
    if (st != NBL_SUCCESS) {
        B = Bufs();  // nothing may point into the released block
        p.have_count = false;
        return st;
    }
    char *base = static_cast<char *>(p.ws.base);
    auto at = [&](size_t off) { return static_cast<void *>(base + off); };
    B.pos = b.pos_on_device ? const_cast<double *>(b.positions) : (double *)at(o_pos);
    B.per_atom = b.per_atom ? (b.aux_on_device ? const_cast<double *>(b.per_atom)
                                               : (double *)at(o_pa))
                            : nullptr;
    B.types = b.types ? (b.aux_on_device ? const_cast<int32_t *>(b.types)
                                         : (int32_t *)at(o_ty))
                      : nullptr;
    B.sys = (SysDev *)at(o_sys);
    B.tab_sab = o_sab - o_sys;
    B.tab_pt64 = o_pt64 - o_sys;
    B.tab_pt32 = o_pt32 - o_sys;
    B.tab_bytes = tab_end - o_sys;
    B.visit = nvis ? (VisitDev *)at(o_vis) : nullptr;
    B.sys_atom_base = (int64_t *)at(o_sab);
    B.pt64 = (double *)at(o_pt64);
    B.pt32 = (float *)at(o_pt32);
    B.keys = (uint32_t *)at(o_keys);
    B.vals = (int32_t *)at(o_vals);
    B.keys2 = (uint32_t *)at(o_keys2);
    B.vals2 = (int32_t *)at(o_vals2);
    B.hist = (int32_t *)at(o_hist);
    B.hist_scan = (int32_t *)at(o_hscan);
    B.scan32 = (int32_t *)at(o_sscr32);
    B.scan64 = (int64_t *)at(o_sscr64);
    B.table = (int2 *)at(o_table);
    B.hkey = b.grid == kGridHashed ? (unsigned long long *)at(o_hkey) : nullptr;
    B.pos64 = (double4 *)at(o_pos64);
    B.pos32 = (float4 *)at(o_pos32);
    B.aux = (int4 *)at(o_aux);
    B.amax = (float *)at(o_amax);
    B.home = (HomeCell *)at(o_home);
    B.counts = (int32_t *)at(o_cnt);
    B.offsets = (int64_t *)at(o_off);
    B.small = reinterpret_cast<int *>(B.offsets + N + 1);
    B.mask_pool = (uint32_t *)at(o_mask);
    B.mask_cap = mask_cap;
    B.home_mask = (long long *)at(o_hmask);
    B.items = (WorkItem *)at(o_items);
    B.lj_part = (double *)at(o_ljp);
    return NBL_SUCCESS;
}

// ---------------------------------------------------------------------------
// batch planning
// ---------------------------------------------------------------------------

nbl_status finish_batch(Batch &b, int grid_req) {
    const int64_t nsys = (int64_t)b.sys.size();
    if (b.natoms > INT32_MAX - 1)
        return set_error(NBL_ERROR_INVALID_ARGUMENT, "more than 2^31-2 atoms");
    int64_t total_cells = 0, total_morton = 0;
    bool morton_ok = true;
    for (int64_t s = 0; s < nsys; s++) {
        const SysDev &S = b.sys[s];
        total_cells += b.ncells[s];
        const int32_t nmax = std::max(S.n[0], std::max(S.n[1], S.n[2]));
        if (nmax > 1024) morton_ok = false;
        const int mb = bits_for((uint64_t)(nmax - 1));
        total_morton += int64_t(1) << (3 * mb);
        if (b.ncells[s] >= (int64_t(1) << kHashSysShift))
            return set_error(NBL_ERROR_INVALID_ARGUMENT, "cell grid too large");
    }
    if (nsys >= (int64_t(1) << (64 - kHashSysShift - 1)))
        return set_error(NBL_ERROR_INVALID_ARGUMENT, "too many systems");
    const int64_t budget = std::max<int64_t>(int64_t(1) << 20, 8 * b.natoms);
    int grid = grid_req;
    if (grid == NBL_GRID_AUTO) grid = total_cells > budget ? NBL_GRID_HASHED : NBL_GRID_DENSE;
    if ((grid == NBL_GRID_DENSE || grid == NBL_GRID_MORTON) &&
        total_cells > (int64_t(1) << 31) - 2)
        grid = NBL_GRID_HASHED;
    if (grid == NBL_GRID_MORTON && (!morton_ok || total_morton > (int64_t(1) << 32) - 2))
        grid = NBL_GRID_DENSE;
    b.grid = grid == NBL_GRID_HASHED ? kGridHashed
             : (grid == NBL_GRID_MORTON ? kGridMorton : kGridDense);
    int64_t cell_base = 0, key_base = 0;
    for (int64_t s = 0; s < nsys; s++) {
        SysDev &S = b.sys[s];
        S.cell_base = cell_base;
        S.key_base = (b.grid == kGridMorton) ? key_base : cell_base;
        cell_base += b.ncells[s];
        const int32_t nmax = std::max(S.n[0], std::max(S.n[1], S.n[2]));
        key_base += int64_t(1) << (3 * bits_for((uint64_t)(nmax - 1)));
    }
    if (b.grid == kGridHashed) {
        int64_t cap = 1;
        const int64_t forced = g_inject_hash_capacity.load();
        while (cap < (forced > 0 ? forced : 2 * std::max<int64_t>(b.natoms, 1) + 1)) cap <<= 1;
        b.table_size = cap;
        b.key_bits = bits_for((uint64_t)(cap - 1));
    } else {
        b.table_size = std::max<int64_t>(total_cells, 1);
        b.key_bits = b.grid == kGridMorton ? bits_for((uint64_t)(key_base - 1))
                                           : bits_for((uint64_t)(total_cells - 1));
    }
    return NBL_SUCCESS;
}

// ---------------------------------------------------------------------------
// count / fill
// ---------------------------------------------------------------------------

// Persistent-style grid: `mult` CTAs per SM (four warps each, one work item
// per warp at a time; mult <= 0: kAutoWaves full waves of the kernel's
// resident CTAs), capped by the number of work items.  The warps take work
// items in a fixed stride, so a grid that is not a whole number of waves
// leaves its last partial wave running alone.
static int traverse_grid(const Plan &p, int64_t natoms, int mult, int mode, bool fp32,
                         int kind, const TravShape &shape, bool lj) {
    if (mult <= 0)
        mult = kAutoWaves * std::max(1, traverse_blocks_per_sm(mode, fp32, kind, shape, lj,
                                                               p.targs.runs != 0));
    const int64_t items = std::max<int64_t>((natoms + 3) / 4, 1);
    return (int)std::min<int64_t>((int64_t)p.num_sms * mult, items);
}

// Home cells per work item the tile builder may join: runs need the dense
// grid (a run's atoms are contiguous in sorted order), the FP32 filter (the
// plain FP64 sweep reads each segment's own offset) and the systems' visit
// tables (a pair's offset vector is looked up there).
static int run_limit(const Plan &p, const Batch &b) {
    if (b.grid != kGridDense || !b.fp32 || p.bufs.visit == nullptr) return 1;
    // left to the device only where the grid is sparse on average (below two
    // atoms per cell); denser grids keep one cell per item and the kernels
    // without run handling
    if (p.max_run == 0 && (double)b.natoms >= 2.0 * (double)b.table_size) return 1;
    return p.max_run;
}

// Atoms per work item (the cell-occupancy tile) for batch b: the launch
// configuration's, or by default chosen from the atom count.  A small system
// has few work items however its cells are cut, and its call time is the
// latency of the longest item, so it is cut finer: single calls through the
// C-ABI measured on one B200 (count + fill + synchronisation) took, at tiles
// of 32 / 16 / 8 / 4 atoms, 122 / 99 / 86 / 79 us for 1,000 atoms (15.6 per
// cell) and 212 / 150 / 117 / 101 us on average over 300 of the batched
// small periodic systems (691 / 397 / 244 / 167 us with the plain FP64
// test).  Large systems keep 32: their cells hold fewer atoms than that.
static int tile_of(const Plan &p, const Batch &b) {
    if (!p.itile_auto) return p.itile;
    if (b.natoms <= 4096) return 4;
    if (b.natoms <= 16384) return 8;
    if (b.natoms <= 65536) return 16;
    return p.itile;
}

// Whether the pair passes run one thread per atom (nbl_trav_atoms.cu) for
// batch b: every system needs its visit table; by default only where the
// occupied cells hold fewer than two atoms on average, so that a warp's work
// item would hold one or two atoms.  The occupied cells are known once a
// count of the same sizes has run on the plan; before that, fewer atoms than
// cells stands in for it.  Measured on 200,000-atom uniform gases (count +
// fill): 2.7x faster at 0.25 atoms per cell (1.1 per occupied cell), 2.0x at
// 0.5 (1.3), 1.35x at 1 (1.6), even at 2 (2.3), slower above; even on a slab
// of 2 atoms per occupied cell.  The force sink always takes the work items.
static bool atom_mode(const Plan &p, const Batch &b) {
    if (p.no_atoms || p.atom_threads < 0 || p.bufs.visit == nullptr) return false;
    if (p.atom_threads > 0) return true;
    if (p.occ_cells > 0 && p.occ_natoms == b.natoms && p.occ_table == b.table_size)
        return (double)b.natoms < 2.0 * (double)p.occ_cells;
    double cells = 0.0;
    for (int64_t n : b.ncells) cells += (double)n;
    return (double)b.natoms < cells;
}

// Size the workspace for a batch and copy its inputs and host tables in.
nbl_status upload_batch(Plan &p, const Batch &b, cudaStream_t st) {
    nbl_status s = layout_workspace(p, b);
    if (s != NBL_SUCCESS) return s;
    Bufs &B = p.bufs;
    const int64_t N = b.natoms;
    const int nsys = (int)b.sys.size();
    p.batch_natoms = N;
    p.batch_nsys = nsys;
    p.batch_fp32 = b.fp32;
    p.batch_grid = b.grid;
    p.have_count = false;

    if (!b.pos_on_device && N > 0)
        NBL_CUDA(cudaMemcpyAsync(B.pos, b.positions, sizeof(double) * 3 * N,
                                 cudaMemcpyHostToDevice, st), "copy positions");
    if (b.per_atom && !b.aux_on_device && N > 0)
        NBL_CUDA(cudaMemcpyAsync(B.per_atom, b.per_atom, sizeof(double) * N,
                                 cudaMemcpyHostToDevice, st), "copy per-atom cutoffs");
    if (b.types && !b.aux_on_device && N > 0)
        NBL_CUDA(cudaMemcpyAsync(B.types, b.types, sizeof(int32_t) * N,
                                 cudaMemcpyHostToDevice, st), "copy types");
    // Small host tables go through the plan's pinned staging so the copies
    // are truly asynchronous and the staging stays valid until they run.
    {
        size_t need = B.tab_bytes + 64;
        if (need > p.host_stage_bytes) {
            if (p.host_stage) {
                cudaStreamSynchronize(st);
                cudaFreeHost(p.host_stage);
            }
            p.host_stage = nullptr;
            p.host_stage_bytes = 0;
            NBL_CUDA(cudaMallocHost(&p.host_stage, need * 2), "pinned staging");
            p.host_stage_bytes = need * 2;
        } else if (p.stage_in_flight) {
            // The previous call's staging copies must have run before reuse.
            NBL_CUDA(cudaEventSynchronize(p.stage_done), "staging reuse");
        }
        // the same layout as the device block at B.sys: one copy
        char *h = static_cast<char *>(p.host_stage);
        std::memcpy(h, b.sys.data(), sizeof(SysDev) * nsys);
        if (B.visit != nullptr) {
            SysDev *hs = reinterpret_cast<SysDev *>(h);
            int64_t base = 0;
            for (int s2 = 0; s2 < nsys; s2++) {
                hs[s2].visit_base = base;
                base += hs[s2].nvisit;
            }
        }
        int64_t *sab = reinterpret_cast<int64_t *>(h + B.tab_sab);
        for (int s2 = 0; s2 < nsys; s2++) sab[s2] = b.sys[s2].atom_base;
        if (!b.pt64.empty()) {
            double *p64 = reinterpret_cast<double *>(h + B.tab_pt64);
            std::memcpy(p64, b.pt64.data(), sizeof(double) * b.pt64.size());
            float *p32 = reinterpret_cast<float *>(h + B.tab_pt32);
            for (size_t k = 0; k < b.pt64.size(); k++) p32[k] = (float)b.pt64[k];
        }
        NBL_CUDA(cudaMemcpyAsync(B.sys, h, B.tab_bytes, cudaMemcpyHostToDevice, st),
                 "copy systems");
        NBL_CUDA(cudaEventRecord(p.stage_done, st), "staging event");
        p.stage_in_flight = true;
    }
    return NBL_SUCCESS;
}

// The argument blocks of the count phase's stages for batch b: binning,
// gather (over the sorted keys / values), and the pair passes' (into
// p.targs, with the passes' grids).
static void bin_args(const Plan &p, const Batch &b, BinArgs &ba) {
    const Bufs &B = p.bufs;
    ba.sys = B.sys;
    ba.sys_atom_base = B.sys_atom_base;
    ba.nsys = (int)b.sys.size();
    ba.grid = b.grid;
    ba.positions = B.pos;
    ba.natoms = b.natoms;
    ba.keys = B.keys;
    ba.vals = B.vals;
    ba.hkey = B.hkey;
    ba.hmask = (unsigned long long)(b.table_size - 1);
    ba.err = B.small + 1;
}

static void gather_args(const Plan &p, const Batch &b, const uint32_t *skeys,
                        const int32_t *svals, GatherArgs &ga) {
    const Bufs &B = p.bufs;
    ga.sys = B.sys;
    ga.sys_atom_base = B.sys_atom_base;
    ga.nsys = (int)b.sys.size();
    ga.grid = b.grid;
    ga.positions = B.pos;
    ga.per_atom = B.per_atom;
    ga.types = B.types;
    ga.natoms = b.natoms;
    ga.keys = skeys;
    ga.vals = svals;
    ga.table = B.table;
    ga.pos64 = B.pos64;
    ga.pos32 = B.pos32;
    ga.aux = B.aux;
    ga.amax = B.amax;
    ga.home = B.home;
    ga.n_home = B.small + 0;
}

static void traverse_args(Plan &p, const Batch &b) {
    const Bufs &B = p.bufs;
    const int64_t N = b.natoms;
    TraverseArgs &ta = p.targs;
    std::memset(&ta, 0, sizeof(ta));
    ta.sys = B.sys;
    ta.visit = B.visit;
    ta.home = B.home;
    ta.n_home = B.small + 0;
    ta.items = B.items;
    ta.n_items = B.small + 3;
    ta.grid = b.grid;
    ta.table = B.table;
    ta.hkey = B.hkey;
    ta.hmask = (unsigned long long)(b.table_size - 1);
    ta.pos64 = B.pos64;
    ta.pos32 = B.pos32;
    ta.aux = B.aux;
    ta.amax = B.amax;
    ta.pt32 = B.pt32;
    ta.pt64 = B.pt64;
    ta.counts = B.counts;
    ta.offsets = B.offsets;
    ta.mask_pool = B.mask_pool;
    ta.mask_cursor = reinterpret_cast<unsigned long long *>(B.small + 4);
    ta.item_next = p.count_tickets ? B.small + 6 : nullptr;
    ta.mask_cap = B.mask_cap;
    ta.home_mask = B.home_mask;
    ta.err = B.small + 1;
    ta.i_lo = p.i_lo;
    ta.i_hi = p.i_hi;
    ta.itile = tile_of(p, b);
    ta.natoms = N;
    ta.runs = run_limit(p, b) != 1 ? 1 : 0;
    ta.atoms = atom_mode(p, b) ? 1 : 0;
    ta.sys_atom_base = B.sys_atom_base;
    ta.nsys = (int)b.sys.size();
    p.batch_kind = b.sys.empty() ? kCutScalar : b.sys[0].cutoff_kind;
    p.trav_grid = traverse_grid(p, N, p.count_mult, kModeCount, b.fp32, p.batch_kind,
                                p.count_shape, false);
    p.fill_grid = traverse_grid(p, N, p.fill_mult, kModeFill, b.fp32, p.batch_kind,
                                p.fill_shape, false);
}

// Enqueue the count phase (bin, sort, gather, work items, count, scan) on a
// batch whose inputs are resident: no host synchronisation, no allocation,
// so it can be captured in a CUDA graph.
nbl_status enqueue_count(Plan &p, const Batch &b, cudaStream_t st) {
    StageRange whole("nbl.count_phase");
    Bufs &B = p.bufs;
    const int64_t N = b.natoms;
    const int nsys = (int)b.sys.size();
    NBL_CUDA(launch_init(B.sys, nsys, B.visit, B.small, B.table, b.table_size, B.amax,
                         b.grid == kGridHashed ? B.hkey : nullptr, p.num_sms, st),
             "k_init");
    BinArgs ba;
    bin_args(p, b, ba);
    {
        StageRange r("nbl.bin");
        NBL_CUDA(launch_bin(ba, st), "k_bin");
    }
    bool in_alt = false;
    {
        StageRange r("nbl.sort");
        NBL_CUDA(radix_sort_pairs(B.keys, B.vals, B.keys2, B.vals2, N, b.key_bits, B.hist,
                                  B.hist_scan, B.scan32, st, &in_alt),
                 "radix sort");
    }
    GatherArgs ga;
    gather_args(p, b, in_alt ? B.keys2 : B.keys, in_alt ? B.vals2 : B.vals, ga);
    const bool atoms = atom_mode(p, b);
    {
        StageRange r("nbl.gather");
        NBL_CUDA(launch_gather(ga, st), "k_gather");
        if (!atoms)  // the thread-per-atom passes need no work items
            NBL_CUDA(launch_tiles(B.home, ga.n_home, B.table, B.sys, B.items, B.small + 3, N,
                                  p.num_sms, tile_of(p, b), run_limit(p, b), st),
                     "k_tiles");
    }
    traverse_args(p, b);
    p.targs.skeys = in_alt ? B.keys2 : B.keys;
    if (p.i_lo > 0 || p.i_hi < N)
        NBL_CUDA(cudaMemsetAsync(B.counts, 0, sizeof(int32_t) * N, st), "memset counts");
    {
        StageRange r("nbl.count");
        TraverseArgs tc = p.targs;
        tc.ticket_ready = 1;  // k_init cleared the ticket
        NBL_CUDA(launch_traverse(kModeCount, b.fp32, p.batch_kind, tc, p.trav_grid, st,
                                 p.count_shape),
                 "count pass");
    }
    {
        StageRange r("nbl.scan");
        NBL_CUDA(exclusive_scan_i32_i64(B.counts, N, B.offsets, B.scan64, st), "scan");
    }
    return NBL_SUCCESS;
}

// Whether batch b takes the one-launch count phase (nbl_small.cu): one system of
// up to p.small_atoms atoms on a dense grid of at most kSmallMaxCells cells,
// every row.
static bool small_path(const Plan &p, const Batch &b) {
    return p.small_atoms > 0 && b.sys.size() == 1 && b.natoms >= 1 &&
           b.natoms <= std::min<int64_t>(p.small_atoms, kSmallMaxAtoms) &&
           b.grid == kGridDense && b.table_size <= kSmallMaxCells && p.i_lo <= 0 &&
           p.i_hi >= b.natoms;
}

// The count phase of a small system as one launch: the same buffers as
// enqueue_count leaves (the fill and the other consumers follow unchanged).
static nbl_status enqueue_count_small(Plan &p, const Batch &b, cudaStream_t st) {
    StageRange whole("nbl.count_phase");
    Bufs &B = p.bufs;
    SmallCountArgs sa;
    bin_args(p, b, sa.bin);
    gather_args(p, b, B.keys, B.vals, sa.gather);
    traverse_args(p, b);
    p.targs.atoms = 0;  // the one-launch count builds work items for the warp passes
    // Work items of at most 8 atoms: a small system's passes are bound by the
    // latency of one item, which shrinks with its tile (100 atoms: 74 -> 62 us
    // for count + fill + synchronisation against 32-atom items).
    p.targs.itile = p.itile_auto ? kSmallTile : std::min(p.itile, kSmallTile);
    sa.trav = p.targs;
    sa.trav.item_next = p.count_tickets ? B.small + 6 : nullptr;
    sa.ncells = b.table_size;
    sa.small = B.small;
    sa.items_count = B.small + 3;
    sa.offsets = B.offsets;
    // one CTA up to 128 atoms, else a cluster of up to 8 (about one work item
    // per warp)
    const int ctas = (int)std::min<int64_t>(kSmallMaxCtas, (b.natoms + 127) / 128);
    NBL_CUDA(launch_count_small(b.fp32, p.batch_kind, sa, ctas, st), "one-launch count phase");
    return NBL_SUCCESS;
}

void drop_count_graph(Plan &p) {
    if (p.count_graph) cudaGraphExecDestroy(p.count_graph);
    p.count_graph = nullptr;
    p.have_last_key = false;
}

static CountKey count_key(const Plan &p, const Batch &b) {
    CountKey k;
    k.ws_base = p.ws.base;
    k.pos = p.bufs.pos;
    k.per_atom = p.bufs.per_atom;
    k.types = p.bufs.types;
    k.natoms = b.natoms;
    k.table_size = b.table_size;
    k.mask_cap = p.bufs.mask_cap;
    k.pt_size = (int64_t)b.pt64.size();
    k.i_lo = p.i_lo;
    k.i_hi = p.i_hi;
    k.nsys = (int32_t)b.sys.size();
    k.grid = b.grid;
    k.key_bits = b.key_bits;
    k.fp32 = b.fp32 ? 1 : 0;
    k.kind = b.sys.empty() ? kCutScalar : b.sys[0].cutoff_kind;
    k.itile = tile_of(p, b);
    k.max_run = run_limit(p, b);
    k.nvisit_tab = p.bufs.visit != nullptr ? 1 : 0;
    k.count_mult = p.count_mult;
    k.count_warps = p.count_shape.warps;
    k.count_cand = p.count_shape.cand;
    k.count_group = p.count_shape.group;
    k.count_tickets = p.count_tickets ? 1 : 0;
    k.atoms = atom_mode(p, b) ? 1 : 0;
    return k;
}

// Captures the count phase into p.count_graph (on the plan's own stream; the
// capture runs nothing).  False if the capture fails: direct launches then.
static bool capture_count(Plan &p, const Batch &b, const CountKey &k) {
    if (!p.capture_stream &&
        cudaStreamCreateWithFlags(&p.capture_stream, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    const long long before = g_launches;
    if (cudaStreamBeginCapture(p.capture_stream, cudaStreamCaptureModeThreadLocal) !=
        cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    const nbl_status s = enqueue_count(p, b, p.capture_stream);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(p.capture_stream, &g);
    if (s != NBL_SUCCESS || e != cudaSuccess || g == nullptr) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        return false;
    }
    if (p.count_graph) cudaGraphExecDestroy(p.count_graph);
    p.count_graph = nullptr;
    const cudaError_t ie = cudaGraphInstantiate(&p.count_graph, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) {
        p.count_graph = nullptr;
        cudaGetLastError();
        return false;
    }
    p.graph_launches = g_launches - before;
    count_launch((int)-p.graph_launches);  // nothing ran yet: counted at each replay
    p.graph_key = k;
    p.graph_targs = p.targs;
    p.graph_trav_grid = p.trav_grid;
    p.graph_kind = p.batch_kind;
    return true;
}

nbl_status run_count(Plan &p, const Batch &b, cudaStream_t st, bool sync) {
    nbl_status s = upload_batch(p, b, st);
    if (s != NBL_SUCCESS) return s;
    const bool small = sync && small_path(p, b);
    // Single calls: replay the captured count phase while the launch key
    // repeats (captured on the second call with the same key); a small
    // system's count phase is one launch already.
    bool replay = false;
    if (sync && !small && !p.graphs_off) {
        const CountKey k = count_key(p, b);
        if (p.count_graph && k == p.graph_key) {
            replay = true;
        } else if (p.have_last_key && k == p.last_key) {
            replay = capture_count(p, b, k);
            if (!replay) {
                p.graphs_off = true;
                drop_count_graph(p);
            }
        }
        p.last_key = k;
        p.have_last_key = true;
    }
    if (replay) {
        p.targs = p.graph_targs;
        p.trav_grid = p.graph_trav_grid;
        p.batch_kind = p.graph_kind;
        // the fill's shape is not part of the count key
        p.fill_grid = traverse_grid(p, b.natoms, p.fill_mult, kModeFill, b.fp32, p.batch_kind,
                                    p.fill_shape, false);
        NBL_CUDA(cudaGraphLaunch(p.count_graph, st), "count-phase graph");
        count_launch((int)p.graph_launches);
    } else {
        s = small ? enqueue_count_small(p, b, st) : enqueue_count(p, b, st);
        if (s != NBL_SUCCESS) return s;
    }
    Bufs &B = p.bufs;
    const int64_t N = b.natoms;
    if (sync) {
        // pair count and flags in one copy (the flag block follows offsets[N])
        NBL_CUDA(cudaMemcpyAsync(p.host_small, B.offsets + N, sizeof(int64_t) + sizeof(int) * 6,
                                 cudaMemcpyDeviceToHost, st), "read pair count and flags");
        NBL_CUDA(cudaStreamSynchronize(st), "count phase");
        p.stage_in_flight = false;
        int flags[6];
        std::memcpy(flags, p.host_small + 1, sizeof(flags));
        p.npairs = p.host_small[0];
        if (flags[0] > 0) {  // occupied cells, for the next call's choice of passes
            p.occ_natoms = N;
            p.occ_table = b.table_size;
            p.occ_cells = flags[0];
        }
        unsigned long long demand = 0;  // mask-pool words the count asked for
        std::memcpy(&demand, flags + 4, sizeof(demand));
        p.mask_hint = (int64_t)demand;
        if (flags[1] & kErrRange)
            return set_error(NBL_ERROR_RANGE,
                             "positions must be finite and within 2^29 cells of the box");
        if (flags[1] & kErrInternal)
            return set_error(NBL_ERROR_INTERNAL, "device-side bound exceeded in count phase");
    }
    p.have_count = true;
    return NBL_SUCCESS;
}

nbl_status run_fill(Plan &p, const nbl_outputs &o, int64_t capacity, cudaStream_t st) {
    if (!p.have_count)
        return set_error(NBL_ERROR_INVALID_ARGUMENT, "nbl_fill without a preceding nbl_count");
    TraverseArgs ta = p.targs;
    ta.item_next = p.fill_tickets ? p.bufs.small + 6 : nullptr;
    ta.first = o.first;
    ta.second = o.second;
    ta.distvec = o.distvec;
    ta.absdist = o.absdist;
    ta.shift = o.shift;
    ta.capacity = capacity;
    if (!(o.first || o.second || o.distvec || o.absdist || o.shift)) return NBL_SUCCESS;
    StageRange r("nbl.fill");
    NBL_CUDA(launch_traverse(kModeFill, p.batch_fp32, p.batch_kind, ta, p.fill_grid, st,
                             p.fill_shape),
             "fill pass");
    return NBL_SUCCESS;
}

// The device flags of the last count / fill as a status; with `copy`, first
// reads them (synchronising `st`), else they were read already.
nbl_status read_flags(Plan &p, cudaStream_t st, bool copy) {
    if (copy) {
        NBL_CUDA(cudaMemcpyAsync(p.host_small + 1, p.bufs.small, sizeof(int) * 2,
                                 cudaMemcpyDeviceToHost, st), "read flags");
        NBL_CUDA(cudaStreamSynchronize(st), "check");
    }
    int flags[2];
    std::memcpy(flags, p.host_small + 1, sizeof(flags));
    if (flags[1] & kErrRange)
        return set_error(NBL_ERROR_RANGE,
                         "positions must be finite and within 2^29 cells of the box");
    if (flags[1] & kErrCapacity)
        return set_error(NBL_ERROR_CAPACITY, "output capacity smaller than the pair count");
    if (flags[1] & kErrInternal)
        return set_error(NBL_ERROR_INTERNAL, "device-side bound exceeded");
    return NBL_SUCCESS;
}

// The plan's launch configuration in C-ABI form.
void launch_config_of(const Plan &p, nbl_launch_config *cfg) {
    cfg->count_ctas_per_sm = p.count_mult;
    cfg->fill_ctas_per_sm = p.fill_mult;
    cfg->count_strided = p.count_tickets ? 0 : 1;
    cfg->fill_strided = p.fill_tickets ? 0 : 1;
    cfg->count_warps = p.count_shape.warps;
    cfg->fill_warps = p.fill_shape.warps;
    cfg->count_group = p.count_shape.group;
    cfg->count_large_staging = p.count_shape.cand;
    cfg->atoms_per_item = p.itile_auto ? 0 : p.itile;
    cfg->cells_per_item = p.max_run;
    cfg->one_launch_atoms = p.small_atoms == kSmallDefaultAtoms ? 0
                            : p.small_atoms > 0                ? p.small_atoms
                                                               : -1;
    cfg->thread_per_atom = p.atom_threads;
}

// Request -> one-system batch.
nbl_status batch_from_request(const nbl_request *req, Batch &b) {
    if (!req) return set_error(NBL_ERROR_INVALID_ARGUMENT, "null request");
    if (req->quantities & ~31)
        return set_error(NBL_ERROR_INVALID_ARGUMENT, "Unsupported quantity specified.");
    if (req->nat < 0) return set_error(NBL_ERROR_INVALID_ARGUMENT, "negative atom count");
    if (!req->cell_origin || !req->cell || !req->inv_cell || !req->pbc)
        return set_error(NBL_ERROR_INVALID_ARGUMENT, "missing geometry");
    if (req->nat > 0 && !req->positions)
        return set_error(NBL_ERROR_INVALID_ARGUMENT, "missing positions");
    if (req->per_type_cutoff_sq && req->ncutoffs < 0)
        return set_error(NBL_ERROR_INVALID_ARGUMENT, "negative ncutoffs");
    if (req->precision != NBL_PRECISION_FP32_FILTER && req->precision != NBL_PRECISION_FP64)
        return set_error(NBL_ERROR_INVALID_ARGUMENT, "unknown precision");
    if (req->grid < NBL_GRID_AUTO || req->grid > NBL_GRID_HASHED)
        return set_error(NBL_ERROR_INVALID_ARGUMENT, "unknown grid");
    b = Batch();
    SysDev S;
    int64_t ncells = 0;
    nbl_status st = plan_system(req->cell_origin, req->cell, req->inv_cell, req->pbc,
                                req->cutoff, S, ncells);
    if (st != NBL_SUCCESS) return st;
    S.nat = (int32_t)req->nat;
    S.atom_base = 0;
    if (req->per_atom_cutoff) {
        S.cutoff_kind = kCutPerAtom;
    } else if (req->per_type_cutoff_sq && req->types) {
        S.cutoff_kind = kCutPerType;
        S.ncutoffs = req->ncutoffs;
        S.pt_base = 0;
        b.pt64.assign(req->per_type_cutoff_sq,
                      req->per_type_cutoff_sq + (size_t)req->ncutoffs * req->ncutoffs);
    } else {
        S.cutoff_kind = kCutScalar;
    }
    b.sys.push_back(S);
    b.ncells.push_back(ncells);
    b.natoms = req->nat;
    b.positions = req->positions;
    b.pos_on_device = req->positions_on_device != 0;
    b.per_atom = S.cutoff_kind == kCutPerAtom ? req->per_atom_cutoff : nullptr;
    b.types = S.cutoff_kind == kCutPerType ? req->types : nullptr;
    b.aux_on_device = req->aux_on_device != 0;
    b.fp32 = req->precision == NBL_PRECISION_FP32_FILTER;
    b.quantities = req->quantities;
    return finish_batch(b, req->grid);
}

// RAII device switch.
struct DeviceGuard {
    int prev = -1;
    bool ok = true;
    explicit DeviceGuard(int dev) {
        int cur = 0;
        if (cudaGetDevice(&cur) != cudaSuccess) {
            ok = false;
            return;
        }
        if (dev >= 0 && dev != cur) {
            if (cudaSetDevice(dev) != cudaSuccess) ok = false;
            prev = cur;
        }
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

nbl_status plan_init(Plan &p, int device_id) {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return set_error(NBL_ERROR_NO_DEVICE, "no CUDA device available");
    }
    int dev = device_id;
    if (dev < 0) NBL_CUDA(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev >= ndev) return set_error(NBL_ERROR_INVALID_ARGUMENT, "no device %d", dev);
    p.device = dev;
    DeviceGuard g(dev);
    NBL_CUDA(cudaDeviceGetAttribute(&p.num_sms, cudaDevAttrMultiProcessorCount, dev),
             "device query");
    NBL_CUDA(cudaMallocHost(&p.host_small, sizeof(int64_t) * 4), "pinned");
    NBL_CUDA(cudaEventCreateWithFlags(&p.stage_done, cudaEventDisableTiming), "event");
    return NBL_SUCCESS;
}

void plan_free(Plan &p) {
    DeviceGuard g(p.device);
    if (p.stage_done) cudaEventSynchronize(p.stage_done);
    drop_count_graph(p);
    if (p.capture_stream) cudaStreamDestroy(p.capture_stream);
    p.capture_stream = nullptr;
    p.ws.release();
    if (p.host_small) cudaFreeHost(p.host_small);
    if (p.host_stage) cudaFreeHost(p.host_stage);
    if (p.host_out) cudaFreeHost(p.host_out);
    if (p.stage_done) cudaEventDestroy(p.stage_done);
    p.host_small = nullptr;
    p.host_stage = nullptr;
    p.host_out = nullptr;
    p.host_out_bytes = 0;
    p.stage_done = nullptr;
}

}  // namespace nbl

using namespace nbl;

struct nbl_plan {
    Plan p;
};

extern "C" {

nbl_status nbl_plan_create(int device_id, nbl_plan **plan) {
    clear_error();
    if (!plan) return set_error(NBL_ERROR_INVALID_ARGUMENT, "null plan pointer");
    *plan = nullptr;
    nbl_plan *np = new (std::nothrow) nbl_plan();
    if (!np) return set_error(NBL_ERROR_OUT_OF_MEMORY, "host allocation failed");
    nbl_status st = plan_init(np->p, device_id);
    if (st != NBL_SUCCESS) {
        plan_free(np->p);
        delete np;
        return st;
    }
    *plan = np;
    return NBL_SUCCESS;
}

nbl_status nbl_plan_destroy(nbl_plan *plan) {
    clear_error();
    if (!plan) return NBL_SUCCESS;
    plan_free(plan->p);
    delete plan;
    return NBL_SUCCESS;
}

nbl_status nbl_plan_trim(nbl_plan *plan) {
    clear_error();
    if (!plan) return set_error(NBL_ERROR_INVALID_ARGUMENT, "null plan");
    DeviceGuard g(plan->p.device);
    cudaDeviceSynchronize();
    drop_count_graph(plan->p);
    plan->p.ws.release();
    plan->p.have_count = false;
    return NBL_SUCCESS;
}

nbl_status nbl_set_atom_range(nbl_plan *plan, int64_t lo, int64_t hi) {
    clear_error();
    if (!plan) return set_error(NBL_ERROR_INVALID_ARGUMENT, "null plan");
    if (hi < 0) hi = INT64_MAX;
    if (lo < 0 || lo > hi)
        return set_error(NBL_ERROR_INVALID_ARGUMENT, "bad atom range [%lld, %lld)",
                         (long long)lo, (long long)hi);
    plan->p.i_lo = lo;
    plan->p.i_hi = hi;
    return NBL_SUCCESS;
}

nbl_status nbl_debug_inject(int what, int64_t value) {
    clear_error();
    if (value < 0) return set_error(NBL_ERROR_INVALID_ARGUMENT, "negative injection value");
    if (what == NBL_INJECT_ALLOC_FAILURES) {
        g_inject_alloc_failures.store(value);
    } else if (what == NBL_INJECT_HASH_CAPACITY) {
        if (value > (int64_t(1) << 40))
            return set_error(NBL_ERROR_INVALID_ARGUMENT, "hash capacity too large");
        g_inject_hash_capacity.store(value);
    } else {
        return set_error(NBL_ERROR_INVALID_ARGUMENT, "unknown injection %d", what);
    }
    return NBL_SUCCESS;
}

nbl_status nbl_plan_set_launch(nbl_plan *plan, int count_ctas_per_sm, int count_group,
                               int fill_ctas_per_sm) {
    clear_error();
    if (!plan) return set_error(NBL_ERROR_INVALID_ARGUMENT, "null plan");
    if (count_ctas_per_sm < 0 || count_ctas_per_sm > 64 || fill_ctas_per_sm < 0 ||
        fill_ctas_per_sm > 64 || !(count_group == 0 || count_group == 2 || count_group == 4))
        return set_error(NBL_ERROR_INVALID_ARGUMENT,
                         "launch: CTAs per SM in [0, 64], count group 0, 2 or 4");
    plan->p.count_mult = count_ctas_per_sm;
    plan->p.fill_mult = fill_ctas_per_sm;
    plan->p.count_shape.group = count_group == 0 ? 4 : count_group;
    return NBL_SUCCESS;
}

nbl_status nbl_plan_set_launch_config(nbl_plan *plan, const nbl_launch_config *cfg) {
    clear_error();
    if (!plan || !cfg) return set_error(NBL_ERROR_INVALID_ARGUMENT, "null argument");
    TravShape cs, fs;
    cs.warps = cfg->count_warps == 0 ? 4 : cfg->count_warps;
    cs.cand = cfg->count_large_staging;
    cs.group = cfg->count_group == 0 ? 4 : cfg->count_group;
    fs.warps = cfg->fill_warps == 0 ? default_fill_shape().warps : cfg->fill_warps;
    const int itile = cfg->atoms_per_item == 0 ? 32 : cfg->atoms_per_item;
    if (cfg->count_ctas_per_sm < 0 || cfg->count_ctas_per_sm > 64 || cfg->fill_ctas_per_sm < 0 ||
        cfg->fill_ctas_per_sm > 64 || itile < 1 || itile > 32 || cfg->cells_per_item < 0 ||
        cfg->cells_per_item > kMaxRun || cfg->one_launch_atoms < -1 ||
        cfg->one_launch_atoms > kSmallMaxAtoms || !traverse_shape_ok(kModeCount, true, cs) ||
        !traverse_shape_ok(kModeFill, true, fs) || cfg->thread_per_atom < -1 ||
        cfg->thread_per_atom > 1)
        return set_error(NBL_ERROR_INVALID_ARGUMENT,
                         "launch config: CTAs per SM in [0, 64], warps 2, 4 or 8, count group "
                         "2 or 4, large candidate staging 0 or 1, atoms per item in [1, 32], "
                         "cells per item in [0, %d], single-CTA atoms in [-1, %d], thread per "
                         "atom -1, 0 or 1", kMaxRun, kSmallMaxAtoms);
    plan->p.count_mult = cfg->count_ctas_per_sm;
    plan->p.fill_mult = cfg->fill_ctas_per_sm;
    plan->p.count_tickets = cfg->count_strided == 0;
    plan->p.fill_tickets = cfg->fill_strided == 0;
    plan->p.count_shape = cs;
    plan->p.fill_shape = fs;
    plan->p.itile = itile;
    plan->p.itile_auto = cfg->atoms_per_item == 0;
    plan->p.max_run = cfg->cells_per_item;
    plan->p.small_atoms = cfg->one_launch_atoms == 0   ? kSmallDefaultAtoms
                          : cfg->one_launch_atoms < 0 ? 0
                                                      : cfg->one_launch_atoms;
    plan->p.atom_threads = cfg->thread_per_atom;
    return NBL_SUCCESS;
}

nbl_status nbl_plan_get_launch_config(nbl_plan *plan, nbl_launch_config *cfg) {
    clear_error();
    if (!plan || !cfg) return set_error(NBL_ERROR_INVALID_ARGUMENT, "null argument");
    launch_config_of(plan->p, cfg);
    return NBL_SUCCESS;
}

nbl_status nbl_count(nbl_plan *plan, const nbl_request *req, void *stream,
                     int64_t *npairs) {
    clear_error();
    if (!plan || !npairs) return set_error(NBL_ERROR_INVALID_ARGUMENT, "null argument");
    *npairs = 0;
    plan->p.have_count = false;
    Batch b;
    nbl_status st = batch_from_request(req, b);
    if (st != NBL_SUCCESS) return st;
    if (req->device_id >= 0 && req->device_id != plan->p.device)
        return set_error(NBL_ERROR_INVALID_ARGUMENT, "request device %d != plan device %d",
                         req->device_id, plan->p.device);
    DeviceGuard g(plan->p.device);
    if (!g.ok) return set_error(NBL_ERROR_CUDA, "cannot select device %d", plan->p.device);
    st = run_count(plan->p, b, static_cast<cudaStream_t>(stream), true);
    if (st != NBL_SUCCESS) return st;
    plan->p.quantities = req->quantities;
    *npairs = plan->p.npairs;
    return NBL_SUCCESS;
}

nbl_status nbl_fill(nbl_plan *plan, const nbl_outputs *out, void *stream) {
    clear_error();
    if (!plan || !out) return set_error(NBL_ERROR_INVALID_ARGUMENT, "null argument");
    DeviceGuard g(plan->p.device);
    return run_fill(plan->p, *out, plan->p.npairs, static_cast<cudaStream_t>(stream));
}

nbl_status nbl_fill_host(nbl_plan *plan, const nbl_outputs *host_out, void *stream) {
    clear_error();
    if (!plan || !host_out) return set_error(NBL_ERROR_INVALID_ARGUMENT, "null argument");
    Plan &p = plan->p;
    if (!p.have_count)
        return set_error(NBL_ERROR_INVALID_ARGUMENT, "nbl_fill_host without nbl_count");
    DeviceGuard g(p.device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int64_t np = p.npairs;
    if (np == 0) return NBL_SUCCESS;
    const nbl_outputs &h = *host_out;
    Layout L;
    size_t o_i = h.first ? L.add(sizeof(int32_t) * np) : 0;
    size_t o_j = h.second ? L.add(sizeof(int32_t) * np) : 0;
    size_t o_D = h.distvec ? L.add(sizeof(double) * 3 * np) : 0;
    size_t o_d = h.absdist ? L.add(sizeof(double) * np) : 0;
    size_t o_S = h.shift ? L.add(sizeof(int32_t) * 3 * np) : 0;
    nbl_status s = ensure(p.ws.out_base, p.ws.out_bytes, std::max<size_t>(L.total, 256),
                          "output scratch");
    if (s != NBL_SUCCESS) return s;
    char *base = static_cast<char *>(p.ws.out_base);
    nbl_outputs d;
    d.first = h.first ? (int32_t *)(base + o_i) : nullptr;
    d.second = h.second ? (int32_t *)(base + o_j) : nullptr;
    d.distvec = h.distvec ? (double *)(base + o_D) : nullptr;
    d.absdist = h.absdist ? (double *)(base + o_d) : nullptr;
    d.shift = h.shift ? (int32_t *)(base + o_S) : nullptr;
    s = run_fill(p, d, np, st);
    if (s != NBL_SUCCESS) return s;
    // Small lists: one copy of the contiguous outputs (and the flags) into the
    // plan's pinned landing area, then host copies into the caller's arrays --
    // cheaper than one device->host copy per quantity below a few hundred KB.
    constexpr size_t kOneCopyBytes = 256 << 10;
    if (L.total <= kOneCopyBytes) {
        if (L.total > p.host_out_bytes) {
            if (p.host_out) cudaFreeHost(p.host_out);
            p.host_out = nullptr;
            p.host_out_bytes = 0;
            NBL_CUDA(cudaMallocHost(&p.host_out, kOneCopyBytes), "pinned landing area");
            p.host_out_bytes = kOneCopyBytes;
        }
        NBL_CUDA(cudaMemcpyAsync(p.host_out, base, L.total, cudaMemcpyDeviceToHost, st),
                 "copy outputs");
        NBL_CUDA(cudaMemcpyAsync(p.host_small + 1, p.bufs.small, sizeof(int) * 2,
                                 cudaMemcpyDeviceToHost, st), "read flags");
        NBL_CUDA(cudaStreamSynchronize(st), "fill");
        const char *hb = static_cast<const char *>(p.host_out);
        if (h.first) std::memcpy(h.first, hb + o_i, sizeof(int32_t) * np);
        if (h.second) std::memcpy(h.second, hb + o_j, sizeof(int32_t) * np);
        if (h.distvec) std::memcpy(h.distvec, hb + o_D, sizeof(double) * 3 * np);
        if (h.absdist) std::memcpy(h.absdist, hb + o_d, sizeof(double) * np);
        if (h.shift) std::memcpy(h.shift, hb + o_S, sizeof(int32_t) * 3 * np);
        return read_flags(p, st, false);
    }
    if (h.first)
        NBL_CUDA(cudaMemcpyAsync(h.first, d.first, sizeof(int32_t) * np,
                                 cudaMemcpyDeviceToHost, st), "copy i");
    if (h.second)
        NBL_CUDA(cudaMemcpyAsync(h.second, d.second, sizeof(int32_t) * np,
                                 cudaMemcpyDeviceToHost, st), "copy j");
    if (h.distvec)
        NBL_CUDA(cudaMemcpyAsync(h.distvec, d.distvec, sizeof(double) * 3 * np,
                                 cudaMemcpyDeviceToHost, st), "copy D");
    if (h.absdist)
        NBL_CUDA(cudaMemcpyAsync(h.absdist, d.absdist, sizeof(double) * np,
                                 cudaMemcpyDeviceToHost, st), "copy d");
    if (h.shift)
        NBL_CUDA(cudaMemcpyAsync(h.shift, d.shift, sizeof(int32_t) * 3 * np,
                                 cudaMemcpyDeviceToHost, st), "copy S");
    return read_flags(p, st);
}

nbl_status nbl_fill_matrix(nbl_plan *plan, int32_t max_neighbours, int32_t *idx,
                           double *dist, int32_t *count, int *overflow, void *stream) {
    clear_error();
    if (!plan || !idx || !dist || !count || !overflow || max_neighbours <= 0)
        return set_error(NBL_ERROR_INVALID_ARGUMENT, "bad neighbour-matrix arguments");
    Plan &p = plan->p;
    if (!p.have_count) return set_error(NBL_ERROR_INVALID_ARGUMENT, "no count phase");
    DeviceGuard g(p.device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int64_t n = p.batch_natoms;
    const size_t nk = (size_t)n * (size_t)max_neighbours;
    *overflow = 0;
    if (n == 0) return NBL_SUCCESS;
    NBL_CUDA(cudaMemsetAsync(idx, 0, sizeof(int32_t) * nk, st), "memset matrix");
    NBL_CUDA(cudaMemsetAsync(dist, 0, sizeof(double) * 3 * nk, st), "memset matrix");
    NBL_CUDA(cudaMemsetAsync(count, 0, sizeof(int32_t) * n, st), "memset matrix");
    NBL_CUDA(cudaMemsetAsync(p.bufs.small + 2, 0, sizeof(int), st), "memset flag");
    TraverseArgs ta = p.targs;
    ta.item_next = p.fill_tickets ? p.bufs.small + 6 : nullptr;
    ta.mat_k = max_neighbours;
    ta.mat_idx = idx;
    ta.mat_dist = dist;
    ta.mat_count = count;
    ta.mat_overflow = p.bufs.small + 2;
    ta.capacity = 0;
    NBL_CUDA(launch_traverse(kModeFill, p.batch_fp32, p.batch_kind, ta, p.fill_grid, st,
                             p.fill_shape),
             "matrix fill");
    NBL_CUDA(cudaMemcpyAsync(p.host_small + 2, p.bufs.small + 2, sizeof(int),
                             cudaMemcpyDeviceToHost, st), "read overflow");
    nbl_status r = read_flags(p, st);
    int ov = 0;
    std::memcpy(&ov, p.host_small + 2, sizeof(int));
    *overflow = ov ? 1 : 0;
    return r;
}

nbl_status nbl_lj_forces(nbl_plan *plan, const nbl_request *req, double epsilon,
                         double sigma, double *forces, double *energy, void *stream) {
    clear_error();
    if (!plan || !req || !energy || (!forces && req->nat > 0))
        return set_error(NBL_ERROR_INVALID_ARGUMENT, "null argument");
    if (!(std::isfinite(epsilon) && std::isfinite(sigma)))
        return set_error(NBL_ERROR_INVALID_ARGUMENT, "epsilon and sigma must be finite");
    plan->p.have_count = false;
    Batch b;
    nbl_status st = batch_from_request(req, b);
    if (st != NBL_SUCCESS) return st;
    if (req->device_id >= 0 && req->device_id != plan->p.device)
        return set_error(NBL_ERROR_INVALID_ARGUMENT, "request device %d != plan device %d",
                         req->device_id, plan->p.device);
    DeviceGuard g(plan->p.device);
    if (!g.ok) return set_error(NBL_ERROR_CUDA, "cannot select device %d", plan->p.device);
    cudaStream_t cs = static_cast<cudaStream_t>(stream);
    Plan &p = plan->p;
    p.no_atoms = true;  // the force sink takes the work items
    st = run_count(p, b, cs, false);
    p.no_atoms = false;
    if (st != NBL_SUCCESS) return st;
    if (b.natoms == 0) {
        NBL_CUDA(cudaMemsetAsync(energy, 0, sizeof(double), cs), "memset energy");
        return NBL_SUCCESS;
    }
    TraverseArgs ta = p.targs;
    ta.item_next = p.fill_tickets ? p.bufs.small + 6 : nullptr;
    ta.first = ta.second = nullptr;
    ta.distvec = ta.absdist = nullptr;
    ta.shift = nullptr;
    ta.capacity = 0;
    ta.lj_force = forces;
    ta.lj_energy = p.bufs.lj_part;
    ta.lj_eps4 = 4.0 * epsilon;
    ta.lj_eps24 = 24.0 * epsilon;
    ta.lj_sig2 = sigma * sigma;
    const int grid = traverse_grid(p, b.natoms, p.fill_mult, kModeFill, p.batch_fp32,
                                   p.batch_kind, TravShape(), true);
    NBL_CUDA(launch_traverse(kModeFill, p.batch_fp32, p.batch_kind, ta, grid, cs),
             "force pass");
    NBL_CUDA(launch_lj_energy(p.bufs.lj_part, b.natoms, p.bufs.lj_part + b.natoms, energy,
                              cs),
             "energy");
    return NBL_SUCCESS;
}

nbl_status nbl_counts(nbl_plan *plan, int32_t *counts, void *stream) {
    clear_error();
    if (!plan || !counts) return set_error(NBL_ERROR_INVALID_ARGUMENT, "null argument");
    Plan &p = plan->p;
    if (!p.have_count) return set_error(NBL_ERROR_INVALID_ARGUMENT, "no count phase");
    DeviceGuard g(p.device);
    if (p.batch_natoms > 0)
        NBL_CUDA(cudaMemcpyAsync(counts, p.bufs.counts, sizeof(int32_t) * p.batch_natoms,
                                 cudaMemcpyDeviceToDevice, static_cast<cudaStream_t>(stream)),
                 "copy counts");
    return NBL_SUCCESS;
}

nbl_status nbl_row_offsets(nbl_plan *plan, int64_t *offsets, void *stream) {
    clear_error();
    if (!plan || !offsets) return set_error(NBL_ERROR_INVALID_ARGUMENT, "null argument");
    Plan &p = plan->p;
    if (!p.have_count) return set_error(NBL_ERROR_INVALID_ARGUMENT, "no count phase");
    DeviceGuard g(p.device);
    NBL_CUDA(cudaMemcpyAsync(offsets, p.bufs.offsets, sizeof(int64_t) * (p.batch_natoms + 1),
                             cudaMemcpyDeviceToDevice, static_cast<cudaStream_t>(stream)),
             "copy offsets");
    return NBL_SUCCESS;
}

nbl_status nbl_check(nbl_plan *plan, void *stream) {
    clear_error();
    if (!plan) return set_error(NBL_ERROR_INVALID_ARGUMENT, "null plan");
    DeviceGuard g(plan->p.device);
    return read_flags(plan->p, static_cast<cudaStream_t>(stream));
}

nbl_status nbl_neighbour_list_device(const nbl_request *req, void *stream,
                                     nbl_device_result *result) {
    clear_error();
    if (!req || !result) return set_error(NBL_ERROR_INVALID_ARGUMENT, "null argument");
    std::memset(result, 0, sizeof(*result));
    // One cached plan per (host thread, device).
    static thread_local std::vector<nbl_plan *> plans;
    int dev = req->device_id;
    if (dev < 0) {
        if (cudaGetDevice(&dev) != cudaSuccess) {
            cudaGetLastError();
            return set_error(NBL_ERROR_NO_DEVICE, "no CUDA device available");
        }
    }
    if ((int)plans.size() <= dev) plans.resize(dev + 1, nullptr);
    if (!plans[dev]) {
        nbl_status st = nbl_plan_create(dev, &plans[dev]);
        if (st != NBL_SUCCESS) return st;
    }
    nbl_plan *plan = plans[dev];
    int64_t np = 0;
    nbl_status st = nbl_count(plan, req, stream, &np);
    if (st != NBL_SUCCESS) return st;
    DeviceGuard g(dev);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    result->npairs = np;
    result->device_id = dev;
    const int q = req->quantities;
    const size_t n1 = std::max<int64_t>(np, 1);
    nbl_outputs o;
    std::memset(&o, 0, sizeof(o));
    if (q & NBL_QUANTITY_FIRST)
        NBL_CUDA(cudaMallocAsync((void **)&result->first, sizeof(int32_t) * n1, s), "alloc i");
    if (q & NBL_QUANTITY_SECOND)
        NBL_CUDA(cudaMallocAsync((void **)&result->second, sizeof(int32_t) * n1, s), "alloc j");
    if (q & NBL_QUANTITY_DISTVEC)
        NBL_CUDA(cudaMallocAsync((void **)&result->distvec, sizeof(double) * 3 * n1, s),
                 "alloc D");
    if (q & NBL_QUANTITY_ABSDIST)
        NBL_CUDA(cudaMallocAsync((void **)&result->absdist, sizeof(double) * n1, s), "alloc d");
    if (q & NBL_QUANTITY_SHIFT)
        NBL_CUDA(cudaMallocAsync((void **)&result->shift, sizeof(int32_t) * 3 * n1, s),
                 "alloc S");
    o.first = result->first;
    o.second = result->second;
    o.distvec = result->distvec;
    o.absdist = result->absdist;
    o.shift = result->shift;
    return run_fill(plan->p, o, np, s);
}

nbl_status nbl_device_result_free(nbl_device_result *r, void *stream) {
    clear_error();
    if (!r) return NBL_SUCCESS;
    DeviceGuard g(r->device_id);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (r->first) cudaFreeAsync(r->first, s);
    if (r->second) cudaFreeAsync(r->second, s);
    if (r->distvec) cudaFreeAsync(r->distvec, s);
    if (r->absdist) cudaFreeAsync(r->absdist, s);
    if (r->shift) cudaFreeAsync(r->shift, s);
    std::memset(r, 0, sizeof(*r));
    return NBL_SUCCESS;
}

const char *nbl_last_error(void) { return g_last_error.c_str(); }

long long nbl_launch_count(int reset) {
    const long long n = g_launches;
    if (reset) g_launches = 0;
    return n;
}

int nbl_has_gpu(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return n > 0 ? 1 : 0;
}

int nbl_device_type(void) { return 2; }

const char *nbl_version(void) {
    return kChecked ? "nbl_b200 0.1.0 (sm_100a, checked)" : "nbl_b200 0.1.0 (sm_100a)";
}

}  // extern "C"
