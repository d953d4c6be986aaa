// nbl_noalloc.cu -- the allocation-free entry point nbl_neighbour_list_noalloc.
//
// Some callers cannot allocate device memory when they need a neighbour list:
// MD engines whose time-step loop forbids any allocation after start-up,
// applications that hand (nearly) all device memory to their own pool
// allocator up front so that a cudaMalloc would fail, and services with a
// fixed per-process memory budget.  For them this entry point runs the same
// pipeline as nbl_count + nbl_fill (the same kernels, the same bit-identical
// output) with every piece of device scratch taken from one file-scope
// __device__ array of fixed size, g_noalloc_scratch, instead of a plan's
// workspace.  The caller passes the inputs and the output buffers (with their
// capacity); nothing here calls cudaMalloc, cudaMallocAsync, cudaFree,
// cudaMallocHost or any library routine that allocates device memory.
//
// Properties a caller must know:
//   * every GPU that loads the library holds the array (kNoAllocScratchBytes,
//     8 MiB) until the process exits;
//   * systems are limited to NBL_NOALLOC_MAX_ATOMS atoms and to grids whose
//     scratch fits the array; larger requests are rejected with
//     NBL_ERROR_INVALID_ARGUMENT and a message naming the limit;
//   * all calls on a device share the one array and it keeps the last call's
//     contents; each call clears what must start at zero, but two calls that
//     overlap on the GPU (different streams, or different host threads) race
//     on it and must be serialised by the caller;
//   * the first call on a device looks up the array's device address with
//     cudaGetSymbolAddress (that device current) and caches it per device
//     ordinal for the life of the process; make that first call before
//     starting any stream capture.  The cache assumes the process keeps one
//     (primary) context per device: after cudaDeviceReset, or under a context
//     of its own on that device, the cached address is stale;
//   * the call returns after the fill has finished (it synchronises `stream`
//     twice: for the pair count and at the end) and reports errors the device
//     flagged in either pass.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <mutex>

#include <cuda_runtime.h>

#include "nbl_b200.h"
#include "nbl_build.cuh"
#include "nbl_internal.cuh"
#include "nbl_plan.hh"
#include "nbl_sort.cuh"

namespace nbl {

// Request -> one-system batch (nbl_api.cu).
nbl_status batch_from_request(const nbl_request *req, Batch &b);

constexpr size_t kNoAllocScratchBytes = size_t(8) << 20;  // 8 MiB
constexpr int kNoAllocMaxDevices = 64;

// The scratch.  In host code this name is only a host-side stand-in; its
// device address comes from cudaGetSymbolAddress (noalloc_scratch_ptr).
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {

std::mutex g_noalloc_mutex;
void *g_noalloc_ptr[kNoAllocMaxDevices] = {nullptr};

nbl_status noalloc_scratch_ptr(int dev, unsigned char **out) {
    if (dev < 0 || dev >= kNoAllocMaxDevices)
        return set_error(NBL_ERROR_INVALID_ARGUMENT, "device %d out of range", dev);
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_ptr[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_status(e, "cudaGetSymbolAddress(scratch)");
        g_noalloc_ptr[dev] = p;
    }
    *out = static_cast<unsigned char *>(g_noalloc_ptr[dev]);
    return NBL_SUCCESS;
}

struct Carve {
    unsigned char *base;
    size_t used = 0;
    size_t cap;
    bool ok = true;
    template <typename T>
    T *take(size_t count) {
        const size_t bytes = (sizeof(T) * count + 255) & ~size_t(255);
        if (used + bytes > cap) {
            ok = false;
            return nullptr;
        }
        T *p = reinterpret_cast<T *>(base + used);
        used += bytes;
        return p;
    }
};

}  // namespace

}  // namespace nbl

using namespace nbl;

extern "C" NBL_API nbl_status nbl_neighbour_list_noalloc(const nbl_request *req,
                                                         const nbl_outputs *out,
                                                         int64_t capacity,
                                                         int64_t *npairs,
                                                         void *stream) {
    if (!req || !out || !npairs || capacity < 0)
        return set_error(NBL_ERROR_INVALID_ARGUMENT, "null argument");
    *npairs = 0;
    if (req->nat > NBL_NOALLOC_MAX_ATOMS)
        return set_error(NBL_ERROR_INVALID_ARGUMENT,
                         "nbl_neighbour_list_noalloc: %lld atoms exceed the limit of %d "
                         "(use nbl_count/nbl_fill)",
                         (long long)req->nat, NBL_NOALLOC_MAX_ATOMS);
    int dev = req->device_id;
    if (dev < 0 && cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return set_error(NBL_ERROR_NO_DEVICE, "no CUDA device available");
    }
    int cur = 0;
    if (cudaGetDevice(&cur) != cudaSuccess) {
        cudaGetLastError();
        return set_error(NBL_ERROR_NO_DEVICE, "no CUDA device available");
    }
    if (cur != dev)
        return set_error(NBL_ERROR_INVALID_ARGUMENT,
                         "nbl_neighbour_list_noalloc: make device %d current first", dev);

    // Plan the system on the host as nbl_count does, with one difference: a
    // dense or Morton table of more than 2^18 cells (whether the caller asked
    // for it or the automatic rule chose it) is replaced by the hashed table,
    // whose size follows the atom count, so that it fits the static scratch.
    // Every grid gives the same output.
    nbl_request r = *req;
    Batch b;
    nbl_status st = batch_from_request(&r, b);
    if (st != NBL_SUCCESS) return st;
    if (b.grid != kGridHashed && b.table_size > (int64_t(1) << 18)) {
        r.grid = NBL_GRID_HASHED;
        st = batch_from_request(&r, b);
        if (st != NBL_SUCCESS) return st;
    }
    const int64_t N = b.natoms;

    unsigned char *scratch = nullptr;
    st = noalloc_scratch_ptr(dev, &scratch);
    if (st != NBL_SUCCESS) return st;
    cudaStream_t s = static_cast<cudaStream_t>(stream);

    // Carve the buffers of one call out of the static array.
    Carve c{scratch, 0, kNoAllocScratchBytes};
    const int64_t hist = radix_hist_elems(std::max<int64_t>(N, 1));
    double *pos = b.pos_on_device ? const_cast<double *>(b.positions)
                                  : c.take<double>(3 * N);
    double *per_atom = nullptr;
    int32_t *types = nullptr;
    if (b.per_atom) per_atom = b.aux_on_device ? const_cast<double *>(b.per_atom)
                                               : c.take<double>(N);
    if (b.types) types = b.aux_on_device ? const_cast<int32_t *>(b.types)
                                         : c.take<int32_t>(N);
    SysDev *sys = c.take<SysDev>(1);
    int64_t *sab = c.take<int64_t>(1);
    const size_t npt = std::max<size_t>(b.pt64.size(), 1);
    double *pt64 = c.take<double>(npt);
    float *pt32 = c.take<float>(npt);
    uint32_t *keys = c.take<uint32_t>(N), *keys2 = c.take<uint32_t>(N);
    int32_t *vals = c.take<int32_t>(N), *vals2 = c.take<int32_t>(N);
    int32_t *hst = c.take<int32_t>(hist), *hscan = c.take<int32_t>(hist);
    int32_t *scan32 = c.take<int32_t>(scan_scratch_elems(hist));
    int64_t *scan64 = c.take<int64_t>(scan_scratch_elems(N + 1));
    int2 *table = c.take<int2>(b.table_size);
    unsigned long long *hkey =
        b.grid == kGridHashed ? c.take<unsigned long long>(b.table_size) : nullptr;
    double4 *pos64 = c.take<double4>(N);
    float4 *pos32 = c.take<float4>(N);
    int4 *aux = c.take<int4>(N);
    float *amax = c.take<float>(1);
    HomeCell *home = c.take<HomeCell>(N);
    int32_t *counts = c.take<int32_t>(N + 1);
    int64_t *offsets = c.take<int64_t>(N + 1);
    int *small = c.take<int>(8);
    WorkItem *items = c.take<WorkItem>(std::max<int64_t>(N, 1));
    if (!c.ok)
        return set_error(NBL_ERROR_INVALID_ARGUMENT,
                         "nbl_neighbour_list_noalloc: the request needs more than the "
                         "%zu bytes of static scratch (grid too large for %lld atoms)",
                         kNoAllocScratchBytes, (long long)N);

#define NA_CUDA(call, where)                                    \
    do {                                                        \
        cudaError_t e_ = (call);                                \
        if (e_ != cudaSuccess) return cuda_status(e_, where);   \
    } while (0)

    // Small host tables: pageable copies (staged by the driver, no allocation).
    SysDev S0 = b.sys[0];
    const int64_t zero64 = 0;
    NA_CUDA(cudaMemcpyAsync(sys, &S0, sizeof(SysDev), cudaMemcpyHostToDevice, s), "copy");
    NA_CUDA(cudaMemcpyAsync(sab, &zero64, sizeof(int64_t), cudaMemcpyHostToDevice, s),
            "copy");
    if (!b.pt64.empty()) {
        NA_CUDA(cudaMemcpyAsync(pt64, b.pt64.data(), sizeof(double) * b.pt64.size(),
                                cudaMemcpyHostToDevice, s), "copy");
        std::vector<float> p32(b.pt64.begin(), b.pt64.end());
        NA_CUDA(cudaMemcpyAsync(pt32, p32.data(), sizeof(float) * p32.size(),
                                cudaMemcpyHostToDevice, s), "copy");
        NA_CUDA(cudaStreamSynchronize(s), "copy");
    }
    if (!b.pos_on_device && N > 0)
        NA_CUDA(cudaMemcpyAsync(pos, b.positions, sizeof(double) * 3 * N,
                                cudaMemcpyHostToDevice, s), "copy positions");
    if (b.per_atom && !b.aux_on_device && N > 0)
        NA_CUDA(cudaMemcpyAsync(per_atom, b.per_atom, sizeof(double) * N,
                                cudaMemcpyHostToDevice, s), "copy cutoffs");
    if (b.types && !b.aux_on_device && N > 0)
        NA_CUDA(cudaMemcpyAsync(types, b.types, sizeof(int32_t) * N,
                                cudaMemcpyHostToDevice, s), "copy types");

    // Everything that must start at zero (the array keeps the last call's data).
    NA_CUDA(cudaMemsetAsync(small, 0, sizeof(int) * 8, s), "memset");
    NA_CUDA(cudaMemsetAsync(table, 0, sizeof(int2) * b.table_size, s), "memset");
    if (hkey)
        NA_CUDA(cudaMemsetAsync(hkey, 0xff, sizeof(unsigned long long) * b.table_size, s),
                "memset");
    NA_CUDA(cudaMemsetAsync(amax, 0, sizeof(float), s), "memset");

    BinArgs ba{};
    ba.sys = sys;
    ba.sys_atom_base = sab;
    ba.nsys = 1;
    ba.grid = b.grid;
    ba.positions = pos;
    ba.natoms = N;
    ba.keys = keys;
    ba.vals = vals;
    ba.hkey = hkey;
    ba.hmask = (unsigned long long)(b.table_size - 1);
    ba.err = small + 1;
    NA_CUDA(launch_bin(ba, s), "k_bin");
    bool in_alt = false;
    NA_CUDA(radix_sort_pairs(keys, vals, keys2, vals2, N, b.key_bits, hst, hscan, scan32,
                             s, &in_alt), "radix sort");
    GatherArgs ga{};
    ga.sys = sys;
    ga.sys_atom_base = sab;
    ga.nsys = 1;
    ga.grid = b.grid;
    ga.positions = pos;
    ga.per_atom = per_atom;
    ga.types = types;
    ga.natoms = N;
    ga.keys = in_alt ? keys2 : keys;
    ga.vals = in_alt ? vals2 : vals;
    ga.table = table;
    ga.pos64 = pos64;
    ga.pos32 = pos32;
    ga.aux = aux;
    ga.amax = amax;
    ga.home = home;
    ga.n_home = small;
    NA_CUDA(launch_gather(ga, s), "k_gather");
    int nsm_tiles = 148;
    cudaDeviceGetAttribute(&nsm_tiles, cudaDevAttrMultiProcessorCount, dev);
    NA_CUDA(launch_tiles(home, small, table, sys, items, small + 3, N, nsm_tiles, 32, 1, s),
            "k_tiles");

    TraverseArgs ta{};
    ta.sys = sys;
    ta.home = home;
    ta.n_home = small;
    ta.items = items;
    ta.n_items = small + 3;
    ta.grid = b.grid;
    ta.table = table;
    ta.hkey = hkey;
    ta.hmask = (unsigned long long)(b.table_size - 1);
    ta.pos64 = pos64;
    ta.pos32 = pos32;
    ta.aux = aux;
    ta.amax = amax;
    ta.pt32 = pt32;
    ta.pt64 = pt64;
    ta.counts = counts;
    ta.offsets = offsets;
    ta.err = small + 1;
    ta.item_next = small + 6;
    ta.i_lo = 0;
    ta.i_hi = INT64_MAX;
    ta.itile = 32;
    ta.natoms = N;
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    // two whole waves of each pass's resident CTAs
    const int kind = b.sys[0].cutoff_kind;
    const int count_grid = (int)std::min<int64_t>(
        (int64_t)nsm * 2 * std::max(1, traverse_blocks_per_sm(kModeCount, b.fp32, kind)),
        std::max<int64_t>(N, 1));
    const int fill_grid = (int)std::min<int64_t>(
        (int64_t)nsm * 2 * std::max(1, traverse_blocks_per_sm(kModeFill, b.fp32, kind)),
        std::max<int64_t>(N, 1));
    NA_CUDA(launch_traverse(kModeCount, b.fp32, kind, ta, count_grid, s), "count pass");
    NA_CUDA(exclusive_scan_i32_i64(counts, N, offsets, scan64, s), "scan");

    // Pair count and error bits back through pageable host memory.
    int64_t total = 0;
    int flags[2] = {0, 0};
    NA_CUDA(cudaMemcpyAsync(&total, offsets + N, sizeof(int64_t), cudaMemcpyDeviceToHost, s),
            "read pair count");
    NA_CUDA(cudaMemcpyAsync(flags, small, sizeof(flags), cudaMemcpyDeviceToHost, s),
            "read flags");
    NA_CUDA(cudaStreamSynchronize(s), "count phase");
    *npairs = total;
    if (flags[1] & kErrRange)
        return set_error(NBL_ERROR_RANGE,
                         "positions must be finite and within 2^29 cells of the box");
    if (flags[1] & kErrInternal)
        return set_error(NBL_ERROR_INTERNAL, "device-side bound exceeded in count phase");
    if (total > capacity)
        return set_error(NBL_ERROR_CAPACITY,
                         "nbl_neighbour_list_noalloc: %lld pairs exceed the output "
                         "capacity %lld",
                         (long long)total, (long long)capacity);
    if (total == 0 || !(out->first || out->second || out->distvec || out->absdist ||
                        out->shift))
        return NBL_SUCCESS;
    ta.first = out->first;
    ta.second = out->second;
    ta.distvec = out->distvec;
    ta.absdist = out->absdist;
    ta.shift = out->shift;
    ta.capacity = capacity;
    NA_CUDA(launch_traverse(kModeFill, b.fp32, kind, ta, fill_grid, s), "fill pass");
    // The call returns only when the fill has finished with the shared scratch,
    // and reports what the device flagged during it.
    NA_CUDA(cudaMemcpyAsync(flags, small, sizeof(flags), cudaMemcpyDeviceToHost, s),
            "read flags");
    NA_CUDA(cudaStreamSynchronize(s), "fill pass");
    if (flags[1] & kErrCapacity)
        return set_error(NBL_ERROR_CAPACITY,
                         "nbl_neighbour_list_noalloc: a pair fell outside the output "
                         "capacity %lld", (long long)capacity);
    if (flags[1] & kErrInternal)
        return set_error(NBL_ERROR_INTERNAL, "device-side bound exceeded in fill pass");
#undef NA_CUDA
    return NBL_SUCCESS;
}
