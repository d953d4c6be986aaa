// nbl_small.cu -- the whole count phase of one small system in one launch.
//
// For a system of about a hundred atoms the count phase's own work is a few
// microseconds; its cost is the chain of launches (init, bin, the sort's
// passes, gather, work items, count, the scan's passes) that the multi-CTA
// path needs between its grid-wide steps.  Here one 16-warp CTA runs every
// stage, separated by __syncthreads, on the same data layout: the cell table,
// sorted positions, work items, hit words, counts and row offsets it leaves
// behind are exactly what the multi-CTA path leaves, so the ordinary fill
// pass (and nbl_counts, nbl_row_offsets, nbl_fill_matrix) follows it
// unchanged.  The stage bodies are the multi-CTA kernels' own
// (nbl_stages.cuh, nbl_traverse.cuh); the sort is a bitonic sort of
// (cell key, atom index) pairs in shared memory, which gives the radix
// sort's stable order.
//
// Above 128 atoms the launch is a thread-block cluster of up to 8 such CTAs:
// every stage is spread over the cluster's threads, the sort and the scan
// run in CTA 0, and the barriers are cluster-wide.  The warps still take the
// work items one after another, so the path pays off only while the system
// has about as many items as the launch has warps: measured on a B200, a
// 100-atom system's count + fill + synchronisation takes 68 us this way
// against 81 us for the multi-kernel sequence, even at 300 atoms, and 94
// against 82 us at 1000 -- hence the 128-atom default.  A thread-per-atom
// exact count in one CTA was measured as well and lost: each thread walks a
// few hundred candidates serially.
#include <cstdint>

#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include "nbl_build.cuh"
#include "nbl_internal.cuh"
#include "nbl_stages.cuh"
#include "nbl_traverse.cuh"

namespace nbl {
namespace {

constexpr int kSmallThreads = 512;  // 16 warps
constexpr int kSmallWarps = kSmallThreads / 32;

// Per-CTA dynamic shared memory: the sort buffer, then (reused) the count
// pass's per-warp state.
template <bool FP32>
constexpr size_t small_smem_bytes() {
    constexpr size_t sort = sizeof(unsigned long long) * kSmallMaxAtoms;
    constexpr size_t count = count_smem_bytes<FP32, FP32 ? 384 : 192>(kSmallWarps);
    return sort > count ? sort : count;
}

// Barrier across every CTA of the launch (a thread-block cluster, or the one
// CTA), ordering the global and shared memory accesses before it.
template <bool CLUSTER>
__device__ __forceinline__ void small_sync() {
    if constexpr (CLUSTER)
        cooperative_groups::this_cluster().sync();
    else
        __syncthreads();
}

template <bool FP32, int KIND, bool CLUSTER>
__global__ void __launch_bounds__(kSmallThreads, 1)
k_count_small(SmallCountArgs p) {
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    __shared__ long long warp_sum[kSmallWarps];
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int lane = tid & 31, warp = tid >> 5;
    // this CTA's rank in the launch and the launch's threads: the stages run
    // over all of them, the sort and the scan in CTA 0
    const int rank = blockIdx.x, nctas = gridDim.x;
    const int grank = rank * nthr + tid, gsize = nctas * nthr;
    const int64_t N = p.bin.natoms;
    const SysDev &S = p.bin.sys[0];

    // --- init: flag block, cell table, per-system maximum, visit table -------
    if (grank < 8) p.small[grank] = 0;
    for (int64_t i = grank; i < p.ncells; i += gsize) p.gather.table[i] = make_int2(0, 0);
    if (grank == 0) p.gather.amax[0] = 0.f;
    if (p.trav.visit != nullptr)
        visit_fill(S, const_cast<VisitDev *>(p.trav.visit), grank, gsize);
    small_sync<CLUSTER>();

    // --- bin ----------------------------------------------------------------
    for (int64_t t = grank; t < N; t += gsize) bin_one(p.bin, t);
    small_sync<CLUSTER>();

    // --- stable sort by cell key (CTA 0): bitonic on (key << 32 | atom) ------
    if (rank == 0) {
        unsigned long long *srt = reinterpret_cast<unsigned long long *>(dyn_smem);
        int P = 1;
        while (P < N) P <<= 1;
        for (int i = tid; i < P; i += nthr)
            srt[i] = i < N ? ((unsigned long long)p.bin.keys[i] << 32) |
                                 (unsigned long long)(uint32_t)p.bin.vals[i]
                           : ~0ull;
        __syncthreads();
        for (int k = 2; k <= P; k <<= 1) {
            for (int j = k >> 1; j > 0; j >>= 1) {
                for (int i = tid; i < P; i += nthr) {
                    const int l = i ^ j;
                    if (l > i) {
                        const unsigned long long x = srt[i], y = srt[l];
                        const bool up = (i & k) == 0;
                        if ((x > y) == up) {
                            srt[i] = y;
                            srt[l] = x;
                        }
                    }
                }
                __syncthreads();
            }
        }
        for (int i = tid; i < N; i += nthr) {
            p.bin.keys[i] = (uint32_t)(srt[i] >> 32);
            p.bin.vals[i] = (int32_t)(uint32_t)srt[i];
        }
    }
    small_sync<CLUSTER>();

    // --- gather: positions, cell slices, occupied cells ----------------------
    for (int64_t b = (int64_t)rank * nthr; b < N; b += gsize) gather_one(p.gather, b + tid);
    small_sync<CLUSTER>();

    // --- work items -----------------------------------------------------------
    {
        const int nh = *p.gather.n_home;
        for (int b = rank * nthr; b < nh; b += gsize)
            tiles_one(p.gather.home, p.gather.table, p.trav.sys,
                      const_cast<WorkItem *>(p.trav.items), p.items_count, p.trav.itile, 1,
                      b + tid, nh);
    }
    small_sync<CLUSTER>();

    // --- count pass: all warps of the launch over the items -------------------
    count_items<FP32, KIND, 4, FP32 ? 384 : 192, false>(p.trav, dyn_smem,
                                                        rank * kSmallWarps + warp,
                                                        nctas * kSmallWarps);
    small_sync<CLUSTER>();
    if (rank != 0) return;

    // --- row offsets (CTA 0): exclusive scan of the counts, original order ---
    constexpr int kPer = kSmallMaxAtoms / kSmallThreads;
    long long local[kPer];
    long long sum = 0;
#pragma unroll
    for (int q = 0; q < kPer; q++) {
        const int64_t i = (int64_t)tid * kPer + q;
        local[q] = i < N ? (long long)p.trav.counts[i] : 0ll;
        sum += local[q];
    }
    long long incl = sum;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const long long o = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= d) incl += o;
    }
    if (lane == 31) warp_sum[warp] = incl;
    __syncthreads();
    long long base = 0;
    for (int w = 0; w < warp; w++) base += warp_sum[w];
    long long run = base + incl - sum;
#pragma unroll
    for (int q = 0; q < kPer; q++) {
        const int64_t i = (int64_t)tid * kPer + q;
        if (i < N) p.offsets[i] = run;
        run += local[q];
    }
    if (tid == nthr - 1) p.offsets[N] = run;
}

template <bool FP32, bool CLUSTER>
TravKernel small_kernel(int kind) {
    // (the type only carries the pointer to prepare_kernel and the launch)
    if (kind == kCutPerAtom)
        return reinterpret_cast<TravKernel>(k_count_small<FP32, kCutPerAtom, CLUSTER>);
    if (kind == kCutPerType)
        return reinterpret_cast<TravKernel>(k_count_small<FP32, kCutPerType, CLUSTER>);
    return reinterpret_cast<TravKernel>(k_count_small<FP32, kCutScalar, CLUSTER>);
}

// One CTA, or a cluster of `ctas` CTAs (one per SM: each holds 16 warps'
// count state) for systems with more work items than one CTA has warps.
template <bool FP32>
cudaError_t launch_small(int kind, const SmallCountArgs &a, int ctas, cudaStream_t st) {
    const bool cluster = ctas > 1;
    const TravKernel k = cluster ? small_kernel<FP32, true>(kind) : small_kernel<FP32, false>(kind);
    const size_t smem = small_smem_bytes<FP32>();
    cudaError_t e = prepare_kernel(k, smem);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)ctas);
    cfg.blockDim = dim3(kSmallThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    if (cluster) {
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = (unsigned)ctas;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
    }
    void *args[] = {const_cast<SmallCountArgs *>(&a)};
    e = cudaLaunchKernelExC(&cfg, reinterpret_cast<const void *>(k), args);
    count_launch();
    return e;
}

}  // namespace

cudaError_t launch_count_small(bool fp32, int kind, const SmallCountArgs &a, int ctas,
                               cudaStream_t st) {
    if (a.bin.natoms < 1 || a.bin.natoms > kSmallMaxAtoms || a.ncells > kSmallMaxCells ||
        a.bin.nsys != 1 || a.bin.grid != kGridDense || ctas < 1 || ctas > kSmallMaxCtas)
        return cudaErrorInvalidValue;
    return fp32 ? launch_small<true>(kind, a, ctas, st) : launch_small<false>(kind, a, ctas, st);
}

}  // namespace nbl
