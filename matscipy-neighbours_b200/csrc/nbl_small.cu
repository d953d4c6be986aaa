// nbl_small.cu -- the whole count phase of one small system in one CTA.
//
// For a system of a few hundred atoms the count phase's own work is a few
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
// The CTA's warps take the work items one after another, each at the latency
// of one item, so the path pays off while the system has about as many
// items as the CTA has warps: measured on a B200, a 100-atom system's count +
// fill + synchronisation takes 62 us this way against 65 us for the
// multi-kernel sequence, while at 200 atoms the sequence is already faster
// (62 against 74 us) -- hence the 128-atom default.  A thread-per-atom exact
// count in one CTA was measured as well and lost: each thread walks a few
// hundred candidates serially.
#include <cstdint>

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

template <bool FP32, int KIND>
__global__ void __launch_bounds__(kSmallThreads, 1)
k_count_small(SmallCountArgs p) {
    extern __shared__ __align__(16) unsigned char dyn_smem[];
    __shared__ long long warp_sum[kSmallWarps];
    const int tid = threadIdx.x, nthr = blockDim.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int64_t N = p.bin.natoms;
    const SysDev &S = p.bin.sys[0];

    // --- init: flag block, cell table, per-system maximum, visit table -------
    if (tid < 8) p.small[tid] = 0;
    for (int64_t i = tid; i < p.ncells; i += nthr) p.gather.table[i] = make_int2(0, 0);
    if (tid == 0) p.gather.amax[0] = 0.f;
    if (p.trav.visit != nullptr) visit_fill(S, const_cast<VisitDev *>(p.trav.visit), tid, nthr);
    __syncthreads();

    // --- bin ----------------------------------------------------------------
    for (int64_t t = tid; t < N; t += nthr) bin_one(p.bin, t);
    __syncthreads();

    // --- stable sort by cell key: bitonic on (key << 32 | atom) ---------------
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
    __syncthreads();

    // --- gather: positions, cell slices, occupied cells ----------------------
    for (int64_t b = 0; b < N; b += nthr) gather_one(p.gather, b + tid);
    __syncthreads();

    // --- work items -----------------------------------------------------------
    {
        const int nh = *p.gather.n_home;
        for (int b = 0; b < nh; b += nthr)
            tiles_one(p.gather.home, p.gather.table, p.trav.sys,
                      const_cast<WorkItem *>(p.trav.items), p.items_count, p.trav.itile, 1,
                      b + tid, nh);
    }
    __syncthreads();

    // --- count pass: the CTA's warps over the items ---------------------------
    count_items<FP32, KIND, 4, FP32 ? 384 : 192, false>(p.trav, dyn_smem, warp, kSmallWarps);
    __syncthreads();

    // --- row offsets: exclusive scan of the counts (original atom order) ------
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

template <bool FP32>
cudaError_t launch_small(int kind, const SmallCountArgs &a, cudaStream_t st) {
    TravKernel k = nullptr;  // (the type only carries the pointer to prepare_kernel)
    if (kind == kCutPerAtom)
        k = reinterpret_cast<TravKernel>(k_count_small<FP32, kCutPerAtom>);
    else if (kind == kCutPerType)
        k = reinterpret_cast<TravKernel>(k_count_small<FP32, kCutPerType>);
    else
        k = reinterpret_cast<TravKernel>(k_count_small<FP32, kCutScalar>);
    const size_t smem = small_smem_bytes<FP32>();
    cudaError_t e = prepare_kernel(k, smem);
    if (e != cudaSuccess) return e;
    void *args[] = {const_cast<SmallCountArgs *>(&a)};
    e = cudaLaunchKernel(reinterpret_cast<const void *>(k), dim3(1), dim3(kSmallThreads), args,
                         smem, st);
    count_launch();
    return e;
}

}  // namespace

cudaError_t launch_count_small(bool fp32, int kind, const SmallCountArgs &a, cudaStream_t st) {
    if (a.bin.natoms < 1 || a.bin.natoms > kSmallMaxAtoms || a.ncells > kSmallMaxCells ||
        a.bin.nsys != 1 || a.bin.grid != kGridDense)
        return cudaErrorInvalidValue;
    return fp32 ? launch_small<true>(kind, a, st) : launch_small<false>(kind, a, st);
}

}  // namespace nbl
