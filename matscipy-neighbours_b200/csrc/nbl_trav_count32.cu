// nbl_trav_count32.cu -- the count pass with the FP32 filter, every launch
// shape (warps per CTA x staged candidates x atoms per sweep x cutoff kind),
// for one-cell work items.  nbl_trav_count32r.cu compiles the same file with
// NBL_TRAV_RUNS = 1: the instantiations that also take runs of home cells.
#include "nbl_traverse.cuh"

#ifndef NBL_TRAV_RUNS
#define NBL_TRAV_RUNS 0
#endif
#if NBL_TRAV_RUNS
#define NBL_TRAV_NAME(x) x##_runs
#else
#define NBL_TRAV_NAME(x) x
#endif

namespace nbl {
namespace {

template <int K, int G, int W, int C>
TravKernel pick(size_t &smem) {
    smem = count_smem_bytes<true, C>(W);
    return k_count<true, K, G, W, C, NBL_TRAV_RUNS != 0>;
}

template <int K, int W>
TravKernel pick_w(const TravShape &s, size_t &smem) {
    const bool big = s.cand != 0, g2 = s.group == 2;
    if (big) return g2 ? pick<K, 2, W, 768>(smem) : pick<K, 4, W, 768>(smem);
    return g2 ? pick<K, 2, W, 384>(smem) : pick<K, 4, W, 384>(smem);
}

template <int K>
TravKernel pick_k(const TravShape &s, size_t &smem) {
    if (s.warps == 2) return pick_w<K, 2>(s, smem);
    if (s.warps == 8) return pick_w<K, 8>(s, smem);
    return pick_w<K, 4>(s, smem);
}

TravKernel kernel_for(int kind, const TravShape &s, size_t &smem) {
    if (kind == kCutPerAtom) return pick_k<kCutPerAtom>(s, smem);
    if (kind == kCutPerType) return pick_k<kCutPerType>(s, smem);
    return pick_k<kCutScalar>(s, smem);
}

}  // namespace

cudaError_t NBL_TRAV_NAME(launch_count_fp32)(int kind, const TraverseArgs &a, int grid, cudaStream_t st,
                              const TravShape &shape) {
    size_t smem = 0;
    const TravKernel k = kernel_for(kind, shape, smem);
    return launch_kernel(k, smem, shape.warps, a, grid, st);
}

int NBL_TRAV_NAME(occupancy_count_fp32)(int kind, const TravShape &shape) {
    size_t smem = 0;
    const TravKernel k = kernel_for(kind, shape, smem);
    return occupancy_kernel(k, smem, shape.warps);
}

}  // namespace nbl
