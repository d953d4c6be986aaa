// nbl_trav_fill32.cu -- the fill pass (after the FP32-filter count),
// every launch shape (warps per CTA x cutoff kind, all five outputs or any subset),
// and the Lennard-Jones force sink (four-warp CTAs only), for one-cell work
// items.  nbl_trav_fill32r.cu compiles the same file with NBL_TRAV_RUNS = 1:
// the instantiations that also take runs of home cells.
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

template <int K, int W>
TravKernel pick_w(bool lj, bool all5, size_t &smem) {
    if (lj) {
        smem = fill_smem_bytes<true>(4, true);
        return k_fill<true, K, true, false, 4, NBL_TRAV_RUNS != 0>;
    }
    if (all5) {
        smem = fill_smem_bytes<true>(W, false);
        return k_fill<true, K, false, true, W, NBL_TRAV_RUNS != 0>;
    }
    smem = fill_smem_bytes<true>(W, false);
    return k_fill<true, K, false, false, W, NBL_TRAV_RUNS != 0>;
}

template <int K>
TravKernel pick_k(const TravShape &s, bool lj, bool all5, size_t &smem) {
    if (s.warps == 2) return pick_w<K, 2>(lj, all5, smem);
    if (s.warps == 8) return pick_w<K, 8>(lj, all5, smem);
    return pick_w<K, 4>(lj, all5, smem);
}

TravKernel kernel_for(int kind, const TravShape &s, bool lj, bool all5, size_t &smem) {
    if (kind == kCutPerAtom) return pick_k<kCutPerAtom>(s, lj, all5, smem);
    if (kind == kCutPerType) return pick_k<kCutPerType>(s, lj, all5, smem);
    return pick_k<kCutScalar>(s, lj, all5, smem);
}

}  // namespace

cudaError_t NBL_TRAV_NAME(launch_fill_fp32)(int kind, const TraverseArgs &a, int grid, cudaStream_t st,
                             const TravShape &shape) {
    const bool lj = a.lj_force != nullptr;
    const bool all5 = !lj && a.first && a.second && a.distvec && a.absdist && a.shift &&
                      a.mat_k == 0;
    size_t smem = 0;
    const TravKernel k = kernel_for(kind, shape, lj, all5, smem);
    return launch_kernel(k, smem, lj ? 4 : shape.warps, a, grid, st);
}

int NBL_TRAV_NAME(occupancy_fill_fp32)(int kind, const TravShape &shape, bool lj) {
    size_t smem = 0;
    const TravKernel k = kernel_for(kind, shape, lj, false, smem);
    return occupancy_kernel(k, smem, lj ? 4 : shape.warps);
}

}  // namespace nbl
