// nbl_trav_count64.cu -- the count pass with the plain FP64 test, every
// launch shape (warps per CTA x staged candidates x cutoff kind).
#include "nbl_traverse.cuh"

namespace nbl {
namespace {

template <int K, int W, int C>
TravKernel pick(size_t &smem) {
    smem = count_smem_bytes<false, C>(W);
    return k_count<false, K, 4, W, C, false>;
}

template <int K, int W>
TravKernel pick_w(const TravShape &s, size_t &smem) {
    return s.cand != 0 ? pick<K, W, 384>(smem) : pick<K, W, 192>(smem);
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

cudaError_t launch_count_fp64(int kind, const TraverseArgs &a, int grid, cudaStream_t st,
                              const TravShape &shape) {
    size_t smem = 0;
    const TravKernel k = kernel_for(kind, shape, smem);
    return launch_kernel(k, smem, shape.warps, a, grid, st);
}

int occupancy_count_fp64(int kind, const TravShape &shape) {
    size_t smem = 0;
    const TravKernel k = kernel_for(kind, shape, smem);
    return occupancy_kernel(k, smem, shape.warps);
}

}  // namespace nbl
