// ref_gpu_shim.cu -- TEST INFRASTRUCTURE ONLY: a C entry point over the
// reference's own CUDA backend, neighbour_list_gpu_device
// (src/libneighbours/neighbour_list_gpu.cc:518, declared in
// neighbour_list_gpu.hh:95-96), compiled from the reference's sources by
// `make -C oracle ref_gpu` into oracle/_ref/libref_gpu.so.  bench.py times it
// on the same B200 as a secondary comparator; nothing in the engine links or
// loads it.
//
// The reference aborts the process on any CUDA error (device.hh:68-74), so
// callers give it only inputs the engine has already handled on the same
// device.
#include <cstdint>
#include <cstring>

#include <cuda_runtime.h>

#include "neighbour_list_gpu.hh"

namespace {
void copy_out(void *dst, const void *src, size_t bytes) {
    if (dst && src && bytes) cudaMemcpy(dst, src, bytes, cudaMemcpyDeviceToDevice);
}
}  // namespace

// One device build of the `quantities` of a system whose positions are on
// the device (scalar cutoff).  *npairs receives the pair count and *build_ms
// the device time of the reference's call (CUDA events on the legacy default
// stream, which the reference uses throughout).  When the output pointers are
// non-null and capacity >= npairs, the pairs are copied into them (device
// memory) after the timed call.
extern "C" __attribute__((visibility("default"))) int refgpu_neighbour_list(
    int quantities, const double *origin, const double *cell, const double *inv_cell,
    const int *pbc, int nat, const double *d_positions, double cutoff, int64_t *npairs,
    float *build_ms, int *first, int *second, double *distvec, double *absdist, int *shift,
    int64_t capacity) {
    using namespace matscipy;
    bool pb[3] = {pbc[0] != 0, pbc[1] != 0, pbc[2] != 0};
    NeighbourListRequest req;
    req.quantities = quantities;
    req.cell_origin = origin;
    req.cell = cell;
    req.inv_cell = inv_cell;
    req.pbc = pb;
    req.nat = nat;
    req.positions = d_positions;
    req.positions_on_device = true;
    req.cutoff = cutoff;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    int st = 0;
    {
        NeighbourListDevice out;
        cudaEventRecord(e0, 0);
        st = (int)neighbour_list_gpu_device(req, out);
        cudaEventRecord(e1, 0);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (build_ms) *build_ms = ms;
        if (npairs) *npairs = (int64_t)out.npairs;
        if (st == 0 && capacity >= (int64_t)out.npairs) {
            const size_t n = (size_t)out.npairs;
            copy_out(first, out.first.data(), n * sizeof(int));
            copy_out(second, out.secnd.data(), n * sizeof(int));
            copy_out(distvec, out.distvec.data(), 3 * n * sizeof(double));
            copy_out(absdist, out.absdist.data(), n * sizeof(double));
            copy_out(shift, out.shift.data(), 3 * n * sizeof(int));
            cudaDeviceSynchronize();
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return st;
}
