// nbl_verlet.cu -- reuse of a pair list across molecular-dynamics steps
// (a Verlet list): a list built once with cutoff rc + skin keeps every pair
// within rc for as long as no atom has moved more than skin / 2 since the
// build.  Per step the caller measures the largest displacement
// (nbl_max_displacement) and, while it is below skin / 2, refreshes the
// stored list instead of rebuilding it (nbl_verlet_refresh): D and d are
// recomputed from the current positions for every stored pair and the pairs
// with d < rc are kept, in the stored order (rows ascending in i).
//
// The reference rebuilds its list every step in its MD example
// (examples/lj_langevin/lj_langevin_gpu.cu:171-179); this is an addition.
// The refreshed pair set equals neighbour_list(rc) at the current positions;
// D is formed as r_j - r_i + sum over periodic axes of S_m cell[m], which
// rounds differently from the traversal's cell-relative arithmetic (ulps).
#include <algorithm>
#include <cstdint>
#include <cstring>

#include <cuda_runtime.h>

#include "nbl_b200.h"
#include "nbl_internal.cuh"
#include "nbl_plan.hh"
#include "nbl_sort.cuh"

namespace nbl {
namespace {

constexpr int kVThreads = 256;

// Block b: max over atoms [kVChunk b, kVChunk (b + 1)) of |r - r0|^2, in a
// fixed tree (max is order independent anyway).
constexpr int kVChunk = 2048;

__global__ void __launch_bounds__(kVThreads)
k_disp2(const double *__restrict__ r, const double *__restrict__ r0, int64_t n,
        double *__restrict__ out) {
    __shared__ double s[kVThreads];
    double m = 0.0;
    const int64_t a0 = (int64_t)blockIdx.x * kVChunk;
    for (int64_t a = a0 + threadIdx.x; a < n && a < a0 + kVChunk; a += kVThreads) {
        const double dx = r[3 * a] - r0[3 * a];
        const double dy = r[3 * a + 1] - r0[3 * a + 1];
        const double dz = r[3 * a + 2] - r0[3 * a + 2];
        const double d2 = dx * dx + dy * dy + dz * dz;
        // NaN positions must not pass as "no movement"
        m = (d2 > m || d2 != d2) ? d2 : m;
    }
    s[threadIdx.x] = m;
    __syncthreads();
    for (int h = kVThreads / 2; h > 0; h >>= 1) {
        if ((int)threadIdx.x < h) {
            const double o = s[threadIdx.x + h];
            if (o > s[threadIdx.x] || o != o) s[threadIdx.x] = o;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) out[blockIdx.x] = s[0];
}

__global__ void __launch_bounds__(kVThreads)
k_max_of(const double *__restrict__ v, int64_t n, double *__restrict__ out) {
    __shared__ double s[kVThreads];
    double m = 0.0;
    for (int64_t k = threadIdx.x; k < n; k += kVThreads) {
        const double x = v[k];
        m = (x > m || x != x) ? x : m;
    }
    s[threadIdx.x] = m;
    __syncthreads();
    for (int h = kVThreads / 2; h > 0; h >>= 1) {
        if ((int)threadIdx.x < h) {
            const double o = s[threadIdx.x + h];
            if (o > s[threadIdx.x] || o != o) s[threadIdx.x] = o;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = sqrt(s[0]);
}

struct Cell {
    double c[9];
    int pbc_bits;
};

__device__ __forceinline__ void pair_d(const Cell &C, const double *r, int32_t i, int32_t j,
                                       const int32_t *S, double &dx, double &dy, double &dz) {
    const double s0 = (C.pbc_bits & 1) ? (double)S[0] : 0.0;
    const double s1 = (C.pbc_bits & 2) ? (double)S[1] : 0.0;
    const double s2 = (C.pbc_bits & 4) ? (double)S[2] : 0.0;
    dx = r[3 * (int64_t)j] - r[3 * (int64_t)i] + (s0 * C.c[0] + s1 * C.c[3] + s2 * C.c[6]);
    dy = r[3 * (int64_t)j + 1] - r[3 * (int64_t)i + 1] +
         (s0 * C.c[1] + s1 * C.c[4] + s2 * C.c[7]);
    dz = r[3 * (int64_t)j + 2] - r[3 * (int64_t)i + 2] +
         (s0 * C.c[2] + s1 * C.c[5] + s2 * C.c[8]);
}

// Refresh in two passes over the stored pairs, kRTile pairs per block in
// kRTile / kRThreads sub-tiles of one pair per thread: the first counts the
// kept pairs of each block, the second (after a scan of the block counts)
// recomputes the test and writes the kept pairs at the block's offset plus
// their rank inside the block, so the stored order is kept.
constexpr int kRThreads = 256;
constexpr int kRTile = 2048;
constexpr int kRWarps = kRThreads / 32;

__device__ __forceinline__ bool refresh_keep(const Cell &C, const int32_t *__restrict__ fi,
                                             const int32_t *__restrict__ fj,
                                             const int32_t *__restrict__ fS,
                                             const double *__restrict__ r, int64_t p,
                                             int64_t np, double rc2, double &dx, double &dy,
                                             double &dz) {
    if (p >= np) return false;
    pair_d(C, r, fi[p], fj[p], fS + 3 * p, dx, dy, dz);
    return (dx * dx + dy * dy + dz * dz) < rc2;
}

__global__ void __launch_bounds__(kRThreads)
k_refresh_count(Cell C, const int32_t *__restrict__ fi, const int32_t *__restrict__ fj,
                const int32_t *__restrict__ fS, const double *__restrict__ r, int64_t np,
                double rc2, int32_t *__restrict__ blk) {
    __shared__ int wsum[kRWarps];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t p0 = (int64_t)blockIdx.x * kRTile;
    int c = 0;
#pragma unroll 2
    for (int k = 0; k < kRTile / kRThreads; k++) {
        double dx, dy, dz;
        const bool keep = refresh_keep(C, fi, fj, fS, r, p0 + k * kRThreads + threadIdx.x, np,
                                       rc2, dx, dy, dz);
        c += __popc(__ballot_sync(0xffffffffu, keep));
    }
    if (lane == 0) wsum[warp] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        int t = 0;
        for (int w = 0; w < kRWarps; w++) t += wsum[w];
        blk[blockIdx.x] = t;
    }
}

__global__ void __launch_bounds__(kRThreads)
k_refresh_write(Cell C, const int32_t *__restrict__ fi, const int32_t *__restrict__ fj,
                const int32_t *__restrict__ fS, const double *__restrict__ r, int64_t np,
                double rc2, const int64_t *__restrict__ blk_off, nbl_outputs o) {
    __shared__ int wcnt[kRWarps];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t p0 = (int64_t)blockIdx.x * kRTile;
    int64_t base = blk_off[blockIdx.x];
    for (int k = 0; k < kRTile / kRThreads; k++) {
        const int64_t p = p0 + k * kRThreads + threadIdx.x;
        double dx, dy, dz;
        const bool keep = refresh_keep(C, fi, fj, fS, r, p, np, rc2, dx, dy, dz);
        const unsigned m = __ballot_sync(0xffffffffu, keep);
        if (lane == 0) wcnt[warp] = __popc(m);
        __syncthreads();
        int before = 0, total = 0;
#pragma unroll
        for (int w = 0; w < kRWarps; w++) {
            const int x = wcnt[w];
            before += (w < warp) ? x : 0;
            total += x;
        }
        __syncthreads();  // wcnt is rewritten by the next sub-tile
        if (keep) {
            const int64_t q = base + before + __popc(m & ((1u << lane) - 1u));
            if (o.first) o.first[q] = fi[p];
            if (o.second) o.second[q] = fj[p];
            if (o.distvec) {
                o.distvec[3 * q] = dx;
                o.distvec[3 * q + 1] = dy;
                o.distvec[3 * q + 2] = dz;
            }
            if (o.absdist) o.absdist[q] = sqrt(dx * dx + dy * dy + dz * dz);
            if (o.shift) {
                o.shift[3 * q] = fS[3 * p];
                o.shift[3 * q + 1] = fS[3 * p + 1];
                o.shift[3 * q + 2] = fS[3 * p + 2];
            }
        }
        base += total;
    }
}

}  // namespace
}  // namespace nbl

using namespace nbl;

#define V_CUDA(call, where)                                                    \
    do {                                                                       \
        cudaError_t e_ = (call);                                               \
        if (e_ != cudaSuccess) {                                               \
            status = cuda_status(e_, where);                                   \
            goto done;                                                         \
        }                                                                      \
    } while (0)

extern "C" NBL_API nbl_status nbl_max_displacement(int64_t n, const double *positions,
                                                   const double *reference, double *out,
                                                   void *stream) {
    if (n < 0 || !out || (n > 0 && (!positions || !reference)))
        return set_error(NBL_ERROR_INVALID_ARGUMENT, "bad max_displacement arguments");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    nbl_status status = NBL_SUCCESS;
    const int64_t nb = std::max<int64_t>((n + kVChunk - 1) / kVChunk, 1);
    double *part = nullptr;
    int dev = 0;
    cudaGetDevice(&dev);
    {
        cudaMemPool_t pool = nullptr;
        V_CUDA(scratch_pool(dev, &pool), "scratch pool");
        V_CUDA(cudaMallocFromPoolAsync((void **)&part, sizeof(double) * nb, pool, st),
               "scratch");
        if (n > 0) {
            k_disp2<<<(unsigned)nb, kVThreads, 0, st>>>(positions, reference, n, part);
            count_launch();
            V_CUDA(cudaGetLastError(), "displacement");
        } else {
            V_CUDA(cudaMemsetAsync(part, 0, sizeof(double), st), "memset");
        }
        k_max_of<<<1, kVThreads, 0, st>>>(part, nb, out);
        count_launch();
        V_CUDA(cudaGetLastError(), "displacement max");
    }
done:
    if (part) cudaFreeAsync(part, st);
    return status;
}

extern "C" NBL_API nbl_status nbl_verlet_refresh(int64_t npairs, const int32_t *first,
                                                 const int32_t *second, const int32_t *shift,
                                                 const double *positions, const double *cell,
                                                 const uint8_t *pbc, double cutoff,
                                                 const nbl_outputs *out, int64_t capacity,
                                                 int64_t *nkept, void *stream) {
    if (npairs < 0 || !nkept || !cell || !pbc || !(cutoff >= 0.0) ||
        (npairs > 0 && (!first || !second || !shift || !positions)))
        return set_error(NBL_ERROR_INVALID_ARGUMENT, "bad verlet_refresh arguments");
    if (npairs >= INT32_MAX)
        return set_error(NBL_ERROR_INVALID_ARGUMENT, "verlet_refresh supports < 2^31 pairs");
    *nkept = 0;
    if (npairs == 0) return NBL_SUCCESS;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    nbl_status status = NBL_SUCCESS;
    Cell C;
    std::memcpy(C.c, cell, sizeof(C.c));
    C.pbc_bits = (pbc[0] ? 1 : 0) | (pbc[1] ? 2 : 0) | (pbc[2] ? 4 : 0);
    const double rc2 = cutoff * cutoff;
    const int64_t nblk = (npairs + kRTile - 1) / kRTile;
    char *scratch = nullptr;
    int dev = 0;
    cudaGetDevice(&dev);
    size_t bytes = 0;
    auto add = [&](size_t b) {
        const size_t o = bytes;
        bytes += (b + 255) & ~size_t(255);
        return o;
    };
    const size_t o_blk = add(sizeof(int32_t) * nblk);
    const size_t o_off = add(sizeof(int64_t) * (nblk + 1));
    const size_t o_s = add(sizeof(int64_t) * scan_scratch_elems(nblk + 1));
    // With room for every stored pair the write pass needs no count first:
    // one synchronisation at the end reads the total.
    const bool direct = out != nullptr && capacity >= npairs;
    {
        cudaMemPool_t pool = nullptr;
        V_CUDA(scratch_pool(dev, &pool), "scratch pool");
        V_CUDA(cudaMallocFromPoolAsync((void **)&scratch, bytes, pool, st), "scratch");
        int32_t *blk = reinterpret_cast<int32_t *>(scratch + o_blk);
        int64_t *off = reinterpret_cast<int64_t *>(scratch + o_off);
        int64_t *sscr = reinterpret_cast<int64_t *>(scratch + o_s);
        k_refresh_count<<<(unsigned)nblk, kRThreads, 0, st>>>(C, first, second, shift, positions,
                                                              npairs, rc2, blk);
        count_launch();
        V_CUDA(cudaGetLastError(), "refresh count");
        V_CUDA(exclusive_scan_i32_i64(blk, nblk, off, sscr, st), "scan");
        if (direct) {
            k_refresh_write<<<(unsigned)nblk, kRThreads, 0, st>>>(C, first, second, shift,
                                                                  positions, npairs, rc2, off,
                                                                  *out);
            count_launch();
            V_CUDA(cudaGetLastError(), "refresh write");
        }
        int64_t total = 0;  // pageable: the copy completes before it returns
        V_CUDA(cudaMemcpyAsync(&total, off + nblk, sizeof(int64_t), cudaMemcpyDeviceToHost, st),
               "read count");
        V_CUDA(cudaStreamSynchronize(st), "refresh count");
        *nkept = total;
        if (!out || direct || total == 0) goto done;
        if (capacity < total) {
            status = set_error(NBL_ERROR_CAPACITY, "verlet_refresh: %lld pairs, capacity %lld",
                               (long long)total, (long long)capacity);
            goto done;
        }
        k_refresh_write<<<(unsigned)nblk, kRThreads, 0, st>>>(C, first, second, shift, positions,
                                                              npairs, rc2, off, *out);
        count_launch();
        V_CUDA(cudaGetLastError(), "refresh write");
    }
done:
    if (scratch) cudaFreeAsync(scratch, st);
    return status;
}
