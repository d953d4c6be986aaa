// nbl_backward.cu -- gradients of a loss through the pair list.
//
// For a fixed pair list (i, j, S) the reference's distance vector is
//     D = r_j - r_i + sum_m c_m cell[m],    c_m = S_m on periodic axes, 0 else
// (on a non-periodic axis the reference's shift can be non-zero for atoms
// outside the box -- neighbour_visit.hh:112-114 -- but it never enters D,
// whose cell-relative terms cancel there), and d = |D|.  Given dL/dD and
// dL/dd per pair, with g = dL/dD + (dL/dd) D / d:
//     dL/dr_i -= g,   dL/dr_j += g,   dL/dcell[m][k] += c_m g_k.
//
// Default: one thread per pair (a flat, fully coalesced pass over the pairs);
// the i-side sums each warp's runs of equal i with a segmented shuffle scan
// and adds one FP64 atomic per run, the j-side adds FP64 atomics per pair.
// Deterministic: pairs are sorted by i, so each atom's row is contiguous and
// a warp reduces it without atomics; the j-side is a stable radix sort of the
// pairs by j followed by the same per-atom reduction.  Cell: per-CTA partial
// sums reduced in a fixed order.  With `deterministic` every result is
// bit-reproducible run to run.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <mutex>

#include <cuda_runtime.h>

#include "nbl_b200.h"
#include "nbl_internal.cuh"
#include "nbl_plan.hh"
#include "nbl_sort.cuh"

namespace nbl {

namespace {

constexpr int kBwdThreads = 256;
constexpr int kBwdWarps = kBwdThreads / 32;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
    return v;
}

struct PairGrad {
    const double *gD;   // [3P] or null
    const double *gd;   // [P] or null
    const double *D;    // [3P]
    const double *d;    // [P]
    __device__ __forceinline__ void at(int64_t p, double &g0, double &g1, double &g2) const {
        g0 = g1 = g2 = 0.0;
        if (gD) {
            g0 = gD[3 * p + 0];
            g1 = gD[3 * p + 1];
            g2 = gD[3 * p + 2];
        }
        if (gd) {
            const double dd = d[p];
            if (dd > 0.0) {
                const double s = gd[p] / dd;
                g0 += s * D[3 * p + 0];
                g1 += s * D[3 * p + 1];
                g2 += s * D[3 * p + 2];
            }
        }
    }
};

// Row starts of a sorted index array: start[v] = first p with idx[p] == v,
// for every v in [idx[p-1]+1, idx[p]] (empty rows get the next start).
__global__ void k_row_starts(const int32_t *__restrict__ idx, int64_t n, int64_t nat,
                             int64_t *__restrict__ start) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p > n) return;
    const int64_t lo = (p == 0) ? 0 : (int64_t)idx[p - 1] + 1;
    const int64_t hi = (p == n) ? nat : (int64_t)idx[p];
    for (int64_t v = lo; v <= hi && v <= nat; v++) start[v] = p;
}

// i-side rows and cell partials.  One warp per atom row.
__global__ void __launch_bounds__(kBwdThreads)
k_bwd_rows(PairGrad pg, const int64_t *__restrict__ off, int64_t nat,
           const int32_t *__restrict__ shift, const int32_t *__restrict__ second,
           int pbc_bits, double *__restrict__ grad_i, double *__restrict__ grad_j_atomic,
           double *__restrict__ cell_part) {
    __shared__ double s_cell[kBwdWarps][9];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double c[9];
#pragma unroll
    for (int k = 0; k < 9; k++) c[k] = 0.0;
    const int64_t gw = (int64_t)blockIdx.x * kBwdWarps + warp;
    const int64_t nw = (int64_t)gridDim.x * kBwdWarps;
    for (int64_t a = gw; a < nat; a += nw) {
        double gi0 = 0.0, gi1 = 0.0, gi2 = 0.0;
        for (int64_t p = off[a] + lane; p < off[a + 1]; p += 32) {
            double g0, g1, g2;
            pg.at(p, g0, g1, g2);
            gi0 += g0;
            gi1 += g1;
            gi2 += g2;
            const double s0 = (pbc_bits & 1) ? (double)shift[3 * p + 0] : 0.0;
            const double s1 = (pbc_bits & 2) ? (double)shift[3 * p + 1] : 0.0;
            const double s2 = (pbc_bits & 4) ? (double)shift[3 * p + 2] : 0.0;
            c[0] += s0 * g0; c[1] += s0 * g1; c[2] += s0 * g2;
            c[3] += s1 * g0; c[4] += s1 * g1; c[5] += s1 * g2;
            c[6] += s2 * g0; c[7] += s2 * g1; c[8] += s2 * g2;
            if (grad_j_atomic) {
                const int64_t j = second[p];
                atomicAdd(grad_j_atomic + 3 * j + 0, g0);
                atomicAdd(grad_j_atomic + 3 * j + 1, g1);
                atomicAdd(grad_j_atomic + 3 * j + 2, g2);
            }
        }
        gi0 = warp_sum(gi0);
        gi1 = warp_sum(gi1);
        gi2 = warp_sum(gi2);
        if (lane == 0) {
            grad_i[3 * a + 0] = gi0;
            grad_i[3 * a + 1] = gi1;
            grad_i[3 * a + 2] = gi2;
        }
    }
#pragma unroll
    for (int k = 0; k < 9; k++) c[k] = warp_sum(c[k]);
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < 9; k++) s_cell[warp][k] = c[k];
    }
    __syncthreads();
    if (threadIdx.x < 9) {
        double t = 0.0;
        for (int w = 0; w < kBwdWarps; w++) t += s_cell[w][threadIdx.x];
        cell_part[9 * blockIdx.x + threadIdx.x] = t;
    }
}

// Default path: thread per pair.  grad_pos must be zeroed; receives
// sum_j-side g - sum_i-side g through FP64 atomics.
__global__ void __launch_bounds__(kBwdThreads)
k_bwd_pairs(PairGrad pg, const int32_t *__restrict__ first,
            const int32_t *__restrict__ second, const int32_t *__restrict__ shift, int64_t P,
            int pbc_bits, double *__restrict__ grad_pos, double *__restrict__ cell_part) {
    __shared__ double s_cell[kBwdWarps][9];
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double c[9];
#pragma unroll
    for (int k = 0; k < 9; k++) c[k] = 0.0;
    const int64_t stride = (int64_t)gridDim.x * kBwdThreads;
    for (int64_t base = (int64_t)blockIdx.x * kBwdThreads + warp * 32; base < P;
         base += stride) {
        const int64_t p = base + lane;
        const bool act = p < P;
        double g0 = 0.0, g1 = 0.0, g2 = 0.0;
        int i = -1;
        if (act) {
            pg.at(p, g0, g1, g2);
            i = first[p];
            const int64_t j = second[p];
            const double s0 = (pbc_bits & 1) ? (double)shift[3 * p + 0] : 0.0;
            const double s1 = (pbc_bits & 2) ? (double)shift[3 * p + 1] : 0.0;
            const double s2 = (pbc_bits & 4) ? (double)shift[3 * p + 2] : 0.0;
            c[0] += s0 * g0; c[1] += s0 * g1; c[2] += s0 * g2;
            c[3] += s1 * g0; c[4] += s1 * g1; c[5] += s1 * g2;
            c[6] += s2 * g0; c[7] += s2 * g1; c[8] += s2 * g2;
            atomicAdd(grad_pos + 3 * j + 0, g0);
            atomicAdd(grad_pos + 3 * j + 1, g1);
            atomicAdd(grad_pos + 3 * j + 2, g2);
        }
        // runs of equal i are contiguous: segmented inclusive scan over lanes
        double r0 = g0, r1 = g1, r2 = g2;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const double t0 = __shfl_up_sync(full, r0, d);
            const double t1 = __shfl_up_sync(full, r1, d);
            const double t2 = __shfl_up_sync(full, r2, d);
            const int ii = __shfl_up_sync(full, i, d);
            if (lane >= d && ii == i) {
                r0 += t0;
                r1 += t1;
                r2 += t2;
            }
        }
        const int inext = __shfl_down_sync(full, i, 1);
        if (act && (lane == 31 || inext != i)) {
            atomicAdd(grad_pos + 3 * (int64_t)i + 0, -r0);
            atomicAdd(grad_pos + 3 * (int64_t)i + 1, -r1);
            atomicAdd(grad_pos + 3 * (int64_t)i + 2, -r2);
        }
    }
#pragma unroll
    for (int k = 0; k < 9; k++) c[k] = warp_sum(c[k]);
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < 9; k++) s_cell[warp][k] = c[k];
    }
    __syncthreads();
    if (threadIdx.x < 9) {
        double t = 0.0;
        for (int w = 0; w < kBwdWarps; w++) t += s_cell[w][threadIdx.x];
        cell_part[9 * blockIdx.x + threadIdx.x] = t;
    }
}

// j-side in deterministic order: perm lists the pairs sorted by j (stable).
__global__ void __launch_bounds__(kBwdThreads)
k_bwd_cols(PairGrad pg, const int64_t *__restrict__ coff, const int32_t *__restrict__ perm,
           int64_t nat, double *__restrict__ grad_j) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int64_t gw = (int64_t)blockIdx.x * kBwdWarps + warp;
    const int64_t nw = (int64_t)gridDim.x * kBwdWarps;
    for (int64_t a = gw; a < nat; a += nw) {
        double g0s = 0.0, g1s = 0.0, g2s = 0.0;
        for (int64_t q = coff[a] + lane; q < coff[a + 1]; q += 32) {
            double g0, g1, g2;
            pg.at(perm[q], g0, g1, g2);
            g0s += g0;
            g1s += g1;
            g2s += g2;
        }
        g0s = warp_sum(g0s);
        g1s = warp_sum(g1s);
        g2s = warp_sum(g2s);
        if (lane == 0) {
            grad_j[3 * a + 0] = g0s;
            grad_j[3 * a + 1] = g1s;
            grad_j[3 * a + 2] = g2s;
        }
    }
}

__global__ void k_bwd_combine(const double *__restrict__ gi, const double *__restrict__ gj,
                              int64_t n3, double *__restrict__ out) {
    const int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n3) out[t] = gj[t] - gi[t];
}

// Sum of the per-CTA cell partials in a fixed order: thread t of one block
// takes partials t, t + blockDim, ...; then a fixed tree over the threads.
__global__ void __launch_bounds__(kBwdThreads)
k_bwd_cell(const double *__restrict__ part, int nblocks, double *__restrict__ grad_cell) {
    __shared__ double s[kBwdThreads][9];
    double t[9];
#pragma unroll
    for (int k = 0; k < 9; k++) t[k] = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += kBwdThreads) {
#pragma unroll
        for (int k = 0; k < 9; k++) t[k] += part[9 * b + k];
    }
#pragma unroll
    for (int k = 0; k < 9; k++) s[threadIdx.x][k] = t[k];
    __syncthreads();
    for (int h = kBwdThreads / 2; h > 0; h >>= 1) {
        if ((int)threadIdx.x < h) {
#pragma unroll
            for (int k = 0; k < 9; k++) s[threadIdx.x][k] += s[threadIdx.x + h][k];
        }
        __syncthreads();
    }
    if (threadIdx.x < 9) grad_cell[threadIdx.x] = s[0][threadIdx.x];
}

__global__ void k_iota_keys(const int32_t *__restrict__ second, int64_t n,
                            uint32_t *__restrict__ keys, int32_t *__restrict__ vals) {
    const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    keys[p] = (uint32_t)second[p];
    vals[p] = (int32_t)p;
}

}  // namespace

// Stream-ordered scratch comes from a pool of this library's own per device
// that keeps its memory between calls (the default pool would hand it back to
// the driver at every synchronisation and map it again on the next call).
namespace {
constexpr int kMaxPoolDevices = 64;
std::mutex g_pool_mutex;
cudaMemPool_t g_pools[kMaxPoolDevices] = {};
}  // namespace

cudaError_t scratch_pool(int dev, cudaMemPool_t *pool) {
    if (dev < 0 || dev >= kMaxPoolDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_pool_mutex);
    if (!g_pools[dev]) {
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t p = nullptr;
        cudaError_t e = cudaMemPoolCreate(&p, &props);
        if (e != cudaSuccess) return e;
        uint64_t keep = UINT64_MAX;
        e = cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
        if (e != cudaSuccess) {
            cudaMemPoolDestroy(p);
            return e;
        }
        g_pools[dev] = p;
    }
    *pool = g_pools[dev];
    return cudaSuccess;
}

}  // namespace nbl

using namespace nbl;

#define NBL_CUDA(call, where)                                  \
    do {                                                       \
        cudaError_t e_ = (call);                               \
        if (e_ != cudaSuccess) { status = cuda_status(e_, where); goto done; } \
    } while (0)

extern "C" NBL_API nbl_status nbl_backward(const nbl_backward_args *g, void *stream) {
    if (!g || g->npairs < 0 || g->nat < 0 || !g->grad_positions || !g->grad_cell)
        return set_error(NBL_ERROR_INVALID_ARGUMENT, "bad backward arguments");
    if (g->npairs > 0 && (!g->first || !g->second || !g->shift ||
                          (!g->grad_distvec && !g->grad_absdist) ||
                          (g->grad_absdist && (!g->distvec || !g->absdist))))
        return set_error(NBL_ERROR_INVALID_ARGUMENT, "backward needs i, j, S and a gradient");
    if (g->npairs >= INT32_MAX)
        return set_error(NBL_ERROR_INVALID_ARGUMENT, "backward supports < 2^31 pairs");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    nbl_status status = NBL_SUCCESS;
    const int64_t P = g->npairs, N = g->nat;
    int nsm = 148, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const int rows_grid =
        g->deterministic
            ? (int)std::max<int64_t>(1, std::min<int64_t>((N + kBwdWarps - 1) / kBwdWarps,
                                                          (int64_t)nsm * 8))
            : (int)std::max<int64_t>(1, std::min<int64_t>((P + kBwdThreads - 1) / kBwdThreads,
                                                          (int64_t)nsm * 8));
    const int pbc_bits = (g->pbc && g->pbc[0] ? 1 : 0) | (g->pbc && g->pbc[1] ? 2 : 0) |
                         (g->pbc && g->pbc[2] ? 4 : 0);
    PairGrad pg{g->grad_distvec, g->grad_absdist, g->distvec, g->absdist};
    // Scratch (stream-ordered): row starts, i/j partial gradients, cell partials,
    // and for the deterministic j-side the sort buffers.
    char *scratch = nullptr;
    size_t bytes = 0, o_off, o_gi, o_gj, o_cell, o_keys = 0, o_vals = 0, o_keys2 = 0,
           o_vals2 = 0, o_hist = 0, o_hscan = 0, o_s32 = 0, o_coff = 0;
    const int64_t hist = radix_hist_elems(std::max<int64_t>(P, 1));
    auto add = [&](size_t b) {
        const size_t o = bytes;
        bytes += (b + 255) & ~size_t(255);
        return o;
    };
    o_off = add(sizeof(int64_t) * (N + 1));
    o_gi = add(sizeof(double) * 3 * std::max<int64_t>(N, 1));
    o_gj = add(sizeof(double) * 3 * std::max<int64_t>(N, 1));
    o_cell = add(sizeof(double) * 9 * rows_grid);
    if (g->deterministic) {
        o_keys = add(sizeof(uint32_t) * P);
        o_vals = add(sizeof(int32_t) * P);
        o_keys2 = add(sizeof(uint32_t) * P);
        o_vals2 = add(sizeof(int32_t) * P);
        o_hist = add(sizeof(int32_t) * hist);
        o_hscan = add(sizeof(int32_t) * hist);
        o_s32 = add(sizeof(int32_t) * scan_scratch_elems(hist));
        o_coff = add(sizeof(int64_t) * (N + 1));
    }
    {
        cudaMemPool_t pool = nullptr;
        NBL_CUDA(scratch_pool(dev, &pool), "backward scratch pool");
        NBL_CUDA(cudaMallocFromPoolAsync((void **)&scratch, std::max<size_t>(bytes, 256), pool,
                                         st),
                 "backward scratch");
        int64_t *off = reinterpret_cast<int64_t *>(scratch + o_off);
        double *gi = reinterpret_cast<double *>(scratch + o_gi);
        double *gj = reinterpret_cast<double *>(scratch + o_gj);
        double *cell_part = reinterpret_cast<double *>(scratch + o_cell);
        if (!g->deterministic) {
            // the default path reads no row offsets
        } else if (g->row_offsets) {
            NBL_CUDA(cudaMemcpyAsync(off, g->row_offsets, sizeof(int64_t) * (N + 1),
                                     cudaMemcpyDeviceToDevice, st), "row offsets");
        } else {
            k_row_starts<<<(unsigned)((P + 1 + 255) / 256), 256, 0, st>>>(g->first, P, N, off);
            count_launch();
            NBL_CUDA(cudaGetLastError(), "row starts");
        }
        if (!g->deterministic) {
            NBL_CUDA(cudaMemsetAsync(g->grad_positions, 0,
                                     sizeof(double) * 3 * std::max<int64_t>(N, 1), st),
                     "memset");
            k_bwd_pairs<<<rows_grid, kBwdThreads, 0, st>>>(pg, g->first, g->second, g->shift,
                                                           P, pbc_bits, g->grad_positions,
                                                           cell_part);
            count_launch();
            NBL_CUDA(cudaGetLastError(), "backward pairs");
        } else {
            k_bwd_rows<<<rows_grid, kBwdThreads, 0, st>>>(pg, off, N, g->shift, g->second,
                                                          pbc_bits, gi, nullptr, cell_part);
            count_launch();
            NBL_CUDA(cudaGetLastError(), "backward rows");
        }
        if (g->deterministic && P > 0) {
            uint32_t *keys = reinterpret_cast<uint32_t *>(scratch + o_keys);
            int32_t *vals = reinterpret_cast<int32_t *>(scratch + o_vals);
            uint32_t *keys2 = reinterpret_cast<uint32_t *>(scratch + o_keys2);
            int32_t *vals2 = reinterpret_cast<int32_t *>(scratch + o_vals2);
            k_iota_keys<<<(unsigned)((P + 255) / 256), 256, 0, st>>>(g->second, P, keys, vals);
            count_launch();
            NBL_CUDA(cudaGetLastError(), "sort keys");
            int bits = 0;
            while (bits < 32 && ((uint64_t)std::max<int64_t>(N - 1, 0) >> bits) != 0) bits++;
            bool alt = false;
            NBL_CUDA(radix_sort_pairs(keys, vals, keys2, vals2, P, bits,
                                      reinterpret_cast<int32_t *>(scratch + o_hist),
                                      reinterpret_cast<int32_t *>(scratch + o_hscan),
                                      reinterpret_cast<int32_t *>(scratch + o_s32), st, &alt),
                     "sort by j");
            const uint32_t *sk = alt ? keys2 : keys;
            const int32_t *perm = alt ? vals2 : vals;
            int64_t *coff = reinterpret_cast<int64_t *>(scratch + o_coff);
            k_row_starts<<<(unsigned)((P + 1 + 255) / 256), 256, 0, st>>>(
                reinterpret_cast<const int32_t *>(sk), P, N, coff);
            count_launch();
            NBL_CUDA(cudaGetLastError(), "column starts");
            k_bwd_cols<<<rows_grid, kBwdThreads, 0, st>>>(pg, coff, perm, N, gj);
            count_launch();
            NBL_CUDA(cudaGetLastError(), "backward columns");
        }
        if (N > 0 && g->deterministic) {
            k_bwd_combine<<<(unsigned)((3 * N + 255) / 256), 256, 0, st>>>(gi, gj, 3 * N,
                                                                           g->grad_positions);
            count_launch();
            NBL_CUDA(cudaGetLastError(), "combine");
        }
        k_bwd_cell<<<1, kBwdThreads, 0, st>>>(cell_part, rows_grid, g->grad_cell);
        count_launch();
        NBL_CUDA(cudaGetLastError(), "cell gradient");
    }
done:
    if (scratch) cudaFreeAsync(scratch, st);
    return status;
}
