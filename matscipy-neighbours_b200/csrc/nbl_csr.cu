// nbl_csr.cu -- the CSR helpers of a pair list on the device: row starts
// (first_neighbours) and triplets of pairs sharing a first atom
// (triplet_list), with the reference's semantics and output order.
//
// first_neighbours (first_neighbours.cc:15-38): seed[k] = first pair of atom
// k; -1 for atoms before the first atom with pairs, nn (the pair count) after
// the last, and an empty row's seed is the next row's start.  One thread per
// pair writes the seeds between its atom and the previous pair's.
//
// triplet_list (triplet_list.cc:15-34): for each row r = [first_i[r],
// first_i[r+1]), every ordered pair (ij, ik), ij != ik, of the row's pairs
// whose distance is below the cutoff (all of them without distances), ij
// major.  With m kept pairs a row has m (m - 1) triplets; triplet
// q = a (m - 1) + c' of the row is (kept[a], kept[c' + (c' >= a)]).  Three
// passes, one warp per row: count m, compact the kept pairs, write the
// triplets lane-parallel (consecutive lanes, consecutive triplets).
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

constexpr int kCsrThreads = 256;
constexpr int kCsrWarps = kCsrThreads / 32;
constexpr int kMaxKept = 46340;  // m (m - 1) stays below 2^31

__global__ void k_seed_init(int64_t n, int32_t v, int32_t *__restrict__ seed) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k <= n) seed[k] = v;
}

// Atom indices outside [0, n) write nothing (the reference leaves that
// undefined).
__global__ void k_seed_scatter(const int32_t *__restrict__ i, int64_t nn, int64_t n,
                               int32_t *__restrict__ seed) {
    const int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= nn) return;
    const int64_t cur = i[k];
    if (k == 0) {
        if (cur >= 0 && cur <= n) seed[cur] = 0;
    } else {
        const int64_t prev = i[k - 1];
        if (cur != prev) {
            for (int64_t l = std::max<int64_t>(prev + 1, 0); l <= cur && l <= n; l++)
                seed[l] = (int32_t)k;
        }
    }
    if (k == nn - 1) {
        for (int64_t l = std::max<int64_t>(cur + 1, 0); l <= n; l++) seed[l] = (int32_t)nn;
    }
}

__device__ __forceinline__ bool kept(const double *d, double cutoff, int64_t p) {
    return d == nullptr || d[p] < cutoff;
}

// m per row; triplet count m (m - 1) per row.  Rows that start before 0
// (the seeds of atoms before the first one with pairs) hold no triplets.
__global__ void __launch_bounds__(kCsrThreads)
k_trip_count(const int32_t *__restrict__ first, int64_t nrows, const double *__restrict__ d,
             double cutoff, int32_t *__restrict__ mcount, int32_t *__restrict__ tcount,
             int *__restrict__ err) {
    const int lane = threadIdx.x & 31;
    const int64_t gw = ((int64_t)blockIdx.x * kCsrThreads + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * kCsrThreads) >> 5;
    for (int64_t r = gw; r < nrows; r += nw) {
        const int64_t b = first[r], e = first[r + 1];
        int m = 0;
        if (b >= 0) {
            for (int64_t p0 = b; p0 < e; p0 += 32) {
                const int64_t p = p0 + lane;
                m += __popc(__ballot_sync(0xffffffffu, p < e && kept(d, cutoff, p)));
            }
        }
        if (lane == 0) {
            if (m > kMaxKept) {
                atomicOr(err, 1);
                m = 0;
            }
            mcount[r] = m;
            tcount[r] = m * (m - 1) > 0 ? m * (m - 1) : 0;
        }
    }
}

// The kept pairs of each row, in order, at moff[r].
__global__ void __launch_bounds__(kCsrThreads)
k_trip_kept(const int32_t *__restrict__ first, int64_t nrows, const double *__restrict__ d,
            double cutoff, const int64_t *__restrict__ moff, int32_t *__restrict__ keep) {
    const int lane = threadIdx.x & 31;
    const int64_t gw = ((int64_t)blockIdx.x * kCsrThreads + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * kCsrThreads) >> 5;
    const unsigned lt = (1u << lane) - 1u;
    for (int64_t r = gw; r < nrows; r += nw) {
        const int64_t b = first[r], e = first[r + 1];
        if (b < 0 || moff[r + 1] == moff[r]) continue;
        int64_t out = moff[r];
        for (int64_t p0 = b; p0 < e; p0 += 32) {
            const int64_t p = p0 + lane;
            const bool k = p < e && kept(d, cutoff, p);
            const unsigned bal = __ballot_sync(0xffffffffu, k);
            if (k) keep[out + __popc(bal & lt)] = (int32_t)p;
            out += __popc(bal);
        }
    }
}

__global__ void __launch_bounds__(kCsrThreads)
k_trip_fill(int64_t nrows, const int64_t *__restrict__ moff, const int64_t *__restrict__ toff,
            const int32_t *__restrict__ keep, int32_t *__restrict__ ij,
            int32_t *__restrict__ ik) {
    const int lane = threadIdx.x & 31;
    const int64_t gw = ((int64_t)blockIdx.x * kCsrThreads + threadIdx.x) >> 5;
    const int64_t nw = ((int64_t)gridDim.x * kCsrThreads) >> 5;
    for (int64_t r = gw; r < nrows; r += nw) {
        const int m = (int)(moff[r + 1] - moff[r]);
        if (m < 2) continue;
        const int64_t kb = moff[r], tb = toff[r];
        const int t = m * (m - 1), m1 = m - 1;
        for (int q = lane; q < t; q += 32) {
            const int a = q / m1;
            const int c1 = q - a * m1;
            const int c = c1 + (c1 >= a ? 1 : 0);
            __stcs(ij + tb + q, keep[kb + a]);
            __stcs(ik + tb + q, keep[kb + c]);
        }
    }
}

}  // namespace
}  // namespace nbl

using namespace nbl;

#define CSR_CUDA(call, where)                                                  \
    do {                                                                       \
        cudaError_t e_ = (call);                                               \
        if (e_ != cudaSuccess) {                                               \
            status = cuda_status(e_, where);                                   \
            goto done;                                                         \
        }                                                                      \
    } while (0)

extern "C" NBL_API nbl_status nbl_first_neighbours(int64_t n, int64_t npairs,
                                                   const int32_t *first, int32_t *seed,
                                                   void *stream) {
    if (n < 0 || npairs < 0 || !seed || (npairs > 0 && !first))
        return set_error(NBL_ERROR_INVALID_ARGUMENT, "bad first_neighbours arguments");
    if (n >= INT32_MAX || npairs >= INT32_MAX)
        return set_error(NBL_ERROR_INVALID_ARGUMENT, "first_neighbours supports < 2^31 rows");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    k_seed_init<<<(unsigned)((n + 1 + 255) / 256), 256, 0, st>>>(n, npairs > 0 ? -1 : 0,
                                                                 seed);
    count_launch();
    if (npairs > 0) {
        k_seed_scatter<<<(unsigned)((npairs + 255) / 256), 256, 0, st>>>(first, npairs, n,
                                                                         seed);
        count_launch();
    }
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? NBL_SUCCESS : cuda_status(e, "first_neighbours");
}

extern "C" NBL_API nbl_status nbl_triplet_list(int64_t nfirst, const int32_t *first_i,
                                               const double *absdist, double cutoff,
                                               int32_t *ij, int32_t *ik, int64_t capacity,
                                               int64_t *ntriplets, void *stream) {
    if (!ntriplets || nfirst < 0 || (nfirst > 0 && !first_i))
        return set_error(NBL_ERROR_INVALID_ARGUMENT, "bad triplet_list arguments");
    *ntriplets = 0;
    if (nfirst < 2) return NBL_SUCCESS;
    if (nfirst >= INT32_MAX)
        return set_error(NBL_ERROR_INVALID_ARGUMENT, "triplet_list supports < 2^31 rows");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    nbl_status status = NBL_SUCCESS;
    const int64_t nrows = nfirst - 1;
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const int grid = (int)std::max<int64_t>(
        1, std::min<int64_t>((nrows + kCsrWarps - 1) / kCsrWarps, (int64_t)nsm * 8));
    char *scratch = nullptr;
    int64_t host[4] = {0, 0, 0, 0};  // pageable: the copies complete before they return
    size_t bytes = 0;
    auto add = [&](size_t b) {
        const size_t o = bytes;
        bytes += (b + 255) & ~size_t(255);
        return o;
    };
    const size_t o_m = add(sizeof(int32_t) * nrows);
    const size_t o_t = add(sizeof(int32_t) * nrows);
    const size_t o_mo = add(sizeof(int64_t) * (nrows + 1));
    const size_t o_to = add(sizeof(int64_t) * (nrows + 1));
    const size_t o_s = add(sizeof(int64_t) * scan_scratch_elems(nrows + 1));
    const size_t o_err = add(sizeof(int) * 2);
    {
        cudaMemPool_t pool = nullptr;
        CSR_CUDA(scratch_pool(dev, &pool), "triplet scratch pool");
        CSR_CUDA(cudaMallocFromPoolAsync((void **)&scratch, bytes, pool, st), "triplet scratch");
        int32_t *mcount = reinterpret_cast<int32_t *>(scratch + o_m);
        int32_t *tcount = reinterpret_cast<int32_t *>(scratch + o_t);
        int64_t *moff = reinterpret_cast<int64_t *>(scratch + o_mo);
        int64_t *toff = reinterpret_cast<int64_t *>(scratch + o_to);
        int64_t *sscr = reinterpret_cast<int64_t *>(scratch + o_s);
        int *err = reinterpret_cast<int *>(scratch + o_err);
        CSR_CUDA(cudaMemsetAsync(err, 0, sizeof(int), st), "memset");
        k_trip_count<<<grid, kCsrThreads, 0, st>>>(first_i, nrows, absdist, cutoff, mcount,
                                                   tcount, err);
        count_launch();
        CSR_CUDA(cudaGetLastError(), "triplet count");
        CSR_CUDA(exclusive_scan_i32_i64(mcount, nrows, moff, sscr, st), "scan");
        CSR_CUDA(exclusive_scan_i32_i64(tcount, nrows, toff, sscr, st), "scan");
        CSR_CUDA(cudaMemcpyAsync(host, toff + nrows, sizeof(int64_t), cudaMemcpyDeviceToHost,
                                 st),
                 "read count");
        CSR_CUDA(cudaMemcpyAsync(host + 1, moff + nrows, sizeof(int64_t),
                                 cudaMemcpyDeviceToHost, st),
                 "read count");
        CSR_CUDA(cudaMemcpyAsync(host + 2, err, sizeof(int), cudaMemcpyDeviceToHost, st),
                 "read flags");
        CSR_CUDA(cudaStreamSynchronize(st), "triplet count");
        int flag = 0;
        std::memcpy(&flag, host + 2, sizeof(int));
        if (flag) {
            status = set_error(NBL_ERROR_INVALID_ARGUMENT,
                               "triplet_list: a row keeps more than %d pairs", kMaxKept);
            goto done;
        }
        *ntriplets = host[0];
        if (!ij || !ik || host[0] == 0) goto done;
        if (capacity < host[0]) {
            status = set_error(NBL_ERROR_CAPACITY, "triplet_list: %lld triplets, capacity %lld",
                               (long long)host[0], (long long)capacity);
            goto done;
        }
        {
            int32_t *keep = nullptr;
            CSR_CUDA(cudaMallocFromPoolAsync((void **)&keep,
                                             sizeof(int32_t) * std::max<int64_t>(host[1], 1),
                                             pool, st),
                     "triplet scratch");
            k_trip_kept<<<grid, kCsrThreads, 0, st>>>(first_i, nrows, absdist, cutoff, moff,
                                                      keep);
            count_launch();
            cudaError_t e = cudaGetLastError();
            if (e == cudaSuccess) {
                k_trip_fill<<<grid, kCsrThreads, 0, st>>>(nrows, moff, toff, keep, ij, ik);
                count_launch();
                e = cudaGetLastError();
            }
            cudaFreeAsync(keep, st);
            CSR_CUDA(e, "triplet fill");
        }
    }
done:
    if (scratch) cudaFreeAsync(scratch, st);
    return status;
}
