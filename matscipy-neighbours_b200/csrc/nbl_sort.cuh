// nbl_sort.cuh -- device scan / radix sort entry points (nbl_sort.cu).
#pragma once

#include <cstdint>

#include <cuda_runtime.h>

namespace nbl {

// Scratch elements (of the accumulator type) needed by a scan of n items.
int64_t scan_scratch_elems(int64_t n);

// out[k] = sum(in[0..k)), k < n, and out[n] = sum(in[0..n)).
cudaError_t exclusive_scan_i32_i64(const int32_t *in, int64_t n, int64_t *out,
                                   int64_t *scratch, cudaStream_t st);
// out[k] = sum(in[0..k)), k < n.
cudaError_t exclusive_scan_i32_i32(const int32_t *in, int64_t n, int32_t *out,
                                   int32_t *scratch, cudaStream_t st);

// int32 entries needed for the digit histogram of one radix pass over n keys.
int64_t radix_hist_elems(int64_t n);

// Stable sort of (keys, vals) by the low `bits` bits of keys.  Ping-pongs
// between the two buffer pairs; *result_in_alt tells where the result is.
cudaError_t radix_sort_pairs(uint32_t *keys, int32_t *vals, uint32_t *keys_alt,
                             int32_t *vals_alt, int64_t n, int bits,
                             int32_t *hist, int32_t *hist_scan,
                             int32_t *scan_scratch, cudaStream_t st,
                             bool *result_in_alt);

}  // namespace nbl
