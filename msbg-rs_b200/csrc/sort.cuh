// sort.cuh -- stable LSD radix sort of (u64 key, u32 value) pairs and a
// device exclusive scan, shared by the Morton sort, bucket_indices and P2G.
#pragma once

#include "common.cuh"

namespace msbg {

// Scratch bytes radix_sort_pairs needs for n pairs.
size_t radix_sort_scratch_bytes(size_t n);

// Stable ascending sort of (keys, vals) by key bits [0, end_bit).  Inputs are
// read from keys_in/vals_in; the sorted result lands in keys_out/vals_out.
// `tmp` must hold radix_sort_scratch_bytes(n).  vals_in == nullptr means the
// identity 0..n-1.  All buffers are device memory on ctx's stream.
void radix_sort_pairs(msbg_ctx* ctx, const uint64_t* keys_in, const uint32_t* vals_in, uint64_t* keys_out,
                      uint32_t* vals_out, size_t n, int end_bit, void* tmp);

// Exclusive scan of n uint32 values into out (may alias in); total to
// *d_total (device) if non-null.  `tmp` needs scan_scratch_bytes(n).
size_t scan_scratch_bytes(size_t n);
void exclusive_scan_u32(msbg_ctx* ctx, const uint32_t* in, uint32_t* out, size_t n, uint32_t* d_total, void* tmp);

// Number of significant bits of the largest key (device reduction, synchronises).
int key_bits(msbg_ctx* ctx, const uint64_t* d_keys, size_t n, void* tmp8);

// Segment boundaries of a sorted key array: for each distinct key, its first
// index (starts[k]) and the key (uniq[k]); starts[count] = n.  Returns count
// (synchronises).  tmp needs segment_scratch_bytes(n).
size_t segment_scratch_bytes(size_t n);
size_t sorted_segments(msbg_ctx* ctx, const uint64_t* d_sorted, size_t n, uint64_t shift, uint64_t* d_uniq,
                       uint64_t* d_starts, void* tmp);

// Morton key of the truncated cell coordinate of each particle ([n][3] f32).
void morton_keys(msbg_ctx* ctx, const float* d_pos, size_t n, uint64_t* d_keys);

}  // namespace msbg
