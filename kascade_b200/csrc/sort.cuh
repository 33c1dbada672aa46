// Device-wide exclusive scan and stable LSD radix sort of (uint32 key,
// uint32 value) pairs, both hand-written for this library.
#pragma once

#include "ctx.cuh"

namespace ks {

// out[i] = sum(in[0..i)), count < 2^31; *total (device) receives the sum if
// non-null.  `in` and `out` may alias.
kascade_status exclusive_scan_u32(kascade_ctx& ctx, const uint32_t* in, uint32_t* out, uint64_t count,
                                  uint32_t* total, cudaStream_t s);

// Source of the first sort pass: keys from a uint64 parent array (key =
// parent[i], value = i; out-of-range parents raise KASCADE_ERR_OUT_OF_RANGE
// and sort as their own index), or from uint32 key/value arrays.
struct SortSource {
  const uint64_t* parent = nullptr;
  const uint32_t* keys = nullptr;
  const uint32_t* vals = nullptr;
};

// Stable sort of n pairs by key, keys < 2^key_bits.  Scratch comes from the
// arena.  On return *keys_out / *vals_out point at the sorted arrays (arena
// memory).
kascade_status radix_sort_pairs(kascade_ctx& ctx, const SortSource& src, uint32_t n, int key_bits,
                                uint32_t** keys_out, uint32_t** vals_out, cudaStream_t s);

}  // namespace ks
