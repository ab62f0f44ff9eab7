// Radix sort of (uint64 key, uint32 value) pairs on one stream.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace tpm {
// Scratch bytes radix_sort_u64 needs for n pairs (ping-pong copies, per-tile
// digit counts and offsets, the 8x256 histogram).
size_t radix_sort_scratch_bytes(int64_t n);
// Stable ascending sort of keys[0..n) (low key_bits bits) carrying vals.
// Synchronises the stream once (to skip constant-digit passes).
void radix_sort_u64(uint64_t* keys, uint32_t* vals, int64_t n, int key_bits, void* scratch, size_t scratch_bytes,
                    cudaStream_t s);
// Same sort with every digit pass run unconditionally: no host
// synchronisation and no device-to-host copy, so it can run on memory the
// caller cannot free or reallocate mid-stream.
void radix_sort_u64_all_passes(uint64_t* keys, uint32_t* vals, int64_t n, void* scratch, size_t scratch_bytes,
                               cudaStream_t s);
}  // namespace tpm
