// Exclusive prefix sums on one stream.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace tpm {
size_t scan_scratch_bytes(int64_t n);
// out[i] = sum_{j<i} in[j]; *total_dev (if non-null) = sum of all.  in == out is allowed.
void exclusive_scan_u32(const uint32_t* in, uint32_t* out, int64_t n, uint32_t* total_dev, void* scratch,
                        cudaStream_t s);
}  // namespace tpm
