// Exclusive prefix sum of uint32 counts into uint32 offsets (three kernels:
// per-block sums, a single-block scan of the block sums, per-block apply).
#include "common.cuh"
#include "scan.cuh"

namespace tpm {
namespace {

constexpr int SCAN_BLOCK = 1024;
constexpr int SCAN_ITEMS = 4;
constexpr int SCAN_TILE = SCAN_BLOCK * SCAN_ITEMS;

__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t* total, uint32_t* sh) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  uint32_t x = v;
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  if (lane == 31) sh[warp] = x;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = lane < nw ? sh[lane] : 0u;
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += y;
    }
    sh[lane] = w;
  }
  __syncthreads();
  uint32_t r = (warp > 0 ? sh[warp - 1] : 0u) + x - v;
  *total = sh[nw - 1];
  __syncthreads();
  return r;
}

__global__ void k_block_sums(const uint32_t* __restrict__ in, int64_t n, uint32_t* __restrict__ sums) {
  __shared__ uint32_t sh[32];
  int64_t base = (int64_t)blockIdx.x * SCAN_TILE;
  uint32_t s = 0;
  for (int j = 0; j < SCAN_ITEMS; ++j) {
    int64_t i = base + (int64_t)j * SCAN_BLOCK + threadIdx.x;
    if (i < n) s += in[i];
  }
  uint32_t tot;
  block_excl_scan(s, &tot, sh);
  if (threadIdx.x == 0) sums[blockIdx.x] = tot;
}

__global__ void k_scan_sums(uint32_t* __restrict__ sums, int64_t nb, uint32_t* __restrict__ total_out) {
  __shared__ uint32_t sh[32];
  uint32_t carry = 0;
  for (int64_t c0 = 0; c0 < nb; c0 += blockDim.x) {
    int64_t i = c0 + threadIdx.x;
    uint32_t v = i < nb ? sums[i] : 0u;
    uint32_t tot;
    uint32_t e = block_excl_scan(v, &tot, sh);
    if (i < nb) sums[i] = carry + e;
    carry += tot;
  }
  if (threadIdx.x == 0 && total_out) *total_out = carry;
}

__global__ void k_apply(const uint32_t* __restrict__ in, int64_t n, const uint32_t* __restrict__ sums,
                        uint32_t* __restrict__ out) {
  __shared__ uint32_t sh[32];
  int64_t base = (int64_t)blockIdx.x * SCAN_TILE;
  // thread-contiguous items keep the scan order exact
  uint32_t v[SCAN_ITEMS];
  uint32_t s = 0;
  for (int j = 0; j < SCAN_ITEMS; ++j) {
    int64_t i = base + (int64_t)threadIdx.x * SCAN_ITEMS + j;
    v[j] = i < n ? in[i] : 0u;
    s += v[j];
  }
  uint32_t tot;
  uint32_t e = block_excl_scan(s, &tot, sh) + sums[blockIdx.x];
  for (int j = 0; j < SCAN_ITEMS; ++j) {
    int64_t i = base + (int64_t)threadIdx.x * SCAN_ITEMS + j;
    if (i < n) out[i] = e;
    e += v[j];
  }
}

}  // namespace

size_t scan_scratch_bytes(int64_t n) { return (size_t)((n + SCAN_TILE - 1) / SCAN_TILE + 1) * sizeof(uint32_t) + 256; }

void exclusive_scan_u32(const uint32_t* in, uint32_t* out, int64_t n, uint32_t* total_dev, void* scratch,
                        cudaStream_t s) {
  if (n <= 0) {
    if (total_dev) TPM_CUDA(cudaMemsetAsync(total_dev, 0, sizeof(uint32_t), s));
    return;
  }
  int64_t nb = (n + SCAN_TILE - 1) / SCAN_TILE;
  uint32_t* sums = (uint32_t*)scratch;
  k_block_sums<<<(unsigned)nb, SCAN_BLOCK, 0, s>>>(in, n, sums);
  TPM_LAUNCH_CHECK();
  k_scan_sums<<<1, SCAN_BLOCK, 0, s>>>(sums, nb, total_dev);
  TPM_LAUNCH_CHECK();
  k_apply<<<(unsigned)nb, SCAN_BLOCK, 0, s>>>(in, n, sums, out);
  TPM_LAUNCH_CHECK();
}

}  // namespace tpm
