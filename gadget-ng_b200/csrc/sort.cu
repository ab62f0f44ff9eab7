// LSD radix sort of (uint64 key, uint32 value) pairs — 8-bit digits, stable.
//
// One pass = upsweep (per-tile digit counts) -> per-digit scan over tiles ->
// downsweep (stable scatter).  Ranks inside a tile come from warp match/ballot
// (no shared-memory atomics on the scatter path), so the order of equal keys
// is the input order.  A single histogram kernel reads the keys once for all
// eight digit positions; passes whose digit is constant are skipped.  No
// kernel waits on another block, so nothing can spin.
#include "common.cuh"
#include "sort.cuh"

namespace tpm {

namespace {

constexpr int SORT_WARPS = SORT_BLOCK / 32;

__global__ void k_hist8(const uint64_t* __restrict__ keys, int64_t n, uint32_t* __restrict__ hist) {
  __shared__ uint32_t h[8][256];
  for (int i = threadIdx.x; i < 8 * 256; i += blockDim.x) (&h[0][0])[i] = 0;
  __syncthreads();
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    uint64_t k = keys[i];
#pragma unroll
    for (int d = 0; d < 8; ++d) atomicAdd(&h[d][(k >> (8 * d)) & 255u], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 8 * 256; i += blockDim.x) {
    uint32_t v = (&h[0][0])[i];
    if (v) atomicAdd(&hist[i], v);
  }
}

__global__ void k_upsweep(const uint64_t* __restrict__ keys, int64_t n, int shift, int64_t ntiles,
                          uint32_t* __restrict__ tile_counts) {
  __shared__ uint32_t h[256];
  for (int i = threadIdx.x; i < 256; i += blockDim.x) h[i] = 0;
  __syncthreads();
  int64_t base = (int64_t)blockIdx.x * SORT_TILE;
#pragma unroll 4
  for (int j = 0; j < SORT_ITEMS; ++j) {
    int64_t idx = base + (int64_t)j * SORT_BLOCK + threadIdx.x;
    if (idx < n) atomicAdd(&h[(keys[idx] >> shift) & 255u], 1u);
  }
  __syncthreads();
  for (int d = threadIdx.x; d < 256; d += blockDim.x) tile_counts[(int64_t)d * ntiles + blockIdx.x] = h[d];
}

// One block per digit: offsets[d][t] = base(d) + sum_{t' < t} tile_counts[d][t'].
__global__ void k_scan_tiles(const uint32_t* __restrict__ tile_counts, const uint32_t* __restrict__ digit_hist,
                             int64_t ntiles, uint32_t* __restrict__ offsets) {
  __shared__ uint32_t warp_sums[32];
  __shared__ uint32_t s_base;
  const int d = blockIdx.x;
  if (threadIdx.x < 32) {
    uint32_t s = 0;
    for (int i = threadIdx.x; i < d; i += 32) s += digit_hist[i];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) s_base = s;
  }
  __syncthreads();
  uint32_t carry = s_base;
  const uint32_t* row = tile_counts + (int64_t)d * ntiles;
  uint32_t* orow = offsets + (int64_t)d * ntiles;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int64_t c0 = 0; c0 < ntiles; c0 += blockDim.x) {
    int64_t i = c0 + threadIdx.x;
    uint32_t v = i < ntiles ? row[i] : 0u;
    uint32_t x = v;  // inclusive warp scan
    for (int o = 1; o < 32; o <<= 1) {
      uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
      if (lane >= o) x += y;
    }
    if (lane == 31) warp_sums[warp] = x;
    __syncthreads();
    if (warp == 0) {
      uint32_t w = lane < nw ? warp_sums[lane] : 0u;
      for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
        if (lane >= o) w += y;
      }
      warp_sums[lane] = w;  // inclusive over warps
    }
    __syncthreads();
    uint32_t before = (warp > 0 ? warp_sums[warp - 1] : 0u) + x - v;
    if (i < ntiles) orow[i] = carry + before;
    uint32_t total = warp_sums[nw - 1];
    __syncthreads();
    carry += total;
  }
}

// Stable scatter of one tile: items are ranked per digit (warp match, warps
// in order), placed in digit order in shared memory, then written out as
// contiguous runs per digit, so consecutive threads store to consecutive
// addresses.
static_assert(SORT_BLOCK == 256, "the downsweep's digit scan maps one thread to one digit");
constexpr size_t DOWNSWEEP_SMEM = (size_t)SORT_TILE * (sizeof(uint64_t) + sizeof(uint32_t)) +
                                  (size_t)SORT_WARPS * 256 * sizeof(uint32_t) + 2 * 256 * sizeof(uint32_t);

__global__ void __launch_bounds__(SORT_BLOCK) k_downsweep(const uint64_t* __restrict__ keys_in,
                                                          const uint32_t* __restrict__ vals_in,
                                                          uint64_t* __restrict__ keys_out,
                                                          uint32_t* __restrict__ vals_out, int64_t n, int shift,
                                                          int64_t ntiles, const uint32_t* __restrict__ offsets) {
  extern __shared__ __align__(16) unsigned char ds_smem[];
  uint64_t* s_k = reinterpret_cast<uint64_t*>(ds_smem);
  uint32_t* s_v = reinterpret_cast<uint32_t*>(s_k + SORT_TILE);
  uint32_t(*wcnt)[256] = reinterpret_cast<uint32_t(*)[256]>(s_v + SORT_TILE);  // per-warp counts, then offsets
  uint32_t* toff = reinterpret_cast<uint32_t*>(wcnt + SORT_WARPS);             // global start of each digit
  uint32_t* lstart = toff + 256;                                                // start of each digit in the tile
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  for (int i = tid; i < SORT_WARPS * 256; i += SORT_BLOCK) (&wcnt[0][0])[i] = 0;
  for (int d = tid; d < 256; d += SORT_BLOCK) toff[d] = offsets[(int64_t)d * ntiles + blockIdx.x];
  __syncthreads();
  const int64_t tile0 = (int64_t)blockIdx.x * SORT_TILE;
  const int64_t seg = tile0 + (int64_t)warp * (32 * SORT_ITEMS);
  const unsigned lt_mask = (1u << lane) - 1u;
  uint64_t k[SORT_ITEMS];
  uint32_t v[SORT_ITEMS];
  uint32_t rk[SORT_ITEMS];
  uint32_t dg[SORT_ITEMS];
#pragma unroll
  for (int j = 0; j < SORT_ITEMS; ++j) {
    int64_t idx = seg + (int64_t)j * 32 + lane;
    bool ok = idx < n;
    k[j] = ok ? keys_in[idx] : 0ull;
    v[j] = ok ? vals_in[idx] : 0u;
    uint32_t d = ok ? (uint32_t)((k[j] >> shift) & 255u) : 256u;
    unsigned peers = __match_any_sync(0xffffffffu, d);
    int leader = __ffs(peers) - 1;
    uint32_t c = d < 256u ? wcnt[warp][d] : 0u;
    __syncwarp();
    if (lane == leader && d < 256u) wcnt[warp][d] = c + __popc(peers);
    __syncwarp();
    rk[j] = c + __popc(peers & lt_mask);
    dg[j] = d;
  }
  __syncthreads();
  // per digit: warp offsets (in place) and the tile total; then the digit
  // starts inside the tile by a block-wide exclusive scan (256 threads)
  uint32_t tot = 0;
  {
    const int d = tid;
#pragma unroll
    for (int w = 0; w < SORT_WARPS; ++w) {
      const uint32_t c = wcnt[w][d];
      wcnt[w][d] = tot;
      tot += c;
    }
  }
  uint32_t x = tot;  // inclusive scan of tot over the 256 threads
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
    if (lane >= o) x += y;
  }
  __shared__ uint32_t wsum[SORT_WARPS];
  if (lane == 31) wsum[warp] = x;
  __syncthreads();
  uint32_t before = 0;
  for (int w = 0; w < warp; ++w) before += wsum[w];
  lstart[tid] = before + x - tot;
  __syncthreads();
#pragma unroll
  for (int j = 0; j < SORT_ITEMS; ++j) {
    const uint32_t d = dg[j];
    if (d < 256u) {
      const uint32_t pos = lstart[d] + wcnt[warp][d] + rk[j];
      s_k[pos] = k[j];
      s_v[pos] = v[j];
    }
  }
  __syncthreads();
  const int count = (int)min((int64_t)SORT_TILE, n - tile0);
  for (int i = tid; i < count; i += SORT_BLOCK) {
    const uint64_t key = s_k[i];
    const uint32_t d = (uint32_t)((key >> shift) & 255u);
    const uint32_t pos = toff[d] + ((uint32_t)i - lstart[d]);
    keys_out[pos] = key;
    vals_out[pos] = s_v[i];
  }
}

}  // namespace

void radix_sort_u64(uint64_t* keys, uint32_t* vals, int64_t n, int key_bits, void* scratch, size_t scratch_bytes,
                    cudaStream_t s) {
  if (n <= 1) return;
  if (scratch_bytes < radix_sort_scratch_bytes(n)) throw Error(1, "radix sort scratch too small");
  int64_t ntiles = (n + SORT_TILE - 1) / SORT_TILE;
  char* p = (char*)scratch;
  auto carve = [&](size_t bytes) {
    char* r = p;
    p += (bytes + 255) & ~(size_t)255;
    return (void*)r;
  };
  uint64_t* keys_alt = (uint64_t*)carve((size_t)n * sizeof(uint64_t));
  uint32_t* vals_alt = (uint32_t*)carve((size_t)n * sizeof(uint32_t));
  uint32_t* tile_counts = (uint32_t*)carve((size_t)ntiles * 256 * sizeof(uint32_t));
  uint32_t* offsets = (uint32_t*)carve((size_t)ntiles * 256 * sizeof(uint32_t));
  uint32_t* hist = (uint32_t*)carve(8 * 256 * sizeof(uint32_t));
  (void)p;

  TPM_CUDA(cudaFuncSetAttribute(k_downsweep, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)DOWNSWEEP_SMEM));
  TPM_CUDA(cudaMemsetAsync(hist, 0, 8 * 256 * sizeof(uint32_t), s));
  k_hist8<<<grid_for(n, 256, 148 * 8), 256, 0, s>>>(keys, n, hist);
  TPM_LAUNCH_CHECK();
  uint32_t hh[8 * 256];
  TPM_CUDA(cudaMemcpyAsync(hh, hist, sizeof(hh), cudaMemcpyDeviceToHost, s));
  TPM_CUDA(cudaStreamSynchronize(s));

  uint64_t* kin = keys;
  uint32_t* vin = vals;
  uint64_t* kout = keys_alt;
  uint32_t* vout = vals_alt;
  int npass = (key_bits + 7) / 8;
  if (npass > 8) npass = 8;
  for (int pass = 0; pass < npass; ++pass) {
    bool constant = false;
    for (int d = 0; d < 256; ++d)
      if (hh[pass * 256 + d] == (uint32_t)n) constant = true;
    if (constant) continue;
    int shift = 8 * pass;
    k_upsweep<<<(unsigned)ntiles, SORT_BLOCK, 0, s>>>(kin, n, shift, ntiles, tile_counts);
    TPM_LAUNCH_CHECK();
    k_scan_tiles<<<256, 1024, 0, s>>>(tile_counts, hist + pass * 256, ntiles, offsets);
    TPM_LAUNCH_CHECK();
    k_downsweep<<<(unsigned)ntiles, SORT_BLOCK, DOWNSWEEP_SMEM, s>>>(kin, vin, kout, vout, n, shift, ntiles, offsets);
    TPM_LAUNCH_CHECK();
    std::swap(kin, kout);
    std::swap(vin, vout);
  }
  if (kin != keys) {
    TPM_CUDA(cudaMemcpyAsync(keys, kin, (size_t)n * sizeof(uint64_t), cudaMemcpyDeviceToDevice, s));
    TPM_CUDA(cudaMemcpyAsync(vals, vin, (size_t)n * sizeof(uint32_t), cudaMemcpyDeviceToDevice, s));
  }
}

void radix_sort_u64_all_passes(uint64_t* keys, uint32_t* vals, int64_t n, void* scratch, size_t scratch_bytes,
                               cudaStream_t s) {
  if (n <= 1) return;
  if (scratch_bytes < radix_sort_scratch_bytes(n)) throw Error(1, "radix sort scratch too small");
  int64_t ntiles = (n + SORT_TILE - 1) / SORT_TILE;
  char* p = (char*)scratch;
  auto carve = [&](size_t bytes) {
    char* r = p;
    p += (bytes + 255) & ~(size_t)255;
    return (void*)r;
  };
  uint64_t* keys_alt = (uint64_t*)carve((size_t)n * sizeof(uint64_t));
  uint32_t* vals_alt = (uint32_t*)carve((size_t)n * sizeof(uint32_t));
  uint32_t* tile_counts = (uint32_t*)carve((size_t)ntiles * 256 * sizeof(uint32_t));
  uint32_t* offsets = (uint32_t*)carve((size_t)ntiles * 256 * sizeof(uint32_t));
  uint32_t* hist = (uint32_t*)carve(8 * 256 * sizeof(uint32_t));
  TPM_CUDA(cudaFuncSetAttribute(k_downsweep, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)DOWNSWEEP_SMEM));
  TPM_CUDA(cudaMemsetAsync(hist, 0, 8 * 256 * sizeof(uint32_t), s));
  k_hist8<<<grid_for(n, 256, 148 * 8), 256, 0, s>>>(keys, n, hist);
  TPM_LAUNCH_CHECK();
  uint64_t* kin = keys;
  uint32_t* vin = vals;
  uint64_t* kout = keys_alt;
  uint32_t* vout = vals_alt;
  for (int pass = 0; pass < 8; ++pass) {  // eight passes: the result ends in keys / vals
    const int shift = 8 * pass;
    k_upsweep<<<(unsigned)ntiles, SORT_BLOCK, 0, s>>>(kin, n, shift, ntiles, tile_counts);
    TPM_LAUNCH_CHECK();
    k_scan_tiles<<<256, 1024, 0, s>>>(tile_counts, hist + pass * 256, ntiles, offsets);
    TPM_LAUNCH_CHECK();
    k_downsweep<<<(unsigned)ntiles, SORT_BLOCK, DOWNSWEEP_SMEM, s>>>(kin, vin, kout, vout, n, shift, ntiles, offsets);
    TPM_LAUNCH_CHECK();
    std::swap(kin, kout);
    std::swap(vin, vout);
  }
}

}  // namespace tpm
