// Domain-decomposed TreePM: halo selection, packing, append and compaction
// on the device (see domain.cuh).
#include "common.cuh"
#include "domain.cuh"
#include "scan.cuh"

namespace tpm {
namespace {

__global__ void k_bounds(const uint32_t* __restrict__ qx, const uint32_t* __restrict__ qy,
                         const uint32_t* __restrict__ qz, int64_t n, uint32_t* out6) {
  uint32_t mn[3] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu}, mx[3] = {0u, 0u, 0u};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    const uint32_t q[3] = {qx[i], qy[i], qz[i]};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      mn[d] = min(mn[d], q[d]);
      mx[d] = max(mx[d], q[d]);
    }
  }
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    mn[d] = __reduce_min_sync(0xffffffffu, mn[d]);
    mx[d] = __reduce_max_sync(0xffffffffu, mx[d]);
  }
  if ((threadIdx.x & 31) == 0) {
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      atomicMin(&out6[2 * d], mn[d]);
      atomicMax(&out6[2 * d + 1], mx[d]);
    }
  }
}

// min_dist2_to_aabb_3d_periodic (crates/gadget-ng-parallel/src/halo3d.rs:237-251):
// centre and half extents of the box, minimum image of centre - p per axis
// (minimum_image_scalar, halo3d.rs, the same expression as short_range.rs:53-63),
// excess = max(|d| - half, 0), summed in axis order; float64 without contraction.
__device__ __forceinline__ double aabb_dist2_periodic(const double p[3], const double* a, double box) {
  double d2 = 0.0;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const double lo = a[2 * k], hi = a[2 * k + 1];
    const double com = dmul(dadd(lo, hi), 0.5);
    const double half = dmul(dsub(hi, lo), 0.5);
    const double d = minimum_image(dsub(com, p[k]), box);
    const double x = dsub(fabs(d), half);
    const double e = x > 0.0 ? x : 0.0;
    d2 = dadd(d2, dmul(e, e));
  }
  return d2;
}

__global__ void k_halo_flags(const uint32_t* __restrict__ qx, const uint32_t* __restrict__ qy,
                             const uint32_t* __restrict__ qz, int64_t n, double scale, double box, AabbTable t,
                             int n_ranks, int rank, double w2, uint64_t* __restrict__ flags,
                             unsigned long long* __restrict__ counts) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const bool live = i < n;
  uint64_t f = 0;
  if (live) {
    const double p[3] = {decode(qx[i], scale), decode(qy[i], scale), decode(qz[i], scale)};
    for (int r = 0; r < n_ranks; ++r) {
      if (r == rank) continue;
      const double* a = &t.v[6 * r];
      // Aabb3::is_valid: lo <= hi on every axis (false for the empty box and NaN)
      if (!(a[0] <= a[1] && a[2] <= a[3] && a[4] <= a[5])) continue;
      if (aabb_dist2_periodic(p, a, box) < w2) f |= 1ull << r;
    }
    flags[i] = f;
  }
  // per-rank counts, one atomic per warp and rank
  const uint64_t any = __reduce_or_sync(0xffffffffu, (uint32_t)f) | ((uint64_t)__reduce_or_sync(0xffffffffu, (uint32_t)(f >> 32)) << 32);
  uint64_t rest = any;
  while (rest) {
    const int r = __ffsll((long long)rest) - 1;
    rest &= rest - 1;
    const unsigned c = __popc(__ballot_sync(0xffffffffu, (f >> r) & 1ull));
    if ((threadIdx.x & 31) == 0) atomicAdd(&counts[r], (unsigned long long)c);
  }
}

__device__ __forceinline__ int cell_of(uint32_t q, int g) { return (int)(((uint64_t)q * (uint64_t)g) >> 32); }

__global__ void k_occupancy(const uint32_t* __restrict__ qx, const uint32_t* __restrict__ qy,
                            const uint32_t* __restrict__ qz, int64_t n, int g, uint32_t* __restrict__ bits) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t c = ((int64_t)cell_of(qz[i], g) * g + cell_of(qy[i], g)) * g + cell_of(qx[i], g);
  const uint32_t w = (uint32_t)(c >> 5), b = 1u << (c & 31);
  // one atomic per word and warp
  const uint32_t peers = __match_any_sync(__activemask(), w);
  const uint32_t m = __reduce_or_sync(peers, b);
  if ((threadIdx.x & 31) == __ffs(peers) - 1) atomicOr(&bits[w], m);
}

// the gap between coordinate x (in cell ci) and the neighbour cell at offset o
__device__ __forceinline__ double face_gap(double x, int ci, int o, double cell) {
  if (o == 0) return 0.0;
  return o > 0 ? dsub(dmul((double)(ci + 1), cell), x) : dsub(x, dmul((double)ci, cell));
}

__global__ void k_halo_flags_cells(const uint32_t* __restrict__ qx, const uint32_t* __restrict__ qy,
                                   const uint32_t* __restrict__ qz, int64_t n, double scale, double cell, int g,
                                   const uint32_t* __restrict__ bits, int64_t words, int n_ranks, int rank,
                                   double w2, uint64_t* __restrict__ flags, unsigned long long* __restrict__ counts) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const bool live = i < n;
  uint64_t f = 0;
  if (live) {
    const uint32_t q[3] = {qx[i], qy[i], qz[i]};
    int ci[3];
    double x[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      ci[k] = cell_of(q[k], g);
      x[k] = decode(q[k], scale);
    }
    for (int oz = -1; oz <= 1; ++oz)
      for (int oy = -1; oy <= 1; ++oy)
        for (int ox = -1; ox <= 1; ++ox) {
          const double gx = face_gap(x[0], ci[0], ox, cell), gy = face_gap(x[1], ci[1], oy, cell);
          const double gz = face_gap(x[2], ci[2], oz, cell);
          if (!(dadd(dadd(dmul(gx, gx), dmul(gy, gy)), dmul(gz, gz)) < w2)) continue;
          const int cx = (ci[0] + ox + g) % g, cy = (ci[1] + oy + g) % g, cz = (ci[2] + oz + g) % g;
          const int64_t c = ((int64_t)cz * g + cy) * g + cx;
          for (int r = 0; r < n_ranks; ++r)
            if (r != rank && ((__ldg(&bits[r * words + (c >> 5)]) >> (c & 31)) & 1u)) f |= 1ull << r;
        }
    flags[i] = f;
  }
  const uint64_t any = __reduce_or_sync(0xffffffffu, (uint32_t)f) |
                       ((uint64_t)__reduce_or_sync(0xffffffffu, (uint32_t)(f >> 32)) << 32);
  uint64_t rest = any;
  while (rest) {
    const int r = __ffsll((long long)rest) - 1;
    rest &= rest - 1;
    const unsigned cnt = __popc(__ballot_sync(0xffffffffu, (f >> r) & 1ull));
    if ((threadIdx.x & 31) == 0) atomicAdd(&counts[r], (unsigned long long)cnt);
  }
}

__global__ void k_bit(const uint64_t* __restrict__ flags, int64_t n, int r, uint32_t* __restrict__ bit) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) bit[i] = (uint32_t)((flags[i] >> r) & 1ull);
}

__global__ void k_pack(const uint32_t* __restrict__ qx, const uint32_t* __restrict__ qy,
                       const uint32_t* __restrict__ qz, const uint32_t* __restrict__ id, const double* __restrict__ mass,
                       int64_t n, const uint32_t* __restrict__ bit, const uint32_t* __restrict__ pos,
                       HaloRecord* __restrict__ out) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n || !bit[i]) return;
  HaloRecord r;
  r.q[0] = qx[i];
  r.q[1] = qy[i];
  r.q[2] = qz[i];
  r.id = id[i];
  r.mass = mass[i];
  out[pos[i]] = r;
}

__global__ void k_owned_flag(const uint32_t* __restrict__ id, int64_t n, uint32_t n_owned, uint32_t* __restrict__ flag) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) flag[i] = id[i] < n_owned ? 1u : 0u;
}

__global__ void k_compact(Particles src, Particles dst, int64_t n, const uint32_t* __restrict__ flag,
                          const uint32_t* __restrict__ pos, const float* __restrict__ ax, const float* __restrict__ ay,
                          const float* __restrict__ az, float* __restrict__ tx, float* __restrict__ ty,
                          float* __restrict__ tz) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n || !flag[i]) return;
  const uint32_t j = pos[i];
  dst.qx[j] = src.qx[i];
  dst.qy[j] = src.qy[i];
  dst.qz[j] = src.qz[i];
  dst.vx[j] = src.vx[i];
  dst.vy[j] = src.vy[i];
  dst.vz[j] = src.vz[i];
  dst.mass[j] = src.mass[i];
  dst.massf[j] = src.massf[i];
  dst.id[j] = src.id[i];
  tx[j] = ax[i];
  ty[j] = ay[i];
  tz[j] = az[i];
}

__global__ void k_append(Particles P, int64_t first, const HaloRecord* __restrict__ rec, int64_t m) {
  const int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k >= m) return;
  const HaloRecord r = rec[k];
  const int64_t j = first + k;
  P.qx[j] = r.q[0];
  P.qy[j] = r.q[1];
  P.qz[j] = r.q[2];
  P.vx[j] = 0.f;
  P.vy[j] = 0.f;
  P.vz[j] = 0.f;
  P.mass[j] = r.mass;
  P.massf[j] = (float)r.mass;
  P.id[j] = (uint32_t)j;
}

__global__ void k_owned_mask(const uint32_t* __restrict__ id, int64_t n, uint32_t n_owned, uint8_t* __restrict__ mask) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) mask[i] = id[i] < n_owned ? 1 : 0;
}

unsigned blocks_of(int64_t n) { return (unsigned)((n + 255) / 256 > 0 ? (n + 255) / 256 : 1); }

}  // namespace

void owned_bounds(const Particles& P, int64_t n, uint32_t* scratch6, uint32_t out6[6], cudaStream_t s) {
  const uint32_t init[6] = {0xFFFFFFFFu, 0u, 0xFFFFFFFFu, 0u, 0xFFFFFFFFu, 0u};
  TPM_CUDA(cudaMemcpyAsync(scratch6, init, sizeof(init), cudaMemcpyHostToDevice, s));
  if (n > 0) {
    k_bounds<<<grid_for(n, 256, 148 * 8), 256, 0, s>>>(P.qx, P.qy, P.qz, n, scratch6);
    TPM_LAUNCH_CHECK();
  }
  TPM_CUDA(cudaMemcpyAsync(out6, scratch6, sizeof(uint32_t) * 6, cudaMemcpyDeviceToHost, s));
  TPM_CUDA(cudaStreamSynchronize(s));
}

void halo_flags(const Particles& P, int64_t n, double scale, double box, const AabbTable& t, int n_ranks, int rank,
                double w2, uint64_t* flags, unsigned long long* counts_dev, cudaStream_t s) {
  TPM_CUDA(cudaMemsetAsync(counts_dev, 0, sizeof(unsigned long long) * MAX_RANKS, s));
  if (n == 0) return;
  k_halo_flags<<<blocks_of(n), 256, 0, s>>>(P.qx, P.qy, P.qz, n, scale, box, t, n_ranks, rank, w2, flags, counts_dev);
  TPM_LAUNCH_CHECK();
}

void occupancy(const Particles& P, int64_t n, int grid, uint32_t* bits, cudaStream_t s) {
  const int64_t words = ((int64_t)grid * grid * grid + 31) / 32;
  TPM_CUDA(cudaMemsetAsync(bits, 0, sizeof(uint32_t) * words, s));
  if (n == 0) return;
  k_occupancy<<<blocks_of(n), 256, 0, s>>>(P.qx, P.qy, P.qz, n, grid, bits);
  TPM_LAUNCH_CHECK();
}

void halo_flags_cells(const Particles& P, int64_t n, double scale, double cell, int grid, const uint32_t* bits,
                      int64_t words, int n_ranks, int rank, double w2, uint64_t* flags,
                      unsigned long long* counts_dev, cudaStream_t s) {
  TPM_CUDA(cudaMemsetAsync(counts_dev, 0, sizeof(unsigned long long) * MAX_RANKS, s));
  if (n == 0) return;
  k_halo_flags_cells<<<blocks_of(n), 256, 0, s>>>(P.qx, P.qy, P.qz, n, scale, cell, grid, bits, words, n_ranks, rank,
                                                  w2, flags, counts_dev);
  TPM_LAUNCH_CHECK();
}

void halo_pack(const Particles& P, int64_t n, const uint64_t* flags, int r, uint32_t* bit, uint32_t* pos,
               void* scan_scratch, HaloRecord* out, cudaStream_t s) {
  if (n == 0) return;
  k_bit<<<blocks_of(n), 256, 0, s>>>(flags, n, r, bit);
  TPM_LAUNCH_CHECK();
  exclusive_scan_u32(bit, pos, n, nullptr, scan_scratch, s);
  k_pack<<<blocks_of(n), 256, 0, s>>>(P.qx, P.qy, P.qz, P.id, P.mass, n, bit, pos, out);
  TPM_LAUNCH_CHECK();
}

void compact_owned(const Particles& src, const Particles& dst, int64_t n, uint32_t n_owned, const float* ax,
                   const float* ay, const float* az, float* tx, float* ty, float* tz, uint32_t* flag, uint32_t* pos,
                   void* scan_scratch, cudaStream_t s) {
  if (n == 0) return;
  k_owned_flag<<<blocks_of(n), 256, 0, s>>>(src.id, n, n_owned, flag);
  TPM_LAUNCH_CHECK();
  exclusive_scan_u32(flag, pos, n, nullptr, scan_scratch, s);
  k_compact<<<blocks_of(n), 256, 0, s>>>(src, dst, n, flag, pos, ax, ay, az, tx, ty, tz);
  TPM_LAUNCH_CHECK();
}

void append_halos(const Particles& P, int64_t first, const HaloRecord* rec, int64_t m, cudaStream_t s) {
  if (m == 0) return;
  k_append<<<blocks_of(m), 256, 0, s>>>(P, first, rec, m);
  TPM_LAUNCH_CHECK();
}

void owned_mask(const uint32_t* id, int64_t n, uint32_t n_owned, uint8_t* mask, cudaStream_t s) {
  if (n == 0) return;
  k_owned_mask<<<blocks_of(n), 256, 0, s>>>(id, n, n_owned, mask);
  TPM_LAUNCH_CHECK();
}

}  // namespace tpm
