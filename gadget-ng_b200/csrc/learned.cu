// Learned short range inside a force evaluation.  The network runs once over
// the whole periodic mesh: the features are padded by 3 nodes on each side,
// so three valid convolutions leave exactly one output per mesh node, each
// seeing its 7^3 neighbourhood (the same values a tiling of patches would
// give).  Particles whose 8 CIC nodes are all at or below the density limit
// read the head there by the PM gather's CIC weights; the rest keep the tree
// walk, run only over the walk groups that hold them.
#include <cuda_bf16.h>

#include <cmath>

#include "common.cuh"
#include "learned.cuh"
#include "scan.cuh"

namespace tpm {
namespace {

struct Feat {
  float shift[cnn::MAX_CIN];
  float scale[cnn::MAX_CIN];
};

__global__ void k_mesh_features(const float* __restrict__ rho, const float* __restrict__ phi,
                                const float* __restrict__ oct, int nm, float inv_mcell, float cell_over_mcell,
                                int c_in, Feat f, __nv_bfloat16* __restrict__ vol) {
  const int P = nm + 6;
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= (int64_t)P * P * P) return;
  const int x = (int)(i % P), y = (int)((i / P) % P), z = (int)(i / ((int64_t)P * P));
  const int mx = (x - 3 + nm) % nm, my = (y - 3 + nm) % nm, mz = (z - 3 + nm) % nm;
  const int64_t node = ((int64_t)mz * nm + my) * nm + mx;
  float v[16];
#pragma unroll
  for (int c = 0; c < 16; ++c)
    v[c] = c < c_in ? (raw_feature(c, node, rho, phi, oct, inv_mcell, cell_over_mcell) - f.shift[c]) * f.scale[c]
                    : 0.f;
  uint32_t w[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    __nv_bfloat162 h = __floats2bfloat162_rn(v[2 * k], v[2 * k + 1]);
    w[k] = *reinterpret_cast<uint32_t*>(&h);
  }
  uint4* d = reinterpret_cast<uint4*>(vol) + i * 2;
  d[0] = make_uint4(w[0], w[1], w[2], w[3]);
  d[1] = make_uint4(w[4], w[5], w[6], w[7]);
}

__global__ void k_octant_deposit(const uint32_t* __restrict__ qx, const uint32_t* __restrict__ qy,
                                 const uint32_t* __restrict__ qz, const float* __restrict__ m, int64_t n,
                                 double scale, double inv_cell, int nm, float* __restrict__ oct) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t q[3] = {qx[i], qy[i], qz[i]};
  int node[3], bits = 0;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double c = rem_euclid(dmul(decode(q[d], scale), inv_cell), (double)nm) + 0.5;
    const double f = floor(c);
    node[d] = ((int)f) % nm;
    bits |= (c - f >= 0.5 ? 1 : 0) << d;
  }
  atomicAdd(&oct[((((int64_t)node[2] * nm + node[1]) * nm + node[0]) << 3) + bits], m[i]);
}

__device__ __forceinline__ int cic_cell(uint32_t q, double scale, double inv_cell, int nm) {
  const double c = rem_euclid(dmul(decode(q, scale), inv_cell), (double)nm);
  return min((int)floor(c), nm - 1);
}

__global__ void k_cell_count(const uint32_t* __restrict__ qx, const uint32_t* __restrict__ qy,
                             const uint32_t* __restrict__ qz, int64_t n, double scale, double inv_cell, int nm,
                             uint32_t* __restrict__ cell_of, uint32_t* __restrict__ counts) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int x = cic_cell(qx[i], scale, inv_cell, nm), y = cic_cell(qy[i], scale, inv_cell, nm),
            z = cic_cell(qz[i], scale, inv_cell, nm);
  const uint32_t c = (uint32_t)(((int64_t)z * nm + y) * nm + x);
  cell_of[i] = c;
  atomicAdd(&counts[c], 1u);
}

__global__ void k_cell_fill(const uint32_t* __restrict__ cell_of, int64_t n, const uint32_t* __restrict__ start,
                            uint32_t* __restrict__ cursor, uint32_t* __restrict__ items) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t c = cell_of[i];
  items[start[c] + atomicAdd(&cursor[c], 1u)] = (uint32_t)i;
}

__global__ void k_near(NearField f, float scale, float r_near2, float inv_s2rs, float eps2) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= f.n || (f.skip && f.skip[i])) return;
  const int nm = f.nm;
  const uint32_t c = f.cell_of[i];
  const int cx = (int)(c % nm), cy = (int)((c / nm) % nm), cz = (int)(c / ((uint32_t)nm * nm));
  const uint32_t qi[3] = {f.qx[i], f.qy[i], f.qz[i]};
  float ax = 0.f, ay = 0.f, az = 0.f;
  for (int d = 0; d < 27; ++d) {
    const int x = (cx + d % 3 - 1 + nm) % nm, y = (cy + (d / 3) % 3 - 1 + nm) % nm, z = (cz + d / 9 - 1 + nm) % nm;
    const int64_t nc = ((int64_t)z * nm + y) * nm + x;
    const uint32_t e = f.start[nc + 1];
    for (uint32_t k = f.start[nc]; k < e; ++k) {
      const uint32_t j = f.items[k];
      if (j == (uint32_t)i) continue;
      // exact minimum image of the fixed-point difference, then one rounding
      const float dx = (float)(int32_t)(f.qx[j] - qi[0]) * scale;
      const float dy = (float)(int32_t)(f.qy[j] - qi[1]) * scale;
      const float dz = (float)(int32_t)(f.qz[j] - qi[2]) * scale;
      const float r2b = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
      if (r2b >= r_near2) continue;
      const float r2 = r2b + eps2;
      const float r = sqrtf(r2);
      const float xx = r * inv_s2rs;
      const float w = erfcf(xx) + 1.1283791670955126f * xx * expf(-xx * xx);
      const float g = f.mass[j] * w / (r2 * r);
      ax = fmaf(g, dx, ax);
      ay = fmaf(g, dy, ay);
      az = fmaf(g, dz, az);
    }
  }
  f.nx[i] = ax;
  f.ny[i] = ay;
  f.nz[i] = az;
}

struct Nodes {
  int i0[3], i1[3];
  float w0[3], w1[3];
};

// CIC nodes and weights of the PM gather (cic.rs:100-170 arithmetic).
__device__ __forceinline__ Nodes nodes_of(uint32_t qx, uint32_t qy, uint32_t qz, double scale, double inv_cell,
                                          int nm) {
  Nodes r;
  const uint32_t q[3] = {qx, qy, qz};
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double c = rem_euclid(dmul(decode(q[d], scale), inv_cell), (double)nm);
    const double f = floor(c);
    const int i0 = (int)f;
    const double t = dsub(c, f);
    r.i0[d] = i0;
    r.i1[d] = (i0 + 1) % nm;
    r.w0[d] = (float)dsub(1.0, t);
    r.w1[d] = (float)t;
  }
  return r;
}

__device__ __forceinline__ int64_t corner(const Nodes& r, int k, int nm) {
  const int x = (k & 1) ? r.i1[0] : r.i0[0], y = ((k >> 1) & 1) ? r.i1[1] : r.i0[1], z = (k >> 2) ? r.i1[2] : r.i0[2];
  return ((int64_t)z * nm + y) * nm + x;
}

__global__ void k_learned_mask(const uint32_t* __restrict__ qx, const uint32_t* __restrict__ qy,
                               const uint32_t* __restrict__ qz, int64_t n, double scale, double inv_cell, int nm,
                               const float* __restrict__ rho, float rho_max, uint8_t* __restrict__ fallback,
                               unsigned long long* __restrict__ count) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  bool net = false;
  if (i < n) {
    const Nodes r = nodes_of(qx[i], qy[i], qz[i], scale, inv_cell, nm);
    net = true;
#pragma unroll
    for (int k = 0; k < 8; ++k) net = net && rho[corner(r, k, nm)] <= rho_max;
    fallback[i] = net ? 0 : 1;
  }
  const unsigned m = __ballot_sync(0xffffffffu, net);
  if ((threadIdx.x & 31) == 0 && m) atomicAdd(count, (unsigned long long)__popc(m));
}

__global__ void k_learned_groups(const uint32_t* __restrict__ gfirst, const uint32_t* __restrict__ gsize,
                                 int64_t ngroups, const uint8_t* __restrict__ fallback, uint32_t* __restrict__ of,
                                 uint32_t* __restrict__ os, uint32_t* __restrict__ oc) {
  const int64_t g = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (g >= ngroups) return;
  const uint32_t f = gfirst[g], c = gsize[g];
  bool any = false;
  for (uint32_t k = 0; k < c && !any; ++k) any = fallback[f + k] != 0;
  if (!any) return;
  const uint32_t slot = atomicAdd(oc, 1u);
  of[slot] = f;
  os[slot] = c;
}

__global__ void k_learned_apply(const uint32_t* __restrict__ qx, const uint32_t* __restrict__ qy,
                                const uint32_t* __restrict__ qz, int64_t n, double scale, double inv_cell, int nm,
                                const uint8_t* __restrict__ fallback, const __nv_bfloat16* __restrict__ a3,
                                const float* __restrict__ p, int64_t wh, int64_t bh, float out_unit, int add,
                                float* __restrict__ srx, float* __restrict__ sry, float* __restrict__ srz) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n || fallback[i]) return;
  const Nodes r = nodes_of(qx[i], qy[i], qz[i], scale, inv_cell, nm);
  float acc[16];
#pragma unroll
  for (int k = 0; k < 16; ++k) acc[k] = 0.f;
  // the head is linear: interpolate the 16 activations, then apply it once
#pragma unroll 1
  for (int k = 0; k < 8; ++k) {
    const float wk = ((k & 1) ? r.w1[0] : r.w0[0]) * (((k >> 1) & 1) ? r.w1[1] : r.w0[1]) *
                     ((k >> 2) ? r.w1[2] : r.w0[2]);
    const uint4* src = reinterpret_cast<const uint4*>(a3) + corner(r, k, nm) * 2;
    const uint4 u0 = src[0], u1 = src[1];
    const uint32_t u[8] = {u0.x, u0.y, u0.z, u0.w, u1.x, u1.y, u1.z, u1.w};
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const float2 v = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&u[j]));
      acc[2 * j] = fmaf(wk, v.x, acc[2 * j]);
      acc[2 * j + 1] = fmaf(wk, v.y, acc[2 * j + 1]);
    }
  }
  float o[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    float s = p[bh + c];
#pragma unroll
    for (int k = 0; k < 16; ++k) s = fmaf(p[wh + c * 16 + k], acc[k], s);
    o[c] = s * out_unit;
  }
  if (add) {
    srx[i] += o[0];
    sry[i] += o[1];
    srz[i] += o[2];
  } else {
    srx[i] = o[0];
    sry[i] = o[1];
    srz[i] = o[2];
  }
}

}  // namespace

void learned_mesh(const LearnedNet& net, const LearnedMesh& m, uint32_t* err, cudaStream_t s) {
  const int nm = m.nm, P = nm + 6;
  const double cell = m.box / nm;
  Feat f{};
  for (int k = 0; k < cnn::MAX_CIN; ++k) {
    f.shift[k] = net.shift[k];
    f.scale[k] = net.scale[k];
  }
  const int64_t np = (int64_t)P * P * P;
  k_mesh_features<<<grid_for(np, 256, 1ll << 30), 256, 0, s>>>(m.rho, m.phi, m.octants, nm, (float)(1.0 / m.m_cell),
                                                               (float)(cell / m.m_cell), net.L.c_in, f, m.vol_a);
  TPM_LAUNCH_CHECK();
  cnn::conv_forward(m.vol_a, cnn::Vol{1, P, P, P}, m.vol_b, nullptr, net.fwd[0], net.params + net.L.b[0], err, s);
  cnn::conv_forward(m.vol_b, cnn::Vol{1, P - 2, P - 2, P - 2}, m.vol_a, nullptr, net.fwd[1],
                    net.params + net.L.b[1], err, s);
  cnn::conv_forward(m.vol_a, cnn::Vol{1, P - 4, P - 4, P - 4}, m.vol_b, nullptr, net.fwd[2],
                    net.params + net.L.b[2], err, s);
}

void octant_deposit(const uint32_t* qx, const uint32_t* qy, const uint32_t* qz, const float* mass, int64_t n,
                    int nm, double box, float* oct, cudaStream_t s) {
  TPM_CUDA(cudaMemsetAsync(oct, 0, sizeof(float) * 8 * (size_t)nm * nm * nm, s));
  if (n == 0) return;
  k_octant_deposit<<<grid_for(n, 256, 1ll << 30), 256, 0, s>>>(qx, qy, qz, mass, n, box / TWO32, nm / box, nm, oct);
  TPM_LAUNCH_CHECK();
}

void cell_list(const uint32_t* qx, const uint32_t* qy, const uint32_t* qz, int64_t n, int nm, double box,
               uint32_t* cell_of, uint32_t* cursor, uint32_t* start, uint32_t* items, void* scan_scratch,
               cudaStream_t s) {
  const int64_t nm3 = (int64_t)nm * nm * nm;
  TPM_CUDA(cudaMemsetAsync(cursor, 0, sizeof(uint32_t) * (nm3 + 1), s));
  if (n > 0) {
    k_cell_count<<<grid_for(n, 256, 1ll << 30), 256, 0, s>>>(qx, qy, qz, n, box / TWO32, nm / box, nm, cell_of, cursor);
    TPM_LAUNCH_CHECK();
  }
  exclusive_scan_u32(cursor, start, nm3 + 1, nullptr, scan_scratch, s);
  TPM_CUDA(cudaMemsetAsync(cursor, 0, sizeof(uint32_t) * (nm3 + 1), s));
  if (n > 0) {
    k_cell_fill<<<grid_for(n, 256, 1ll << 30), 256, 0, s>>>(cell_of, n, start, cursor, items);
    TPM_LAUNCH_CHECK();
  }
}

void near_field(const NearField& f, cudaStream_t s) {
  if (f.n == 0) return;
  const float rn = (float)f.r_near;
  k_near<<<grid_for(f.n, 128, 1ll << 30), 128, 0, s>>>(f, (float)(f.box / TWO32), rn * rn,
                                                       (float)(1.0 / (std::sqrt(2.0) * f.r_split)), (float)f.eps2);
  TPM_LAUNCH_CHECK();
}

void learned_mask(const uint32_t* qx, const uint32_t* qy, const uint32_t* qz, int64_t n, const LearnedNet& net,
                  const LearnedMesh& m, uint8_t* fallback, unsigned long long* count, cudaStream_t s) {
  if (n == 0) return;
  const float rho_max = (float)((1.0 + net.delta_max) * m.m_cell);
  k_learned_mask<<<grid_for(n, 256, 1ll << 30), 256, 0, s>>>(qx, qy, qz, n, m.box / TWO32, m.nm / m.box, m.nm, m.rho,
                                                             rho_max, fallback, count);
  TPM_LAUNCH_CHECK();
}

void learned_groups(const uint32_t* gfirst, const uint32_t* gsize, int64_t ngroups, const uint8_t* fallback,
                    uint32_t* out_first, uint32_t* out_size, uint32_t* out_count, cudaStream_t s) {
  TPM_CUDA(cudaMemsetAsync(out_count, 0, sizeof(uint32_t), s));
  if (ngroups == 0) return;
  k_learned_groups<<<grid_for(ngroups, 256, 1ll << 30), 256, 0, s>>>(gfirst, gsize, ngroups, fallback, out_first,
                                                                     out_size, out_count);
  TPM_LAUNCH_CHECK();
}

void learned_apply(const uint32_t* qx, const uint32_t* qy, const uint32_t* qz, int64_t n, const LearnedNet& net,
                   const LearnedMesh& m, const uint8_t* fallback, float* srx, float* sry, float* srz,
                   cudaStream_t s) {
  if (n == 0) return;
  const double cell = m.box / m.nm;
  const float out_unit = (float)(net.out_scale * m.m_cell / (cell * cell));
  k_learned_apply<<<grid_for(n, 256, 1ll << 30), 256, 0, s>>>(qx, qy, qz, n, m.box / TWO32, m.nm / m.box, m.nm,
                                                              fallback, m.vol_b, net.params, net.L.wh, net.L.bh,
                                                              out_unit, net.near_cells > 0.f ? 1 : 0, srx, sry, srz);
  TPM_LAUNCH_CHECK();
}

}  // namespace tpm
