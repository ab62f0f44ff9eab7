// C ABI of the learned short-range network: parameters, forward and
// gradients on host batches (for the checks against the CPU restatement),
// Adam, the training set captured from solver handles and the training loop.
// No counterpart exists in the reference.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "../../include/treepm_b200.h"
#include "cnn_api.h"
#include "common.cuh"
#include "learned.cuh"
#include "scan.cuh"

using tpm::Error;
using tpm::grid_for;
namespace cn = tpm::cnn;

namespace {

constexpr int PATCH_IN = 14;   // input side of a training patch
constexpr int PATCH_OUT = 8;   // output side (three valid convolutions)
constexpr int PATCH_CELLS = 7;  // particles of the inner 7^3 cells are read inside the output
constexpr int PCAP = 2048;     // particle slots of one patch

struct Norm {
  float shift[cn::MAX_CIN];
  float scale[cn::MAX_CIN];
};

struct BoxView {
  int nm;
  const float* feats;
  const uint32_t* start;
  const float4* pdat;
  const float4* ptgt;
};

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__device__ __forceinline__ void store16f(__nv_bfloat16* dst, const float* v) {
  uint32_t w[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    __nv_bfloat162 h = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
    w[i] = *reinterpret_cast<uint32_t*>(&h);
  }
  uint4* d = reinterpret_cast<uint4*>(dst);
  d[0] = make_uint4(w[0], w[1], w[2], w[3]);
  d[1] = make_uint4(w[4], w[5], w[6], w[7]);
}

__global__ void k_x0_from_f32(const float* __restrict__ x, int64_t nodes, int c_in, __nv_bfloat16* __restrict__ x0) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= nodes) return;
  float v[16];
#pragma unroll
  for (int c = 0; c < 16; ++c) v[c] = c < c_in ? x[i * c_in + c] : 0.f;
  store16f(x0 + i * 16, v);
}

// ---- capture of a training box ------------------------------------------------
__global__ void k_box_feats(const float* __restrict__ rho, const float* __restrict__ phi,
                            const float* __restrict__ oct, int64_t nm3, float inv_mcell, float cell_over_mcell,
                            int c_in, float* __restrict__ feats) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= nm3) return;
  for (int c = 0; c < c_in; ++c) feats[i * c_in + c] = tpm::raw_feature(c, i, rho, phi, oct, inv_mcell, cell_over_mcell);
}

struct Capture {
  int64_t n;
  const uint32_t *qx, *qy, *qz;
  double scale, inv_cell;
  int nm;
  const float* rho;
  float rho_max;
  const float *srx, *sry, *srz, *lrx, *lry, *lrz;
  const float *nrx, *nry, *nrz;
  float inv_g, a_unit_inv;
};

// Target of particle i: the short range minus its exact near-field part.
__device__ __forceinline__ float3 target_of(const Capture& c, int64_t i) {
  float3 t = make_float3(c.srx[i], c.sry[i], c.srz[i]);
  if (c.nrx) {
    t.x -= c.nrx[i];
    t.y -= c.nry[i];
    t.z -= c.nrz[i];
  }
  return make_float3(t.x * c.a_unit_inv, t.y * c.a_unit_inv, t.z * c.a_unit_inv);
}

__device__ __forceinline__ void node_coord(uint32_t q, double scale, double inv_cell, int nm, int* i0, float* s) {
  const double c = tpm::rem_euclid(tpm::dmul(tpm::decode(q, scale), inv_cell), (double)nm);
  const double f = floor(c);
  *i0 = min((int)f, nm - 1);
  *s = (float)c;
}

// Cell of each particle whose 8 CIC nodes are all at or below rho_max (-1
// otherwise), the per-cell counts and sums for the normalisation.
__global__ void k_box_pass1(Capture c, int32_t* __restrict__ cell_of, uint32_t* __restrict__ counts,
                            double* __restrict__ sums) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= c.n) return;
  int ix, iy, iz;
  float s[3];
  node_coord(c.qx[i], c.scale, c.inv_cell, c.nm, &ix, &s[0]);
  node_coord(c.qy[i], c.scale, c.inv_cell, c.nm, &iy, &s[1]);
  node_coord(c.qz[i], c.scale, c.inv_cell, c.nm, &iz, &s[2]);
  const int nm = c.nm;
  bool ok = true;
  for (int k = 0; k < 8 && ok; ++k) {
    const int x = (ix + (k & 1)) % nm, y = (iy + ((k >> 1) & 1)) % nm, z = (iz + (k >> 2)) % nm;
    ok = c.rho[((int64_t)z * nm + y) * nm + x] <= c.rho_max;
  }
  const int64_t lin = ((int64_t)iz * nm + iy) * nm + ix;
  cell_of[i] = ok ? (int32_t)lin : -1;
  if (!ok) return;
  atomicAdd(&counts[lin], 1u);
  const float ax = (c.lrx[i] * c.inv_g + c.srx[i]) * c.a_unit_inv;
  const float ay = (c.lry[i] * c.inv_g + c.sry[i]) * c.a_unit_inv;
  const float az = (c.lrz[i] * c.inv_g + c.srz[i]) * c.a_unit_inv;
  const float3 t = target_of(c, i);
  const float tx = t.x, ty = t.y, tz = t.z;
  atomicAdd(&sums[0], (double)(ax * ax + ay * ay + az * az));
  atomicAdd(&sums[1], (double)(tx * tx + ty * ty + tz * tz));
  atomicAdd(&sums[2], 1.0);
}

// Particles into their cells' slots: node coordinates, the weight
// 1 / (|a|^2 + a_floor^2) (a relative-error loss) and the target (units of
// a_unit).
__global__ void k_box_pass2(Capture c, const int32_t* __restrict__ cell_of, const uint32_t* __restrict__ start,
                            uint32_t* __restrict__ cursor, float a_floor2, float wnorm,
                            float4* __restrict__ pdat, float4* __restrict__ ptgt) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= c.n) return;
  const int32_t lin = cell_of[i];
  if (lin < 0) return;
  int i0;
  float s[3];
  node_coord(c.qx[i], c.scale, c.inv_cell, c.nm, &i0, &s[0]);
  node_coord(c.qy[i], c.scale, c.inv_cell, c.nm, &i0, &s[1]);
  node_coord(c.qz[i], c.scale, c.inv_cell, c.nm, &i0, &s[2]);
  const float ax = (c.lrx[i] * c.inv_g + c.srx[i]) * c.a_unit_inv;
  const float ay = (c.lry[i] * c.inv_g + c.sry[i]) * c.a_unit_inv;
  const float az = (c.lrz[i] * c.inv_g + c.srz[i]) * c.a_unit_inv;
  const float w = wnorm / (ax * ax + ay * ay + az * az + a_floor2);
  const uint32_t slot = start[lin] + atomicAdd(&cursor[lin], 1u);
  const float3 t = target_of(c, i);
  const float tx = t.x, ty = t.y, tz = t.z;
  pdat[slot] = make_float4(s[0], s[1], s[2], w);
  ptgt[slot] = make_float4(tx, ty, tz, 0.f);
}

__global__ void k_scale_targets(float4* __restrict__ t, int64_t n, float f) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  float4 v = t[i];
  t[i] = make_float4(v.x * f, v.y * f, v.z * f, 0.f);
}

// ---- batches of patches ------------------------------------------------------------
// Patch b: box and output origin from picks[b] (x = box, yzw = origin) or, with
// picks == nullptr, drawn from (seed, b).  Writes the 14^3 input volume and the
// particles of the inner 7^3 cells (local node coordinates of the 8^3 output).
__global__ void __launch_bounds__(512) k_batch(const BoxView* __restrict__ boxes, int nboxes,
                                               const int4* __restrict__ picks, uint64_t seed, int c_in, Norm nrm,
                                               __nv_bfloat16* __restrict__ x0, int32_t* __restrict__ pb,
                                               float* __restrict__ ps, float* __restrict__ tgt,
                                               float* __restrict__ w, float* __restrict__ wsum) {
  __shared__ int4 pick;
  __shared__ uint32_t cnt[512];
  __shared__ float red[16];
  const int b = blockIdx.x, tid = threadIdx.x;
  if (tid == 0) {
    if (picks) {
      pick = picks[b];
    } else {
      const uint64_t h = mix64(seed * 0x100000001B3ull + (uint64_t)b);
      const int k = (int)(h % (uint64_t)nboxes);
      const int nm = boxes[k].nm;
      const uint64_t h2 = mix64(h);
      pick = make_int4(k, (int)(h2 % nm), (int)((h2 >> 21) % nm), (int)((h2 >> 42) % nm));
    }
  }
  __syncthreads();
  const BoxView bv = boxes[pick.x];
  const int nm = bv.nm;
  // input features, periodic
  for (int i = tid; i < PATCH_IN * PATCH_IN * PATCH_IN; i += blockDim.x) {
    const int xx = i % PATCH_IN, yy = (i / PATCH_IN) % PATCH_IN, zz = i / (PATCH_IN * PATCH_IN);
    const int x = (pick.y + xx - 3 + 2 * nm) % nm, y = (pick.z + yy - 3 + 2 * nm) % nm,
              z = (pick.w + zz - 3 + 2 * nm) % nm;
    const int64_t node = ((int64_t)z * nm + y) * nm + x;
    float v[16];
#pragma unroll
    for (int c = 0; c < 16; ++c)
      v[c] = c < c_in ? (bv.feats[node * c_in + c] - nrm.shift[c]) * nrm.scale[c] : 0.f;
    store16f(x0 + ((int64_t)b * PATCH_IN * PATCH_IN * PATCH_IN + i) * 16, v);
  }
  // particle counts of the inner cells, then an exclusive scan
  uint32_t first = 0, mine = 0;
  if (tid < PATCH_CELLS * PATCH_CELLS * PATCH_CELLS) {
    const int cx = (pick.y + tid % 7) % nm, cy = (pick.z + (tid / 7) % 7) % nm, cz = (pick.w + tid / 49) % nm;
    const int64_t lin = ((int64_t)cz * nm + cy) * nm + cx;
    first = bv.start[lin];
    mine = bv.start[lin + 1] - first;
  }
  cnt[tid] = mine;
  __syncthreads();
  for (int off = 1; off < 512; off <<= 1) {
    const uint32_t add = tid >= off ? cnt[tid - off] : 0u;
    __syncthreads();
    cnt[tid] += add;
    __syncthreads();
  }
  const uint32_t total = cnt[511];
  const uint32_t base = cnt[tid] - mine;
  float wsum_t = 0.f;
  const int64_t slot0 = (int64_t)b * PCAP;
  for (uint32_t j = 0; j < mine; ++j) {
    const uint32_t slot = base + j;
    if (slot >= (uint32_t)PCAP) break;
    const float4 p = bv.pdat[first + j];
    const float4 t = bv.ptgt[first + j];
    float lx = p.x - (float)pick.y, ly = p.y - (float)pick.z, lz = p.z - (float)pick.w;
    if (lx < 0.f) lx += (float)nm;
    if (ly < 0.f) ly += (float)nm;
    if (lz < 0.f) lz += (float)nm;
    const int64_t o = slot0 + slot;
    pb[o] = b;
    ps[3 * o] = lx;
    ps[3 * o + 1] = ly;
    ps[3 * o + 2] = lz;
    tgt[3 * o] = t.x;
    tgt[3 * o + 1] = t.y;
    tgt[3 * o + 2] = t.z;
    w[o] = p.w;
    wsum_t += p.w;
  }
  for (uint32_t s = min(total, (uint32_t)PCAP) + tid; s < (uint32_t)PCAP; s += blockDim.x) {
    w[slot0 + s] = 0.f;
    pb[slot0 + s] = b;
    ps[3 * (slot0 + s)] = ps[3 * (slot0 + s) + 1] = ps[3 * (slot0 + s) + 2] = 0.f;
  }
  for (int o = 16; o > 0; o >>= 1) wsum_t += __shfl_down_sync(0xffffffffu, wsum_t, o);
  if ((tid & 31) == 0) red[tid >> 5] = wsum_t;
  __syncthreads();
  if (tid == 0) {
    float s = 0.f;
    for (int k = 0; k < 16; ++k) s += red[k];
    atomicAdd(wsum, s);
  }
}

// ---- host side -----------------------------------------------------------------
template <class T>
T* ws_alloc(tpm_cnn* c, size_t count) {
  void* p = nullptr;
  TPM_CUDA(cudaMalloc(&p, std::max<size_t>(count * sizeof(T), 16)));
  c->ws_allocs.push_back(p);
  return (T*)p;
}

void ensure_workspace(tpm_cnn* c, int B, int D, int64_t nparticles) {
  if (B <= c->ws_b && D == c->ws_d && nparticles <= c->ws_p) return;
  for (void* p : c->ws_allocs) cudaFree(p);
  c->ws_allocs.clear();
  B = std::max(B, c->ws_b);
  nparticles = std::max<int64_t>(nparticles, c->ws_p);
  const int64_t n0 = (int64_t)B * D * D * D, n1 = (int64_t)B * (D - 2) * (D - 2) * (D - 2);
  const int64_t n2 = (int64_t)B * (D - 4) * (D - 4) * (D - 4), n3 = (int64_t)B * (D - 6) * (D - 6) * (D - 6);
  c->x0f = ws_alloc<float>(c, n0 * c->c_in);
  c->x0 = ws_alloc<__nv_bfloat16>(c, n0 * 16);
  c->z1 = ws_alloc<__nv_bfloat16>(c, n1 * 16);
  c->a1 = ws_alloc<__nv_bfloat16>(c, n1 * 16);
  c->dz1 = ws_alloc<__nv_bfloat16>(c, n1 * 16);
  c->z2 = ws_alloc<__nv_bfloat16>(c, n2 * 16);
  c->a2 = ws_alloc<__nv_bfloat16>(c, n2 * 16);
  c->dz2 = ws_alloc<__nv_bfloat16>(c, n2 * 16);
  c->z3 = ws_alloc<__nv_bfloat16>(c, n3 * 16);
  c->a3 = ws_alloc<__nv_bfloat16>(c, n3 * 16);
  c->dz3 = ws_alloc<__nv_bfloat16>(c, n3 * 16);
  c->dout = ws_alloc<float>(c, n3 * 3);
  c->pb = ws_alloc<int32_t>(c, nparticles);
  c->ps = ws_alloc<float>(c, nparticles * 3);
  c->tgt = ws_alloc<float>(c, nparticles * 3);
  c->w = ws_alloc<float>(c, nparticles);
  c->ws_b = B;
  c->ws_d = D;
  c->ws_p = nparticles;
}

cn::Vol vol(int B, int D) { return cn::Vol{B, D, D, D}; }

void forward_pass(tpm_cnn* c, int B, int D, bool keep_z) {
  cudaStream_t s = c->stream;
  cn::conv_forward(c->x0, vol(B, D), c->a1, keep_z ? c->z1 : nullptr, c->P.fwd[0], c->params + c->L.b[0],
                   c->err_dev, s);
  cn::conv_forward(c->a1, vol(B, D - 2), c->a2, keep_z ? c->z2 : nullptr, c->P.fwd[1], c->params + c->L.b[1],
                   c->err_dev, s);
  cn::conv_forward(c->a2, vol(B, D - 4), c->a3, keep_z ? c->z3 : nullptr, c->P.fwd[2], c->params + c->L.b[2],
                   c->err_dev, s);
}

// Loss of the particles in the workspace (n slots) into *loss_dev and the
// parameter gradient into c->grad.
void backward_pass(tpm_cnn* c, int B, int D, int64_t n, const float* wsum_dev, float* loss_dev) {
  cudaStream_t s = c->stream;
  const cn::Vol v3 = vol(B, D - 6);
  TPM_CUDA(cudaMemsetAsync(c->grad, 0, sizeof(float) * c->L.total, s));
  TPM_CUDA(cudaMemsetAsync(c->dout, 0, sizeof(float) * 3 * v3.nodes(), s));
  cn::head_loss(c->a3, v3, c->params, c->L, n, c->pb, c->ps, c->tgt, c->w, wsum_dev, c->dout, loss_dev, s);
  cn::head_backward(c->a3, c->z3, c->dout, v3.nodes(), c->params, c->L, c->dz3, c->grad, s);
  cn::conv_backward_weights(c->a2, vol(B, D - 4), c->dz3, cn::CH, c->grad + c->L.w[2], c->grad + c->L.b[2], s);
  cn::conv_backward_data(c->dz3, v3, c->dz2, c->z2, c->P.bwd[2], c->err_dev, s);
  cn::conv_backward_weights(c->a1, vol(B, D - 2), c->dz2, cn::CH, c->grad + c->L.w[1], c->grad + c->L.b[1], s);
  cn::conv_backward_data(c->dz2, vol(B, D - 4), c->dz1, c->z1, c->P.bwd[1], c->err_dev, s);
  cn::conv_backward_weights(c->x0, vol(B, D), c->dz1, c->c_in, c->grad + c->L.w[0], c->grad + c->L.b[0], s);
}

void check_err(tpm_cnn* c) {
  uint32_t e = 0;
  TPM_CUDA(cudaMemcpyAsync(&e, c->err_dev, sizeof(e), cudaMemcpyDeviceToHost, c->stream));
  TPM_CUDA(cudaStreamSynchronize(c->stream));
  if (e & tpm::DEV_ERR_MMA_TIMEOUT) throw Error(TPM_ERR_CUDA, "tensor-core wait timed out");
}

int cnn_fail(tpm_cnn* c, const Error& e) {
  if (c) c->err = e.what();
  return e.code ? e.code : TPM_ERR_CUDA;
}

std::vector<BoxView> box_views(const tpm_cnn* c, bool held_out) {
  std::vector<BoxView> v;
  for (const auto& b : c->boxes)
    if (b.held_out == held_out) v.push_back(BoxView{b.nm, b.feats, b.start, b.pdat, b.ptgt});
  return v;
}

Norm norm_of(const tpm_cnn* c) {
  Norm n{};
  for (int k = 0; k < cn::MAX_CIN; ++k) {
    n.shift[k] = c->shift[k];
    n.scale[k] = c->scale[k];
  }
  return n;
}

}  // namespace

namespace tpm {
namespace cnn {

void add_box(tpm_cnn* c, const BoxSource& b, bool held_out) {
  cudaStream_t s = c->stream;
  const int nm = b.nm;
  const int64_t nm3 = (int64_t)nm * nm * nm;
  const double cell = b.box / nm;
  const double m_cell = b.m_total / (double)nm3;
  const double a_unit = m_cell / (cell * cell);  // acceleration of one cell's mean mass at one cell, per unit G
  tpm_cnn::Box bx;
  bx.nm = nm;
  bx.held_out = held_out;
  auto balloc = [&](size_t bytes) {
    void* p = nullptr;
    TPM_CUDA(cudaMalloc(&p, std::max<size_t>(bytes, 16)));
    c->box_allocs.push_back(p);
    return p;
  };
  bx.feats = (float*)balloc(sizeof(float) * nm3 * c->c_in);
  float* oct = nullptr;
  TPM_CUDA(cudaMalloc(&oct, sizeof(float) * 8 * nm3));
  octant_deposit(b.qx, b.qy, b.qz, b.massf, b.n, nm, b.box, oct, s);
  k_box_feats<<<grid_for(nm3, 256, 1ll << 30), 256, 0, s>>>(b.rho, b.phi, oct, nm3, (float)(1.0 / m_cell),
                                                            (float)(cell / m_cell), c->c_in, bx.feats);
  TPM_LAUNCH_CHECK();
  TPM_CUDA(cudaStreamSynchronize(s));
  cudaFree(oct);
  // normalisation from the first box
  if (!c->scales_set) {
    std::vector<float> h((size_t)nm3 * c->c_in);
    TPM_CUDA(cudaMemcpyAsync(h.data(), bx.feats, sizeof(float) * h.size(), cudaMemcpyDeviceToHost, s));
    TPM_CUDA(cudaStreamSynchronize(s));
    for (int k = 0; k < c->c_in; ++k) {
      double s1 = 0, s2 = 0;
      for (int64_t i = 0; i < nm3; ++i) {
        const double v = h[(size_t)i * c->c_in + k];
        s1 += v;
        s2 += v * v;
      }
      const double mean = s1 / nm3, var = std::max(s2 / nm3 - mean * mean, 1e-12);
      c->shift[k] = (float)mean;
      c->scale[k] = (float)(1.0 / std::sqrt(var));
    }
  }
  Capture cap{};
  cap.n = b.n;
  cap.qx = b.qx;
  cap.qy = b.qy;
  cap.qz = b.qz;
  cap.scale = b.box / TWO32;
  cap.inv_cell = nm / b.box;
  cap.nm = nm;
  cap.rho = b.rho;
  cap.rho_max = (float)((1.0 + c->delta_max) * m_cell);
  cap.srx = b.srx;
  cap.sry = b.sry;
  cap.srz = b.srz;
  cap.lrx = b.lrx;
  cap.lry = b.lry;
  cap.lrz = b.lrz;
  cap.nrx = b.nrx;
  cap.nry = b.nry;
  cap.nrz = b.nrz;
  cap.inv_g = (float)(1.0 / b.g);
  cap.a_unit_inv = (float)(1.0 / a_unit);
  int32_t* cell_of = (int32_t*)balloc(sizeof(int32_t) * std::max<int64_t>(b.n, 1));
  uint32_t* counts = (uint32_t*)balloc(sizeof(uint32_t) * (nm3 + 1));
  bx.start = (uint32_t*)balloc(sizeof(uint32_t) * (nm3 + 1));
  double* sums = (double*)balloc(sizeof(double) * 4);
  void* scratch = balloc(scan_scratch_bytes(nm3 + 1));
  TPM_CUDA(cudaMemsetAsync(counts, 0, sizeof(uint32_t) * (nm3 + 1), s));
  TPM_CUDA(cudaMemsetAsync(sums, 0, sizeof(double) * 4, s));
  k_box_pass1<<<grid_for(b.n, 256, 1ll << 30), 256, 0, s>>>(cap, cell_of, counts, sums);
  TPM_LAUNCH_CHECK();
  exclusive_scan_u32(counts, bx.start, nm3 + 1, nullptr, scratch, s);
  double hs[4];
  TPM_CUDA(cudaMemcpyAsync(hs, sums, sizeof(hs), cudaMemcpyDeviceToHost, s));
  TPM_CUDA(cudaStreamSynchronize(s));
  const double kept = hs[2];
  if (kept < 1) throw Error(TPM_ERR_INVALID_ARGUMENT, "no particle of the box lies in cells below delta_max");
  const double mean_a2 = hs[0] / kept;
  bx.n = (int64_t)kept;
  bx.pdat = (float4*)balloc(sizeof(float4) * bx.n);
  bx.ptgt = (float4*)balloc(sizeof(float4) * bx.n);
  TPM_CUDA(cudaMemsetAsync(counts, 0, sizeof(uint32_t) * (nm3 + 1), s));
  k_box_pass2<<<grid_for(b.n, 256, 1ll << 30), 256, 0, s>>>(cap, cell_of, bx.start, counts,
                                                            (float)(0.01 * mean_a2), (float)mean_a2, bx.pdat,
                                                            bx.ptgt);
  TPM_LAUNCH_CHECK();
  TPM_CUDA(cudaStreamSynchronize(s));
  // output unit from the first box: the loss-weighted rms of the targets with
  // the largest 1 % left out (particles whose short and long range nearly
  // cancel would dominate it), so that predicting zero costs a loss near 1
  if (!c->scales_set) {
    std::vector<float4> hp((size_t)bx.n), ht((size_t)bx.n);
    TPM_CUDA(cudaMemcpy(hp.data(), bx.pdat, sizeof(float4) * bx.n, cudaMemcpyDeviceToHost));
    TPM_CUDA(cudaMemcpy(ht.data(), bx.ptgt, sizeof(float4) * bx.n, cudaMemcpyDeviceToHost));
    std::vector<float> t2((size_t)bx.n);
    for (int64_t i = 0; i < bx.n; ++i) t2[i] = ht[i].x * ht[i].x + ht[i].y * ht[i].y + ht[i].z * ht[i].z;
    std::vector<float> sorted = t2;
    const size_t k99 = (size_t)(0.99 * (double)(sorted.size() - 1));
    std::nth_element(sorted.begin(), sorted.begin() + k99, sorted.end());
    const float cut = sorted[k99];
    double sw = 0.0, swt = 0.0;
    for (int64_t i = 0; i < bx.n; ++i)
      if (t2[i] <= cut) {
        sw += hp[i].w;
        swt += (double)hp[i].w * t2[i];
      }
    c->out_scale = (float)std::sqrt(std::max(swt / std::max(sw, 1e-300), 1e-30));
    c->scales_set = true;
  }
  k_scale_targets<<<grid_for(bx.n, 256, 1ll << 30), 256, 0, s>>>(bx.ptgt, bx.n, 1.f / c->out_scale);
  TPM_LAUNCH_CHECK();
  TPM_CUDA(cudaStreamSynchronize(s));
  c->boxes.push_back(bx);
}

}  // namespace cnn
}  // namespace tpm

extern "C" {

int64_t tpm_cnn_param_count(int32_t c_in) {
  if (c_in < 1 || c_in > cn::MAX_CIN) return -TPM_ERR_INVALID_ARGUMENT;
  return cn::layout(c_in).total;
}

int tpm_cnn_create(int32_t c_in, int32_t device, tpm_cnn** out) {
  if (!out) return TPM_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  if (c_in < 1 || c_in > cn::MAX_CIN) return TPM_ERR_INVALID_ARGUMENT;
  tpm_cnn* c = new (std::nothrow) tpm_cnn();
  if (!c) return TPM_ERR_OUT_OF_MEMORY;
  try {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
      cudaGetLastError();
      throw Error(TPM_ERR_NO_DEVICE, "no CUDA device");
    }
    if (device < 0 || device >= ndev) throw Error(TPM_ERR_INVALID_ARGUMENT, "device ordinal out of range");
    cudaDeviceProp prop;
    TPM_CUDA(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10) throw Error(TPM_ERR_NO_DEVICE, std::string("device is not sm_100: ") + prop.name);
    TPM_CUDA(cudaSetDevice(device));
    c->device = device;
    c->c_in = c_in;
    c->L = cn::layout(c_in);
    TPM_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
    const size_t pb = sizeof(float) * c->L.total;
    TPM_CUDA(cudaMalloc(&c->params, pb));
    TPM_CUDA(cudaMalloc(&c->m, pb));
    TPM_CUDA(cudaMalloc(&c->v, pb));
    TPM_CUDA(cudaMalloc(&c->grad, pb));
    TPM_CUDA(cudaMalloc(&c->pack, sizeof(uint4) * cn::WPACK_U4 * 5));
    TPM_CUDA(cudaMalloc(&c->scal, sizeof(float) * 4));
    TPM_CUDA(cudaMalloc(&c->err_dev, sizeof(uint32_t)));
    TPM_CUDA(cudaMemset(c->params, 0, pb));
    TPM_CUDA(cudaMemset(c->m, 0, pb));
    TPM_CUDA(cudaMemset(c->v, 0, pb));
    TPM_CUDA(cudaMemset(c->err_dev, 0, sizeof(uint32_t)));
    for (int l = 0; l < 3; ++l) c->P.fwd[l] = c->pack + (size_t)l * cn::WPACK_U4;
    c->P.bwd[0] = nullptr;
    c->P.bwd[1] = c->pack + (size_t)3 * cn::WPACK_U4;
    c->P.bwd[2] = c->pack + (size_t)4 * cn::WPACK_U4;
    for (int k = 0; k < cn::MAX_CIN; ++k) c->scale[k] = 1.f;
    cn::pack_weights(c->params, c->L, c->P, c->stream);
    TPM_CUDA(cudaStreamSynchronize(c->stream));
  } catch (const Error& e) {
    const int rc = e.code ? e.code : TPM_ERR_CUDA;
    tpm_cnn_destroy(c);
    return rc;
  }
  *out = c;
  return TPM_OK;
}

int tpm_cnn_destroy(tpm_cnn* c) {
  if (!c) return TPM_OK;
  cudaSetDevice(c->device);
  if (c->stream) cudaStreamSynchronize(c->stream);
  for (void* p : c->ws_allocs) cudaFree(p);
  for (void* p : c->box_allocs) cudaFree(p);
  cudaFree(c->params);
  cudaFree(c->m);
  cudaFree(c->v);
  cudaFree(c->grad);
  cudaFree(c->pack);
  cudaFree(c->scal);
  cudaFree(c->err_dev);
  cudaFree(c->loss_hist);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return TPM_OK;
}

const char* tpm_cnn_last_error(const tpm_cnn* c) { return c ? c->err.c_str() : "null network"; }

int tpm_cnn_set_params(tpm_cnn* c, const float* params, int64_t n) {
  if (!c || !params || n != c->L.total) return TPM_ERR_INVALID_ARGUMENT;
  try {
    TPM_CUDA(cudaSetDevice(c->device));
    TPM_CUDA(cudaMemcpyAsync(c->params, params, sizeof(float) * n, cudaMemcpyHostToDevice, c->stream));
    TPM_CUDA(cudaMemsetAsync(c->m, 0, sizeof(float) * n, c->stream));
    TPM_CUDA(cudaMemsetAsync(c->v, 0, sizeof(float) * n, c->stream));
    c->step = 0;
    cn::pack_weights(c->params, c->L, c->P, c->stream);
    TPM_CUDA(cudaStreamSynchronize(c->stream));
  } catch (const Error& e) {
    return cnn_fail(c, e);
  }
  return TPM_OK;
}

int tpm_cnn_get_params(tpm_cnn* c, float* params, int64_t n) {
  if (!c || !params || n != c->L.total) return TPM_ERR_INVALID_ARGUMENT;
  try {
    TPM_CUDA(cudaSetDevice(c->device));
    TPM_CUDA(cudaMemcpyAsync(params, c->params, sizeof(float) * n, cudaMemcpyDeviceToHost, c->stream));
    TPM_CUDA(cudaStreamSynchronize(c->stream));
  } catch (const Error& e) {
    return cnn_fail(c, e);
  }
  return TPM_OK;
}

int tpm_cnn_set_scales(tpm_cnn* c, const float* shift, const float* scale, float out_scale, float delta_max) {
  if (!c || !shift || !scale || !(out_scale > 0.f) || !(delta_max > 0.f)) return TPM_ERR_INVALID_ARGUMENT;
  for (int k = 0; k < c->c_in; ++k) {
    c->shift[k] = shift[k];
    c->scale[k] = scale[k];
  }
  c->out_scale = out_scale;
  c->delta_max = delta_max;
  c->scales_set = true;
  return TPM_OK;
}

int tpm_cnn_set_near(tpm_cnn* c, float near_cells) {
  if (!c || !(near_cells >= 0.f && near_cells <= 1.f)) return TPM_ERR_INVALID_ARGUMENT;
  if (!c->boxes.empty()) {
    c->err = "the near-field radius defines the captured targets: set it before tpm_cnn_add_box";
    return TPM_ERR_INVALID_ARGUMENT;
  }
  c->near_cells = near_cells;
  return TPM_OK;
}

float tpm_cnn_get_near(const tpm_cnn* c) { return c ? c->near_cells : -1.f; }

int tpm_cnn_get_scales(const tpm_cnn* c, float* shift, float* scale, float* out_scale, float* delta_max) {
  if (!c || !shift || !scale || !out_scale || !delta_max) return TPM_ERR_INVALID_ARGUMENT;
  for (int k = 0; k < c->c_in; ++k) {
    shift[k] = c->shift[k];
    scale[k] = c->scale[k];
  }
  *out_scale = c->out_scale;
  *delta_max = c->delta_max;
  return TPM_OK;
}

int tpm_cnn_forward(tpm_cnn* c, const float* x0, int32_t batch, int32_t d, float* out) {
  if (!c || !x0 || !out || batch < 1 || d < 7) return TPM_ERR_INVALID_ARGUMENT;
  try {
    TPM_CUDA(cudaSetDevice(c->device));
    ensure_workspace(c, batch, d, 1);
    const int64_t n0 = (int64_t)batch * d * d * d, n3 = (int64_t)batch * (d - 6) * (d - 6) * (d - 6);
    TPM_CUDA(cudaMemcpyAsync(c->x0f, x0, sizeof(float) * n0 * c->c_in, cudaMemcpyHostToDevice, c->stream));
    k_x0_from_f32<<<tpm::grid_for(n0, 256, 1ll << 30), 256, 0, c->stream>>>(c->x0f, n0, c->c_in, c->x0);
    TPM_LAUNCH_CHECK();
    forward_pass(c, batch, d, false);
    float* field = c->dout;
    cn::head_field(c->a3, n3, c->params, c->L, field, c->stream);
    TPM_CUDA(cudaMemcpyAsync(out, field, sizeof(float) * 3 * n3, cudaMemcpyDeviceToHost, c->stream));
    check_err(c);
  } catch (const Error& e) {
    return cnn_fail(c, e);
  }
  return TPM_OK;
}

int tpm_cnn_loss_grad(tpm_cnn* c, const float* x0, int32_t batch, int32_t d, int64_t n, const int32_t* pb,
                      const float* ps, const float* target, const float* weight, float* loss, float* grad) {
  if (!c || !x0 || batch < 1 || d < 7 || n < 1 || !pb || !ps || !target || !weight || !loss || !grad)
    return TPM_ERR_INVALID_ARGUMENT;
  const int dout = d - 6;
  double wsum = 0.0;
  for (int64_t i = 0; i < n; ++i) {
    if (pb[i] < 0 || pb[i] >= batch || !(weight[i] >= 0.f)) return TPM_ERR_INVALID_ARGUMENT;
    for (int k = 0; k < 3; ++k)
      if (!(ps[3 * i + k] >= 0.f && ps[3 * i + k] <= (float)(dout - 1))) return TPM_ERR_INVALID_ARGUMENT;
    wsum += weight[i];
  }
  if (!(wsum > 0.0)) return TPM_ERR_INVALID_ARGUMENT;
  try {
    TPM_CUDA(cudaSetDevice(c->device));
    ensure_workspace(c, batch, d, n);
    cudaStream_t s = c->stream;
    const int64_t n0 = (int64_t)batch * d * d * d;
    TPM_CUDA(cudaMemcpyAsync(c->x0f, x0, sizeof(float) * n0 * c->c_in, cudaMemcpyHostToDevice, s));
    TPM_CUDA(cudaMemcpyAsync(c->pb, pb, sizeof(int32_t) * n, cudaMemcpyHostToDevice, s));
    TPM_CUDA(cudaMemcpyAsync(c->ps, ps, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, s));
    TPM_CUDA(cudaMemcpyAsync(c->tgt, target, sizeof(float) * 3 * n, cudaMemcpyHostToDevice, s));
    TPM_CUDA(cudaMemcpyAsync(c->w, weight, sizeof(float) * n, cudaMemcpyHostToDevice, s));
    const float hs[2] = {(float)wsum, 0.f};
    TPM_CUDA(cudaMemcpyAsync(c->scal, hs, sizeof(hs), cudaMemcpyHostToDevice, s));
    k_x0_from_f32<<<tpm::grid_for(n0, 256, 1ll << 30), 256, 0, s>>>(c->x0f, n0, c->c_in, c->x0);
    TPM_LAUNCH_CHECK();
    forward_pass(c, batch, d, true);
    backward_pass(c, batch, d, n, c->scal, c->scal + 1);
    TPM_CUDA(cudaMemcpyAsync(loss, c->scal + 1, sizeof(float), cudaMemcpyDeviceToHost, s));
    TPM_CUDA(cudaMemcpyAsync(grad, c->grad, sizeof(float) * c->L.total, cudaMemcpyDeviceToHost, s));
    check_err(c);
  } catch (const Error& e) {
    return cnn_fail(c, e);
  }
  return TPM_OK;
}

int tpm_cnn_adam_step(tpm_cnn* c, const float* grad, float lr, float beta1, float beta2, float eps) {
  if (!c || !(lr > 0.f) || !(beta1 >= 0.f && beta1 < 1.f) || !(beta2 >= 0.f && beta2 < 1.f) || !(eps > 0.f))
    return TPM_ERR_INVALID_ARGUMENT;
  try {
    TPM_CUDA(cudaSetDevice(c->device));
    if (grad)
      TPM_CUDA(cudaMemcpyAsync(c->grad, grad, sizeof(float) * c->L.total, cudaMemcpyHostToDevice, c->stream));
    ++c->step;
    cn::adam(c->params, c->m, c->v, c->grad, c->L.total, lr, beta1, beta2, eps, c->step, c->stream);
    cn::pack_weights(c->params, c->L, c->P, c->stream);
    TPM_CUDA(cudaStreamSynchronize(c->stream));
  } catch (const Error& e) {
    return cnn_fail(c, e);
  }
  return TPM_OK;
}

int tpm_cnn_box_count(const tpm_cnn* c, int32_t held_out) {
  if (!c) return -TPM_ERR_INVALID_ARGUMENT;
  int k = 0;
  for (const auto& b : c->boxes) k += (b.held_out == (held_out != 0)) ? 1 : 0;
  return k;
}

int tpm_cnn_train(tpm_cnn* c, int32_t steps, int32_t batch, float lr, uint64_t seed, float* loss_history) {
  if (!c || steps < 1 || batch < 1 || batch > 1024 || !(lr > 0.f)) return TPM_ERR_INVALID_ARGUMENT;
  try {
    TPM_CUDA(cudaSetDevice(c->device));
    const std::vector<BoxView> views = box_views(c, false);
    if (views.empty()) throw Error(TPM_ERR_NOT_READY, "no training box captured");
    cudaStream_t s = c->stream;
    ensure_workspace(c, batch, PATCH_IN, (int64_t)batch * PCAP);
    if (c->loss_cap < steps) {
      cudaFree(c->loss_hist);
      c->loss_hist = nullptr;
      TPM_CUDA(cudaMalloc(&c->loss_hist, sizeof(float) * steps));
      c->loss_cap = steps;
    }
    BoxView* dv = nullptr;
    TPM_CUDA(cudaMalloc(&dv, sizeof(BoxView) * views.size()));
    TPM_CUDA(cudaMemcpyAsync(dv, views.data(), sizeof(BoxView) * views.size(), cudaMemcpyHostToDevice, s));
    TPM_CUDA(cudaMemsetAsync(c->loss_hist, 0, sizeof(float) * steps, s));
    const Norm nrm = norm_of(c);
    const int64_t np = (int64_t)batch * PCAP;
    for (int32_t it = 0; it < steps; ++it) {
      TPM_CUDA(cudaMemsetAsync(c->scal, 0, sizeof(float), s));
      k_batch<<<batch, 512, 0, s>>>(dv, (int)views.size(), nullptr, seed + (uint64_t)c->step + 1, c->c_in, nrm, c->x0,
                                    c->pb, c->ps, c->tgt, c->w, c->scal);
      TPM_LAUNCH_CHECK();
      forward_pass(c, batch, PATCH_IN, true);
      backward_pass(c, batch, PATCH_IN, np, c->scal, c->loss_hist + it);
      ++c->step;
      cn::adam(c->params, c->m, c->v, c->grad, c->L.total, lr, 0.9f, 0.999f, 1e-8f, c->step, s);
      cn::pack_weights(c->params, c->L, c->P, s);
    }
    if (loss_history)
      TPM_CUDA(cudaMemcpyAsync(loss_history, c->loss_hist, sizeof(float) * steps, cudaMemcpyDeviceToHost, s));
    check_err(c);
    cudaFree(dv);
  } catch (const Error& e) {
    return cnn_fail(c, e);
  }
  return TPM_OK;
}

// Weighted loss over every patch of a tiling (stride 7) of the held-out (or
// training) boxes.
int tpm_cnn_evaluate(tpm_cnn* c, int32_t held_out, int32_t batch, float* loss) {
  if (!c || !loss || batch < 1 || batch > 1024) return TPM_ERR_INVALID_ARGUMENT;
  try {
    TPM_CUDA(cudaSetDevice(c->device));
    std::vector<BoxView> views;
    std::vector<int4> picks;
    int k = 0;
    for (const auto& b : c->boxes) {
      if (b.held_out != (held_out != 0)) continue;
      views.push_back(BoxView{b.nm, b.feats, b.start, b.pdat, b.ptgt});
      const int nt = (b.nm + PATCH_CELLS - 1) / PATCH_CELLS;
      for (int z = 0; z < nt; ++z)
        for (int y = 0; y < nt; ++y)
          for (int x = 0; x < nt; ++x)
            picks.push_back(make_int4(k, (x * PATCH_CELLS) % b.nm, (y * PATCH_CELLS) % b.nm, (z * PATCH_CELLS) % b.nm));
      ++k;
    }
    if (views.empty()) throw Error(TPM_ERR_NOT_READY, "no box of that kind captured");
    cudaStream_t s = c->stream;
    ensure_workspace(c, batch, PATCH_IN, (int64_t)batch * PCAP);
    BoxView* dv = nullptr;
    int4* dp = nullptr;
    float* acc = nullptr;  // [0] sum w, [1] sum w err^2, [2] unit weight sum
    TPM_CUDA(cudaMalloc(&dv, sizeof(BoxView) * views.size()));
    TPM_CUDA(cudaMalloc(&dp, sizeof(int4) * picks.size()));
    TPM_CUDA(cudaMalloc(&acc, sizeof(float) * 4));
    TPM_CUDA(cudaMemcpyAsync(dv, views.data(), sizeof(BoxView) * views.size(), cudaMemcpyHostToDevice, s));
    TPM_CUDA(cudaMemcpyAsync(dp, picks.data(), sizeof(int4) * picks.size(), cudaMemcpyHostToDevice, s));
    const float init[4] = {0.f, 0.f, 1.f, 0.f};
    TPM_CUDA(cudaMemcpyAsync(acc, init, sizeof(init), cudaMemcpyHostToDevice, s));
    const Norm nrm = norm_of(c);
    for (size_t p0 = 0; p0 < picks.size(); p0 += batch) {
      const int B = (int)std::min<size_t>(batch, picks.size() - p0);
      k_batch<<<B, 512, 0, s>>>(dv, (int)views.size(), dp + p0, 0, c->c_in, nrm, c->x0, c->pb, c->ps, c->tgt, c->w,
                                acc);
      TPM_LAUNCH_CHECK();
      forward_pass(c, B, PATCH_IN, true);
      TPM_CUDA(cudaMemsetAsync(c->dout, 0, sizeof(float) * 3 * (int64_t)B * 512, s));
      cn::head_loss(c->a3, vol(B, PATCH_OUT), c->params, c->L, (int64_t)B * PCAP, c->pb, c->ps, c->tgt, c->w, acc + 2,
                    c->dout, acc + 1, s);
    }
    float h[2];
    TPM_CUDA(cudaMemcpyAsync(h, acc, sizeof(h), cudaMemcpyDeviceToHost, s));
    check_err(c);
    cudaFree(dv);
    cudaFree(dp);
    cudaFree(acc);
    *loss = h[0] > 0.f ? h[1] / h[0] : 0.f;
  } catch (const Error& e) {
    return cnn_fail(c, e);
  }
  return TPM_OK;
}

int tpm_selftest_bounded_wait(int32_t device, double* waited_seconds) {
  try {
    TPM_CUDA(cudaSetDevice(device));
    cudaStream_t s;
    TPM_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    double t = 0.0;
    try {
      t = cn::conv_wait_selftest(s);
    } catch (...) {
      cudaStreamDestroy(s);
      throw;
    }
    cudaStreamDestroy(s);
    if (waited_seconds) *waited_seconds = t;
  } catch (const Error& e) {
    return e.code;
  }
  return TPM_OK;
}

}  // extern "C"
