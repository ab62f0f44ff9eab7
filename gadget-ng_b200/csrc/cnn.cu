// Learned short-range network: kernels.
//
// Convolutions are implicit GEMMs on the tcgen05 tensor cores.  One CTA
// computes an output tile of 8 (x) x 16 (y) x 4 (z) nodes: for each z slice
// the 128 nodes are the M = 128 rows of a tcgen05.mma (kind::f16, BF16 in,
// FP32 accumulate in tensor memory), N = 16 output channels, K = 16 input
// channels per tap; the 27 taps accumulate into the same TMEM columns.  The
// input tile with its one-node halo sits in shared memory as two planes of
// 8 channels ([channel group][z][y][x], 16 bytes a node), which is the
// canonical no-swizzle K-major operand layout: 8 consecutive x nodes form one
// 8 x 16-byte core matrix, the next y row is the next core matrix along M
// (SBO = 10 nodes x 16 bytes) and the second channel group is the next core
// matrix along K (LBO = one plane).  A tap is a shift of the descriptor's
// start address, so no im2col copy is made.  Weights of all 27 taps
// (13.5 KB) are staged once per CTA.  One thread issues the 108 MMAs, one
// tcgen05.commit signals an mbarrier, and the four warps read their 32 TMEM
// lanes back with tcgen05.ld for the epilogue (bias + GELU forward, or the
// GELU derivative backward).  Waits on the mbarrier are bounded in time and
// report DEV_ERR_MMA_TIMEOUT instead of hanging.
//
// Weight gradients reduce over all nodes of a batch into 27 x 16 x 16 sums;
// they are small, irregular contractions and run on the CUDA cores in FP32.
#include <cuda_bf16.h>

#include <cmath>

#include "cnn.cuh"
#include "common.cuh"

namespace tpm {
namespace cnn {

Layout layout(int c_in) {
  Layout L{};
  L.c_in = c_in;
  int64_t o = 0;
  const int cin[3] = {c_in, CH, CH};
  for (int l = 0; l < 3; ++l) {
    L.w[l] = o;
    o += 27 * CH * cin[l];
    L.b[l] = o;
    o += CH;
  }
  L.wh = o;
  o += NOUT * CH;
  L.bh = o;
  o += NOUT;
  L.total = o;
  return L;
}

namespace {

constexpr int TX = 8, TY = 16, TZ = 4;
constexpr int HX = TX + 2, HY = TY + 2, HZ = TZ + 2;
constexpr int HALO = HX * HY * HZ;        // input nodes of one tile
constexpr int SIN_BYTES = 2 * HALO * 16;  // two planes of 8 channels
constexpr int SW_BYTES = WPACK_U4 * 16;
constexpr int CONV_SMEM = SIN_BYTES + SW_BYTES + 16;
constexpr uint32_t TMEM_COLS = 64;  // TZ accumulators of 16 FP32 columns (a power of two >= 32)
constexpr int CONV_THREADS = 128;

// Instruction descriptor of tcgen05.mma kind::f16: D FP32 (bits 4-5 = 1), A and
// B BF16 (bits 7-9 and 10-12 = 1), both K-major, N >> 3 at bit 17, M >> 4 at bit 24.
constexpr uint32_t IDESC = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(CH >> 3) << 17) | ((128u >> 4) << 24);

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor, no swizzle: start address, leading byte
// offset (next core matrix along K), stride byte offset (next 8-row group
// along M or N), each in 16-byte units; descriptor version 1 at bit 46.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((addr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__device__ __forceinline__ void umma_bf16(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(IDESC), "r"(acc));
}

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Wait for phase `parity` of an mbarrier; false after 2 s.
__device__ __forceinline__ bool mbar_wait(uint32_t addr, uint32_t parity) {
  const uint64_t t0 = global_ns();
  for (;;) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(addr), "r"(parity)
        : "memory");
    if (done) return true;
    if (global_ns() - t0 > 2000000000ull) return false;
  }
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

__device__ __forceinline__ float gelu_f(float z) { return 0.5f * z * (1.f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad_f(float z) {
  return 0.5f * (1.f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * expf(-0.5f * z * z);
}

__device__ __forceinline__ void store16(uint4* dst, const float* v) {
  uint32_t w[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    __nv_bfloat162 h = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
    w[i] = *reinterpret_cast<uint32_t*>(&h);
  }
  dst[0] = make_uint4(w[0], w[1], w[2], w[3]);
  dst[1] = make_uint4(w[4], w[5], w[6], w[7]);
}

__device__ __forceinline__ void load16(const uint4* src, float* v) {
  const uint4 a = src[0], b = src[1];
  const uint32_t w[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    __nv_bfloat162 h = *reinterpret_cast<const __nv_bfloat162*>(&w[i]);
    const float2 f = __bfloat1622float2(h);
    v[2 * i] = f.x;
    v[2 * i + 1] = f.y;
  }
}

// ---- convolution on the tensor cores -----------------------------------------
template <bool BWD>
__global__ void __launch_bounds__(CONV_THREADS) k_conv_tc(const __nv_bfloat16* __restrict__ in, Vol vin, int pad,
                                                          __nv_bfloat16* __restrict__ out, int oz, int oy, int ox,
                                                          __nv_bfloat16* __restrict__ zout,
                                                          const __nv_bfloat16* __restrict__ zprev,
                                                          const uint4* __restrict__ wpack,
                                                          const float* __restrict__ bias, uint32_t* err, int issue) {
  extern __shared__ __align__(128) unsigned char smem[];
  uint4* s_in = reinterpret_cast<uint4*>(smem);
  uint4* s_w = reinterpret_cast<uint4*>(smem + SIN_BYTES);
  uint64_t* mbar = reinterpret_cast<uint64_t*>(smem + SIN_BYTES + SW_BYTES);
  uint32_t* s_tmem = reinterpret_cast<uint32_t*>(smem + SIN_BYTES + SW_BYTES + 8);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int ntx = (ox + TX - 1) / TX;
  const int x0 = (int)(blockIdx.x % ntx) * TX, y0 = (int)(blockIdx.x / ntx) * TY, z0 = (int)blockIdx.y * TZ;
  const int b = blockIdx.z;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(s_tmem)),
                 "r"(TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(mbar)));
    asm volatile("fence.mbarrier_init.release.cluster;");
  }
  for (int i = tid; i < WPACK_U4; i += CONV_THREADS) s_w[i] = wpack[i];
  for (int i = tid; i < HALO; i += CONV_THREADS) {
    const int xs = i % HX, ys = (i / HX) % HY, zs = i / (HX * HY);
    const int xi = x0 - pad + xs, yi = y0 - pad + ys, zi = z0 - pad + zs;
    uint4 v0 = make_uint4(0u, 0u, 0u, 0u), v1 = v0;
    if (xi >= 0 && xi < vin.x && yi >= 0 && yi < vin.y && zi >= 0 && zi < vin.z) {
      const uint4* src =
          reinterpret_cast<const uint4*>(in) + ((((int64_t)b * vin.z + zi) * vin.y + yi) * vin.x + xi) * 2;
      v0 = src[0];
      v1 = src[1];
    }
    s_in[i] = v0;
    s_in[HALO + i] = v1;
  }
  // generic-proxy stores must be visible to the tensor cores' async proxy
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *s_tmem;

  // issue == 0 (the bounded-wait self-test): no MMA and no commit, so the
  // mbarrier never completes and the wait below must give up and report
  if (tid == 0 && issue) {
    const uint32_t a0 = smem_u32(s_in), w0 = smem_u32(s_w);
    for (int zz = 0; zz < TZ; ++zz) {
#pragma unroll 1
      for (int t = 0; t < 27; ++t) {
        const int dx = t % 3, dy = (t / 3) % 3, dz = t / 9;
        const uint64_t ad =
            smem_desc(a0 + (uint32_t)((((zz + dz) * HY + dy) * HX + dx) * 16), (uint32_t)(HALO * 16), HX * 16);
        const uint64_t bd = smem_desc(w0 + (uint32_t)(t * 512), 256u, 128u);
        umma_bf16(tmem + (uint32_t)(zz * CH), ad, bd, t > 0 ? 1u : 0u);
      }
    }
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(mbar))
                 : "memory");
  }
  const bool ok = __syncthreads_and(mbar_wait(smem_u32(mbar), 0u)) != 0;
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");

  const int r = warp * 32 + lane;  // TMEM lane = row of D = node of the tile
  const int xo = x0 + (r & 7), yo = y0 + (r >> 3);
  for (int zz = 0; zz < TZ; ++zz) {
    float v[16];
    if (ok) tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(zz * CH), v);
    const int zo = z0 + zz;
    if (!ok || xo >= ox || yo >= oy || zo >= oz) continue;
    const int64_t node = (((int64_t)b * oz + zo) * oy + yo) * ox + xo;
    uint4* dst = reinterpret_cast<uint4*>(out) + node * 2;
    if (!BWD) {
      float a[16];
#pragma unroll
      for (int c = 0; c < 16; ++c) {
        v[c] += bias[c];
        a[c] = gelu_f(v[c]);
      }
      if (zout) store16(reinterpret_cast<uint4*>(zout) + node * 2, v);
      store16(dst, a);
    } else {
      float zp[16];
      load16(reinterpret_cast<const uint4*>(zprev) + node * 2, zp);
#pragma unroll
      for (int c = 0; c < 16; ++c) v[c] *= gelu_grad_f(zp[c]);
      store16(dst, v);
    }
  }
  if (!ok && tid == 0) atomicOr(err, DEV_ERR_MMA_TIMEOUT);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
  }
}

// ---- weight gradients (CUDA cores) -------------------------------------------
constexpr int DZT = 2;  // output z slices per block
constexpr int DHZ = DZT + 2;
__global__ void __launch_bounds__(256) k_conv_dw(const __nv_bfloat16* __restrict__ x, Vol vin,
                                                 const __nv_bfloat16* __restrict__ dz, int oz, int oy, int ox,
                                                 int cin, float* __restrict__ dw, float* __restrict__ db) {
  __shared__ uint4 s_x[DHZ * HY * HX * 2];
  __shared__ uint4 s_d[DZT * TY * TX * 2];
  const int ntx = (ox + TX - 1) / TX;
  const int x0 = (int)(blockIdx.x % ntx) * TX, y0 = (int)(blockIdx.x / ntx) * TY, z0 = (int)blockIdx.y * DZT;
  const int b = blockIdx.z;
  for (int i = threadIdx.x; i < DHZ * HY * HX; i += blockDim.x) {
    const int xs = i % HX, ys = (i / HX) % HY, zs = i / (HX * HY);
    const int xi = x0 + xs, yi = y0 + ys, zi = z0 + zs;
    uint4 v0 = make_uint4(0u, 0u, 0u, 0u), v1 = v0;
    if (xi < vin.x && yi < vin.y && zi < vin.z) {
      const uint4* src =
          reinterpret_cast<const uint4*>(x) + ((((int64_t)b * vin.z + zi) * vin.y + yi) * vin.x + xi) * 2;
      v0 = src[0];
      v1 = src[1];
    }
    s_x[2 * i] = v0;
    s_x[2 * i + 1] = v1;
  }
  for (int i = threadIdx.x; i < DZT * TY * TX; i += blockDim.x) {
    const int xx = i % TX, yy = (i / TX) % TY, zz = i / (TX * TY);
    const int xo = x0 + xx, yo = y0 + yy, zo = z0 + zz;
    uint4 v0 = make_uint4(0u, 0u, 0u, 0u), v1 = v0;
    if (xo < ox && yo < oy && zo < oz) {
      const uint4* src = reinterpret_cast<const uint4*>(dz) + ((((int64_t)b * oz + zo) * oy + yo) * ox + xo) * 2;
      v0 = src[0];
      v1 = src[1];
    }
    s_d[2 * i] = v0;
    s_d[2 * i + 1] = v1;
  }
  __syncthreads();
  const int co = threadIdx.x >> 4, ci = threadIdx.x & 15;
  const __nv_bfloat16* sx = reinterpret_cast<const __nv_bfloat16*>(s_x);
  const __nv_bfloat16* sd = reinterpret_cast<const __nv_bfloat16*>(s_d);
  float acc[27];
#pragma unroll
  for (int t = 0; t < 27; ++t) acc[t] = 0.f;
  float dbs = 0.f;
  for (int v = 0; v < DZT * TY * TX; ++v) {
    const int xx = v % TX, yy = (v / TX) % TY, zz = v / (TX * TY);
    const float g = __bfloat162float(sd[v * 16 + co]);
    dbs += g;
    const int base = (zz * HY + yy) * HX + xx;
#pragma unroll
    for (int t = 0; t < 27; ++t) {
      const int node = base + ((t / 9) * HY + (t / 3) % 3) * HX + t % 3;
      acc[t] = fmaf(g, __bfloat162float(sx[node * 16 + ci]), acc[t]);
    }
  }
  if (ci < cin) {
#pragma unroll
    for (int t = 0; t < 27; ++t) atomicAdd(&dw[(t * CH + co) * cin + ci], acc[t]);
  }
  if (ci == 0) atomicAdd(&db[co], dbs);
}

// ---- packing of the operands ---------------------------------------------------
// Packed element e of a layer: tap t = e / 256, then [k group][n group][row][col]
// with n = output row of the MMA, k = reduction channel.
__global__ void k_pack(const float* __restrict__ p, Layout L, Packed P) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  const int per = 27 * 256;
  if (e >= 5 * per) return;
  const int which = e / per, r = e % per;
  const int t = r / 256, rem = r % 256;
  const int kg = rem / 128, ng = (rem / 64) & 1, row = (rem / 8) & 7, col = rem & 7;
  const int n = ng * 8 + row, k = kg * 8 + col;
  float val = 0.f;
  __nv_bfloat16* dst;
  if (which < 3) {  // forward: n = output channel, k = input channel
    const int l = which, cin = l == 0 ? L.c_in : CH;
    if (k < cin) val = p[L.w[l] + ((int64_t)t * CH + n) * cin + k];
    dst = reinterpret_cast<__nv_bfloat16*>(P.fwd[l]);
  } else {  // input gradient of layer 2 or 3: taps flipped, n = input channel, k = output channel
    const int l = which - 2;
    val = p[L.w[l] + ((int64_t)(26 - t) * CH + k) * CH + n];
    dst = reinterpret_cast<__nv_bfloat16*>(P.bwd[l]);
  }
  dst[r] = __float2bfloat16_rn(val);
}

// ---- head ------------------------------------------------------------------------
struct Corners {
  int64_t node[8];
  float w[8];
};

__device__ __forceinline__ Corners corners_local(Vol v, int b, float sx, float sy, float sz, bool periodic) {
  Corners c;
  const float s[3] = {sx, sy, sz};
  const int dim[3] = {v.x, v.y, v.z};
  int i0[3], i1[3];
  float f[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    int i = (int)floorf(s[d]);
    if (periodic) {
      i = ((i % dim[d]) + dim[d]) % dim[d];
      i1[d] = i + 1 == dim[d] ? 0 : i + 1;
    } else {
      i = min(max(i, 0), dim[d] - 2);
      i1[d] = i + 1;
    }
    i0[d] = i;
    f[d] = fminf(fmaxf(s[d] - floorf(s[d]), 0.f), 1.f);
  }
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const int ox = k & 1, oy = (k >> 1) & 1, oz = k >> 2;
    const int xx = ox ? i1[0] : i0[0], yy = oy ? i1[1] : i0[1], zz = oz ? i1[2] : i0[2];
    c.node[k] = (((int64_t)b * v.z + zz) * v.y + yy) * v.x + xx;
    c.w[k] = (ox ? f[0] : 1.f - f[0]) * (oy ? f[1] : 1.f - f[1]) * (oz ? f[2] : 1.f - f[2]);
  }
  return c;
}

__device__ __forceinline__ void head_node(const __nv_bfloat16* a3, int64_t node, const float* __restrict__ p,
                                          const Layout& L, float* o) {
  float a[16];
  load16(reinterpret_cast<const uint4*>(a3) + node * 2, a);
#pragma unroll
  for (int c = 0; c < NOUT; ++c) {
    float s = p[L.bh + c];
#pragma unroll
    for (int k = 0; k < CH; ++k) s = fmaf(p[L.wh + c * CH + k], a[k], s);
    o[c] = s;
  }
}

__global__ void k_head_field(const __nv_bfloat16* __restrict__ a3, int64_t nodes, const float* __restrict__ p,
                             Layout L, float* __restrict__ out) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= nodes) return;
  float o[NOUT];
  head_node(a3, i, p, L, o);
  for (int c = 0; c < NOUT; ++c) out[i * NOUT + c] = o[c];
}

__global__ void k_head_particles(const __nv_bfloat16* __restrict__ a3, Vol v3, const float* __restrict__ p,
                                 Layout L, HeadParticles hp, int periodic) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= hp.n) return;
  const int b = hp.pb ? hp.pb[i] : 0;
  const Corners c = corners_local(v3, b, hp.ps[3 * i], hp.ps[3 * i + 1], hp.ps[3 * i + 2], periodic != 0);
  float pred[NOUT] = {0.f, 0.f, 0.f};
#pragma unroll 1
  for (int k = 0; k < 8; ++k) {
    float o[NOUT];
    head_node(a3, c.node[k], p, L, o);
    for (int j = 0; j < NOUT; ++j) pred[j] = fmaf(c.w[k], o[j], pred[j]);
  }
  for (int j = 0; j < NOUT; ++j) hp.out[3 * i + j] = pred[j];
}

// Loss sum_p w_p |pred_p - t_p|^2 / sum w and its gradient with respect to the
// head output at the nodes (scattered with the trilinear weights).
__global__ void k_head_loss(const __nv_bfloat16* __restrict__ a3, Vol v3, const float* __restrict__ p, Layout L,
                            int64_t n, const int32_t* __restrict__ pb, const float* __restrict__ ps,
                            const float* __restrict__ tgt, const float* __restrict__ w,
                            const float* __restrict__ wsum, float* __restrict__ dout, float* __restrict__ loss) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  float contrib = 0.f;
  if (i < n && w[i] > 0.f) {
    const int b = pb ? pb[i] : 0;
    const Corners c = corners_local(v3, b, ps[3 * i], ps[3 * i + 1], ps[3 * i + 2], false);
    float pred[NOUT] = {0.f, 0.f, 0.f};
#pragma unroll 1
    for (int k = 0; k < 8; ++k) {
      float o[NOUT];
      head_node(a3, c.node[k], p, L, o);
      for (int j = 0; j < NOUT; ++j) pred[j] = fmaf(c.w[k], o[j], pred[j]);
    }
    const float lw = w[i] / *wsum;
    float g[NOUT];
    for (int j = 0; j < NOUT; ++j) {
      const float d = pred[j] - tgt[3 * i + j];
      contrib = fmaf(lw * d, d, contrib);
      g[j] = 2.f * lw * d;
    }
    for (int k = 0; k < 8; ++k)
      for (int j = 0; j < NOUT; ++j) atomicAdd(&dout[c.node[k] * NOUT + j], c.w[k] * g[j]);
  }
  for (int o = 16; o > 0; o >>= 1) contrib += __shfl_down_sync(0xffffffffu, contrib, o);
  if ((threadIdx.x & 31) == 0 && contrib != 0.f) atomicAdd(loss, contrib);
}

// Head backward: dZ3 = (Wh^T dout) * GELU'(z3); dWh, dbh accumulated.
__global__ void __launch_bounds__(256) k_head_bwd(const __nv_bfloat16* __restrict__ a3,
                                                  const __nv_bfloat16* __restrict__ z3,
                                                  const float* __restrict__ dout, int64_t nodes,
                                                  const float* __restrict__ p, Layout L,
                                                  __nv_bfloat16* __restrict__ dz3, float* __restrict__ grad) {
  __shared__ float red[NOUT * CH + NOUT];
  for (int k = threadIdx.x; k < NOUT * CH + NOUT; k += blockDim.x) red[k] = 0.f;
  __syncthreads();
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  float d[NOUT] = {0.f, 0.f, 0.f}, a[16];
  if (i < nodes) {
    for (int j = 0; j < NOUT; ++j) d[j] = dout[i * NOUT + j];
    float z[16], g[16];
    load16(reinterpret_cast<const uint4*>(a3) + i * 2, a);
    load16(reinterpret_cast<const uint4*>(z3) + i * 2, z);
#pragma unroll
    for (int k = 0; k < CH; ++k) {
      float s = 0.f;
      for (int j = 0; j < NOUT; ++j) s = fmaf(p[L.wh + j * CH + k], d[j], s);
      g[k] = s * gelu_grad_f(z[k]);
    }
    store16(reinterpret_cast<uint4*>(dz3) + i * 2, g);
  } else {
#pragma unroll
    for (int k = 0; k < CH; ++k) a[k] = 0.f;
  }
  // block reduction of dWh (3 x 16) and dbh (3)
  for (int j = 0; j < NOUT; ++j) {
#pragma unroll
    for (int k = 0; k <= CH; ++k) {
      float v = k < CH ? d[j] * a[k] : d[j];
      for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
      if ((threadIdx.x & 31) == 0) atomicAdd(&red[k < CH ? j * CH + k : NOUT * CH + j], v);
    }
  }
  __syncthreads();
  for (int k = threadIdx.x; k < NOUT * CH + NOUT; k += blockDim.x) {
    const int64_t dst = k < NOUT * CH ? L.wh + k : L.bh + (k - NOUT * CH);
    atomicAdd(&grad[dst], red[k]);
  }
}

__global__ void k_adam(float* __restrict__ p, float* __restrict__ m, float* __restrict__ v,
                       const float* __restrict__ g, int64_t n, float lr, float b1, float b2, float eps, float c1,
                       float c2) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi * c1) / (sqrtf(vi * c2) + eps);
}

}  // namespace

// ---- host wrappers -----------------------------------------------------------------
static void conv_launch(bool bwd, const __nv_bfloat16* in, Vol vin, int pad, __nv_bfloat16* out, Vol vout,
                        __nv_bfloat16* zout, const __nv_bfloat16* zprev, const uint4* w, const float* bias,
                        uint32_t* err, cudaStream_t s) {
  static bool attr_set[2] = {false, false};
  if (!attr_set[bwd]) {
    if (bwd)
      TPM_CUDA(cudaFuncSetAttribute(k_conv_tc<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, CONV_SMEM));
    else
      TPM_CUDA(cudaFuncSetAttribute(k_conv_tc<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, CONV_SMEM));
    attr_set[bwd] = true;
  }
  if (vout.x <= 0 || vout.y <= 0 || vout.z <= 0 || vout.b <= 0) return;
  const dim3 grid((unsigned)(((vout.x + TX - 1) / TX) * ((vout.y + TY - 1) / TY)), (unsigned)((vout.z + TZ - 1) / TZ),
                  (unsigned)vout.b);
  if (bwd)
    k_conv_tc<true><<<grid, CONV_THREADS, CONV_SMEM, s>>>(in, vin, pad, out, vout.z, vout.y, vout.x, zout, zprev, w,
                                                           bias, err, 1);
  else
    k_conv_tc<false><<<grid, CONV_THREADS, CONV_SMEM, s>>>(in, vin, pad, out, vout.z, vout.y, vout.x, zout, zprev,
                                                            w, bias, err, 1);
  TPM_LAUNCH_CHECK();
}

// One conv tile whose tensor-core work is never issued, then one normal tile:
// the first must end by its wait's time limit with DEV_ERR_MMA_TIMEOUT set
// (TMEM freed, nothing in flight), the second must run cleanly on the same
// context.  Returns the seconds the first launch took; throws on a failure.
double conv_wait_selftest(cudaStream_t s) {
  conv_launch(false, nullptr, Vol{0, 0, 0, 0}, 0, nullptr, Vol{0, 0, 0, 0}, nullptr, nullptr, nullptr, nullptr,
              nullptr, s);  // sets the shared-memory attribute only
  const Vol vin{1, TZ + 2, TY + 2, TX + 2};
  const int64_t in_bytes = vin.nodes() * CH * 2, out_bytes = (int64_t)TZ * TY * TX * CH * 2;
  char* buf = nullptr;
  const size_t total = (size_t)(in_bytes + out_bytes) + WPACK_U4 * 16 + CH * 4 + 16;
  TPM_CUDA(cudaMalloc(&buf, total));
  struct Free {
    char* p;
    ~Free() { cudaFree(p); }
  } guard{buf};
  TPM_CUDA(cudaMemsetAsync(buf, 0, total, s));
  auto* in = reinterpret_cast<__nv_bfloat16*>(buf);
  auto* out = reinterpret_cast<__nv_bfloat16*>(buf + in_bytes);
  auto* w = reinterpret_cast<uint4*>(buf + in_bytes + out_bytes);
  auto* bias = reinterpret_cast<float*>(buf + in_bytes + out_bytes + WPACK_U4 * 16);
  auto* err = reinterpret_cast<uint32_t*>(buf + in_bytes + out_bytes + WPACK_U4 * 16 + CH * 4);
  cudaEvent_t e0, e1;
  TPM_CUDA(cudaEventCreate(&e0));
  TPM_CUDA(cudaEventCreate(&e1));
  TPM_CUDA(cudaEventRecord(e0, s));
  k_conv_tc<false><<<dim3(1, 1, 1), CONV_THREADS, CONV_SMEM, s>>>(in, vin, 0, out, TZ, TY, TX, nullptr, nullptr, w,
                                                                   bias, err, 0);
  TPM_LAUNCH_CHECK();
  TPM_CUDA(cudaEventRecord(e1, s));
  uint32_t flag = 0;
  TPM_CUDA(cudaMemcpyAsync(&flag, err, 4, cudaMemcpyDeviceToHost, s));
  TPM_CUDA(cudaStreamSynchronize(s));
  float ms = 0.f;
  TPM_CUDA(cudaEventElapsedTime(&ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (!(flag & DEV_ERR_MMA_TIMEOUT)) throw Error(2, "the unissued tensor-core wait was not reported");
  TPM_CUDA(cudaMemsetAsync(err, 0, 4, s));
  k_conv_tc<false><<<dim3(1, 1, 1), CONV_THREADS, CONV_SMEM, s>>>(in, vin, 0, out, TZ, TY, TX, nullptr, nullptr, w,
                                                                   bias, err, 1);
  TPM_LAUNCH_CHECK();
  TPM_CUDA(cudaMemcpyAsync(&flag, err, 4, cudaMemcpyDeviceToHost, s));
  TPM_CUDA(cudaStreamSynchronize(s));
  if (flag != 0) throw Error(2, "a normal tensor-core tile failed after the timed-out one");
  return ms * 1e-3;
}

void conv_forward(const __nv_bfloat16* in, Vol vin, __nv_bfloat16* out, __nv_bfloat16* zout, const uint4* wpack,
                  const float* bias, uint32_t* err, cudaStream_t s) {
  const Vol vout{vin.b, vin.z - 2, vin.y - 2, vin.x - 2};
  conv_launch(false, in, vin, 0, out, vout, zout, nullptr, wpack, bias, err, s);
}

void conv_backward_data(const __nv_bfloat16* dz, Vol vdz, __nv_bfloat16* dzprev, const __nv_bfloat16* zprev,
                        const uint4* wpack_bwd, uint32_t* err, cudaStream_t s) {
  const Vol vout{vdz.b, vdz.z + 2, vdz.y + 2, vdz.x + 2};
  conv_launch(true, dz, vdz, 2, dzprev, vout, nullptr, zprev, wpack_bwd, nullptr, err, s);
}

void conv_backward_weights(const __nv_bfloat16* x, Vol vin, const __nv_bfloat16* dz, int cin, float* dw, float* db,
                           cudaStream_t s) {
  const int ox = vin.x - 2, oy = vin.y - 2, oz = vin.z - 2;
  if (ox <= 0 || oy <= 0 || oz <= 0) return;
  const dim3 grid((unsigned)(((ox + TX - 1) / TX) * ((oy + TY - 1) / TY)), (unsigned)((oz + DZT - 1) / DZT),
                  (unsigned)vin.b);
  k_conv_dw<<<grid, 256, 0, s>>>(x, vin, dz, oz, oy, ox, cin, dw, db);
  TPM_LAUNCH_CHECK();
}

void pack_weights(const float* params, const Layout& L, const Packed& P, cudaStream_t s) {
  k_pack<<<(5 * 27 * 256 + 255) / 256, 256, 0, s>>>(params, L, P);
  TPM_LAUNCH_CHECK();
}

void head_at_particles(const __nv_bfloat16* a3, Vol v3, const float* params, const Layout& L,
                       const HeadParticles& hp, cudaStream_t s) {
  if (hp.n == 0) return;
  k_head_particles<<<grid_for(hp.n, 256, 1ll << 30), 256, 0, s>>>(a3, v3, params, L, hp, 0);
  TPM_LAUNCH_CHECK();
}

void head_periodic(const __nv_bfloat16* a3, Vol v3, const float* params, const Layout& L, const HeadParticles& hp,
                   cudaStream_t s) {
  if (hp.n == 0) return;
  k_head_particles<<<grid_for(hp.n, 256, 1ll << 30), 256, 0, s>>>(a3, v3, params, L, hp, 1);
  TPM_LAUNCH_CHECK();
}

void head_field(const __nv_bfloat16* a3, int64_t nodes, const float* params, const Layout& L, float* out,
                cudaStream_t s) {
  k_head_field<<<grid_for(nodes, 256, 1ll << 30), 256, 0, s>>>(a3, nodes, params, L, out);
  TPM_LAUNCH_CHECK();
}

void head_loss(const __nv_bfloat16* a3, Vol v3, const float* params, const Layout& L, int64_t n, const int32_t* pb,
               const float* ps, const float* tgt, const float* w, const float* wsum, float* dout, float* loss,
               cudaStream_t s) {
  if (n == 0) return;
  k_head_loss<<<grid_for(n, 256, 1ll << 30), 256, 0, s>>>(a3, v3, params, L, n, pb, ps, tgt, w, wsum, dout, loss);
  TPM_LAUNCH_CHECK();
}

void head_backward(const __nv_bfloat16* a3, const __nv_bfloat16* z3, const float* dout, int64_t nodes,
                   const float* params, const Layout& L, __nv_bfloat16* dz3, float* grad, cudaStream_t s) {
  k_head_bwd<<<grid_for(nodes, 256, 1ll << 30), 256, 0, s>>>(a3, z3, dout, nodes, params, L, dz3, grad);
  TPM_LAUNCH_CHECK();
}

void adam(float* p, float* m, float* v, const float* g, int64_t n, float lr, float b1, float b2, float eps, int64_t step,
          cudaStream_t s) {
  const float c1 = (float)(1.0 / (1.0 - std::pow((double)b1, (double)step)));
  const float c2 = (float)(1.0 / (1.0 - std::pow((double)b2, (double)step)));
  k_adam<<<grid_for(n, 256, 1ll << 30), 256, 0, s>>>(p, m, v, g, n, lr, b1, b2, eps, c1, c2);
  TPM_LAUNCH_CHECK();
}

}  // namespace cnn
}  // namespace tpm
