// Long-range PM on the device.
//
// Reference path: cic::assign (crates/gadget-ng-pm/src/cic.rs:37-93, :260-292)
// -> fft_poisson::solve_forces_filtered (fft_poisson.rs:87-103, :306-476) ->
// cic::interpolate (cic.rs:100-170, :298-346).
//
// The reference transforms a complex copy of the real density with three
// passes of 1D c2c FFTs (x, y, z), multiplies by -4 pi G W(k)/k^2, forms
// F_a = -i k_a phi, transforms back (z, y, x) and keeps the real part / N^3.
// Here the density is real, so only the kx in [0, N/2] half spectrum is
// carried (the other half is its conjugate): an x pass real -> half spectrum,
// a y pass, one kernel that does the forward z pass, the Green's function,
// the filter and the gradient for all three components and their inverse z
// passes without leaving shared memory, then inverse y and x passes back to
// three real force meshes.  Taking the real part in the reference zeroes the
// derivative's Nyquist plane (F_x at kx = N/2 and so on); the derivative table
// is zero there, so the half spectrum is exactly Hermitian.  Every 1D
// transform is a two-stage register transform (fft_reg.cuh) with one
// shared-memory exchange; the y and z passes stage their pencils (CTX
// adjacent kx columns of a z plane or a y row) with TMA tensor copies, the x
// passes their contiguous rows with one bulk copy per block.  Half-spectrum
// rows are padded to an even length (nhp) for the copies' 16-byte rule.
// Linear in G: the meshes hold forces per unit G, the gather multiplies by g.
#include <cuda.h>
#include <cudaTypedefs.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "../../include/treepm_b200.h"
#include "common.cuh"
#include "fft_reg.cuh"
#include "pm.cuh"

namespace tpm {
namespace {

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }

// Twiddle exp(-+2 pi i m / n) from the half table tw[m] = exp(-2 pi i m / n), m < n/2.
__device__ __forceinline__ float2 twiddle(const float2* tw, int m, int n, bool inv) {
  const int half = n >> 1;
  float2 w = m < half ? tw[m] : make_float2(-tw[m - half].x, -tw[m - half].y);
  if (inv) w.y = -w.y;
  return w;
}

__device__ __forceinline__ void load_twiddles(float2* s_tw, const float2* tw, int n) {
  for (int i = threadIdx.x; i < (n >> 1); i += blockDim.x) s_tw[i] = tw[i];
}

// ---- pencil passes (y and z): TMA-staged tiles, register transforms ----------------
// A block transforms CTX adjacent kx columns of one y row (z pass) or one z
// plane (y pass) of a half spectrum.  One thread issues the bulk tensor copy
// of the n x CTX tile into shared memory (8-byte complex elements, rows of CTX
// values); every thread then runs its share of the two-stage transform of
// fft_reg.cuh and the valid columns are written back with coalesced stores.

// Columns per tile: 16 (128-byte rows), 8 for the longest transforms.
template <int LOGN> struct Pencil {
  static constexpr int N = 1 << LOGN;
  static constexpr int CTX = N > 512 ? 8 : 16;
  static constexpr int THREADS = CTX * fftr::Split<LOGN>::N2;
  static constexpr int ROWS_PER_COPY = N < 256 ? N : 256;  // a tensor-map box spans at most 256 rows
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ uint64_t globaltimer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Stage the tile; false (and DEV_ERR_TMA_TIMEOUT) when the copy does not
// complete within 2 s.  axis 0: y pencils (rows are y of plane `fixed`), 1: z
// pencils (rows are z of row `fixed`); zbase = comp * nm.
template <int LOGN>
__device__ bool stage_pencil(float2* tile, uint64_t* bar, const CUtensorMap* map, int axis, int kx0, int fixed,
                             int zbase, uint32_t* err) {
  using P = Pencil<LOGN>;
  const uint32_t b = smem_u32(bar);
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(b));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b),
                 "r"((uint32_t)(P::N * P::CTX * sizeof(float2)))
                 : "memory");
    for (int r0 = 0; r0 < P::N; r0 += P::ROWS_PER_COPY) {
      const uint32_t dst = smem_u32(tile + (size_t)r0 * P::CTX);
      const int y = axis == 0 ? r0 : fixed, z = axis == 0 ? zbase + fixed : zbase + r0;
      asm volatile(
          "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
          "[%5];" ::"r"(dst),
          "l"(map), "r"(kx0), "r"(y), "r"(z), "r"(b)
          : "memory");
    }
  }
  __syncthreads();  // the barrier is initialised before anyone waits on it
  bool done = false;
  const uint64_t t0 = globaltimer_ns();
  for (;;) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(b)
        : "memory");
    if (ok) {
      done = true;
      break;
    }
    if (globaltimer_ns() - t0 > 2000000000ull) break;
  }
  if (!done && threadIdx.x == 0) atomicOr(err, DEV_ERR_TMA_TIMEOUT);
  return __syncthreads_and(done) != 0;
}

// In-place length-N transform of the CTX columns of a [N][CTX] tile (element
// j of column c at tile[j * CTX + c]); natural order in and out.
template <int LOGN, bool INV>
__device__ __forceinline__ void pencil_fft(float2* tile, const float2* s_tw) {
  using S = fftr::Split<LOGN>;
  constexpr int N = S::N, N1 = S::N1, N2 = S::N2, R = S::R, CTX = Pencil<LOGN>::CTX;
  const int c = threadIdx.x % CTX, t = threadIdx.x / CTX;  // t in [0, N2)
  // stage 1: thread t = j2 holds x[N2 j1 + j2], j1 < N1
  float2 v[N1];
#pragma unroll
  for (int j1 = 0; j1 < N1; ++j1) v[j1] = tile[(N2 * j1 + t) * CTX + c];
  fftr::dft<N1, INV>(v);
#pragma unroll
  for (int k1 = 1; k1 < N1; ++k1) v[k1] = cmul(v[k1], twiddle(s_tw, (t * k1) & (N - 1), N, INV));
  __syncthreads();
#pragma unroll
  for (int k1 = 0; k1 < N1; ++k1) tile[(k1 * N2 + t) * CTX + c] = v[k1];
  __syncthreads();
  // stage 2: N2-point transforms over j2 for k1 = t + N2 r
  float2 w[R][N2];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int k1 = t + N2 * r;
#pragma unroll
    for (int j2 = 0; j2 < N2; ++j2) w[r][j2] = tile[(k1 * N2 + j2) * CTX + c];
    fftr::dft<N2, INV>(w[r]);
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int k1 = t + N2 * r;
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) tile[(k1 + N1 * k2) * CTX + c] = w[r][k2];
  }
  __syncthreads();
}

// Shared memory of a pencil kernel: `tiles` tiles, the N/2 twiddles, the barrier.
template <int LOGN> constexpr size_t pencil_smem(int tiles) {
  return (size_t)tiles * Pencil<LOGN>::N * Pencil<LOGN>::CTX * sizeof(float2) +
         (size_t)(Pencil<LOGN>::N / 2 > 0 ? Pencil<LOGN>::N / 2 : 1) * sizeof(float2) + 16;
}

// Store the valid columns (kx < nh) of a tile back to [comp][z][y][kx]:
// prow y rows per z plane, ppc z planes per component.
template <int LOGN>
__device__ __forceinline__ void store_pencil(const float2* tile, float2* __restrict__ data, int axis, int kx0,
                                             int fixed, int comp, int nh, int nhp, int prow, int ppc) {
  using P = Pencil<LOGN>;
  const int64_t plane = (int64_t)prow * nhp;
  float2* base = data + (int64_t)comp * ppc * plane;
  for (int idx = threadIdx.x; idx < P::N * P::CTX; idx += blockDim.x) {
    const int r = idx / P::CTX, c = idx % P::CTX, kx = kx0 + c;
    if (kx >= nh) continue;
    const int64_t a = axis == 0 ? fixed * plane + (int64_t)r * nhp + kx : r * plane + (int64_t)fixed * nhp + kx;
    base[a] = tile[idx];
  }
}

template <int LOGN>
__device__ __forceinline__ void pencil_layout(unsigned char* sm, float2*& tile, float2*& tile2, float2*& s_tw,
                                              uint64_t*& bar, int tiles) {
  using P = Pencil<LOGN>;
  tile = reinterpret_cast<float2*>(sm);
  tile2 = tiles > 1 ? tile + P::N * P::CTX : nullptr;
  s_tw = tile + (size_t)tiles * P::N * P::CTX;
  bar = reinterpret_cast<uint64_t*>(s_tw + (P::N / 2 > 0 ? P::N / 2 : 1));
}

// c2c pass along y (axis 0) or z (axis 1) of ncomp half spectra, in place:
// prow y rows per z plane, ppc z planes per component (the full mesh: nm
// and nm; a z slab: nm and its planes; a y slab: its rows and nm).
template <int LOGN, bool INV>
__global__ void __launch_bounds__(Pencil<LOGN>::THREADS) k_pencil(const __grid_constant__ CUtensorMap map,
                                                                  float2* __restrict__ data, int axis, int nh,
                                                                  int nhp, int prow, int ppc,
                                                                  const float2* __restrict__ tw,
                                                                  uint32_t* __restrict__ err) {
  extern __shared__ __align__(128) unsigned char psm[];
  float2 *tile, *tile2, *s_tw;
  uint64_t* bar;
  pencil_layout<LOGN>(psm, tile, tile2, s_tw, bar, 1);
  load_twiddles(s_tw, tw, Pencil<LOGN>::N);
  const int kx0 = blockIdx.x * Pencil<LOGN>::CTX, fixed = blockIdx.y, comp = blockIdx.z;
  if (!stage_pencil<LOGN>(tile, bar, &map, axis, kx0, fixed, comp * ppc, err)) return;
  pencil_fft<LOGN, INV>(tile, s_tw);
  store_pencil<LOGN>(tile, data, axis, kx0, fixed, comp, nh, nhp, prow, ppc);
}

// Forward z pass, Green's function x filter x gradient, and the inverse z
// passes of the ncomp components (4: the potential itself as well).
// prow: y rows per z plane of the input and output layouts (nm, or a y
// slab's rows starting at global row y0).
template <int LOGN>
__global__ void __launch_bounds__(Pencil<LOGN>::THREADS) k_pencil_poisson(
    const __grid_constant__ CUtensorMap map, float2* __restrict__ spec3, int nh, int nhp, int prow, int y0,
    const float2* __restrict__ tw, const float* __restrict__ kval, const float* __restrict__ kfilter,
    const float* __restrict__ kderiv, float kcoef, int ncomp, uint32_t* __restrict__ err) {
  using P = Pencil<LOGN>;
  extern __shared__ __align__(128) unsigned char psm[];
  float2 *tile, *phi, *s_tw;
  uint64_t* bar;
  pencil_layout<LOGN>(psm, tile, phi, s_tw, bar, 2);
  load_twiddles(s_tw, tw, P::N);
  const int kx0 = blockIdx.x * P::CTX, yl = blockIdx.y, y = y0 + yl;
  if (!stage_pencil<LOGN>(tile, bar, &map, 1, kx0, yl, 0, err)) return;
  pencil_fft<LOGN, false>(tile, s_tw);
  // phi(k) = rho(k) kcoef W(k) / k^2
  for (int idx = threadIdx.x; idx < P::N * P::CTX; idx += blockDim.x) {
    const int z = idx / P::CTX, kx = kx0 + idx % P::CTX;
    float2 v = make_float2(0.f, 0.f);
    if (kx < nh) {
      const float k2 = kval[kx] * kval[kx] + kval[y] * kval[y] + kval[z] * kval[z];
      if (k2 > 0.f) {
        const float sc = kcoef * kfilter[kx] * kfilter[y] * kfilter[z] / k2;
        v = make_float2(tile[idx].x * sc, tile[idx].y * sc);
      }
    }
    phi[idx] = v;
  }
  __syncthreads();
  for (int comp = 0; comp < ncomp; ++comp) {
    for (int idx = threadIdx.x; idx < P::N * P::CTX; idx += blockDim.x) {
      const int z = idx / P::CTX, kx = min(kx0 + idx % P::CTX, nh - 1);
      const float2 ph = phi[idx];
      if (comp == 3) {  // the potential itself
        tile[idx] = ph;
        continue;
      }
      const float d = comp == 0 ? kderiv[kx] : (comp == 1 ? kderiv[y] : kderiv[z]);
      tile[idx] = make_float2(d * ph.y, -d * ph.x);  // -i D phi
    }
    __syncthreads();
    pencil_fft<LOGN, true>(tile, s_tw);
    store_pencil<LOGN>(tile, spec3, 1, kx0, yl, comp, nh, nhp, prow, P::N);
    __syncthreads();
  }
}

__device__ __forceinline__ double pk_sinc(int k, int nm) {
  if (k == 0) return 1.0;
  const double x = (double)k / (double)nm;
  return sinpi(x) / (M_PI * x);
}

// Forward z pass of the half spectrum, then every mode into its |k| shell:
// sum of |rho_k|^2 / W^2 and the mode count, modes with 0 < kx < nm/2 twice
// (their conjugates are not stored), as power_spectrum.rs:74-110 over the full
// cube.
template <int LOGN>
__global__ void __launch_bounds__(Pencil<LOGN>::THREADS) k_pencil_pk(
    const __grid_constant__ CUtensorMap map, int nh, const float2* __restrict__ tw, double* __restrict__ pk_sum,
    unsigned long long* __restrict__ pk_n, uint32_t* __restrict__ err) {
  using P = Pencil<LOGN>;
  constexpr int nm = P::N, nb = P::N / 2;
  extern __shared__ __align__(128) unsigned char psm[];
  float2 *tile, *unused, *s_tw;
  uint64_t* bar;
  pencil_layout<LOGN>(psm, tile, unused, s_tw, bar, 1);
  double* hs = reinterpret_cast<double*>(psm + pencil_smem<LOGN>(1));
  unsigned long long* hn = reinterpret_cast<unsigned long long*>(hs + nb);
  load_twiddles(s_tw, tw, nm);
  for (int i = threadIdx.x; i < nb; i += blockDim.x) {
    hs[i] = 0.0;
    hn[i] = 0ull;
  }
  const int kx0 = blockIdx.x * P::CTX, y = blockIdx.y;
  if (!stage_pencil<LOGN>(tile, bar, &map, 1, kx0, y, 0, err)) return;
  pencil_fft<LOGN, false>(tile, s_tw);
  const int fy = y <= nb ? y : y - nm;
  for (int idx = threadIdx.x; idx < nm * P::CTX; idx += blockDim.x) {
    const int z = idx / P::CTX, kx = kx0 + idx % P::CTX;
    if (kx >= nh) continue;
    const int fz = z <= nb ? z : z - nm;
    const double k2 = (double)kx * kx + (double)fy * fy + (double)fz * fz;
    if (k2 == 0.0) continue;
    const double bf = sqrt(k2) - 0.5;
    if (bf < 0.0 || bf >= (double)nb) continue;
    const int bin = (int)bf;
    const double w = pk_sinc(kx, nm) * pk_sinc(fy, nm) * pk_sinc(fz, nm);
    const double re = tile[idx].x, im = tile[idx].y;
    const int mult = (kx == 0 || kx == nb) ? 1 : 2;
    atomicAdd(&hs[bin], mult * (re * re + im * im) / (w * w));
    atomicAdd(&hn[bin], (unsigned long long)mult);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < nb; i += blockDim.x)
    if (hn[i]) {
      atomicAdd(&pk_sum[i], hs[i]);
      atomicAdd(&pk_n[i], hn[i]);
    }
}

// ---- CIC deposit (cic.rs:37-93) ------------------------------------------------
struct Cic {
  int ix[2], iy[2], iz[2];
  float wx[2], wy[2], wz[2];
};

// One CIC axis with the integer <-> float64 conversions done by float64
// adds instead of conversion instructions (the conversion pipe was 93 % busy
// in the deposit, ahead of every other unit): the exact float64 of q as the
// bit pattern of 2^52 + q minus 2^52, and floor(c) as the low word of the
// round-down sum c + 2^52 (c in [0, nm)).  Same values as (double)q, floor and
// (int) on these ranges; the upper node index wraps without a division.
constexpr double TWO52 = 4503599627370496.0;
__device__ __forceinline__ double u32_to_f64(uint32_t q) {
  return dsub(__hiloint2double(0x43300000, (int)q), TWO52);
}

__device__ __forceinline__ void cic_axis(uint32_t q, double scale, double inv_cell, double nmf, int nm, int* i,
                                         float* w) {
  const double c = rem_once(dmul(dmul(u32_to_f64(q), scale), inv_cell), nmf);
  const double t = __dadd_rd(c, TWO52);  // 2^52 + floor(c)
  const int i0 = __double2loint(t);
  const double d = dsub(c, dsub(t, TWO52));
  i[0] = i0;
  i[1] = i0 + 1 == nm ? 0 : i0 + 1;
  w[0] = (float)dsub(1.0, d);
  w[1] = (float)d;
}

__device__ __forceinline__ Cic cic_of(uint32_t qx, uint32_t qy, uint32_t qz, double scale, double inv_cell, int nm) {
  Cic c;
  const double nmf = (double)nm;
  cic_axis(qx, scale, inv_cell, nmf, nm, c.ix, c.wx);
  cic_axis(qy, scale, inv_cell, nmf, nm, c.iy, c.wy);
  cic_axis(qz, scale, inv_cell, nmf, nm, c.iz, c.wz);
  return c;
}

// The particles arrive in octree order, so a warp's 32 particles sit in a
// compact region and lanes often share a CIC cell.  Lanes with the same base
// cell are grouped with match_any and the group's first lane sums their 8
// weighted masses through shuffles.  Those leaders then add their 8 sums into
// a per-warp 8 x 8 x 8 node window in shared memory placed at the warp's
// smallest base cell, one corner slot at a time (within a slot every leader
// writes a different node, so a plain read-modify-write suffices); the
// window's non-zero nodes then go to the mesh with one atomic each, lanes on
// consecutive x of a window row so that one atomic instruction covers four
// mesh rows.  A warp whose base cells do not fit in the window adds its sums
// to the mesh directly.  At 256^3 (16.7 M particles) the deposit went from
// 512 to 330 us with the window, the used-rows flush and the segmented sums:
// neighbouring particles' shared corner nodes take one atomic instead of up
// to eight.
constexpr int DEP_THREADS = 256;
constexpr int DEP_WIN = 8;  // window side (nodes); the flush indexes x, y, z by 3-bit fields
static_assert(DEP_WIN == 8, "the flush maps eight lanes to a window row");

// d in (-nm, nm) to the periodic offset in [-nm/2, nm/2)
__device__ __forceinline__ int wrap_offset(int d, int nm) {
  return d >= nm / 2 ? d - nm : (d < -nm / 2 ? d + nm : d);
}

__global__ void __launch_bounds__(DEP_THREADS) k_deposit(const uint32_t* __restrict__ qx, const uint32_t* __restrict__ qy,
                          const uint32_t* __restrict__ qz, const float* __restrict__ m, int64_t n, double scale,
                          double inv_cell, int nm, float* __restrict__ rho, const uint32_t* __restrict__ id,
                          uint32_t id_limit) {
  __shared__ __align__(16) float s_win[DEP_THREADS / 32][DEP_WIN * DEP_WIN * DEP_WIN];
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;
  float* win = s_win[threadIdx.x >> 5];
  const bool live = i < n && (!id || id[i] < id_limit);
  Cic c{};
  float mi = 0.f;
  uint32_t key = 0xFFFFFFFFu;
  if (live) {
    c = cic_of(qx[i], qy[i], qz[i], scale, inv_cell, nm);
    mi = m[i];
    key = (uint32_t)(((int64_t)c.iz[0] * nm + c.iy[0]) * nm + c.ix[0]);
  }
  const uint32_t peers = __match_any_sync(0xffffffffu, key);
  const int rounds = __reduce_max_sync(0xffffffffu, (unsigned)__popc(peers));
  float sum[8];
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b)
#pragma unroll
      for (int d = 0; d < 2; ++d) sum[a * 4 + b * 2 + d] = mi * c.wx[d] * c.wy[b] * c.wz[a];
  if (rounds > 1) {
    // groups of consecutive lanes (octree order makes them the rule): a
    // segmented suffix sum, five shuffle steps whatever the group size; the
    // group's first lane ends with its total
    const int end = 32 - __clz(peers);
    if (__all_sync(0xffffffffu, __popc(peers) == end - (__ffs(peers) - 1))) {
#pragma unroll
      for (int off = 1; off < 32; off <<= 1) {
#pragma unroll
        for (int k = 0; k < 8; ++k) {
          const float y = __shfl_down_sync(0xffffffffu, sum[k], off);
          if (lane + off < end) sum[k] += y;
        }
      }
    } else {  // scattered groups: the leader gathers its members one at a time
#pragma unroll
      for (int k = 0; k < 8; ++k) sum[k] = 0.f;
      uint32_t rest = peers;
      for (int r = 0; r < rounds; ++r) {  // the same count on every lane: full-warp shuffles
        const int src = rest ? __ffs(rest) - 1 : lane;
        const bool take = rest != 0u;
        rest &= rest - 1u;
        const float sm = __shfl_sync(0xffffffffu, mi, src);
        const float x0 = __shfl_sync(0xffffffffu, c.wx[0], src), x1 = __shfl_sync(0xffffffffu, c.wx[1], src);
        const float y0 = __shfl_sync(0xffffffffu, c.wy[0], src), y1 = __shfl_sync(0xffffffffu, c.wy[1], src);
        const float z0 = __shfl_sync(0xffffffffu, c.wz[0], src), z1 = __shfl_sync(0xffffffffu, c.wz[1], src);
        if (take) {
          sum[0] += sm * x0 * y0 * z0;
          sum[1] += sm * x1 * y0 * z0;
          sum[2] += sm * x0 * y1 * z0;
          sum[3] += sm * x1 * y1 * z0;
          sum[4] += sm * x0 * y0 * z1;
          sum[5] += sm * x1 * y0 * z1;
          sum[6] += sm * x0 * y1 * z1;
          sum[7] += sm * x1 * y1 * z1;
        }
      }
    }
  }
  const bool lead = live && lane == __ffs(peers) - 1;
  const uint32_t leaders = __ballot_sync(0xffffffffu, lead);
  if (leaders == 0u) return;
  const int f = __ffs(leaders) - 1;
  const int o[3] = {__shfl_sync(0xffffffffu, c.ix[0], f), __shfl_sync(0xffffffffu, c.iy[0], f),
                    __shfl_sync(0xffffffffu, c.iz[0], f)};
  const int mine[3] = {c.ix[0], c.iy[0], c.iz[0]};
  int rel[3], lo[3], ext[3];
  bool fits = true;
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    rel[d] = wrap_offset(mine[d] - o[d], nm);
    lo[d] = __reduce_min_sync(0xffffffffu, lead ? rel[d] : 0x7FFFFFFF);
    const int hi = __reduce_max_sync(0xffffffffu, lead ? rel[d] : -0x7FFFFFFF);
    ext[d] = hi - lo[d] + 2;  // nodes used along this axis
    fits = fits && ext[d] <= DEP_WIN;
  }
  const int64_t nm2 = (int64_t)nm * nm;
  if (!fits) {
    if (!lead) return;
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int b = 0; b < 2; ++b)
#pragma unroll
        for (int d = 0; d < 2; ++d) atomicAdd(&rho[c.iz[a] * nm2 + (int64_t)c.iy[b] * nm + c.ix[d]], sum[a * 4 + b * 2 + d]);
    return;
  }
#pragma unroll
  for (int k = 0; k < DEP_WIN * DEP_WIN * DEP_WIN / 128; ++k)
    reinterpret_cast<float4*>(win)[lane + 32 * k] = make_float4(0.f, 0.f, 0.f, 0.f);
  __syncwarp();
  const int base = ((rel[2] - lo[2]) * DEP_WIN + (rel[1] - lo[1])) * DEP_WIN + (rel[0] - lo[0]);
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    if (lead) {
      const int w = base + ((k >> 2) * DEP_WIN + ((k >> 1) & 1)) * DEP_WIN + (k & 1);
      win[w] += sum[k];
    }
    __syncwarp();
  }
  // the used rows of the window to the mesh, four rows per pass with
  // consecutive lanes on consecutive x, so one atomic instruction touches four
  // mesh rows; row r is (y, z) = (r mod ext_y, r div ext_y), the division by
  // a multiply (r < 64, ext_y <= 8)
  const int rows = ext[1] * ext[2];
  const uint32_t mdiv = (65536u + (uint32_t)ext[1] - 1u) / (uint32_t)ext[1];
  const int x = lane & 7;
  for (int r0 = 0; r0 < rows; r0 += 4) {
    const int r = r0 + (lane >> 3);
    if (r >= rows || x >= ext[0]) continue;
    const int zz = (int)(((uint32_t)r * mdiv) >> 16), yy = r - zz * ext[1];
    const float v = win[(zz * DEP_WIN + yy) * DEP_WIN + x];
    if (v == 0.f) continue;
    int gx = o[0] + lo[0] + x, gy = o[1] + lo[1] + yy, gz = o[2] + lo[2] + zz;
    gx = gx < 0 ? gx + nm : (gx >= nm ? gx - nm : gx);
    gy = gy < 0 ? gy + nm : (gy >= nm ? gy - nm : gy);
    gz = gz < 0 ? gz + nm : (gz >= nm ? gz - nm : gz);
    atomicAdd(&rho[gz * nm2 + (int64_t)gy * nm + gx], v);
  }
}

__global__ void k_cells(const uint32_t* __restrict__ qx, const uint32_t* __restrict__ qy,
                        const uint32_t* __restrict__ qz, const uint32_t* __restrict__ id, int64_t n, double scale,
                        double inv_cell, int nm, int32_t* __restrict__ out) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const Cic c = cic_of(qx[i], qy[i], qz[i], scale, inv_cell, nm);
  const int64_t o = 3 * (int64_t)id[i];
  out[o] = c.ix[0];
  out[o + 1] = c.iy[0];
  out[o + 2] = c.iz[0];
}

// ---- x passes: a real row of nm samples as one complex row of h = nm/2 -------
// (x[2j], x[2j+1]) is packed as z[j] = x[2j] + i x[2j+1] and transformed at
// half length.  Forward: X[k] = E[k] + e^{-2 pi i k/nm} O[k] with
// E = (Z[k] + conj Z[h-k]) / 2 and O = (Z[k] - conj Z[h-k]) / 2i, k = 0..h.
// Inverse: Z[k] = X[k] (1 + i W_k) + conj(X[h-k]) (1 - i W_k), W_k =
// e^{2 pi i k/nm}, k < h; the unnormalised inverse of Z gives x[2j] and
// x[2j+1] as its real and imaginary parts (the row spectrum is Hermitian, so
// X[0] and X[h] are real up to rounding).
//
// RX rows per block, N2 threads per row (Split<log2 h>).  The block's input
// rows are one contiguous range of global memory: one bulk copy (no tensor
// map) stages them in shared memory.  Stage 1 reads a row's elements from
// there; the exchange between the stages goes through a padded buffer (row of
// N2 x (N1 + 1)), so neither stage's shared-memory accesses collide in a bank.

template <int LOGH> struct RowPass {
  using S = fftr::Split<LOGH>;
  static constexpr int H = 1 << LOGH;
  static constexpr int RX = 256 / S::N2 > 0 ? 256 / S::N2 : 1;  // rows per block: 256 threads
  static constexpr int THREADS = RX * S::N2;
  static constexpr int YP = S::N2 * (S::N1 + 1);  // padded exchange row
};

// One bulk copy of `bytes` contiguous bytes into shared memory; false (and
// DEV_ERR_TMA_TIMEOUT) when it does not complete within 2 s.
__device__ bool stage_bulk(void* dst, const void* src, uint32_t bytes, uint64_t* bar, uint32_t* err) {
  const uint32_t b = smem_u32(bar);
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(b));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(bytes) : "memory");
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(b)
                 : "memory");
  }
  __syncthreads();
  bool done = false;
  const uint64_t t0 = globaltimer_ns();
  for (;;) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(ok)
        : "r"(b)
        : "memory");
    if (ok) {
      done = true;
      break;
    }
    if (globaltimer_ns() - t0 > 2000000000ull) break;
  }
  if (!done && threadIdx.x == 0) atomicOr(err, DEV_ERR_TMA_TIMEOUT);
  return __syncthreads_and(done) != 0;
}

// Real rows of nm samples -> half spectra (pitch nhp): the half-length
// transform of the packed row, then the even / odd split above.
template <int LOGH>
__global__ void __launch_bounds__(RowPass<LOGH>::THREADS) k_row_r2c(const float* __restrict__ rho,
                                                                   float2* __restrict__ spec, int nhp,
                                                                   int64_t nrows, const float2* __restrict__ tw,
                                                                   uint32_t* __restrict__ err) {
  using RP = RowPass<LOGH>;
  using S = typename RP::S;
  constexpr int H = RP::H, N1 = S::N1, N2 = S::N2, R = S::R, RX = RP::RX, NM = 2 * H;
  extern __shared__ __align__(128) unsigned char rsm[];
  float2* rows = reinterpret_cast<float2*>(rsm);             // RX x H (input, then the transform)
  float2* ybuf = rows + RX * H;                              // RX x YP
  float2* s_tw = ybuf + RX * RP::YP;                         // NM / 2 twiddles of length NM
  uint64_t* bar = reinterpret_cast<uint64_t*>(s_tw + NM / 2);
  for (int i = threadIdx.x; i < NM / 2; i += blockDim.x) s_tw[i] = tw[i];
  const int64_t row0 = (int64_t)blockIdx.x * RX;
  const int nr = (int)min((int64_t)RX, nrows - row0);
  if (!stage_bulk(rows, rho + row0 * NM, (uint32_t)(nr * NM * sizeof(float)), bar, err)) return;
  const int rr = threadIdx.x / N2, t = threadIdx.x % N2;
  float2 out[R][N2];
  const float2* row = rows + rr * H;
  {
    float2 v[N1];
#pragma unroll
    for (int j1 = 0; j1 < N1; ++j1) v[j1] = row[N2 * j1 + t];
    fftr::dft<N1, false>(v);
#pragma unroll
    for (int k1 = 1; k1 < N1; ++k1) v[k1] = cmul(v[k1], twiddle(s_tw, 2 * ((t * k1) & (H - 1)), NM, false));
    float2* yb = ybuf + rr * RP::YP;
#pragma unroll
    for (int k1 = 0; k1 < N1; ++k1) yb[k1 + t * (N1 + 1)] = v[k1];
    __syncthreads();
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int k1 = t + N2 * r;
#pragma unroll
      for (int j2 = 0; j2 < N2; ++j2) out[r][j2] = yb[k1 + j2 * (N1 + 1)];
      fftr::dft<N2, false>(out[r]);
    }
  }
  __syncthreads();
  // Z[k] in natural order into the row buffer
#pragma unroll
  for (int r = 0; r < R; ++r)
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) rows[rr * H + (t + N2 * r) + N1 * k2] = out[r][k2];
  __syncthreads();
  // split: X[k] = E + w_NM^k O, k = 0..H
  for (int idx = threadIdx.x; idx < nr * (H + 1); idx += blockDim.x) {
    const int r = idx / (H + 1), k = idx % (H + 1);
    const float2 zk = rows[r * H + (k == H ? 0 : k)];
    const float2 zm = rows[r * H + (k == 0 || k == H ? 0 : H - k)];
    const float2 e = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
    const float2 o = make_float2(0.5f * (zk.y + zm.y), -0.5f * (zk.x - zm.x));
    spec[(row0 + r) * nhp + k] = cadd(e, cmul(twiddle(s_tw, k, NM, false), o));
  }
}

// Half spectra (pitch nhp) of ncomp components -> real rows: the merge
// above, the inverse half-length transform, real / imaginary parts as the
// even / odd samples.
template <int LOGH>
__global__ void __launch_bounds__(RowPass<LOGH>::THREADS) k_row_c2r(const float2* __restrict__ spec3,
                                                                   float* __restrict__ force, int nhp,
                                                                   int64_t nrows, const float2* __restrict__ tw,
                                                                   uint32_t* __restrict__ err) {
  using RP = RowPass<LOGH>;
  using S = typename RP::S;
  constexpr int H = RP::H, N1 = S::N1, N2 = S::N2, R = S::R, RX = RP::RX, NM = 2 * H;
  extern __shared__ __align__(128) unsigned char rsm[];
  float2* rows = reinterpret_cast<float2*>(rsm);  // RX x nhp (input spectra)
  float2* ybuf = rows + (size_t)RX * nhp;         // RX x YP
  float2* s_tw = ybuf + RX * RP::YP;
  uint64_t* bar = reinterpret_cast<uint64_t*>(s_tw + NM / 2);
  for (int i = threadIdx.x; i < NM / 2; i += blockDim.x) s_tw[i] = tw[i];
  const int comp = blockIdx.y;
  const float2* in = spec3 + (int64_t)comp * nrows * nhp;
  float2* out_rows = reinterpret_cast<float2*>(force + (int64_t)comp * nrows * NM);
  const int64_t row0 = (int64_t)blockIdx.x * RX;
  const int nr = (int)min((int64_t)RX, nrows - row0);
  if (!stage_bulk(rows, in + row0 * nhp, (uint32_t)(nr * nhp * sizeof(float2)), bar, err)) return;
  const int rr = threadIdx.x / N2, t = threadIdx.x % N2;
  const float2* X = rows + (size_t)rr * nhp;
  // Z[k] = X[k] (1 + i W) + conj(X[h - k]) (1 - i W), W = w_NM^-k; Im X[0], Im X[h] drop out
  auto zin = [&](int k) {
    float2 xk = X[k], xm = X[H - k];
    if (k == 0) xk.y = xm.y = 0.f;
    const float2 w = twiddle(s_tw, k, NM, true);
    const float2 p = make_float2(1.f - w.y, w.x), q = make_float2(1.f + w.y, -w.x);
    return cadd(cmul(xk, p), cmul(make_float2(xm.x, -xm.y), q));
  };
  float2 v[N1];
#pragma unroll
  for (int j1 = 0; j1 < N1; ++j1) v[j1] = rr < nr ? zin(N2 * j1 + t) : make_float2(0.f, 0.f);
  fftr::dft<N1, true>(v);
#pragma unroll
  for (int k1 = 1; k1 < N1; ++k1) v[k1] = cmul(v[k1], twiddle(s_tw, 2 * ((t * k1) & (H - 1)), NM, true));
  float2* yb = ybuf + rr * RP::YP;
#pragma unroll
  for (int k1 = 0; k1 < N1; ++k1) yb[k1 + t * (N1 + 1)] = v[k1];
  __syncthreads();
  float2 o[R][N2];
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const int k1 = t + N2 * r;
#pragma unroll
    for (int j2 = 0; j2 < N2; ++j2) o[r][j2] = yb[k1 + j2 * (N1 + 1)];
    fftr::dft<N2, true>(o[r]);
  }
  if (rr < nr) {
#pragma unroll
    for (int r = 0; r < R; ++r)
#pragma unroll
      for (int k2 = 0; k2 < N2; ++k2) out_rows[(row0 + rr) * H + (t + N2 * r) + N1 * k2] = o[r][k2];
  }
}

template <int LOGH> constexpr size_t row_smem(int cols) {
  return ((size_t)RowPass<LOGH>::RX * cols + (size_t)RowPass<LOGH>::RX * RowPass<LOGH>::YP + RowPass<LOGH>::H) *
             sizeof(float2) + 16;
}

// ---- gather (cic.rs:100-170) fused with the sum LR + SR and the kick -------------
__global__ void k_gather_kick(GatherArgs a, const float* __restrict__ fx, const float* __restrict__ fy,
                              const float* __restrict__ fz, double scale, double inv_cell, int nm) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= a.n) return;
  const Cic c = cic_of(a.qx[i], a.qy[i], a.qz[i], scale, inv_cell, nm);
  const int64_t nm2 = (int64_t)nm * nm;
  float lx = 0.f, ly = 0.f, lz = 0.f;
#pragma unroll
  for (int u = 0; u < 2; ++u)
#pragma unroll
    for (int v = 0; v < 2; ++v)
#pragma unroll
      for (int w = 0; w < 2; ++w) {
        const float wt = c.wx[w] * c.wy[v] * c.wz[u];
        const int64_t idx = c.iz[u] * nm2 + (int64_t)c.iy[v] * nm + c.ix[w];
        lx = fmaf(fx[idx], wt, lx);
        ly = fmaf(fy[idx], wt, ly);
        lz = fmaf(fz[idx], wt, lz);
      }
  const float g = (float)a.g;
  float sx = 0.f, sy = 0.f, sz = 0.f;
  if (a.srx) {
    sx = a.srx[i];
    sy = a.sry[i];
    sz = a.srz[i];
  }
  const float tx = g * (lx + sx), ty = g * (ly + sy), tz = g * (lz + sz);
  a.ax[i] = tx;
  a.ay[i] = ty;
  a.az[i] = tz;
  if (a.lrx) {
    a.lrx[i] = g * lx;
    a.lry[i] = g * ly;
    a.lrz[i] = g * lz;
  }
  if (a.vx) {
    const float k = (float)a.kick;
    a.vx[i] = fmaf(tx, k, a.vx[i]);
    a.vy[i] = fmaf(ty, k, a.vy[i]);
    a.vz[i] = fmaf(tz, k, a.vz[i]);
  }
}

inline int ilog2(int n) {
  int l = 0;
  while ((1 << l) < n) ++l;
  return l;
}
// rows of one x-pass block: 4096 complex values, never more than the mesh has
// ---- power spectrum (crates/gadget-ng-analysis/src/power_spectrum.rs) --------------
// CIC assignment of power_spectrum.rs:146-166: fx = x / cell, floor, weights
// (1 - t, t), indices rem_euclid(n), m * wx * wy * wz; stored z-major like the
// PM mesh (the binned spectrum does not depend on the axis order).
// CIC cells and weights of power_spectrum.rs:146-166 (float64, division by
// the cell size), the eight corners in (dx, dy, dz) order.
__device__ __forceinline__ void pk_cic(double x, double y, double z, double m, double cell, int nm, int64_t idx[8],
                                       float w[8]) {
  const double f[3] = {ddiv(x, cell), ddiv(y, cell), ddiv(z, cell)};
  int i0[3];
  double t[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double fl = floor(f[d]);
    i0[d] = (int)fl;
    t[d] = dsub(f[d], fl);
  }
  const int msk = nm - 1;  // nm is a power of two: & wraps negative indices too (rem_euclid)
#pragma unroll
  for (int dx = 0; dx < 2; ++dx)
#pragma unroll
    for (int dy = 0; dy < 2; ++dy)
#pragma unroll
      for (int dz = 0; dz < 2; ++dz) {
        const double wx = dx ? t[0] : dsub(1.0, t[0]), wy = dy ? t[1] : dsub(1.0, t[1]);
        const double wz = dz ? t[2] : dsub(1.0, t[2]);
        const int jx = (i0[0] + dx) & msk, jy = (i0[1] + dy) & msk, jz = (i0[2] + dz) & msk;
        const int k = dx * 4 + dy * 2 + dz;
        idx[k] = ((int64_t)jz * nm + jy) * nm + jx;
        w[k] = (float)dmul(dmul(dmul(m, wx), wy), wz);
      }
}

// Add the eight corner weights of each live lane; lanes whose particles share
// a base cell sum their weights in registers first (warp match), so one lane
// per cell issues the eight atomics.
__device__ __forceinline__ void pk_add_aggregated(bool live, const int64_t idx[8], const float w[8], float* rho) {
  const int lane = threadIdx.x & 31;
  const uint32_t key = live ? (uint32_t)idx[0] : 0xFFFFFFFFu;
  const uint32_t peers = __match_any_sync(0xffffffffu, key);
  const int rounds = __reduce_max_sync(0xffffffffu, (unsigned)__popc(peers));
  if (rounds == 1) {
    if (!live) return;
#pragma unroll
    for (int k = 0; k < 8; ++k) atomicAdd(&rho[idx[k]], w[k]);
    return;
  }
  float sum[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) sum[k] = 0.f;
  uint32_t rest = peers;
  for (int r = 0; r < rounds; ++r) {  // the same count on every lane: full-warp shuffles
    const int src = rest ? __ffs(rest) - 1 : lane;
    const bool take = rest != 0u;
    rest &= rest - 1u;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const float v = __shfl_sync(0xffffffffu, w[k], src);
      if (take) sum[k] += v;
    }
  }
  if (!live || lane != __ffs(peers) - 1) return;
#pragma unroll
  for (int k = 0; k < 8; ++k) atomicAdd(&rho[idx[k]], sum[k]);
}

__global__ void k_pk_deposit_pos(const double* __restrict__ pos, const double* __restrict__ m, int64_t n,
                                 double cell, int nm, float* __restrict__ rho) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const bool live = i < n;
  int64_t idx[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  float w[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  if (live) pk_cic(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2], m[i], cell, nm, idx, w);
  pk_add_aggregated(live, idx, w, rho);
}

__global__ void k_pk_deposit_q(const uint32_t* __restrict__ qx, const uint32_t* __restrict__ qy,
                               const uint32_t* __restrict__ qz, const double* __restrict__ m, int64_t n,
                               double scale, double cell, int nm, float* __restrict__ rho) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const bool live = i < n;
  int64_t idx[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  float w[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
  if (live) pk_cic(decode(qx[i], scale), decode(qy[i], scale), decode(qz[i], scale), m[i], cell, nm, idx, w);
  pk_add_aggregated(live, idx, w, rho);
}

// ---- pencil launches, one instantiation per transform length (4 .. 1024) ------------
enum PencilOp { PEN_Y_FWD, PEN_Y_INV, PEN_Z_FWD, PEN_Z_INV, PEN_POISSON, PEN_PK };

template <int LOGN>
void pencil_launch_t(const PmPlan& p, PencilOp op, int ncomp, double* pk_sum, unsigned long long* pk_n,
                     cudaStream_t s) {
  using P = Pencil<LOGN>;
  const int nm = p.nm, ntx = (p.nh + P::CTX - 1) / P::CTX;
  const CUtensorMap* spec_y = reinterpret_cast<const CUtensorMap*>(p.tmap[0]);
  const CUtensorMap* spec_z = reinterpret_cast<const CUtensorMap*>(p.tmap[1]);
  const CUtensorMap* spec3_y = reinterpret_cast<const CUtensorMap*>(p.tmap[2]);
  const CUtensorMap* spec3_z = reinterpret_cast<const CUtensorMap*>(p.tmap[3]);
  const size_t sm1 = pencil_smem<LOGN>(1), sm2 = pencil_smem<LOGN>(2);
  switch (op) {
    case PEN_Y_FWD:
    case PEN_Z_FWD: {
      auto k = k_pencil<LOGN, false>;
      TPM_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm1));
      k<<<dim3(ntx, nm, 1), P::THREADS, sm1, s>>>(op == PEN_Y_FWD ? *spec_y : *spec_z, p.spec,
                                                  op == PEN_Y_FWD ? 0 : 1, p.nh, p.nhp, nm, nm, p.twiddle, p.err);
      break;
    }
    case PEN_Y_INV:
    case PEN_Z_INV: {
      auto k = k_pencil<LOGN, true>;
      TPM_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm1));
      k<<<dim3(ntx, nm, ncomp), P::THREADS, sm1, s>>>(op == PEN_Y_INV ? *spec3_y : *spec3_z, p.spec3,
                                                      op == PEN_Y_INV ? 0 : 1, p.nh, p.nhp, nm, nm, p.twiddle,
                                                      p.err);
      break;
    }
    case PEN_POISSON: {
      auto k = k_pencil_poisson<LOGN>;
      TPM_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm2));
      k<<<dim3(ntx, nm), P::THREADS, sm2, s>>>(*spec_z, p.spec3, p.nh, p.nhp, nm, 0, p.twiddle, p.kval,
                                               p.kfilter, p.kderiv, p.kcoef, p.ncomp, p.err);
      break;
    }
    case PEN_PK: {
      auto k = k_pencil_pk<LOGN>;
      const size_t smk = sm1 + (sizeof(double) + sizeof(unsigned long long)) * (size_t)(nm / 2);
      TPM_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smk));
      k<<<dim3(ntx, nm), P::THREADS, smk, s>>>(*spec_z, p.nh, p.twiddle, pk_sum, pk_n, p.err);
      break;
    }
  }
  TPM_LAUNCH_CHECK();
}

void pencil_launch(const PmPlan& p, PencilOp op, int ncomp = 1, double* pk_sum = nullptr,
                   unsigned long long* pk_n = nullptr, cudaStream_t s = 0) {
  switch (p.logn) {
    case 2: pencil_launch_t<2>(p, op, ncomp, pk_sum, pk_n, s); break;
    case 3: pencil_launch_t<3>(p, op, ncomp, pk_sum, pk_n, s); break;
    case 4: pencil_launch_t<4>(p, op, ncomp, pk_sum, pk_n, s); break;
    case 5: pencil_launch_t<5>(p, op, ncomp, pk_sum, pk_n, s); break;
    case 6: pencil_launch_t<6>(p, op, ncomp, pk_sum, pk_n, s); break;
    case 7: pencil_launch_t<7>(p, op, ncomp, pk_sum, pk_n, s); break;
    case 8: pencil_launch_t<8>(p, op, ncomp, pk_sum, pk_n, s); break;
    case 9: pencil_launch_t<9>(p, op, ncomp, pk_sum, pk_n, s); break;
    case 10: pencil_launch_t<10>(p, op, ncomp, pk_sum, pk_n, s); break;
    default: throw Error(TPM_ERR_INVALID_ARGUMENT, "mesh size outside 4..1024");
  }
}

// ---- slab pencil launches ------------------------------------------------------------
template <int LOGN>
void slab_pencil_t(const PmPlan& p, const PmSlab& sl, int op, cudaStream_t s) {
  using P = Pencil<LOGN>;
  const int nm = p.nm, ntx = (p.nh + P::CTX - 1) / P::CTX;
  const size_t sm1 = pencil_smem<LOGN>(1), sm2 = pencil_smem<LOGN>(2);
  if (op == 0) {  // forward y on this rank's planes
    auto k = k_pencil<LOGN, false>;
    TPM_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm1));
    k<<<dim3(ntx, sl.nzl, 1), P::THREADS, sm1, s>>>(*reinterpret_cast<const CUtensorMap*>(sl.tmap[0]), sl.spec, 0,
                                                    p.nh, p.nhp, nm, sl.nzl, p.twiddle, p.err);
  } else if (op == 1) {  // z passes + Poisson on the received y rows
    auto k = k_pencil_poisson<LOGN>;
    TPM_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm2));
    k<<<dim3(ntx, sl.nyl), P::THREADS, sm2, s>>>(*reinterpret_cast<const CUtensorMap*>(sl.tmap[2]), sl.t3, p.nh,
                                                 p.nhp, sl.nyl, sl.rank * sl.nyl, p.twiddle, p.kval, p.kfilter,
                                                 p.kderiv, p.kcoef, sl.ncomp, p.err);
  } else {  // inverse y of the force spectra of this rank's planes
    auto k = k_pencil<LOGN, true>;
    TPM_CUDA(cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm1));
    k<<<dim3(ntx, sl.nzl, sl.ncomp), P::THREADS, sm1, s>>>(*reinterpret_cast<const CUtensorMap*>(sl.tmap[1]),
                                                           sl.spec3, 0, p.nh, p.nhp, nm, sl.nzl, p.twiddle, p.err);
  }
  TPM_LAUNCH_CHECK();
}

void slab_pencil(const PmPlan& p, const PmSlab& sl, int op, cudaStream_t s) {
  switch (p.logn) {
    case 2: slab_pencil_t<2>(p, sl, op, s); break;
    case 3: slab_pencil_t<3>(p, sl, op, s); break;
    case 4: slab_pencil_t<4>(p, sl, op, s); break;
    case 5: slab_pencil_t<5>(p, sl, op, s); break;
    case 6: slab_pencil_t<6>(p, sl, op, s); break;
    case 7: slab_pencil_t<7>(p, sl, op, s); break;
    case 8: slab_pencil_t<8>(p, sl, op, s); break;
    case 9: slab_pencil_t<9>(p, sl, op, s); break;
    case 10: slab_pencil_t<10>(p, sl, op, s); break;
    default: throw Error(TPM_ERR_INVALID_ARGUMENT, "mesh size outside 4..1024");
  }
}

// ---- x-pass launches (rows of h = nm/2 packed complex values) ---------------------
// nrows rows of the real meshes `real` and spectra `spec` (per component:
// nrows rows each).
template <int LOGH>
void row_launch_t(const PmPlan& p, bool forward, float* real, float2* spec, int64_t nrows, int ncomp,
                  cudaStream_t s) {
  using RP = RowPass<LOGH>;
  const unsigned blocks = (unsigned)((nrows + RP::RX - 1) / RP::RX);
  if (forward) {
    const size_t sm = row_smem<LOGH>(RP::H);
    TPM_CUDA(cudaFuncSetAttribute(k_row_r2c<LOGH>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    k_row_r2c<LOGH><<<blocks, RP::THREADS, sm, s>>>(real, spec, p.nhp, nrows, p.twiddle, p.err);
  } else {
    const size_t sm = row_smem<LOGH>(p.nhp);
    TPM_CUDA(cudaFuncSetAttribute(k_row_c2r<LOGH>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
    k_row_c2r<LOGH><<<dim3(blocks, ncomp), RP::THREADS, sm, s>>>(spec, real, p.nhp, nrows, p.twiddle, p.err);
  }
  TPM_LAUNCH_CHECK();
}

void row_launch(const PmPlan& p, bool forward, float* real, float2* spec, int64_t nrows, int ncomp, cudaStream_t s) {
  switch (p.logn - 1) {
    case 1: row_launch_t<1>(p, forward, real, spec, nrows, ncomp, s); break;
    case 2: row_launch_t<2>(p, forward, real, spec, nrows, ncomp, s); break;
    case 3: row_launch_t<3>(p, forward, real, spec, nrows, ncomp, s); break;
    case 4: row_launch_t<4>(p, forward, real, spec, nrows, ncomp, s); break;
    case 5: row_launch_t<5>(p, forward, real, spec, nrows, ncomp, s); break;
    case 6: row_launch_t<6>(p, forward, real, spec, nrows, ncomp, s); break;
    case 7: row_launch_t<7>(p, forward, real, spec, nrows, ncomp, s); break;
    case 8: row_launch_t<8>(p, forward, real, spec, nrows, ncomp, s); break;
    case 9: row_launch_t<9>(p, forward, real, spec, nrows, ncomp, s); break;
    default: throw Error(TPM_ERR_INVALID_ARGUMENT, "mesh size outside 4..1024");
  }
}
void row_launch(const PmPlan& p, bool forward, int ncomp, cudaStream_t s) {
  row_launch(p, forward, forward ? p.rho : p.force, forward ? p.spec : p.spec3, (int64_t)p.nm * p.nm, ncomp, s);
}

// cuTensorMapEncodeTiled from the driver, looked up once (no libcuda link).
PFN_cuTensorMapEncodeTiled_v12000 encode_tiled() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    TPM_CUDA(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q));
    if (q != cudaDriverEntryPointSuccess || !f) throw Error(TPM_ERR_CUDA, "cuTensorMapEncodeTiled is unavailable");
    fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
  }
  return fn;
}

// Tensor map of half spectra [plane][y][kx] (8-byte complex elements, rows of
// nhp, ny rows per plane, `planes` planes over all components): box of ctx
// columns by `rows_y` y rows by `rows_z` planes.
void encode_spectrum_map(void* out, float2* base, int ny, int nhp, int64_t planes, int ctx, int rows_y, int rows_z) {
  CUtensorMap* m = reinterpret_cast<CUtensorMap*>(out);
  const cuuint64_t dims[3] = {(cuuint64_t)nhp, (cuuint64_t)ny, (cuuint64_t)planes};
  const cuuint64_t strides[2] = {(cuuint64_t)nhp * sizeof(float2), (cuuint64_t)nhp * sizeof(float2) * (cuuint64_t)ny};
  const cuuint32_t box[3] = {(cuuint32_t)ctx, (cuuint32_t)rows_y, (cuuint32_t)rows_z};
  const cuuint32_t estr[3] = {1, 1, 1};
  const CUresult r = encode_tiled()(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3, base, dims, strides, box, estr,
                                    CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                                    CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) throw Error(TPM_ERR_CUDA, "cuTensorMapEncodeTiled failed: " + std::to_string((int)r));
}

}  // namespace

void pm_plan_init(PmPlan& p, int nm, double box, double r_split, uint32_t flags, int device) {
  (void)device;
  p.nm = nm;
  p.logn = ilog2(nm);
  p.nh = nm / 2 + 1;
  p.nhp = (p.nh + 1) & ~1;  // even: 16-byte rows
  p.box = box;
  const int64_t nm3 = (int64_t)nm * nm * nm;
  const int64_t nspec = (int64_t)nm * nm * p.nhp;
  std::vector<float2> tw(nm / 2);
  for (int m = 0; m < nm / 2; ++m) {
    const double ang = -2.0 * M_PI * (double)m / (double)nm;
    tw[m] = make_float2((float)std::cos(ang), (float)std::sin(ang));
  }
  // float64 tables: k = 2 pi n / L with n = freq_index (fft_poisson.rs:724-730)
  const double dk = 2.0 * M_PI / box, cell = box / nm;
  std::vector<float> kval(nm), kfil(nm), kder(nm);
  for (int i = 0; i < nm; ++i) {
    const int64_t f = i <= nm / 2 ? i : (int64_t)i - nm;
    const double k = dk * (double)f;
    kval[i] = (float)k;
    double fil = 1.0;
    if (r_split > 0.0) fil *= std::exp(-0.5 * k * k * r_split * r_split);  // per-axis factor of exp(-k^2 r_s^2 / 2)
    if (flags & 2u) {  // CIC deconvolution: divide by W_cic^2 = prod sinc^4
      const double h = 0.5 * k * cell;
      const double sn = i == 0 ? 1.0 : std::sin(h) / h;
      fil /= (sn * sn) * (sn * sn);
    }
    kfil[i] = (float)fil;
    double d = k;
    if (flags & 4u) d = (8.0 * std::sin(k * cell) - std::sin(2.0 * k * cell)) / (6.0 * cell);
    if (i == nm / 2) d = 0.0;  // the real part of the reference's c2c inverse drops it
    kder[i] = (float)d;
  }
  const double vcell = cell * (cell * cell);
  p.kcoef = (float)(-4.0 * M_PI / vcell / (double)nm3);
  TPM_CUDA(cudaMalloc(&p.twiddle, sizeof(float2) * (nm / 2)));
  TPM_CUDA(cudaMalloc(&p.kval, sizeof(float) * nm));
  TPM_CUDA(cudaMalloc(&p.kfilter, sizeof(float) * nm));
  TPM_CUDA(cudaMalloc(&p.kderiv, sizeof(float) * nm));
  TPM_CUDA(cudaMalloc(&p.rho, sizeof(float) * nm3));
  TPM_CUDA(cudaMalloc(&p.spec, sizeof(float2) * nspec));
  p.ncomp = (flags & (1u << 6)) ? 4 : 3;
  TPM_CUDA(cudaMalloc(&p.spec3, sizeof(float2) * nspec * p.ncomp));
  TPM_CUDA(cudaMalloc(&p.force, sizeof(float) * nm3 * p.ncomp));
  TPM_CUDA(cudaMemcpy(p.twiddle, tw.data(), sizeof(float2) * (nm / 2), cudaMemcpyHostToDevice));
  TPM_CUDA(cudaMemcpy(p.kval, kval.data(), sizeof(float) * nm, cudaMemcpyHostToDevice));
  TPM_CUDA(cudaMemcpy(p.kfilter, kfil.data(), sizeof(float) * nm, cudaMemcpyHostToDevice));
  TPM_CUDA(cudaMemcpy(p.kderiv, kder.data(), sizeof(float) * nm, cudaMemcpyHostToDevice));
  // the padding column (kx = nh) is never written: zero it once
  TPM_CUDA(cudaMemset(p.spec, 0, sizeof(float2) * nspec));
  TPM_CUDA(cudaMemset(p.spec3, 0, sizeof(float2) * nspec * p.ncomp));
  TPM_CUDA(cudaMalloc(&p.err, sizeof(uint32_t)));
  TPM_CUDA(cudaMemset(p.err, 0, sizeof(uint32_t)));
  // pencil tiles: ctx columns by min(nm, 256) rows along y or z
  const int ctx = nm > 512 ? 8 : 16, rows = nm < 256 ? nm : 256;
  encode_spectrum_map(p.tmap[0], p.spec, nm, p.nhp, nm, ctx, rows, 1);
  encode_spectrum_map(p.tmap[1], p.spec, nm, p.nhp, nm, ctx, 1, rows);
  encode_spectrum_map(p.tmap[2], p.spec3, nm, p.nhp, (int64_t)nm * p.ncomp, ctx, rows, 1);
  encode_spectrum_map(p.tmap[3], p.spec3, nm, p.nhp, (int64_t)nm * p.ncomp, ctx, 1, rows);
}

void pm_check(const PmPlan& p, cudaStream_t s) {
  uint32_t e = 0;
  TPM_CUDA(cudaMemcpyAsync(&e, p.err, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
  TPM_CUDA(cudaStreamSynchronize(s));
  if (!e) return;
  TPM_CUDA(cudaMemsetAsync(p.err, 0, sizeof(uint32_t), s));
  throw Error(TPM_ERR_CUDA, "a transform pass's bulk tensor copy did not complete within its time limit");
}

void pm_plan_free(PmPlan& p) {
  cudaFree(p.twiddle);
  cudaFree(p.kval);
  cudaFree(p.kfilter);
  cudaFree(p.kderiv);
  cudaFree(p.rho);
  cudaFree(p.spec);
  cudaFree(p.spec3);
  cudaFree(p.force);
  cudaFree(p.err);
  p = PmPlan();
}

void pm_deposit(const PmPlan& p, const uint32_t* qx, const uint32_t* qy, const uint32_t* qz, const float* massf,
                int64_t n, cudaStream_t s, const uint32_t* id, uint32_t id_limit) {
  const int64_t nm3 = (int64_t)p.nm * p.nm * p.nm;
  TPM_CUDA(cudaMemsetAsync(p.rho, 0, sizeof(float) * nm3, s));
  if (n == 0) return;
  k_deposit<<<grid_for(n, DEP_THREADS, 1ll << 30), DEP_THREADS, 0, s>>>(qx, qy, qz, massf, n, p.box / TWO32, (double)p.nm / p.box,
                                                        p.nm, p.rho, id, id_limit);
  TPM_LAUNCH_CHECK();
}

void pm_solve(const PmPlan& p, cudaStream_t s) {
  row_launch(p, true, 1, s);
  pencil_launch(p, PEN_Y_FWD, 1, nullptr, nullptr, s);
  pencil_launch(p, PEN_POISSON, p.ncomp, nullptr, nullptr, s);
  pencil_launch(p, PEN_Y_INV, p.ncomp, nullptr, nullptr, s);
  row_launch(p, false, p.ncomp, s);
}

void pm_gather_kick(const PmPlan& p, const GatherArgs& a, cudaStream_t s) {
  if (a.n == 0) return;
  const int64_t nm3 = (int64_t)p.nm * p.nm * p.nm;
  k_gather_kick<<<grid_for(a.n, 256, 1ll << 30), 256, 0, s>>>(a, p.force, p.force + nm3, p.force + 2 * nm3,
                                                              p.box / TWO32, (double)p.nm / p.box, p.nm);
  TPM_LAUNCH_CHECK();
}

void pm_cells(const PmPlan& p, const uint32_t* qx, const uint32_t* qy, const uint32_t* qz, const uint32_t* id,
              int64_t n, int32_t* cells_by_id, cudaStream_t s) {
  if (n == 0) return;
  k_cells<<<grid_for(n, 256, 1ll << 30), 256, 0, s>>>(qx, qy, qz, id, n, p.box / TWO32, (double)p.nm / p.box, p.nm,
                                                      cells_by_id);
  TPM_LAUNCH_CHECK();
}

void pm_forward_real(const PmPlan& p, cudaStream_t s) {
  row_launch(p, true, 1, s);
  pencil_launch(p, PEN_Y_FWD, 1, nullptr, nullptr, s);
  pencil_launch(p, PEN_Z_FWD, 1, nullptr, nullptr, s);
}

void pm_inverse_components(const PmPlan& p, int ncomp, cudaStream_t s) {
  pencil_launch(p, PEN_Z_INV, ncomp, nullptr, nullptr, s);
  pencil_launch(p, PEN_Y_INV, ncomp, nullptr, nullptr, s);
  row_launch(p, false, ncomp, s);
}

void pm_power_spectrum(const PmPlan& p, const double* pos, const uint32_t* qx, const uint32_t* qy,
                       const uint32_t* qz, const double* mass, int64_t n, double total_mass, double* pk_sum,
                       unsigned long long* pk_n, double* k_out, double* pk_out, unsigned long long* n_out,
                       cudaStream_t s) {
  const int nm = p.nm, nb = nm / 2;
  const int64_t nm3 = (int64_t)nm * nm * nm;
  const double cell = p.box / nm;
  TPM_CUDA(cudaMemsetAsync(p.rho, 0, sizeof(float) * nm3, s));
  TPM_CUDA(cudaMemsetAsync(pk_sum, 0, sizeof(double) * nb, s));
  TPM_CUDA(cudaMemsetAsync(pk_n, 0, sizeof(unsigned long long) * nb, s));
  if (n > 0) {
    if (pos)
      k_pk_deposit_pos<<<grid_for(n, 256, 1ll << 30), 256, 0, s>>>(pos, mass, n, cell, nm, p.rho);
    else
      k_pk_deposit_q<<<grid_for(n, 256, 1ll << 30), 256, 0, s>>>(qx, qy, qz, mass, n, p.box / TWO32, cell, nm,
                                                                 p.rho);
    TPM_LAUNCH_CHECK();
  }
  row_launch(p, true, 1, s);
  pencil_launch(p, PEN_Y_FWD, 1, nullptr, nullptr, s);
  pencil_launch(p, PEN_PK, 1, pk_sum, pk_n, s);
  std::vector<double> hs((size_t)nb);
  std::vector<unsigned long long> hn((size_t)nb);
  TPM_CUDA(cudaMemcpyAsync(hs.data(), pk_sum, sizeof(double) * nb, cudaMemcpyDeviceToHost, s));
  TPM_CUDA(cudaMemcpyAsync(hn.data(), pk_n, sizeof(unsigned long long) * nb, cudaMemcpyDeviceToHost, s));
  TPM_CUDA(cudaStreamSynchronize(s));
  // delta_k = rho_k / (mean_rho V_cell) = rho_k nm^3 / M for k != 0; norm (V / nm^3)^2
  const double vol = p.box * p.box * p.box;
  const double scale = (double)nm3 / total_mass, norm = (vol / (double)nm3) * (vol / (double)nm3);
  for (int i = 0; i < nb; ++i) {
    k_out[i] = (i + 1.0) * 2.0 * M_PI / p.box;
    n_out[i] = hn[i];
    pk_out[i] = hn[i] ? hs[i] * scale * scale * norm / (double)hn[i] : 0.0;
  }
}

// ---- z-slab decomposition ---------------------------------------------------------
void pm_slab_init(PmSlab& sl, const PmPlan& p, int rank, int ranks) {
  const int nm = p.nm;
  if (ranks < 1 || rank < 0 || rank >= ranks || nm % ranks != 0)
    throw Error(TPM_ERR_INVALID_ARGUMENT, "pm_grid_size must be a multiple of the rank count");
  pm_slab_free(sl);
  sl.rank = rank;
  sl.ranks = ranks;
  sl.nzl = nm / ranks;
  sl.nyl = nm / ranks;
  sl.ncomp = 3;
  const int64_t nhp = p.nhp, nm2 = (int64_t)nm * nm;
  const int64_t slab_spec = (int64_t)sl.nzl * nm * nhp, ycols = (int64_t)nm * sl.nyl * nhp;
  TPM_CUDA(cudaMalloc(&sl.rho, sizeof(float) * sl.nzl * nm2));
  TPM_CUDA(cudaMalloc(&sl.spec, sizeof(float2) * slab_spec));
  TPM_CUDA(cudaMalloc(&sl.send, sizeof(float2) * ycols * sl.ncomp));
  TPM_CUDA(cudaMalloc(&sl.recv, sizeof(float2) * ycols * sl.ncomp));
  TPM_CUDA(cudaMalloc(&sl.t3, sizeof(float2) * ycols * sl.ncomp));
  TPM_CUDA(cudaMalloc(&sl.spec3, sizeof(float2) * slab_spec * sl.ncomp));
  TPM_CUDA(cudaMalloc(&sl.force, sizeof(float) * sl.nzl * nm2 * sl.ncomp));
  // padding columns (kx = nh) are never written
  TPM_CUDA(cudaMemset(sl.spec, 0, sizeof(float2) * slab_spec));
  TPM_CUDA(cudaMemset(sl.send, 0, sizeof(float2) * ycols * sl.ncomp));
  TPM_CUDA(cudaMemset(sl.recv, 0, sizeof(float2) * ycols * sl.ncomp));
  TPM_CUDA(cudaMemset(sl.t3, 0, sizeof(float2) * ycols * sl.ncomp));
  TPM_CUDA(cudaMemset(sl.spec3, 0, sizeof(float2) * slab_spec * sl.ncomp));
  sl.send_bytes = sizeof(float2) * (size_t)slab_spec;  // the forward transpose; the return one sends ncomp times as much
  const int ctx = nm > 512 ? 8 : 16, rows = nm < 256 ? nm : 256;
  encode_spectrum_map(sl.tmap[0], sl.spec, nm, p.nhp, sl.nzl, ctx, rows, 1);
  encode_spectrum_map(sl.tmap[1], sl.spec3, nm, p.nhp, (int64_t)sl.nzl * sl.ncomp, ctx, rows, 1);
  encode_spectrum_map(sl.tmap[2], sl.recv, sl.nyl, p.nhp, nm, ctx, 1, rows);
}

void pm_slab_free(PmSlab& sl) {
  cudaFree(sl.rho);
  cudaFree(sl.spec);
  cudaFree(sl.send);
  cudaFree(sl.recv);
  cudaFree(sl.t3);
  cudaFree(sl.spec3);
  cudaFree(sl.force);
  sl = PmSlab();
}

void pm_slab_forward(const PmPlan& p, const PmSlab& sl, cudaStream_t s) {
  const int nm = p.nm;
  const int64_t nhp = p.nhp;
  row_launch(p, true, sl.rho, sl.spec, (int64_t)sl.nzl * nm, 1, s);
  slab_pencil(p, sl, 0, s);
  // send[dest][zl][yl][kx] = spec[zl][dest nyl + yl][kx]
  const size_t w = sizeof(float2) * (size_t)sl.nyl * nhp;
  for (int d = 0; d < sl.ranks; ++d)
    TPM_CUDA(cudaMemcpy2DAsync(sl.send + (int64_t)d * sl.nzl * sl.nyl * nhp, w, sl.spec + (int64_t)d * sl.nyl * nhp,
                               sizeof(float2) * (size_t)nm * nhp, w, sl.nzl, cudaMemcpyDeviceToDevice, s));
}

void pm_slab_poisson(const PmPlan& p, const PmSlab& sl, cudaStream_t s) {
  // recv is [src][zl][yl][kx] = [z][yl][kx]: every z of this rank's y rows
  slab_pencil(p, sl, 1, s);
  // send[dest][comp][zl][yl][kx] = t3[comp][dest nzl + zl][yl][kx]
  const int64_t blk = (int64_t)sl.nzl * sl.nyl * p.nhp;
  for (int d = 0; d < sl.ranks; ++d)
    for (int c = 0; c < sl.ncomp; ++c)
      TPM_CUDA(cudaMemcpyAsync(sl.send + ((int64_t)d * sl.ncomp + c) * blk,
                               sl.t3 + (int64_t)c * p.nm * sl.nyl * p.nhp + (int64_t)d * blk, sizeof(float2) * blk,
                               cudaMemcpyDeviceToDevice, s));
}

void pm_slab_inverse(const PmPlan& p, const PmSlab& sl, cudaStream_t s) {
  const int nm = p.nm;
  const int64_t nhp = p.nhp, blk = (int64_t)sl.nzl * sl.nyl * nhp;
  // spec3[comp][zl][src nyl + yl][kx] = recv[src][comp][zl][yl][kx]
  const size_t w = sizeof(float2) * (size_t)sl.nyl * nhp;
  for (int r = 0; r < sl.ranks; ++r)
    for (int c = 0; c < sl.ncomp; ++c)
      TPM_CUDA(cudaMemcpy2DAsync(sl.spec3 + (int64_t)c * sl.nzl * nm * nhp + (int64_t)r * sl.nyl * nhp,
                                 sizeof(float2) * (size_t)nm * nhp, sl.recv + ((int64_t)r * sl.ncomp + c) * blk, w, w,
                                 sl.nzl, cudaMemcpyDeviceToDevice, s));
  slab_pencil(p, sl, 2, s);
  row_launch(p, false, sl.force, sl.spec3, (int64_t)sl.nzl * nm, sl.ncomp, s);
}

}  // namespace tpm
