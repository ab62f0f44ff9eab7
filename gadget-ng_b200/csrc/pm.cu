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
// transform is a radix-2 Stockham autosort FFT in shared memory.  Linear in G:
// the meshes hold forces per unit G, the gather multiplies by g.
#include <cmath>
#include <vector>

#include "common.cuh"
#include "pm.cuh"

namespace tpm {
namespace {

__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }

// Batched Stockham FFT in shared memory.  ROWMAJOR: element (j, c) at
// a[c * n + j]; otherwise at a[j * cols + c].  Returns the buffer holding the
// result (a or b).
template <bool ROWMAJOR>
__device__ __forceinline__ int fft_addr(int c, int j, int n, int cols) {
  return ROWMAJOR ? c * n + j : j * cols + c;
}

// Twiddle exp(-+2 pi i m / n) from the half table tw[m] = exp(-2 pi i m / n), m < n/2.
__device__ __forceinline__ float2 twiddle(const float2* tw, int m, int n, bool inv) {
  const int half = n >> 1;
  float2 w = m < half ? tw[m] : make_float2(-tw[m - half].x, -tw[m - half].y);
  if (inv) w.y = -w.y;
  return w;
}

// Stockham radix-4 passes (one radix-2 pass last when log2 n is odd): each
// pass reads a, writes b, then swaps; between passes only shared memory and
// one barrier.  Pass with Ns outputs done so far: element j of a column,
// k = j mod Ns, inputs a[j + i n/4] twiddled by w^(i k) with w = exp(-2 pi i /
// (4 Ns)), a 4-point DFT, outputs b[(j / Ns) 4 Ns + k + i Ns].  cols is a
// power of two (log2 = lcols).
template <bool ROWMAJOR>
__device__ float2* fft_smem(float2* a, float2* b, int n, int logn, int cols, const float2* tw, bool inv) {
  const int lcols = __ffs(cols) - 1;
  int Ns = 1, lNs = 0;
  while (logn - lNs >= 2) {
    const int q = n >> 2, lq = logn - 2;
    const int total = q << lcols;
    for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
      int j, c;
      if (ROWMAJOR) {
        j = idx & (q - 1);
        c = idx >> lq;
      } else {
        c = idx & (cols - 1);
        j = idx >> lcols;
      }
      const int k = j & (Ns - 1);
      float2 v0 = a[fft_addr<ROWMAJOR>(c, j, n, cols)];
      float2 v1 = a[fft_addr<ROWMAJOR>(c, j + q, n, cols)];
      float2 v2 = a[fft_addr<ROWMAJOR>(c, j + 2 * q, n, cols)];
      float2 v3 = a[fft_addr<ROWMAJOR>(c, j + 3 * q, n, cols)];
      if (k) {  // w^(i k) = exp(-2 pi i i k / (4 Ns)) = tw[i k n / (4 Ns)]
        const int sh = logn - lNs - 2;
        v1 = cmul(v1, twiddle(tw, k << sh, n, inv));
        v2 = cmul(v2, twiddle(tw, (2 * k) << sh, n, inv));
        v3 = cmul(v3, twiddle(tw, (3 * k) << sh, n, inv));
      }
      const float2 a0 = cadd(v0, v2), a1 = csub(v0, v2), a2 = cadd(v1, v3), d = csub(v1, v3);
      // (v1 - v3) * (-i) forward, * (+i) inverse
      const float2 a3 = inv ? make_float2(-d.y, d.x) : make_float2(d.y, -d.x);
      const int o = ((j - k) << 2) + k;
      b[fft_addr<ROWMAJOR>(c, o, n, cols)] = cadd(a0, a2);
      b[fft_addr<ROWMAJOR>(c, o + Ns, n, cols)] = cadd(a1, a3);
      b[fft_addr<ROWMAJOR>(c, o + 2 * Ns, n, cols)] = csub(a0, a2);
      b[fft_addr<ROWMAJOR>(c, o + 3 * Ns, n, cols)] = csub(a1, a3);
    }
    __syncthreads();
    float2* t = a;
    a = b;
    b = t;
    Ns <<= 2;
    lNs += 2;
  }
  if (lNs < logn) {  // the last radix-2 pass
    const int half = n >> 1;
    const int total = half << lcols;
    for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
      int j, c;
      if (ROWMAJOR) {
        j = idx & (half - 1);
        c = idx >> (logn - 1);
      } else {
        c = idx & (cols - 1);
        j = idx >> lcols;
      }
      const int k = j & (Ns - 1);
      const float2 w = twiddle(tw, k << (logn - 1 - lNs), n, inv);
      const float2 x0 = a[fft_addr<ROWMAJOR>(c, j, n, cols)];
      const float2 t = cmul(a[fft_addr<ROWMAJOR>(c, j + half, n, cols)], w);
      const int o = ((j - k) << 1) + k;
      b[fft_addr<ROWMAJOR>(c, o, n, cols)] = cadd(x0, t);
      b[fft_addr<ROWMAJOR>(c, o + Ns, n, cols)] = csub(x0, t);
    }
    __syncthreads();
    float2* t = a;
    a = b;
    b = t;
  }
  return a;
}

__device__ __forceinline__ void load_twiddles(float2* s_tw, const float2* tw, int n) {
  for (int i = threadIdx.x; i < (n >> 1); i += blockDim.x) s_tw[i] = tw[i];
}

// ---- CIC deposit (cic.rs:37-93) ------------------------------------------------
struct Cic {
  int ix[2], iy[2], iz[2];
  float wx[2], wy[2], wz[2];
};

__device__ __forceinline__ void cic_axis(uint32_t q, double scale, double inv_cell, double nmf, int nm, int* i,
                                         float* w) {
  const double c = rem_euclid(dmul(decode(q, scale), inv_cell), nmf);
  const double f = floor(c);
  const int i0 = (int)f;
  const double d = dsub(c, f);
  i[0] = i0;
  i[1] = (i0 + 1) % nm;
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

// The particles arrive in octree order, so lanes of a warp often share a
// CIC cell (in a Plummer core, hundreds of particles share one).  Lanes with
// the same base cell (hence the same 8 nodes) are grouped with match_any; the
// group's first lane sums their 8 weighted masses through shuffles and issues
// the 8 atomics for all of them.  The cell index and the weights are the
// reference's (float64 position arithmetic, product m wx wy wz).
__global__ void k_deposit(const uint32_t* __restrict__ qx, const uint32_t* __restrict__ qy,
                          const uint32_t* __restrict__ qz, const float* __restrict__ m, int64_t n, double scale,
                          double inv_cell, int nm, float* __restrict__ rho, const uint32_t* __restrict__ id,
                          uint32_t id_limit) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int lane = threadIdx.x & 31;
  const bool live = i < n && (!id || id[i] < id_limit);  // halo copies deposit nothing
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
  const int64_t nm2 = (int64_t)nm * nm;
  if (rounds == 1) {  // no two lanes share a cell
    if (!live) return;
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int b = 0; b < 2; ++b)
#pragma unroll
        for (int d = 0; d < 2; ++d)
          atomicAdd(&rho[c.iz[a] * nm2 + (int64_t)c.iy[b] * nm + c.ix[d]], mi * c.wx[d] * c.wy[b] * c.wz[a]);
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
  if (!live || lane != __ffs(peers) - 1) return;
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b)
#pragma unroll
      for (int d = 0; d < 2; ++d) atomicAdd(&rho[c.iz[a] * nm2 + (int64_t)c.iy[b] * nm + c.ix[d]], sum[a * 4 + b * 2 + d]);
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
// X[0] and X[h] are real up to rounding).  Shared memory: the nm/2 twiddles of
// length nm, the h/2 of length h, two work rows of h per row.
__device__ __forceinline__ void load_x_twiddles(float2* s_tw, float2* s_th, const float2* tw, int nm) {
  const int h = nm >> 1;
  for (int i = threadIdx.x; i < h; i += blockDim.x) s_tw[i] = tw[i];
  for (int i = threadIdx.x; i < (h >> 1); i += blockDim.x) s_th[i] = tw[2 * i];
}

__global__ void k_fft_x_r2c(const float* __restrict__ rho, float2* __restrict__ spec, int nm, int logn, int nh,
                            int rows, int64_t nrows, const float2* __restrict__ tw) {
  extern __shared__ float2 sm[];
  const int h = nm >> 1;
  float2* s_tw = sm;
  float2* s_th = sm + h;
  float2* a = s_th + (h >> 1 > 0 ? h >> 1 : 1);
  float2* b = a + rows * h;
  load_x_twiddles(s_tw, s_th, tw, nm);
  const int64_t row0 = (int64_t)blockIdx.x * rows;
  const float2* src = reinterpret_cast<const float2*>(rho);
  for (int idx = threadIdx.x; idx < rows * h; idx += blockDim.x) {
    const int r = idx / h, j = idx % h;
    a[idx] = row0 + r < nrows ? src[(row0 + r) * h + j] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  const float2* res = fft_smem<true>(a, b, h, logn - 1, rows, s_th, false);
  for (int idx = threadIdx.x; idx < rows * nh; idx += blockDim.x) {
    const int r = idx / nh, k = idx % nh;
    if (row0 + r >= nrows) continue;
    const float2 zk = res[r * h + (k == h ? 0 : k)];
    const float2 zm = res[r * h + (k == 0 || k == h ? 0 : h - k)];
    const float2 e = make_float2(0.5f * (zk.x + zm.x), 0.5f * (zk.y - zm.y));
    const float2 o = make_float2(0.5f * (zk.y + zm.y), -0.5f * (zk.x - zm.x));  // (Zk - conj Zm) / 2i
    spec[(row0 + r) * nh + k] = cadd(e, cmul(twiddle(s_tw, k, nm, false), o));
  }
}

__global__ void k_fft_x_c2r(const float2* __restrict__ spec3, float* __restrict__ force, int nm, int logn, int nh,
                            int rows, int64_t nrows, const float2* __restrict__ tw) {
  extern __shared__ float2 sm[];
  const int h = nm >> 1;
  float2* s_tw = sm;
  float2* s_th = sm + h;
  float2* a = s_th + (h >> 1 > 0 ? h >> 1 : 1);
  float2* b = a + rows * h;
  load_x_twiddles(s_tw, s_th, tw, nm);
  __syncthreads();  // the unpacking below reads s_tw
  const int comp = blockIdx.y;
  const float2* in = spec3 + comp * nrows * nh;
  float2* out = reinterpret_cast<float2*>(force + comp * nrows * nm);
  const int64_t row0 = (int64_t)blockIdx.x * rows;
  for (int idx = threadIdx.x; idx < rows * h; idx += blockDim.x) {
    const int r = idx / h, k = idx % h;
    float2 z = make_float2(0.f, 0.f);
    if (row0 + r < nrows) {
      float2 xk = in[(row0 + r) * nh + k];
      float2 xm = in[(row0 + r) * nh + (h - k)];
      if (k == 0) xk.y = xm.y = 0.f;  // the real part of the full inverse: Im X[0], Im X[h] drop out
      const float2 w = twiddle(s_tw, k, nm, true);  // e^{+2 pi i k / nm}
      // X[k] (1 + i W) + conj(X[h - k]) (1 - i W)
      const float2 p = make_float2(1.f - w.y, w.x), q = make_float2(1.f + w.y, -w.x);
      z = cadd(cmul(xk, p), cmul(make_float2(xm.x, -xm.y), q));
    }
    a[idx] = z;
  }
  __syncthreads();
  const float2* res = fft_smem<true>(a, b, h, logn - 1, rows, s_th, true);
  for (int idx = threadIdx.x; idx < rows * h; idx += blockDim.x) {
    const int r = idx / h, j = idx % h;
    if (row0 + r < nrows) out[(row0 + r) * h + j] = res[idx];
  }
}

// ---- y pass (c2c) on [z][y][kx] half spectra, one component per blockIdx.z --------
__global__ void k_fft_y(float2* __restrict__ spec, int64_t comp_stride, int nm, int logn, int nh, int tx,
                        const float2* __restrict__ tw, int inv) {
  extern __shared__ float2 sm[];
  float2* s_tw = sm;
  float2* a = sm + (nm >> 1);
  float2* b = a + nm * tx;
  load_twiddles(s_tw, tw, nm);
  const int kx0 = blockIdx.x * tx, z = blockIdx.y;
  float2* base = spec + blockIdx.z * comp_stride + (int64_t)z * nm * nh;
  for (int idx = threadIdx.x; idx < nm * tx; idx += blockDim.x) {
    const int y = idx / tx, c = idx % tx;
    a[idx] = (kx0 + c < nh) ? base[(int64_t)y * nh + kx0 + c] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  const float2* res = fft_smem<false>(a, b, nm, logn, tx, s_tw, inv != 0);
  for (int idx = threadIdx.x; idx < nm * tx; idx += blockDim.x) {
    const int y = idx / tx, c = idx % tx;
    if (kx0 + c < nh) base[(int64_t)y * nh + kx0 + c] = res[idx];
  }
}

// ---- z pass (c2c) on [z][y][kx] half spectra, one component per blockIdx.z --------
__global__ void k_fft_z_c2c(float2* __restrict__ spec, int64_t comp_stride, int nm, int logn, int nh, int tx,
                            const float2* __restrict__ tw, int inv) {
  extern __shared__ float2 sm[];
  float2* s_tw = sm;
  float2* a = sm + (nm >> 1);
  float2* b = a + nm * tx;
  load_twiddles(s_tw, tw, nm);
  const int kx0 = blockIdx.x * tx, y = blockIdx.y;
  const int64_t plane = (int64_t)nm * nh;
  float2* base = spec + blockIdx.z * comp_stride + (int64_t)y * nh;
  for (int idx = threadIdx.x; idx < nm * tx; idx += blockDim.x) {
    const int z = idx / tx, c = idx % tx;
    a[idx] = (kx0 + c < nh) ? base[z * plane + kx0 + c] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  const float2* res = fft_smem<false>(a, b, nm, logn, tx, s_tw, inv != 0);
  for (int idx = threadIdx.x; idx < nm * tx; idx += blockDim.x) {
    const int z = idx / tx, c = idx % tx;
    if (kx0 + c < nh) base[z * plane + kx0 + c] = res[idx];
  }
}

// ---- z pass + Green's function x filter x gradient + inverse z pass ---------------
__global__ void k_fft_z_poisson(const float2* __restrict__ spec, float2* __restrict__ spec3, int nm, int logn,
                                int nh, int tx, const float2* __restrict__ tw, const float* __restrict__ kval,
                                const float* __restrict__ kfilter, const float* __restrict__ kderiv, float kcoef,
                                int ncomp) {
  extern __shared__ float2 sm[];
  float2* s_tw = sm;
  float2* a = sm + (nm >> 1);
  float2* b = a + nm * tx;
  float2* c3 = b + nm * tx;
  load_twiddles(s_tw, tw, nm);
  const int kx0 = blockIdx.x * tx, y = blockIdx.y;
  const int64_t plane = (int64_t)nm * nh;
  for (int idx = threadIdx.x; idx < nm * tx; idx += blockDim.x) {
    const int z = idx / tx, c = idx % tx;
    a[idx] = (kx0 + c < nh) ? spec[z * plane + (int64_t)y * nh + kx0 + c] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  float2* rho_k = fft_smem<false>(a, b, nm, logn, tx, s_tw, false);
  float2* spare = rho_k == a ? b : a;
  // phi(k) = rho(k) * kcoef * W(k) / k^2 ; F_a = -i D_a phi
  for (int idx = threadIdx.x; idx < nm * tx; idx += blockDim.x) {
    const int z = idx / tx, c = idx % tx;
    const int kx = kx0 + c;
    float2 v = make_float2(0.f, 0.f);
    if (kx < nh) {
      const float k2 = kval[kx] * kval[kx] + kval[y] * kval[y] + kval[z] * kval[z];
      if (k2 > 0.f) {
        const float s = kcoef * kfilter[kx] * kfilter[y] * kfilter[z] / k2;
        v = make_float2(rho_k[idx].x * s, rho_k[idx].y * s);
      }
    }
    rho_k[idx] = v;  // phi
  }
  __syncthreads();
  for (int comp = 0; comp < ncomp; ++comp) {
    for (int idx = threadIdx.x; idx < nm * tx; idx += blockDim.x) {
      const int z = idx / tx, c = idx % tx;
      const int kx = kx0 + c < nh ? kx0 + c : 0;
      const float2 ph = rho_k[idx];
      if (comp == 3) {  // the potential itself
        c3[idx] = ph;
        continue;
      }
      const float d = comp == 0 ? kderiv[kx] : (comp == 1 ? kderiv[y] : kderiv[z]);
      c3[idx] = make_float2(d * ph.y, -d * ph.x);
    }
    __syncthreads();
    const float2* res = fft_smem<false>(c3, spare, nm, logn, tx, s_tw, true);
    float2* out = spec3 + comp * (int64_t)nm * plane;
    for (int idx = threadIdx.x; idx < nm * tx; idx += blockDim.x) {
      const int z = idx / tx, c = idx % tx;
      if (kx0 + c < nh) out[z * plane + (int64_t)y * nh + kx0 + c] = res[idx];
    }
    __syncthreads();
    if (res == spare) {  // keep c3 as the scratch input of the next component
      float2* t = spare;
      spare = c3;
      c3 = t;
    }
  }
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

__device__ __forceinline__ double pk_sinc(int k, int nm) {
  if (k == 0) return 1.0;
  const double x = (double)k / (double)nm;
  return sinpi(x) / (M_PI * x);
}

// Forward z pass of the half spectrum, then every mode into its |k| shell:
// sum of |rho_k|^2 / W^2 and the mode count, modes with 0 < kx < nm/2 twice
// (their conjugates are not stored), as power_spectrum.rs:74-110 over the full
// cube.
__global__ void k_fft_z_pk(const float2* __restrict__ spec, int nm, int logn, int nh, int tx,
                           const float2* __restrict__ tw, double* __restrict__ pk_sum,
                           unsigned long long* __restrict__ pk_n) {
  extern __shared__ float2 sm[];
  float2* s_tw = sm;
  float2* a = sm + (nm >> 1);
  float2* b = a + nm * tx;
  double* hs = reinterpret_cast<double*>(b + nm * tx);
  unsigned long long* hn = reinterpret_cast<unsigned long long*>(hs + (nm >> 1));
  load_twiddles(s_tw, tw, nm);
  for (int i = threadIdx.x; i < (nm >> 1); i += blockDim.x) {
    hs[i] = 0.0;
    hn[i] = 0ull;
  }
  const int kx0 = blockIdx.x * tx, y = blockIdx.y;
  const int64_t plane = (int64_t)nm * nh;
  for (int idx = threadIdx.x; idx < nm * tx; idx += blockDim.x) {
    const int z = idx / tx, c = idx % tx;
    a[idx] = (kx0 + c < nh) ? spec[z * plane + (int64_t)y * nh + kx0 + c] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  const float2* res = fft_smem<false>(a, b, nm, logn, tx, s_tw, false);
  const int nb = nm >> 1;
  const int fy = y <= nb ? y : y - nm;
  for (int idx = threadIdx.x; idx < nm * tx; idx += blockDim.x) {
    const int z = idx / tx, c = idx % tx;
    const int kx = kx0 + c;
    if (kx >= nh) continue;
    const int fz = z <= nb ? z : z - nm;
    const double k2 = (double)kx * kx + (double)fy * fy + (double)fz * fz;
    if (k2 == 0.0) continue;
    const double bf = sqrt(k2) - 0.5;
    if (bf < 0.0 || bf >= (double)nb) continue;
    const int bin = (int)bf;
    const double w = pk_sinc(kx, nm) * pk_sinc(fy, nm) * pk_sinc(fz, nm);
    const double re = res[idx].x, im = res[idx].y;
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

// Threads per block of the FFT passes: the passes loop over their butterflies
// by blockDim, and 512 threads hide the shared-memory latency of the 2-3
// resident blocks per SM better than 256 (PM 2.04 -> 1.67 ms at 256^3) or 1024.
constexpr int FFT_THREADS = 512;

// Full-length rows and columns (y, z passes) per block: 2048 elements per block
// (8 x 8 at nm = 256: PM 1.67 -> 1.61 ms against 16 x 16; 32-wide tiles are
// slower), at least 8 columns so a block still reads 64-byte runs.
inline int rows_for(int nm) {
  int r = nm >= 2048 ? 1 : 2048 / nm;
  return r > nm * nm ? nm * nm : r;
}
inline int tx_for(int nm) {
  int t = 2048 / nm;
  return t < 8 ? 8 : (t > 16 ? 16 : t);
}

// The x passes: rows per block (the half-length rows of 2048 / nm complex
// elements each make the same 2048-element tile), shared memory, blocks.
struct XPass {
  int rows;
  size_t smem;
  int blocks;
};
inline XPass x_pass(int nm, int64_t nrows) {
  const int h = nm >> 1;
  int rows = rows_for(nm) * 2;
  if ((int64_t)rows > nrows) rows = (int)nrows;
  const size_t smem = sizeof(float2) * ((size_t)h + (size_t)(h >> 1 > 0 ? h >> 1 : 1) + 2 * (size_t)rows * h);
  return XPass{rows, smem, (int)((nrows + rows - 1) / rows)};
}

}  // namespace

void pm_plan_init(PmPlan& p, int nm, double box, double r_split, uint32_t flags, int device) {
  (void)device;
  p.nm = nm;
  p.logn = ilog2(nm);
  p.nh = nm / 2 + 1;
  p.box = box;
  const int64_t nm3 = (int64_t)nm * nm * nm;
  const int64_t nspec = (int64_t)nm * nm * p.nh;
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
  // shared-memory opt-in for the largest variants
  const int big = 227 * 1024;
  TPM_CUDA(cudaFuncSetAttribute(k_fft_x_r2c, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  TPM_CUDA(cudaFuncSetAttribute(k_fft_y, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  TPM_CUDA(cudaFuncSetAttribute(k_fft_z_poisson, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
  TPM_CUDA(cudaFuncSetAttribute(k_fft_x_c2r, cudaFuncAttributeMaxDynamicSharedMemorySize, big));
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
  p = PmPlan();
}

void pm_deposit(const PmPlan& p, const uint32_t* qx, const uint32_t* qy, const uint32_t* qz, const float* massf,
                int64_t n, cudaStream_t s, const uint32_t* id, uint32_t id_limit) {
  const int64_t nm3 = (int64_t)p.nm * p.nm * p.nm;
  TPM_CUDA(cudaMemsetAsync(p.rho, 0, sizeof(float) * nm3, s));
  if (n == 0) return;
  k_deposit<<<grid_for(n, 256, 1ll << 30), 256, 0, s>>>(qx, qy, qz, massf, n, p.box / TWO32, (double)p.nm / p.box,
                                                        p.nm, p.rho, id, id_limit);
  TPM_LAUNCH_CHECK();
}

void pm_solve(const PmPlan& p, cudaStream_t s) {
  const int nm = p.nm, nh = p.nh, logn = p.logn;
  const int tx = tx_for(nm);
  const int64_t nrows = (int64_t)nm * nm;
  const XPass xp = x_pass(nm, nrows);
  const size_t sm_y = sizeof(float2) * ((size_t)(nm / 2) + 2 * (size_t)nm * tx);
  const size_t sm_z = sizeof(float2) * ((size_t)(nm / 2) + 3 * (size_t)nm * tx);
  const int ntx = (nh + tx - 1) / tx;
  k_fft_x_r2c<<<xp.blocks, FFT_THREADS, xp.smem, s>>>(p.rho, p.spec, nm, logn, nh, xp.rows, nrows, p.twiddle);
  TPM_LAUNCH_CHECK();
  k_fft_y<<<dim3(ntx, nm, 1), FFT_THREADS, sm_y, s>>>(p.spec, 0, nm, logn, nh, tx, p.twiddle, 0);
  TPM_LAUNCH_CHECK();
  k_fft_z_poisson<<<dim3(ntx, nm), FFT_THREADS, sm_z, s>>>(p.spec, p.spec3, nm, logn, nh, tx, p.twiddle, p.kval, p.kfilter,
                                                   p.kderiv, p.kcoef, p.ncomp);
  TPM_LAUNCH_CHECK();
  k_fft_y<<<dim3(ntx, nm, p.ncomp), FFT_THREADS, sm_y, s>>>(p.spec3, nrows * nh, nm, logn, nh, tx, p.twiddle, 1);
  TPM_LAUNCH_CHECK();
  k_fft_x_c2r<<<dim3(xp.blocks, p.ncomp), FFT_THREADS, xp.smem, s>>>(p.spec3, p.force, nm, logn, nh, xp.rows, nrows,
                                                                      p.twiddle);
  TPM_LAUNCH_CHECK();
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
  const int nm = p.nm, nh = p.nh, logn = p.logn;
  const int tx = tx_for(nm);
  const int64_t nrows = (int64_t)nm * nm;
  const XPass xp = x_pass(nm, nrows);
  const size_t sm_y = sizeof(float2) * ((size_t)(nm / 2) + 2 * (size_t)nm * tx);
  TPM_CUDA(cudaFuncSetAttribute(k_fft_z_c2c, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024));
  const int ntx = (nh + tx - 1) / tx;
  k_fft_x_r2c<<<xp.blocks, FFT_THREADS, xp.smem, s>>>(p.rho, p.spec, nm, logn, nh, xp.rows, nrows, p.twiddle);
  TPM_LAUNCH_CHECK();
  k_fft_y<<<dim3(ntx, nm, 1), FFT_THREADS, sm_y, s>>>(p.spec, 0, nm, logn, nh, tx, p.twiddle, 0);
  TPM_LAUNCH_CHECK();
  k_fft_z_c2c<<<dim3(ntx, nm, 1), FFT_THREADS, sm_y, s>>>(p.spec, 0, nm, logn, nh, tx, p.twiddle, 0);
  TPM_LAUNCH_CHECK();
}

void pm_inverse_components(const PmPlan& p, int ncomp, cudaStream_t s) {
  const int nm = p.nm, nh = p.nh, logn = p.logn;
  const int tx = tx_for(nm);
  const int64_t nrows = (int64_t)nm * nm;
  const XPass xp = x_pass(nm, nrows);
  const size_t sm_y = sizeof(float2) * ((size_t)(nm / 2) + 2 * (size_t)nm * tx);
  TPM_CUDA(cudaFuncSetAttribute(k_fft_z_c2c, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024));
  const int ntx = (nh + tx - 1) / tx;
  k_fft_z_c2c<<<dim3(ntx, nm, ncomp), FFT_THREADS, sm_y, s>>>(p.spec3, nrows * nh, nm, logn, nh, tx, p.twiddle, 1);
  TPM_LAUNCH_CHECK();
  k_fft_y<<<dim3(ntx, nm, ncomp), FFT_THREADS, sm_y, s>>>(p.spec3, nrows * nh, nm, logn, nh, tx, p.twiddle, 1);
  TPM_LAUNCH_CHECK();
  k_fft_x_c2r<<<dim3(xp.blocks, ncomp), FFT_THREADS, xp.smem, s>>>(p.spec3, p.force, nm, logn, nh, xp.rows, nrows,
                                                                    p.twiddle);
  TPM_LAUNCH_CHECK();
}

void pm_power_spectrum(const PmPlan& p, const double* pos, const uint32_t* qx, const uint32_t* qy,
                       const uint32_t* qz, const double* mass, int64_t n, double total_mass, double* pk_sum,
                       unsigned long long* pk_n, double* k_out, double* pk_out, unsigned long long* n_out,
                       cudaStream_t s) {
  const int nm = p.nm, nh = p.nh, logn = p.logn, nb = nm / 2;
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
  const int tx = tx_for(nm);
  const int64_t nrows = (int64_t)nm * nm;
  const XPass xp = x_pass(nm, nrows);
  const size_t sm_y = sizeof(float2) * ((size_t)(nm / 2) + 2 * (size_t)nm * tx);
  const size_t sm_pk = sm_y + (sizeof(double) + sizeof(unsigned long long)) * (size_t)nb;
  TPM_CUDA(cudaFuncSetAttribute(k_fft_z_pk, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024));
  const int ntx = (nh + tx - 1) / tx;
  k_fft_x_r2c<<<xp.blocks, FFT_THREADS, xp.smem, s>>>(p.rho, p.spec, nm, logn, nh, xp.rows, nrows, p.twiddle);
  TPM_LAUNCH_CHECK();
  k_fft_y<<<dim3(ntx, nm, 1), FFT_THREADS, sm_y, s>>>(p.spec, 0, nm, logn, nh, tx, p.twiddle, 0);
  TPM_LAUNCH_CHECK();
  k_fft_z_pk<<<dim3(ntx, nm), FFT_THREADS, sm_pk, s>>>(p.spec, nm, logn, nh, tx, p.twiddle, pk_sum, pk_n);
  TPM_LAUNCH_CHECK();
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

}  // namespace tpm
