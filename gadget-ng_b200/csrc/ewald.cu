// FP64 Ewald summation: the accuracy reference for the TreePM force.
//
// No counterpart in the reference (it has no Ewald code).  Written from the
// mathematics (Ewald 1921; Hernquist, Bouchet & Suto 1991, ApJS 75, 231): the
// periodic 1/r^2 force splits into a real-space sum with the kernel
// erfc(a r) + (2 a r / sqrt(pi)) exp(-a^2 r^2) over minimum images within r_c
// and a k-space sum (4 pi / V) sum_{k != 0} (k / k^2) exp(-k^2 / 4a^2)
// Im(exp(-i k.x_i) S(k)) with structure factors S(k) = sum_j m_j exp(i k.x_j).
// The k = 0 term is dropped (uniform neutralising background, as the PM does).
// Nearest-image pairs closer than r_soft get the Plummer correction
// m (1/(r^2+eps^2)^{3/2} - 1/r^3) r_vec, so the reference is softened where
// the TreePM short range softens.  All arithmetic is float64; this is a
// checker, run outside any timed region.
#include <cmath>
#include <vector>

#include "../../include/treepm_b200.h"
#include "common.cuh"

namespace {

__global__ void k_ewald_real(const double* __restrict__ pos, const double* __restrict__ mass, int64_t n, double box,
                             const int64_t* __restrict__ targets, double alpha, double rc2, double eps2,
                             double rsoft2, double* __restrict__ out) {
  const int64_t t = blockIdx.x;
  const int64_t i = targets[t];
  const double xi = pos[3 * i], yi = pos[3 * i + 1], zi = pos[3 * i + 2];
  const double half = 0.5 * box;
  const double two_over_sqrtpi = 1.1283791670955126;
  double ax = 0.0, ay = 0.0, az = 0.0;
  for (int64_t j = threadIdx.x; j < n; j += blockDim.x) {
    if (j == i) continue;
    double dx = pos[3 * j] - xi, dy = pos[3 * j + 1] - yi, dz = pos[3 * j + 2] - zi;
    dx -= box * rint(dx / box);
    dy -= box * rint(dy / box);
    dz -= box * rint(dz / box);
    (void)half;
    const double r2 = dx * dx + dy * dy + dz * dz;
    if (r2 >= rc2) continue;
    const double r = sqrt(r2);
    const double ar = alpha * r;
    double s = (erfc(ar) + two_over_sqrtpi * ar * exp(-ar * ar)) / (r2 * r);
    if (r2 < rsoft2) {  // Plummer softening of the nearest image
      const double rs2 = r2 + eps2;
      s += 1.0 / (rs2 * sqrt(rs2)) - 1.0 / (r2 * r);
    }
    s *= mass[j];
    ax += s * dx;
    ay += s * dy;
    az += s * dz;
  }
  // block reduction
  __shared__ double red[3][32];
  for (int o = 16; o > 0; o >>= 1) {
    ax += __shfl_down_sync(0xffffffffu, ax, o);
    ay += __shfl_down_sync(0xffffffffu, ay, o);
    az += __shfl_down_sync(0xffffffffu, az, o);
  }
  const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) {
    red[0][w] = ax;
    red[1][w] = ay;
    red[2][w] = az;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double sx = 0, sy = 0, sz = 0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
      sx += red[0][k];
      sy += red[1][k];
      sz += red[2][k];
    }
    out[3 * t] = sx;
    out[3 * t + 1] = sy;
    out[3 * t + 2] = sz;
  }
}

// S(k) for the listed modes (integer triples), one block per mode.
__global__ void k_ewald_structure(const double* __restrict__ pos, const double* __restrict__ mass, int64_t n,
                                  double box, const int* __restrict__ modes, double* __restrict__ sk) {
  const int m = blockIdx.x;
  const double w = 2.0 * M_PI / box;
  const double kx = w * modes[3 * m], ky = w * modes[3 * m + 1], kz = w * modes[3 * m + 2];
  double re = 0.0, im = 0.0;
  for (int64_t j = threadIdx.x; j < n; j += blockDim.x) {
    double s, c;
    sincos(kx * pos[3 * j] + ky * pos[3 * j + 1] + kz * pos[3 * j + 2], &s, &c);
    re += mass[j] * c;
    im += mass[j] * s;
  }
  __shared__ double red[2][32];
  for (int o = 16; o > 0; o >>= 1) {
    re += __shfl_down_sync(0xffffffffu, re, o);
    im += __shfl_down_sync(0xffffffffu, im, o);
  }
  const int wi = threadIdx.x >> 5, l = threadIdx.x & 31;
  if (l == 0) {
    red[0][wi] = re;
    red[1][wi] = im;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0, b = 0;
    for (int k = 0; k < (int)(blockDim.x >> 5); ++k) {
      a += red[0][k];
      b += red[1][k];
    }
    sk[2 * m] = a;
    sk[2 * m + 1] = b;
  }
}

// k-space acceleration at each target from the half-space modes (x2).
__global__ void k_ewald_kspace(const double* __restrict__ pos, const int64_t* __restrict__ targets, int64_t nt,
                               double box, const int* __restrict__ modes, const double* __restrict__ sk, int nmodes,
                               double alpha, double* __restrict__ out) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= nt) return;
  const int64_t i = targets[t];
  const double xi = pos[3 * i], yi = pos[3 * i + 1], zi = pos[3 * i + 2];
  const double w = 2.0 * M_PI / box;
  const double pref = 2.0 * 4.0 * M_PI / (box * box * box);
  double ax = 0.0, ay = 0.0, az = 0.0;
  for (int m = 0; m < nmodes; ++m) {
    const double kx = w * modes[3 * m], ky = w * modes[3 * m + 1], kz = w * modes[3 * m + 2];
    const double k2 = kx * kx + ky * ky + kz * kz;
    double s, c;
    sincos(kx * xi + ky * yi + kz * zi, &s, &c);
    // Im(exp(-i k.x) S) = c * Im S - s * Re S
    const double im = c * sk[2 * m + 1] - s * sk[2 * m];
    const double f = pref * exp(-k2 / (4.0 * alpha * alpha)) / k2 * im;
    ax += f * kx;
    ay += f * ky;
    az += f * kz;
  }
  out[3 * t] += ax;
  out[3 * t + 1] += ay;
  out[3 * t + 2] += az;
}

}  // namespace

extern "C" int tpm_ewald(const double* pos, const double* mass, int64_t n, double box, double g, double eps2,
                         double r_soft, const int64_t* targets, int64_t nt, double alpha, double r_c, int n_max,
                         int device, double* out) {
  if (!pos || !mass || !targets || !out || n <= 0 || nt <= 0 || !(box > 0) || n_max < 1)
    return TPM_ERR_INVALID_ARGUMENT;
  for (int64_t t = 0; t < nt; ++t)
    if (targets[t] < 0 || targets[t] >= n) return TPM_ERR_INVALID_ARGUMENT;
  double *dpos = nullptr, *dmass = nullptr, *dout = nullptr, *dsk = nullptr;
  int64_t* dt = nullptr;
  int* dmodes = nullptr;
  int rc = TPM_OK;
  try {
    TPM_CUDA(cudaSetDevice(device));
    // half space of integer modes with 0 < |n| <= n_max
    std::vector<int> modes;
    for (int x = 0; x <= n_max; ++x)
      for (int y = -n_max; y <= n_max; ++y)
        for (int z = -n_max; z <= n_max; ++z) {
          if (x * x + y * y + z * z > n_max * n_max) continue;
          const bool upper = x > 0 || (x == 0 && (y > 0 || (y == 0 && z > 0)));
          if (!upper) continue;
          modes.push_back(x);
          modes.push_back(y);
          modes.push_back(z);
        }
    const int nmodes = (int)(modes.size() / 3);
    TPM_CUDA(cudaMalloc(&dpos, sizeof(double) * 3 * n));
    TPM_CUDA(cudaMalloc(&dmass, sizeof(double) * n));
    TPM_CUDA(cudaMalloc(&dt, sizeof(int64_t) * nt));
    TPM_CUDA(cudaMalloc(&dout, sizeof(double) * 3 * nt));
    TPM_CUDA(cudaMalloc(&dmodes, sizeof(int) * 3 * nmodes));
    TPM_CUDA(cudaMalloc(&dsk, sizeof(double) * 2 * nmodes));
    TPM_CUDA(cudaMemcpy(dpos, pos, sizeof(double) * 3 * n, cudaMemcpyHostToDevice));
    TPM_CUDA(cudaMemcpy(dmass, mass, sizeof(double) * n, cudaMemcpyHostToDevice));
    TPM_CUDA(cudaMemcpy(dt, targets, sizeof(int64_t) * nt, cudaMemcpyHostToDevice));
    TPM_CUDA(cudaMemcpy(dmodes, modes.data(), sizeof(int) * 3 * nmodes, cudaMemcpyHostToDevice));
    k_ewald_real<<<(unsigned)nt, 256>>>(dpos, dmass, n, box, dt, alpha, r_c * r_c, eps2, r_soft * r_soft, dout);
    TPM_LAUNCH_CHECK();
    k_ewald_structure<<<(unsigned)nmodes, 256>>>(dpos, dmass, n, box, dmodes, dsk);
    TPM_LAUNCH_CHECK();
    k_ewald_kspace<<<(unsigned)((nt + 127) / 128), 128>>>(dpos, dt, nt, box, dmodes, dsk, nmodes, alpha, dout);
    TPM_LAUNCH_CHECK();
    TPM_CUDA(cudaMemcpy(out, dout, sizeof(double) * 3 * nt, cudaMemcpyDeviceToHost));
    for (int64_t k = 0; k < 3 * nt; ++k) out[k] *= g;
  } catch (const tpm::Error& e) {
    rc = e.code ? e.code : TPM_ERR_CUDA;
  }
  cudaFree(dpos);
  cudaFree(dmass);
  cudaFree(dt);
  cudaFree(dout);
  cudaFree(dmodes);
  cudaFree(dsk);
  return rc;
}
