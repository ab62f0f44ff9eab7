// Shared definitions of the sm_100a TreePM library.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdio>
#include <stdexcept>
#include <string>

namespace tpm {

// ---- error handling (host) -------------------------------------------------
struct Error : public std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define TPM_CUDA(call)                                                                          \
  do {                                                                                          \
    cudaError_t e_ = (call);                                                                    \
    if (e_ != cudaSuccess)                                                                      \
      throw ::tpm::Error(e_ == cudaErrorMemoryAllocation ? 3 : 2,                               \
                         std::string(#call) + ": " + cudaGetErrorString(e_));                   \
  } while (0)

// Kernel launches on this host thread (every launch site ends with
// TPM_LAUNCH_CHECK); the bench reports the per-step count.
extern thread_local unsigned long long g_kernel_launches;
#define TPM_LAUNCH_CHECK()          \
  do {                              \
    ++::tpm::g_kernel_launches;     \
    TPM_CUDA(cudaGetLastError());   \
  } while (0)

// Device-side error flags (bit set in a status word, read by the host after
// the stream synchronises).  Kernels never trap: they record and return.
enum : uint32_t {
  DEV_ERR_STACK = 1u << 0,
  DEV_ERR_DEFERRED = 1u << 1,
  DEV_ERR_COINCIDENT = 1u << 2,
  DEV_ERR_LIST = 1u << 3,
  DEV_ERR_TIE_RUN = 1u << 4,
  DEV_ERR_NONFINITE = 1u << 5,
  DEV_ERR_MMA_TIMEOUT = 1u << 6,  // a tensor-core wait ran past its time limit
  DEV_ERR_TMA_TIMEOUT = 1u << 7,  // a TMA (bulk tensor copy) wait ran past its time limit
};

// ---- fixed point --------------------------------------------------------------
// x = q * scale, scale = L * 2^-32.  Positions wrap modulo 2^32 exactly.
constexpr double TWO32 = 4294967296.0;

inline __host__ __device__ double decode(uint32_t q, double scale) { return (double)q * scale; }

// ---- float64 arithmetic that the compiler may not contract into FMA --------
// The reference's decisions (octant choice, cell index, culls) are f64
// expressions evaluated without FMA; these wrappers keep the device results
// bit-identical.
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }

// Rust f64::rem_euclid.
__device__ __forceinline__ double rem_euclid(double a, double b) {
  double r = fmod(a, b);
  return r < 0.0 ? dadd(r, fabs(b)) : r;
}

// rem_euclid(c, m) for c in [0, 2 m): c, or c - m (exact, Sterbenz) from m
// on.  A decoded fixed-point coordinate times nm / L lies in [0, nm], so the
// CIC cell coordinate needs no general remainder.
__device__ __forceinline__ double rem_once(double c, double m) { return c >= m ? dsub(c, m) : c; }

// minimum_image (crates/gadget-ng-treepm/src/short_range.rs:53-63), exact f64.
__device__ __forceinline__ double minimum_image(double dx, double box) {
  double half = dmul(box, 0.5);
  double d = dsub(dx, dmul(box, round(ddiv(dx, box))));
  if (d > half) d = dsub(d, box);
  else if (d < -half) d = dadd(d, box);
  return d;
}

// ---- hardware approximations (PTX ISA: rsqrt/rcp/ex2 .approx) --------------
__device__ __forceinline__ float rsqrt_approx(float x) {
  float y;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float rcp_approx(float x) {
  float y;
  asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}
__device__ __forceinline__ float ex2_approx(float x) {
  float y;
  asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
  return y;
}

// ---- the erfc-truncated pair kernel, FP32 -----------------------------------
// Abramowitz & Stegun 7.1.26 with the coefficients of
// crates/gadget-ng-treepm/src/short_range.rs:91-101.
struct ErfcConst {
  static constexpr float P = 0.3275911f;
  static constexpr float A1 = 0.254829592f;
  static constexpr float A2 = -0.284496736f;
  static constexpr float A3 = 1.421413741f;
  static constexpr float A4 = -1.453152027f;
  static constexpr float A5 = 1.061405429f;
};

// ---- launch helpers ---------------------------------------------------------------
inline unsigned grid_for(int64_t n, int block, int64_t cap = 148 * 64) {
  int64_t g = (n + block - 1) / block;
  if (g < 1) g = 1;
  if (g > cap) g = cap;
  return (unsigned)g;
}

}  // namespace tpm
