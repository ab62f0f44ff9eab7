// Register-resident DFTs and the two-stage column transform of the PM passes.
//
// A length n = N1 * N2 transform (Cooley-Tukey, index j = N2 j1 + j2 in,
// k = k1 + N1 k2 out) runs on N2 threads per column: thread j2 holds the N1
// elements x[N2 j1 + j2] in registers and does an N1-point DFT there, scales
// by w_n^(j2 k1), writes its results to shared memory, and after one barrier
// each thread does N1 / N2 of the N2-point DFTs over j2 (k1 = t + N2 r) and
// holds X[k1 + N1 k2].  One shared-memory exchange per transform, instead of
// one per radix-4 pass.  Small DFTs are unrolled radix-2 recursions whose
// twiddles are compile-time constants (values of cos / sin at multiples of
// 2 pi / 32).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace tpm {
namespace fftr {

__device__ __forceinline__ float2 c_add(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 c_sub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 c_mul(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}

// cos(2 pi m / 32), m = 0..8 (the rest by symmetry)
__host__ __device__ constexpr double cos32_q(int m) {
  return m == 0   ? 1.0
         : m == 1 ? 0.98078528040323044912618223613424
         : m == 2 ? 0.92387953251128675612818318939679
         : m == 3 ? 0.83146961230254523707878837761791
         : m == 4 ? 0.70710678118654752440084436210485
         : m == 5 ? 0.55557023301960222474283081394853
         : m == 6 ? 0.38268343236508977172845998403040
         : m == 7 ? 0.19509032201612826784828486847702
                  : 0.0;
}

// cos and sin of 2 pi m / 32 for integer m (constant-folded when m is).
__host__ __device__ constexpr double cos32(int m) {
  m = ((m % 32) + 32) % 32;
  return m <= 8 ? cos32_q(m) : m <= 16 ? -cos32_q(16 - m) : m <= 24 ? -cos32_q(m - 16) : cos32_q(32 - m);
}
__host__ __device__ constexpr double sin32(int m) { return cos32(m - 8); }

// w_N^k = exp(-+2 pi i k / N) for N dividing 32 (INV: the + sign).
template <int N, bool INV>
__device__ __forceinline__ float2 root(int k) {
  const int m = (32 / N) * k;
  return make_float2((float)cos32(m), INV ? (float)sin32(m) : -(float)sin32(m));
}

// Multiply by w_N^k with the trivial cases (1, -i, -1, i) folded.
template <int N, bool INV>
__device__ __forceinline__ float2 twiddle_mul(float2 v, int k) {
  const int kk = ((k % N) + N) % N;
  if (kk == 0) return v;
  if (4 * kk == N) return INV ? make_float2(-v.y, v.x) : make_float2(v.y, -v.x);
  if (2 * kk == N) return make_float2(-v.x, -v.y);
  if (4 * kk == 3 * N) return INV ? make_float2(v.y, -v.x) : make_float2(-v.y, v.x);
  return c_mul(v, root<N, INV>(kk));
}

// In-place N-point DFT of x[0..N) at stride S in the array (natural order in
// and out), radix-2 decimation in time, fully unrolled.
template <int N, int S, bool INV>
struct Dft {
  __device__ __forceinline__ static void run(float2* x) {
    Dft<N / 2, 2 * S, INV>::run(x);      // even samples
    Dft<N / 2, 2 * S, INV>::run(x + S);  // odd samples
    // even results at x[2 S k], odd at x[2 S k + S], k < N/2
    float2 t[N];
#pragma unroll
    for (int k = 0; k < N / 2; ++k) {
      const float2 e = x[2 * S * k], o = twiddle_mul<N, INV>(x[2 * S * k + S], k);
      t[k] = c_add(e, o);
      t[k + N / 2] = c_sub(e, o);
    }
#pragma unroll
    for (int k = 0; k < N; ++k) x[S * k] = t[k];
  }
};
template <int S, bool INV>
struct Dft<1, S, INV> {
  __device__ __forceinline__ static void run(float2*) {}
};

template <int N, bool INV>
__device__ __forceinline__ void dft(float2 (&x)[N]) {
  static_assert(N >= 1 && N <= 32 && (N & (N - 1)) == 0, "register DFT sizes 1..32");
  Dft<N, 1, INV>::run(x);
}

// Factors of the two-stage transform: N1 = 2^ceil(log2 n / 2), N2 = n / N1.
template <int LOGN> struct Split {
  static constexpr int N = 1 << LOGN;
  static constexpr int N1 = 1 << ((LOGN + 1) / 2);
  static constexpr int N2 = N / N1;
  static constexpr int R = N1 / N2;  // step-2 DFTs per thread (1 or 2)
};

}  // namespace fftr
}  // namespace tpm
