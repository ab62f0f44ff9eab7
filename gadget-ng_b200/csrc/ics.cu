// Zel'dovich initial conditions on the device, written straight into a
// solver handle (crates/gadget-ng-core/src/ic_zeldovich.rs:287-760).
//
// The Gaussian field is generated on the half spectrum [z][y][kx] that the
// mesh FFT uses: modes with kx > 0 are their own representatives; in the kx = 0
// plane a mode and its conjugate twin share the representative with the
// smaller packed index ix n^2 + iy n + iz (the reference's rule), so
// delta(-k) = conj(delta(k)).  DC and every mode with a Nyquist component are
// zero, as in the reference.  Psi_a(k) = i n_a / |n|^2 delta(k) for the three
// axes, three inverse transforms, then particles on the lattice in the
// reference's order (gid = ix n^2 + iy n + iz) at cell centres plus Psi, and
// momenta a^2 f H Psi.  Each mode's seed is the reference's mode_seed of its
// representative; the two uniforms behind its Gaussian come from SplitMix64
// seeded there instead of the reference's StdRng (ChaCha12 in rand 0.10), so a
// realisation is reproducible here but not equal to the reference's; spectrum,
// symmetry, displacement and momentum conventions are the reference's.
#include <cmath>
#include <vector>

#include "../../include/treepm_b200.h"
#include "common.cuh"
#include "pm.cuh"
#include "tree.cuh"

namespace tpm {

// Per-mode standard deviation sigma(|n|) (ic_zeldovich.rs:387-466 with the
// Eisenstein-Hu no-wiggle transfer of transfer_fn.rs:89-127).
struct IcSpectrum {
  int kind;        // 0 power law, 1 Eisenstein-Hu
  double amp;      // A (sigma_8 already applied)
  double n_s;
  double omega_m, omega_b, h;
  double two_pi_h_over_bsm;
  double inv_sqrt_n3;
};

__host__ __device__ inline double eh_transfer(double k, double omega_m, double omega_b, double h) {
  if (k <= 0.0) return 1.0;
  const double om_h2 = omega_m * h * h, ob_h2 = omega_b * h * h, fb = omega_b / omega_m;
  const double s = 44.5 * log(9.83 / om_h2) / sqrt(1.0 + 10.0 * pow(ob_h2, 0.75));
  const double ag = 1.0 - 0.328 * log(431.0 * om_h2) * fb + 0.38 * log(22.3 * om_h2) * fb * fb;
  const double ks = 0.43 * (k * h) * s;
  const double ks2 = ks * ks;
  const double gamma = omega_m * h * (ag + (1.0 - ag) / (1.0 + ks2 * ks2));
  const double q = k / (gamma > 1e-30 ? gamma : 1e-30);
  const double l0 = log(2.718281828459045 * 2.0 + 1.8 * q);
  const double c0 = 14.2 + 731.0 / (1.0 + 62.5 * q);
  const double t = l0 / (l0 + c0 * q * q);
  return t < 0.0 ? 0.0 : (t > 1.0 ? 1.0 : t);
}

__host__ __device__ inline double ic_sigma(const IcSpectrum& sp, double n_abs) {
  if (n_abs <= 0.0) return 0.0;
  if (sp.kind == 0) return sp.amp * pow(n_abs, sp.n_s / 4.0) * sp.inv_sqrt_n3;
  const double k = sp.two_pi_h_over_bsm * n_abs;
  return sp.amp * pow(k, sp.n_s / 2.0) * eh_transfer(k, sp.omega_m, sp.omega_b, sp.h) * sp.inv_sqrt_n3;
}

namespace {

// Murmur3's 64-bit finalizer, the reference's hash_u64 (ic_zeldovich.rs:27-35);
// per-mode seeds are the reference's mode_seed (:38-42) unchanged.
__device__ __forceinline__ uint64_t fmix64(uint64_t x) {
  x ^= x >> 33;
  x *= 0xff51afd7ed558ccdull;
  x ^= x >> 33;
  x *= 0xc4ceb9fe1a85ec53ull;
  x ^= x >> 33;
  return x;
}

// SplitMix64 (Steele, Lea and Flood 2014): the uniform stream behind each
// mode's Gaussian, standing in for the reference's StdRng seeded by mode_seed.
__device__ __forceinline__ uint64_t splitmix_next(uint64_t& state) {
  state += 0x9E3779B97F4A7C15ull;
  uint64_t z = state;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

__device__ __forceinline__ double u53(uint64_t x) { return (double)(x >> 11) * (1.0 / 9007199254740992.0); }

// gaussian_std (ic_zeldovich.rs:51-57): Box-Muller on the first two uniforms
// of the stream seeded by `seed`.
__device__ __forceinline__ double gaussian_std(uint64_t seed) {
  uint64_t st = seed;
  const double u1 = fmax(u53(splitmix_next(st)), 1e-300);
  const double u2 = u53(splitmix_next(st));
  return sqrt(-2.0 * log(u1)) * cos(6.283185307179586 * u2);
}

__device__ __forceinline__ int mode_int(int j, int n) { return j <= n / 2 ? j : j - n; }

// The integrand of sigma^2(8 Mpc/h) for A = 1 (transfer_fn.rs:146-184): k^(n_s+3)
// T(k)^2 W(kR)^2 on 8193 log-spaced points of [1e-5, 5e2] h/Mpc.
__host__ __device__ inline double sigma_integrand(double k, double r, double n_s, double om, double ob, double h) {
  const double t = eh_transfer(k, om, ob, h);
  const double x = k * r;
  const double w = fabs(x) < 1e-4 ? 1.0 - x * x / 10.0 : 3.0 * (sin(x) - x * cos(x)) / (x * x * x);
  return pow(k, n_s + 3.0) * t * t * w * w;
}

constexpr int SIGMA_STEPS = 8192;

// One block: the trapezoid of sigma^2(8) (weights 1/2 at both ends) and the
// amplitude A = sigma_8 / sqrt(sigma^2) into amp_out (amplitude_for_sigma8,
// transfer_fn.rs:222-228); the sum's order differs from the reference's
// running sum only in rounding.
__global__ void k_ic_sigma8(IcSpectrum sp, double sigma8, double* __restrict__ amp_out) {
  __shared__ double part[32];
  const double lk0 = log(1e-5), lk1 = log(5e2), dl = (lk1 - lk0) / SIGMA_STEPS;
  double acc = 0.0;
  for (int i = threadIdx.x; i <= SIGMA_STEPS; i += blockDim.x) {
    const double k = i == 0 ? 1e-5 : exp(lk0 + i * dl);
    const double wgt = (i == 0 || i == SIGMA_STEPS) ? 0.5 : 1.0;
    acc += wgt * sigma_integrand(k, 8.0, sp.n_s, sp.omega_m, sp.omega_b, sp.h);
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double v = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v += part[w];
    v = v * dl / (2.0 * M_PI * M_PI);
    *amp_out = v > 0.0 ? sigma8 / sqrt(v) : sigma8;
  }
}

// sigma(sqrt(n2)) for every integer n2 <= n2_max; the amplitude from amp_dev
// when given (sigma_8 normalisation), else the configured one.
__global__ void k_ic_sigma_table(IcSpectrum sp, const double* __restrict__ amp_dev, int64_t n2_max,
                                 double* __restrict__ table) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i > n2_max) return;
  if (amp_dev) sp.amp = *amp_dev;
  table[i] = ic_sigma(sp, sqrt((double)i));
}

// delta(k) of every half-spectrum mode from the mode seeds, written as the
// three Psi1 components i n_a / |n|^2 delta (ic_zeldovich.rs:541-585) and,
// when `delta_out` is given, as delta itself for the second-order fields.
__global__ void k_ic_modes(int n, int nh, int nhp, uint64_t seed, const double* __restrict__ sigma_of_n2,
                           float2* __restrict__ spec3, int64_t comp_stride, float2* __restrict__ delta_out) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t total = (int64_t)n * n * nhp;  // rows of nhp: kx >= nh is padding
  if (i >= total) return;
  const int kx = (int)(i % nhp), y = (int)((i / nhp) % n), z = (int)(i / ((int64_t)n * nhp));
  if (kx >= nh) return;
  const int nx = kx, ny = mode_int(y, n), nz = mode_int(z, n), half = n / 2;
  const double n2 = (double)nx * nx + (double)ny * ny + (double)nz * nz;
  float2 out[3] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
  float2 dk = make_float2(0.f, 0.f);
  if (n2 > 0.0 && nx != half && abs(ny) != half && abs(nz) != half) {
    // representative of the pair {k, -k} and whether this mode is its twin
    const int64_t self = ((int64_t)kx * n + y) * n + z;
    bool twin = false;
    int64_t rep = self;
    if (kx == 0) {
      const int yn = (n - y) % n, zn = (n - z) % n;
      const int64_t other = (int64_t)yn * n + zn;
      if (other < self) {
        rep = other;
        twin = true;
      }
    }
    const double sig = sigma_of_n2[(int64_t)n2];
    const uint64_t ms = fmix64(seed ^ fmix64((uint64_t)rep));
    double re = sig * gaussian_std(ms), im = sig * gaussian_std(fmix64(ms ^ 0x9E3779B97F4A7C15ull));
    if (twin) im = -im;
    const double inv_n2 = 1.0 / n2;
    const double na[3] = {(double)nx, (double)ny, (double)nz};
#pragma unroll
    for (int c = 0; c < 3; ++c)  // i n_a / |n|^2 (re + i im)
      out[c] = make_float2((float)(-na[c] * im * inv_n2), (float)(na[c] * re * inv_n2));
    dk = make_float2((float)re, (float)im);
  }
  for (int c = 0; c < 3; ++c) spec3[c * comp_stride + i] = out[c];
  if (delta_out) delta_out[i] = dk;
}

// Second derivatives of phi from the stored delta (ic_2lpt.rs:86-140):
// -n_a^2 / |n|^2 delta for a = x, y, z (off_diagonal 0) or -n_a n_b / |n|^2
// delta for ab = xy, xz, yz (off_diagonal 1).
__global__ void k_ic_phi_ab(const float2* __restrict__ delta, int n, int nh, int nhp, float2* __restrict__ spec3,
                            int64_t comp_stride, int off_diagonal) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t total = (int64_t)n * n * nhp;
  if (i >= total) return;
  const int kx = (int)(i % nhp), y = (int)((i / nhp) % n), z = (int)(i / ((int64_t)n * nhp));
  if (kx >= nh) return;
  const float na[3] = {(float)kx, (float)mode_int(y, n), (float)mode_int(z, n)};
  const float n2 = na[0] * na[0] + na[1] * na[1] + na[2] * na[2];
  const float2 dk = delta[i];
  const int a0[3] = {0, 0, 1}, b0[3] = {1, 2, 2};
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const float f = n2 > 0.f ? (off_diagonal ? -na[a0[c]] * na[b0[c]] : -na[c] * na[c]) / n2 : 0.f;
    spec3[c * comp_stride + i] = make_float2(f * dk.x, f * dk.y);
  }
}

// The 2LPT source (ic_2lpt.rs:146-165) from unnormalised inverse transforms of
// phi_ab (scaled by 1/n^3 here): the diagonal pass sets rho to
// xx yy + yy zz + zz xx, the off-diagonal pass subtracts xy^2 + xz^2 + yz^2.
__global__ void k_ic_source(const float* __restrict__ f, float* __restrict__ rho, int64_t n3, float inv_n3,
                            int off_diagonal) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n3) return;
  const float a = f[i] * inv_n3, b = f[n3 + i] * inv_n3, c = f[2 * n3 + i] * inv_n3;
  if (!off_diagonal)
    rho[i] = fmaf(a, b, fmaf(b, c, c * a));
  else
    rho[i] -= fmaf(a, a, fmaf(b, b, c * c));
}

// Psi2_a(k) = -i n_a / |n|^2 S(k), zero at DC and on the Nyquist planes
// (ic_2lpt.rs:181-240).
__global__ void k_ic_psi2_modes(const float2* __restrict__ src, int n, int nh, int nhp, float2* __restrict__ spec3,
                                int64_t comp_stride) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t total = (int64_t)n * n * nhp;
  if (i >= total) return;
  const int kx = (int)(i % nhp), y = (int)((i / nhp) % n), z = (int)(i / ((int64_t)n * nhp));
  if (kx >= nh) return;
  const int nx = kx, ny = mode_int(y, n), nz = mode_int(z, n), half = n / 2;
  const float n2 = (float)(nx * nx + ny * ny + nz * nz);
  float2 out[3] = {make_float2(0.f, 0.f), make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
  if (n2 > 0.f && nx != half && abs(ny) != half && abs(nz) != half) {
    const float2 sk = src[i];
    const float na[3] = {(float)nx, (float)ny, (float)nz};
#pragma unroll
    for (int c = 0; c < 3; ++c) out[c] = make_float2(na[c] * sk.y / n2, -na[c] * sk.x / n2);
  }
  for (int c = 0; c < 3; ++c) spec3[c * comp_stride + i] = out[c];
}

// Particles are stored in the mesh's [z][y][x] order (slot = mesh node, so
// reads of the displacement fields and writes of the state coalesce); each
// carries its reference global id gid = ix n^2 + iy n + iz, through which every
// host view of the state is ordered.
__device__ __forceinline__ uint32_t lattice_of(int64_t slot, int n, int ii[3]) {
  ii[0] = (int)(slot % n);
  ii[1] = (int)((slot / n) % n);
  ii[2] = (int)(slot / ((int64_t)n * n));
  return (uint32_t)(((int64_t)ii[0] * n + ii[1]) * n + ii[2]);
}

// Lattice position at the cell centre + Psi1, wrapped; momentum vel1 Psi1
// (ic_zeldovich.rs:726-757).
__global__ void k_ic_particles(int n, double box, double psi_scale, double vel1, const float* __restrict__ psi,
                               int64_t n3, Particles p) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n3) return;
  int ii[3];
  const uint32_t gid = lattice_of(i, n, ii);
  const double d = box / n;
  uint32_t q[3];
  float v[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const double s1 = (double)psi[c * n3 + i] * psi_scale;
    double u = ((ii[c] + 0.5) * d + s1) / box;
    u = u - floor(u);
    q[c] = (uint32_t)((unsigned long long)llrint(u * TWO32) & 0xFFFFFFFFull);
    v[c] = (float)(s1 * vel1);
  }
  p.qx[i] = q[0];
  p.qy[i] = q[1];
  p.qz[i] = q[2];
  p.vx[i] = v[0];
  p.vy[i] = v[1];
  p.vz[i] = v[2];
  const double m = 1.0 / (double)n3;
  p.mass[i] = m;
  p.massf[i] = (float)m;
  p.id[i] = gid;
}

// Second order on top of the first (ic_2lpt.rs:520-548): x += D2/D1^2 Psi2
// as a fixed-point offset (the uint32 sum wraps periodically, as rem_euclid
// does), p += vel2 Psi2.
__global__ void k_ic_add_psi2(int n, double box, double psi2_scale, double d21, double vel2,
                              const float* __restrict__ psi2, int64_t n3, Particles p) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n3) return;
  uint32_t* q[3] = {p.qx, p.qy, p.qz};
  float* v[3] = {p.vx, p.vy, p.vz};
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const double s2 = (double)psi2[c * n3 + i] * psi2_scale;
    q[c][i] += (uint32_t)llrint(d21 * s2 / box * TWO32);
    v[c][i] = (float)((double)v[c][i] + s2 * vel2);
  }
}

// transfer_fn.rs:146-184, :190-199, :222-228 (host, the reference's running sum)
double sigma_sq_unit(double r, double n_s, double om, double ob, double h) {
  const double lk0 = std::log(1e-5), lk1 = std::log(5e2);
  const double dl = (lk1 - lk0) / SIGMA_STEPS;
  double sum = 0.0, fprev = sigma_integrand(1e-5, r, n_s, om, ob, h);
  for (int i = 1; i <= SIGMA_STEPS; ++i) {
    const double f = sigma_integrand(std::exp(lk0 + i * dl), r, n_s, om, ob, h);
    sum += 0.5 * (fprev + f) * dl;
    fprev = f;
  }
  return sum / (2.0 * M_PI * M_PI);
}

}  // namespace

// Growth and momentum factors of a configuration.
struct IcFactors {
  double vel1;   // a^2 f1 H
  double scale;  // D(a_init)/D(1) when rescaled, else 1
  double d21;    // D2/D1^2 = -3/7 Omega_m(a)^(-1/143)
  double vel2;   // a^2 f2 H D2/D1^2, f2 = 2 Omega_m(a)^(6/11)
};

// Spectrum and factors of a configuration (host); false when it is invalid.
bool zeldovich_factors(const tpm_zeldovich* c, IcSpectrum* sp, IcFactors* fa, bool host_sigma8 = true) {
  if (!c || c->n_side < 4 || c->n_side > 1024 || (c->n_side & (c->n_side - 1)) != 0) return false;
  if (c->transfer != 0 && c->transfer != 1) return false;
  if (c->use_2lpt != 0 && c->use_2lpt != 1) return false;
  if (c->transfer == 1 && !(c->omega_m > 0.0 && c->omega_b >= 0.0 && c->h > 0.0 && c->box_size_mpc_h > 0.0))
    return false;
  const double n3 = (double)c->n_side * c->n_side * c->n_side;
  sp->kind = c->transfer;
  sp->n_s = c->spectral_index;
  sp->omega_m = c->omega_m;
  sp->omega_b = c->omega_b;
  sp->h = c->h;
  sp->two_pi_h_over_bsm = c->transfer == 1 ? 2.0 * M_PI * c->h / c->box_size_mpc_h : 0.0;
  sp->inv_sqrt_n3 = 1.0 / std::sqrt(n3);
  sp->amp = c->amplitude;
  if (host_sigma8 && c->transfer == 1 && c->sigma8 > 0.0) {
    const double v = sigma_sq_unit(8.0, c->spectral_index, c->omega_m, c->omega_b, c->h);
    sp->amp = v > 0.0 ? c->sigma8 / std::sqrt(v) : c->sigma8;
  }
  // cosmology.rs:509-520 (H, LCDM), :598-610 (f), :650-666 / :736-742 (CPT92
  // ratio); without cosmology a = 1, Omega_m = 1, Omega_L = 0, H = H0
  double a = 1.0, om = 1.0, ol = 0.0;
  if (c->cosmology) {
    a = c->a_init;
    om = c->omega_m;
    ol = c->omega_lambda;
  }
  if (!(a > 0.0) || !(c->h0 > 0.0)) return false;
  const double hh = c->h0 * std::sqrt(std::max(om / (a * a * a) + ol, 0.0));
  const double om_a = std::max(om / (a * a * a) / ((hh / c->h0) * (hh / c->h0)), 0.0);
  const double f1 = std::pow(om_a, 0.55);
  fa->vel1 = a * a * f1 * hh;
  // ic_2lpt.rs:420-446 (Bouchet et al. 1995 fits)
  const double f2 = 2.0 * std::pow(om_a, 6.0 / 11.0);
  fa->d21 = -3.0 / 7.0 * std::pow(om_a, -1.0 / 143.0);
  fa->vel2 = a * a * f2 * hh * fa->d21;
  fa->scale = 1.0;
  if (c->rescale_to_a_init && c->cosmology) {
    auto growth = [&](double aa) {
      const double a3 = aa * aa * aa, den = om + ol * a3;
      if (den <= 0.0) return aa;
      const double oma = om / den, ola = ol * a3 / den;
      const double br = std::pow(std::max(oma, 0.0), 4.0 / 7.0) - ola + (1.0 + oma / 2.0) * (1.0 + ola / 70.0);
      return br <= 0.0 ? aa : aa * 2.5 * oma / br;
    };
    const double d1 = growth(1.0);
    fa->scale = d1 == 0.0 ? 1.0 : growth(a) / d1;
  }
  return true;
}

// `mesh` is a plan of the solver whose buffers may be overwritten; it is used
// when its mesh is the IC lattice (no allocation), otherwise a temporary plan
// of n_side^3 is made and freed.  Sequence: delta -> Psi1 -> particles; for
// 2LPT then phi_aa -> source, phi_ab -> source, forward transform -> Psi2,
// added to the particles.
void zeldovich_fill(const tpm_zeldovich* c, double box, const Particles& out, cudaStream_t s, PmPlan* mesh) {
  IcSpectrum sp{};
  IcFactors fa{};
  if (!zeldovich_factors(c, &sp, &fa, false)) throw Error(TPM_ERR_INVALID_ARGUMENT, "bad Zel'dovich configuration");
  const int n = c->n_side;
  const bool reuse = mesh && mesh->nm == n && mesh->ncomp >= 3 && mesh->spec3 && mesh->force && mesh->rho &&
                     mesh->spec;
  PmPlan temp;
  PmPlan& plan = reuse ? *mesh : temp;
  try {
    if (!reuse) {
      int dev = 0;
      TPM_CUDA(cudaGetDevice(&dev));
      pm_plan_init(temp, n, box, 0.0, 0u, dev);
    }
    const int64_t nh = n / 2 + 1, plane = (int64_t)n * n * plan.nhp, n3 = (int64_t)n * n * n;
    const unsigned gm = grid_for(plane, 256, 1ll << 30), gp = grid_for(n3, 256, 1ll << 30);
    const double cell_over_n3 = (box / n) / (double)n3;  // rustfft's inverse is unnormalised
    // sigma(|n|) tabulated by |n|^2 in the density buffer (6 n^2 + 16 bytes of
    // its 4 n^3), the sigma_8 amplitude first when asked for
    double* table = reinterpret_cast<double*>(plan.rho);
    const int64_t n2_max = 3ll * (n / 2) * (n / 2);
    double* amp_dev = nullptr;
    if (c->transfer == 1 && c->sigma8 > 0.0) {
      amp_dev = table + n2_max + 1;
      k_ic_sigma8<<<1, 256, 0, s>>>(sp, c->sigma8, amp_dev);
      TPM_LAUNCH_CHECK();
    }
    k_ic_sigma_table<<<grid_for(n2_max + 1, 256, 1ll << 30), 256, 0, s>>>(sp, amp_dev, n2_max, table);
    TPM_LAUNCH_CHECK();
    // first order; delta kept in the spectrum work array for the second
    k_ic_modes<<<gm, 256, 0, s>>>(n, (int)nh, plan.nhp, c->seed, table, plan.spec3, plane, c->use_2lpt ? plan.spec : nullptr);
    TPM_LAUNCH_CHECK();
    pm_inverse_components(plan, 3, s);
    k_ic_particles<<<gp, 256, 0, s>>>(n, box, cell_over_n3 * fa.scale, fa.vel1, plan.force, n3, out);
    TPM_LAUNCH_CHECK();
    if (c->use_2lpt) {
      const float inv_n3 = (float)(1.0 / (double)n3);
      for (int off = 0; off < 2; ++off) {
        k_ic_phi_ab<<<gm, 256, 0, s>>>(plan.spec, n, (int)nh, plan.nhp, plan.spec3, plane, off);
        TPM_LAUNCH_CHECK();
        pm_inverse_components(plan, 3, s);
        k_ic_source<<<gp, 256, 0, s>>>(plan.force, plan.rho, n3, inv_n3, off);
        TPM_LAUNCH_CHECK();
      }
      pm_forward_real(plan, s);  // S(k) replaces delta in the work array
      k_ic_psi2_modes<<<gm, 256, 0, s>>>(plan.spec, n, (int)nh, plan.nhp, plan.spec3, plane);
      TPM_LAUNCH_CHECK();
      pm_inverse_components(plan, 3, s);
      k_ic_add_psi2<<<gp, 256, 0, s>>>(n, box, cell_over_n3 * fa.scale * fa.scale, fa.d21, fa.vel2, plan.force, n3,
                                       out);
      TPM_LAUNCH_CHECK();
    }
    TPM_CUDA(cudaStreamSynchronize(s));
    pm_check(plan, s);
  } catch (...) {
    if (!reuse) pm_plan_free(temp);
    throw;
  }
  if (!reuse) pm_plan_free(temp);
}

}  // namespace tpm

extern "C" int tpm_zeldovich_sigma(const tpm_zeldovich* c, const double* n_abs, int64_t count, double* sigma,
                                   double* factors) {
  tpm::IcSpectrum sp{};
  tpm::IcFactors fa{};
  if (!tpm::zeldovich_factors(c, &sp, &fa) || count < 0 || (count > 0 && (!n_abs || !sigma)))
    return TPM_ERR_INVALID_ARGUMENT;
  for (int64_t i = 0; i < count; ++i) sigma[i] = tpm::ic_sigma(sp, n_abs[i]);
  if (factors) {
    factors[0] = sp.amp;
    factors[1] = fa.vel1;
    factors[2] = fa.scale;
    factors[3] = fa.d21;
    factors[4] = fa.vel2;
  }
  return TPM_OK;
}
