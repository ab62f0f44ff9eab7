// Long-range PM: CIC deposit, 3D FFT Poisson solve with the Gaussian
// long-range filter and spectral gradient, CIC gather fused with the kick.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace tpm {

struct PmPlan {
  int nm = 0, logn = 0, nh = 0;
  int nhp = 0;                // row pitch of the half spectra: nh rounded up to even (16-byte rows, for TMA)
  double box = 0.0;
  float2* twiddle = nullptr;  // e^{-2 pi i m / nm}, m < nm/2
  float* kfilter = nullptr;   // per-axis factor of the filter (and CIC deconvolution)
  float* kderiv = nullptr;    // per-axis derivative (exact i k or 4-point), 0 at Nyquist
  float* kval = nullptr;      // per-axis wavenumber k (for k^2)
  float* rho = nullptr;       // nm^3 real, mass per cell
  float2* spec = nullptr;     // nm*nm*nh complex work array
  float2* spec3 = nullptr;    // ncomp x nm*nm*nh
  float* force = nullptr;     // ncomp x nm^3 real, per unit G: -dphi/dx, -dphi/dy, -dphi/dz [, phi]
  int ncomp = 3;              // 4 keeps the long-range potential itself (learned short range)
  float kcoef = 0.f;          // -4 pi / V_cell / N^3
  uint32_t* err = nullptr;    // device status word (DEV_ERR_TMA_TIMEOUT)
  // TMA tensor maps (CUtensorMap, 128 bytes each) of the half spectra as
  // [comp * nm + z][y][kx] arrays of 8-byte complex values: spec and spec3,
  // each with a y-pencil box (CTX x rows x 1) and a z-pencil box (CTX x 1 x rows)
  alignas(64) unsigned char tmap[4][128];
};

// Build tables for mesh nm, box L, split r_s (<= 0: no filter), flags
// (bit 1 CIC deconvolution, bit 2 four-point gradient, bit 6 keep phi).
void pm_plan_init(PmPlan& p, int nm, double box, double r_split, uint32_t flags, int device);
void pm_plan_free(PmPlan& p);
// Throws if a transform pass recorded an error (a TMA wait past its time limit).
void pm_check(const PmPlan& p, cudaStream_t s);

struct GatherArgs {
  int64_t n;
  const uint32_t* qx;
  const uint32_t* qy;
  const uint32_t* qz;
  const float* srx;  // short range (physical, per unit G); may be null
  const float* sry;
  const float* srz;
  float* ax;  // total acceleration out
  float* ay;
  float* az;
  float* lrx;  // long-range part out (optional)
  float* lry;
  float* lrz;
  float* vx;  // kick target (optional)
  float* vy;
  float* vz;
  double g;
  double kick;
};

// CIC deposit of particles [0, n) into p.rho (cleared first); with `id`,
// only the particles whose id is below id_limit (the owned ones) deposit.
void pm_deposit(const PmPlan& p, const uint32_t* qx, const uint32_t* qy, const uint32_t* qz, const float* massf,
                int64_t n, cudaStream_t s, const uint32_t* id = nullptr, uint32_t id_limit = 0xFFFFFFFFu);
void pm_solve(const PmPlan& p, cudaStream_t s);
void pm_gather_kick(const PmPlan& p, const GatherArgs& a, cudaStream_t s);
void pm_cells(const PmPlan& p, const uint32_t* qx, const uint32_t* qy, const uint32_t* qz, const uint32_t* id,
              int64_t n, int32_t* cells_by_id, cudaStream_t s);

struct Particles;

// z-slab decomposition of the PM solve over `ranks` processes (slab_fft.rs
// :209-330): rank r owns z planes [r nzl, (r+1) nzl) of the density and the
// force meshes and, between the two transposes, y rows [r nyl, (r+1) nyl) of
// the half spectrum with every z.  The caller moves the buffers between the
// ranks (reduce-scatter of the density into `rho`, two equal-split
// all-to-alls from `send` into `recv`, all-gather of `force`).
struct PmSlab {
  int rank = 0, ranks = 0, nzl = 0, nyl = 0, ncomp = 3;
  float* rho = nullptr;     // nzl x nm x nm: this rank's planes of the summed density
  float2* spec = nullptr;   // nzl x nm x nhp: after the x and y passes
  float2* send = nullptr;   // transpose send buffer (ncomp x nm x nyl x nhp)
  float2* recv = nullptr;   // transpose receive buffer, same size
  float2* t3 = nullptr;     // ncomp x nm x nyl x nhp: force spectra, [z][y - y0][kx]
  float2* spec3 = nullptr;  // ncomp x nzl x nm x nhp: force spectra of this rank's planes
  float* force = nullptr;   // ncomp x nzl x nm x nm: force slabs, per unit G
  size_t send_bytes = 0;    // bytes of one transpose (every rank sends and receives as many)
  alignas(64) unsigned char tmap[3][128];  // spec y pencils, spec3 y pencils, recv z pencils
};
void pm_slab_init(PmSlab& sl, const PmPlan& p, int rank, int ranks);
void pm_slab_free(PmSlab& sl);
// x and y passes of this rank's density planes, then the forward transpose's send buffer.
void pm_slab_forward(const PmPlan& p, const PmSlab& sl, cudaStream_t s);
// After the forward all-to-all: z passes with the Green's function, filter
// and gradient on the received y rows, then the return transpose's send buffer.
void pm_slab_poisson(const PmPlan& p, const PmSlab& sl, cudaStream_t s);
// After the return all-to-all: inverse y and x passes into the force slabs.
void pm_slab_inverse(const PmPlan& p, const PmSlab& sl, cudaStream_t s);

// Unnormalised forward 3D transform of the real field p.rho into the half
// spectrum p.spec ([z][y][kx], kx <= nm/2, row pitch nhp).
void pm_forward_real(const PmPlan& p, cudaStream_t s);

// Unnormalised inverse 3D transforms of the first ncomp half spectra in
// spec3 ([z][y][kx] each, row pitch nhp) into the real grids
// force[c * nm^3 + (z nm + y) nm + x].
void pm_inverse_components(const PmPlan& p, int ncomp, cudaStream_t s);

// Power spectrum of power_spectrum.rs: CIC assignment (from float64 positions
// pos, or from fixed-point q when pos is null), the plan's FFT passes, shells
// of |k|.  pk_sum / pk_n: device scratch of nm/2; outputs (host, nm/2 each):
// k, P(k) (0 where a shell has no modes) and the mode counts.  Overwrites the
// plan's density and spectrum work arrays.
void pm_power_spectrum(const PmPlan& p, const double* pos, const uint32_t* qx, const uint32_t* qy,
                       const uint32_t* qz, const double* mass, int64_t n, double total_mass, double* pk_sum,
                       unsigned long long* pk_n, double* k_out, double* pk_out, unsigned long long* n_out,
                       cudaStream_t s);

}  // namespace tpm
