// Host orchestration of one TreePM force evaluation and the C ABI.
//
// One handle = one solver (TreePmSolver / PmSolver of the reference) on one
// device and one stream, with device-resident particle state.  A force
// evaluation runs: bounding box -> octant-path keys -> radix sort -> particle
// permutation -> radix tree -> octree -> bit-exact moments -> walk groups ->
// short-range walk -> CIC deposit -> FFT Poisson -> gather (+ kick).  A
// domain-decomposed step runs the same stages in three calls around the
// caller's density all-reduce, with halo copies of other ranks' particles
// resident for one evaluation.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <thread>
#include <vector>

#include "../../include/treepm_b200.h"
#include "cnn_api.h"
#include "common.cuh"
#include "domain.cuh"
#include "learned.cuh"
#include "pm.cuh"
#include "scan.cuh"
#include "snapshot.cuh"
#include "sort.cuh"
#include "tree.cuh"
#include "walk.cuh"

namespace tpm {
thread_local unsigned long long g_kernel_launches = 0;
void zeldovich_fill(const tpm_zeldovich* c, double box, const Particles& out, cudaStream_t s, PmPlan* mesh);
}

using namespace tpm;

namespace {

constexpr int STACK_CAP = 2048;
constexpr uint32_t DEFERRED_CAP = 1u << 16;

__global__ void k_encode(const double* __restrict__ pos, const double* __restrict__ vel,
                         const double* __restrict__ mass, int64_t n, double box, Particles p,
                         uint32_t* __restrict__ err) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  uint32_t q[3];
  for (int d = 0; d < 3; ++d) {
    const double x = pos[3 * i + d];
    if (!isfinite(x)) atomicOr(err, DEV_ERR_NONFINITE);
    double u = x / box;
    u = u - floor(u);
    q[d] = (uint32_t)((unsigned long long)llrint(u * TWO32) & 0xFFFFFFFFull);
  }
  p.qx[i] = q[0];
  p.qy[i] = q[1];
  p.qz[i] = q[2];
  p.vx[i] = vel ? (float)vel[3 * i] : 0.f;
  p.vy[i] = vel ? (float)vel[3 * i + 1] : 0.f;
  p.vz[i] = vel ? (float)vel[3 * i + 2] : 0.f;
  const double m = mass[i];
  if (!isfinite(m)) atomicOr(err, DEV_ERR_NONFINITE);
  p.mass[i] = m;
  p.massf[i] = (float)m;
  p.id[i] = (uint32_t)i;
}

// Does the staged host state (positions, velocities, masses by original
// index) equal the resident state?  Clears *same on any difference.
// Host-buffer steps: are this call's inputs (pin, vin, min; original order)
// bit for bit the state the previous call returned (prev: positions then
// momenta, original order) with the resident masses?
__global__ void k_match_returned(const double* __restrict__ pin, const double* __restrict__ vin,
                                 const double* __restrict__ min, const double* __restrict__ prev, int64_t n,
                                 Particles p, uint32_t* __restrict__ same) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t o = p.id[i];
  bool eq = min[o] == p.mass[i];
  const unsigned long long* a = reinterpret_cast<const unsigned long long*>(pin);
  const unsigned long long* b = reinterpret_cast<const unsigned long long*>(vin);
  const unsigned long long* c = reinterpret_cast<const unsigned long long*>(prev);
  for (int d = 0; d < 3; ++d) {
    eq = eq && a[3 * i + d] == c[3 * i + d];
    eq = eq && b[3 * i + d] == c[3 * n + 3 * i + d];
  }
  if (!eq) atomicAnd(same, 0u);
}

__global__ void k_sum_mass(const double* __restrict__ m, int64_t n, double* __restrict__ out) {
  double s = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    s += m[i];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(out, s);
}

__global__ void k_decode_state(Particles p, int64_t n, double scale, const float* ax, const float* ay,
                               const float* az, double* pos, double* vel, double* acc) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const int64_t o = 3 * (int64_t)p.id[i];
  if (pos) {
    pos[o] = decode(p.qx[i], scale);
    pos[o + 1] = decode(p.qy[i], scale);
    pos[o + 2] = decode(p.qz[i], scale);
  }
  if (vel) {
    vel[o] = p.vx[i];
    vel[o + 1] = p.vy[i];
    vel[o + 2] = p.vz[i];
  }
  if (acc) {
    acc[o] = ax[i];
    acc[o + 1] = ay[i];
    acc[o + 2] = az[i];
  }
}

// out[id] = (x, y, z) * mul for the particles with id < limit (halo copies have none)
__global__ void k_scatter_xyz(const uint32_t* __restrict__ id, int64_t n, const float* x, const float* y,
                              const float* z, double mul, double* out, uint32_t limit = 0xFFFFFFFFu) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n || id[i] >= limit) return;
  const int64_t o = 3 * (int64_t)id[i];
  out[o] = x[i] * mul;
  out[o + 1] = y[i] * mul;
  out[o + 2] = z[i] * mul;
}

__global__ void k_inverse_perm(const uint32_t* __restrict__ id, int64_t n, uint32_t* __restrict__ inv) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n) inv[id[i]] = (uint32_t)i;
}

__global__ void k_pick(const uint32_t* __restrict__ inv, const uint64_t* __restrict__ idx, int64_t m,
                       const float* ax, const float* ay, const float* az, double* out) {
  int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (k >= m) return;
  const uint32_t s = inv[idx[k]];
  out[3 * k] = ax[s];
  out[3 * k + 1] = ay[s];
  out[3 * k + 2] = az[s];
}

__global__ void k_kick_drift(Particles p, int64_t n, const float* __restrict__ ax, const float* __restrict__ ay,
                             const float* __restrict__ az, float kick, double drift_q) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float vx = fmaf(ax[i], kick, p.vx[i]);
  const float vy = fmaf(ay[i], kick, p.vy[i]);
  const float vz = fmaf(az[i], kick, p.vz[i]);
  p.vx[i] = vx;
  p.vy[i] = vy;
  p.vz[i] = vz;
  // x += v * drift, then wrap into the box (exact modulo 2^32 in fixed point)
  p.qx[i] += (uint32_t)(int64_t)llrint((double)vx * drift_q);
  p.qy[i] += (uint32_t)(int64_t)llrint((double)vy * drift_q);
  p.qz[i] += (uint32_t)(int64_t)llrint((double)vz * drift_q);
}

__global__ void k_scatter_u64(const uint32_t* __restrict__ id, int64_t n, const uint64_t* __restrict__ in,
                              uint64_t* __restrict__ out, uint32_t* __restrict__ vals) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[id[i]] = in[i];
  vals[i] = (uint32_t)i;
}

__global__ void k_export_nodes(int64_t n, int64_t n_int, double scale, const uint8_t* o_depth,
                               const double* o_mass, const double* o_com, const double* o_quad,
                               const uint8_t* leaf_depth, Particles p, int32_t* depth, double* mass, double* com,
                               double* quad, int64_t* particle) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n_int + n) return;
  if (i < n_int) {
    depth[i] = o_depth[i];
    mass[i] = o_mass[i];
    for (int d = 0; d < 3; ++d) com[3 * i + d] = o_com[3 * i + d];
    for (int k = 0; k < 6; ++k) quad[6 * i + k] = o_quad[6 * i + k];
    particle[i] = -1;
  } else {
    const int64_t j = i - n_int;
    depth[i] = leaf_depth ? leaf_depth[j] : 0;
    mass[i] = p.mass[j];
    com[3 * i] = decode(p.qx[j], scale);
    com[3 * i + 1] = decode(p.qy[j], scale);
    com[3 * i + 2] = decode(p.qz[j], scale);
    for (int k = 0; k < 6; ++k) quad[6 * i + k] = 0.0;
    particle[i] = p.id[j];
  }
}

// LambdaCDM cosmology (crates/gadget-ng-core/src/cosmology.rs:150-233), FP64.
struct Cosmo {
  double om, ol, h0;
  double da_dt(double a) const {
    double h_sq = (om + 0.0) / (a * a * a) + ol;
    return a * h0 * std::sqrt(std::max(h_sq, 0.0));
  }
  double advance_a(double a, double dt) const {
    double k1 = da_dt(a);
    double k2 = da_dt(a + 0.5 * dt * k1);
    double k3 = da_dt(a + 0.5 * dt * k2);
    double k4 = da_dt(a + dt * k3);
    return a + dt / 6.0 * (k1 + 2.0 * k2 + 2.0 * k3 + k4);
  }
};

}  // namespace

struct tpm_handle {
  tpm_config cfg{};
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  double r_s = 0, r_cut = 0, rc2 = 0, thr = 0;
  bool periodic = true, pm_only = false;
  std::string err;
  int64_t n = 0, cap = 0;
  // particles with id < n_owned are this rank's; the rest (n - n_owned) are
  // halo copies of other ranks' particles for one domain-decomposed evaluation
  int64_t n_owned = 0;
  Particles P[2]{};
  int cur = 0;
  float *ax = nullptr, *ay = nullptr, *az = nullptr;
  float *srx = nullptr, *sry = nullptr, *srz = nullptr;
  float *lrx = nullptr, *lry = nullptr, *lrz = nullptr;
  uint32_t* pcounts = nullptr;
  TreeBuffers T{};
  PmPlan pm;
  PmSlab slab;  // z-slab decomposition of the PM solve (domain-decomposed runs)
  void* sort_scratch = nullptr;
  size_t sort_bytes = 0;
  void* scan_scratch = nullptr;
  uint32_t* stack = nullptr;
  int walk_grid = 0;
  uint2* deferred = nullptr;
  uint32_t* ndeferred = nullptr;
  unsigned long long* stats_dev = nullptr;
  uint32_t* work = nullptr;
  double* staging = nullptr;  // float64 host-exchange buffer (n x 3 + n)
  size_t staging_elems = 0;
  bool forces_valid = false;
  bool parts_valid = false;  // lr / sr parts and interaction counts match the particle order
  double g_acc = 0, eps2_acc = -1;
  int64_t n_int = 0, n_groups = 0;
  TreeParams params_host{};
  tpm_stats stats{};
  cudaEvent_t ev[10]{};
  // learned short range (TPM_FLAG_LEARNED)
  bool learned = false;
  bool net_attached = false;
  LearnedNet net{};
  double m_total = 0.0;      // total mass (learned path), summed on the device when first needed
  bool m_total_valid = false;
  __nv_bfloat16* vol_a = nullptr;  // (nm + 6)^3 x 16
  __nv_bfloat16* vol_b = nullptr;  // (nm + 4)^3 x 16
  float* octants = nullptr;        // nm^3 x 8 octant masses
  uint8_t* fallback = nullptr;     // per particle: 1 = the tree walk, 0 = the network
  uint32_t* lgrp_first = nullptr;  // walk groups holding fallback particles
  uint32_t* lgrp_size = nullptr;
  uint32_t* lgrp_count = nullptr;
  unsigned long long* learned_count = nullptr;
  double* pk_sum = nullptr;        // power-spectrum shells (nm/2)
  unsigned long long* pk_n = nullptr;
  uint32_t* cell_of = nullptr;     // near field: cell of each particle, particles by cell
  uint32_t* cell_items = nullptr;
  uint32_t* cell_start = nullptr;  // nm^3 + 1
  uint32_t* cell_cursor = nullptr;
  void* cell_scan = nullptr;
  size_t mem_used = 0;
  // every device allocation with its size; `group` 0 = persistent,
  // 1 = sized by the particle capacity, 2 = sized by the octree, 3 = the
  // learned network's buffers, 4 = the host-buffer step's buffers
  struct Alloc {
    void* p;
    size_t bytes;
    int group;
  };
  std::vector<Alloc> allocs;
  bool tree_valid = false;
  bool quad_valid = false;  // the octree's quadrupoles (made for tpm_export_tree only)
  // domain decomposition scratch (sized by the particle capacity)
  uint8_t* owned_mask = nullptr;
  uint64_t* dom_flags = nullptr;
  uint32_t* dom_a = nullptr;
  uint32_t* dom_b = nullptr;
  unsigned long long* dom_counts = nullptr;  // MAX_RANKS, persistent
  uint32_t* dom_bits = nullptr;              // every rank's cell occupancy, MAX_RANKS x 64^3 bits, persistent
  // Host-buffer steps (tpm_kdk_step_host): the state the last call returned
  // (original order; positions then momenta, 6n float64) in two buffers, the
  // inputs of this call (7n) and a flag word; the state version that state
  // belongs to (every change of the resident state or its accelerations bumps
  // `version`), a copy stream and two events.
  double* e2e_out[2] = {nullptr, nullptr};
  double* e2e_in = nullptr;
  uint32_t* e2e_flag = nullptr;
  int e2e_buf = 0;
  uint64_t version = 0, e2e_version = ~0ull;
  // positions and momenta of a few particles as the last host-buffer step
  // returned them (E2E_SAMPLE evenly spaced indices, 6 values each)
  std::vector<double> e2e_sample;
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t ev_pos = nullptr, ev_done = nullptr;
  // state carried between the stages of one force evaluation
  struct Stage {
    int phase = 0;  // 0 idle, 1 sorted + deposited, 2 short range done (domain-decomposed calls)
    unsigned long long launches0 = 0;
    bool use_net = false;
    int64_t walk_groups = 0;
    double eps2 = 0.0;
  } fe;

  template <class T_>
  T_* alloc(size_t count, int group) {
    size_t bytes = count * sizeof(T_);
    if (bytes == 0) bytes = 16;
    if (cfg.memory_cap_bytes > 0 && mem_used + bytes > (size_t)cfg.memory_cap_bytes)
      throw Error(TPM_ERR_OUT_OF_MEMORY, "device memory cap of the handle reached (" +
                                             std::to_string(cfg.memory_cap_bytes) + " bytes)");
    void* p = nullptr;
    TPM_CUDA(cudaMalloc(&p, bytes));
    mem_used += bytes;
    allocs.push_back({p, bytes, group});
    return (T_*)p;
  }
  void release_group(int group) {
    std::vector<Alloc> keep;
    for (const Alloc& a : allocs) {
      if (a.group == group) {
        cudaFree(a.p);
        mem_used -= std::min(mem_used, a.bytes);
      } else {
        keep.push_back(a);
      }
    }
    allocs.swap(keep);
  }
};

namespace {

int fail(tpm_handle* h, const Error& e) {
  if (h) h->err = e.what();
  return e.code ? e.code : TPM_ERR_CUDA;
}

void check_dev_err(tpm_handle* h) {
  if (h->pm.err) pm_check(h->pm, h->stream);
  uint32_t e = 0;
  TPM_CUDA(cudaMemcpyAsync(&e, h->T.err, sizeof(uint32_t), cudaMemcpyDeviceToHost, h->stream));
  TPM_CUDA(cudaStreamSynchronize(h->stream));
  if (!e) return;
  TPM_CUDA(cudaMemsetAsync(h->T.err, 0, sizeof(uint32_t), h->stream));
  if (e & DEV_ERR_NONFINITE) throw Error(TPM_ERR_NONFINITE, "non-finite position or mass");
  if (e & DEV_ERR_COINCIDENT)
    throw Error(TPM_ERR_COINCIDENT, "two particles share a position: the insertion octree cannot separate them");
  if (e & DEV_ERR_TIE_RUN) throw Error(TPM_ERR_COINCIDENT, "too many particles share a 21-level octree cell");
  if (e & DEV_ERR_STACK) throw Error(TPM_ERR_WALK_STACK, "tree-walk stack capacity exceeded");
  if (e & DEV_ERR_DEFERRED) throw Error(TPM_ERR_DEFERRED, "exact-fallback work list overflowed");
  throw Error(TPM_ERR_CUDA, "device error flag " + std::to_string(e));
}

void ensure_capacity(tpm_handle* h, int64_t n) {
  if (n <= h->cap) return;
  h->release_group(4);
  h->e2e_out[0] = h->e2e_out[1] = h->e2e_in = nullptr;
  h->e2e_flag = nullptr;
  h->e2e_version = ~0ull;
  h->release_group(2);
  h->release_group(1);
  TreeBuffers& T = h->T;
  T.cap_int = 0;
  T.cap_groups = 0;
  const int64_t c = n;
  for (int k = 0; k < 2; ++k) {
    Particles& P = h->P[k];
    P.qx = h->alloc<uint32_t>(c, 1);
    P.qy = h->alloc<uint32_t>(c, 1);
    P.qz = h->alloc<uint32_t>(c, 1);
    P.vx = h->alloc<float>(c, 1);
    P.vy = h->alloc<float>(c, 1);
    P.vz = h->alloc<float>(c, 1);
    P.mass = h->alloc<double>(c, 1);
    P.massf = h->alloc<float>(c, 1);
    P.id = h->alloc<uint32_t>(c, 1);
  }
  h->ax = h->alloc<float>(c, 1);
  h->ay = h->alloc<float>(c, 1);
  h->az = h->alloc<float>(c, 1);
  h->srx = h->alloc<float>(c, 1);
  h->sry = h->alloc<float>(c, 1);
  h->srz = h->alloc<float>(c, 1);
  h->lrx = h->alloc<float>(c, 1);
  h->lry = h->alloc<float>(c, 1);
  h->lrz = h->alloc<float>(c, 1);
  h->pcounts = h->alloc<uint32_t>(2 * c, 1);
  T.key_hi = h->alloc<uint64_t>(c, 1);
  T.key_lo = h->alloc<uint64_t>(c, 1);
  T.key_lo_tmp = h->alloc<uint64_t>(c, 1);
  T.perm = h->alloc<uint32_t>(c, 1);
  const int64_t cb = c > 1 ? c - 1 : 1;
  T.bin_left = h->alloc<uint32_t>(cb, 1);
  T.bin_right = h->alloc<uint32_t>(cb, 1);
  T.bin_prefix = h->alloc<int32_t>(cb, 1);
  T.bin_first = h->alloc<uint32_t>(cb, 1);
  T.bin_last = h->alloc<uint32_t>(cb, 1);
  T.bin_parent = h->alloc<int32_t>(cb, 1);
  T.oct_count = h->alloc<uint32_t>(cb, 1);
  T.oct_base = h->alloc<uint32_t>(cb, 1);
  T.leaf_bparent = h->alloc<int32_t>(c, 1);
  T.leaf_oparent = h->alloc<int32_t>(c, 1);
  T.leaf_depth = h->alloc<uint8_t>(c, 1);
  h->sort_bytes = radix_sort_scratch_bytes(c);
  h->sort_scratch = h->alloc<char>(h->sort_bytes, 1);
  h->scan_scratch = h->alloc<char>(scan_scratch_bytes(4 * c + 16), 1);
  if (h->learned) {
    h->cell_of = h->alloc<uint32_t>(c, 1);
    h->cell_items = h->alloc<uint32_t>(c, 1);
    h->fallback = h->alloc<uint8_t>(c, 1);
    h->lgrp_first = h->alloc<uint32_t>(c + 1, 1);
    h->lgrp_size = h->alloc<uint32_t>(c + 1, 1);
  }
  h->owned_mask = h->alloc<uint8_t>(c, 1);
  h->dom_flags = h->alloc<uint64_t>(c, 1);
  h->dom_a = h->alloc<uint32_t>(c, 1);
  h->dom_b = h->alloc<uint32_t>(c, 1);
  h->staging_elems = (size_t)9 * c + 1;  // positions, velocities, accelerations (n x 3 float64 each), a scratch word
  h->staging = h->alloc<double>(h->staging_elems, 1);
  h->cap = n;
}

// The accurate walk with the relative opening criterion ([gravity]
// opening_criterion = "relative").
bool relative_mac(const tpm_handle* h) {
  return (h->cfg.flags & TPM_FLAG_ACCURATE) && h->cfg.opening_criterion == 1;
}

void ensure_tree_capacity(tpm_handle* h, int64_t n_int) {
  TreeBuffers& T = h->T;
  if (n_int <= T.cap_int) return;
  h->release_group(2);
  const int64_t c = std::max<int64_t>(n_int + n_int / 8, 1024);
  T.o_parent = h->alloc<int32_t>(c, 2);
  T.o_depth = h->alloc<uint8_t>(c, 2);
  T.o_first = h->alloc<uint32_t>(c, 2);
  T.o_last = h->alloc<uint32_t>(c, 2);
  T.o_slots = h->alloc<uint32_t>(8 * c, 2);
  T.o_nchild = h->alloc<uint32_t>(c, 2);
  T.o_child_first = h->alloc<uint32_t>(c, 2);
  T.o_cnt = h->alloc<uint32_t>(c, 2);
  T.child_ids = h->alloc<uint32_t>(c + h->cap + 8, 2);
  T.o_mass = h->alloc<double>(c, 2);
  T.o_com = h->alloc<double>(3 * c, 2);
  T.o_quad = h->alloc<double>(6 * c, 2);
  T.o_walk = h->alloc<uint4>(c, 2);
  T.o_cell = h->alloc<uint4>(c, 2);
  T.recs = h->alloc<WalkNode>(c + h->cap + 8, 2);
  T.grp_count_per_node = h->alloc<uint32_t>(c, 2);
  T.grp_base = h->alloc<uint32_t>(c, 2);
  T.grp_first = h->alloc<uint32_t>(h->cap + 1, 2);
  T.grp_size = h->alloc<uint32_t>(h->cap + 1, 2);
  T.cap_int = c;
  T.cap_groups = h->cap + 1;
}

float ms_between(cudaEvent_t a, cudaEvent_t b) {
  float ms = 0.f;
  cudaEventElapsedTime(&ms, a, b);
  return ms;
}

double total_mass(tpm_handle* h) {
  if (!h->m_total_valid) {
    double* d = h->staging + h->staging_elems - 1;  // a scratch word at the end of the staging buffer
    TPM_CUDA(cudaMemsetAsync(d, 0, sizeof(double), h->stream));
    k_sum_mass<<<grid_for(h->n, 256, 148 * 8), 256, 0, h->stream>>>(h->P[h->cur].mass, h->n, d);
    TPM_LAUNCH_CHECK();
    TPM_CUDA(cudaMemcpyAsync(&h->m_total, d, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    TPM_CUDA(cudaStreamSynchronize(h->stream));
    h->m_total_valid = true;
  }
  return h->m_total;
}

LearnedMesh learned_mesh_of(tpm_handle* h) {
  LearnedMesh m{};
  m.nm = h->pm.nm;
  m.box = h->cfg.box_size;
  m.m_cell = total_mass(h) / ((double)m.nm * m.nm * m.nm);
  m.rho = h->pm.rho;
  m.phi = h->pm.force + 3 * (int64_t)m.nm * m.nm * m.nm;
  m.octants = h->octants;
  m.vol_a = h->vol_a;
  m.vol_b = h->vol_b;
  return m;
}

// Exact near-field short range (radius near_cells cells, default: the
// attached network's) of the resident particles into (nx, ny, nz); targets
// with skip[i] != 0 are left untouched.
void near_of(tpm_handle* h, double eps2, const uint8_t* skip, float* nx, float* ny, float* nz,
             float near_cells = -1.f) {
  const Particles& P = h->P[h->cur];
  const int nm = h->pm.nm;
  const double box = h->cfg.box_size;
  cell_list(P.qx, P.qy, P.qz, h->n, nm, box, h->cell_of, h->cell_cursor, h->cell_start, h->cell_items, h->cell_scan,
            h->stream);
  NearField f{};
  f.n = h->n;
  f.qx = P.qx;
  f.qy = P.qy;
  f.qz = P.qz;
  f.mass = P.massf;
  f.nm = nm;
  f.box = box;
  f.cell_of = h->cell_of;
  f.start = h->cell_start;
  f.items = h->cell_items;
  f.skip = skip;
  f.r_near = (near_cells >= 0.f ? near_cells : h->net.near_cells) * box / nm;
  f.r_split = h->r_s;
  f.eps2 = eps2;
  f.nx = nx;
  f.ny = ny;
  f.nz = nz;
  near_field(f, h->stream);
}

// The stages of one force evaluation of the resident particles.
// fe_sort: events, keys and sort (tree solvers).
void fe_sort(tpm_handle* h) {
  cudaStream_t s = h->stream;
  const int64_t n = h->n;
  if (n == 0) throw Error(TPM_ERR_NOT_READY, "no particles set");
  TreeBuffers& T = h->T;
  const double box = h->cfg.box_size;
  h->fe.launches0 = g_kernel_launches;
  TPM_CUDA(cudaEventRecord(h->ev[0], s));
  TPM_CUDA(cudaMemsetAsync(h->stats_dev, 0, 8 * sizeof(unsigned long long), s));
  const bool need_tree = !h->pm_only;
  h->fe.use_net = need_tree && h->learned && h->net_attached;
  h->fe.walk_groups = 0;
  h->tree_valid = false;
  if (need_tree) {
    launch_bbox_root(h->P[h->cur], n, box, T, s);
    launch_tree_keys(h->P[h->cur], n, box, T, s);
    TPM_CUDA(cudaEventRecord(h->ev[1], s));
    radix_sort_u64(T.key_hi, T.perm, n, 63, h->sort_scratch, h->sort_bytes, s);
    launch_fix_ties(h->P[h->cur], n, box, T, s);
    launch_permute(h->P[h->cur], h->P[1 - h->cur], n, T.perm, s);
    h->cur = 1 - h->cur;
    TPM_CUDA(cudaEventRecord(h->ev[2], s));
  } else {
    TPM_CUDA(cudaEventRecord(h->ev[1], s));
    TPM_CUDA(cudaEventRecord(h->ev[2], s));
  }
}

// fe_tree_walk: octree, moments, walk groups and the short-range walk (the
// learned path also runs its mesh stages here).  only: per sorted particle,
// 1 = a walk target (null: all).
void fe_tree_walk(tpm_handle* h, double eps2, const uint8_t* only) {
  cudaStream_t s = h->stream;
  const int64_t n = h->n;
  TreeBuffers& T = h->T;
  const double box = h->cfg.box_size;
  const bool need_tree = !h->pm_only;
  const bool use_net = h->fe.use_net;
  int64_t walk_groups = 0;
  h->fe.eps2 = eps2;
  if (need_tree) {
    // ---- tree
    h->n_int = 0;
    if (n >= 2) {
      TPM_CUDA(cudaMemsetAsync(T.scalars, 0, 4 * sizeof(uint32_t), s));
      launch_karras(n, T, s);
      exclusive_scan_u32(T.oct_count, T.oct_base, n - 1, &T.scalars[0], h->scan_scratch, s);
      uint32_t sc[4];
      TPM_CUDA(cudaMemcpyAsync(sc, T.scalars, sizeof(sc), cudaMemcpyDeviceToHost, s));
      TPM_CUDA(cudaMemcpyAsync(&h->params_host, T.params, sizeof(TreeParams), cudaMemcpyDeviceToHost, s));
      TPM_CUDA(cudaStreamSynchronize(s));
      h->n_int = sc[0];
      ensure_tree_capacity(h, h->n_int);
      launch_octree_nodes(n, T, s);
      launch_octree_links(n, h->n_int, T, h->scan_scratch, s);
      // the accurate walk's relative opening criterion reads |Q|_F and the
      // cell centres: the quadrupole pass runs only for it
      const bool rel = relative_mac(h);
      launch_aggregate(h->P[h->cur], n, h->n_int, box, T, s, rel);
      h->quad_valid = rel;
      if (rel) launch_cell_q(h->n_int, box, T, s);
      launch_walk_records(h->P[h->cur], n, h->n_int, h->thr, T, s);
      launch_groups(n, h->n_int, walk_targets_per_warp(), T, h->scan_scratch, s);
      TPM_CUDA(cudaMemcpyAsync(sc, T.scalars, sizeof(sc), cudaMemcpyDeviceToHost, s));
      TPM_CUDA(cudaStreamSynchronize(s));
      h->n_groups = sc[1];
      h->stats.max_tree_depth = (int32_t)sc[2];
    } else {
      TPM_CUDA(cudaMemcpyAsync(&h->params_host, T.params, sizeof(TreeParams), cudaMemcpyDeviceToHost, s));
      TPM_CUDA(cudaStreamSynchronize(s));
      h->n_groups = 0;
    }
    h->tree_valid = true;
    TPM_CUDA(cudaEventRecord(h->ev[3], s));
    walk_groups = h->n_groups;
    if (use_net) {
      // the network and the dense-cell mask read the mesh: long range first
      const Particles& P = h->P[h->cur];
      pm_deposit(h->pm, P.qx, P.qy, P.qz, P.massf, n, s);
      pm_solve(h->pm, s);
      TPM_CUDA(cudaEventRecord(h->ev[7], s));
      const LearnedMesh lm = learned_mesh_of(h);
      octant_deposit(P.qx, P.qy, P.qz, P.massf, n, lm.nm, box, h->octants, s);
      learned_mesh(h->net, lm, T.err, s);
      TPM_CUDA(cudaMemsetAsync(h->learned_count, 0, sizeof(unsigned long long), s));
      learned_mask(P.qx, P.qy, P.qz, n, h->net, lm, h->fallback, h->learned_count, s);
      if (h->net.near_cells > 0.f) {  // exact pairs below the mesh scale for the network's particles
        near_of(h, eps2, h->fallback, h->srx, h->sry, h->srz);
      }
      learned_groups(T.grp_first, T.grp_size, h->n_groups, h->fallback, h->lgrp_first, h->lgrp_size, h->lgrp_count,
                     s);
      uint32_t ng = 0;
      TPM_CUDA(cudaMemcpyAsync(&ng, h->lgrp_count, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
      TPM_CUDA(cudaStreamSynchronize(s));
      walk_groups = ng;
      TPM_CUDA(cudaEventRecord(h->ev[8], s));
    }
    // ---- short-range walk
    if (n >= 2) {
      const double scale = box / TWO32;
      const double h0 = h->params_host.half;
      const int U = (int)std::lround(std::log2(h->r_cut / scale));
      const double u = std::ldexp(scale, U);
      WalkArgs a{};
      a.n = n;
      a.n_int = h->n_int;
      const Particles& P = h->P[h->cur];
      a.qx = P.qx; a.qy = P.qy; a.qz = P.qz; a.massf = P.massf;
      a.recs = T.recs;
      a.walk = T.o_walk; a.depth = T.o_depth; a.nchild = T.o_nchild; a.child_first = T.o_child_first;
      a.child_ids = T.child_ids; a.o_com = T.o_com; a.leaf_depth = T.leaf_depth;
      a.gfirst = use_net ? h->lgrp_first : T.grp_first;
      a.gsize = use_net ? h->lgrp_size : T.grp_size;
      a.ngroups = walk_groups;
      a.work = h->work;
      a.scale = scale; a.box = box; a.rc2 = h->rc2; a.thr = h->thr; a.h0 = h0;
      a.periodic = h->periodic ? 1 : 0;
      a.u_inv = (float)std::ldexp(1.0, -U);
      a.box_u = (float)std::ldexp(1.0, 32 - U);
      a.h0_u = (float)(h0 / u);
      const double rc2_u = h->rc2 / (u * u);
      a.rc2_lo = (float)(rc2_u * (1.0 - 1e-4));
      a.rc2_hi = (float)(rc2_u * (1.0 + 1e-4));
      // The pair loop's band: near r_cut its FP32 distance carries a relative
      // error below 2.4e-7 (1 + E / r_cut) + 2e-7, E = the widest group the
      // walk accepts (1/16 of the box; coordinates are group-relative floats),
      // since periodic leaves have no half side and monopoles h < 0.1 r_cut;
      // 8 times that (at least 1e-5) leaves every pair the FP32 path could
      // misjudge to the float64 test.  The aperiodic walk's leaves carry their
      // cell's half side (cancellation against it): the node band of 1e-4.
      {
        const double e_over_rc = (box / 16.0) / h->r_cut;
        const double pband = h->periodic ? std::max(1e-5, 8.0 * (2.4e-7 * (1.0 + e_over_rc) + 2e-7)) : 1e-4;
        a.prc2_lo = (float)(rc2_u * (1.0 - pband));
        a.prc2_hi = (float)(rc2_u * (1.0 + pband));
        uint32_t lo_bits, hi_bits;
        std::memcpy(&lo_bits, &a.prc2_lo, 4);
        std::memcpy(&hi_bits, &a.prc2_hi, 4);
        a.prc2_lo_bits = lo_bits;
        a.pband_bits = hi_bits - lo_bits;
      }
      a.grc2_lo = (float)(rc2_u * (1.0 - 4e-4));
      a.grc2_hi = (float)(rc2_u * (1.0 + 4e-4));
      a.eps2_u = (float)(eps2 / (u * u));
      const double cx = u / (std::sqrt(2.0) * h->r_s);
      a.pcx = (float)(0.3275911 * cx);
      a.ex2k = (float)(-(cx * cx) / std::log(2.0));
      const double tq = std::ldexp(4.0, -U);
      a.tiny_u = (float)(tq * tq);
      a.out_scale = (float)(1.0 / (u * u));
      a.accurate = (h->cfg.flags & TPM_FLAG_ACCURATE) ? 1 : 0;
      a.gkc = a.accurate ? (float)(2.0 / std::sqrt(M_PI) * cx) : 0.f;
      {
        const double th = h->cfg.theta > 0.0 ? h->cfg.theta : 0.5;
        a.theta2 = (float)(th * th);
      }
      // relative criterion (octree.rs:769-796): accept a node when the
      // quadrupole estimate g |Q|_F / d^5 is below err_tol times the monopole
      // g M / (d^2 + eps^2).  The reference leaves g out of the quadrupole
      // term, which makes its ratio scale with 1/g and with the length unit;
      // with g on both sides the tolerance is the relative truncation error
      // the reference documents.  With d and eps in walk units and |Q|_F
      // physical: |Q|_F (d^2 + eps^2) < err_tol u^3 M d^5
      a.relative = relative_mac(h) ? 1 : 0;
      a.cellq = T.o_cell;
      a.rel_k = (float)(h->cfg.err_tol_force_acc * u * u * u);
      if (a.accurate) {  // no reference decisions to reproduce: no float64 band, no COM-on-target opening
        a.rc2_lo = a.rc2_hi = (float)rc2_u;
        a.prc2_lo = a.prc2_hi = a.rc2_lo;
        std::memcpy(&a.prc2_lo_bits, &a.prc2_lo, 4);
        a.pband_bits = 0u;
        a.tiny_u = -1.f;
      }
      a.ax = h->srx; a.ay = h->sry; a.az = h->srz;
      a.stats = h->stats_dev; a.err = T.err;
      a.deferred = h->deferred; a.ndeferred = h->ndeferred; a.cap_deferred = DEFERRED_CAP;
      a.stack = h->stack; a.stack_cap = STACK_CAP;
      a.single_target = h->r_cut > 0.2 * box ? 1 : 0;
      a.pcounts = h->pcounts;
      a.only = use_net ? h->fallback : only;
      {
        // a group spans at most L/16 (wider ones are walked target by target),
        // so for a node of cull half side hc the +-L images lie at least
        // 7L/16 - hc away: beyond r_cut once hc < 7L/16 - r_cut (hc <= 2 h)
        const double box_u = std::ldexp(1.0, 32 - U), rc_u = std::sqrt(rc2_u) * 1.001;
        int dimg = 0;
        while (dimg < 64 && !(7.0 / 16.0 * box_u - 2.0 * std::ldexp(a.h0_u, -dimg) > rc_u)) ++dimg;
        a.img_depth = dimg;
      }
      TPM_CUDA(cudaMemsetAsync(h->work, 0, sizeof(uint32_t), s));
      TPM_CUDA(cudaMemsetAsync(h->ndeferred, 0, sizeof(uint32_t), s));
      launch_walk(a, h->walk_grid, s);
      uint32_t nd = 0;
      TPM_CUDA(cudaMemcpyAsync(&nd, h->ndeferred, sizeof(uint32_t), cudaMemcpyDeviceToHost, s));
      TPM_CUDA(cudaStreamSynchronize(s));
      if (nd) launch_deferred(a, std::min(nd, DEFERRED_CAP), s);
      double thr_depth = h0;
      int dstar = 0;
      while (!(thr_depth < h->thr) && dstar < 200) {
        thr_depth = std::ldexp(h0, -(++dstar));
      }
      h->stats.terminal_depth = dstar;
    } else {
      TPM_CUDA(cudaMemsetAsync(h->srx, 0, sizeof(float) * n, s));
      TPM_CUDA(cudaMemsetAsync(h->sry, 0, sizeof(float) * n, s));
      TPM_CUDA(cudaMemsetAsync(h->srz, 0, sizeof(float) * n, s));
    }
    if (use_net) {
      const Particles& P = h->P[h->cur];
      learned_apply(P.qx, P.qy, P.qz, n, h->net, learned_mesh_of(h), h->fallback, h->srx, h->sry, h->srz, s);
    }
  } else {
    TPM_CUDA(cudaEventRecord(h->ev[3], s));
  }
  TPM_CUDA(cudaEventRecord(h->ev[4], s));
  h->fe.walk_groups = walk_groups;
}

// fe_long_range: CIC deposit (unless the caller deposited already), FFT
// Poisson solve, gather fused with the short-range sum and the kick, stats.
void fe_long_range(tpm_handle* h, double g, double kick, bool deposit, bool solve = true) {
  cudaStream_t s = h->stream;
  const int64_t n = h->n;
  const bool use_net = h->fe.use_net;
  const int64_t walk_groups = h->fe.walk_groups;
  const double eps2 = h->fe.eps2;
  const Particles& P = h->P[h->cur];
  if (!use_net) {
    if (deposit) pm_deposit(h->pm, P.qx, P.qy, P.qz, P.massf, n, s);
    if (solve) pm_solve(h->pm, s);
  }
  TPM_CUDA(cudaEventRecord(h->ev[5], s));
  GatherArgs ga{};
  ga.n = n;
  ga.qx = P.qx; ga.qy = P.qy; ga.qz = P.qz;
  ga.srx = h->pm_only ? nullptr : h->srx;
  ga.sry = h->pm_only ? nullptr : h->sry;
  ga.srz = h->pm_only ? nullptr : h->srz;
  ga.ax = h->ax; ga.ay = h->ay; ga.az = h->az;
  ga.lrx = h->lrx; ga.lry = h->lry; ga.lrz = h->lrz;
  if (kick != 0.0) {
    ga.vx = P.vx; ga.vy = P.vy; ga.vz = P.vz;
  }
  ga.g = g;
  ga.kick = kick;
  pm_gather_kick(h->pm, ga, s);
  TPM_CUDA(cudaEventRecord(h->ev[6], s));
  check_dev_err(h);
  unsigned long long st[8];
  TPM_CUDA(cudaMemcpy(st, h->stats_dev, sizeof(st), cudaMemcpyDeviceToHost));
  h->stats.n_particles = n;
  h->stats.n_tree_nodes = h->n_int;
  h->stats.n_groups = h->n_groups;
  h->stats.leaf_pairs = (int64_t)st[0];
  h->stats.monopoles = (int64_t)st[1];
  h->stats.evaluated_pairs = (int64_t)st[2];
  h->stats.exact_fallbacks = (int64_t)st[3];
  h->stats.deferred_opens = (int64_t)st[4];
  h->stats.ms_bbox_keys = ms_between(h->ev[0], h->ev[1]);
  h->stats.ms_sort = ms_between(h->ev[1], h->ev[2]);
  h->stats.ms_build = ms_between(h->ev[2], h->ev[3]);
  if (use_net) {
    unsigned long long nl = 0;
    TPM_CUDA(cudaMemcpy(&nl, h->learned_count, sizeof(nl), cudaMemcpyDeviceToHost));
    h->stats.learned_particles = (int64_t)nl;
    h->stats.walk_groups = walk_groups;
    h->stats.ms_pm = ms_between(h->ev[3], h->ev[7]);
    h->stats.ms_learned = ms_between(h->ev[7], h->ev[8]);
    h->stats.ms_walk = ms_between(h->ev[8], h->ev[4]);
  } else {
    h->stats.learned_particles = 0;
    h->stats.walk_groups = walk_groups;
    h->stats.ms_learned = 0.f;
    h->stats.ms_walk = ms_between(h->ev[3], h->ev[4]);
    h->stats.ms_pm = ms_between(h->ev[4], h->ev[5]);
  }
  h->stats.ms_gather_kick = ms_between(h->ev[5], h->ev[6]);
  h->stats.ms_total = ms_between(h->ev[0], h->ev[6]);
  h->stats.kernel_launches = (int64_t)(g_kernel_launches - h->fe.launches0);
  h->stats.force_evaluations += 1;
  h->forces_valid = true;
  h->parts_valid = true;
  h->g_acc = g;
  h->eps2_acc = eps2;
  h->fe.phase = 0;
  ++h->version;
}

// Drop the halo copies: the owned particles (id < n_owned) move, in their
// current order and with their accelerations, to the front.  The force parts
// and interaction counts of the last evaluation are not carried.
void drop_halos(tpm_handle* h) {
  if (h->n <= h->n_owned) return;
  cudaStream_t s = h->stream;
  const Particles& src = h->P[h->cur];
  const Particles& dst = h->P[1 - h->cur];
  compact_owned(src, dst, h->n, (uint32_t)h->n_owned, h->ax, h->ay, h->az, h->srx, h->sry, h->srz, h->dom_a,
                h->dom_b, h->scan_scratch, s);
  const size_t b = sizeof(float) * (size_t)h->n_owned;
  TPM_CUDA(cudaMemcpyAsync(h->ax, h->srx, b, cudaMemcpyDeviceToDevice, s));
  TPM_CUDA(cudaMemcpyAsync(h->ay, h->sry, b, cudaMemcpyDeviceToDevice, s));
  TPM_CUDA(cudaMemcpyAsync(h->az, h->srz, b, cudaMemcpyDeviceToDevice, s));
  h->cur = 1 - h->cur;
  h->n = h->n_owned;
  h->tree_valid = false;
  h->parts_valid = false;
  h->fe.phase = 0;
  ++h->version;
}

// Grow the particle capacity to at least `need` keeping the resident
// particles [0, n) and their accelerations (through one temporary buffer).
void grow_keeping_state(tpm_handle* h, int64_t need) {
  if (need <= h->cap) return;
  cudaStream_t s = h->stream;
  const int64_t n = h->n;
  const Particles& P = h->P[h->cur];
  const void* src[12] = {P.qx, P.qy, P.qz, P.vx, P.vy, P.vz, P.mass, P.massf, P.id, h->ax, h->ay, h->az};
  const size_t esz[12] = {4, 4, 4, 4, 4, 4, 8, 4, 4, 4, 4, 4};
  size_t total = 0;
  for (int k = 0; k < 12; ++k) total += esz[k] * (size_t)n;
  char* tmp = nullptr;
  if (n > 0) {
    TPM_CUDA(cudaMalloc(&tmp, total));
    size_t off = 0;
    for (int k = 0; k < 12; ++k) {
      TPM_CUDA(cudaMemcpyAsync(tmp + off, src[k], esz[k] * n, cudaMemcpyDeviceToDevice, s));
      off += esz[k] * (size_t)n;
    }
    TPM_CUDA(cudaStreamSynchronize(s));
  }
  try {
    ensure_capacity(h, need + need / 4);
  } catch (...) {
    cudaFree(tmp);
    throw;
  }
  h->cur = 0;
  const Particles& Q = h->P[0];
  void* dst[12] = {Q.qx, Q.qy, Q.qz, Q.vx, Q.vy, Q.vz, Q.mass, Q.massf, Q.id, h->ax, h->ay, h->az};
  size_t off = 0;
  for (int k = 0; k < 12 && n > 0; ++k) {
    TPM_CUDA(cudaMemcpyAsync(dst[k], tmp + off, esz[k] * n, cudaMemcpyDeviceToDevice, s));
    off += esz[k] * (size_t)n;
  }
  TPM_CUDA(cudaStreamSynchronize(s));
  cudaFree(tmp);
  h->tree_valid = false;
}

// One force evaluation of all resident particles (halo copies dropped
// first).  kick != 0 applies v += a * kick in the gather.
void force_eval(tpm_handle* h, double eps2, double g, double kick) {
  drop_halos(h);
  fe_sort(h);
  fe_tree_walk(h, eps2, nullptr);
  fe_long_range(h, g, kick, true);
}

// leapfrog_cosmo_kdk_step on the resident state: the opening half kick with
// the cached acceleration rescaled to this step's coupling, the drift, and a
// force evaluation with the closing half kick fused into the gather.
void kdk_device(tpm_handle* h, double kick_half, double drift, double kick_half2, double eps2, double g) {
  drop_halos(h);
  if (h->n == 0) throw Error(TPM_ERR_NOT_READY, "no particles set");
  if (!h->forces_valid || h->eps2_acc != eps2 || h->g_acc == 0.0) force_eval(h, eps2, g, 0.0);
  const double k1 = kick_half * (g / h->g_acc);
  const Particles& P = h->P[h->cur];
  k_kick_drift<<<grid_for(h->n, 256, 1ll << 30), 256, 0, h->stream>>>(P, h->n, h->ax, h->ay, h->az, (float)k1,
                                                                      drift * TWO32 / h->cfg.box_size);
  TPM_LAUNCH_CHECK();
  force_eval(h, eps2, g, kick_half2);
  h->stats.kernel_launches += 1;  // the kick-drift kernel
}

void upload(tpm_handle* h, const double* pos, const double* vel, const double* mass, int64_t n) {
  if (n < 0 || n >= (int64_t)1 << 31) throw Error(TPM_ERR_INVALID_ARGUMENT, "particle count out of range");
  if (n > 0 && (!pos || !mass)) throw Error(TPM_ERR_INVALID_ARGUMENT, "positions and masses are required");
  ensure_capacity(h, std::max<int64_t>(n, 1));
  h->n = n;
  h->n_owned = n;
  h->cur = 0;
  ++h->version;
  h->forces_valid = false;
  h->m_total_valid = false;
  if (n == 0) return;
  cudaStream_t s = h->stream;
  double* dpos = h->staging;
  double* dmass = h->staging + 3 * n;
  TPM_CUDA(cudaMemcpyAsync(dpos, pos, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, s));
  TPM_CUDA(cudaMemcpyAsync(dmass, mass, sizeof(double) * n, cudaMemcpyHostToDevice, s));
  double* dvel = nullptr;
  if (vel) {
    dvel = h->staging + 4 * n;
    TPM_CUDA(cudaMemcpyAsync(dvel, vel, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, s));
  }
  k_encode<<<grid_for(n, 256, 1ll << 30), 256, 0, s>>>(dpos, dvel, dmass, n, h->cfg.box_size, h->P[0], h->T.err);
  TPM_LAUNCH_CHECK();
  check_dev_err(h);
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
extern "C" {

int tpm_version(void) { return 10000; }

int tpm_create(const tpm_config* cfg, tpm_handle** out) {
  if (!cfg || !out) return TPM_ERR_INVALID_ARGUMENT;
  *out = nullptr;
  tpm_handle* h = new (std::nothrow) tpm_handle();
  if (!h) return TPM_ERR_OUT_OF_MEMORY;
  try {
    h->cfg = *cfg;
    const int nm = cfg->grid_size;
    if (nm < 4 || nm > 1024 || (nm & (nm - 1)) != 0)
      throw Error(TPM_ERR_INVALID_ARGUMENT, "pm_grid_size must be a power of two in [4, 1024]");
    if (!(cfg->box_size > 0.0) || !std::isfinite(cfg->box_size))
      throw Error(TPM_ERR_INVALID_ARGUMENT, "box_size must be positive");
    // accurate mode: a cell holding the target has s/d >= 1/sqrt(3) for any
    // centre of mass inside it, so theta below that never accepts one
    if ((cfg->flags & TPM_FLAG_ACCURATE) && !(cfg->theta == 0.0 || (cfg->theta > 0.0 && cfg->theta < 0.577)))
      throw Error(TPM_ERR_INVALID_ARGUMENT, "accurate mode needs theta in (0, 0.577)");
    if ((cfg->flags & TPM_FLAG_ACCURATE) && cfg->opening_criterion == 1 &&
        !(cfg->err_tol_force_acc > 0.0 && std::isfinite(cfg->err_tol_force_acc)))
      throw Error(TPM_ERR_INVALID_ARGUMENT, "the relative opening criterion needs err_tol_force_acc > 0");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
      cudaGetLastError();
      throw Error(TPM_ERR_NO_DEVICE, "no CUDA device");
    }
    if (cfg->device < 0 || cfg->device >= ndev) throw Error(TPM_ERR_INVALID_ARGUMENT, "device ordinal out of range");
    cudaDeviceProp prop;
    TPM_CUDA(cudaGetDeviceProperties(&prop, cfg->device));
    if (prop.major != 10) throw Error(TPM_ERR_NO_DEVICE, std::string("device is not sm_100: ") + prop.name);
    TPM_CUDA(cudaSetDevice(cfg->device));
    // solver.rs:56-62 (auto r_s = 2.5 cells), :80 (r_cut = 5 r_s)
    h->r_s = cfg->r_split > 0.0 ? cfg->r_split : 2.5 * cfg->box_size / (double)nm;
    const double f = cfg->r_cut_factor > 0.0 ? cfg->r_cut_factor : 5.0;
    h->r_cut = f * h->r_s;
    h->rc2 = h->r_cut * h->r_cut;
    h->thr = 0.1 * std::sqrt(h->rc2);  // short_range.rs:320
    h->periodic = !(cfg->flags & TPM_FLAG_APERIODIC_WALK);
    h->pm_only = (cfg->flags & TPM_FLAG_PM_ONLY) != 0;
    h->learned = (cfg->flags & TPM_FLAG_LEARNED) != 0;
    if (h->learned && h->pm_only) throw Error(TPM_ERR_INVALID_ARGUMENT, "the learned short range needs the TreePM solver");
    if (!(h->r_cut > 0.0) || !std::isfinite(h->r_cut)) throw Error(TPM_ERR_INVALID_ARGUMENT, "r_cut must be positive");
    TPM_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    h->own_stream = true;
    for (auto& e : h->ev) TPM_CUDA(cudaEventCreate(&e));
    h->T.params = h->alloc<TreeParams>(1, 0);
    h->T.bbox = h->alloc<uint32_t>(6, 0);
    h->T.scalars = h->alloc<uint32_t>(8, 0);
    h->T.depth_tab = h->alloc<uint32_t>(3 * DEPTH_BINS + 1, 0);
    h->T.err = h->alloc<uint32_t>(1, 0);
    h->stats_dev = h->alloc<unsigned long long>(8, 0);
    h->work = h->alloc<uint32_t>(1, 0);
    h->dom_counts = h->alloc<unsigned long long>(MAX_RANKS + 8, 0);
    h->lgrp_count = h->alloc<uint32_t>(1, 0);
    if (h->learned) {
      const int64_t nm3 = (int64_t)nm * nm * nm;
      h->cell_start = h->alloc<uint32_t>(nm3 + 1, 0);
      h->cell_cursor = h->alloc<uint32_t>(nm3 + 1, 0);
      h->cell_scan = h->alloc<char>(scan_scratch_bytes(nm3 + 1), 0);
    }
    h->learned_count = h->alloc<unsigned long long>(1, 0);
    h->ndeferred = h->alloc<uint32_t>(1, 0);
    h->deferred = h->alloc<uint2>(DEFERRED_CAP, 0);
    int sms = prop.multiProcessorCount;
    h->walk_grid = sms * walk_blocks_per_sm((cfg->flags & TPM_FLAG_ACCURATE) != 0);
    h->stack = h->alloc<uint32_t>(walk_stack_words(h->walk_grid, STACK_CAP), 0);
    TPM_CUDA(cudaMemset(h->T.err, 0, sizeof(uint32_t)));
    pm_plan_init(h->pm, nm, cfg->box_size, h->pm_only ? 0.0 : h->r_s, cfg->flags, cfg->device);
    h->mem_used += (size_t)nm * nm * nm * 4 * 4 + (size_t)nm * nm * (nm / 2 + 1) * 8 * 4;  // PM meshes
  } catch (const Error& e) {
    int code = e.code;
    delete h;
    (void)code;
    return code ? code : TPM_ERR_CUDA;
  }
  *out = h;
  return TPM_OK;
}

void tpm_destroy(tpm_handle* h) {
  if (!h) return;
  cudaSetDevice(h->cfg.device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  for (const auto& a : h->allocs) cudaFree(a.p);
  pm_slab_free(h->slab);
  pm_plan_free(h->pm);
  for (auto& e : h->ev)
    if (e) cudaEventDestroy(e);
  if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
  if (h->copy_stream) cudaStreamDestroy(h->copy_stream);
  if (h->ev_pos) cudaEventDestroy(h->ev_pos);
  if (h->ev_done) cudaEventDestroy(h->ev_done);
  delete h;
}

const char* tpm_last_error(const tpm_handle* h) { return h ? h->err.c_str() : "null handle"; }

int tpm_set_stream(tpm_handle* h, void* stream) {
  if (!h) return TPM_ERR_INVALID_ARGUMENT;
  try {
    TPM_CUDA(cudaSetDevice(h->cfg.device));
    TPM_CUDA(cudaStreamSynchronize(h->stream));
    if (h->own_stream) cudaStreamDestroy(h->stream);
    h->stream = (cudaStream_t)stream;
    h->own_stream = false;
  } catch (const Error& e) {
    return fail(h, e);
  }
  return TPM_OK;
}

void* tpm_get_stream(const tpm_handle* h) { return h ? (void*)h->stream : nullptr; }

// ---- domain-decomposed TreePM ----------------------------------------------
static_assert(sizeof(tpm_halo_record) == sizeof(HaloRecord), "halo record layout");
static_assert(sizeof(tpm_halo_record) == 24, "halo record size");

int tpm_owned_aabb(tpm_handle* h, double aabb6[6]) {
  if (!h || !aabb6) return TPM_ERR_INVALID_ARGUMENT;
  try {
    TPM_CUDA(cudaSetDevice(h->cfg.device));
    drop_halos(h);
    if (h->n_owned == 0) {  // Aabb3::empty
      for (int d = 0; d < 3; ++d) {
        aabb6[2 * d] = INFINITY;
        aabb6[2 * d + 1] = -INFINITY;
      }
      return TPM_OK;
    }
    uint32_t b[6];
    owned_bounds(h->P[h->cur], h->n_owned, reinterpret_cast<uint32_t*>(h->dom_counts), b, h->stream);
    // decode is monotone, so the bounds of the decoded positions are the
    // decoded bounds (compute_aabb_3d, halo3d.rs)
    const double scale = h->cfg.box_size / TWO32;
    for (int k = 0; k < 6; ++k) aabb6[k] = decode(b[k], scale);
  } catch (const Error& e) {
    return fail(h, e);
  }
  return TPM_OK;
}

int tpm_halo_select(tpm_handle* h, const double* aabbs, int32_t n_ranks, int32_t rank, double width,
                    int64_t* counts, tpm_halo_record* send, int64_t cap) {
  if (!h || !aabbs || !counts || n_ranks < 1 || n_ranks > MAX_RANKS || rank < 0 || rank >= n_ranks ||
      !(width >= 0.0) || cap < 0)
    return TPM_ERR_INVALID_ARGUMENT;
  try {
    TPM_CUDA(cudaSetDevice(h->cfg.device));
    drop_halos(h);
    cudaStream_t s = h->stream;
    AabbTable t{};
    std::memcpy(t.v, aabbs, sizeof(double) * 6 * (size_t)n_ranks);
    const int64_t n = h->n_owned;
    const Particles& P = h->P[h->cur];
    halo_flags(P, n, h->cfg.box_size / TWO32, h->cfg.box_size, t, n_ranks, rank, width * width, h->dom_flags,
               h->dom_counts, s);
    unsigned long long c[MAX_RANKS];
    TPM_CUDA(cudaMemcpyAsync(c, h->dom_counts, sizeof(c), cudaMemcpyDeviceToHost, s));
    TPM_CUDA(cudaStreamSynchronize(s));
    int64_t total = 0;
    for (int r = 0; r < n_ranks; ++r) {
      counts[r] = (int64_t)c[r];
      total += (int64_t)c[r];
    }
    if (!send) return TPM_OK;
    if (total > cap) throw Error(TPM_ERR_INVALID_ARGUMENT, "halo send buffer holds " + std::to_string(cap) +
                                                               " records, " + std::to_string(total) + " selected");
    int64_t off = 0;
    for (int r = 0; r < n_ranks; ++r) {
      if (c[r] == 0) continue;
      halo_pack(P, n, h->dom_flags, r, h->dom_a, h->dom_b, h->scan_scratch,
                reinterpret_cast<HaloRecord*>(send) + off, s);
      off += (int64_t)c[r];
    }
    TPM_CUDA(cudaStreamSynchronize(s));
  } catch (const Error& e) {
    return fail(h, e);
  }
  return TPM_OK;
}

// The occupancy grid for a halo width: cells at least `width` wide, at most
// 64 per axis.
static int occupancy_grid(double box, double width) {
  const double g = width > 0.0 ? std::floor(box / width) : 64.0;
  return (int)std::max(1.0, std::min(64.0, g));
}

int tpm_occupancy(tpm_handle* h, double width, int32_t* grid, uint32_t* bits) {
  if (!h || !grid || !(width >= 0.0)) return TPM_ERR_INVALID_ARGUMENT;
  try {
    TPM_CUDA(cudaSetDevice(h->cfg.device));
    drop_halos(h);
    const int g = occupancy_grid(h->cfg.box_size, width);
    *grid = g;
    if (!bits) return TPM_OK;
    if (!h->dom_bits) h->dom_bits = h->alloc<uint32_t>((size_t)MAX_RANKS * 8192, 0);
    const int64_t words = ((int64_t)g * g * g + 31) / 32;
    occupancy(h->P[h->cur], h->n_owned, g, h->dom_bits, h->stream);
    TPM_CUDA(cudaMemcpyAsync(bits, h->dom_bits, sizeof(uint32_t) * words, cudaMemcpyDeviceToHost, h->stream));
    TPM_CUDA(cudaStreamSynchronize(h->stream));
  } catch (const Error& e) {
    return fail(h, e);
  }
  return TPM_OK;
}

int tpm_halo_select_cells(tpm_handle* h, const uint32_t* bits, int32_t grid, int32_t n_ranks, int32_t rank,
                          double width, int64_t* counts, tpm_halo_record* send, int64_t cap) {
  if (!h || !bits || !counts || n_ranks < 1 || n_ranks > MAX_RANKS || rank < 0 || rank >= n_ranks ||
      !(width >= 0.0) || cap < 0 || grid != occupancy_grid(h->cfg.box_size, width))
    return TPM_ERR_INVALID_ARGUMENT;
  try {
    TPM_CUDA(cudaSetDevice(h->cfg.device));
    drop_halos(h);
    cudaStream_t s = h->stream;
    const int64_t words = ((int64_t)grid * grid * grid + 31) / 32;
    if (!h->dom_bits) h->dom_bits = h->alloc<uint32_t>((size_t)MAX_RANKS * 8192, 0);
    TPM_CUDA(cudaMemcpyAsync(h->dom_bits, bits, sizeof(uint32_t) * words * n_ranks, cudaMemcpyHostToDevice, s));
    const int64_t n = h->n_owned;
    const Particles& P = h->P[h->cur];
    // the halo width with a relative margin of 1e-9 for the float64 face gaps
    const double w2 = width * width * (1.0 + 1e-9);
    halo_flags_cells(P, n, h->cfg.box_size / TWO32, h->cfg.box_size / grid, grid, h->dom_bits, words, n_ranks, rank,
                     w2, h->dom_flags, h->dom_counts, s);
    unsigned long long c[MAX_RANKS];
    TPM_CUDA(cudaMemcpyAsync(c, h->dom_counts, sizeof(c), cudaMemcpyDeviceToHost, s));
    TPM_CUDA(cudaStreamSynchronize(s));
    int64_t total = 0;
    for (int r = 0; r < n_ranks; ++r) {
      counts[r] = (int64_t)c[r];
      total += (int64_t)c[r];
    }
    if (!send) return TPM_OK;
    if (total > cap) throw Error(TPM_ERR_INVALID_ARGUMENT, "halo send buffer holds " + std::to_string(cap) +
                                                               " records, " + std::to_string(total) + " selected");
    int64_t off = 0;
    for (int r = 0; r < n_ranks; ++r) {
      if (c[r] == 0) continue;
      halo_pack(P, n, h->dom_flags, r, h->dom_a, h->dom_b, h->scan_scratch,
                reinterpret_cast<HaloRecord*>(send) + off, s);
      off += (int64_t)c[r];
    }
    TPM_CUDA(cudaStreamSynchronize(s));
  } catch (const Error& e) {
    return fail(h, e);
  }
  return TPM_OK;
}

int tpm_set_halos(tpm_handle* h, const tpm_halo_record* recv, int64_t n) {
  if (!h || n < 0 || (n > 0 && !recv)) return TPM_ERR_INVALID_ARGUMENT;
  try {
    TPM_CUDA(cudaSetDevice(h->cfg.device));
    drop_halos(h);
    if (h->n_owned + n >= ((int64_t)1 << 31)) throw Error(TPM_ERR_INVALID_ARGUMENT, "particle count out of range");
    grow_keeping_state(h, std::max<int64_t>(h->n_owned + n, 1));
    append_halos(h->P[h->cur], h->n_owned, reinterpret_cast<const HaloRecord*>(recv), n, h->stream);
    h->n = h->n_owned + n;
    h->tree_valid = false;
    h->parts_valid = false;
    h->m_total_valid = false;
    ++h->version;
    TPM_CUDA(cudaStreamSynchronize(h->stream));  // the receive buffer is free on return
  } catch (const Error& e) {
    return fail(h, e);
  }
  return TPM_OK;
}

int tpm_force_begin(tpm_handle* h) {
  if (!h) return TPM_ERR_INVALID_ARGUMENT;
  try {
    TPM_CUDA(cudaSetDevice(h->cfg.device));
    if (h->learned) throw Error(TPM_ERR_INVALID_ARGUMENT, "the learned short range runs on one domain only");
    h->fe.phase = 0;
    if (h->n == 0) {  // an empty rank still contributes its (empty) density to the sum
      h->fe.launches0 = g_kernel_launches;
      h->fe.use_net = false;
      TPM_CUDA(cudaMemsetAsync(h->pm.rho, 0, sizeof(float) * (size_t)h->pm.nm * h->pm.nm * h->pm.nm, h->stream));
    } else {
      fe_sort(h);
      const Particles& P = h->P[h->cur];
      pm_deposit(h->pm, P.qx, P.qy, P.qz, P.massf, h->n, h->stream, P.id, (uint32_t)h->n_owned);
    }
    h->fe.phase = 1;
  } catch (const Error& e) {
    return fail(h, e);
  }
  return TPM_OK;
}

int tpm_mesh_density(tpm_handle* h, float** density, int64_t* cells) {
  if (!h || !density || !cells) return TPM_ERR_INVALID_ARGUMENT;
  *density = h->pm.rho;
  *cells = (int64_t)h->pm.nm * h->pm.nm * h->pm.nm;
  return TPM_OK;
}

int tpm_force_short_range(tpm_handle* h, double eps2) {
  if (!h) return TPM_ERR_INVALID_ARGUMENT;
  try {
    TPM_CUDA(cudaSetDevice(h->cfg.device));
    if (h->fe.phase != 1) throw Error(TPM_ERR_NOT_READY, "tpm_force_begin first");
    if (h->n > 0) {
      const uint8_t* only = nullptr;
      if (h->n_owned < h->n) {
        owned_mask(h->P[h->cur].id, h->n, (uint32_t)h->n_owned, h->owned_mask, h->stream);
        only = h->owned_mask;
      }
      fe_tree_walk(h, eps2, only);
    } else {
      h->fe.eps2 = eps2;
    }
    h->fe.phase = 2;
  } catch (const Error& e) {
    return fail(h, e);
  }
  return TPM_OK;
}

static int force_end(tpm_handle* h, double g, double kick, bool solve) {
  if (!h) return TPM_ERR_INVALID_ARGUMENT;
  try {
    TPM_CUDA(cudaSetDevice(h->cfg.device));
    if (h->fe.phase != 2) throw Error(TPM_ERR_NOT_READY, "tpm_force_short_range first");
    if (h->n > 0) {
      fe_long_range(h, g, kick, false, solve);
    } else {
      h->fe.phase = 0;
      h->forces_valid = true;
      h->parts_valid = true;
      h->g_acc = g;
      h->eps2_acc = h->fe.eps2;
    }
  } catch (const Error& e) {
    return fail(h, e);
  }
  return TPM_OK;
}

int tpm_force_end(tpm_handle* h, double g, double kick) { return force_end(h, g, kick, true); }
int tpm_force_end_solved(tpm_handle* h, double g, double kick) { return force_end(h, g, kick, false); }

int tpm_pm_slab_setup(tpm_handle* h, int32_t rank, int32_t ranks, tpm_slab_buffers* out) {
  if (!h || !out) return TPM_ERR_INVALID_ARGUMENT;
  try {
    TPM_CUDA(cudaSetDevice(h->cfg.device));
    if (h->pm_only || h->learned) throw Error(TPM_ERR_INVALID_ARGUMENT, "the slab PM serves the TreePM solver");
    if (ranks < 1 || ranks > MAX_RANKS || rank < 0 || rank >= ranks)
      throw Error(TPM_ERR_INVALID_ARGUMENT, "rank out of range");
    if (h->slab.ranks != ranks || h->slab.rank != rank) pm_slab_init(h->slab, h->pm, rank, ranks);
    const PmSlab& sl = h->slab;
    const int64_t nm = h->pm.nm;
    out->density_slab = sl.rho;
    out->send = sl.send;
    out->recv = sl.recv;
    out->forward_bytes = (int64_t)sl.send_bytes;
    out->return_bytes = (int64_t)sl.send_bytes * sl.ncomp;
    out->force_slab = sl.force;
    out->force_mesh = h->pm.force;
    out->planes = sl.nzl;
    out->slab_cells = (int64_t)sl.nzl * nm * nm;
    out->mesh_cells = nm * nm * nm;
  } catch (const Error& e) {
    return fail(h, e);
  }
  return TPM_OK;
}

static int slab_stage(tpm_handle* h, int stage) {
  if (!h) return TPM_ERR_INVALID_ARGUMENT;
  try {
    TPM_CUDA(cudaSetDevice(h->cfg.device));
    if (h->slab.ranks < 1) throw Error(TPM_ERR_NOT_READY, "tpm_pm_slab_setup first");
    if (stage == 0) pm_slab_forward(h->pm, h->slab, h->stream);
    else if (stage == 1) pm_slab_poisson(h->pm, h->slab, h->stream);
    else pm_slab_inverse(h->pm, h->slab, h->stream);
  } catch (const Error& e) {
    return fail(h, e);
  }
  return TPM_OK;
}
int tpm_pm_slab_forward(tpm_handle* h) { return slab_stage(h, 0); }
int tpm_pm_slab_poisson(tpm_handle* h) { return slab_stage(h, 1); }
int tpm_pm_slab_inverse(tpm_handle* h) { return slab_stage(h, 2); }

int tpm_kick_drift(tpm_handle* h, double kick_half, double drift, double g) {
  if (!h) return TPM_ERR_INVALID_ARGUMENT;
  try {
    TPM_CUDA(cudaSetDevice(h->cfg.device));
    drop_halos(h);
    if (h->n == 0) return TPM_OK;
    if (!h->forces_valid || h->g_acc == 0.0) throw Error(TPM_ERR_NOT_READY, "no forces computed");
    const double k1 = kick_half * (g / h->g_acc);
    const Particles& P = h->P[h->cur];
    k_kick_drift<<<grid_for(h->n, 256, 1ll << 30), 256, 0, h->stream>>>(P, h->n, h->ax, h->ay, h->az, (float)k1,
                                                                        drift * TWO32 / h->cfg.box_size);
    TPM_LAUNCH_CHECK();
    ++h->version;
  } catch (const Error& e) {
    return fail(h, e);
  }
  return TPM_OK;
}

int tpm_particle_counts(const tpm_handle* h, int64_t* n_owned, int64_t* n_resident) {
  if (!h) return TPM_ERR_INVALID_ARGUMENT;
  if (n_owned) *n_owned = h->n_owned;
  if (n_resident) *n_resident = h->n;
  return TPM_OK;
}

int tpm_accelerations_for_indices(tpm_handle* h, const double* pos, const double* mass, int64_t n, double eps2,
                                  double g, const uint64_t* idx, int64_t n_idx, double* out) {
  if (!h) return TPM_ERR_INVALID_ARGUMENT;
  try {
    TPM_CUDA(cudaSetDevice(h->cfg.device));
    if (n_idx < 0 || (n_idx > 0 && (!idx || !out))) throw Error(TPM_ERR_INVALID_ARGUMENT, "bad index arrays");
    for (int64_t k = 0; k < n_idx; ++k)
      if ((int64_t)idx[k] >= n) throw Error(TPM_ERR_INVALID_ARGUMENT, "global index out of range");
    upload(h, pos, nullptr, mass, n);
    if (n_idx == 0) return TPM_OK;
    force_eval(h, eps2, g, 0.0);
    cudaStream_t s = h->stream;
    uint32_t* inv = h->T.perm;  // free after the build
    k_inverse_perm<<<grid_for(n, 256, 1ll << 30), 256, 0, s>>>(h->P[h->cur].id, n, inv);
    TPM_LAUNCH_CHECK();
    uint64_t* didx = (uint64_t*)h->sort_scratch;
    double* dout = h->staging;
    for (int64_t k0 = 0; k0 < n_idx; k0 += n) {  // chunks of at most n indices
      const int64_t m = std::min<int64_t>(n, n_idx - k0);
      TPM_CUDA(cudaMemcpyAsync(didx, idx + k0, sizeof(uint64_t) * m, cudaMemcpyHostToDevice, s));
      k_pick<<<grid_for(m, 256, 1ll << 30), 256, 0, s>>>(inv, didx, m, h->ax, h->ay, h->az, dout);
      TPM_LAUNCH_CHECK();
      TPM_CUDA(cudaMemcpyAsync(out + 3 * k0, dout, sizeof(double) * 3 * m, cudaMemcpyDeviceToHost, s));
    }
    TPM_CUDA(cudaStreamSynchronize(s));
  } catch (const Error& e) {
    return fail(h, e);
  }
  return TPM_OK;
}

int tpm_set_particles(tpm_handle* h, const double* pos, const double* vel, const double* mass, int64_t n) {
  if (!h) return TPM_ERR_INVALID_ARGUMENT;
  try {
    TPM_CUDA(cudaSetDevice(h->cfg.device));
    upload(h, pos, vel, mass, n);
  } catch (const Error& e) {
    return fail(h, e);
  }
  return TPM_OK;
}

int tpm_set_particles_fixed(tpm_handle* h, const uint32_t* q, const float* vel, const double* mass, int64_t n) {
  if (!h) return TPM_ERR_INVALID_ARGUMENT;
  try {
    TPM_CUDA(cudaSetDevice(h->cfg.device));
    if (n <= 0 || !q || !mass) throw Error(TPM_ERR_INVALID_ARGUMENT, "positions and masses are required");
    ensure_capacity(h, n);
    h->n = n;
    h->n_owned = n;
    h->cur = 0;
    ++h->version;
    h->forces_valid = false;
    h->m_total_valid = false;
    cudaStream_t s = h->stream;
    std::vector<uint32_t> tmp((size_t)n);
    Particles& P = h->P[0];
    uint32_t* dst[3] = {P.qx, P.qy, P.qz};
    for (int d = 0; d < 3; ++d) {
      for (int64_t i = 0; i < n; ++i) tmp[i] = q[3 * i + d];
      TPM_CUDA(cudaMemcpyAsync(dst[d], tmp.data(), sizeof(uint32_t) * n, cudaMemcpyHostToDevice, s));
      TPM_CUDA(cudaStreamSynchronize(s));
    }
    std::vector<float> fv((size_t)n);
    float* vd[3] = {P.vx, P.vy, P.vz};
    for (int d = 0; d < 3; ++d) {
      for (int64_t i = 0; i < n; ++i) fv[i] = vel ? vel[3 * i + d] : 0.f;
      TPM_CUDA(cudaMemcpyAsync(vd[d], fv.data(), sizeof(float) * n, cudaMemcpyHostToDevice, s));
      TPM_CUDA(cudaStreamSynchronize(s));
    }
    TPM_CUDA(cudaMemcpyAsync(P.mass, mass, sizeof(double) * n, cudaMemcpyHostToDevice, s));
    for (int64_t i = 0; i < n; ++i) fv[i] = (float)mass[i];
    TPM_CUDA(cudaMemcpyAsync(P.massf, fv.data(), sizeof(float) * n, cudaMemcpyHostToDevice, s));
    std::vector<uint32_t> ids((size_t)n);
    for (int64_t i = 0; i < n; ++i) ids[i] = (uint32_t)i;
    TPM_CUDA(cudaMemcpyAsync(P.id, ids.data(), sizeof(uint32_t) * n, cudaMemcpyHostToDevice, s));
    TPM_CUDA(cudaStreamSynchronize(s));
  } catch (const Error& e) {
    return fail(h, e);
  }
  return TPM_OK;
}

int tpm_compute_forces(tpm_handle* h, double eps2, double g) {
  if (!h) return TPM_ERR_INVALID_ARGUMENT;
  try {
    TPM_CUDA(cudaSetDevice(h->cfg.device));
    force_eval(h, eps2, g, 0.0);
  } catch (const Error& e) {
    return fail(h, e);
  }
  return TPM_OK;
}

int tpm_kdk_step(tpm_handle* h, double kick_half, double drift, double kick_half2, double eps2, double g) {
  if (!h) return TPM_ERR_INVALID_ARGUMENT;
  try {
    TPM_CUDA(cudaSetDevice(h->cfg.device));
    kdk_device(h, kick_half, drift, kick_half2, eps2, g);
  } catch (const Error& e) {
    return fail(h, e);
  }
  return TPM_OK;
}

int tpm_get_state(tpm_handle* h, double* pos, double* vel, double* acc) {
  if (!h) return TPM_ERR_INVALID_ARGUMENT;
  try {
    TPM_CUDA(cudaSetDevice(h->cfg.device));
    // owned particles only (ids below n_owned), read in place: halo copies
    // land past the owned block of each staging area and are not copied
    const int64_t n = h->n, no = h->n_owned;
    if (n == 0) return TPM_OK;
    if (acc && !h->forces_valid) throw Error(TPM_ERR_NOT_READY, "no forces computed");
    cudaStream_t s = h->stream;
    double* dp = h->staging;
    double* dv = h->staging + 3 * n;
    double* da = h->staging + 6 * n;
    k_decode_state<<<grid_for(n, 256, 1ll << 30), 256, 0, s>>>(h->P[h->cur], n, h->cfg.box_size / TWO32, nullptr,
                                                               nullptr, nullptr, pos ? dp : nullptr,
                                                               vel ? dv : nullptr, nullptr);
    TPM_LAUNCH_CHECK();
    if (pos) TPM_CUDA(cudaMemcpyAsync(pos, dp, sizeof(double) * 3 * no, cudaMemcpyDeviceToHost, s));
    if (vel) TPM_CUDA(cudaMemcpyAsync(vel, dv, sizeof(double) * 3 * no, cudaMemcpyDeviceToHost, s));
    TPM_CUDA(cudaStreamSynchronize(s));
    if (acc) {
      double* buf = da;
      k_scatter_xyz<<<grid_for(n, 256, 1ll << 30), 256, 0, s>>>(h->P[h->cur].id, n, h->ax, h->ay, h->az, 1.0, buf,
                                                                (uint32_t)no);
      TPM_LAUNCH_CHECK();
      TPM_CUDA(cudaMemcpyAsync(acc, buf, sizeof(double) * 3 * no, cudaMemcpyDeviceToHost, s));
      TPM_CUDA(cudaStreamSynchronize(s));
    }
  } catch (const Error& e) {
    return fail(h, e);
  }
  return TPM_OK;
}

// A restart from another state (a new initial condition, a rewind) would
// otherwise be stepped speculatively on the resident state first and then
// again from the upload: a few returned values decide it on the host before
// any work is queued.  A match still goes through the full device check.
constexpr int64_t E2E_SAMPLE = 256;
static void e2e_take_sample(tpm_handle* h, const double* pos, const double* vel, int64_t n) {
  h->e2e_sample.resize(6 * E2E_SAMPLE);
  for (int64_t k = 0; k < E2E_SAMPLE; ++k) {
    const int64_t i = k * n / E2E_SAMPLE;
    for (int d = 0; d < 3; ++d) {
      h->e2e_sample[6 * k + d] = pos[3 * i + d];
      h->e2e_sample[6 * k + 3 + d] = vel[3 * i + d];
    }
  }
}
static bool e2e_sample_matches(const tpm_handle* h, const double* pos, const double* vel, int64_t n) {
  if ((int64_t)h->e2e_sample.size() != 6 * E2E_SAMPLE) return false;
  for (int64_t k = 0; k < E2E_SAMPLE; ++k) {
    const int64_t i = k * n / E2E_SAMPLE;
    for (int d = 0; d < 3; ++d)  // bit patterns, as the device check compares them
      if (std::memcmp(&h->e2e_sample[6 * k + d], &pos[3 * i + d], sizeof(double)) != 0 ||
          std::memcmp(&h->e2e_sample[6 * k + 3 + d], &vel[3 * i + d], sizeof(double)) != 0)
        return false;
  }
  return true;
}

int tpm_kdk_step_host(tpm_handle* h, double* pos, double* vel, const double* mass, int64_t n, double kick_half,
                      double drift, double kick_half2, double eps2, double g) {
  if (!h) return TPM_ERR_INVALID_ARGUMENT;
  if (n < 0 || (n > 0 && (!pos || !mass))) return TPM_ERR_INVALID_ARGUMENT;
  // An integrator hands back the state the previous call returned.  When the
  // resident state is still the one returned then (its version) the step runs
  // on it at once, while a copy stream uploads this call's inputs, checks them
  // bit for bit against the returned state and copies the new positions back
  // (final after the drift) during the force evaluation; only the momenta
  // (final after the closing kick) are copied after it.  Inputs that differ
  // are stepped from the upload instead (two force evaluations, as for any
  // new state).
  try {
    TPM_CUDA(cudaSetDevice(h->cfg.device));
    const double scale = h->cfg.box_size / TWO32;
    cudaStream_t s = h->stream;
    // the buffers follow the particle capacity (ensure_capacity releases them)
    auto ensure_buffers = [&]() {
      if (h->e2e_in) return;
      h->e2e_out[0] = h->alloc<double>(6 * (size_t)h->cap, 4);
      h->e2e_out[1] = h->alloc<double>(6 * (size_t)h->cap, 4);
      h->e2e_in = h->alloc<double>(7 * (size_t)h->cap, 4);
      h->e2e_flag = h->alloc<uint32_t>(4, 4);
      h->e2e_version = ~0ull;
    };
    if (!h->copy_stream) TPM_CUDA(cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking));
    if (!h->ev_pos) TPM_CUDA(cudaEventCreateWithFlags(&h->ev_pos, cudaEventDisableTiming));
    if (!h->ev_done) TPM_CUDA(cudaEventCreateWithFlags(&h->ev_done, cudaEventDisableTiming));
    cudaStream_t c = h->copy_stream;
    // the state after a step, decoded into output buffer b and copied to the host
    auto return_state = [&](int b) {
      double* out = h->e2e_out[b];
      const Particles& P = h->P[h->cur];
      k_decode_state<<<grid_for(n, 256, 1ll << 30), 256, 0, s>>>(P, n, scale, nullptr, nullptr, nullptr, out,
                                                                 out + 3 * n, nullptr);
      TPM_LAUNCH_CHECK();
      TPM_CUDA(cudaMemcpyAsync(pos, out, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, s));
      if (vel) TPM_CUDA(cudaMemcpyAsync(vel, out + 3 * n, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, s));
      TPM_CUDA(cudaStreamSynchronize(s));
      h->e2e_buf = b;
      h->e2e_version = vel ? h->version : ~0ull;
      if (vel) e2e_take_sample(h, pos, vel, n);
    };
    const bool spec = n > 0 && vel && h->e2e_version == h->version && n == h->n && n == h->n_owned &&
                      h->forces_valid && h->eps2_acc == eps2 && h->g_acc != 0.0 &&
                      e2e_sample_matches(h, pos, vel, n);
    if (!spec) {
      h->e2e_version = ~0ull;
      upload(h, pos, vel, mass, n);
      if (n == 0) return TPM_OK;
      kdk_device(h, kick_half, drift, kick_half2, eps2, g);
      ensure_buffers();
      return_state(1 - h->e2e_buf);
      return TPM_OK;
    }
    ensure_buffers();
    const int ob = h->e2e_buf, nb = 1 - ob;
    const double* prev = h->e2e_out[ob];
    double* out = h->e2e_out[nb];
    double* din = h->e2e_in;  // positions 3n, momenta 3n, masses n
    const Particles before = h->P[h->cur];
    h->e2e_version = ~0ull;
    // opening half: kick with the cached acceleration, drift; positions out
    const double k1 = kick_half * (g / h->g_acc);
    k_kick_drift<<<grid_for(n, 256, 1ll << 30), 256, 0, s>>>(before, n, h->ax, h->ay, h->az, (float)k1,
                                                             drift * TWO32 / h->cfg.box_size);
    TPM_LAUNCH_CHECK();
    ++h->version;
    k_decode_state<<<grid_for(n, 256, 1ll << 30), 256, 0, s>>>(before, n, scale, nullptr, nullptr, nullptr, out,
                                                               nullptr, nullptr);
    TPM_LAUNCH_CHECK();
    TPM_CUDA(cudaEventRecord(h->ev_pos, s));
    // the copy stream, driven from a second host thread so that pageable host
    // buffers (whose copies block the calling thread) overlap as well
    cudaError_t copy_err = cudaSuccess;
    const int dev = h->cfg.device;
    uint32_t* same = h->e2e_flag;
    cudaEvent_t ev_pos = h->ev_pos;
    std::thread copier([&, dev, same, ev_pos] {
      auto chk = [&](cudaError_t e) {
        if (e != cudaSuccess && copy_err == cudaSuccess) copy_err = e;
      };
      chk(cudaSetDevice(dev));
      chk(cudaMemcpyAsync(din, pos, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, c));
      chk(cudaMemcpyAsync(din + 3 * n, vel, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, c));
      chk(cudaMemcpyAsync(din + 6 * n, mass, sizeof(double) * n, cudaMemcpyHostToDevice, c));
      chk(cudaMemsetAsync(same, 0xFF, sizeof(uint32_t), c));
      k_match_returned<<<grid_for(n, 256, 1ll << 30), 256, 0, c>>>(din, din + 3 * n, din + 6 * n, prev, n, before,
                                                                    same);
      chk(cudaGetLastError());
      chk(cudaStreamWaitEvent(c, ev_pos, 0));
      chk(cudaMemcpyAsync(pos, out, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, c));
    });
    try {
      force_eval(h, eps2, g, kick_half2);  // closing half: the kick is fused into the gather
      k_decode_state<<<grid_for(n, 256, 1ll << 30), 256, 0, s>>>(h->P[h->cur], n, scale, nullptr, nullptr, nullptr,
                                                                 nullptr, out + 3 * n, nullptr);
      TPM_LAUNCH_CHECK();
      TPM_CUDA(cudaEventRecord(h->ev_done, s));
    } catch (...) {
      copier.join();
      cudaStreamSynchronize(c);  // no copy into the caller's buffers after the return
      throw;
    }
    copier.join();
    g_kernel_launches += 1;  // the check kernel on the copy stream
    h->stats.kernel_launches += 4;  // kick-drift, the two decodes, the check
    if (copy_err != cudaSuccess) throw Error(TPM_ERR_CUDA, std::string("host-buffer copies: ") + cudaGetErrorString(copy_err));
    TPM_CUDA(cudaStreamWaitEvent(c, h->ev_done, 0));
    TPM_CUDA(cudaMemcpyAsync(vel, out + 3 * n, sizeof(double) * 3 * n, cudaMemcpyDeviceToHost, c));
    uint32_t flag = 0;
    TPM_CUDA(cudaMemcpyAsync(&flag, same, sizeof(uint32_t), cudaMemcpyDeviceToHost, c));
    TPM_CUDA(cudaStreamSynchronize(c));
    if (flag != 0u) {
      h->e2e_buf = nb;
      h->e2e_version = h->version;
      e2e_take_sample(h, pos, vel, n);
      return TPM_OK;
    }
    // the inputs were another state: encode the uploaded copy and step it
    ensure_capacity(h, n);  // (no-op: the capacity holds n)
    h->n = n;
    h->n_owned = n;
    h->cur = 0;
    h->forces_valid = false;
    h->m_total_valid = false;
    ++h->version;
    k_encode<<<grid_for(n, 256, 1ll << 30), 256, 0, s>>>(din, din + 3 * n, din + 6 * n, n, h->cfg.box_size, h->P[0],
                                                         h->T.err);
    TPM_LAUNCH_CHECK();
    check_dev_err(h);
    kdk_device(h, kick_half, drift, kick_half2, eps2, g);
    return_state(nb);
  } catch (const Error& e) {
    h->e2e_version = ~0ull;
    return fail(h, e);
  }
  return TPM_OK;
}

int tpm_set_particles_zeldovich(tpm_handle* h, const tpm_zeldovich* cfg) {
  if (!h || !cfg) return TPM_ERR_INVALID_ARGUMENT;
  try {
    TPM_CUDA(cudaSetDevice(h->cfg.device));
    if (cfg->n_side < 4 || cfg->n_side > 1024 || (cfg->n_side & (cfg->n_side - 1)) != 0)
      throw Error(TPM_ERR_INVALID_ARGUMENT, "n_side must be a power of two in [4, 1024]");
    const int64_t n = (int64_t)cfg->n_side * cfg->n_side * cfg->n_side;
    if (n >= ((int64_t)1 << 31)) throw Error(TPM_ERR_INVALID_ARGUMENT, "too many particles");
    ensure_capacity(h, n);
    h->n = n;
    h->n_owned = n;
    h->cur = 0;
    ++h->version;
    h->forces_valid = false;
    h->m_total_valid = false;
    zeldovich_fill(cfg, h->cfg.box_size, h->P[0], h->stream, &h->pm);
  } catch (const Error& e) {
    return fail(h, e);
  }
  return TPM_OK;
}

int tpm_write_snapshot(tpm_handle* h, const char* out_dir, int32_t format, const tpm_snapshot_env* env,
                       const tpm_provenance* prov) {
  if (!h || !out_dir || !env || !prov) return TPM_ERR_INVALID_ARGUMENT;
  try {
    TPM_CUDA(cudaSetDevice(h->cfg.device));
    drop_halos(h);
    snapshot_write(out_dir, format, env, prov, DeviceState{h->P[h->cur], h->n, h->cfg.box_size, h->staging, h->stream});
  } catch (const Error& e) {
    return fail(h, e);
  } catch (const std::exception& e) {
    return fail(h, Error(TPM_ERR_IO, e.what()));
  }
  return TPM_OK;
}

int tpm_read_snapshot(tpm_handle* h, const char* dir, int32_t format, tpm_snapshot_env* env_out) {
  if (!h || !dir) return TPM_ERR_INVALID_ARGUMENT;
  try {
    std::vector<double> pos, vel, mass;
    std::vector<uint64_t> ids;
    snapshot_read(dir, format, env_out, pos, vel, mass, ids);
    order_by_id(pos, vel, mass, ids);
    const int rc = tpm_set_particles(h, pos.data(), vel.data(), mass.data(), (int64_t)ids.size());
    if (rc != TPM_OK) return rc;
  } catch (const Error& e) {
    return fail(h, e);
  } catch (const std::exception& e) {
    return fail(h, Error(TPM_ERR_IO, e.what()));
  }
  return TPM_OK;
}

// save_checkpoint (checkpoint.rs:47-105): the JSONL writer with the default
// SnapshotEnv (time 0, redshift 0, box 1) and the provenance ("checkpoint",
// no commit, "release", no features, no command line, config hash).
int tpm_write_checkpoint(tpm_handle* h, const char* out_dir, uint64_t completed_step, double a_current,
                         const char* config_hash) {
  if (!h || !out_dir || !config_hash) return TPM_ERR_INVALID_ARGUMENT;
  try {
    TPM_CUDA(cudaSetDevice(h->cfg.device));
    drop_halos(h);
    const std::string ck = std::string(out_dir) + "/checkpoint";
    tpm_snapshot_env env{};
    env.box_size = 1.0;
    const tpm_provenance prov{"checkpoint", nullptr, "release", nullptr, 0, 0, nullptr, config_hash};
    snapshot_write(ck, TPM_SNAPSHOT_JSONL, &env, &prov,
                   DeviceState{h->P[h->cur], h->n, h->cfg.box_size, h->staging, h->stream});
    checkpoint_write_meta(ck, completed_step, a_current, config_hash, h->n);
  } catch (const Error& e) {
    return fail(h, e);
  } catch (const std::exception& e) {
    return fail(h, Error(TPM_ERR_IO, e.what()));
  }
  return TPM_OK;
}

// load_checkpoint (checkpoint.rs:112-178) for one rank holding every particle.
int tpm_read_checkpoint(tpm_handle* h, const char* resume_dir, uint64_t* completed_step, double* a_current,
                        char* config_hash, int64_t config_hash_capacity) {
  if (!h || !resume_dir || !completed_step || !a_current) return TPM_ERR_INVALID_ARGUMENT;
  try {
    const std::string ck = std::string(resume_dir) + "/checkpoint";
    std::string hash;
    int64_t total = 0;
    checkpoint_read_meta(ck, completed_step, a_current, &hash, &total);
    if (config_hash) {
      if (config_hash_capacity < (int64_t)hash.size() + 1)
        throw Error(TPM_ERR_INVALID_ARGUMENT, "config_hash buffer too small");
      std::memcpy(config_hash, hash.c_str(), hash.size() + 1);
    }
    std::vector<double> pos, vel, mass;
    std::vector<uint64_t> ids;
    snapshot_read(ck, TPM_SNAPSHOT_JSONL, nullptr, pos, vel, mass, ids);
    if ((int64_t)ids.size() != total) throw Error(TPM_ERR_IO, "checkpoint particle count differs from checkpoint.json");
    order_by_id(pos, vel, mass, ids);
    const int rc = tpm_set_particles(h, pos.data(), vel.data(), mass.data(), total);
    if (rc != TPM_OK) return rc;
  } catch (const Error& e) {
    return fail(h, e);
  } catch (const std::exception& e) {
    return fail(h, Error(TPM_ERR_IO, e.what()));
  }
  return TPM_OK;
}

int tpm_power_spectrum(const double* pos, const double* mass, int64_t n, double box, int32_t mesh, int32_t device,
                       double* k, double* pk, uint64_t* n_modes) {
  if (!pos || !mass || !k || !pk || !n_modes || n < 1 || !(box > 0.0) || !std::isfinite(box) || mesh < 4 ||
      mesh > 1024 || (mesh & (mesh - 1)) != 0)
    return TPM_ERR_INVALID_ARGUMENT;
  PmPlan plan;
  double *dpos = nullptr, *dmass = nullptr, *dsum = nullptr;
  unsigned long long* dn = nullptr;
  int rc = TPM_OK;
  try {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
      cudaGetLastError();
      throw Error(TPM_ERR_NO_DEVICE, "no CUDA device");
    }
    if (device < 0 || device >= ndev) throw Error(TPM_ERR_INVALID_ARGUMENT, "device ordinal out of range");
    TPM_CUDA(cudaSetDevice(device));
    double mtot = 0.0;
    for (int64_t i = 0; i < n; ++i) mtot += mass[i];
    if (!(mtot > 0.0) || !std::isfinite(mtot)) throw Error(TPM_ERR_INVALID_ARGUMENT, "total mass must be positive");
    pm_plan_init(plan, mesh, box, 0.0, 0u, device);
    TPM_CUDA(cudaMalloc(&dpos, sizeof(double) * 3 * n));
    TPM_CUDA(cudaMalloc(&dmass, sizeof(double) * n));
    TPM_CUDA(cudaMalloc(&dsum, sizeof(double) * (mesh / 2)));
    TPM_CUDA(cudaMalloc(&dn, sizeof(unsigned long long) * (mesh / 2)));
    TPM_CUDA(cudaMemcpy(dpos, pos, sizeof(double) * 3 * n, cudaMemcpyHostToDevice));
    TPM_CUDA(cudaMemcpy(dmass, mass, sizeof(double) * n, cudaMemcpyHostToDevice));
    std::vector<unsigned long long> hn((size_t)mesh / 2);
    pm_power_spectrum(plan, dpos, nullptr, nullptr, nullptr, dmass, n, mtot, dsum, dn, k, pk, hn.data(), 0);
    pm_check(plan, 0);
    for (int i = 0; i < mesh / 2; ++i) n_modes[i] = hn[i];
  } catch (const Error& e) {
    rc = e.code ? e.code : TPM_ERR_CUDA;
  }
  cudaFree(dpos);
  cudaFree(dmass);
  cudaFree(dsum);
  cudaFree(dn);
  pm_plan_free(plan);
  return rc;
}

int tpm_get_power_spectrum(tpm_handle* h, double* k, double* pk, uint64_t* n_modes) {
  if (!h || !k || !pk || !n_modes) return TPM_ERR_INVALID_ARGUMENT;
  try {
    TPM_CUDA(cudaSetDevice(h->cfg.device));
    drop_halos(h);
    if (h->n == 0) throw Error(TPM_ERR_NOT_READY, "no particles set");
    const int nb = h->pm.nm / 2;
    if (!h->pk_sum) {
      h->pk_sum = h->alloc<double>(nb, 0);
      h->pk_n = h->alloc<unsigned long long>(nb, 0);
    }
    const Particles& P = h->P[h->cur];
    std::vector<unsigned long long> hn((size_t)nb);
    pm_power_spectrum(h->pm, nullptr, P.qx, P.qy, P.qz, P.mass, h->n, total_mass(h), h->pk_sum, h->pk_n, k, pk,
                      hn.data(), h->stream);
    for (int i = 0; i < nb; ++i) n_modes[i] = hn[i];
  } catch (const Error& e) {
    return fail(h, e);
  }
  return TPM_OK;
}

int tpm_set_learned(tpm_handle* h, const tpm_cnn* c) {
  if (!h) return TPM_ERR_INVALID_ARGUMENT;
  try {
    TPM_CUDA(cudaSetDevice(h->cfg.device));
    if (!h->learned) throw Error(TPM_ERR_INVALID_ARGUMENT, "the handle was not created with TPM_FLAG_LEARNED");
    TPM_CUDA(cudaStreamSynchronize(h->stream));
    h->net_attached = false;
    h->forces_valid = false;
    h->release_group(3);
    if (!c) return TPM_OK;
    if (c->device != h->cfg.device) throw Error(TPM_ERR_INVALID_ARGUMENT, "network and solver are on different devices");
    if (c->c_in > cnn::N_FEATURES) throw Error(TPM_ERR_INVALID_ARGUMENT, "the mesh provides 10 input features");
    TPM_CUDA(cudaStreamSynchronize(c->stream));
    LearnedNet& net = h->net;
    net.L = c->L;
    float* params = h->alloc<float>(c->L.total, 3);
    TPM_CUDA(cudaMemcpyAsync(params, c->params, sizeof(float) * c->L.total, cudaMemcpyDeviceToDevice, h->stream));
    uint4* pack = h->alloc<uint4>((size_t)cnn::WPACK_U4 * 5, 3);
    cnn::Packed P{};
    for (int l = 0; l < 3; ++l) P.fwd[l] = pack + (size_t)l * cnn::WPACK_U4;
    P.bwd[1] = pack + (size_t)3 * cnn::WPACK_U4;
    P.bwd[2] = pack + (size_t)4 * cnn::WPACK_U4;
    cnn::pack_weights(params, c->L, P, h->stream);
    net.params = params;
    for (int l = 0; l < 3; ++l) net.fwd[l] = P.fwd[l];
    for (int k = 0; k < cnn::MAX_CIN; ++k) {
      net.shift[k] = c->shift[k];
      net.scale[k] = c->scale[k];
    }
    net.out_scale = c->out_scale;
    net.delta_max = c->delta_max;
    net.near_cells = c->near_cells;
    const int64_t nm = h->pm.nm;
    h->vol_a = h->alloc<__nv_bfloat16>((size_t)(nm + 6) * (nm + 6) * (nm + 6) * cnn::CH, 3);
    h->vol_b = h->alloc<__nv_bfloat16>((size_t)(nm + 4) * (nm + 4) * (nm + 4) * cnn::CH, 3);
    h->octants = h->alloc<float>((size_t)8 * nm * nm * nm, 3);
    TPM_CUDA(cudaStreamSynchronize(h->stream));
    h->net_attached = true;
  } catch (const Error& e) {
    return fail(h, e);
  }
  return TPM_OK;
}

int tpm_cnn_add_box(tpm_cnn* c, tpm_handle* h, int32_t held_out) {
  if (!c || !h) return TPM_ERR_INVALID_ARGUMENT;
  try {
    TPM_CUDA(cudaSetDevice(h->cfg.device));
    if (!h->learned) throw Error(TPM_ERR_INVALID_ARGUMENT, "the handle was not created with TPM_FLAG_LEARNED");
    if (h->net_attached)
      throw Error(TPM_ERR_INVALID_ARGUMENT, "training targets come from the walk: detach the network first");
    if (!h->forces_valid) throw Error(TPM_ERR_NOT_READY, "no forces computed");
    if (c->device != h->cfg.device) throw Error(TPM_ERR_INVALID_ARGUMENT, "network and solver are on different devices");
    if (c->c_in > cnn::N_FEATURES) throw Error(TPM_ERR_INVALID_ARGUMENT, "the mesh provides 10 input features");
    TPM_CUDA(cudaStreamSynchronize(h->stream));
    const Particles& P = h->P[h->cur];
    cnn::BoxSource b{};
    b.nm = h->pm.nm;
    b.box = h->cfg.box_size;
    b.n = h->n;
    b.qx = P.qx;
    b.qy = P.qy;
    b.qz = P.qz;
    b.massf = P.massf;
    b.rho = h->pm.rho;
    b.phi = h->pm.force + 3 * (int64_t)b.nm * b.nm * b.nm;
    b.srx = h->srx;
    b.sry = h->sry;
    b.srz = h->srz;
    b.lrx = h->lrx;
    b.lry = h->lry;
    b.lrz = h->lrz;
    b.g = h->g_acc;
    b.m_total = total_mass(h);
    float* near = nullptr;
    if (c->near_cells > 0.f) {
      TPM_CUDA(cudaMalloc(&near, sizeof(float) * 3 * std::max<int64_t>(h->n, 1)));
      near_of(h, h->eps2_acc, nullptr, near, near + h->n, near + 2 * h->n, c->near_cells);
      TPM_CUDA(cudaStreamSynchronize(h->stream));
      b.nrx = near;
      b.nry = near + h->n;
      b.nrz = near + 2 * h->n;
    }
    if (!(b.g > 0.0)) {
      cudaFree(near);
      throw Error(TPM_ERR_INVALID_ARGUMENT, "the last force evaluation had g <= 0");
    }
    try {
      cnn::add_box(c, b, held_out != 0);
    } catch (...) {
      cudaFree(near);
      throw;
    }
    cudaFree(near);
  } catch (const Error& e) {
    c->err = e.what();
    return e.code ? e.code : TPM_ERR_CUDA;
  }
  return TPM_OK;
}

int tpm_get_force_parts(tpm_handle* h, double* acc_lr, double* acc_sr) {
  if (!h) return TPM_ERR_INVALID_ARGUMENT;
  try {
    TPM_CUDA(cudaSetDevice(h->cfg.device));
    if (!h->forces_valid || !h->parts_valid) throw Error(TPM_ERR_NOT_READY, "no forces computed");
    const int64_t n = h->n, no = h->n_owned;  // owned particles only
    const uint32_t lim = (uint32_t)no;
    cudaStream_t s = h->stream;
    if (acc_lr) {
      k_scatter_xyz<<<grid_for(n, 256, 1ll << 30), 256, 0, s>>>(h->P[h->cur].id, n, h->lrx, h->lry, h->lrz, 1.0,
                                                                h->staging, lim);
      TPM_LAUNCH_CHECK();
      TPM_CUDA(cudaMemcpyAsync(acc_lr, h->staging, sizeof(double) * 3 * no, cudaMemcpyDeviceToHost, s));
      TPM_CUDA(cudaStreamSynchronize(s));
    }
    if (acc_sr) {
      if (h->pm_only) {
        std::memset(acc_sr, 0, sizeof(double) * 3 * no);
      } else {
        k_scatter_xyz<<<grid_for(n, 256, 1ll << 30), 256, 0, s>>>(h->P[h->cur].id, n, h->srx, h->sry, h->srz,
                                                                  h->g_acc, h->staging, lim);
        TPM_LAUNCH_CHECK();
        TPM_CUDA(cudaMemcpyAsync(acc_sr, h->staging, sizeof(double) * 3 * no, cudaMemcpyDeviceToHost, s));
        TPM_CUDA(cudaStreamSynchronize(s));
      }
    }
  } catch (const Error& e) {
    return fail(h, e);
  }
  return TPM_OK;
}

int tpm_get_interaction_counts(tpm_handle* h, int64_t* counts) {
  if (!h || !counts) return TPM_ERR_INVALID_ARGUMENT;
  try {
    TPM_CUDA(cudaSetDevice(h->cfg.device));
    if (!h->forces_valid || !h->parts_valid || h->pm_only || h->n < 2)
      throw Error(TPM_ERR_NOT_READY, "no short-range walk computed");
    const int64_t n = h->n;
    std::vector<uint32_t> c((size_t)2 * n), id((size_t)n);
    TPM_CUDA(cudaMemcpyAsync(c.data(), h->pcounts, sizeof(uint32_t) * 2 * n, cudaMemcpyDeviceToHost, h->stream));
    TPM_CUDA(cudaMemcpyAsync(id.data(), h->P[h->cur].id, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, h->stream));
    TPM_CUDA(cudaStreamSynchronize(h->stream));
    for (int64_t i = 0; i < n; ++i) {
      if ((int64_t)id[i] >= h->n_owned) continue;  // halo copies
      counts[2 * (int64_t)id[i]] = c[2 * i];
      counts[2 * (int64_t)id[i] + 1] = c[2 * i + 1];
    }
  } catch (const Error& e) {
    return fail(h, e);
  }
  return TPM_OK;
}

int tpm_get_stats(const tpm_handle* h, tpm_stats* out) {
  if (!h || !out) return TPM_ERR_INVALID_ARGUMENT;
  *out = h->stats;
  return TPM_OK;
}

int tpm_drift_kick_factors(double omega_m, double omega_lambda, double h0, double a0, double dt, double* out3) {
  if (!out3) return TPM_ERR_INVALID_ARGUMENT;
  const Cosmo c{omega_m, omega_lambda, h0};
  const uint32_t N_SUB = 16;
  const double sub_dt = dt / (double)N_SUB;
  double a = a0, drift = 0.0, kh = 0.0, kh2 = 0.0;
  for (uint32_t sidx = 0; sidx < N_SUB; ++sidx) {
    const double al = a, am = c.advance_a(a, sub_dt * 0.5), ar = c.advance_a(a, sub_dt);
    drift += sub_dt / 6.0 * (1.0 / (al * al) + 4.0 / (am * am) + 1.0 / (ar * ar));
    const double k = sub_dt / 6.0 * (1.0 / al + 4.0 / am + 1.0 / ar);
    if (sidx < N_SUB / 2) kh += k; else kh2 += k;
    a = ar;
  }
  out3[0] = drift;
  out3[1] = kh;
  out3[2] = kh2;
  return TPM_OK;
}

double tpm_advance_a(double omega_m, double omega_lambda, double h0, double a, double dt) {
  return Cosmo{omega_m, omega_lambda, h0}.advance_a(a, dt);
}

int tpm_hilbert_keys(tpm_handle* h, uint64_t* keys, int64_t* order) {
  if (!h || !keys) return TPM_ERR_INVALID_ARGUMENT;
  try {
    TPM_CUDA(cudaSetDevice(h->cfg.device));
    drop_halos(h);
    const int64_t n = h->n;
    if (n == 0) return TPM_OK;
    cudaStream_t s = h->stream;
    launch_bbox_root(h->P[h->cur], n, h->cfg.box_size, h->T, s);
    uint64_t* k_store = h->T.key_lo_tmp;
    uint64_t* k_by_id = h->T.key_hi;
    uint32_t* vals = h->T.perm;
    launch_hilbert_keys(h->P[h->cur], n, h->cfg.box_size, h->T.params, k_store, vals, s);
    k_scatter_u64<<<grid_for(n, 256, 1ll << 30), 256, 0, s>>>(h->P[h->cur].id, n, k_store, k_by_id, vals);
    TPM_LAUNCH_CHECK();
    TPM_CUDA(cudaMemcpyAsync(keys, k_by_id, sizeof(uint64_t) * n, cudaMemcpyDeviceToHost, s));
    if (order) {
      radix_sort_u64(k_by_id, vals, n, 63, h->sort_scratch, h->sort_bytes, s);
      std::vector<uint32_t> o((size_t)n);
      TPM_CUDA(cudaMemcpyAsync(o.data(), vals, sizeof(uint32_t) * n, cudaMemcpyDeviceToHost, s));
      TPM_CUDA(cudaStreamSynchronize(s));
      for (int64_t i = 0; i < n; ++i) order[i] = o[i];
    }
    TPM_CUDA(cudaStreamSynchronize(s));
    h->tree_valid = false;
  } catch (const Error& e) {
    return fail(h, e);
  }
  return TPM_OK;
}

int tpm_sfc_keys(tpm_handle* h, const double bbox6[6], int32_t kind, uint64_t* keys) {
  if (!h || !bbox6 || !keys || (kind != TPM_SFC_HILBERT && kind != TPM_SFC_MORTON)) return TPM_ERR_INVALID_ARGUMENT;
  try {
    TPM_CUDA(cudaSetDevice(h->cfg.device));
    drop_halos(h);
    const int64_t n = h->n;
    if (n == 0) return TPM_OK;
    cudaStream_t s = h->stream;
    // the normalisation of particle_hilbert / particle_morton (sfc.rs:64-81,
    // :187-204): origin lo, extent max(hi - lo, f64::EPSILON) per axis
    TreeParams prm{};
    for (int d = 0; d < 3; ++d) {
      prm.hlo[d] = bbox6[2 * d];
      prm.hlen[d] = std::max(bbox6[2 * d + 1] - bbox6[2 * d], 2.220446049250313e-16);
    }
    TPM_CUDA(cudaMemcpyAsync(h->T.params, &prm, sizeof(prm), cudaMemcpyHostToDevice, s));
    uint64_t* k_store = h->T.key_lo_tmp;
    uint64_t* k_by_id = h->T.key_hi;
    uint32_t* vals = h->T.perm;
    if (kind == TPM_SFC_HILBERT)
      launch_hilbert_keys(h->P[h->cur], n, h->cfg.box_size, h->T.params, k_store, vals, s);
    else
      launch_morton_keys(h->P[h->cur], n, h->cfg.box_size, h->T.params, k_store, vals, s);
    k_scatter_u64<<<grid_for(n, 256, 1ll << 30), 256, 0, s>>>(h->P[h->cur].id, n, k_store, k_by_id, vals);
    TPM_LAUNCH_CHECK();
    TPM_CUDA(cudaMemcpyAsync(keys, k_by_id, sizeof(uint64_t) * n, cudaMemcpyDeviceToHost, s));
    TPM_CUDA(cudaStreamSynchronize(s));
    h->tree_valid = false;
  } catch (const Error& e) {
    return fail(h, e);
  }
  return TPM_OK;
}

int tpm_cic_cells(tpm_handle* h, int32_t* cells) {
  if (!h || !cells) return TPM_ERR_INVALID_ARGUMENT;
  try {
    TPM_CUDA(cudaSetDevice(h->cfg.device));
    drop_halos(h);
    const int64_t n = h->n;
    if (n == 0) return TPM_OK;
    int32_t* d = (int32_t*)h->staging;
    const Particles& P = h->P[h->cur];
    pm_cells(h->pm, P.qx, P.qy, P.qz, P.id, n, d, h->stream);
    TPM_CUDA(cudaMemcpyAsync(cells, d, sizeof(int32_t) * 3 * n, cudaMemcpyDeviceToHost, h->stream));
    TPM_CUDA(cudaStreamSynchronize(h->stream));
  } catch (const Error& e) {
    return fail(h, e);
  }
  return TPM_OK;
}

int64_t tpm_tree_node_count(const tpm_handle* h) {
  if (!h || !h->tree_valid) return 0;
  return h->n_int + h->n;
}

int64_t tpm_export_tree(tpm_handle* h, int64_t cap, int32_t* depth, double* mass, double* com, double* quad,
                        int64_t* particle, uint64_t* path_hi, uint64_t* path_lo) {
  if (!h) return -TPM_ERR_INVALID_ARGUMENT;
  try {
    TPM_CUDA(cudaSetDevice(h->cfg.device));
    if (!h->tree_valid) throw Error(TPM_ERR_NOT_READY, "no tree built");
    const int64_t n = h->n, ni = h->n_int, tot = n + ni;
    if (cap < tot) return tot;
    if (!depth || !mass || !com || !quad || !particle || !path_hi || !path_lo)
      throw Error(TPM_ERR_INVALID_ARGUMENT, "null export array");
    cudaStream_t s = h->stream;
    if (!h->quad_valid && ni > 0) {  // the force evaluation made mass and centre of mass only
      launch_aggregate(h->P[h->cur], n, ni, h->cfg.box_size, h->T, s, true);
      h->quad_valid = true;
    }
    int32_t* dd;
    double *dm, *dc, *dq;
    int64_t* dp;
    uint64_t *nh, *nl;
    TPM_CUDA(cudaMalloc(&dd, sizeof(int32_t) * tot));
    TPM_CUDA(cudaMalloc(&dm, sizeof(double) * tot));
    TPM_CUDA(cudaMalloc(&dc, sizeof(double) * 3 * tot));
    TPM_CUDA(cudaMalloc(&dq, sizeof(double) * 6 * tot));
    TPM_CUDA(cudaMalloc(&dp, sizeof(int64_t) * tot));
    TPM_CUDA(cudaMalloc(&nh, sizeof(uint64_t) * tot));
    TPM_CUDA(cudaMalloc(&nl, sizeof(uint64_t) * tot));
    k_export_nodes<<<grid_for(tot, 256, 1ll << 30), 256, 0, s>>>(n, ni, h->cfg.box_size / TWO32, h->T.o_depth,
                                                                 h->T.o_mass, h->T.o_com, h->T.o_quad,
                                                                 n > 1 ? h->T.leaf_depth : nullptr, h->P[h->cur], dd,
                                                                 dm, dc, dq, dp);
    TPM_LAUNCH_CHECK();
    launch_export_paths(n, ni, h->T, nh, nl, nh + ni, nl + ni, s);
    TPM_CUDA(cudaMemcpyAsync(depth, dd, sizeof(int32_t) * tot, cudaMemcpyDeviceToHost, s));
    TPM_CUDA(cudaMemcpyAsync(mass, dm, sizeof(double) * tot, cudaMemcpyDeviceToHost, s));
    TPM_CUDA(cudaMemcpyAsync(com, dc, sizeof(double) * 3 * tot, cudaMemcpyDeviceToHost, s));
    TPM_CUDA(cudaMemcpyAsync(quad, dq, sizeof(double) * 6 * tot, cudaMemcpyDeviceToHost, s));
    TPM_CUDA(cudaMemcpyAsync(particle, dp, sizeof(int64_t) * tot, cudaMemcpyDeviceToHost, s));
    TPM_CUDA(cudaMemcpyAsync(path_hi, nh, sizeof(uint64_t) * tot, cudaMemcpyDeviceToHost, s));
    TPM_CUDA(cudaMemcpyAsync(path_lo, nl, sizeof(uint64_t) * tot, cudaMemcpyDeviceToHost, s));
    TPM_CUDA(cudaStreamSynchronize(s));
    cudaFree(dd); cudaFree(dm); cudaFree(dc); cudaFree(dq); cudaFree(dp); cudaFree(nh); cudaFree(nl);
    return tot;
  } catch (const Error& e) {
    fail(h, e);
    return -(int64_t)(e.code ? e.code : TPM_ERR_CUDA);
  }
}

int tpm_get_mesh(tpm_handle* h, float* density, float* fx, float* fy, float* fz) {
  if (!h) return TPM_ERR_INVALID_ARGUMENT;
  try {
    TPM_CUDA(cudaSetDevice(h->cfg.device));
    if (!h->forces_valid) throw Error(TPM_ERR_NOT_READY, "no forces computed");
    const int64_t nm3 = (int64_t)h->pm.nm * h->pm.nm * h->pm.nm;
    cudaStream_t s = h->stream;
    if (density) TPM_CUDA(cudaMemcpyAsync(density, h->pm.rho, sizeof(float) * nm3, cudaMemcpyDeviceToHost, s));
    float* f[3] = {fx, fy, fz};
    for (int c = 0; c < 3; ++c)
      if (f[c]) TPM_CUDA(cudaMemcpyAsync(f[c], h->pm.force + c * nm3, sizeof(float) * nm3, cudaMemcpyDeviceToHost, s));
    TPM_CUDA(cudaStreamSynchronize(s));
    const float g = (float)h->g_acc;
    for (int c = 0; c < 3; ++c)
      if (f[c])
        for (int64_t i = 0; i < nm3; ++i) f[c][i] *= g;
  } catch (const Error& e) {
    return fail(h, e);
  }
  return TPM_OK;
}

}  // extern "C"
