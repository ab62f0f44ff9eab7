// Learned short range inside a force evaluation: mesh features, the network
// over the whole periodic mesh, the dense-cell mask and the per-particle read.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "cnn.cuh"

namespace tpm {

struct LearnedNet {
  float near_cells = 0.f;  // radius of the exact near-field sum, in cells (0: none)
  cnn::Layout L{};
  const float* params = nullptr;
  const uint4* fwd[3] = {nullptr, nullptr, nullptr};
  float shift[cnn::MAX_CIN] = {};
  float scale[cnn::MAX_CIN] = {};
  float out_scale = 1.f;
  float delta_max = 200.f;
};

struct LearnedMesh {
  int nm;
  double box;
  double m_cell;       // mean mass of a cell
  const float* rho;    // mass per cell
  const float* phi;    // long-range potential per unit G
  float* octants;      // nm^3 x 8: mass in each octant around a node
  __nv_bfloat16* vol_a;  // (nm + 6)^3 x 16
  __nv_bfloat16* vol_b;  // (nm + 4)^3 x 16
};

// Raw input feature c of mesh node `node`: 0 = ln(1 + rho / m_cell) (CIC),
// 1 = phi * cell / m_cell, 2..9 = ln(1 + 8 m_oct / m_cell) for the 8 octants
// of the node's own cell [i - 1/2, i + 1/2)^3 (nearest-node assignment, octant
// by the sign of the offset: bit 0 x, bit 1 y, bit 2 z).
constexpr int N_RAW_FEATURES = 10;
__device__ __forceinline__ float raw_feature(int c, int64_t node, const float* __restrict__ rho,
                                             const float* __restrict__ phi, const float* __restrict__ oct,
                                             float inv_mcell, float cell_over_mcell) {
  if (c == 0) return log1pf(fmaxf(rho[node], 0.f) * inv_mcell);
  if (c == 1) return phi[node] * cell_over_mcell;
  return log1pf(8.f * oct[node * 8 + (c - 2)] * inv_mcell);
}

// Particles by mesh cell (the CIC cell floor(x nm / L)): per-cell start
// offsets (nm^3 + 1) and the particle indices; `cell_of` and `cursor` are
// scratch of n and nm^3 + 1 entries, `scan_scratch` sized by
// scan_scratch_bytes(nm^3 + 1).
void cell_list(const uint32_t* qx, const uint32_t* qy, const uint32_t* qz, int64_t n, int nm, double box,
               uint32_t* cell_of, uint32_t* cursor, uint32_t* start, uint32_t* items, void* scan_scratch,
               cudaStream_t s);

// Exact short-range pairs closer than r_near (complete split kernel, Plummer
// softened, minimum image): the part of the short range below the mesh
// scale.  Targets with skip[i] != 0 are left untouched (skip may be null).
struct NearField {
  int64_t n;
  const uint32_t *qx, *qy, *qz;
  const float* mass;
  int nm;
  double box;
  const uint32_t* cell_of;
  const uint32_t* start;
  const uint32_t* items;
  const uint8_t* skip;
  double r_near, r_split, eps2;
  float *nx, *ny, *nz;  // per unit G
};
void near_field(const NearField& f, cudaStream_t s);

// Octant masses of every node (zeroed here); positions in fixed point.
void octant_deposit(const uint32_t* qx, const uint32_t* qy, const uint32_t* qz, const float* mass, int64_t n,
                    int nm, double box, float* oct, cudaStream_t s);

// Features of the padded periodic mesh and the three convolutions; the head
// input (layer-3 activation, nm^3 x 16) ends in vol_b.
void learned_mesh(const LearnedNet& net, const LearnedMesh& m, uint32_t* err, cudaStream_t s);

// fallback[i] = 1 where any of particle i's 8 CIC nodes has rho > (1 +
// delta_max) m_cell; *count (device) += particles taken by the network.
void learned_mask(const uint32_t* qx, const uint32_t* qy, const uint32_t* qz, int64_t n, const LearnedNet& net,
                  const LearnedMesh& m, uint8_t* fallback, unsigned long long* count, cudaStream_t s);

// Walk groups holding at least one fallback particle, compacted; *ngroups (device).
void learned_groups(const uint32_t* gfirst, const uint32_t* gsize, int64_t ngroups, const uint8_t* fallback,
                    uint32_t* out_first, uint32_t* out_size, uint32_t* out_count, cudaStream_t s);

// Short-range acceleration per unit G of the particles the network takes:
// the network's prediction plus the near-field sum already in sr (when the
// network has a near field) or alone.
void learned_apply(const uint32_t* qx, const uint32_t* qy, const uint32_t* qz, int64_t n, const LearnedNet& net,
                   const LearnedMesh& m, const uint8_t* fallback, float* srx, float* sry, float* srz,
                   cudaStream_t s);

}  // namespace tpm
