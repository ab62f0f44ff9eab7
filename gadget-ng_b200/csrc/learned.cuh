// Learned short range inside a force evaluation: mesh features, the network
// over the whole periodic mesh, the dense-cell mask and the per-particle read.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "cnn.cuh"

namespace tpm {

struct LearnedNet {
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
  __nv_bfloat16* vol_a;  // (nm + 6)^3 x 16
  __nv_bfloat16* vol_b;  // (nm + 4)^3 x 16
};

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

// Short-range acceleration per unit G of the particles the network takes.
void learned_apply(const uint32_t* qx, const uint32_t* qy, const uint32_t* qz, int64_t n, const LearnedNet& net,
                   const LearnedMesh& m, const uint8_t* fallback, float* srx, float* sry, float* srz,
                   cudaStream_t s);

}  // namespace tpm
