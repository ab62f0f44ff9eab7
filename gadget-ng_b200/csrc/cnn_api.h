// Host object of the learned short-range network (tpm_cnn): parameters, Adam
// state, the tensor-core operand packs, a workspace for batches of patches,
// and the device-resident training set captured from solver handles.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "cnn.cuh"

struct tpm_cnn {
  int device = 0;
  int c_in = 2;
  tpm::cnn::Layout L{};
  std::string err;
  cudaStream_t stream = nullptr;
  float* params = nullptr;  // float32 master parameters
  float* m = nullptr;       // Adam moments
  float* v = nullptr;
  float* grad = nullptr;
  uint4* pack = nullptr;  // 5 packed layers
  tpm::cnn::Packed P{};
  int64_t step = 0;
  // feature normalisation x = (raw - shift) * scale and the output unit
  float shift[tpm::cnn::MAX_CIN] = {};
  float scale[tpm::cnn::MAX_CIN] = {};
  float out_scale = 1.f;
  float delta_max = 200.f;
  float near_cells = 0.f;  // exact near-field radius (cells); the network learns the rest
  bool scales_set = false;
  // batch workspace (volumes of side ws_d, ws_b of them; ws_p particle slots)
  int ws_b = 0, ws_d = 0;
  int64_t ws_p = 0;
  float* x0f = nullptr;
  __nv_bfloat16 *x0 = nullptr, *z1 = nullptr, *a1 = nullptr, *z2 = nullptr, *a2 = nullptr, *z3 = nullptr,
                *a3 = nullptr, *dz1 = nullptr, *dz2 = nullptr, *dz3 = nullptr;
  float* dout = nullptr;
  int32_t* pb = nullptr;
  float *ps = nullptr, *tgt = nullptr, *w = nullptr;
  float* scal = nullptr;  // [0] weight sum, [1] loss
  float* loss_hist = nullptr;
  int64_t loss_cap = 0;
  uint32_t* err_dev = nullptr;
  std::vector<void*> ws_allocs;
  // training set: one entry per captured box
  struct Box {
    int nm = 0;
    bool held_out = false;
    int64_t n = 0;         // particles kept (all 8 CIC nodes at or below delta_max)
    float* feats = nullptr;   // nm^3 x c_in raw features
    uint32_t* start = nullptr;  // nm^3 + 1 offsets of the particles of each cell
    float4* pdat = nullptr;     // (sx, sy, sz, weight), node units
    float4* ptgt = nullptr;     // target short-range acceleration, network units
  };
  std::vector<Box> boxes;
  std::vector<void*> box_allocs;
};

namespace tpm {
namespace cnn {

// What a solver handle hands over for one training box (device pointers, the
// particles in the handle's storage order).
struct BoxSource {
  int nm;
  double box;
  int64_t n;
  const uint32_t *qx, *qy, *qz;
  const float* massf;  // particle masses
  const float* rho;  // mass per mesh cell
  const float* phi;  // long-range potential per unit G
  const float *srx, *sry, *srz;  // short-range acceleration per unit G
  const float *lrx, *lry, *lrz;  // long-range acceleration (times g)
  const float *nrx, *nry, *nrz;  // near-field part of the short range (per unit G), or null
  double g;
  double m_total;
};
void add_box(tpm_cnn* c, const BoxSource& b, bool held_out);

// Raw (unnormalised) input features of a mesh: see raw_feature (learned.cuh).
constexpr int N_FEATURES = 10;

}  // namespace cnn
}  // namespace tpm
