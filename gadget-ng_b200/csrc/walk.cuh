// Short-range erfc tree walk (crates/gadget-ng-treepm/src/short_range.rs).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "tree.cuh"

namespace tpm {

struct WalkArgs {
  int64_t n, n_int;
  // particles, sorted order
  const uint32_t* qx;
  const uint32_t* qy;
  const uint32_t* qz;
  const float* massf;
  // octree
  const WalkNode* recs;  // walk records, children contiguous
  const uint4* walk;  // internal nodes: fixed-point COM + float mass bits
  const uint8_t* depth;
  const uint32_t* nchild;
  const uint32_t* child_first;
  const uint32_t* child_ids;
  const double* o_com;
  const uint8_t* leaf_depth;
  // groups
  const uint32_t* gfirst;
  const uint32_t* gsize;
  int64_t ngroups;
  uint32_t* work;
  // geometry (float64 = the reference's decisions; float32 = the fast path)
  double scale, box, rc2, thr, h0;
  int periodic;
  float u_inv;    // 2^-U: quanta -> walk units u = scale * 2^U
  float box_u;    // box side in walk units (2^32 quanta)
  float h0_u;     // root half side in u
  float rc2_lo, rc2_hi;    // per-target ambiguity band around r_cut^2 (u^2): node refinement
  float prc2_lo, prc2_hi;  // the pair loop's (narrower) band: leaf pairs and monopoles
  uint32_t prc2_lo_bits, pband_bits;  // the pair band as float bit patterns: (lo, lo + band]
  float grc2_lo, grc2_hi;  // group-level band
  float eps2_u;
  float pcx;      // 0.3275911 * scale*2^U / (sqrt(2) r_s)
  float ex2k;     // -(scale*2^U / (sqrt(2) r_s))^2 * log2(e)
  float tiny_u;   // (4 quanta)^2 in u^2
  float out_scale;  // 1/u^2 in physical units
  int accurate;      // extension mode: complete split kernel + opening angle
  float theta2;      // opening angle squared (accurate mode)
  float gkc;         // (2/sqrt(pi)) * u/(sqrt(2) r_s): the Gaussian term of the split
  int relative;      // accurate mode: relative opening criterion instead of the opening angle
  float rel_k;       // err_tol * u^3 (relative criterion, walk units)
  const uint4* cellq;  // per internal node: fixed-point cell centre, |Q|_F float bits
  // outputs (physical, per unit G), sorted order
  float* ax;
  float* ay;
  float* az;
  unsigned long long* stats;  // [0] leaf pairs [1] monopoles [2] evaluated [3] exact fallbacks [4] deferred
  uint32_t* err;
  uint2* deferred;
  uint32_t* ndeferred;
  uint32_t cap_deferred;
  uint32_t* stack;
  int stack_cap;
  int single_target;     // walk every target alone (r_cut above a quarter box)
  uint32_t* pcounts;     // per target (sorted order): leaf pairs, monopoles
  const uint8_t* only;   // nullptr, or: walk only the targets p with only[p] != 0
  int img_depth;         // periodic: nodes shallower than this need the +-L images in the group cull
};

int walk_blocks_per_sm(bool accurate);
int walk_targets_per_warp();
int walk_threads();
size_t walk_stack_words(int grid, int stack_cap);
void launch_walk(const WalkArgs& a, int grid, cudaStream_t s);
void launch_deferred(const WalkArgs& a, uint32_t n_items, cudaStream_t s);

}  // namespace tpm
