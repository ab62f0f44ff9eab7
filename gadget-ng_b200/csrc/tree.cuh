// Octree of the insertion algorithm of crates/gadget-ng-tree/src/octree.rs,
// rebuilt in parallel from sorted octant-path keys.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace tpm {

constexpr uint32_t LEAF_BIT = 0x80000000u;
constexpr uint32_t EMPTY_SLOT = 0xFFFFFFFFu;
constexpr int KEY_LEVELS = 42;  // 21 octant digits in each of two 64-bit words

// One node of the walk, 32 bytes.  Records are laid out so that the children
// of every internal node are contiguous (root at 0, the children of internal
// node P at 1 + child_first[P] ...), so the walk reads a node's children with
// one coalesced load.
struct __align__(16) WalkNode {
  uint32_t cq[3];    // fixed-point centre of mass (leaf: the particle)
  float mass;
  uint32_t first;    // record index of the first child (internal nodes)
  uint32_t info;     // nchild [0,4) | depth [4,10) | leaf bit 10 | terminal bit 11
  uint32_t ref;      // leaf: sorted particle index; internal: octree node id
  uint32_t pad;
};
constexpr uint32_t WN_LEAF = 1u << 10;
constexpr uint32_t WN_TERMINAL = 1u << 11;
__host__ __device__ inline uint32_t wn_nchild(uint32_t info) { return info & 15u; }
__host__ __device__ inline int wn_depth(uint32_t info) { return (int)((info >> 4) & 63u); }

// Geometry of one force evaluation, computed on the device.
struct TreeParams {
  double center[3];  // bounding_cube centre (octree.rs:1306-1332)
  double half;       // bounding_cube half side, padded
  double hlo[3];     // Hilbert normalisation origin (sfc.rs:187-204)
  double hlen[3];    // Hilbert normalisation extent
  uint32_t qmin[3], qmax[3];
};

// Particle arrays (structure of arrays, current storage order).
struct Particles {
  uint32_t* qx;
  uint32_t* qy;
  uint32_t* qz;
  float* vx;
  float* vy;
  float* vz;
  double* mass;
  float* massf;
  uint32_t* id;  // original index
};

struct TreeBuffers {
  // keys (sorted order after the sort)
  uint64_t* key_hi;
  uint64_t* key_lo;      // by storage index before the permutation, sorted after
  uint64_t* key_lo_tmp;
  uint32_t* perm;
  // binary radix tree over the sorted keys (n - 1 internal nodes)
  uint32_t* bin_left;
  uint32_t* bin_right;
  int32_t* bin_prefix;
  uint32_t* bin_first;
  uint32_t* bin_last;
  int32_t* bin_parent;
  int32_t* leaf_bparent;
  uint32_t* oct_count;
  uint32_t* oct_base;
  // octree internal nodes
  int64_t cap_int;
  int32_t* o_parent;
  uint8_t* o_depth;
  uint32_t* o_first;
  uint32_t* o_last;
  uint32_t* o_slots;  // 8 per node, EMPTY_SLOT or child id (LEAF_BIT | particle)
  uint32_t* o_nchild;
  uint32_t* o_child_first;
  uint32_t* o_cnt;      // internal node ids bucketed by depth (aggregation order)
  uint32_t* child_ids;  // compacted, same encoding as o_slots
  double* o_mass;
  double* o_com;   // 3 per node
  double* o_quad;  // 6 per node
  uint4* o_walk;   // fixed-point COM (x, y, z) and float mass bits
  uint4* o_cell;   // relative opening criterion: fixed-point cell centre (x, y, z), |Q|_F float bits
  WalkNode* recs;  // n_int + n walk records
  // leaves
  int32_t* leaf_oparent;
  uint8_t* leaf_depth;
  // walk groups
  uint32_t* grp_count_per_node;
  uint32_t* grp_base;
  uint32_t* grp_first;
  uint32_t* grp_size;
  int64_t cap_groups;
  // params and scalars
  TreeParams* params;
  uint32_t* bbox;       // 6 words
  uint32_t* scalars;    // [0] octree internal count, [1] groups, [2] max depth, [3] child total
  uint32_t* depth_tab;  // DEPTH_BINS counts, offsets, cursors of internal nodes per depth
  uint32_t* err;
};

constexpr int DEPTH_BINS = 64;  // octree depths are at most KEY_LEVELS

void launch_bbox_root(const Particles& p, int64_t n, double box, TreeBuffers& t, cudaStream_t s);
void launch_tree_keys(const Particles& p, int64_t n, double box, TreeBuffers& t, cudaStream_t s);
void launch_fix_ties(const Particles& p, int64_t n, double box, TreeBuffers& t, cudaStream_t s);
void launch_permute(const Particles& src, const Particles& dst, int64_t n, const uint32_t* perm, cudaStream_t s);
void launch_karras(int64_t n, TreeBuffers& t, cudaStream_t s);
void launch_octree_nodes(int64_t n, TreeBuffers& t, cudaStream_t s);
void launch_octree_links(int64_t n, int64_t n_int, TreeBuffers& t, void* scan_scratch, cudaStream_t s);
// Level-synchronous moments, deepest level first: mass and centre of mass, and
// with_quad the quadrupole tensors too.
void launch_aggregate(const Particles& p, int64_t n, int64_t n_int, double box, TreeBuffers& t, cudaStream_t s,
                      bool with_quad = false);
void launch_walk_records(const Particles& p, int64_t n, int64_t n_int, double thr, TreeBuffers& t, cudaStream_t s);
// Per internal node: the centre of its octree cell (child_center replayed
// along the node's octant path, octree.rs:446-465) in fixed point and the
// Frobenius norm of its six stored quadrupole components (the relative
// opening criterion's estimate, octree.rs:769-796).  Needs the quadrupoles.
void launch_cell_q(int64_t n_int, double box, TreeBuffers& t, cudaStream_t s);
void launch_groups(int64_t n, int64_t n_int, int group_max, TreeBuffers& t, void* scan_scratch, cudaStream_t s);
void launch_hilbert_keys(const Particles& p, int64_t n, double box, const TreeParams* prm, uint64_t* keys,
                         uint32_t* vals, cudaStream_t s);
// Morton keys (particle_morton, sfc.rs:54-81) with the normalisation of prm's
// hlo / hlen, like launch_hilbert_keys.
void launch_morton_keys(const Particles& p, int64_t n, double box, const TreeParams* prm, uint64_t* keys,
                        uint32_t* vals, cudaStream_t s);
void launch_export_paths(int64_t n, int64_t n_int, const TreeBuffers& t, uint64_t* node_hi, uint64_t* node_lo,
                         uint64_t* leaf_hi, uint64_t* leaf_lo, cudaStream_t s);

}  // namespace tpm
