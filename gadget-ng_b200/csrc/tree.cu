// Octree construction on the device.
//
// The reference builds its octree by inserting particles one at a time
// (crates/gadget-ng-tree/src/octree.rs:474-540): one particle per leaf, all
// eight children created on each split, octant chosen by `p >= centre`
// comparisons against float64 child centres (octant_of :423-435,
// child_center :447-465).  The resulting node set does not depend on the
// insertion order: a cell is internal iff it holds two or more particles.
// So the device computes, per particle, the exact sequence of octant choices
// the insertion would make (same float64 centres, same comparisons), sorts by
// that path key, and recovers the nodes from the sorted keys with a binary
// radix tree (Karras 2012, "Maximizing parallelism in the construction of
// BVHs, octrees and k-d trees"), whose prefix lengths, read in 3-bit digits,
// give the octree levels.  Mass, centre of mass and quadrupole are then
// aggregated bottom-up in float64 with the reference's operation order
// (aggregate :547-629), so they are bit-identical to the reference's nodes.
#include "common.cuh"
#include "scan.cuh"
#include "tree.cuh"

namespace tpm {
namespace {

constexpr double F64_EPSILON = 2.220446049250313e-16;

// ---------------------------------------------------------------------------
// bounding box and root cube
// ---------------------------------------------------------------------------
// Seeds the min/max words on the stream (no host copy, so nothing pageable is
// read and the sequence stays stream-ordered).
__global__ void k_bbox_init(uint32_t* __restrict__ out) {
  if (threadIdx.x < 6) out[threadIdx.x] = threadIdx.x < 3 ? 0xFFFFFFFFu : 0u;
}

__global__ void k_bbox(const uint32_t* __restrict__ qx, const uint32_t* __restrict__ qy,
                       const uint32_t* __restrict__ qz, int64_t n, uint32_t* __restrict__ out) {
  uint32_t mn[3] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu}, mx[3] = {0u, 0u, 0u};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    uint32_t a = qx[i], b = qy[i], c = qz[i];
    mn[0] = min(mn[0], a); mx[0] = max(mx[0], a);
    mn[1] = min(mn[1], b); mx[1] = max(mx[1], b);
    mn[2] = min(mn[2], c); mx[2] = max(mx[2], c);
  }
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    uint32_t a = __reduce_min_sync(0xffffffffu, mn[d]);
    uint32_t b = __reduce_max_sync(0xffffffffu, mx[d]);
    if ((threadIdx.x & 31) == 0) {
      atomicMin(&out[d], a);
      atomicMax(&out[3 + d], b);
    }
  }
}

// bounding_cube (octree.rs:1306-1332) and the Hilbert box (sfc.rs:187-204,
// with the extent from SfcDecomposition::build_with_kind, :250-280).
__global__ void k_root(const uint32_t* __restrict__ bb, double scale, TreeParams* __restrict__ prm) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  double mn[3], mx[3];
  for (int d = 0; d < 3; ++d) {
    mn[d] = decode(bb[d], scale);
    mx[d] = decode(bb[3 + d], scale);
    prm->qmin[d] = bb[d];
    prm->qmax[d] = bb[3 + d];
  }
  double hx = dmul(dsub(mx[0], mn[0]), 0.5), hy = dmul(dsub(mx[1], mn[1]), 0.5), hz = dmul(dsub(mx[2], mn[2]), 0.5);
  for (int d = 0; d < 3; ++d) prm->center[d] = dmul(0.5, dadd(mn[d], mx[d]));
  double half = fmax(fmax(hx, hy), hz);
  double pad = fmax(dmul(half, 1e-6), 1e-12);
  prm->half = dadd(half, pad);
  for (int d = 0; d < 3; ++d) {
    prm->hlo[d] = mn[d];
    prm->hlen[d] = fmax(dsub(mx[d], mn[d]), F64_EPSILON);
  }
}

// ---------------------------------------------------------------------------
// octant-path keys
// ---------------------------------------------------------------------------
// 21 octant levels of the reference's insertion octree from the cell state
// (centre, half side) onward: the digit is the octant of the particle against
// the centre, then child_center moves the centre by +/- half/2 per axis, all
// in float64 as the reference does.  The levels are unrolled so the digit
// shifts are constants.
__device__ __forceinline__ uint64_t octant_word(double x, double y, double z, double& cx, double& cy, double& cz,
                                               double& h) {
  uint64_t key = 0;
#pragma unroll
  for (int l = 1; l <= KEY_LEVELS / 2; ++l) {
    const double q = dmul(h, 0.5);
    const bool ox = x >= cx, oy = y >= cy, oz = z >= cz;
    const uint64_t digit = (uint64_t)ox | ((uint64_t)oy << 1) | ((uint64_t)oz << 2);
    cx = dadd(cx, ox ? q : -q);
    cy = dadd(cy, oy ? q : -q);
    cz = dadd(cz, oz ? q : -q);
    h = q;
    key |= digit << (63 - 3 * l);
  }
  return key;
}

// Levels 1..21 of every particle (the sort key).  Levels 22..42 only
// separate particles that share the first 21 (tie runs), so k_tie_low makes
// them for those alone.
__global__ void k_tree_keys(const uint32_t* __restrict__ qx, const uint32_t* __restrict__ qy,
                            const uint32_t* __restrict__ qz, int64_t n, double scale,
                            const TreeParams* __restrict__ prm, uint64_t* __restrict__ key_hi,
                            uint32_t* __restrict__ perm) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double x = decode(qx[i], scale), y = decode(qy[i], scale), z = decode(qz[i], scale);
  double cx = prm->center[0], cy = prm->center[1], cz = prm->center[2], h = prm->half;
  key_hi[i] = octant_word(x, y, z, cx, cy, cz, h);
  perm[i] = (uint32_t)i;
}

// After the sort: the low word (levels 22..42) of every particle in a run of
// equal high keys, stored by original index for k_fix_ties.
__global__ void k_tie_low(const uint32_t* __restrict__ qx, const uint32_t* __restrict__ qy,
                          const uint32_t* __restrict__ qz, int64_t n, double scale,
                          const TreeParams* __restrict__ prm, const uint64_t* __restrict__ hi,
                          const uint32_t* __restrict__ perm, uint64_t* __restrict__ lo_by_index) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint64_t k = hi[i];
  if (!((i > 0 && hi[i - 1] == k) || (i + 1 < n && hi[i + 1] == k))) return;
  const uint32_t j = perm[i];
  const double x = decode(qx[j], scale), y = decode(qy[j], scale), z = decode(qz[j], scale);
  double cx = prm->center[0], cy = prm->center[1], cz = prm->center[2], h = prm->half;
  (void)octant_word(x, y, z, cx, cy, cz, h);
  lo_by_index[j] = octant_word(x, y, z, cx, cy, cz, h);
}

// Runs of equal high keys (particles sharing the first 21 octant levels) are
// ordered by the low key.  Equal full keys mean coincident positions.
constexpr int MAX_TIE_RUN = 1 << 14;

__global__ void k_fix_ties(int64_t n, const uint64_t* __restrict__ hi, uint32_t* __restrict__ perm,
                           const uint64_t* __restrict__ lo_by_index, uint64_t* __restrict__ lo_sorted,
                           uint32_t* __restrict__ err) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint64_t k = hi[i];
  const bool starts = (i == 0 || hi[i - 1] != k) && (i + 1 < n && hi[i + 1] == k);
  const bool inside = (i > 0 && hi[i - 1] == k);
  if (!starts) {
    if (!inside) lo_sorted[i] = 0;  // a particle alone in its level-21 cell: its low word is never read
    return;
  }
  int64_t e = i + 1;
  while (e + 1 < n && hi[e + 1] == k && e - i < MAX_TIE_RUN) ++e;
  if (e - i >= MAX_TIE_RUN) {
    atomicOr(err, DEV_ERR_TIE_RUN);
    return;
  }
  // insertion sort of perm[i..e] by the low key (stable)
  for (int64_t a = i + 1; a <= e; ++a) {
    uint32_t pa = perm[a];
    uint64_t ka = lo_by_index[pa];
    int64_t b = a - 1;
    while (b >= i && lo_by_index[perm[b]] > ka) {
      perm[b + 1] = perm[b];
      --b;
    }
    perm[b + 1] = pa;
  }
  for (int64_t a = i; a <= e; ++a) {
    lo_sorted[a] = lo_by_index[perm[a]];
    if (a > i && lo_sorted[a] == lo_sorted[a - 1]) atomicOr(err, DEV_ERR_COINCIDENT);
  }
}

__global__ void k_permute(Particles src, Particles dst, int64_t n, const uint32_t* __restrict__ perm) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t j = perm[i];
  dst.qx[i] = src.qx[j];
  dst.qy[i] = src.qy[j];
  dst.qz[i] = src.qz[j];
  dst.vx[i] = src.vx[j];
  dst.vy[i] = src.vy[j];
  dst.vz[i] = src.vz[j];
  dst.mass[i] = src.mass[j];
  dst.massf[i] = src.massf[j];
  dst.id[i] = src.id[j];
}

// ---------------------------------------------------------------------------
// binary radix tree (Karras 2012, section 4)
// ---------------------------------------------------------------------------
// Common prefix, in bits of the 126-bit digit string, of sorted keys i
// (preloaded) and j; j out of [0, n) on either side gives -1.
__device__ __forceinline__ int delta_i(const uint64_t* __restrict__ hi, const uint64_t* __restrict__ lo, int64_t n,
                                       uint64_t hi_i, uint64_t lo_i, int64_t i, int64_t j) {
  if ((uint64_t)j >= (uint64_t)n) return -1;
  const uint64_t a = hi_i ^ __ldg(&hi[j]);
  if (a) return __clzll((long long)a) - 1;
  const uint64_t b = lo_i ^ __ldg(&lo[j]);
  if (b) return 63 + __clzll((long long)b) - 1;
  return 126 + __clzll((long long)(i ^ j));
}

__global__ void k_karras(int64_t n, const uint64_t* __restrict__ hi, const uint64_t* __restrict__ lo,
                         uint32_t* __restrict__ bl, uint32_t* __restrict__ br, int32_t* __restrict__ bpre,
                         uint32_t* __restrict__ bfirst, uint32_t* __restrict__ blast, int32_t* __restrict__ bparent,
                         int32_t* __restrict__ leaf_bparent) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n - 1) return;
  const uint64_t hi_i = hi[i], lo_i = lo[i];
  // the direction d and the steps along it (i + k d as a sign choice, not a product)
  const bool up = delta_i(hi, lo, n, hi_i, lo_i, i, i + 1) - delta_i(hi, lo, n, hi_i, lo_i, i, i - 1) >= 0;
  auto at = [&](int64_t k) { return up ? i + k : i - k; };
  const int dmin = delta_i(hi, lo, n, hi_i, lo_i, i, at(-1));
  int64_t lmax = 2;
  while (delta_i(hi, lo, n, hi_i, lo_i, i, at(lmax)) > dmin) lmax <<= 1;
  int64_t l = 0;
  for (int64_t t = lmax >> 1; t >= 1; t >>= 1)
    if (delta_i(hi, lo, n, hi_i, lo_i, i, at(l + t)) > dmin) l += t;
  const int64_t j = at(l);
  const int dnode = delta_i(hi, lo, n, hi_i, lo_i, i, j);
  int64_t s = 0, t = l;
  do {
    t = (t + 1) >> 1;
    if (delta_i(hi, lo, n, hi_i, lo_i, i, at(s + t)) > dnode) s += t;
  } while (t > 1);
  const int64_t gamma = at(s) + (up ? 0 : -1);
  const int64_t first = i < j ? i : j, last = i < j ? j : i;
  const bool left_leaf = first == gamma, right_leaf = last == gamma + 1;
  bl[i] = (uint32_t)gamma | (left_leaf ? LEAF_BIT : 0u);
  br[i] = (uint32_t)(gamma + 1) | (right_leaf ? LEAF_BIT : 0u);
  bpre[i] = dnode;
  bfirst[i] = (uint32_t)first;
  blast[i] = (uint32_t)last;
  if (left_leaf) leaf_bparent[gamma] = (int32_t)i; else bparent[gamma] = (int32_t)i;
  if (right_leaf) leaf_bparent[gamma + 1] = (int32_t)i; else bparent[gamma + 1] = (int32_t)i;
  if (i == 0) bparent[0] = -1;
}

// Octree nodes owned by binary node B: depths floor(p_parent/3)+1 .. floor(p_B/3).
__global__ void k_oct_count(int64_t nb, const int32_t* __restrict__ bpre, const int32_t* __restrict__ bparent,
                            uint32_t* __restrict__ cnt) {
  int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (b >= nb) return;
  const int par = bparent[b];
  const int dpar = par < 0 ? -1 : bpre[par] / 3;
  cnt[b] = (uint32_t)(bpre[b] / 3 - dpar);
}

__device__ __forceinline__ int32_t owner_deepest(int32_t b, const int32_t* __restrict__ bparent,
                                                 const uint32_t* __restrict__ cnt,
                                                 const uint32_t* __restrict__ base) {
  // at most three binary levels share one 3-bit octree level
  for (int guard = 0; cnt[b] == 0 && guard < 8; ++guard) b = bparent[b];
  return (int32_t)(base[b] + cnt[b] - 1);
}

__device__ __forceinline__ uint32_t digit_at(uint64_t hi, uint64_t lo, int depth) {
  // octant digit chosen at the split of the node at depth-1 (depth >= 1)
  return depth <= 21 ? (uint32_t)((hi >> (63 - 3 * depth)) & 7u) : (uint32_t)((lo >> (63 - 3 * (depth - 21))) & 7u);
}

__global__ void k_oct_nodes(int64_t nb, const int32_t* __restrict__ bpre, const int32_t* __restrict__ bparent,
                            const uint32_t* __restrict__ bfirst, const uint32_t* __restrict__ blast,
                            const uint32_t* __restrict__ cnt, const uint32_t* __restrict__ base,
                            int32_t* __restrict__ o_parent, uint8_t* __restrict__ o_depth,
                            uint32_t* __restrict__ o_first, uint32_t* __restrict__ o_last,
                            uint32_t* __restrict__ max_depth) {
  int64_t b = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  uint32_t deep = 0;
  const uint32_t c = b < nb ? cnt[b] : 0u;
  if (c != 0) {
    const int32_t par = bparent[b];
    const int start = (par < 0 ? -1 : bpre[par] / 3) + 1;
    const int32_t p0 = par < 0 ? -1 : owner_deepest(par, bparent, cnt, base);
    const uint32_t id0 = base[b];
    for (uint32_t k = 0; k < c; ++k) {
      const uint32_t id = id0 + k;
      o_parent[id] = k == 0 ? p0 : (int32_t)(id - 1);
      o_depth[id] = (uint8_t)(start + k);
      o_first[id] = bfirst[b];
      o_last[id] = blast[b];
    }
    deep = (uint32_t)(start + c);
  }
  // deepest leaf bound: one atomic per warp (one per thread on a single
  // address serialised the kernel)
  deep = __reduce_max_sync(0xffffffffu, deep);
  if ((threadIdx.x & 31) == 0 && deep) atomicMax(max_depth, deep);
}

__global__ void k_leaf_parents(int64_t n, const int32_t* __restrict__ leaf_bparent,
                               const int32_t* __restrict__ bparent, const uint32_t* __restrict__ cnt,
                               const uint32_t* __restrict__ base, const uint8_t* __restrict__ o_depth,
                               int32_t* __restrict__ leaf_oparent, uint8_t* __restrict__ leaf_depth) {
  int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int32_t P = owner_deepest(leaf_bparent[p], bparent, cnt, base);
  leaf_oparent[p] = P;
  leaf_depth[p] = (uint8_t)(o_depth[P] + 1);
}

__global__ void k_oct_slots_nodes(int64_t n_int, const int32_t* __restrict__ o_parent,
                                  const uint8_t* __restrict__ o_depth, const uint32_t* __restrict__ o_first,
                                  const uint64_t* __restrict__ hi, const uint64_t* __restrict__ lo,
                                  uint32_t* __restrict__ slots) {
  int64_t id = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (id >= n_int) return;
  const int32_t P = o_parent[id];
  if (P < 0) return;
  const uint32_t f = o_first[id];
  slots[(int64_t)P * 8 + digit_at(hi[f], lo[f], o_depth[id])] = (uint32_t)id;
}

__global__ void k_oct_slots_leaves(int64_t n, const int32_t* __restrict__ leaf_oparent,
                                   const uint8_t* __restrict__ leaf_depth, const uint64_t* __restrict__ hi,
                                   const uint64_t* __restrict__ lo, uint32_t* __restrict__ slots) {
  int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (p >= n) return;
  slots[(int64_t)leaf_oparent[p] * 8 + digit_at(hi[p], lo[p], leaf_depth[p])] = (uint32_t)p | LEAF_BIT;
}

__global__ void k_oct_nchild(int64_t n_int, const uint32_t* __restrict__ slots, uint32_t* __restrict__ nchild) {
  int64_t id = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (id >= n_int) return;
  uint32_t c = 0;
#pragma unroll
  for (int s = 0; s < 8; ++s) c += slots[id * 8 + s] != EMPTY_SLOT;
  nchild[id] = c;
}

__global__ void k_oct_childlist(int64_t n_int, const uint32_t* __restrict__ slots,
                                const uint32_t* __restrict__ first, uint32_t* __restrict__ ids) {
  int64_t id = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (id >= n_int) return;
  uint32_t w = first[id];
#pragma unroll
  for (int s = 0; s < 8; ++s) {
    uint32_t c = slots[id * 8 + s];
    if (c != EMPTY_SLOT) ids[w++] = c;
  }
}

// ---------------------------------------------------------------------------
// bottom-up aggregation (octree.rs:547-629), float64, reference order
// ---------------------------------------------------------------------------
// Mass and centre of mass of an octree child (leaf: the particle).
__device__ __forceinline__ void child_moments(uint32_t c, double scale, const uint32_t* __restrict__ qx,
                                              const uint32_t* __restrict__ qy, const uint32_t* __restrict__ qz,
                                              const double* __restrict__ pmass, const double* o_mass,
                                              const double* o_com, double* m, double* x, double* y, double* z) {
  if (c & LEAF_BIT) {
    const uint32_t j = c & ~LEAF_BIT;
    *m = pmass[j];
    *x = decode(qx[j], scale);
    *y = decode(qy[j], scale);
    *z = decode(qz[j], scale);
  } else {
    *m = __ldcg(&o_mass[c]);
    *x = __ldcg(&o_com[3 * (int64_t)c]);
    *y = __ldcg(&o_com[3 * (int64_t)c + 1]);
    *z = __ldcg(&o_com[3 * (int64_t)c + 2]);
  }
}

// Internal nodes by depth: per-block histograms, then one reserved range per
// (block, depth) into the depth buckets (the order inside a bucket is free).
__global__ void k_depth_count(int64_t n_int, const uint8_t* __restrict__ o_depth, uint32_t* __restrict__ hist) {
  __shared__ uint32_t sh[DEPTH_BINS];
  if (threadIdx.x < DEPTH_BINS) sh[threadIdx.x] = 0u;
  __syncthreads();
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n_int) atomicAdd(&sh[o_depth[i] & (DEPTH_BINS - 1)], 1u);
  __syncthreads();
  if (threadIdx.x < DEPTH_BINS && sh[threadIdx.x]) atomicAdd(&hist[threadIdx.x], sh[threadIdx.x]);
}

// hist -> exclusive offsets (DEPTH_BINS + 1) and cursors; one warp
__global__ void k_depth_offsets(uint32_t* tab) {
  uint32_t* hist = tab;
  uint32_t* off = tab + DEPTH_BINS;
  uint32_t* cur = tab + 2 * DEPTH_BINS + 1;
  if (threadIdx.x == 0) {
    uint32_t acc = 0;
    for (int d = 0; d < DEPTH_BINS; ++d) {
      off[d] = acc;
      cur[d] = acc;
      acc += hist[d];
    }
    off[DEPTH_BINS] = acc;
  }
}

__global__ void k_depth_scatter(int64_t n_int, const uint8_t* __restrict__ o_depth, uint32_t* __restrict__ cur,
                                uint32_t* __restrict__ by_depth) {
  __shared__ uint32_t cnt[DEPTH_BINS], base[DEPTH_BINS];
  if (threadIdx.x < DEPTH_BINS) cnt[threadIdx.x] = 0u;
  __syncthreads();
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  int d = 0;
  uint32_t r = 0;
  if (i < n_int) {
    d = o_depth[i] & (DEPTH_BINS - 1);
    r = atomicAdd(&cnt[d], 1u);
  }
  __syncthreads();
  if (threadIdx.x < DEPTH_BINS && cnt[threadIdx.x]) base[threadIdx.x] = atomicAdd(&cur[threadIdx.x], cnt[threadIdx.x]);
  __syncthreads();
  if (i < n_int) by_depth[base[d] + r] = (uint32_t)i;
}

// Moments of the internal nodes at one depth (octree.rs:547-629) from their
// children, which are leaves or nodes one level deeper (finished by the
// previous launch): mass and centre of mass summed over the children in
// octant order, then the quadrupole by the parallel-axis theorem
// (outer_traceless :197-207), all float64 in the reference's operation order.
// QUAD: also the quadrupole tensors (the walk reads mass and centre of mass
// only; the quadrupoles are made when the tree is exported).
template <bool QUAD>
__global__ void k_aggregate_level(const uint32_t* __restrict__ nodes, int64_t count, double scale,
                                  const uint32_t* __restrict__ qx, const uint32_t* __restrict__ qy,
                                  const uint32_t* __restrict__ qz, const double* __restrict__ pmass,
                                  const uint32_t* __restrict__ slots, double* o_mass, double* o_com, double* o_quad) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= count) return;
  const uint32_t P = nodes[i];
  // pass 1: mass and centre of mass over the children in octant order
  uint32_t cs[8];
  double mt = 0.0, ax = 0.0, ay = 0.0, az = 0.0;
#pragma unroll
  for (int s = 0; s < 8; ++s) {
    const uint32_t c = slots[(int64_t)P * 8 + s];
    cs[s] = c;
    if (c == EMPTY_SLOT) continue;
    double m, x, y, z;
    child_moments(c, scale, qx, qy, qz, pmass, o_mass, o_com, &m, &x, &y, &z);
    mt = dadd(mt, m);
    ax = dadd(ax, dmul(x, m));
    ay = dadd(ay, dmul(y, m));
    az = dadd(az, dmul(z, m));
  }
  double comx = 0.0, comy = 0.0, comz = 0.0;
  if (mt > 0.0) {
    comx = ddiv(ax, mt);
    comy = ddiv(ay, mt);
    comz = ddiv(az, mt);
  }
  if (!QUAD) {
    __stcg(&o_mass[P], mt);
    __stcg(&o_com[3 * (int64_t)P], comx);
    __stcg(&o_com[3 * (int64_t)P + 1], comy);
    __stcg(&o_com[3 * (int64_t)P + 2], comz);
    return;
  }
  // pass 2: the children are read again (cache hits) rather than held in registers
  double qd[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll 1
  for (int s = 0; s < 8; ++s) {
    const uint32_t c = cs[s];
    if (c == EMPTY_SLOT) continue;
    double m, x, y, z;
    child_moments(c, scale, qx, qy, qz, pmass, o_mass, o_com, &m, &x, &y, &z);
    if (m == 0.0) continue;
    const double sx = dsub(x, comx), sy = dsub(y, comy), sz = dsub(z, comz);
    const double s2 = dadd(dadd(dmul(sx, sx), dmul(sy, sy)), dmul(sz, sz));
    const double m3 = dmul(m, 3.0);
    double oq[6];
    oq[0] = dmul(m, dsub(dmul(dmul(3.0, sx), sx), s2));
    oq[1] = dmul(dmul(m3, sx), sy);
    oq[2] = dmul(dmul(m3, sx), sz);
    oq[3] = dmul(m, dsub(dmul(dmul(3.0, sy), sy), s2));
    oq[4] = dmul(dmul(m3, sy), sz);
    oq[5] = dmul(m, dsub(dmul(dmul(3.0, sz), sz), s2));
    if (c & LEAF_BIT) {
#pragma unroll
      for (int k = 0; k < 6; ++k) qd[k] = dadd(qd[k], dadd(0.0, oq[k]));
    } else {
#pragma unroll
      for (int k = 0; k < 6; ++k) qd[k] = dadd(qd[k], dadd(__ldcg(&o_quad[6 * (int64_t)c + k]), oq[k]));
    }
  }
  __stcg(&o_mass[P], mt);
  __stcg(&o_com[3 * (int64_t)P], comx);
  __stcg(&o_com[3 * (int64_t)P + 1], comy);
  __stcg(&o_com[3 * (int64_t)P + 2], comz);
#pragma unroll
  for (int k = 0; k < 6; ++k) __stcg(&o_quad[6 * (int64_t)P + k], qd[k]);
}

__global__ void k_walk_nodes(int64_t n_int, double inv_scale, const double* __restrict__ o_mass,
                             const double* __restrict__ o_com, uint4* __restrict__ walk) {
  int64_t id = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (id >= n_int) return;
  uint32_t q[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    double v = o_com[3 * id + d] * inv_scale;  // in [0, 2^32]
    q[d] = (uint32_t)((unsigned long long)llrint(v) & 0xFFFFFFFFull);
  }
  walk[id] = make_uint4(q[0], q[1], q[2], __float_as_uint((float)o_mass[id]));
}

// Cell centre and |Q|_F of each internal node (relative opening criterion).
// The node's octant path is the first `depth` digits of any of its particles'
// keys (sorted order: o_first); the centre follows child_center level by
// level in float64 as k_tree_keys does.
__global__ void k_cell_q(int64_t n_int, double inv_scale, const TreeParams* __restrict__ prm,
                         const uint8_t* __restrict__ o_depth, const uint32_t* __restrict__ o_first,
                         const uint64_t* __restrict__ key_hi, const uint64_t* __restrict__ key_lo,
                         const double* __restrict__ o_quad, uint4* __restrict__ out) {
  int64_t id = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (id >= n_int) return;
  const int dep = o_depth[id];
  const uint32_t p = o_first[id];
  double c[3] = {prm->center[0], prm->center[1], prm->center[2]};
  double h = prm->half;
  for (int l = 1; l <= dep && l <= KEY_LEVELS; ++l) {
    const uint64_t w = l <= KEY_LEVELS / 2 ? key_hi[p] : key_lo[p];
    const int ll = l <= KEY_LEVELS / 2 ? l : l - KEY_LEVELS / 2;
    const uint32_t digit = (uint32_t)(w >> (63 - 3 * ll)) & 7u;
    const double q = dmul(h, 0.5);
#pragma unroll
    for (int d = 0; d < 3; ++d) c[d] = dadd(c[d], ((digit >> d) & 1u) ? q : -q);
    h = q;
  }
  uint32_t cq[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double u = c[d] * inv_scale;  // fixed point, wrapped like positions
    cq[d] = (uint32_t)((unsigned long long)llrint(u) & 0xFFFFFFFFull);
  }
  const double* Q = o_quad + 6 * id;
  double f2 = 0.0;
#pragma unroll
  for (int k = 0; k < 6; ++k) f2 = fma(Q[k], Q[k], f2);
  out[id] = make_uint4(cq[0], cq[1], cq[2], __float_as_uint((float)sqrt(f2)));
}

// ---------------------------------------------------------------------------
// walk records: children of each internal node contiguous
// ---------------------------------------------------------------------------
__device__ __forceinline__ WalkNode make_record(uint32_t c, const uint32_t* __restrict__ qx,
                                                const uint32_t* __restrict__ qy, const uint32_t* __restrict__ qz,
                                                const float* __restrict__ massf, const uint8_t* __restrict__ leaf_depth,
                                                const uint4* __restrict__ walk, const uint8_t* __restrict__ o_depth,
                                                const uint32_t* __restrict__ nchild,
                                                const uint32_t* __restrict__ child_first, double h0, double thr) {
  WalkNode r;
  r.pad = 0;
  if (c & LEAF_BIT) {
    const uint32_t j = c & ~LEAF_BIT;
    r.cq[0] = qx[j];
    r.cq[1] = qy[j];
    r.cq[2] = qz[j];
    r.mass = massf[j];
    r.first = 0;
    r.info = ((uint32_t)leaf_depth[j] << 4) | WN_LEAF;
    r.ref = j;
  } else {
    const uint4 w = walk[c];
    r.cq[0] = w.x;
    r.cq[1] = w.y;
    r.cq[2] = w.z;
    r.mass = __uint_as_float(w.w);
    r.first = 1u + child_first[c];
    const int dep = o_depth[c];
    r.info = nchild[c] | ((uint32_t)dep << 4) | (ldexp(h0, -dep) < thr ? WN_TERMINAL : 0u);
    r.ref = c;
  }
  return r;
}

__global__ void k_walk_records(int64_t n_int, const uint32_t* __restrict__ qx, const uint32_t* __restrict__ qy,
                               const uint32_t* __restrict__ qz, const float* __restrict__ massf,
                               const uint8_t* __restrict__ leaf_depth, const uint4* __restrict__ walk,
                               const uint8_t* __restrict__ o_depth, const uint32_t* __restrict__ nchild,
                               const uint32_t* __restrict__ child_first, const uint32_t* __restrict__ child_ids,
                               const TreeParams* __restrict__ prm, double thr, WalkNode* __restrict__ recs) {
  int64_t P = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (P >= n_int) return;
  const double h0 = prm->half;
  if (P == 0)
    recs[0] = make_record(0u, qx, qy, qz, massf, leaf_depth, walk, o_depth, nchild, child_first, h0, thr);
  const uint32_t f = child_first[P], nc = nchild[P];
  for (uint32_t r = 0; r < nc; ++r)
    recs[1 + (int64_t)f + r] =
        make_record(child_ids[f + r], qx, qy, qz, massf, leaf_depth, walk, o_depth, nchild, child_first, h0, thr);
}

// ---------------------------------------------------------------------------
// walk groups: maximal subtrees of <= group_max particles, consecutive small
// siblings packed together
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t child_count(uint32_t c, const uint32_t* __restrict__ o_first,
                                                const uint32_t* __restrict__ o_last) {
  return (c & LEAF_BIT) ? 1u : o_last[c] - o_first[c] + 1u;
}
__device__ __forceinline__ uint32_t child_first_particle(uint32_t c, const uint32_t* __restrict__ o_first) {
  return (c & LEAF_BIT) ? (c & ~LEAF_BIT) : o_first[c];
}

template <bool WRITE>
__global__ void k_groups(int64_t n_int, int group_max, const uint32_t* __restrict__ slots,
                         const uint32_t* __restrict__ o_first, const uint32_t* __restrict__ o_last,
                         uint32_t* __restrict__ counts, const uint32_t* __restrict__ base,
                         uint32_t* __restrict__ gfirst, uint32_t* __restrict__ gsize) {
  int64_t id = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (id >= n_int) return;
  const uint32_t mine = o_last[id] - o_first[id] + 1u;
  uint32_t ng = 0, w = WRITE ? base[id] : 0u;
  if (mine > (uint32_t)group_max) {
    uint32_t run_first = 0, run_n = 0;
    for (int s = 0; s < 8; ++s) {
      const uint32_t c = slots[id * 8 + s];
      if (c == EMPTY_SLOT) continue;
      const uint32_t k = child_count(c, o_first, o_last);
      if (k > (uint32_t)group_max) {
        if (run_n) {
          if (WRITE) { gfirst[w] = run_first; gsize[w] = run_n; ++w; }
          ++ng;
          run_n = 0;
        }
        continue;
      }
      if (run_n && run_n + k > (uint32_t)group_max) {
        if (WRITE) { gfirst[w] = run_first; gsize[w] = run_n; ++w; }
        ++ng;
        run_n = 0;
      }
      if (!run_n) run_first = child_first_particle(c, o_first);
      run_n += k;
    }
    if (run_n) {
      if (WRITE) { gfirst[w] = run_first; gsize[w] = run_n; ++w; }
      ++ng;
    }
  } else if (id == 0) {  // the whole tree fits in one group
    if (WRITE) { gfirst[w] = o_first[0]; gsize[w] = mine; }
    ng = 1;
  }
  if (!WRITE) counts[id] = ng;
}

// ---------------------------------------------------------------------------
// Hilbert keys (crates/gadget-ng-parallel/src/sfc.rs:95-204)
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint64_t coords_to_hilbert(uint32_t ix, uint32_t iy, uint32_t iz, uint32_t p) {
  uint32_t x[3] = {ix, iy, iz};
  const uint32_t m = 1u << (p - 1);
  for (uint32_t q = m; q > 1; q >>= 1) {
    const uint32_t pm = q - 1;
#pragma unroll
    for (int i = 2; i >= 0; --i) {
      if (x[i] & q) {
        x[0] ^= pm;
      } else {
        uint32_t t = (x[0] ^ x[i]) & pm;
        x[0] ^= t;
        x[i] ^= t;
      }
    }
  }
  x[1] ^= x[0];
  x[2] ^= x[1];
  uint32_t t = 0;
  for (uint32_t q = m; q > 1; q >>= 1)
    if (x[2] & q) t ^= q - 1;
  x[0] ^= t;
  x[1] ^= t;
  x[2] ^= t;
  uint64_t h = 0;
  for (uint32_t k = 0; k < p; ++k) {
    h = (h << 1) | ((x[0] >> k) & 1u);
    h = (h << 1) | ((x[1] >> k) & 1u);
    h = (h << 1) | ((x[2] >> k) & 1u);
  }
  return h;
}

__device__ __forceinline__ uint32_t hilbert_coord(double x, double lo, double len) {
  double v = ddiv(dsub(x, lo), len);
  v = v < 0.0 ? 0.0 : (v > 1.0 - F64_EPSILON ? 1.0 - F64_EPSILON : v);  // f64::clamp
  return (uint32_t)dmul(v, 2097152.0);
}

__global__ void k_hilbert(const uint32_t* __restrict__ qx, const uint32_t* __restrict__ qy,
                          const uint32_t* __restrict__ qz, const uint32_t* __restrict__ id, int64_t n, double scale,
                          const TreeParams* __restrict__ prm, uint64_t* __restrict__ keys,
                          uint32_t* __restrict__ vals) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t ix = hilbert_coord(decode(qx[i], scale), prm->hlo[0], prm->hlen[0]);
  const uint32_t iy = hilbert_coord(decode(qy[i], scale), prm->hlo[1], prm->hlen[1]);
  const uint32_t iz = hilbert_coord(decode(qz[i], scale), prm->hlo[2], prm->hlen[2]);
  keys[i] = coords_to_hilbert(ix, iy, iz, 21);
  vals[i] = id ? id[i] : (uint32_t)i;
}

// spread_bits (crates/gadget-ng-parallel/src/sfc.rs:39-47): the 21 low bits of
// x to every third bit position.
__device__ __forceinline__ uint64_t spread3(uint64_t x) {
  x &= 0x1FFFFFull;
  x = (x | (x << 32)) & 0x1F00000000FFFFull;
  x = (x | (x << 16)) & 0x1F0000FF0000FFull;
  x = (x | (x << 8)) & 0x100F00F00F00F00Full;
  x = (x | (x << 4)) & 0x10C30C30C30C30C3ull;
  x = (x | (x << 2)) & 0x1249249249249249ull;
  return x;
}

// particle_morton (sfc.rs:54-81): the coordinates normalised and quantised as
// for the Hilbert keys, interleaved x | y << 1 | z << 2.
__global__ void k_morton(const uint32_t* __restrict__ qx, const uint32_t* __restrict__ qy,
                         const uint32_t* __restrict__ qz, const uint32_t* __restrict__ id, int64_t n, double scale,
                         const TreeParams* __restrict__ prm, uint64_t* __restrict__ keys,
                         uint32_t* __restrict__ vals) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint32_t ix = hilbert_coord(decode(qx[i], scale), prm->hlo[0], prm->hlen[0]);
  const uint32_t iy = hilbert_coord(decode(qy[i], scale), prm->hlo[1], prm->hlen[1]);
  const uint32_t iz = hilbert_coord(decode(qz[i], scale), prm->hlo[2], prm->hlen[2]);
  keys[i] = spread3(ix) | (spread3(iy) << 1) | (spread3(iz) << 2);
  vals[i] = id ? id[i] : (uint32_t)i;
}

__device__ __forceinline__ void mask_path(uint64_t hi, uint64_t lo, int depth, uint64_t* oh, uint64_t* ol) {
  if (depth <= 0) { *oh = 0; *ol = 0; return; }
  if (depth <= 21) {
    int keep = 3 * depth;  // bits 62..63-keep
    uint64_t m = keep >= 63 ? 0x7FFFFFFFFFFFFFFFull : (((1ull << keep) - 1) << (63 - keep));
    *oh = hi & m;
    *ol = 0;
  } else {
    int keep = 3 * (depth - 21);
    uint64_t m = keep >= 63 ? 0x7FFFFFFFFFFFFFFFull : (((1ull << keep) - 1) << (63 - keep));
    *oh = hi;
    *ol = lo & m;
  }
}

__global__ void k_export_paths(int64_t n, int64_t n_int, const uint8_t* __restrict__ o_depth,
                               const uint32_t* __restrict__ o_first, const uint8_t* __restrict__ leaf_depth,
                               const uint64_t* __restrict__ hi, const uint64_t* __restrict__ lo, uint64_t* nh,
                               uint64_t* nl, uint64_t* lh, uint64_t* ll) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < n_int) {
    uint32_t f = o_first[i];
    mask_path(hi[f], lo[f], o_depth[i], &nh[i], &nl[i]);
  }
  if (i < n) mask_path(hi[i], lo[i], leaf_depth ? leaf_depth[i] : 0, &lh[i], &ll[i]);
}

}  // namespace

// ===========================================================================
// launchers
// ===========================================================================
void launch_bbox_root(const Particles& p, int64_t n, double box, TreeBuffers& t, cudaStream_t s) {
  k_bbox_init<<<1, 32, 0, s>>>(t.bbox);
  TPM_LAUNCH_CHECK();
  k_bbox<<<grid_for(n, 256, 148 * 8), 256, 0, s>>>(p.qx, p.qy, p.qz, n, t.bbox);
  TPM_LAUNCH_CHECK();
  k_root<<<1, 32, 0, s>>>(t.bbox, box / TWO32, t.params);
  TPM_LAUNCH_CHECK();
}

void launch_tree_keys(const Particles& p, int64_t n, double box, TreeBuffers& t, cudaStream_t s) {
  k_tree_keys<<<grid_for(n, 256, 1ll << 30), 256, 0, s>>>(p.qx, p.qy, p.qz, n, box / TWO32, t.params, t.key_hi,
                                                          t.perm);
  TPM_LAUNCH_CHECK();
}

void launch_fix_ties(const Particles& p, int64_t n, double box, TreeBuffers& t, cudaStream_t s) {
  k_tie_low<<<grid_for(n, 256, 1ll << 30), 256, 0, s>>>(p.qx, p.qy, p.qz, n, box / TWO32, t.params, t.key_hi,
                                                        t.perm, t.key_lo_tmp);
  TPM_LAUNCH_CHECK();
  k_fix_ties<<<grid_for(n, 256, 1ll << 30), 256, 0, s>>>(n, t.key_hi, t.perm, t.key_lo_tmp, t.key_lo, t.err);
  TPM_LAUNCH_CHECK();
}

void launch_permute(const Particles& src, const Particles& dst, int64_t n, const uint32_t* perm, cudaStream_t s) {
  k_permute<<<grid_for(n, 256, 1ll << 30), 256, 0, s>>>(src, dst, n, perm);
  TPM_LAUNCH_CHECK();
}

void launch_karras(int64_t n, TreeBuffers& t, cudaStream_t s) {
  if (n < 2) return;
  k_karras<<<grid_for(n - 1, 256, 1ll << 30), 256, 0, s>>>(n, t.key_hi, t.key_lo, t.bin_left, t.bin_right,
                                                           t.bin_prefix, t.bin_first, t.bin_last, t.bin_parent,
                                                           t.leaf_bparent);
  TPM_LAUNCH_CHECK();
  k_oct_count<<<grid_for(n - 1, 256, 1ll << 30), 256, 0, s>>>(n - 1, t.bin_prefix, t.bin_parent, t.oct_count);
  TPM_LAUNCH_CHECK();
}

void launch_octree_nodes(int64_t n, TreeBuffers& t, cudaStream_t s) {
  k_oct_nodes<<<grid_for(n - 1, 256, 1ll << 30), 256, 0, s>>>(n - 1, t.bin_prefix, t.bin_parent, t.bin_first,
                                                              t.bin_last, t.oct_count, t.oct_base, t.o_parent,
                                                              t.o_depth, t.o_first, t.o_last, &t.scalars[2]);
  TPM_LAUNCH_CHECK();
  k_leaf_parents<<<grid_for(n, 256, 1ll << 30), 256, 0, s>>>(n, t.leaf_bparent, t.bin_parent, t.oct_count,
                                                             t.oct_base, t.o_depth, t.leaf_oparent, t.leaf_depth);
  TPM_LAUNCH_CHECK();
}

void launch_octree_links(int64_t n, int64_t n_int, TreeBuffers& t, void* scan_scratch, cudaStream_t s) {
  TPM_CUDA(cudaMemsetAsync(t.o_slots, 0xFF, (size_t)n_int * 8 * sizeof(uint32_t), s));
  k_oct_slots_nodes<<<grid_for(n_int, 256, 1ll << 30), 256, 0, s>>>(n_int, t.o_parent, t.o_depth, t.o_first,
                                                                    t.key_hi, t.key_lo, t.o_slots);
  TPM_LAUNCH_CHECK();
  k_oct_slots_leaves<<<grid_for(n, 256, 1ll << 30), 256, 0, s>>>(n, t.leaf_oparent, t.leaf_depth, t.key_hi,
                                                                 t.key_lo, t.o_slots);
  TPM_LAUNCH_CHECK();
  k_oct_nchild<<<grid_for(n_int, 256, 1ll << 30), 256, 0, s>>>(n_int, t.o_slots, t.o_nchild);
  TPM_LAUNCH_CHECK();
  exclusive_scan_u32(t.o_nchild, t.o_child_first, n_int, &t.scalars[3], scan_scratch, s);
  k_oct_childlist<<<grid_for(n_int, 256, 1ll << 30), 256, 0, s>>>(n_int, t.o_slots, t.o_child_first, t.child_ids);
  TPM_LAUNCH_CHECK();
}

// Level by level from the deepest internal nodes to the root: each launch
// finishes one depth, so every node reads finished children without atomics
// or fences.  One host synchronisation brings the per-depth counts back.
void launch_aggregate(const Particles& p, int64_t n, int64_t n_int, double box, TreeBuffers& t, cudaStream_t s,
                      bool with_quad) {
  (void)n;
  if (n_int <= 0) return;
  uint32_t* hist = t.depth_tab;
  TPM_CUDA(cudaMemsetAsync(hist, 0, DEPTH_BINS * sizeof(uint32_t), s));
  k_depth_count<<<grid_for(n_int, 256, 1ll << 30), 256, 0, s>>>(n_int, t.o_depth, hist);
  TPM_LAUNCH_CHECK();
  k_depth_offsets<<<1, 32, 0, s>>>(t.depth_tab);
  TPM_LAUNCH_CHECK();
  uint32_t counts[DEPTH_BINS];
  TPM_CUDA(cudaMemcpyAsync(counts, hist, sizeof(counts), cudaMemcpyDeviceToHost, s));
  k_depth_scatter<<<grid_for(n_int, 256, 1ll << 30), 256, 0, s>>>(n_int, t.o_depth, t.depth_tab + 2 * DEPTH_BINS + 1,
                                                                   t.o_cnt);
  TPM_LAUNCH_CHECK();
  TPM_CUDA(cudaStreamSynchronize(s));
  int64_t offset[DEPTH_BINS + 1];
  offset[0] = 0;
  for (int d = 0; d < DEPTH_BINS; ++d) offset[d + 1] = offset[d] + counts[d];
  if (offset[DEPTH_BINS] != n_int) throw Error(2, "octree depth buckets do not add up to the node count");
  for (int d = DEPTH_BINS - 1; d >= 0; --d) {
    if (counts[d] == 0) continue;
    if (with_quad)
      k_aggregate_level<true><<<grid_for(counts[d], 128, 1ll << 30), 128, 0, s>>>(
          t.o_cnt + offset[d], counts[d], box / TWO32, p.qx, p.qy, p.qz, p.mass, t.o_slots, t.o_mass, t.o_com,
          t.o_quad);
    else
      k_aggregate_level<false><<<grid_for(counts[d], 128, 1ll << 30), 128, 0, s>>>(
          t.o_cnt + offset[d], counts[d], box / TWO32, p.qx, p.qy, p.qz, p.mass, t.o_slots, t.o_mass, t.o_com,
          t.o_quad);
    TPM_LAUNCH_CHECK();
  }
  k_walk_nodes<<<grid_for(n_int, 256, 1ll << 30), 256, 0, s>>>(n_int, TWO32 / box, t.o_mass, t.o_com, t.o_walk);
  TPM_LAUNCH_CHECK();
}

void launch_cell_q(int64_t n_int, double box, TreeBuffers& t, cudaStream_t s) {
  if (n_int <= 0) return;
  k_cell_q<<<grid_for(n_int, 256, 1ll << 30), 256, 0, s>>>(n_int, TWO32 / box, t.params, t.o_depth, t.o_first,
                                                           t.key_hi, t.key_lo, t.o_quad, t.o_cell);
  TPM_LAUNCH_CHECK();
}

void launch_walk_records(const Particles& p, int64_t n, int64_t n_int, double thr, TreeBuffers& t, cudaStream_t s) {
  (void)n;
  k_walk_records<<<grid_for(n_int, 128, 1ll << 30), 128, 0, s>>>(n_int, p.qx, p.qy, p.qz, p.massf, t.leaf_depth,
                                                                 t.o_walk, t.o_depth, t.o_nchild, t.o_child_first,
                                                                 t.child_ids, t.params, thr, t.recs);
  TPM_LAUNCH_CHECK();
}

void launch_groups(int64_t n, int64_t n_int, int group_max, TreeBuffers& t, void* scan_scratch, cudaStream_t s) {
  (void)n;
  k_groups<false><<<grid_for(n_int, 256, 1ll << 30), 256, 0, s>>>(n_int, group_max, t.o_slots, t.o_first, t.o_last,
                                                                  t.grp_count_per_node, nullptr, nullptr, nullptr);
  TPM_LAUNCH_CHECK();
  exclusive_scan_u32(t.grp_count_per_node, t.grp_base, n_int, &t.scalars[1], scan_scratch, s);
  k_groups<true><<<grid_for(n_int, 256, 1ll << 30), 256, 0, s>>>(n_int, group_max, t.o_slots, t.o_first, t.o_last,
                                                                 nullptr, t.grp_base, t.grp_first, t.grp_size);
  TPM_LAUNCH_CHECK();
}

void launch_hilbert_keys(const Particles& p, int64_t n, double box, const TreeParams* prm, uint64_t* keys,
                         uint32_t* vals, cudaStream_t s) {
  k_hilbert<<<grid_for(n, 256, 1ll << 30), 256, 0, s>>>(p.qx, p.qy, p.qz, p.id, n, box / TWO32, prm, keys, vals);
  TPM_LAUNCH_CHECK();
}

void launch_morton_keys(const Particles& p, int64_t n, double box, const TreeParams* prm, uint64_t* keys,
                        uint32_t* vals, cudaStream_t s) {
  k_morton<<<grid_for(n, 256, 1ll << 30), 256, 0, s>>>(p.qx, p.qy, p.qz, p.id, n, box / TWO32, prm, keys, vals);
  TPM_LAUNCH_CHECK();
}

void launch_export_paths(int64_t n, int64_t n_int, const TreeBuffers& t, uint64_t* node_hi, uint64_t* node_lo,
                         uint64_t* leaf_hi, uint64_t* leaf_lo, cudaStream_t s) {
  int64_t m = n > n_int ? n : n_int;
  k_export_paths<<<grid_for(m, 256, 1ll << 30), 256, 0, s>>>(n, n_int, t.o_depth, t.o_first,
                                                             n > 1 ? t.leaf_depth : nullptr, t.key_hi, t.key_lo,
                                                             node_hi, node_lo, leaf_hi, leaf_lo);
  TPM_LAUNCH_CHECK();
}

}  // namespace tpm
