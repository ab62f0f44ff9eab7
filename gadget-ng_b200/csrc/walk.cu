// Short-range TreePM walk, one warp per target group.
//
// Semantics (crates/gadget-ng-treepm/src/short_range.rs:274-333, periodic;
// :157-208, aperiodic): for each target particle the reference pops nodes
// from a stack, drops a node whose AABB (centred on its centre of mass, half
// side = the cell's half side) lies beyond r_cut, adds the pair force of a
// leaf (periodic walk: only if the bare minimum-image distance is within
// r_cut), takes an internal node whose half side is below 0.1 r_cut as a
// monopole (unless its centre of mass sits on the target), and otherwise
// opens it.  An internal node's cull hides all its descendants, so whether a
// target interacts with a node depends on every ancestor on its path.
//
// Warp design: the 32 lanes hold up to 32 target particles from one compact
// subtree.  The warp walks the tree once for all of them: each stack entry
// carries a 32-bit mask of the targets that still see that node.  Nodes are
// classified against the group's bounding box in FP32 with a safety margin
// (certainly culled / certainly kept for every target / undecided); undecided
// internal nodes get a per-target test when they are popped, which refines the
// mask, so the hierarchical culls of the reference are reproduced exactly.
// Terminal nodes (leaves and monopole-depth cells) go to an interaction list
// in shared memory; the lanes evaluate the list against the group's targets
// with each target's own final test fused into the pair kernel (a group of c
// targets gives every target 32 / c lanes, each on a share of the entries).
// The running per-target sums, the targets' positions and the group box stay
// in shared memory (read where a flush, a refinement or a classification
// needs them), so the traversal keeps its registers: 7 resident blocks per SM
// at 72 registers.  Any decision
// that falls inside a narrow band around r_cut is re-evaluated in float64
// with the reference's exact expression, so the interaction set equals the
// reference's.  Pair arithmetic is FP32: exact fixed-point differences split
// into two floats, rsqrt / rcp / ex2 hardware approximations, the A&S 7.1.26
// erfc, and Kahan-compensated per-target accumulators.
#include <cstdlib>

#include "common.cuh"
#include "tree.cuh"
#include "walk.cuh"

namespace tpm {
namespace {

constexpr int WALK_WARPS = 4;
constexpr int WALK_THREADS = WALK_WARPS * 32;
constexpr int CHUNK_L = 64;  // leaf-list capacity (walk 72.9 -> 72.5 ms at 256^3 against 48; 32 is slower)
// monopole-list capacity: the accurate mode also emits monopoles at pop time
template <bool ACC> constexpr int chunk_m() { return ACC ? 96 : 64; }
constexpr int32_t WIDE_GROUP = 1 << 28;  // quanta: 1/16 of the box


// One interaction-list entry (32 bytes): the source position relative to
// the group's first target in walk units (one rounding of the exact int32
// difference; the group is compact, so the rounding stays far below the
// softening length and the float64 band settles every borderline cut), mass,
// cull half side (0 for periodic leaves), the mask of targets that see it and
// the node (LEAF_BIT | particle for leaves).
struct __align__(16) Entry {
  float x, y, z, m;
  float h;
  uint32_t mask, node, pad;
};

__device__ __forceinline__ int32_t rel32(uint32_t a, uint32_t b, int periodic) {
  if (periodic) return (int32_t)(a - b);  // minimum image modulo 2^32
  int64_t d = (int64_t)a - (int64_t)b;
  d = d > 0x7FFFFFFFll ? 0x7FFFFFFFll : (d < -0x7FFFFFFFll ? -0x7FFFFFFFll : d);
  return (int32_t)d;
}


__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v, int lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    uint32_t y = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += y;
  }
  return v;
}

// h0 * 2^-dep by exponent arithmetic: h0 (the root half side in walk units,
// O(r_cut / cell)) stays a normal float for every tree depth (-1 <= dep < 64).
__device__ __forceinline__ float half_side(float h0, int dep) {
  return __int_as_float(__float_as_int(h0) - dep * (1 << 23));
}

// ---- float64 decisions with the reference's expressions -------------------
__device__ __forceinline__ double aabb_axis(double dc, double h) {
  double e = dsub(fabs(dc), h);
  return e > 0.0 ? e : 0.0;
}

// min_dist2_to_aabb_periodic (short_range.rs:72-84) or its aperiodic twin (:173-181).
__device__ __forceinline__ double d2_aabb(const double xi[3], const double com[3], double h, double box, int periodic) {
  double e[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    double dc = dsub(com[a], xi[a]);
    if (periodic) dc = minimum_image(dc, box);
    e[a] = aabb_axis(dc, h);
  }
  return dadd(dadd(dmul(e[0], e[0]), dmul(e[1], e[1])), dmul(e[2], e[2]));
}

__device__ __forceinline__ void target_pos(const WalkArgs& a, uint32_t p, double xi[3]) {
  xi[0] = decode(a.qx[p], a.scale);
  xi[1] = decode(a.qy[p], a.scale);
  xi[2] = decode(a.qz[p], a.scale);
}

__device__ __forceinline__ void node_com(const WalkArgs& a, uint32_t node, double c[3]) {
  if (node & LEAF_BIT) {
    uint32_t j = node & ~LEAF_BIT;
    c[0] = decode(a.qx[j], a.scale);
    c[1] = decode(a.qy[j], a.scale);
    c[2] = decode(a.qz[j], a.scale);
  } else {
    c[0] = a.o_com[3 * (int64_t)node];
    c[1] = a.o_com[3 * (int64_t)node + 1];
    c[2] = a.o_com[3 * (int64_t)node + 2];
  }
}

// Does target p keep open internal node `node` (cull test only)?
__device__ __forceinline__ bool exact_open_pass(const WalkArgs& a, uint32_t p, uint32_t node) {
  double xi[3], c[3];
  target_pos(a, p, xi);
  node_com(a, node, c);
  double h = ldexp(a.h0, -(int)a.depth[node]);
  return !(d2_aabb(xi, c, h, a.box, a.periodic) > a.rc2);
}

// Terminal node decision: 0 = skip, 1 = interact, 2 = open for this target
// (monopole whose centre of mass coincides with the target).
__device__ __forceinline__ int exact_terminal(const WalkArgs& a, uint32_t p, uint32_t node) {
  double xi[3], c[3];
  target_pos(a, p, xi);
  node_com(a, node, c);
  if (node & LEAF_BIT) {
    uint32_t j = node & ~LEAF_BIT;
    if (a.periodic) {
      double r[3];
#pragma unroll
      for (int k = 0; k < 3; ++k) r[k] = minimum_image(dsub(c[k], xi[k]), a.box);
      double r2 = dadd(dadd(dmul(r[0], r[0]), dmul(r[1], r[1])), dmul(r[2], r[2]));
      return r2 > a.rc2 ? 0 : 1;
    }
    double h = ldexp(a.h0, -(int)a.leaf_depth[j]);
    return d2_aabb(xi, c, h, a.box, 0) > a.rc2 ? 0 : 1;
  }
  double h = ldexp(a.h0, -(int)a.depth[node]);
  if (d2_aabb(xi, c, h, a.box, a.periodic) > a.rc2) return 0;
  double d[3];
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    d[k] = dsub(c[k], xi[k]);
    if (a.periodic) d[k] = minimum_image(d[k], a.box);
  }
  double d2 = dadd(dadd(dmul(d[0], d[0]), dmul(d[1], d[1])), dmul(d[2], d[2]));
  return d2 > 1e-30 ? 1 : 2;
}

__device__ __forceinline__ void defer(const WalkArgs& a, uint32_t p, uint32_t node) {
  uint32_t slot = atomicAdd(a.ndeferred, 1u);
  if (slot < a.cap_deferred) a.deferred[slot] = make_uint2(p, node);
  else atomicOr(a.err, DEV_ERR_DEFERRED);
}

// FP32 pair term: returns m * erfc(x) / r^3 (walk units), x = r/(sqrt2 r_s);
// ACC (accurate mode) adds the Gaussian term (2x/sqrt(pi)) exp(-x^2).
template <bool ACC = false>
__device__ __forceinline__ float pair_factor(const WalkArgs& a, float r2b, float m) {
  float r2 = fmaxf(r2b + a.eps2_u, 1e-30f);
  float ri = rsqrt_approx(r2);
  float r = r2 * ri;
  float tt = rcp_approx(fmaf(a.pcx, r, 1.0f));
  float poly = tt * fmaf(tt, fmaf(tt, fmaf(tt, fmaf(tt, ErfcConst::A5, ErfcConst::A4), ErfcConst::A3), ErfcConst::A2),
                         ErfcConst::A1);
  if (ACC) poly = fmaf(a.gkc, r, poly);
  const float w = poly * ex2_approx(r2 * a.ex2k);
  return m * w * (ri * ri * ri);
}

struct Acc {
  float sx, sy, sz, cx, cy, cz;  // Kahan sums and compensations
  __device__ void add(float x, float y, float z) {
    float t, v;
    v = x - cx; t = sx + v; cx = (t - sx) - v; sx = t;
    v = y - cy; t = sy + v; cy = (t - sy) - v; sy = t;
    v = z - cz; t = sz + v; cz = (t - sz) - v; sz = t;
  }
};

// Lanes of the pair phase.  A group of c targets leaves 32 - c lanes without
// a target of their own, so R = 32 / c lanes share each target: lane l
// evaluates target l % c against entries l / c, l / c + R, ... of each list
// (lanes from R c on evaluate nothing), and the R partial sums of a target
// are folded when its walk ends.  Packed in one register: target | first
// entry << 8 | R << 16.
__device__ __forceinline__ uint32_t pair_lanes(int lane, uint32_t c) {
  const uint32_t r = 32u / c, t = (uint32_t)lane % c, off = (uint32_t)lane / c;
  return t | ((off < r ? off : 255u) << 8) | (r << 16);
}

// Evaluate one interaction list against this lane's pair-phase target.  MONO
// selects the monopole list (AABB-gap test) or the leaf list (bare-distance
// test; the aperiodic walk's leaves carry their half side and take the AABB
// test too).  Borderline pairs are left out here and flagged; resolve_list
// settles them.
template <bool MONO, bool ACC>
__device__ __forceinline__ void flush_list(const WalkArgs& a, const Entry* L, int nl, uint32_t lanes, float tx,
                                           float ty, float tz, float& fx, float& fy, float& fz, uint32_t& nok,
                                           bool& amb_any) {
  const int t = lanes & 0xffu, stride = lanes >> 16;
#pragma unroll 1
  for (int e = (lanes >> 8) & 0xffu; e < nl; e += stride) {
    const float4 A = *reinterpret_cast<const float4*>(&L[e].x);
    const uint4 B = *reinterpret_cast<const uint4*>(&L[e].h);
    const float h = __uint_as_float(B.x);
    const uint32_t mask = B.y;
    const float dx = A.x - tx, dy = A.y - ty, dz = A.z - tz;
    const float r2b = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
    float s = r2b;
    if (MONO || !a.periodic) {
      const float ex = fmaxf(fabsf(dx) - h, 0.f), ey = fmaxf(fabsf(dy) - h, 0.f);
      const float ez = fmaxf(fabsf(dz) - h, 0.f);
      s = fmaf(ex, ex, fmaf(ey, ey, ez * ez));
    }
    const bool in = (mask >> t) & 1u;
    bool ok = in && s <= a.prc2_lo;
    if (!ACC) {  // accurate mode reproduces no float64 decisions
      // s in (prc2_lo, prc2_hi]: positive floats order like their bit patterns
      bool amb = in && (__float_as_uint(s) - a.prc2_lo_bits - 1u) < a.pband_bits;
      if (MONO) {
        // a centre of mass within a few quanta of the target: resolve_list
        // alone decides it (take it, or open it when it is the target's own
        // position), so it must not enter the sum here as well
        const bool near = in && r2b < a.tiny_u;
        amb = amb || near;
        ok = ok && !near;
      }
      amb_any = amb_any || amb;
    }
    float f = pair_factor<ACC>(a, r2b, A.w);
    f = ok ? f : 0.f;
    fx = fmaf(dx, f, fx);
    fy = fmaf(dy, f, fy);
    fz = fmaf(dz, f, fz);
    nok += ok ? 1u : 0u;  // the target's own leaf is masked out at emission
  }
}

// Float64 decisions for this lane's borderline pairs of one list (rare).
template <bool MONO>
__device__ __noinline__ void resolve_list(const WalkArgs& a, const Entry* L, int nl, uint32_t lanes, uint32_t p,
                                          float tx, float ty, float tz, float* f3, uint32_t* nok, uint32_t* nexact) {
  const int t = lanes & 0xffu, stride = lanes >> 16;
  for (int e = (lanes >> 8) & 0xffu; e < nl; e += stride) {
    const float4 A = *reinterpret_cast<const float4*>(&L[e].x);
    const uint4 B = *reinterpret_cast<const uint4*>(&L[e].h);
    const float h = __uint_as_float(B.x);
    const uint32_t mask = B.y, node = B.z;
    const float dx = A.x - tx, dy = A.y - ty, dz = A.z - tz;
    const float r2b = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
    float s = r2b;
    if (MONO || !a.periodic) {
      const float ex = fmaxf(fabsf(dx) - h, 0.f), ey = fmaxf(fabsf(dy) - h, 0.f);
      const float ez = fmaxf(fabsf(dz) - h, 0.f);
      s = fmaf(ex, ex, fmaf(ey, ey, ez * ez));
    }
    const bool in = (mask >> t) & 1u;
    bool amb = in && s > a.prc2_lo && s <= a.prc2_hi;
    if (MONO) amb = amb || (in && r2b < a.tiny_u);
    if (!amb) continue;
    ++*nexact;
    const int d = exact_terminal(a, p, node);
    if (d == 2) defer(a, p, node);
    if (d != 1) continue;
    const float f = pair_factor(a, r2b, A.w);
    f3[0] = fmaf(dx, f, f3[0]);
    f3[1] = fmaf(dy, f, f3[1]);
    f3[2] = fmaf(dz, f, f3[2]);
    ++*nok;
  }
}

// Evaluate both interaction lists against this lane's pair-phase target
// (pair_lanes; its position is read from the lane that holds it, its
// particle is first + target).
// The lane's running sums live in shared memory between flushes (s0 = sx, sy,
// sz, cx; s1 = cy, cz, leaf count, monopole count bits), so they hold no
// registers across the traversal.
template <bool ACC>
__device__ __forceinline__ void flush(const WalkArgs& a, const Entry* Ll, int nll, const Entry* Lm, int nlm, int lane,
                                      uint32_t count, uint32_t first, const float4* tfs, float4* s0, float4* s1,
                                      uint32_t& nexact, uint32_t& neval) {
  const uint32_t lanes = pair_lanes(lane, count);  // recomputed here: one register less across the traversal
  uint32_t nleaf = 0, nmono = 0;
  float fx = 0.f, fy = 0.f, fz = 0.f;
  bool amb_any = false;
  neval += (uint32_t)(nll + nlm);
  const int t = lanes & 0xffu;
  const float4 T = tfs[t];
  const float tx = T.x, ty = T.y, tz = T.z;
  flush_list<false, ACC>(a, Ll, nll, lanes, tx, ty, tz, fx, fy, fz, nleaf, amb_any);
  flush_list<true, ACC>(a, Lm, nlm, lanes, tx, ty, tz, fx, fy, fz, nmono, amb_any);
  if (!ACC && amb_any) {
    float f3[3] = {fx, fy, fz};
    const uint32_t p = first + (uint32_t)t;
    resolve_list<false>(a, Ll, nll, lanes, p, tx, ty, tz, f3, &nleaf, &nexact);
    resolve_list<true>(a, Lm, nlm, lanes, p, tx, ty, tz, f3, &nmono, &nexact);
    fx = f3[0];
    fy = f3[1];
    fz = f3[2];
  }
  __syncwarp();
  const float4 A = s0[lane], B = s1[lane];
  Acc acc = {A.x, A.y, A.z, A.w, B.x, B.y};
  acc.add(fx, fy, fz);
  s0[lane] = make_float4(acc.sx, acc.sy, acc.sz, acc.cx);
  s1[lane] = make_float4(acc.cy, acc.cz, __uint_as_float(__float_as_uint(B.z) + nleaf),
                         __uint_as_float(__float_as_uint(B.w) + nmono));
}

// Stack entry of an open node: its children's record range, mask of the
// targets that see it (refined per target before the push), and the octree id.
struct __align__(16) StackEntry {
  uint32_t first;  // record index of the first child
  uint32_t info;   // the node's record info | INFO_MAC when its opening angle is undecided for the group
  uint32_t mask;
  uint32_t ref;    // octree node id
};
constexpr int STACK_ENTRIES = 1024;  // global, per warp
constexpr uint32_t INFO_MAC = 0x40000000u;  // opening angle undecided for the group

// Walk the tree for targets [first, first + count) (count <= TPW) with one warp.
template <int TPW, bool ACC>
__device__ void walk_targets(const WalkArgs& a, uint32_t first, uint32_t count, Entry* Ll, Entry* Lm, uint8_t* owner,
                             StackEntry* stk, float4* rpos, uint4* rmask, float4* s0, float4* s1, float4* tfs,
                             float4* gbox) {
  const int lane = threadIdx.x & 31;
  const int tgt = lane & (TPW - 1);  // this lane's target within the group
  const uint32_t p = first + ((uint32_t)tgt < count ? (uint32_t)tgt : 0u);
  // targets of this walk: the group's particles, or those of them the caller
  // selected (the group box then covers only those)
  const bool has = (uint32_t)tgt < count && (!a.only || a.only[p] != 0);
  const uint32_t tq[3] = {a.qx[p], a.qy[p], a.qz[p]};
  uint32_t oq[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) oq[d] = __shfl_sync(0xffffffffu, tq[d], 0);
  int32_t tr[3];
  float tf[3], bmin[3], bmax[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    tr[d] = rel32(tq[d], oq[d], a.periodic);
    tf[d] = (float)tr[d] * a.u_inv;
    int32_t mn = __reduce_min_sync(0xffffffffu, has ? tr[d] : 0x7FFFFFFF);
    int32_t mx = __reduce_max_sync(0xffffffffu, has ? tr[d] : -0x7FFFFFFF);
    bmin[d] = (float)mn * a.u_inv;
    bmax[d] = (float)mx * a.u_inv;
  }
  // the group box, its origin and the targets' positions wait in shared
  // memory (read when a node is classified, refined or flushed): registers
  // for the traversal
  tfs[lane] = make_float4(tf[0], tf[1], tf[2], 0.f);
  if (lane == 0) {
    gbox[0] = make_float4(bmin[0], bmin[1], bmin[2], 0.f);
    gbox[1] = make_float4(bmax[0], bmax[1], bmax[2], 0.f);
    reinterpret_cast<uint4*>(gbox)[2] = make_uint4(oq[0], oq[1], oq[2], 0u);
  }
  __syncwarp();
  const uint32_t mask0 = __ballot_sync(0xffffffffu, has && lane < TPW);  // bit t: target t
  s0[lane] = make_float4(0.f, 0.f, 0.f, 0.f);
  s1[lane] = make_float4(0.f, 0.f, 0.f, 0.f);
  uint32_t nexact = 0, neval = 0;
  int nll = 0, nlm = 0, sp = 0;

  // the first item is the root record
  bool have = lane == 0;
  uint32_t item = 0;
  uint32_t imask = mask0;
  // each iteration pops at least one node, so a walk over a well-formed tree
  // ends within (internal nodes + 1) iterations; the cap turns a malformed
  // tree into an error flag instead of an endless loop
  uint32_t iter_left = (uint32_t)(a.n_int + 2 < 0xFFFFFFFFll ? a.n_int + 2 : 0xFFFFFFFFll);

  for (;;) {
    if (iter_left-- == 0u) {
      if (lane == 0) atomicOr(a.err, DEV_ERR_STACK);
      break;
    }
    // ---- classify this lane's item against the group box
    bool emit = false, push = false, ambig = false, is_leaf = false;
    Entry ent;
    StackEntry se;
    float sx = 0.f, sy = 0.f, sz = 0.f, sh = 0.f;  // an undecided open node: group-relative COM, cull half side
    uint32_t simg = 0u;
    if (have && imask != 0u) {
      const uint4 r0 = __ldg(reinterpret_cast<const uint4*>(&a.recs[item]));
      const uint4 r1 = __ldg(reinterpret_cast<const uint4*>(&a.recs[item]) + 1);
      const uint32_t info = r1.y;
      const bool leaf = (info & WN_LEAF) != 0;
      const int dep = wn_depth(info);
      const float hnode = half_side(a.h0_u, dep);
      // cull half side: the COM-centred AABB of the reference, or (accurate
      // mode) twice that, which holds the whole cell
      const float h = (leaf && a.periodic) ? 0.f : (ACC && !leaf ? 2.f * hnode : hnode);
      const uint32_t cq[3] = {r0.x, r0.y, r0.z};
      const float4 GL = gbox[0], GH = gbox[1];
      const uint4 GO = reinterpret_cast<const uint4*>(gbox)[2];
      const float bmin[3] = {GL.x, GL.y, GL.z}, bmax[3] = {GH.x, GH.y, GH.z};
      const uint32_t oq[3] = {GO.x, GO.y, GO.z};
      // Per axis, the targets see the node at the minimum image of S - t for t
      // in [bmin, bmax]: bound min / max of |wrap(S - t)| over that interval
      // (images at 0 and +-L), then the AABB gap.
      float emin2 = 0.f, emax2 = 0.f, dmin2 = 0.f, dmax2 = 0.f;
      int32_t S[3];
      float SF[3];
#pragma unroll
      for (int d = 0; d < 3; ++d) {
        S[d] = rel32(cq[d], oq[d], a.periodic);
        const float sf = (float)S[d] * a.u_inv;
        SF[d] = sf;
        const float lo = sf - bmax[d], hi = sf - bmin[d];
        float dmin = lo > 0.f ? lo : (hi < 0.f ? -hi : 0.f);
        float dmax = fmaxf(fabsf(lo), fabsf(hi));
        // the +-L images can only come within r_cut of a group (narrower than
        // L/16) for nodes of half side near L/2: the top levels
        if (a.periodic && dep < a.img_depth) {
          dmin = fminf(dmin, fminf(a.box_u - hi, lo + a.box_u));
          const float half = 0.5f * a.box_u;
          if (lo <= -half || hi >= half) dmax = half;
          else dmax = fminf(dmax, half);
        }
        const float gap = fmaxf(dmin - h, 0.f);
        const float far = fmaxf(dmax - h, 0.f);
        emin2 = fmaf(gap, gap, emin2);
        emax2 = fmaf(far, far, emax2);
        dmin2 = fmaf(dmin, dmin, dmin2);
        dmax2 = fmaf(dmax, dmax, dmax2);
      }
      bool open, macmix = false;
      if (ACC && !leaf) {
        bool accept_all, open_all;
        if (a.relative) {
          // relative criterion (octree.rs:769-796): accept when the target is
          // outside the node's cell and |Q|_F (d^2 + eps^2) < k M d^5; that
          // bound falls with d, so the group's nearest and farthest COM
          // distances decide it for every target, and a group box touching
          // the cell leaves the node to the per-target test.  Nodes at the
          // top levels (periodic images) are always opened.
          const uint4 cc = __ldg(&a.cellq[r1.z]);
          const float qf = __uint_as_float(cc.w), m = __uint_as_float(r0.w);
          const uint32_t ccq[3] = {cc.x, cc.y, cc.z};
          bool touch = true, inside_all = true;
#pragma unroll
          for (int d = 0; d < 3; ++d) {
            const float c = (float)rel32(ccq[d], oq[d], a.periodic) * a.u_inv;
            const float lo = c - hnode * 1.0001f, hi = c + hnode * 1.0001f;
            touch = touch && lo <= bmax[d] && hi >= bmin[d];
            inside_all = inside_all && lo <= bmin[d] && hi >= bmax[d];
          }
          const float dmn = sqrtf(dmin2), dmx = sqrtf(dmax2);
          accept_all = !touch && dmin2 > 0.f &&
                       qf * (dmin2 + a.eps2_u) < a.rel_k * m * (dmin2 * dmin2 * dmn) * 0.999f;
          open_all = (a.periodic && dep < a.img_depth) || inside_all ||
                     !(qf * (dmax2 + a.eps2_u) < a.rel_k * m * (dmax2 * dmax2 * dmx) * 1.001f);
          accept_all = accept_all && !open_all;
        } else {
          // opening angle s/d < theta, s = 2 * half side (octree.rs:763-809);
          // a margin on both sides leaves the float-rounding cases to the
          // per-target test at pop time
          const float s2 = 4.f * hnode * hnode;
          accept_all = s2 < a.theta2 * dmin2 * 0.999f;
          open_all = s2 >= a.theta2 * dmax2 * 1.001f;
        }
        open = !accept_all;
        macmix = !accept_all && !open_all;
      } else {
        open = !leaf && !(info & WN_TERMINAL);
      }
      if (!(emin2 > a.grc2_hi)) {
        if (open) {
          push = true;
          ambig = !(emax2 < a.grc2_lo);
          se.first = r1.x;
          se.info = info | (macmix ? INFO_MAC : 0u);
          se.mask = imask;
          se.ref = r1.z;
          if (ambig) {
            sx = SF[0];
            sy = SF[1];
            sz = SF[2];
            sh = h;
            simg = (a.periodic && dep < a.img_depth) ? 1u : 0u;
          }
        } else {
          emit = true;
          ent.x = (float)S[0] * a.u_inv;
          ent.y = (float)S[1] * a.u_inv;
          ent.z = (float)S[2] * a.u_inv;
          ent.m = __uint_as_float(r0.w);
          ent.h = h;
          // the reference skips the target's own leaf (j != skip)
          const uint32_t own = leaf ? r1.z - first : 32u;
          ent.mask = own < count ? (imask & ~(1u << own)) : imask;
          ent.node = leaf ? (r1.z | LEAF_BIT) : r1.z;
          is_leaf = leaf;
        }
      }
    }
    // ---- append terminal entries to the leaf and monopole lists
    const uint32_t eml = __ballot_sync(0xffffffffu, emit && is_leaf);
    const uint32_t emm = __ballot_sync(0xffffffffu, emit && !is_leaf);
    if (emit) {
      const unsigned lt = (1u << lane) - 1u;
      Entry* dstE = is_leaf ? &Ll[nll + __popc(eml & lt)] : &Lm[nlm + __popc(emm & lt)];
      float4* dst = reinterpret_cast<float4*>(dstE);
      dst[0] = make_float4(ent.x, ent.y, ent.z, ent.m);
      *reinterpret_cast<uint4*>(&dst[1]) = make_uint4(__float_as_uint(ent.h), ent.mask, ent.node, 0u);
    }
    nll += __popc(eml);
    nlm += __popc(emm);
    // ---- per-target refinement of open nodes undecided for the group, before
    // they are pushed: each node is staged once (group-relative COM, cull half
    // side) in shared memory, then tested against all targets (one per lane)
    // from a broadcast load.  dd = COM - target in float differs from the exact
    // minimum-image difference by ~1e-7 of r_cut, far inside the band that goes
    // to the float64 test.  A node no target sees is not pushed.
    const uint32_t below = (1u << lane) - 1u;
    const uint32_t amb = __ballot_sync(0xffffffffu, push && ambig);
    if (push && ambig) {
      const int j = __popc(amb & below);
      rpos[j] = make_float4(sx, sy, sz, sh);
      rmask[j] = make_uint4(se.mask, se.ref, simg, 0u);
    }
    __syncwarp();
    const int namb = __popc(amb);
    const float4 TF = tfs[lane];
    const float tfl[3] = {TF.x, TF.y, TF.z};
    for (int j = 0; j < namb; ++j) {
      const float4 R = rpos[j];
      const uint4 M = rmask[j];
      bool pass = false;
      if (has && lane < TPW && ((M.x >> tgt) & 1u)) {
        const float rc[3] = {R.x, R.y, R.z};
        float s = 0.f;
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          float dd = rc[d] - tfl[d];
          if (M.z) dd -= a.box_u * rintf(dd / a.box_u);  // top levels: the nearest periodic image
          const float ee = fmaxf(fabsf(dd) - R.w, 0.f);
          s = fmaf(ee, ee, s);
        }
        if (s <= a.rc2_lo) pass = true;
        else if (!ACC && s <= a.rc2_hi) {
          pass = exact_open_pass(a, p, M.y);
          ++nexact;
        }
      }
      const uint32_t nm = __ballot_sync(0xffffffffu, pass);  // lanes < TPW hold the targets
      if (lane == 0) rmask[j].x = nm;
    }
    __syncwarp();
    if (push && ambig) {
      se.mask = rmask[__popc(amb & below)].x;
      push = se.mask != 0u;
    }
    // ---- push open nodes
    const uint32_t pm = __ballot_sync(0xffffffffu, push);
    if (sp + __popc(pm) > STACK_ENTRIES) {
      if (lane == 0) atomicOr(a.err, DEV_ERR_STACK);
      break;
    }
    if (push) {
      const int slot = sp + __popc(pm & ((1u << lane) - 1u));
      *reinterpret_cast<uint4*>(&stk[slot]) = make_uint4(se.first, se.info, se.mask, se.ref);
    }
    sp += __popc(pm);
    __syncwarp();
    // before the next check the pop adds up to 32 monopole entries (accurate
    // mode) and the next classification up to 32 to either list
    // (one call site of the list evaluation, the last flush included: the
    // kernel's code stays small enough for the instruction cache)
    const bool done = sp == 0;
    if (done || nll > CHUNK_L - 32 || nlm > chunk_m<ACC>() - (ACC ? 64 : 32)) {
      if (nll + nlm > 0)
        flush<ACC>(a, Ll, nll, Lm, nlm, lane, count, first, tfs, s0, s1, nexact, neval);
      __syncwarp();
      nll = 0;
      nlm = 0;
    }
    if (done) break;
    // ---- pop a batch whose children fill at most one warp
    const int avail = sp < 32 ? sp : 32;
    uint4 e = make_uint4(0u, 0u, 0u, 0u);
    uint32_t nc = 0;
    if (lane < avail) {
      e = *reinterpret_cast<const uint4*>(&stk[sp - 1 - lane]);
      nc = wn_nchild(e.y);
    }
    const uint32_t incl = warp_incl_scan(nc, lane);
    const uint32_t take = __ballot_sync(0xffffffffu, lane < avail && incl <= 32u);
    const int k = __popc(take);
    sp -= k;
    uint4 wrec = make_uint4(0u, 0u, 0u, 0u), crec = make_uint4(0u, 0u, 0u, 0u);
    if (ACC && lane < k && (e.y & INFO_MAC)) {
      wrec = __ldg(&a.walk[e.w]);
      if (a.relative) crec = __ldg(&a.cellq[e.w]);
    }
    // accurate mode: per-target opening angle for nodes undecided for the
    // group; targets that accept take the node as a monopole now, the rest
    // open it
    uint32_t macm = ACC ? __ballot_sync(0xffffffffu, lane < k && (e.y & INFO_MAC)) : 0u;
    while (macm) {
      const int src = __ffs(macm) - 1;
      macm &= macm - 1;
      const uint32_t node = __shfl_sync(0xffffffffu, e.w, src);
      const uint32_t me = __shfl_sync(0xffffffffu, e.z, src);
      const int dep = wn_depth(__shfl_sync(0xffffffffu, e.y, src));
      const uint4 w = make_uint4(__shfl_sync(0xffffffffu, wrec.x, src), __shfl_sync(0xffffffffu, wrec.y, src),
                                 __shfl_sync(0xffffffffu, wrec.z, src), __shfl_sync(0xffffffffu, wrec.w, src));
      const float hnode = half_side(a.h0_u, dep);
      uint4 cw = make_uint4(0u, 0u, 0u, 0u);
      if (a.relative)
        cw = make_uint4(__shfl_sync(0xffffffffu, crec.x, src), __shfl_sync(0xffffffffu, crec.y, src),
                        __shfl_sync(0xffffffffu, crec.z, src), __shfl_sync(0xffffffffu, crec.w, src));
      bool accept = false;
      if (has && lane < TPW && ((me >> tgt) & 1u)) {
        float d2 = 0.f;
        const uint32_t wq[3] = {w.x, w.y, w.z};
#pragma unroll
        for (int d = 0; d < 3; ++d) {
          const float dd = (float)rel32(wq[d], tq[d], a.periodic) * a.u_inv;
          d2 = fmaf(dd, dd, d2);
        }
        if (a.relative) {
          // point_in_node_cell with a margin (a target on the cell's face
          // opens the node), then the truncation estimate
          const uint32_t cq3[3] = {cw.x, cw.y, cw.z};
          bool inside = true;
#pragma unroll
          for (int d = 0; d < 3; ++d)
            inside = inside && fabsf((float)rel32(cq3[d], tq[d], a.periodic) * a.u_inv) <= hnode * 1.0001f;
          const float qf = __uint_as_float(cw.w), m = __uint_as_float(w.w);
          accept = !inside && d2 > 0.f && qf * (d2 + a.eps2_u) < a.rel_k * m * (d2 * d2 * sqrtf(d2));
        } else {
          accept = 4.f * hnode * hnode < a.theta2 * d2;
        }
      }
      const uint32_t am = __ballot_sync(0xffffffffu, accept);
      if (am) {  // one monopole entry for the accepting targets (same slot on every lane)
        if (lane == src) {
          const uint4 GO = reinterpret_cast<const uint4*>(gbox)[2];
          const uint32_t oq[3] = {GO.x, GO.y, GO.z};
          float4* dst = reinterpret_cast<float4*>(&Lm[nlm]);
          dst[0] = make_float4((float)rel32(w.x, oq[0], a.periodic) * a.u_inv,
                               (float)rel32(w.y, oq[1], a.periodic) * a.u_inv,
                               (float)rel32(w.z, oq[2], a.periodic) * a.u_inv, __uint_as_float(w.w));
          *reinterpret_cast<uint4*>(&dst[1]) = make_uint4(__float_as_uint(2.f * hnode), am, node, 0u);
        }
        ++nlm;
      }
      if (lane == src) e.z = me & ~am;
    }
    __syncwarp();
    // distribute the children of the popped entries over the lanes
    const uint32_t excl = incl - nc;
    if (lane < k)
      for (uint32_t c = 0; c < nc; ++c) owner[excl + c] = (uint8_t)lane;
    __syncwarp();
    const uint32_t total = __shfl_sync(0xffffffffu, incl, k - 1);
    have = (uint32_t)lane < total;
    const int o = have ? owner[lane] : 0;
    const uint32_t ofirst = __shfl_sync(0xffffffffu, e.x, o);
    const uint32_t omask = __shfl_sync(0xffffffffu, e.z, o);
    const uint32_t oexcl = __shfl_sync(0xffffffffu, excl, o);
    __syncwarp();
    if (have) {
      item = ofirst + ((uint32_t)lane - oexcl);
      imask = omask;
    }
  }
  __syncwarp();
  __syncwarp();
  const float4 S0 = s0[lane], S1 = s1[lane];
  Acc acc = {S0.x, S0.y, S0.z, S0.w, S1.x, S1.y};
  uint32_t nleaf = __float_as_uint(S1.z), nmono = __float_as_uint(S1.w);
  // fold the R pair-phase lanes of each target (lanes t + j count) into lane t
  const uint32_t nrep = 32u / count;
  for (uint32_t j = 1; j < nrep; ++j) {
    const int src = lane + (int)(j * count);  // in range for the lanes t < count that keep the result
    const float ox = __shfl_sync(0xffffffffu, acc.sx, src), oy = __shfl_sync(0xffffffffu, acc.sy, src);
    const float oz = __shfl_sync(0xffffffffu, acc.sz, src);
    const float cx = __shfl_sync(0xffffffffu, acc.cx, src), cy = __shfl_sync(0xffffffffu, acc.cy, src);
    const float cz = __shfl_sync(0xffffffffu, acc.cz, src);
    const uint32_t ol = __shfl_sync(0xffffffffu, nleaf, src), om = __shfl_sync(0xffffffffu, nmono, src);
    if ((uint32_t)lane < count) {
      acc.add(ox - cx, oy - cy, oz - cz);
      nleaf += ol;
      nmono += om;
    }
  }
  if (has && lane < TPW) {
    a.ax[p] = (acc.sx - acc.cx) * a.out_scale;
    a.ay[p] = (acc.sy - acc.cy) * a.out_scale;
    a.az[p] = (acc.sz - acc.cz) * a.out_scale;
    a.pcounts[2 * (int64_t)p] = nleaf;
    a.pcounts[2 * (int64_t)p + 1] = nmono;
  }
  if ((uint32_t)lane >= count || lane >= TPW) nleaf = nmono = 0;  // counted once per target
  // statistics
  unsigned long long l = nleaf, m = nmono, x = nexact;
  for (int off = 16; off > 0; off >>= 1) {
    l += __shfl_down_sync(0xffffffffu, l, off);
    m += __shfl_down_sync(0xffffffffu, m, off);
    x += __shfl_down_sync(0xffffffffu, x, off);
  }
  if (lane == 0) {
    atomicAdd(&a.stats[0], l);
    atomicAdd(&a.stats[1], m);
    atomicAdd(&a.stats[2], (unsigned long long)neval * 32ull / nrep);  // lane evaluations
    atomicAdd(&a.stats[3], x);
  }
}

// per warp: the leaf and monopole lists, 32 staged undecided nodes (float4
// position + uint4 mask / node / image flag), the lanes' running sums (two
// float4 each), the child-owner bytes
template <bool ACC> constexpr size_t walk_smem_per_warp() {
  return sizeof(Entry) * (CHUNK_L + chunk_m<ACC>()) + 32 * (sizeof(float4) + sizeof(uint4)) + 100 * sizeof(float4) + 32;
}

template <int MIN_BLOCKS, int TPW, bool ACC>
__global__ void __launch_bounds__(WALK_THREADS, MIN_BLOCKS) k_walk(WalkArgs a) {
  extern __shared__ __align__(16) unsigned char s_walk[];
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  unsigned char* mine = s_walk + wid * walk_smem_per_warp<ACC>();
  Entry* list_l = reinterpret_cast<Entry*>(mine);
  Entry* list_m = list_l + CHUNK_L;
  float4* rpos = reinterpret_cast<float4*>(list_m + chunk_m<ACC>());
  uint4* rmask = reinterpret_cast<uint4*>(rpos + 32);
  float4* s0 = reinterpret_cast<float4*>(rmask + 32);
  float4* s1 = s0 + 32;
  float4* tfs = s1 + 32;   // 32 target positions
  float4* gbox = tfs + 32; // group box corners and origin (3, padded to 4)
  uint8_t* owner = reinterpret_cast<uint8_t*>(gbox + 4);
  const int64_t gw = (int64_t)blockIdx.x * WALK_WARPS + wid;
  StackEntry* stk = reinterpret_cast<StackEntry*>(a.stack) + gw * STACK_ENTRIES;
  for (;;) {
    uint32_t g = 0;
    if (lane == 0) g = atomicAdd(a.work, 1u);
    g = __shfl_sync(0xffffffffu, g, 0);
    if ((int64_t)g >= a.ngroups) break;
    const uint32_t first = a.gfirst[g], count = a.gsize[g];
    // a group wider than 1/16 of the box would break the shared-origin minimum
    // image: walk its targets one at a time instead
    const bool has = (uint32_t)(lane & (TPW - 1)) < count;
    const uint32_t p = first + (has ? (lane & (TPW - 1)) : 0);
    const uint32_t t0[3] = {a.qx[first], a.qy[first], a.qz[first]};
    const uint32_t tq[3] = {a.qx[p], a.qy[p], a.qz[p]};
    bool wide = false;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      int32_t r = rel32(tq[d], t0[d], a.periodic);
      int32_t mn = __reduce_min_sync(0xffffffffu, has ? r : 0x7FFFFFFF);
      int32_t mx = __reduce_max_sync(0xffffffffu, has ? r : -0x7FFFFFFF);
      wide = wide || ((int64_t)mx - (int64_t)mn > WIDE_GROUP);
    }
    wide = wide || a.single_target;
    // one call site: the group at once, or its targets one at a time
    const uint32_t walks = wide ? count : 1u;
    for (uint32_t t = 0; t < walks; ++t)
      walk_targets<TPW, ACC>(a, wide ? first + t : first, wide ? 1u : count, list_l, list_m, owner, stk, rpos, rmask, s0,
                             s1, tfs, gbox);
  }
}

// ---- per-target exact walk below a node whose centre of mass coincides with
// the target (the reference opens such a monopole, short_range.rs:316-330)
__global__ void k_deferred(WalkArgs a, uint32_t n_items) {
  uint32_t it = blockIdx.x * blockDim.x + threadIdx.x;
  if (it >= n_items || it >= a.cap_deferred) return;
  const uint2 job = a.deferred[it];
  const uint32_t p = job.x;
  double xi[3];
  target_pos(a, p, xi);
  const uint32_t tq[3] = {a.qx[p], a.qy[p], a.qz[p]};
  uint32_t stack[8 * 48];
  int sp = 0;
  float fx = 0.f, fy = 0.f, fz = 0.f;
  // open `job.y`: push its children
  {
    const uint32_t nd = job.y;
    const uint32_t f = a.child_first[nd], c = a.nchild[nd];
    for (uint32_t k = 0; k < c; ++k) stack[sp++] = a.child_ids[f + k];
  }
  int64_t guard = 0;
  while (sp > 0) {
    if (++guard > a.n_int + a.n + 2) {
      atomicOr(a.err, DEV_ERR_STACK);
      break;
    }
    const uint32_t node = stack[--sp];
    double c[3];
    node_com(a, node, c);
    float m;
    uint32_t cq[3];
    if (node & LEAF_BIT) {
      const uint32_t j = node & ~LEAF_BIT;
      m = a.massf[j];
      cq[0] = a.qx[j]; cq[1] = a.qy[j]; cq[2] = a.qz[j];
    } else {
      const uint4 w = a.walk[node];
      m = __uint_as_float(w.w);
      cq[0] = w.x; cq[1] = w.y; cq[2] = w.z;
    }
    const int dep = (node & LEAF_BIT) ? a.leaf_depth[node & ~LEAF_BIT] : a.depth[node];
    const double h = ldexp(a.h0, -dep);
    if (d2_aabb(xi, c, h, a.box, a.periodic) > a.rc2) continue;
    bool interact = false;
    if (node & LEAF_BIT) {
      if ((node & ~LEAF_BIT) == p) continue;
      interact = exact_terminal(a, p, node) == 1;
    } else if (h < a.thr) {
      const int d = exact_terminal(a, p, node);
      if (d == 1) interact = true;
      else if (d == 2) {
        const uint32_t f = a.child_first[node], cc = a.nchild[node];
        if (sp + (int)cc > 8 * 48) { atomicOr(a.err, DEV_ERR_STACK); break; }
        for (uint32_t k = 0; k < cc; ++k) stack[sp++] = a.child_ids[f + k];
      }
    } else {
      const uint32_t f = a.child_first[node], cc = a.nchild[node];
      if (sp + (int)cc > 8 * 48) { atomicOr(a.err, DEV_ERR_STACK); break; }
      for (uint32_t k = 0; k < cc; ++k) stack[sp++] = a.child_ids[f + k];
    }
    if (interact) {
      atomicAdd(&a.pcounts[2 * (int64_t)p + ((node & LEAF_BIT) ? 0 : 1)], 1u);
      const float dx = (float)rel32(cq[0], tq[0], a.periodic) * a.u_inv;
      const float dy = (float)rel32(cq[1], tq[1], a.periodic) * a.u_inv;
      const float dz = (float)rel32(cq[2], tq[2], a.periodic) * a.u_inv;
      const float f = pair_factor(a, fmaf(dx, dx, fmaf(dy, dy, dz * dz)), m);
      fx = fmaf(dx, f, fx);
      fy = fmaf(dy, f, fy);
      fz = fmaf(dz, f, fz);
    }
  }
  atomicAdd(&a.ax[p], fx * a.out_scale);
  atomicAdd(&a.ay[p], fy * a.out_scale);
  atomicAdd(&a.az[p], fz * a.out_scale);
  atomicAdd(&a.stats[4], 1ull);
}

}  // namespace

// Variants of the walk: the register budget for 5 to 8 resident blocks of 4
// warps per SM (TPM_WALK_BLOCKS; 7 = 72 registers by default: walk 64.7 ms at
// 7 blocks, 64.8 at 8 on the 256^3 workload) and 32 or 16 targets per warp
// (TPM_WALK_TARGETS; with 16, two lanes share each target).
static int env_choice(const char* name, int dflt, int lo, int hi) {
  const char* e = getenv(name);
  const int v = e ? atoi(e) : dflt;
  return (v >= lo && v <= hi) ? v : dflt;
}
static int walk_blocks_variant() {
  static int v = env_choice("TPM_WALK_BLOCKS", 7, 5, 8);
  return v;
}
int walk_targets_per_warp() {
  static int v = env_choice("TPM_WALK_TARGETS", 32, 16, 32) == 16 ? 16 : 32;
  return v;
}

template <int B, int T, bool ACC>
static int blocks_for() {
  const size_t smem = walk_smem_per_warp<ACC>() * WALK_WARPS;
  TPM_CUDA(cudaFuncSetAttribute(k_walk<B, T, ACC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  int nb = 0;
  TPM_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_walk<B, T, ACC>, WALK_THREADS, smem));
  return nb < 1 ? 1 : nb;
}

// the accurate mode: 5, 6 or 7 (default; 71 registers, no spills: accurate walk 88.6 ms
// at 6, 85.5 at 7 on the 256^3 workload) blocks per SM (TPM_WALK_BLOCKS_ACC)
static int walk_blocks_acc_variant() {
  static int v = env_choice("TPM_WALK_BLOCKS_ACC", 7, 5, 7);
  return v;
}
template <int T>
static int blocks_t(bool accurate) {
  if (accurate) {
    switch (walk_blocks_acc_variant()) {
      case 5: return blocks_for<5, T, true>();
      case 6: return blocks_for<6, T, true>();
      default: return blocks_for<7, T, true>();
    }
  }
  switch (walk_blocks_variant()) {
    case 5: return blocks_for<5, T, false>();
    case 7: return blocks_for<7, T, false>();
    case 6: return blocks_for<6, T, false>();
    case 8: return blocks_for<8, T, false>();
    default: return blocks_for<7, T, false>();
  }
}

int walk_blocks_per_sm(bool accurate) {
  return walk_targets_per_warp() == 16 ? blocks_t<16>(accurate) : blocks_t<32>(accurate);
}

template <int T>
static void launch_t(const WalkArgs& a, int grid, cudaStream_t s) {
  if (a.accurate) {
    const size_t smem = walk_smem_per_warp<true>() * WALK_WARPS;
    switch (walk_blocks_acc_variant()) {
      case 5: k_walk<5, T, true><<<grid, WALK_THREADS, smem, s>>>(a); break;
      case 6: k_walk<6, T, true><<<grid, WALK_THREADS, smem, s>>>(a); break;
      default: k_walk<7, T, true><<<grid, WALK_THREADS, smem, s>>>(a); break;
    }
    return;
  }
  const size_t smem = walk_smem_per_warp<false>() * WALK_WARPS;
  switch (walk_blocks_variant()) {
    case 5: k_walk<5, T, false><<<grid, WALK_THREADS, smem, s>>>(a); break;
    case 7: k_walk<7, T, false><<<grid, WALK_THREADS, smem, s>>>(a); break;
    case 6: k_walk<6, T, false><<<grid, WALK_THREADS, smem, s>>>(a); break;
    case 8: k_walk<8, T, false><<<grid, WALK_THREADS, smem, s>>>(a); break;
    default: k_walk<7, T, false><<<grid, WALK_THREADS, smem, s>>>(a); break;
  }
}

int walk_threads() { return WALK_THREADS; }
size_t walk_stack_words(int grid, int stack_cap) {
  (void)stack_cap;
  return (size_t)grid * WALK_WARPS * STACK_ENTRIES * 4;  // one 16-byte entry = 4 words
}

void launch_walk(const WalkArgs& a, int grid, cudaStream_t s) {
  if (walk_targets_per_warp() == 16) launch_t<16>(a, grid, s);
  else launch_t<32>(a, grid, s);
  TPM_LAUNCH_CHECK();
}

void launch_deferred(const WalkArgs& a, uint32_t n_items, cudaStream_t s) {
  if (n_items == 0) return;
  k_deferred<<<grid_for(n_items, 64, 1ll << 20), 64, 0, s>>>(a, n_items);
  TPM_LAUNCH_CHECK();
}

}  // namespace tpm
