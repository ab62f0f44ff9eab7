// TEST INFRASTRUCTURE ONLY — the oracle for the TreePM force path.
//
// A CPU restatement (C++17, FP64, OpenMP where the reference uses rayon) of
// gadget-ng's TreePM gravity path.  The reference is a Rust workspace that
// cannot be compiled in this environment (no cargo/rustc), so this file
// restates its algorithm statement by statement, in the same floating-point
// operation order, citing the file:line of each function it follows.  Paths
// are relative to the gadget-ng project root.
//
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
// this library, and only as the checker.  The product (the sm_100a library in
// gadget-ng_b200/) never links or calls it.
//
// Parity pinning: the reference ships no golden force vectors for TreePM.
// This restatement is pinned against every known-answer test and invariant
// the reference's own tests hold for this path (ported as assertions in
// tests/test_oracle_pins.py).  Force-level parity is therefore "pinned by
// known-answer tests", not by reference outputs.
//
// rustfft 6.4.1 (Cargo.lock) is the one third-party numeric dependency on the
// path; it computes an exact unnormalised DFT (forward e^{-2πi jk/n}, inverse
// e^{+2πi jk/n}).  It is restated here as an iterative radix-2 FFT, applied
// in the reference's pass order.

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

struct V3 {
  double x, y, z;
};
inline V3 v3(double x, double y, double z) { return V3{x, y, z}; }
inline V3 add(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline V3 sub(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline V3 mul(V3 a, double s) { return v3(a.x * s, a.y * s, a.z * s); }
inline V3 divs(V3 a, double s) { return v3(a.x / s, a.y / s, a.z / s); }

// Rust f64::rem_euclid (core::f64): r = a % b; r < 0 ? r + |b| : r.
inline double rem_euclid(double a, double b) {
  double r = std::fmod(a, b);
  return r < 0.0 ? r + std::fabs(b) : r;
}
// Rust f64::round: half away from zero == C round().
inline double rround(double a) { return std::round(a); }

inline V3 load(const double* p, int64_t i) { return v3(p[3 * i], p[3 * i + 1], p[3 * i + 2]); }

// ---------------------------------------------------------------------------
// CIC — crates/gadget-ng-pm/src/cic.rs:37-93 (assign_batch_scalar),
//        :100-170 (interpolate_batch_scalar), :260-292 (assign), :298-346.
// ---------------------------------------------------------------------------
void cic_assign(const double* pos, const double* mass, int64_t n, double box, int nm, double* out) {
  const double inv_cell = (double)nm / box;  // cic.rs:262
  const int64_t nm2 = (int64_t)nm * nm;
  const double nmf = (double)nm;
  for (int64_t i = 0; i < n; ++i) {
    double cx = rem_euclid(pos[3 * i] * inv_cell, nmf);
    double cy = rem_euclid(pos[3 * i + 1] * inv_cell, nmf);
    double cz = rem_euclid(pos[3 * i + 2] * inv_cell, nmf);
    int64_t ix0 = (int64_t)std::floor(cx), iy0 = (int64_t)std::floor(cy), iz0 = (int64_t)std::floor(cz);
    double dx = cx - (double)ix0, dy = cy - (double)iy0, dz = cz - (double)iz0;
    double wxs[2] = {1.0 - dx, dx}, wys[2] = {1.0 - dy, dy}, wzs[2] = {1.0 - dz, dz};
    int64_t ixs[2] = {ix0, (ix0 + 1) % nm}, iys[2] = {iy0, (iy0 + 1) % nm}, izs[2] = {iz0, (iz0 + 1) % nm};
    double m = mass[i];
    for (int a = 0; a < 2; ++a)
      for (int b = 0; b < 2; ++b)
        for (int c = 0; c < 2; ++c)
          out[izs[a] * nm2 + iys[b] * nm + ixs[c]] += m * wxs[c] * wys[b] * wzs[a];
  }
}

void cic_interpolate(const double* fx, const double* fy, const double* fz, const double* pos, int64_t n,
                     double box, int nm, double* acc) {
  const double inv_cell = (double)nm / box;
  const int64_t nm2 = (int64_t)nm * nm;
  const double nmf = (double)nm;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    double cx = rem_euclid(pos[3 * i] * inv_cell, nmf);
    double cy = rem_euclid(pos[3 * i + 1] * inv_cell, nmf);
    double cz = rem_euclid(pos[3 * i + 2] * inv_cell, nmf);
    int64_t ix0 = (int64_t)std::floor(cx), iy0 = (int64_t)std::floor(cy), iz0 = (int64_t)std::floor(cz);
    double dx = cx - (double)ix0, dy = cy - (double)iy0, dz = cz - (double)iz0;
    double wxs[2] = {1.0 - dx, dx}, wys[2] = {1.0 - dy, dy}, wzs[2] = {1.0 - dz, dz};
    int64_t ixs[2] = {ix0, (ix0 + 1) % nm}, iys[2] = {iy0, (iy0 + 1) % nm}, izs[2] = {iz0, (iz0 + 1) % nm};
    double ax = 0.0, ay = 0.0, az = 0.0;
    for (int a = 0; a < 2; ++a)
      for (int b = 0; b < 2; ++b)
        for (int c = 0; c < 2; ++c) {
          double w = wxs[c] * wys[b] * wzs[a];
          int64_t idx = izs[a] * nm2 + iys[b] * nm + ixs[c];
          ax += fx[idx] * w;
          ay += fy[idx] * w;
          az += fz[idx] * w;
        }
    acc[3 * i] = ax;
    acc[3 * i + 1] = ay;
    acc[3 * i + 2] = az;
  }
}

// ---------------------------------------------------------------------------
// FFT — restatement of rustfft's unnormalised c2c DFT (exact mathematics),
// applied with the pass order of crates/gadget-ng-pm/src/fft_poisson.rs:733-813.
// ---------------------------------------------------------------------------
typedef std::complex<double> cplx;

struct Fft1d {
  int n = 0;
  std::vector<cplx> tw;  // e^{-2πi k/n}
  std::vector<int> rev;
  explicit Fft1d(int n_) : n(n_), tw(n_ / 2 > 0 ? n_ / 2 : 1), rev(n_) {
    for (int k = 0; k < n / 2; ++k) {
      double ang = -2.0 * M_PI * (double)k / (double)n;
      tw[k] = cplx(std::cos(ang), std::sin(ang));
    }
    int lg = 0;
    while ((1 << lg) < n) ++lg;
    for (int i = 0; i < n; ++i) {
      int r = 0;
      for (int b = 0; b < lg; ++b)
        if (i & (1 << b)) r |= 1 << (lg - 1 - b);
      rev[i] = r;
    }
  }
  // inverse: conjugate twiddles (e^{+2πi jk/n}), unnormalised, like rustfft.
  void run(cplx* a, bool inverse) const {
    for (int i = 0; i < n; ++i)
      if (i < rev[i]) std::swap(a[i], a[rev[i]]);
    for (int len = 2; len <= n; len <<= 1) {
      int half = len / 2, step = n / len;
      for (int s = 0; s < n; s += len)
        for (int k = 0; k < half; ++k) {
          cplx w = tw[k * step];
          if (inverse) w = std::conj(w);
          cplx u = a[s + k], v = a[s + k + half] * w;
          a[s + k] = u + v;
          a[s + k + half] = u - v;
        }
    }
  }
};

// fft_poisson.rs:733-771 (x rows, then y columns, then z stacks).
void fft3d(cplx* d, int nm, const Fft1d& f, bool inverse) {
  const int64_t nm2 = (int64_t)nm * nm;
  auto pass_x = [&]() {
#pragma omp parallel for schedule(static)
    for (int64_t r = 0; r < nm2; ++r) f.run(d + r * nm, inverse);
  };
  auto pass_y = [&]() {
#pragma omp parallel
    {
      std::vector<cplx> tmp(nm);
#pragma omp for schedule(static)
      for (int64_t c = 0; c < nm2; ++c) {
        int64_t iz = c / nm, ix = c % nm;
        for (int iy = 0; iy < nm; ++iy) tmp[iy] = d[iz * nm2 + iy * nm + ix];
        f.run(tmp.data(), inverse);
        for (int iy = 0; iy < nm; ++iy) d[iz * nm2 + iy * nm + ix] = tmp[iy];
      }
    }
  };
  auto pass_z = [&]() {
#pragma omp parallel
    {
      std::vector<cplx> tmp(nm);
#pragma omp for schedule(static)
      for (int64_t c = 0; c < nm2; ++c) {
        int64_t iy = c / nm, ix = c % nm;
        for (int iz = 0; iz < nm; ++iz) tmp[iz] = d[iz * nm2 + iy * nm + ix];
        f.run(tmp.data(), inverse);
        for (int iz = 0; iz < nm; ++iz) d[iz * nm2 + iy * nm + ix] = tmp[iz];
      }
    }
  };
  if (!inverse) {
    pass_x();
    pass_y();
    pass_z();
  } else {  // fft_poisson.rs:775-813: z, y, x
    pass_z();
    pass_y();
    pass_x();
  }
}

// fft_poisson.rs:724-730
inline int64_t freq_index(int64_t j, int64_t nm) { return j <= nm / 2 ? j : j - nm; }

// Extension flags (off in parity mode; the reference has neither).
enum { ORC_DECONVOLVE_CIC = 1, ORC_FOUR_POINT_GRADIENT = 2 };

// fft_poisson.rs:306-476 (solve_forces_impl) with the spectral kernel of
// :488-550.  r_split <= 0 means None; plummer_eps <= 0 means None.
void solve_forces(const double* density, double g, int nm, double box, double r_split, double plummer_eps,
                  int flags, double* fx, double* fy, double* fz) {
  const int64_t nm2 = (int64_t)nm * nm, nm3 = nm2 * nm;
  const double cl = box / (double)nm;
  const double cell_vol = cl * (cl * cl);  // f64::powi(3) == x * (x * x)
  const double rho_scale = 1.0 / cell_vol;
  Fft1d f(nm);
  std::vector<cplx> rho(nm3);
  for (int64_t i = 0; i < nm3; ++i) rho[i] = cplx(density[i] * rho_scale, 0.0);
  fft3d(rho.data(), nm, f, false);
  const double dk = 2.0 * M_PI / box;
  const double four_pi_g = 4.0 * M_PI * g;
  const double dx_cell = box / (double)nm;
  std::vector<double> karr(nm), deriv(nm), wcic(nm);
  for (int i = 0; i < nm; ++i) {
    karr[i] = dk * (double)freq_index(i, nm);
    // extension: 4-point finite-difference gradient in Fourier space
    double kd = karr[i] * dx_cell;
    deriv[i] = (flags & ORC_FOUR_POINT_GRADIENT) ? (8.0 * std::sin(kd) - std::sin(2.0 * kd)) / (6.0 * dx_cell)
                                                 : karr[i];
    double h = 0.5 * kd;
    double s = (i == 0) ? 1.0 : std::sin(h) / h;
    wcic[i] = s * s;
  }
  const bool has_rs = r_split > 0.0;
  const double r_split2 = r_split * r_split;
  const bool has_eps = plummer_eps > 0.0;
  const double eps2 = plummer_eps * plummer_eps;
  std::vector<cplx> cx(nm3), cy(nm3), cz(nm3);
#pragma omp parallel for schedule(static)
  for (int64_t flat = 0; flat < nm3; ++flat) {
    int64_t iz = flat / nm2, iy = (flat / nm) % nm, ix = flat % nm;
    double kx = karr[ix], ky = karr[iy], kz = karr[iz];
    double k2 = kx * kx + ky * ky + kz * kz;
    if (k2 < 1e-30) {
      cx[flat] = cy[flat] = cz[flat] = cplx(0.0, 0.0);
      continue;
    }
    double filter = 1.0;
    if (has_rs) filter *= std::exp(-0.5 * k2 * r_split2);
    if (has_eps && eps2 > 0.0) filter *= std::exp(-k2 * eps2);
    if (flags & ORC_DECONVOLVE_CIC) {
      double w = wcic[ix] * wcic[iy] * wcic[iz];
      filter /= (w * w);
    }
    double phi_re = rho[flat].real() * (-four_pi_g * filter / k2);
    double phi_im = rho[flat].imag() * (-four_pi_g * filter / k2);
    double gx = deriv[ix], gy = deriv[iy], gz = deriv[iz];
    cx[flat] = cplx(gx * phi_im, -gx * phi_re);
    cy[flat] = cplx(gy * phi_im, -gy * phi_re);
    cz[flat] = cplx(gz * phi_im, -gz * phi_re);
  }
  const double norm = 1.0 / (double)nm3;
  fft3d(cx.data(), nm, f, true);
  fft3d(cy.data(), nm, f, true);
  fft3d(cz.data(), nm, f, true);
  for (int64_t i = 0; i < nm3; ++i) {
    fx[i] = cx[i].real() * norm;
    fy[i] = cy[i].real() * norm;
    fz[i] = cz[i].real() * norm;
  }
}

// ---------------------------------------------------------------------------
// Octree — crates/gadget-ng-tree/src/octree.rs:153-175 (OctNode), :197-207
// (outer_traceless), :423-435 (octant_of), :447-465 (child_center), :474-540
// (build / insert), :547-629 (aggregate), :1306-1332 (bounding_cube).
// Octupole / hexadecapole moments are not on the TreePM short-range path and
// are not restated.
// ---------------------------------------------------------------------------
const uint32_t NO_CHILD = 0xFFFFFFFFu;

struct Node {
  V3 center;
  double half_size;
  double mass;
  V3 com;
  uint32_t children[8];
  int64_t particle_idx;  // -1 == None
  double quad[6];
  int32_t depth;
};

struct Octree {
  std::vector<Node> nodes;
  uint32_t root = 0;
};

Node empty_leaf(V3 c, double h, int depth) {
  Node n;
  n.center = c;
  n.half_size = h;
  n.mass = 0.0;
  n.com = v3(0, 0, 0);
  for (int i = 0; i < 8; ++i) n.children[i] = NO_CHILD;
  n.particle_idx = -1;
  for (int i = 0; i < 6; ++i) n.quad[i] = 0.0;
  n.depth = depth;
  return n;
}

inline int octant_of(V3 p, V3 c) {
  int o = 0;
  if (p.x >= c.x) o |= 1;
  if (p.y >= c.y) o |= 2;
  if (p.z >= c.z) o |= 4;
  return o;
}

inline V3 child_center(V3 pc, double ph, int oct) {
  double q = ph * 0.5;
  V3 off = v3(0.0, 0.0, 0.0);
  if (oct & 1) off.x += q; else off.x -= q;
  if (oct & 2) off.y += q; else off.y -= q;
  if (oct & 4) off.z += q; else off.z -= q;
  return add(pc, off);
}

void bounding_cube(const double* pos, int64_t n, V3* center, double* half) {
  double min_x = pos[0], max_x = pos[0], min_y = pos[1], max_y = pos[1], min_z = pos[2], max_z = pos[2];
  for (int64_t i = 1; i < n; ++i) {
    min_x = std::min(min_x, pos[3 * i]);
    max_x = std::max(max_x, pos[3 * i]);
    min_y = std::min(min_y, pos[3 * i + 1]);
    max_y = std::max(max_y, pos[3 * i + 1]);
    min_z = std::min(min_z, pos[3 * i + 2]);
    max_z = std::max(max_z, pos[3 * i + 2]);
  }
  *center = v3(0.5 * (min_x + max_x), 0.5 * (min_y + max_y), 0.5 * (min_z + max_z));
  double hx = (max_x - min_x) * 0.5, hy = (max_y - min_y) * 0.5, hz = (max_z - min_z) * 0.5;
  double h = std::max(std::max(hx, hy), hz);
  double pad = std::max(h * 1e-6, 1e-12);
  *half = h + pad;
}

bool is_leaf(const Node& n) {
  for (int i = 0; i < 8; ++i)
    if (n.children[i] != NO_CHILD) return false;
  return true;
}

// octree.rs:501-540, restated iteratively (identical node creation order).
// Returns false when the depth exceeds max_depth (coincident positions make
// the reference recurse without bound).
bool insert(Octree& t, uint32_t node_idx, int64_t pidx, V3 pos, const double* positions, int max_depth) {
  for (;;) {
    Node& nd = t.nodes[node_idx];
    bool all_empty = is_leaf(nd);
    if (all_empty && nd.particle_idx < 0) {
      nd.particle_idx = pidx;
      return true;
    }
    if (all_empty) {
      if (nd.depth >= max_depth) return false;
      int64_t old = nd.particle_idx;
      nd.particle_idx = -1;
      V3 old_pos = load(positions, old);
      V3 center = nd.center;
      double half = nd.half_size;
      double ch_half = half * 0.5;
      int depth = nd.depth;
      uint32_t kids[8];
      for (int oct = 0; oct < 8; ++oct) {
        V3 cc = child_center(center, half, oct);
        kids[oct] = (uint32_t)t.nodes.size();
        t.nodes.push_back(empty_leaf(cc, ch_half, depth + 1));
      }
      Node& nd2 = t.nodes[node_idx];  // vector may have reallocated
      for (int oct = 0; oct < 8; ++oct) nd2.children[oct] = kids[oct];
      int oct_old = octant_of(old_pos, center);
      int oct_new = octant_of(pos, center);
      if (!insert(t, kids[oct_old], old, old_pos, positions, max_depth)) return false;
      node_idx = kids[oct_new];
      continue;
    }
    int oct = octant_of(pos, nd.center);
    node_idx = nd.children[oct];
  }
}

inline void outer_traceless(V3 s, double m, double* q) {
  double s2 = s.x * s.x + s.y * s.y + s.z * s.z;  // Vec3::dot
  q[0] = m * (3.0 * s.x * s.x - s2);
  q[1] = m * 3.0 * s.x * s.y;
  q[2] = m * 3.0 * s.x * s.z;
  q[3] = m * (3.0 * s.y * s.y - s2);
  q[4] = m * 3.0 * s.y * s.z;
  q[5] = m * (3.0 * s.z * s.z - s2);
}

// octree.rs:547-629 (mass, COM, quadrupole; post-order, children 0..7).
void aggregate(Octree& t, uint32_t root, const double* positions, const double* masses) {
  // explicit post-order to avoid deep recursion costs
  struct Frame { uint32_t idx; int stage; };
  std::vector<Frame> st;
  st.push_back({root, 0});
  while (!st.empty()) {
    Frame& fr = st.back();
    Node& nd = t.nodes[fr.idx];
    if (is_leaf(nd)) {
      if (nd.particle_idx >= 0) {
        nd.mass = masses[nd.particle_idx];
        nd.com = load(positions, nd.particle_idx);
      } else {
        nd.mass = 0.0;
        nd.com = v3(0, 0, 0);
      }
      for (int i = 0; i < 6; ++i) nd.quad[i] = 0.0;
      st.pop_back();
      continue;
    }
    if (fr.stage == 0) {
      fr.stage = 1;
      uint32_t idx = fr.idx;
      for (int c = 7; c >= 0; --c) {
        uint32_t ch = t.nodes[idx].children[c];
        if (ch != NO_CHILD) st.push_back({ch, 0});
      }
      continue;
    }
    // all children done
    uint32_t idx = fr.idx;
    st.pop_back();
    Node& n = t.nodes[idx];
    double mtot = 0.0;
    V3 com_acc = v3(0.0, 0.0, 0.0);
    for (int c = 0; c < 8; ++c) {
      uint32_t ch = n.children[c];
      if (ch == NO_CHILD) continue;
      const Node& cn = t.nodes[ch];
      mtot += cn.mass;
      com_acc = add(com_acc, mul(cn.com, cn.mass));
    }
    V3 com = mtot > 0.0 ? divs(com_acc, mtot) : v3(0.0, 0.0, 0.0);
    n.mass = mtot;
    n.com = com;
    double quad[6] = {0, 0, 0, 0, 0, 0};
    for (int c = 0; c < 8; ++c) {
      uint32_t ch = n.children[c];
      if (ch == NO_CHILD) continue;
      const Node& cn = t.nodes[ch];
      if (cn.mass == 0.0) continue;
      V3 s = sub(cn.com, com);
      double oq[6];
      outer_traceless(s, cn.mass, oq);
      for (int i = 0; i < 6; ++i) quad[i] += cn.quad[i] + oq[i];
    }
    for (int i = 0; i < 6; ++i) n.quad[i] = quad[i];
  }
}

// Returns 0 on success, 1 on depth overflow (coincident positions).
int build_octree(const double* pos, const double* mass, int64_t n, Octree& t, int max_depth = 200) {
  t.nodes.clear();
  if (n == 0) {
    t.nodes.push_back(empty_leaf(v3(0, 0, 0), 1.0, 0));
    t.root = 0;
    return 0;
  }
  V3 center;
  double half;
  bounding_cube(pos, n, &center, &half);
  t.nodes.reserve((size_t)(4.2 * (double)n) + 16);
  t.nodes.push_back(empty_leaf(center, half, 0));
  t.root = 0;
  for (int64_t j = 0; j < n; ++j)
    if (!insert(t, t.root, j, load(pos, j), pos, max_depth)) return 1;
  aggregate(t, t.root, pos, mass);
  return 0;
}

// ---------------------------------------------------------------------------
// Short range — crates/gadget-ng-treepm/src/short_range.rs
// ---------------------------------------------------------------------------
// :53-63
inline double minimum_image(double dx, double box) {
  double half = box * 0.5;
  double d = dx - box * rround(dx / box);
  if (d > half) d -= box;
  else if (d < -half) d += box;
  return d;
}
// :72-84
inline double min_dist2_to_aabb_periodic(V3 xi, V3 com, double h, double box) {
  double dxc = minimum_image(com.x - xi.x, box);
  double dyc = minimum_image(com.y - xi.y, box);
  double dzc = minimum_image(com.z - xi.z, box);
  double ex = std::max(std::fabs(dxc) - h, 0.0);
  double ey = std::max(std::fabs(dyc) - h, 0.0);
  double ez = std::max(std::fabs(dzc) - h, 0.0);
  return ex * ex + ey * ey + ez * ez;
}
// :91-101 (A&S 7.1.26)
double erfc_approx(double x) {
  if (x < 0.0) return 2.0 - erfc_approx(-x);
  double t = 1.0 / (1.0 + 0.3275911 * x);
  double poly = t * (0.254829592 + t * (-0.284496736 + t * (1.421413741 + t * (-1.453152027 + t * 1.061405429))));
  return poly * std::exp(-x * x);
}
// :108-111
inline double erfc_factor(double r, double r_split) {
  double x = r / (M_SQRT2 * r_split);
  return erfc_approx(x);
}
// :384-398
inline V3 pair_accel(double rx, double ry, double rz, double mass, double eps2, double g, double r_split) {
  double r2 = rx * rx + ry * ry + rz * rz + eps2;
  double r = std::sqrt(r2);
  double w = erfc_factor(r, r_split);
  double inv3 = g * mass * w / (r2 * r);
  return v3(rx * inv3, ry * inv3, rz * inv3);
}

struct SrParams {
  const double* pos;
  const double* mass;
  double eps2, g, r_split, r_cut2, box;
};

// :274-333 (walk_short_range_periodic).  counts = {leaf pairs, monopoles}.
V3 walk_periodic(const Octree& t, V3 xi, int64_t skip, const SrParams& p, int64_t* counts,
                 std::vector<uint32_t>& stack) {
  V3 a = v3(0, 0, 0);
  stack.clear();
  stack.push_back(t.root);
  const double box = p.box;
  const double rc = std::sqrt(p.r_cut2);
  while (!stack.empty()) {
    uint32_t ni = stack.back();
    stack.pop_back();
    const Node& node = t.nodes[ni];
    if (node.mass == 0.0) continue;
    double d2a = min_dist2_to_aabb_periodic(xi, node.com, node.half_size, box);
    if (d2a > p.r_cut2) continue;
    if (is_leaf(node)) {
      if (node.particle_idx >= 0 && node.particle_idx != skip) {
        V3 rj = load(p.pos, node.particle_idx);
        double rx = minimum_image(rj.x - xi.x, box);
        double ry = minimum_image(rj.y - xi.y, box);
        double rz = minimum_image(rj.z - xi.z, box);
        double r2_bare = rx * rx + ry * ry + rz * rz;
        if (r2_bare > p.r_cut2) continue;
        a = add(a, pair_accel(rx, ry, rz, p.mass[node.particle_idx], p.eps2, p.g, p.r_split));
        if (counts) counts[0]++;
      }
    } else {
      double dx = minimum_image(node.com.x - xi.x, box);
      double dy = minimum_image(node.com.y - xi.y, box);
      double dz = minimum_image(node.com.z - xi.z, box);
      double d2 = dx * dx + dy * dy + dz * dz;
      bool use_mono = node.half_size < 0.1 * rc && d2 > 1e-30;
      if (use_mono) {
        a = add(a, pair_accel(dx, dy, dz, node.mass, p.eps2, p.g, p.r_split));
        if (counts) counts[1]++;
      } else {
        for (int c = 0; c < 8; ++c)
          if (node.children[c] != NO_CHILD) stack.push_back(node.children[c]);
      }
    }
  }
  return a;
}

// :157-208 (walk_short_range, aperiodic).
V3 walk_aperiodic(const Octree& t, V3 xi, int64_t skip, const SrParams& p, int64_t* counts,
                  std::vector<uint32_t>& stack) {
  V3 a = v3(0, 0, 0);
  stack.clear();
  stack.push_back(t.root);
  const double rc = std::sqrt(p.r_cut2);
  while (!stack.empty()) {
    uint32_t ni = stack.back();
    stack.pop_back();
    const Node& node = t.nodes[ni];
    if (node.mass == 0.0) continue;
    double dx = node.com.x - xi.x, dy = node.com.y - xi.y, dz = node.com.z - xi.z;
    double h = node.half_size;
    double ex = std::max(std::fabs(dx) - h, 0.0);
    double ey = std::max(std::fabs(dy) - h, 0.0);
    double ez = std::max(std::fabs(dz) - h, 0.0);
    if (ex * ex + ey * ey + ez * ez > p.r_cut2) continue;
    if (is_leaf(node)) {
      if (node.particle_idx >= 0 && node.particle_idx != skip) {
        V3 rj = load(p.pos, node.particle_idx);
        a = add(a, pair_accel(rj.x - xi.x, rj.y - xi.y, rj.z - xi.z, p.mass[node.particle_idx], p.eps2, p.g,
                              p.r_split));
        if (counts) counts[0]++;
      }
    } else {
      double d2 = dx * dx + dy * dy + dz * dz;
      bool use_mono = h < 0.1 * rc && d2 > 1e-30;
      if (use_mono) {
        a = add(a, pair_accel(dx, dy, dz, node.mass, p.eps2, p.g, p.r_split));
        if (counts) counts[1]++;
      } else {
        for (int c = 0; c < 8; ++c)
          if (node.children[c] != NO_CHILD) stack.push_back(node.children[c]);
      }
    }
  }
  return a;
}

void short_range(const Octree& t, const SrParams& p, bool periodic, const int64_t* targets, int64_t nt,
                 double* out, int64_t* counts) {
#pragma omp parallel
  {
    std::vector<uint32_t> stack;
    stack.reserve(512);
#pragma omp for schedule(dynamic, 64)
    for (int64_t k = 0; k < nt; ++k) {
      int64_t gi = targets[k];
      V3 xi = load(p.pos, gi);
      int64_t c[2] = {0, 0};
      V3 a = periodic ? walk_periodic(t, xi, gi, p, c, stack) : walk_aperiodic(t, xi, gi, p, c, stack);
      out[3 * k] = a.x;
      out[3 * k + 1] = a.y;
      out[3 * k + 2] = a.z;
      if (counts) {
        counts[2 * k] = c[0];
        counts[2 * k + 1] = c[1];
      }
    }
  }
}

// ---------------------------------------------------------------------------
// SFC keys — crates/gadget-ng-parallel/src/sfc.rs:39-60 (Morton), :95-183
// (hilbert3 / coords_to_hilbert, Skilling 2004 AxesToTranspose), :187-204.
// ---------------------------------------------------------------------------
const double F64_EPS = 2.220446049250313e-16;

uint64_t coords_to_hilbert(uint32_t ix, uint32_t iy, uint32_t iz, uint32_t p) {
  uint32_t x[3] = {ix, iy, iz};
  const int n = 3;
  uint32_t m = 1u << (p - 1);
  for (uint32_t q = m; q > 1; q >>= 1) {
    uint32_t p_mask = q - 1;
    for (int i = n - 1; i >= 0; --i) {
      if (x[i] & q) {
        x[0] ^= p_mask;
      } else {
        uint32_t tt = (x[0] ^ x[i]) & p_mask;
        x[0] ^= tt;
        x[i] ^= tt;
      }
    }
  }
  for (int i = 1; i < n; ++i) x[i] ^= x[i - 1];
  {
    uint32_t t = 0;
    for (uint32_t q = m; q > 1; q >>= 1)
      if (x[n - 1] & q) t ^= q - 1;
    for (int i = 0; i < n; ++i) x[i] ^= t;
  }
  uint64_t h = 0;
  // sfc.rs:174-181 packs k = 0..p-1 (bit k of each word), j = 0..n-1
  for (uint32_t k = 0; k < p; ++k)
    for (int j = 0; j < n; ++j) h = (h << 1) | (uint64_t)((x[j] >> k) & 1u);
  return h;
}

inline double clamp01(double v) { return std::min(std::max(v, 0.0), 1.0 - F64_EPS); }

uint64_t hilbert3(double x, double y, double z) {
  const double SCALE = (double)(1ull << 21);
  uint32_t ix = (uint32_t)(clamp01(x) * SCALE);
  uint32_t iy = (uint32_t)(clamp01(y) * SCALE);
  uint32_t iz = (uint32_t)(clamp01(z) * SCALE);
  return coords_to_hilbert(ix, iy, iz, 21);
}

inline uint64_t spread_bits(uint64_t x) {
  x &= 0x001fffffull;
  x = (x | (x << 32)) & 0x1f00000000ffffull;
  x = (x | (x << 16)) & 0x1f0000ff0000ffull;
  x = (x | (x << 8)) & 0x100f00f00f00f00full;
  x = (x | (x << 4)) & 0x10c30c30c30c30c3ull;
  x = (x | (x << 2)) & 0x1249249249249249ull;
  return x;
}

uint64_t morton3(double x, double y, double z) {
  const double SCALE = (double)(1ull << 21);
  uint64_t ix = (uint64_t)(clamp01(x) * SCALE);
  uint64_t iy = (uint64_t)(clamp01(y) * SCALE);
  uint64_t iz = (uint64_t)(clamp01(z) * SCALE);
  return spread_bits(ix) | (spread_bits(iy) << 1) | (spread_bits(iz) << 2);
}

// ---------------------------------------------------------------------------
// Cosmology — crates/gadget-ng-core/src/cosmology.rs:150-233 (ΛCDM branch).
// ---------------------------------------------------------------------------
struct Cosmo {
  double omega_m, omega_lambda, h0;
  double da_dt(double a) const {
    double omega_de = omega_lambda;  // w0 = -1, wa = 0
    double h_sq = (omega_m + 0.0) / (a * a * a) + omega_de;
    return a * h0 * std::sqrt(std::max(h_sq, 0.0));
  }
  double advance_a(double a, double dt) const {
    double k1 = da_dt(a);
    double k2 = da_dt(a + 0.5 * dt * k1);
    double k3 = da_dt(a + 0.5 * dt * k2);
    double k4 = da_dt(a + dt * k3);
    return a + dt / 6.0 * (k1 + 2.0 * k2 + 2.0 * k3 + k4);
  }
  void drift_kick(double a0, double dt, double* drift, double* kh, double* kh2) const {
    const uint32_t N_SUB = 16;
    double sub_dt = dt / (double)N_SUB;
    double a = a0;
    double d = 0.0, k1 = 0.0, k2 = 0.0;
    for (uint32_t s = 0; s < N_SUB; ++s) {
      double al = a;
      double am = advance_a(a, sub_dt * 0.5);
      double ar = advance_a(a, sub_dt);
      double d_sub = sub_dt / 6.0 * (1.0 / (al * al) + 4.0 / (am * am) + 1.0 / (ar * ar));
      d += d_sub;
      double k_sub = sub_dt / 6.0 * (1.0 / al + 4.0 / am + 1.0 / ar);
      if (s < N_SUB / 2) k1 += k_sub; else k2 += k_sub;
      a = ar;
    }
    *drift = d;
    *kh = k1;
    *kh2 = k2;
  }
};

}  // namespace

// ===========================================================================
// C ABI (ctypes) — test infrastructure only.
// ===========================================================================
extern "C" {

int orc_num_threads() {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
void orc_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

double orc_erfc_approx(double x) { return erfc_approx(x); }
double orc_minimum_image(double dx, double box) { return minimum_image(dx, box); }
double orc_min_dist2_aabb_periodic(const double* xi, const double* com, double h, double box) {
  return min_dist2_to_aabb_periodic(v3(xi[0], xi[1], xi[2]), v3(com[0], com[1], com[2]), h, box);
}
void orc_pair_accel(const double* r, double mass, double eps2, double g, double r_split, double* out) {
  V3 a = pair_accel(r[0], r[1], r[2], mass, eps2, g, r_split);
  out[0] = a.x;
  out[1] = a.y;
  out[2] = a.z;
}

void orc_cic_assign(const double* pos, const double* mass, int64_t n, double box, int nm, double* rho) {
  std::memset(rho, 0, sizeof(double) * (size_t)nm * nm * nm);
  cic_assign(pos, mass, n, box, nm, rho);
}
void orc_cic_interpolate(const double* fx, const double* fy, const double* fz, const double* pos, int64_t n,
                         double box, int nm, double* acc) {
  cic_interpolate(fx, fy, fz, pos, n, box, nm, acc);
}
void orc_solve_forces(const double* density, double g, int nm, double box, double r_split, double plummer_eps,
                      int flags, double* fx, double* fy, double* fz) {
  solve_forces(density, g, nm, box, r_split, plummer_eps, flags, fx, fy, fz);
}
// Forward 3D FFT then inverse (unnormalised both ways), for the round-trip pin.
void orc_fft3d_roundtrip(const double* in_re, int nm, double* fwd_re, double* fwd_im, double* back_re) {
  int64_t nm3 = (int64_t)nm * nm * nm;
  Fft1d f(nm);
  std::vector<cplx> d(nm3);
  for (int64_t i = 0; i < nm3; ++i) d[i] = cplx(in_re[i], 0.0);
  fft3d(d.data(), nm, f, false);
  for (int64_t i = 0; i < nm3; ++i) {
    fwd_re[i] = d[i].real();
    fwd_im[i] = d[i].imag();
  }
  fft3d(d.data(), nm, f, true);
  for (int64_t i = 0; i < nm3; ++i) back_re[i] = d[i].real();
}

// Octree export.  Returns the number of nodes (including empty leaves) or a
// negative value on error (-1: coincident positions).  Node fields are
// written only when the output pointers are non-null and cap is large enough.
int64_t orc_octree(const double* pos, const double* mass, int64_t n, int64_t cap, double* center_half,
                   double* mass_com, double* quad, int64_t* particle_idx, int32_t* depth, uint32_t* children,
                   double* root_center_half) {
  Octree t;
  if (build_octree(pos, mass, n, t) != 0) return -1;
  int64_t nn = (int64_t)t.nodes.size();
  if (root_center_half) {
    root_center_half[0] = t.nodes[0].center.x;
    root_center_half[1] = t.nodes[0].center.y;
    root_center_half[2] = t.nodes[0].center.z;
    root_center_half[3] = t.nodes[0].half_size;
  }
  if (cap < nn) return nn;
  for (int64_t i = 0; i < nn; ++i) {
    const Node& d = t.nodes[i];
    if (center_half) {
      center_half[4 * i] = d.center.x;
      center_half[4 * i + 1] = d.center.y;
      center_half[4 * i + 2] = d.center.z;
      center_half[4 * i + 3] = d.half_size;
    }
    if (mass_com) {
      mass_com[4 * i] = d.mass;
      mass_com[4 * i + 1] = d.com.x;
      mass_com[4 * i + 2] = d.com.y;
      mass_com[4 * i + 3] = d.com.z;
    }
    if (quad)
      for (int k = 0; k < 6; ++k) quad[6 * i + k] = d.quad[k];
    if (particle_idx) particle_idx[i] = d.particle_idx;
    if (depth) depth[i] = d.depth;
    if (children)
      for (int k = 0; k < 8; ++k) children[8 * i + k] = d.children[k];
  }
  return nn;
}

// Short-range accelerations for a subset of targets (the tree is built over
// all n particles, like short_range_accels / short_range_accels_periodic).
// counts (optional, 2 per target): leaf pairs and monopoles evaluated.
int orc_short_range(const double* pos, const double* mass, int64_t n, double eps2, double g, double r_split,
                    double r_cut2, double box, int periodic, const int64_t* targets, int64_t nt, double* out,
                    int64_t* counts) {
  if (n == 0) return 0;
  Octree t;
  if (build_octree(pos, mass, n, t) != 0) return 1;
  SrParams p{pos, mass, eps2, g, r_split, r_cut2, box};
  short_range(t, p, periodic != 0, targets, nt, out, counts);
  return 0;
}

// TreePM force evaluation (crates/gadget-ng-treepm/src/solver.rs:66-108),
// with the periodic walk of short_range.rs:234-333 when periodic != 0 (the
// P=1 slab path, distributed.rs:59-99) and the aperiodic walk otherwise.
// r_split <= 0 selects the automatic 2.5 cells (solver.rs:56-62).
// times (optional, 4 doubles): seconds for PM, tree build, walk, total.
int orc_treepm(const double* pos, const double* mass, int64_t n, double eps2, double g, int nm, double box,
               double r_split, double r_cut_factor, int periodic, int pm_flags, const int64_t* targets, int64_t nt,
               double* out, double* out_lr, double* out_sr, int64_t* counts, double* times) {
  double t0 = omp_get_wtime();
  double r_s = r_split > 0.0 ? r_split : 2.5 * box / (double)nm;
  double r_cut = r_cut_factor * r_s;
  int64_t nm3 = (int64_t)nm * nm * nm;
  std::vector<double> rho(nm3, 0.0), fx(nm3), fy(nm3), fz(nm3);
  cic_assign(pos, mass, n, box, nm, rho.data());
  solve_forces(rho.data(), g, nm, box, r_s, 0.0, pm_flags, fx.data(), fy.data(), fz.data());
  std::vector<double> tpos(3 * nt);
  for (int64_t k = 0; k < nt; ++k)
    for (int c = 0; c < 3; ++c) tpos[3 * k + c] = pos[3 * targets[k] + c];
  std::vector<double> lr(3 * nt), sr(3 * nt, 0.0);
  cic_interpolate(fx.data(), fy.data(), fz.data(), tpos.data(), nt, box, nm, lr.data());
  double t1 = omp_get_wtime();
  Octree t;
  if (n > 0 && build_octree(pos, mass, n, t) != 0) return 1;
  double t2 = omp_get_wtime();
  if (n > 0) {
    SrParams p{pos, mass, eps2, g, r_s, r_cut * r_cut, box};
    short_range(t, p, periodic != 0, targets, nt, sr.data(), counts);
  }
  double t3 = omp_get_wtime();
  for (int64_t i = 0; i < 3 * nt; ++i) {
    out[i] = lr[i] + sr[i];
    if (out_lr) out_lr[i] = lr[i];
    if (out_sr) out_sr[i] = sr[i];
  }
  if (times) {
    times[0] = t1 - t0;
    times[1] = t2 - t1;
    times[2] = t3 - t2;
    times[3] = t3 - t0;
  }
  return 0;
}

// Plain PM (crates/gadget-ng-pm/src/solver.rs:74-140, no filter, no softening).
void orc_pm(const double* pos, const double* mass, int64_t n, double g, int nm, double box, int pm_flags,
            const int64_t* targets, int64_t nt, double* out) {
  int64_t nm3 = (int64_t)nm * nm * nm;
  std::vector<double> rho(nm3, 0.0), fx(nm3), fy(nm3), fz(nm3);
  cic_assign(pos, mass, n, box, nm, rho.data());
  solve_forces(rho.data(), g, nm, box, 0.0, 0.0, pm_flags, fx.data(), fy.data(), fz.data());
  std::vector<double> tpos(3 * nt);
  for (int64_t k = 0; k < nt; ++k)
    for (int c = 0; c < 3; ++c) tpos[3 * k + c] = pos[3 * targets[k] + c];
  cic_interpolate(fx.data(), fy.data(), fz.data(), tpos.data(), nt, box, nm, out);
}

// CIC base cells (ix0, iy0, iz0) of each particle: cic.rs:49-55.
void orc_cic_cells(const double* pos, int64_t n, double box, int nm, int32_t* cells) {
  const double inv_cell = (double)nm / box;
  const double nmf = (double)nm;
  for (int64_t i = 0; i < n; ++i)
    for (int c = 0; c < 3; ++c) cells[3 * i + c] = (int32_t)std::floor(rem_euclid(pos[3 * i + c] * inv_cell, nmf));
}

uint64_t orc_hilbert3(double x, double y, double z) { return hilbert3(x, y, z); }
uint64_t orc_morton3(double x, double y, double z) { return morton3(x, y, z); }
uint64_t orc_coords_to_hilbert(uint32_t ix, uint32_t iy, uint32_t iz, uint32_t p) {
  return coords_to_hilbert(ix, iy, iz, p);
}

// particle_hilbert with the bounding box taken from the positions themselves
// (SfcDecomposition::build_with_kind, sfc.rs:250-280), and the (key, index)
// order: keys sorted ascending, ties by original index.
void orc_hilbert_keys(const double* pos, int64_t n, uint64_t* keys, int64_t* order) {
  if (n == 0) return;
  double lo[3], hi[3];
  for (int c = 0; c < 3; ++c) {
    lo[c] = INFINITY;
    hi[c] = -INFINITY;
  }
  for (int64_t i = 0; i < n; ++i)
    for (int c = 0; c < 3; ++c) {
      lo[c] = std::min(lo[c], pos[3 * i + c]);
      hi[c] = std::max(hi[c], pos[3 * i + c]);
    }
  double l[3];
  for (int c = 0; c < 3; ++c) l[c] = std::max(hi[c] - lo[c], F64_EPS);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i)
    keys[i] = hilbert3((pos[3 * i] - lo[0]) / l[0], (pos[3 * i + 1] - lo[1]) / l[1], (pos[3 * i + 2] - lo[2]) / l[2]);
  if (order) {
    for (int64_t i = 0; i < n; ++i) order[i] = i;
    std::sort(order, order + n, [&](int64_t a, int64_t b) { return keys[a] != keys[b] ? keys[a] < keys[b] : a < b; });
  }
}

void orc_drift_kick_factors(double omega_m, double omega_lambda, double h0, double a0, double dt, double* out3) {
  Cosmo c{omega_m, omega_lambda, h0};
  c.drift_kick(a0, dt, &out3[0], &out3[1], &out3[2]);
}
double orc_advance_a(double omega_m, double omega_lambda, double h0, double a, double dt) {
  Cosmo c{omega_m, omega_lambda, h0};
  return c.advance_a(a, dt);
}

// crates/gadget-ng-integrators/src/leapfrog.rs:72-91 with the TreePM force
// (two force evaluations per step), followed by the periodic wrap of
// cosmology.rs:772-778 as stepping/mod.rs:1572-1576 applies it.
int orc_kdk_step_treepm(double* pos, double* vel, const double* mass, int64_t n, double drift, double kick_half,
                        double kick_half2, double eps2, double g, int nm, double box, double r_split,
                        double r_cut_factor, double* acc_out) {
  std::vector<int64_t> all(n);
  for (int64_t i = 0; i < n; ++i) all[i] = i;
  std::vector<double> acc(3 * n);
  if (orc_treepm(pos, mass, n, eps2, g, nm, box, r_split, r_cut_factor, 1, 0, all.data(), n, acc.data(), nullptr,
                 nullptr, nullptr, nullptr))
    return 1;
  for (int64_t i = 0; i < 3 * n; ++i) vel[i] += acc[i] * kick_half;
  for (int64_t i = 0; i < 3 * n; ++i) pos[i] += vel[i] * drift;
  if (orc_treepm(pos, mass, n, eps2, g, nm, box, r_split, r_cut_factor, 1, 0, all.data(), n, acc.data(), nullptr,
                 nullptr, nullptr, nullptr))
    return 1;
  for (int64_t i = 0; i < 3 * n; ++i) vel[i] += acc[i] * kick_half2;
  for (int64_t i = 0; i < 3 * n; ++i) pos[i] = rem_euclid(pos[i], box);
  if (acc_out) std::memcpy(acc_out, acc.data(), sizeof(double) * 3 * n);
  return 0;
}

// Direct periodic Plummer sum over minimum images (DirectGravity,
// crates/gadget-ng-core/src/gravity.rs:59-86, with minimum_image): used by
// the Ewald self-check at tiny N.
void orc_direct_min_image(const double* pos, const double* mass, int64_t n, double eps2, double g, double box,
                          const int64_t* targets, int64_t nt, double* out) {
#pragma omp parallel for schedule(static)
  for (int64_t k = 0; k < nt; ++k) {
    int64_t i = targets[k];
    double ax = 0, ay = 0, az = 0;
    for (int64_t j = 0; j < n; ++j) {
      if (j == i) continue;
      double rx = minimum_image(pos[3 * j] - pos[3 * i], box);
      double ry = minimum_image(pos[3 * j + 1] - pos[3 * i + 1], box);
      double rz = minimum_image(pos[3 * j + 2] - pos[3 * i + 2], box);
      double r2 = rx * rx + ry * ry + rz * rz + eps2;
      double inv = 1.0 / std::sqrt(r2);
      double s = g * mass[j] * inv * inv * inv;
      ax += rx * s;
      ay += ry * s;
      az += rz * s;
    }
    out[3 * k] = ax;
    out[3 * k + 1] = ay;
    out[3 * k + 2] = az;
  }
}

// FP64 Ewald sum (no counterpart in the reference; from the mathematics:
// Ewald 1921, Hernquist, Bouchet & Suto 1991).  Real space over minimum
// images within r_c with the kernel erfc(a r) + 2 a r/sqrt(pi) exp(-a^2 r^2),
// k space over 0 < |n| <= n_max with (4 pi / V)(k/k^2) exp(-k^2/4a^2)
// Im(exp(-i k.x_i) S(k)); nearest images closer than r_soft are Plummer
// softened.  Validates the device checker at small N.
void orc_ewald(const double* pos, const double* mass, int64_t n, double box, double g, double eps2, double r_soft,
               const int64_t* targets, int64_t nt, double alpha, double r_c, int n_max, double* out) {
  const double rc2 = r_c * r_c, rs2 = r_soft * r_soft;
  const double tsp = 1.1283791670955126;
  std::vector<int> modes;
  for (int x = 0; x <= n_max; ++x)
    for (int y = -n_max; y <= n_max; ++y)
      for (int z = -n_max; z <= n_max; ++z) {
        if (x * x + y * y + z * z > n_max * n_max) continue;
        if (!(x > 0 || (x == 0 && (y > 0 || (y == 0 && z > 0))))) continue;
        modes.push_back(x);
        modes.push_back(y);
        modes.push_back(z);
      }
  const int nm = (int)(modes.size() / 3);
  const double w = 2.0 * M_PI / box;
  std::vector<double> sk(2 * (size_t)nm);
#pragma omp parallel for schedule(dynamic, 16)
  for (int m = 0; m < nm; ++m) {
    double re = 0, im = 0;
    const double kx = w * modes[3 * m], ky = w * modes[3 * m + 1], kz = w * modes[3 * m + 2];
    for (int64_t j = 0; j < n; ++j) {
      const double ph = kx * pos[3 * j] + ky * pos[3 * j + 1] + kz * pos[3 * j + 2];
      re += mass[j] * std::cos(ph);
      im += mass[j] * std::sin(ph);
    }
    sk[2 * m] = re;
    sk[2 * m + 1] = im;
  }
  const double pref = 2.0 * 4.0 * M_PI / (box * box * box);
#pragma omp parallel for schedule(dynamic, 4)
  for (int64_t t = 0; t < nt; ++t) {
    const int64_t i = targets[t];
    double a[3] = {0, 0, 0};
    for (int64_t j = 0; j < n; ++j) {
      if (j == i) continue;
      double d[3];
      for (int c = 0; c < 3; ++c) {
        d[c] = pos[3 * j + c] - pos[3 * i + c];
        d[c] -= box * std::rint(d[c] / box);
      }
      const double r2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
      if (r2 >= rc2) continue;
      const double r = std::sqrt(r2), ar = alpha * r;
      double sc = (std::erfc(ar) + tsp * ar * std::exp(-ar * ar)) / (r2 * r);
      if (r2 < rs2) {
        const double q = r2 + eps2;
        sc += 1.0 / (q * std::sqrt(q)) - 1.0 / (r2 * r);
      }
      for (int c = 0; c < 3; ++c) a[c] += mass[j] * sc * d[c];
    }
    for (int m = 0; m < nm; ++m) {
      const double kx = w * modes[3 * m], ky = w * modes[3 * m + 1], kz = w * modes[3 * m + 2];
      const double k2 = kx * kx + ky * ky + kz * kz;
      const double ph = kx * pos[3 * i] + ky * pos[3 * i + 1] + kz * pos[3 * i + 2];
      const double im = std::cos(ph) * sk[2 * m + 1] - std::sin(ph) * sk[2 * m];
      const double f = pref * std::exp(-k2 / (4.0 * alpha * alpha)) / k2 * im;
      a[0] += f * kx;
      a[1] += f * ky;
      a[2] += f * kz;
    }
    for (int c = 0; c < 3; ++c) out[3 * t + c] = g * a[c];
  }
}

}  // extern "C"
