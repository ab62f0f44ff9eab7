/*
 * treepm_b200 — C ABI of the B200 (sm_100a) TreePM gravity solver.
 *
 * Drop-in boundary: gadget-ng's `GravitySolver` trait
 * (crates/gadget-ng-core/src/gravity.rs:14-56), implemented by
 * `TreePmSolver` (crates/gadget-ng-treepm/src/solver.rs:44-108) and
 * `PmSolver` (crates/gadget-ng-pm/src/solver.rs:23-140), constructed by
 * `make_solver` (crates/gadget-ng-cli/src/engine/gravity.rs:352-556).  The
 * integrator-side fused step replaces `leapfrog_cosmo_kdk_step`
 * (crates/gadget-ng-integrators/src/leapfrog.rs:72-91).  The existing CUDA PM
 * FFI of the reference (crates/gadget-ng-cuda/cuda/pm_gravity.h:11-66) is the
 * pattern: an opaque handle, plain pointers and sizes, an int status.
 *
 * Conventions
 *  - Every entry point returns an int status (TPM_OK == 0) and never aborts;
 *    tpm_last_error() gives a message for the last failure on a handle.
 *  - Host buffers are caller-owned and copied synchronously inside the call.
 *    Device state is handle-owned and persists between calls.
 *  - A handle is not thread-safe: one host thread per handle, as the
 *    reference calls its solver from one thread at a time
 *    (crates/gadget-ng-cuda/src/pm_solver.rs:29-34).
 *  - Positions are stored on the device as 32-bit fixed point per axis in
 *    the periodic box (x = q * L / 2^32); inputs on that lattice round-trip
 *    exactly.
 */
#ifndef TREEPM_B200_H
#define TREEPM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------- */
enum {
  TPM_OK = 0,
  TPM_ERR_INVALID_ARGUMENT = 1,
  TPM_ERR_CUDA = 2,            /* a CUDA runtime call failed */
  TPM_ERR_OUT_OF_MEMORY = 3,   /* device allocation refused (or over the handle's memory cap) */
  TPM_ERR_COINCIDENT = 4,      /* two particles at the same position: the reference's
                                  insertion octree recurses without bound on these
                                  (crates/gadget-ng-tree/src/octree.rs:501-540) */
  TPM_ERR_WALK_STACK = 5,      /* tree-walk stack capacity exceeded */
  TPM_ERR_DEFERRED = 6,        /* exact-fallback work list overflowed */
  TPM_ERR_NOT_READY = 7,       /* call needs particles / forces that are not set */
  TPM_ERR_NO_DEVICE = 8,       /* no CUDA device, or the device is not sm_100 */
  TPM_ERR_NONFINITE = 9,       /* non-finite input position or mass */
  TPM_ERR_TOO_LARGE = 10,      /* more particles than tpm_hilbert_sort_noalloc's fixed scratch holds */
  TPM_ERR_IO = 11              /* a snapshot or checkpoint file could not be written, read or parsed */
};

/* ---- configuration flags -------------------------------------------------- */
/* Short range with the aperiodic walk of short_range.rs:120-208 (the
 * trait-level TreePmSolver).  Default: the periodic walk of
 * short_range.rs:234-333 (treepm_slab at P=1). */
#define TPM_FLAG_APERIODIC_WALK     (1u << 0)
/* Divide the Green's function by the CIC window squared (extension; the
 * reference force path has no deconvolution). */
#define TPM_FLAG_DECONVOLVE_CIC     (1u << 1)
/* 4-point finite-difference gradient in k-space instead of the exact i·k of
 * fft_poisson.rs:542-548 (extension). */
#define TPM_FLAG_FOUR_POINT_GRADIENT (1u << 2)
/* Plain PM (PmSolver): no Gaussian filter, no short range. */
#define TPM_FLAG_PM_ONLY            (1u << 3)
/* Group walk targets along the Hilbert curve of sfc.rs:95-204 instead of the
 * octree's own order. */
#define TPM_FLAG_HILBERT_TARGETS    (1u << 4)
/* Accurate short range (extension, validated against Ewald only): the split
 * kernel erfc(x) + (2x/sqrt(pi)) exp(-x^2) that complements the Gaussian
 * long-range filter exactly (the reference's short_range.rs:108-111 keeps
 * erfc(x) alone), and the geometric opening criterion s/d < theta of the
 * reference's Barnes-Hut walk (crates/gadget-ng-tree/src/octree.rs:763-809)
 * instead of the 0.1 r_cut node-size rule, so a node holding the target is
 * never taken as a monopole (theta must lie in (0, 0.577)).  Culls use the
 * node's whole cell. */
#define TPM_FLAG_ACCURATE           (1u << 5)
/* Learned short range (extension): keep the long-range potential on the mesh
 * and, once a network is attached (tpm_set_learned), take the short-range
 * acceleration from it outside dense cells (see tpm_cnn below). */
#define TPM_FLAG_LEARNED            (1u << 6)

typedef struct tpm_config {
  int32_t grid_size;          /* [gravity] pm_grid_size (power of two, 8..1024) */
  double box_size;            /* [simulation] box_size */
  double r_split;             /* [gravity] r_split; <= 0 selects 2.5 cells (solver.rs:56-62) */
  double r_cut_factor;        /* extension key gravity.r_cut_factor; <= 0 selects 5.0 (solver.rs:80) */
  double theta;               /* [gravity] theta: unused by the parity walk; the opening angle of TPM_FLAG_ACCURATE (0 = 0.5) */
  int32_t opening_criterion;  /* [gravity] opening_criterion: 0 geometric, 1 relative (octree.rs:769-796);
                                 read by the TPM_FLAG_ACCURATE walk, not by the parity walk */
  double err_tol_force_acc;   /* [gravity] err_tol_force_acc: the relative criterion's tolerance */
  uint32_t flags;             /* TPM_FLAG_* */
  int32_t device;             /* CUDA device ordinal */
  int64_t memory_cap_bytes;   /* 0 = no cap; otherwise refuse allocations beyond it */
} tpm_config;

typedef struct tpm_stats {
  int64_t n_particles;
  int64_t n_tree_nodes;         /* internal octree nodes (non-empty) */
  int64_t n_groups;             /* walk target groups */
  int64_t leaf_pairs;           /* particle-particle interactions of the last walk */
  int64_t monopoles;            /* particle-node interactions of the last walk */
  int64_t evaluated_pairs;      /* pair evaluations issued, including masked ones */
  int64_t exact_fallbacks;      /* borderline decisions resolved in FP64 */
  int64_t deferred_opens;       /* nodes opened per target (COM on the target) */
  int32_t max_tree_depth;
  int32_t terminal_depth;       /* first depth whose half size is < 0.1 r_cut */
  /* device milliseconds of the last force evaluation, per stage */
  float ms_bbox_keys;
  float ms_sort;
  float ms_build;
  float ms_walk;
  float ms_pm;
  float ms_gather_kick;
  float ms_total;
  int32_t last_error;
  int64_t kernel_launches;      /* kernels launched by the last call that computed forces */
  int64_t learned_particles;    /* particles whose short range came from the network (TPM_FLAG_LEARNED) */
  int64_t walk_groups;          /* walk groups walked (all groups, or those holding fallback particles) */
  float ms_learned;             /* device milliseconds of the network and its mask */
  int64_t force_evaluations;    /* force evaluations since the handle was created */
} tpm_stats;

typedef struct tpm_handle tpm_handle;

/* ---- lifecycle ---------------------------------------------------------- */
/* make_solver (crates/gadget-ng-cli/src/engine/gravity.rs:511-517) +
 * TreePmSolver { grid_size, box_size, r_split } (solver.rs:44-52). */
int tpm_create(const tpm_config* cfg, tpm_handle** out);
void tpm_destroy(tpm_handle* h);
const char* tpm_last_error(const tpm_handle* h);
int tpm_version(void);

/* ---- the GravitySolver call ----------------------------------------------
 * accelerations_for_indices(global_positions, global_masses, eps2, g,
 * global_indices, out) — crates/gadget-ng-core/src/gravity.rs:16-24.
 * positions: n x 3 float64 (AoS, like &[Vec3]); masses: n float64;
 * indices: n_idx uint64 (usize); out: n_idx x 3 float64.
 * out.len() == global_indices.len() is the reference's assertion
 * (solver.rs:75); here n_idx sizes both. */
int tpm_accelerations_for_indices(tpm_handle* h, const double* global_positions, const double* global_masses,
                                  int64_t n, double eps2, double g, const uint64_t* global_indices,
                                  int64_t n_idx, double* out);

/* ---- device-resident state (the fused integrator path) ----------------- */
/* Upload particles: positions n x 3 float64 (wrapped into the box), velocities
 * n x 3 float64 (canonical momentum p = a^2 dx/dt, may be NULL = zero),
 * masses n float64. */
int tpm_set_particles(tpm_handle* h, const double* pos, const double* vel, const double* mass, int64_t n);
/* Same, with positions already in 32-bit fixed point (n x 3). */
int tpm_set_particles_fixed(tpm_handle* h, const uint32_t* q, const float* vel, const double* mass, int64_t n);
/* One force evaluation of all resident particles (results stay on the device). */
int tpm_compute_forces(tpm_handle* h, double eps2, double g);
/* leapfrog_cosmo_kdk_step (leapfrog.rs:72-91) + wrap_position
 * (crates/gadget-ng-core/src/cosmology.rs:772-778) fused on the device.
 * The opening half kick reuses the previous step's closing acceleration,
 * rescaled by g / g_prev when only the coupling G*a^3 changed; it recomputes
 * when eps2 changed or no acceleration is cached. */
int tpm_kdk_step(tpm_handle* h, double kick_half, double drift, double kick_half2, double eps2, double g);
/* Host KDK step: state in host buffers (n x 3 float64 pos / vel), copied to
 * the device, advanced as tpm_kdk_step, copied back (original order).  When
 * the caller hands back the state the previous call returned (and nothing
 * changed the handle's state since), the step runs on the resident state at
 * once with its closing acceleration (one force evaluation) while a second
 * stream uploads the inputs, checks them bit for bit against the returned
 * state and copies the new positions back; the momenta follow the closing
 * kick.  Inputs that differ are re-encoded from the upload and stepped with
 * two force evaluations (the speculative one is discarded). */
int tpm_kdk_step_host(tpm_handle* h, double* pos, double* vel, const double* mass, int64_t n, double kick_half,
                      double drift, double kick_half2, double eps2, double g);
/* Read back state in the original particle order (any pointer may be NULL). */
int tpm_get_state(tpm_handle* h, double* pos, double* vel, double* acc);
/* Long-range and short-range parts of the last force evaluation (original
 * order, n x 3 float64 each; either may be NULL). */
int tpm_get_force_parts(tpm_handle* h, double* acc_lr, double* acc_sr);
int tpm_get_stats(const tpm_handle* h, tpm_stats* out);
/* Interactions of the last short-range walk per particle (original order,
 * n x 2: leaf pairs, monopoles) — the per-target work counters the reference
 * keeps for its walks (crates/gadget-ng-tree/src/octree.rs:77-151). */
int tpm_get_interaction_counts(tpm_handle* h, int64_t* counts);

/* ---- the stream the handle launches on ----------------------------------- */
int tpm_set_stream(tpm_handle* h, void* cuda_stream);
void* tpm_get_stream(const tpm_handle* h);

/* ---- domain-decomposed TreePM (one handle per rank) -----------------------
 * The reference's distributed TreePM with SFC domains: each rank owns its
 * particles; for one force evaluation it also holds halo copies of the other
 * ranks' particles within r_cut of its particle AABB
 * (ParallelRuntime::exchange_halos_3d_periodic,
 * crates/gadget-ng-parallel/src/lib.rs:168 and src/mpi_rt.rs:723-781); the
 * short range walks a tree of owned + halo particles for the owned targets
 * (short_range_accels_sfc, crates/gadget-ng-treepm/src/distributed.rs:119-145)
 * and the long range solves the all-ranks density (the density all-reduce of
 * ParallelRuntime::allreduce_sum_f64_slice, lib.rs:200-210).  The caller
 * performs the three exchanges (AABB allgather, halo alltoallv, density
 * all-reduce); the handle does the device work around them.  Results and
 * state accessors report owned particles only (n_owned of them, original
 * order); any other force call drops the halo copies first. */

/* One halo particle on the wire: 32-bit fixed-point position (x = q L / 2^32),
 * the owner's particle index, mass (24 bytes). */
typedef struct tpm_halo_record {
  uint32_t q[3];
  uint32_t id;
  double mass;
} tpm_halo_record;

/* AABB of the owned particles as the reference packs it (aabb_to_f64,
 * crates/gadget-ng-parallel/src/halo3d.rs): {xlo, xhi, ylo, yhi, zlo, zhi};
 * an empty rank gives lo = +inf, hi = -inf (an invalid box). */
int tpm_owned_aabb(tpm_handle* h, double aabb6[6]);
/* Halo selection for every rank r != rank: the owned particles whose periodic
 * distance to rank r's AABB (aabbs + 6 r; invalid boxes skipped) is below
 * `width` (min_dist2_to_aabb_3d_periodic < width^2, halo3d.rs:237-260).
 * counts[r] (host, n_ranks) receives the number per rank; when `send` (device,
 * cap records) is non-NULL the records follow grouped by destination rank in
 * rank order, each group in the handle's particle order.  A particle can go to
 * several ranks.  n_ranks <= 64.  A total above cap returns
 * TPM_ERR_INVALID_ARGUMENT with counts filled and nothing written. */
int tpm_halo_select(tpm_handle* h, const double* aabbs, int32_t n_ranks, int32_t rank, double width,
                    int64_t* counts, tpm_halo_record* send, int64_t cap);
/* A tighter halo rule than the AABB (extension; the short-range trees then
 * differ from the reference's, the interaction sets within r_cut do not): a
 * periodic grid of *grid = min(64, floor(L / width)) cells per axis (cells at
 * least `width` wide); tpm_occupancy writes the owned particles' occupancy
 * (bit c of bits[c / 32], c = (z g + y) g + x, (g^3 + 31) / 32 words; bits may
 * be NULL to get the grid only).  tpm_halo_select_cells takes every rank's
 * occupancy (n_ranks x words, host) and selects for rank r != rank the owned
 * particles within `width` of a cell that r occupies among the 27 around the
 * particle's own (float64 gaps to the cell faces, width^2 widened by 1e-9
 * relative); counts and send as tpm_halo_select. */
int tpm_occupancy(tpm_handle* h, double width, int32_t* grid, uint32_t* bits);
int tpm_halo_select_cells(tpm_handle* h, const uint32_t* bits, int32_t grid, int32_t n_ranks, int32_t rank,
                          double width, int64_t* counts, tpm_halo_record* send, int64_t cap);
/* Replace the halo copies by n records (device memory, e.g. the halo
 * alltoallv's receive buffer); owned particles are kept. */
int tpm_set_halos(tpm_handle* h, const tpm_halo_record* recv, int64_t n);
/* The three stages of a domain-decomposed force evaluation, on the handle's
 * stream.  tpm_force_begin: keys, sort, and the CIC deposit of the OWNED
 * particles into the density mesh, whose device address and cell count
 * tpm_mesh_density returns (float32, [z][y][x]); the caller then sums that mesh
 * over all ranks in place (after the stream reaches this point) and may
 * overlap the sum with tpm_force_short_range (tree over owned + halo
 * particles, walk for the owned).  tpm_force_end (the summed density in place
 * before the handle's stream reaches it): FFT Poisson solve, gather of long +
 * short range and, kick != 0, v += a kick for the owned particles. */
int tpm_force_begin(tpm_handle* h);
int tpm_mesh_density(tpm_handle* h, float** density, int64_t* cells);
int tpm_force_short_range(tpm_handle* h, double eps2);
int tpm_force_end(tpm_handle* h, double g, double kick);
/* tpm_force_end without the FFT solve: the gather reads the force meshes the
 * caller assembled (the z-slab path below), per unit G, [c][z][y][x]. */
int tpm_force_end_solved(tpm_handle* h, double g, double kick);

/* z-slab decomposition of the PM solve (crates/gadget-ng-pm/src/slab_fft.rs
 * :209-330 and slab_pm.rs:1-30, the reference's `pm_slab` path): instead of
 * summing the whole density mesh on every rank and solving it everywhere,
 * rank r owns z planes [r nzl, (r+1) nzl) (nzl = pm_grid_size / ranks; the
 * mesh size must be a multiple of the rank count).  Between tpm_force_begin
 * and tpm_force_end_solved, with the caller's collectives on the listed device
 * buffers, in this order:
 *   1. reduce-scatter of the tpm_mesh_density mesh over the ranks into
 *      density_slab (rank r gets planes r nzl ..);
 *   2. tpm_pm_slab_forward: x and y transforms of those planes, send filled;
 *   3. all-to-all of forward_bytes (equal splits) from send into recv;
 *   4. tpm_pm_slab_poisson: z transforms, Green's function x filter x
 *      gradient and inverse z transforms of the y rows [r nyl, (r+1) nyl),
 *      send filled again;
 *   5. all-to-all of return_bytes from send into recv;
 *   6. tpm_pm_slab_inverse: inverse y and x transforms into force_slab
 *      (3 x slab_cells floats);
 *   7. all-gather of each component's slab into force_mesh (3 x mesh_cells).
 * Each stage runs on the handle's stream; the caller orders its collectives
 * after it.  tpm_pm_slab_setup allocates the slab buffers once per
 * (rank, ranks) and returns their addresses. */
typedef struct tpm_slab_buffers {
  float* density_slab;    /* slab_cells floats */
  void* send;             /* transpose send buffer (return_bytes) */
  void* recv;             /* transpose receive buffer (return_bytes) */
  int64_t forward_bytes;  /* bytes of the first all-to-all (forward_bytes / ranks per peer) */
  int64_t return_bytes;   /* bytes of the second all-to-all */
  float* force_slab;      /* 3 x slab_cells floats, per unit G */
  float* force_mesh;      /* 3 x mesh_cells floats: the meshes tpm_force_end_solved gathers from */
  int32_t planes;         /* nzl */
  int64_t slab_cells;     /* nzl x nm x nm */
  int64_t mesh_cells;     /* nm^3 */
} tpm_slab_buffers;
int tpm_pm_slab_setup(tpm_handle* h, int32_t rank, int32_t ranks, tpm_slab_buffers* out);
int tpm_pm_slab_forward(tpm_handle* h);
int tpm_pm_slab_poisson(tpm_handle* h);
int tpm_pm_slab_inverse(tpm_handle* h);
/* The opening half of a domain-decomposed KDK step: halo copies dropped,
 * then v += a kick_half (the cached acceleration rescaled by g / g_prev) and
 * the drift with the periodic wrap, for the owned particles. */
int tpm_kick_drift(tpm_handle* h, double kick_half, double drift, double g);
/* SFC keys of the owned particles over a given box {xlo, xhi, ylo, yhi, zlo,
 * zhi} (all ranks' bounding box for SfcDecomposition, sfc.rs:336-393),
 * original order.  kind (SfcKind): TPM_SFC_HILBERT = particle_hilbert
 * (sfc.rs:187-204; its keys pack the coordinate bits lowest level first, so
 * nearby keys need not be nearby in space), TPM_SFC_MORTON = particle_morton
 * (sfc.rs:54-81, Z order). */
#define TPM_SFC_HILBERT 0
#define TPM_SFC_MORTON 1
int tpm_sfc_keys(tpm_handle* h, const double bbox6[6], int32_t kind, uint64_t* keys);
/* Owned and resident (owned + halo) particle counts. */
int tpm_particle_counts(const tpm_handle* h, int64_t* n_owned, int64_t* n_resident);

/* ---- cosmology (FP64 host) ------------------------------------------------
 * CosmologyParams::drift_kick_factors (crates/gadget-ng-core/src/cosmology.rs:188-233)
 * for LambdaCDM: out3 = {drift, kick_half, kick_half2}. */
int tpm_drift_kick_factors(double omega_m, double omega_lambda, double h0, double a0, double dt, double* out3);
/* CosmologyParams::advance_a (cosmology.rs:172-178). */
double tpm_advance_a(double omega_m, double omega_lambda, double h0, double a, double dt);

/* ---- inspection of the hot-path stages (parity tests) ------------------- */
/* Hilbert keys of the resident particles (particle_hilbert, sfc.rs:187-204,
 * bounding box from the positions) and their (key, original index) order. */
int tpm_hilbert_keys(tpm_handle* h, uint64_t* keys, int64_t* order);
/* CIC base cell (ix0, iy0, iz0) of each resident particle, original order
 * (cic.rs:49-55). */
int tpm_cic_cells(tpm_handle* h, int32_t* cells);
/* Number of non-empty octree nodes of the last force evaluation. */
int64_t tpm_tree_node_count(const tpm_handle* h);
/* Export the non-empty octree nodes: per node depth, mass, COM (float64),
 * quadrupole (6), the original index of the particle for leaves (-1 for
 * internal nodes) and the octant path key (3 bits per level, root = 1).  cap
 * is the array capacity; returns the count written (or a negative status). */
int64_t tpm_export_tree(tpm_handle* h, int64_t cap, int32_t* depth, double* mass, double* com, double* quad,
                        int64_t* particle, uint64_t* path_hi, uint64_t* path_lo);
/* The PM mesh of the last force evaluation: density (mass per cell, nm^3)
 * and the three force grids (nm^3 each), float32; any may be NULL. */
int tpm_get_mesh(tpm_handle* h, float* density, float* fx, float* fy, float* fz);

/* ---- allocation-free variant ---------------------------------------------------
 * No counterpart in the reference.  The Hilbert keys and (key, index) order of
 * tpm_hilbert_keys, for callers that cannot call cudaMalloc — a simulation that
 * owns all device memory through its own pool and forbids other allocations,
 * or code running where an allocation would stall or break it.  It allocates
 * nothing: the radix sort's intermediate buffers live in a fixed file-scope
 * device array of about 3.3 MB, held on every GPU that loads this library
 * until the process exits.
 *  - qx, qy, qz: device arrays of n 32-bit fixed-point positions
 *    (x = q * box_size / 2^32); keys_out (n uint64) and order_out (n uint32):
 *    device arrays owned by the caller.  On return keys_out holds the keys
 *    sorted ascending and order_out the input index of each, ties by
 *    ascending index.  Work is queued on `stream` (NULL = legacy default);
 *    the caller synchronises before reading the outputs.
 *  - n above TPM_NOALLOC_MAX_PARTICLES returns TPM_ERR_TOO_LARGE, nothing runs.
 *  - The first call on a device looks up the array's device address with that
 *    device current; make that first call before any stream capture.
 *  - Every call shares the one array: calls that overlap on the GPU race. */
#define TPM_NOALLOC_MAX_PARTICLES (1 << 18)
int tpm_hilbert_sort_noalloc(const uint32_t* qx, const uint32_t* qy, const uint32_t* qz, int64_t n,
                             double box_size, uint64_t* keys_out, uint32_t* order_out, void* stream);

/* ---- measurement -----------------------------------------------------------
 * No counterpart in the reference: FP64 Ewald accelerations of the targets
 * (periodic box `box`, coupling g), the accuracy reference of the TreePM
 * force.  Real space over minimum images within r_c (Ewald parameter alpha),
 * k space over integer modes 0 < |n| <= n_max; nearest images closer than
 * r_soft are Plummer softened with eps2.  Host arrays in and out (n x 3
 * positions, n masses, nt target indices, nt x 3 out); allocates and frees its
 * own device buffers.  A checker: run outside timed regions. */
int tpm_ewald(const double* pos, const double* mass, int64_t n, double box, double g, double eps2, double r_soft,
              const int64_t* targets, int64_t nt, double alpha, double r_c, int n_max, int device, double* out);
/* No counterpart in the reference: FFMA throughput of `device` in TFLOP/s, the
 * FP32 roofline denominator of the short-range walk. */
int tpm_fp32_peak(int device, double* tflops);

/* ---- Zel'dovich initial conditions -----------------------------------------------
 * zeldovich_ics (crates/gadget-ng-core/src/ic_zeldovich.rs:287-760) generated
 * on the device into a handle: n_side^3 particles of mass 1/N on the lattice
 * (cell centres, gid = ix n^2 + iy n + iz) displaced by the 1LPT field of a
 * Gaussian density with per-mode sigma(|n|) = A |n|^(n_s/4) / sqrt(N^3)
 * (transfer 0, power law) or A k^(n_s/2) T_EH(k) / sqrt(N^3) (transfer 1,
 * Eisenstein-Hu no-wiggle, k = 2 pi |n| h / box_size_mpc_h, A from sigma8 when
 * sigma8 > 0); momenta a^2 f(a) H(a) Psi (cosmology != 0) or H0 Psi (a = 1,
 * f = 1).  rescale_to_a_init multiplies Psi by D(a_init)/D(1) (CPT92).  With
 * use_2lpt, x = q + Psi1 + (D2/D1^2) Psi2 and p = a^2 H (f1 Psi1 + f2 (D2/D1^2)
 * Psi2), Psi2 = -i n / |n|^2 S(k) from the sum of the 2x2 minors of phi_ab
 * (Psi2 scaled by the rescale squared).  Each
 * mode is seeded by the reference's mode_seed (murmur3 fmix64 of seed and the
 * packed mode index); the two uniforms of its Box-Muller Gaussians come from
 * SplitMix64 seeded there instead of the reference's StdRng, so realisations
 * are reproducible but differ from the reference's; statistics and
 * conventions match. */
typedef struct tpm_zeldovich {
  int32_t n_side;         /* power of two, 4..1024 */
  int32_t transfer;       /* 0 power law, 1 Eisenstein-Hu no-wiggle */
  uint64_t seed;
  double amplitude;
  double spectral_index;
  double sigma8;          /* <= 0: use amplitude */
  double omega_m, omega_lambda, omega_b, h;
  double box_size_mpc_h;  /* box in Mpc/h for k (Eisenstein-Hu) */
  double a_init;
  double h0;              /* H0 in internal time units */
  int32_t cosmology;      /* 0: a = 1, f = 1, H = h0 */
  int32_t rescale_to_a_init;
  int32_t use_2lpt;       /* 1: second-order displacements (ic_2lpt.rs:386-550) */
  int32_t reserved;       /* 0 */
} tpm_zeldovich;
int tpm_set_particles_zeldovich(tpm_handle* h, const tpm_zeldovich* cfg);
/* Host evaluation of sigma(|n|) for count values and the five factors
 * [A, a^2 f1 H, growth rescale D(a)/D(1), D2/D1^2, a^2 f2 H D2/D1^2]
 * (factors may be NULL). */
int tpm_zeldovich_sigma(const tpm_zeldovich* cfg, const double* n_abs, int64_t count, double* sigma, double* factors);

/* ---- power spectrum (in-situ analysis) ----------------------------------------
 * power_spectrum(positions, masses, box_size, mesh)
 * (crates/gadget-ng-analysis/src/power_spectrum.rs:35-120): CIC assignment,
 * 3D FFT, |delta_k|^2 / (sinc sinc sinc)^2 * (V/mesh^3)^2 averaged in shells
 * floor(|k| - 1/2) of the fundamental.  Outputs hold mesh/2 shells: k (bin + 1)
 * 2 pi / L, P(k) (0 where n_modes is 0 — the reference drops those shells)
 * and the mode counts.  mesh: power of two in [4, 1024]. */
int tpm_power_spectrum(const double* pos, const double* mass, int64_t n, double box, int32_t mesh, int32_t device,
                       double* k, double* pk, uint64_t* n_modes);
/* The same estimator on a handle's resident particles (mesh = its pm_grid_size);
 * overwrites the density mesh that tpm_get_mesh returns. */
int tpm_get_power_spectrum(tpm_handle* h, double* k, double* pk, uint64_t* n_modes);

/* ---- snapshots and checkpoints ---------------------------------------------------
 * The files of gadget-ng's SnapshotWriter implementations: <dir>/meta.json,
 * <dir>/provenance.json and <dir>/particles.jsonl (JsonlWriter,
 * crates/gadget-ng-io/src/snapshot.rs:124-146) or <dir>/particles.bin
 * (BincodeWriter, bincode_writer.rs:16-31), records in global-id order with
 * the current ParticleRecord fields (dark matter: internal_energy and
 * smoothing_length 0, ptype DarkMatter).  Checkpoints are
 * <dir>/checkpoint/{particles.jsonl, meta.json, provenance.json,
 * checkpoint.json} (crates/gadget-ng-cli/src/engine/checkpoint.rs:47-110). */
#define TPM_SNAPSHOT_JSONL 0
#define TPM_SNAPSHOT_BINCODE 1

/* Provenance (crates/gadget-ng-io/src/provenance.rs:4-12); git_commit NULL
 * is written as null. */
typedef struct tpm_provenance {
  const char* crate_version;
  const char* git_commit;
  const char* build_profile;
  const char* const* enabled_features;
  int32_t n_enabled_features;
  int32_t n_command_line;
  const char* const* command_line;
  const char* config_hash;
} tpm_provenance;

/* SnapshotEnv (crates/gadget-ng-io/src/writer.rs:10-37): time, redshift and
 * box size of meta.json, units when has_units != 0. */
typedef struct tpm_snapshot_env {
  double time;
  double redshift;
  double box_size;
  int32_t has_units;
  int32_t reserved;
  double length_in_kpc, mass_in_msun, velocity_in_km_s, time_in_gyr, g_internal;
} tpm_snapshot_env;

/* The resident state (decoded on the device; JSONL formatted by host threads
 * from double-buffered chunk copies; bincode records built on the device). */
int tpm_write_snapshot(tpm_handle* h, const char* out_dir, int32_t format, const tpm_snapshot_env* env,
                       const tpm_provenance* prov);
/* Load a snapshot's particles into the handle (global ids must be 0..n-1);
 * env_out (may be NULL) receives meta.json's time, redshift, box size, units. */
int tpm_read_snapshot(tpm_handle* h, const char* dir, int32_t format, tpm_snapshot_env* env_out);
/* Host arrays (the reference's write_snapshot on a particle slice):
 * positions and velocities n x 3, masses n, global ids n (NULL: 0..n-1). */
int tpm_write_snapshot_host(const char* out_dir, int32_t format, const double* pos, const double* vel,
                            const double* mass, const uint64_t* global_ids, int64_t n,
                            const tpm_snapshot_env* env, const tpm_provenance* prov);
/* Read a snapshot in file order into host arrays of `capacity` records
 * (all four may be NULL to query *n_out only). */
int tpm_read_snapshot_host(const char* dir, int32_t format, int64_t* n_out, double* pos, double* vel,
                           double* mass, uint64_t* global_ids, int64_t capacity, tpm_snapshot_env* env_out);
const char* tpm_snapshot_last_error(void);  /* message of the last failed *_host call on this thread */
/* save_checkpoint / load_checkpoint of the serial engine: the JSONL state and
 * checkpoint.json (completed step, a, config hash, particle count). */
int tpm_write_checkpoint(tpm_handle* h, const char* out_dir, uint64_t completed_step, double a_current,
                         const char* config_hash);
int tpm_read_checkpoint(tpm_handle* h, const char* resume_dir, uint64_t* completed_step, double* a_current,
                        char* config_hash, int64_t config_hash_capacity);

/* ---- learned short-range network (extension) --------------------------------
 * No counterpart in the reference.  A small 3D CNN reads the long-range mesh
 * (density and potential) and predicts the short-range acceleration at each
 * particle; a solver created with TPM_FLAG_LEARNED and given a trained network
 * (tpm_set_learned) uses it instead of the tree walk for particles whose 8
 * CIC nodes all have overdensity <= delta_max, and walks the tree for the
 * rest.  Network: three valid 3x3x3 convolutions to 16 channels with GELU
 * (BF16 on the tensor cores, FP32 accumulation), a linear head 16 -> 3 read
 * by trilinear interpolation.  Parameters are a flat float32 vector
 * [W1 (27,16,c_in), b1 (16), W2 (27,16,16), b2, W3 (27,16,16), b3,
 * Wh (3,16), bh (3)]; tap t = (dz*3 + dy)*3 + dx reads node o + (dx,dy,dz).
 * Host arrays are copied synchronously. */
typedef struct tpm_cnn tpm_cnn;
/* Failure-detection self-test of the tensor-core kernels' bounded waits: one
 * tile whose MMAs are never issued must end by its wait's 2 s limit with the
 * timeout flag set and its TMEM freed, and a normal tile must then run on the
 * same context.  TPM_OK with the seconds the first tile took, else an error. */
int tpm_selftest_bounded_wait(int32_t device, double* waited_seconds);
int64_t tpm_cnn_param_count(int32_t c_in);
int tpm_cnn_create(int32_t c_in, int32_t device, tpm_cnn** out);
int tpm_cnn_destroy(tpm_cnn* c);
const char* tpm_cnn_last_error(const tpm_cnn* c);
int tpm_cnn_set_params(tpm_cnn* c, const float* params, int64_t n);  /* also resets Adam */
int tpm_cnn_get_params(tpm_cnn* c, float* params, int64_t n);
/* Features x = (raw - shift) * scale; raw = (ln(1 + rho/m_cell), phi * cell / m_cell);
 * the head predicts a / (out_scale * m_cell / cell^2).  Captured boxes set
 * them from the first box unless set here. */
int tpm_cnn_set_scales(tpm_cnn* c, const float* shift, const float* scale, float out_scale, float delta_max);
int tpm_cnn_get_scales(const tpm_cnn* c, float* shift, float* scale, float* out_scale, float* delta_max);
/* Radius (in mesh cells, 0..1; default 0) of the exact near-field pair sum the
 * network is combined with: the network predicts the short range minus the
 * pairs closer than this, which the solver sums directly over the 27
 * neighbouring cells.  Set before capturing boxes; 0 = the network alone. */
int tpm_cnn_set_near(tpm_cnn* c, float near_cells);
float tpm_cnn_get_near(const tpm_cnn* c);
/* Forward of a batch of volumes x0 [batch][d][d][d][c_in] -> head output
 * out [batch][d-6][d-6][d-6][3]. */
int tpm_cnn_forward(tpm_cnn* c, const float* x0, int32_t batch, int32_t d, float* out);
/* Loss sum_p w_p |pred_p - target_p|^2 / sum w and its gradient; particle p
 * reads volume pb[p] at node coordinates ps[p] (within [0, d-7]). */
int tpm_cnn_loss_grad(tpm_cnn* c, const float* x0, int32_t batch, int32_t d, int64_t n, const int32_t* pb,
                      const float* ps, const float* target, const float* weight, float* loss, float* grad);
/* One Adam step with `grad` (host; NULL = the last computed gradient). */
int tpm_cnn_adam_step(tpm_cnn* c, const float* grad, float lr, float beta1, float beta2, float eps);
/* Capture a training (or held-out) box from a solver handle created with
 * TPM_FLAG_LEARNED after tpm_compute_forces without a network: the mesh
 * features and, for particles in cells at or below delta_max, the
 * short-range acceleration of the walk as the target. */
int tpm_cnn_add_box(tpm_cnn* c, tpm_handle* solver, int32_t held_out);
int tpm_cnn_box_count(const tpm_cnn* c, int32_t held_out);
/* `steps` Adam steps (lr, beta 0.9 / 0.999, eps 1e-8) on batches of
 * `batch` random 14^3 patches of the training boxes; loss per step out. */
int tpm_cnn_train(tpm_cnn* c, int32_t steps, int32_t batch, float lr, uint64_t seed, float* loss_history);
/* Weighted loss over a tiling of the held-out (or training) boxes. */
int tpm_cnn_evaluate(tpm_cnn* c, int32_t held_out, int32_t batch, float* loss);
/* Give a TPM_FLAG_LEARNED solver a copy of the network (NULL detaches it). */
int tpm_set_learned(tpm_handle* h, const tpm_cnn* c);

#ifdef __cplusplus
}
#endif

#endif /* TREEPM_B200_H */
