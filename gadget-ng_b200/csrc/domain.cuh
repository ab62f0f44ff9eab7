// Domain-decomposed TreePM: the per-rank device work around the exchanges.
//
// A rank holds its owned particles plus, for one force evaluation, halo
// copies of other ranks' particles within r_cut of its domain
// (crates/gadget-ng-parallel/src/mpi_rt.rs:723-781 exchange_halos_3d_periodic,
// crates/gadget-ng-treepm/src/distributed.rs:60-145 short_range_accels_sfc).
// The exchanges themselves (AABB allgather, halo alltoallv, density
// all-reduce) are the caller's; these kernels select, pack, append and drop.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "tree.cuh"

namespace tpm {

constexpr int MAX_RANKS = 64;

// One halo particle on the wire (24 bytes): fixed-point position, the
// owner's particle index, mass.  Layout of tpm_halo_record.
struct HaloRecord {
  uint32_t q[3];
  uint32_t id;
  double mass;
};

// Every rank's particle AABB as the reference packs it (aabb_to_f64:
// xlo, xhi, ylo, yhi, zlo, zhi), passed by value.
struct AabbTable {
  double v[6 * MAX_RANKS];
};

// Fixed-point min / max per axis of particles [0, n): out6 = {xmin, xmax,
// ymin, ymax, zmin, zmax} (host); scratch6: six device words.
void owned_bounds(const Particles& P, int64_t n, uint32_t* scratch6, uint32_t out6[6], cudaStream_t s);

// flags[i]: bit r set when particle i (of [0, n)) is a halo particle of rank
// r != rank: min_dist2_to_aabb_3d_periodic(x_i, aabb_r, box) < w2, skipping
// invalid boxes (halo3d.rs:237-251).  counts_dev[r] (zeroed here) = bits r set.
void halo_flags(const Particles& P, int64_t n, double scale, double box, const AabbTable& t, int n_ranks, int rank,
                double w2, uint64_t* flags, unsigned long long* counts_dev, cudaStream_t s);

// Occupancy of a coarse periodic grid of `grid`^3 cells (cell index
// ((z g + y) g + x), x = (q g) >> 32) by particles [0, n): bit c of words
// bits[c >> 5] (cleared first, (grid^3 + 31) / 32 words).
void occupancy(const Particles& P, int64_t n, int grid, uint32_t* bits, cudaStream_t s);

// flags[i]: bit r set when some cell that rank r occupies (bits + r * words)
// among the 27 around particle i's cell lies within sqrt(w2) of it (periodic
// gaps to the cell's faces, float64); cells are at least the halo width wide,
// so every particle of r within that distance is in one of them.
// counts_dev[r] (zeroed here) = bits r set.
void halo_flags_cells(const Particles& P, int64_t n, double scale, double cell, int grid, const uint32_t* bits,
                      int64_t words, int n_ranks, int rank, double w2, uint64_t* flags,
                      unsigned long long* counts_dev, cudaStream_t s);

// The particles with bit r of flags, in index order, as records at out.
void halo_pack(const Particles& P, int64_t n, const uint64_t* flags, int r, uint32_t* bit, uint32_t* pos,
               void* scan_scratch, HaloRecord* out, cudaStream_t s);

// Stable partition: the particles with id < n_owned of src [0, n) to dst
// [0, n_owned), with their accelerations (ax..az -> tx..tz).  flag / pos:
// n words of scratch each.
void compact_owned(const Particles& src, const Particles& dst, int64_t n, uint32_t n_owned, const float* ax,
                   const float* ay, const float* az, float* tx, float* ty, float* tz, uint32_t* flag, uint32_t* pos,
                   void* scan_scratch, cudaStream_t s);

// Halo records to particles [first, first + m) with ids first + k, zero velocity.
void append_halos(const Particles& P, int64_t first, const HaloRecord* rec, int64_t m, cudaStream_t s);

// mask[i] = id[i] < n_owned (walk targets).
void owned_mask(const uint32_t* id, int64_t n, uint32_t n_owned, uint8_t* mask, cudaStream_t s);

}  // namespace tpm
