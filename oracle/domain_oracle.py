"""CPU restatement (numpy + the C oracle) of gadget-ng's domain-decomposed
TreePM.  Test infrastructure only: the tests compare the library's per-rank
results with these.

Follows
  crates/gadget-ng-parallel/src/halo3d.rs: Aabb3, compute_aabb_3d,
    min_dist2_to_aabb_3d_periodic (:237-251), is_in_periodic_halo (:258-260),
    minimum_image_scalar;
  crates/gadget-ng-parallel/src/mpi_rt.rs:723-781 exchange_halos_3d_periodic
    (AABB allgather; rank q sends to every r != q with a valid AABB the
    particles with min_dist2 < width^2, in q's order; r concatenates what it
    receives in rank order);
  crates/gadget-ng-treepm/src/distributed.rs:60-145 short_range_accels_sfc
    (tree over local + halo, forces for the locals) and the long range of the
    all-ranks density (lib.rs:200-210 allreduce_sum_f64_slice): the serial
    TreePM's long-range part;
  crates/gadget-ng-parallel/src/sfc.rs:336-393, :499-504 (SfcDecomposition
    cut points and rank_for).
"""
from __future__ import annotations

import numpy as np

import oracle as _o


def rust_round(x):
    """f64::round: half away from zero (exact: x - trunc(x) is exact)."""
    x = np.asarray(x, dtype=np.float64)
    t = np.trunc(x)
    return t + np.where(np.abs(x - t) >= 0.5, np.sign(x), 0.0)


def minimum_image_scalar(dx, box):
    half = box * 0.5
    d = dx - box * rust_round(dx / box)
    d = np.where(d > half, d - box, d)
    return np.where(d < -half, d + box, d)


def compute_aabb_3d(pos) -> np.ndarray:
    """{xlo, xhi, ylo, yhi, zlo, zhi}; the empty box (+inf, -inf) for no particles."""
    pos = np.asarray(pos, dtype=np.float64).reshape(-1, 3)
    if pos.shape[0] == 0:
        return np.array([np.inf, -np.inf] * 3)
    lo, hi = pos.min(0), pos.max(0)
    return np.array([lo[0], hi[0], lo[1], hi[1], lo[2], hi[2]])


def aabb_is_valid(a) -> bool:
    return bool(a[0] <= a[1] and a[2] <= a[3] and a[4] <= a[5])


def min_dist2_to_aabb_3d_periodic(pos, a, box) -> np.ndarray:
    """Per particle; +inf for an invalid box."""
    pos = np.asarray(pos, dtype=np.float64).reshape(-1, 3)
    if not aabb_is_valid(a):
        return np.full(pos.shape[0], np.inf)
    d2 = np.zeros(pos.shape[0])
    for k in range(3):
        lo, hi = a[2 * k], a[2 * k + 1]
        com = (lo + hi) * 0.5
        half = (hi - lo) * 0.5
        d = minimum_image_scalar(com - pos[:, k], box)
        e = np.maximum(np.abs(d) - half, 0.0)
        d2 = d2 + e * e
    return d2


def is_in_periodic_halo(p, a, width, box) -> bool:
    return bool(min_dist2_to_aabb_3d_periodic(np.asarray(p)[None, :], a, box)[0] < width * width)


def halo_selection(pos_q, aabbs, q, width, box):
    """Indices (in q's order) that rank q sends to each rank r != q."""
    out = {}
    w2 = width * width
    for r, a in enumerate(aabbs):
        if r == q or not aabb_is_valid(a):
            continue
        sel = np.nonzero(min_dist2_to_aabb_3d_periodic(pos_q, a, box) < w2)[0]
        if sel.size:
            out[r] = sel
    return out


def exchange_halos(parts, width, box):
    """parts: per-rank (n_r, 3) positions.  Returns per rank the list of
    (source rank, index array into that rank's particles) in receive order."""
    aabbs = [compute_aabb_3d(p) for p in parts]
    sends = [halo_selection(parts[q], aabbs, q, width, box) for q in range(len(parts))]
    return [[(q, sends[q][r]) for q in range(len(parts)) if r in sends[q]] for r in range(len(parts))]


def fixed_point(pos, box):
    """The 32-bit fixed-point coordinates of positions on the lattice x = q L / 2^32."""
    u = np.mod(np.asarray(pos, dtype=np.float64) / box, 1.0)
    return (np.rint(u * 2.0 ** 32).astype(np.uint64) & np.uint64(0xFFFFFFFF)).astype(np.uint64)


def occupancy_grid(box, width):
    g = np.floor(box / width) if width > 0 else 64.0
    return int(max(1.0, min(64.0, g)))


def occupied_cells(q, g):
    """Boolean g^3 occupancy of particles with fixed-point coordinates q (n, 3)."""
    c = ((np.asarray(q, dtype=np.uint64).reshape(-1, 3) * np.uint64(g)) >> np.uint64(32)).astype(np.int64)
    occ = np.zeros(g ** 3, dtype=bool)
    occ[(c[:, 2] * g + c[:, 1]) * g + c[:, 0]] = True
    return occ


def cells_halo_selection(q_own, occs, rank, width, box):
    """The cell rule of the library's tpm_halo_select_cells for one rank's
    particles (fixed point q_own): per destination rank, the indices within
    `width` (float64 face gaps, width^2 widened by 1e-9) of a cell that rank
    occupies among the 27 around each particle's cell."""
    g = occupancy_grid(box, width)
    q = np.asarray(q_own, dtype=np.uint64).reshape(-1, 3)
    ci = ((q * np.uint64(g)) >> np.uint64(32)).astype(np.int64)
    x = q.astype(np.float64) * (box / 2.0 ** 32)
    cell = box / g
    w2 = width * width * (1.0 + 1e-9)
    sel = {r: np.zeros(q.shape[0], dtype=bool) for r in range(len(occs)) if r != rank}
    for oz in (-1, 0, 1):
        for oy in (-1, 0, 1):
            for ox in (-1, 0, 1):
                gaps = []
                for k, o in enumerate((ox, oy, oz)):
                    if o == 0:
                        gaps.append(np.zeros(q.shape[0]))
                    elif o > 0:
                        gaps.append((ci[:, k] + 1).astype(np.float64) * cell - x[:, k])
                    else:
                        gaps.append(x[:, k] - ci[:, k].astype(np.float64) * cell)
                ok = (gaps[0] * gaps[0] + gaps[1] * gaps[1]) + gaps[2] * gaps[2] < w2
                c = (((ci[:, 2] + oz) % g) * g + (ci[:, 1] + oy) % g) * g + (ci[:, 0] + ox) % g
                for r in sel:
                    sel[r] |= ok & occs[r][c]
    return {r: np.nonzero(m)[0] for r, m in sel.items() if m.any()}


def exchange_halos_cells(qparts, width, box):
    g = occupancy_grid(box, width)
    occs = [occupied_cells(q, g) for q in qparts]
    sends = [cells_halo_selection(qparts[r], occs, r, width, box) for r in range(len(qparts))]
    return [[(q, sends[q][r]) for q in range(len(qparts)) if r in sends[q]] for r in range(len(qparts))]


def distributed_treepm(pos, mass, owner, eps2, g, nm, box, r_split, r_cut_factor, halo="aabb"):
    """Accelerations of every particle under the decomposition `owner` (rank
    of each particle): the serial TreePM's long range plus, per rank, the
    periodic short range over its particles and its halos.  Returns
    (acc, sr, counts, halos) with acc / sr / counts in global order and halos
    the per-rank receive lists of exchange_halos (as global indices)."""
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    mass = np.ascontiguousarray(mass, dtype=np.float64)
    owner = np.asarray(owner)
    n_ranks = int(owner.max()) + 1 if owner.size else 1
    members = [np.nonzero(owner == r)[0] for r in range(n_ranks)]
    r_cut = r_cut_factor * r_split
    if halo == "aabb":
        halos = exchange_halos([pos[m] for m in members], r_cut, box)
    else:
        q = fixed_point(pos, box)
        halos = exchange_halos_cells([q[m] for m in members], r_cut, box)
    lr = _o.treepm(pos, mass, eps2, g, nm, box, r_split, r_cut_factor, parts=True)["lr"]
    sr = np.zeros_like(pos)
    cnt = np.zeros((pos.shape[0], 2), dtype=np.int64)
    halo_global = []
    for r in range(n_ranks):
        hidx = np.concatenate([members[q][i] for q, i in halos[r]]) if halos[r] else np.zeros(0, dtype=np.int64)
        halo_global.append(hidx)
        allidx = np.concatenate([members[r], hidx])
        if members[r].size == 0:
            continue
        s, c = _o.short_range(pos[allidx], mass[allidx], eps2, g, r_split, r_cut, box,
                              targets=np.arange(members[r].size), counts=True)
        sr[members[r]] = s
        cnt[members[r]] = c
    return lr + sr, sr, cnt, halo_global


def cutpoints(sorted_keys, n_ranks):
    """build_with_bbox_and_kind cut points (sfc.rs:370-377)."""
    n = len(sorted_keys)
    if n == 0:
        return np.full(n_ranks - 1, np.iinfo(np.uint64).max // np.uint64(n_ranks), dtype=np.uint64)
    return np.array([sorted_keys[min(r * n // n_ranks, n - 1)] for r in range(1, n_ranks)], dtype=np.uint64)


def rank_for(key, cuts, n_ranks):
    """sfc.rs:499-504 with a plain binary search."""
    lo, hi = 0, len(cuts)
    while lo < hi:
        mid = (lo + hi) // 2
        if cuts[mid] < key:
            lo = mid + 1
        elif cuts[mid] > key:
            hi = mid
        else:
            return min(mid + 1, n_ranks - 1)
    return min(lo, n_ranks - 1)


def spread_bits(x):
    """sfc.rs:39-47: the 21 low bits of x to every third bit."""
    x = np.asarray(x, dtype=np.uint64) & np.uint64(0x1FFFFF)
    for sh, m in ((32, 0x1F00000000FFFF), (16, 0x1F0000FF0000FF), (8, 0x100F00F00F00F00F),
                  (4, 0x10C30C30C30C30C3), (2, 0x1249249249249249)):
        x = (x | (x << np.uint64(sh))) & np.uint64(m)
    return x


def morton_keys(pos, bbox6):
    """particle_morton (sfc.rs:54-81) over the box {xlo, xhi, ylo, yhi, zlo, zhi}."""
    pos = np.asarray(pos, dtype=np.float64).reshape(-1, 3)
    eps = np.finfo(np.float64).eps
    c = []
    for k in range(3):
        lo, hi = bbox6[2 * k], bbox6[2 * k + 1]
        ln = max(hi - lo, eps)
        v = np.clip((pos[:, k] - lo) / ln, 0.0, 1.0 - eps)
        c.append((v * 2097152.0).astype(np.uint64))
    return spread_bits(c[0]) | (spread_bits(c[1]) << np.uint64(1)) | (spread_bits(c[2]) << np.uint64(2))
