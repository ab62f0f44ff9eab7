"""Domain-decomposed TreePM on the CPU: the oracle pinned by the reference's
own SR-SFC tests, the driver's SFC helpers against the oracle, and the
exchange layer with two gloo ranks.

Pins (crates/gadget-ng-treepm/tests/sr_sfc_geometry.rs,
crates/gadget-ng-physics/tests/treepm_sr_sfc.rs, the unit tests of
crates/gadget-ng-treepm/src/distributed.rs): the periodic halo rule's three
cases and compute_aabb_3d; the short range over local + halo particles pulls
across a domain border, across the periodic diagonal and through the minimum
image; an isolated particle feels nothing; at P = 1 there are no halos and the
result is the serial one.
"""
import os
import socket
import sys

import numpy as np
import pytest

from conftest import REPO, oracle


def dom():
    import domain_oracle
    return domain_oracle


def _sr(local, halo, r_split=0.1, eps2=1e-6, box=1.0):
    pos = np.array(list(local) + list(halo), dtype=np.float64).reshape(-1, 3)
    mass = np.ones(pos.shape[0])
    return oracle().short_range(pos, mass, eps2, 1.0, r_split, 5.0 * r_split, box, targets=np.arange(len(local)))


def test_halo_rule_pins():
    d = dom()
    a0 = np.array([0.0, 0.5, 0.0, 0.5, 0.0, 0.5])
    assert d.is_in_periodic_halo([0.95, 0.95, 0.95], a0, 0.1, 1.0)   # periodic diagonal, d = 0.087
    assert d.is_in_periodic_halo([0.95, 0.25, 0.25], a0, 0.1, 1.0)   # periodic x border, d = 0.05
    assert not d.is_in_periodic_halo([0.75, 0.75, 0.75], a0, 0.1, 1.0)
    a = d.compute_aabb_3d([[0.1, 0.2, 0.3], [0.4, 0.45, 0.48]])
    assert d.aabb_is_valid(a) and abs(a[0] - 0.1) < 1e-12 and abs(a[1] - 0.4) < 1e-12
    e = d.compute_aabb_3d(np.zeros((0, 3)))
    assert not d.aabb_is_valid(e)
    assert np.all(np.isinf(d.min_dist2_to_aabb_3d_periodic([[0.5, 0.5, 0.5]], e, 1.0)))


def test_rust_round_and_minimum_image():
    d = dom()
    x = np.array([0.5, -0.5, 1.5, -2.5, 0.49999999999999994, -0.49999999999999994, 2.4999999999999996])
    assert list(d.rust_round(x)) == [1.0, -1.0, 2.0, -3.0, 0.0, -0.0, 2.0]
    assert d.minimum_image_scalar(np.array([0.9]), 1.0)[0] == pytest.approx(-0.1)
    assert d.minimum_image_scalar(np.array([-0.6]), 1.0)[0] == pytest.approx(0.4)


def test_short_range_over_local_and_halo_pins():
    # border: local x = 0.48, halo x = 0.52 -> pulled towards +x
    out = _sr([[0.48, 0.5, 0.5]], [[0.52, 0.5, 0.5]])
    assert out[0, 0] > 0.0
    # periodic diagonal: halo image at (-0.01, -0.01, -0.01)
    out = _sr([[0.01, 0.01, 0.01]], [[0.99, 0.99, 0.99]])
    assert np.all(out[0] < 0.0)
    # minimum image in z
    out = _sr([[0.5, 0.5, 0.05]], [[0.5, 0.5, 0.95]])
    assert out[0, 2] < 0.0
    # no gaps: the rightmost local particle feels the halo next to it
    local = [[i * 0.08, 0.5, 0.5] for i in range(5)]
    halo = [[0.4 + i * 0.08, 0.5, 0.5] for i in range(5)]
    out = _sr(local, halo)
    assert np.linalg.norm(out[4]) > 0.0
    # an isolated particle feels nothing (no self force)
    assert np.linalg.norm(_sr([[0.5, 0.5, 0.5]], [])[0]) < 1e-14


def _box(n_side=10, seed=3):
    rng = np.random.default_rng(seed)
    g = (np.arange(n_side) + 0.5) / n_side
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    pos = np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1) + rng.normal(0, 0.2 / n_side, (n_side ** 3, 3))
    pos = np.mod(pos, 1.0)
    q = np.floor(pos * 2.0 ** 32).astype(np.uint64) & 0xFFFFFFFF
    return q.astype(np.float64) * (1.0 / 2.0 ** 32), np.full(n_side ** 3, 1.0 / n_side ** 3)


def test_p1_has_no_halos_and_is_serial():
    pos, mass = _box(8)
    nm, rs = 16, 1.25 / 16
    acc, sr, cnt, halos = dom().distributed_treepm(pos, mass, np.zeros(pos.shape[0], dtype=int), 1e-6, 1.0, nm,
                                                   1.0, rs, 4.5)
    assert halos[0].size == 0
    ref = oracle().treepm(pos, mass, 1e-6, 1.0, nm, 1.0, rs, 4.5, parts=True, counts=True)
    np.testing.assert_array_equal(sr, ref["sr"])
    np.testing.assert_array_equal(cnt, ref["counts"])
    np.testing.assert_allclose(acc, ref["acc"], rtol=1e-13, atol=0)


def _sfc_owner(pos, n_ranks):
    keys, _ = oracle().hilbert_keys(pos)
    cuts = dom().cutpoints(np.sort(keys), n_ranks)
    return np.array([dom().rank_for(k, cuts, n_ranks) for k in keys]), keys, cuts


def test_halos_cover_every_pair_within_r_cut():
    """sr_sfc_no_geometric_gaps at scale: every cross-rank pair closer than
    r_cut (periodic) is in the receiving rank's halo."""
    pos, mass = _box(10, 5)
    owner, _, _ = _sfc_owner(pos, 3)
    r_cut = 4.5 * 1.25 / 16
    _, _, _, halos = dom().distributed_treepm(pos, mass, owner, 1e-6, 1.0, 16, 1.0, 1.25 / 16, 4.5)
    for r in range(3):
        mine = np.nonzero(owner == r)[0]
        other = np.nonzero(owner != r)[0]
        d = dom().minimum_image_scalar(pos[mine][:, None, :] - pos[other][None, :, :], 1.0)
        near = other[np.any(np.sum(d * d, axis=2) < r_cut * r_cut, axis=0)]
        assert set(near) <= set(halos[r].tolist())
        assert len(set(halos[r].tolist())) == halos[r].size  # one copy per particle


def test_two_ranks_close_to_serial():
    """The short range differs from the serial one only where a rank's own
    tree takes other monopoles (distributed.rs builds it from local + halo)."""
    pos, mass = _box(10, 7)
    nm, rs = 16, 1.25 / 16
    owner, _, _ = _sfc_owner(pos, 2)
    acc, _, cnt, _ = dom().distributed_treepm(pos, mass, owner, 1e-6, 1.0, nm, 1.0, rs, 4.5)
    ref = oracle().treepm(pos, mass, 1e-6, 1.0, nm, 1.0, rs, 4.5, counts=True)
    rel = np.linalg.norm(acc - ref["acc"], axis=1) / np.linalg.norm(ref["acc"], axis=1)
    assert np.sqrt(np.mean(rel ** 2)) < 1e-2
    assert cnt.sum() > 0


def test_four_ranks_tail_comes_from_shifted_root_cubes():
    """Where the decomposed short range departs from the serial one at P = 4.
    Each rank builds its octree over its own + halo particles
    (distributed.rs:60-145), whose bounding cube is the root cell.  A rank
    whose local + halo particles span the serial root cube has the serial
    cells at every depth and reproduces the serial forces to the r_cut
    boundary's level (only nodes cut by the halo edge change their COM); a
    rank whose cube differs has every cell shifted, so its monopoles group
    other particles, including monopoles that hold the target, and some of
    its particles feel relative differences of order one.  Morton domains of
    a perturbed 20^3 lattice: seed 7 has one such rank (rank 0), seeds 8 and
    9 none."""
    nm, rs, P = 16, 1.25 / 16, 4
    for seed, shifted in ((7, {0}), (8, set()), (9, set())):
        pos, mass = _box(20, seed)
        keys = dom().morton_keys(pos, np.array([0.0, 0.0, 0.0, 1.0, 1.0, 1.0]))
        cuts = dom().cutpoints(np.sort(keys), P)
        owner = np.array([dom().rank_for(k, cuts, P) for k in keys])
        acc, _, _, halos = dom().distributed_treepm(pos, mass, owner, 1e-6, 1.0, nm, 1.0, rs, 4.5)
        ref = oracle().treepm(pos, mass, 1e-6, 1.0, nm, 1.0, rs, 4.5)["acc"]
        rel = np.linalg.norm(acc - ref, axis=1) / np.linalg.norm(ref, axis=1)
        serial = oracle().octree(pos, mass)
        found = set()
        for r in range(P):
            mine = np.nonzero(owner == r)[0]
            tree = oracle().octree(pos[np.concatenate([mine, halos[r]])], mass[np.concatenate([mine, halos[r]])])
            same = np.array_equal(tree["root_center"], serial["root_center"]) and \
                tree["root_half"] == serial["root_half"]
            if same:
                assert rel[mine].max() < 5e-5, (seed, r, rel[mine].max())
            else:
                found.add(r)
                assert rel[mine].max() > 1e-2, (seed, r, rel[mine].max())
        assert found == shifted, (seed, found)


def test_driver_sfc_helpers_match_oracle():
    from treepm import distributed as D
    rng = np.random.default_rng(1)
    for n, P in ((0, 3), (1, 2), (7, 4), (1000, 8), (999, 3)):
        keys = np.unique(rng.integers(0, 2 ** 63, n, dtype=np.uint64)) if n else np.zeros(0, dtype=np.uint64)
        sk = np.sort(keys)
        cuts = D.cutpoints_from_keys(sk, P)
        np.testing.assert_array_equal(cuts, dom().cutpoints(sk, P))
        probe = np.concatenate([keys, cuts, cuts + np.uint64(1)]) if n else cuts
        got = D.rank_for(probe, cuts, P)
        want = np.array([dom().rank_for(k, cuts, P) for k in probe], dtype=np.int64)
        np.testing.assert_array_equal(got, want)
    assert D.union_bbox([np.array([np.inf, -np.inf] * 3)]).tolist() == [0.0] * 6
    u = D.union_bbox([np.array([0.1, 0.2, 0.3, 0.4, 0.5, 0.6]), np.array([0.0, 0.1, 0.35, 0.9, 0.2, 0.3]),
                      np.array([np.inf, -np.inf] * 3)])
    assert u.tolist() == [0.0, 0.2, 0.3, 0.9, 0.2, 0.6]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _exchange_rank(rank, world, port, parts, width, q):
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    sys.path.insert(0, os.path.join(REPO, "gadget-ng_b200"))
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        from treepm.distributed import _Exchange
        import domain_oracle as d
        ex = _Exchange(None, torch.device("cpu"))
        mine = parts[rank]
        aabbs = ex.allgather_f64(d.compute_aabb_3d(mine))
        sel = d.halo_selection(mine, aabbs, rank, width, 1.0)
        counts = np.array([sel[r].size if r in sel else 0 for r in range(world)], dtype=np.int64)
        order = np.concatenate([sel[r] for r in range(world) if r in sel]) if sel else np.zeros(0, dtype=np.int64)
        send = torch.from_numpy(np.ascontiguousarray(mine[order]).view(np.uint8).reshape(-1).copy())
        rc = ex.alltoall_counts(counts)
        recv = ex.alltoallv_bytes(send, counts * 24, rc * 24).numpy()
        got = recv[:int(rc.sum()) * 24].view(np.float64).reshape(-1, 3)
        t = torch.full((5,), float(rank + 1))
        ex.allreduce_sum_(t)
        words = ex.allgather_u32(np.array([0xFFFFFFFF - rank, rank, 1 << 31], dtype=np.uint32))
        q.put((rank, got, aabbs, t.numpy(), words))
    finally:
        dist.destroy_process_group()


def test_exchange_layer_two_gloo_ranks():
    """exchange_halos_3d_periodic over the driver's collectives (allgather,
    count all-to-all, alltoallv of records, all-reduce) equals the oracle's
    all-in-one exchange; the uint32 allgather of the cell rule keeps every bit."""
    import torch.multiprocessing as mp
    pos, _ = _box(8, 11)
    owner, _, _ = _sfc_owner(pos, 2)
    parts = [pos[owner == r] for r in range(2)]
    width = 0.15
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_exchange_rank, args=(r, 2, port, parts, width, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = dict()
    for _ in range(2):
        r, got, aabbs, t, words = q.get(timeout=120)
        res[r] = (got, aabbs, t, words)
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    want = dom().exchange_halos(parts, width, 1.0)
    for r in range(2):
        got, aabbs, t, words = res[r]
        assert words.dtype == np.uint32 and words.tolist() == [[0xFFFFFFFF, 0, 1 << 31], [0xFFFFFFFE, 1, 1 << 31]]
        exp = np.concatenate([parts[s][i] for s, i in want[r]]) if want[r] else np.zeros((0, 3))
        np.testing.assert_array_equal(got, exp)
        np.testing.assert_array_equal(aabbs, np.stack([dom().compute_aabb_3d(p) for p in parts]))
        assert np.all(t == 3.0)


def test_morton_keys_pins():
    """morton_zero_maps_to_zero, morton_order_preserves_locality and
    spread_bits_and_back of crates/gadget-ng-parallel/src/sfc.rs."""
    d = dom()
    unit = [0.0, 1.0, 0.0, 1.0, 0.0, 1.0]
    k = d.morton_keys([[0.0, 0.0, 0.0], [0.1, 0.1, 0.1], [0.15, 0.12, 0.11], [0.9, 0.9, 0.9]], unit)
    assert k[0] == 0 and k[1] < k[3] and k[2] < k[3]
    for x in (0, 1, 42, 1048575, (1 << 21) - 1):
        s = int(d.spread_bits(np.array([x], dtype=np.uint64))[0])
        assert s & ~0x1249249249249249 == 0
        # every third bit of s, gathered, is x again
        assert sum(((s >> (3 * i)) & 1) << i for i in range(21)) == x
    # Z order: the top three key bits are the octant (z, y, x)
    k = d.morton_keys([[0.7, 0.2, 0.6]], unit)[0]
    assert int(k) >> 60 == 0b101


def test_cells_halo_covers_every_pair_and_is_smaller():
    """The cell rule (tpm_halo_select_cells) keeps every cross-rank pair within
    r_cut and, on Morton domains, sends fewer particles than the AABB rule."""
    from treepm import distributed as D
    pos, mass = _box(12, 9)
    keys = dom().morton_keys(pos, dom().compute_aabb_3d(pos))
    P = 4
    owner = D.rank_for(keys, D.cutpoints_from_keys(np.sort(keys), P), P)
    r_cut = 4.5 * 1.25 / 48
    q = dom().fixed_point(pos, 1.0)
    assert np.array_equal(q.astype(np.float64) * 2.0 ** -32, pos)
    cells = dom().exchange_halos_cells([q[owner == r] for r in range(P)], r_cut, 1.0)
    aabb = dom().exchange_halos([pos[owner == r] for r in range(P)], r_cut, 1.0)
    members = [np.nonzero(owner == r)[0] for r in range(P)]
    n_cells = n_aabb = 0
    for r in range(P):
        got = np.concatenate([members[s][i] for s, i in cells[r]]) if cells[r] else np.zeros(0, dtype=int)
        n_cells += got.size
        n_aabb += sum(i.size for _, i in aabb[r])
        other = np.nonzero(owner != r)[0]
        d = dom().minimum_image_scalar(pos[members[r]][:, None, :] - pos[other][None, :, :], 1.0)
        near = other[np.any(np.sum(d * d, axis=2) < r_cut * r_cut, axis=0)]
        assert set(near) <= set(got.tolist())
        assert len(set(got.tolist())) == got.size
    assert n_cells < n_aabb
