"""Domain-decomposed TreePM through the C ABI: two ranks as two processes
that share one GPU, their exchanges over gloo (host staging).  No kernel waits
on another rank's: every cross-rank step is a host collective between the
ranks' force stages.

Parity with the oracle's restatement of the reference's SR-SFC path for the
same decomposition: halo counts and the per-particle interaction sets
bit-exact, accelerations within the serial parity tolerance (1e-5 rms
relative), one KDK step within the serial KDK tolerances, and
exchange_domain_sfc keeping every particle once.
"""
import os
import socket
import sys

import numpy as np
import pytest

from conftest import REPO, oracle

pytestmark = pytest.mark.gpu

NM, BOX, RCF = 64, 100.0, 4.5  # r_cut = 8.8 % of the box: partial halos


def dom():
    import domain_oracle
    return domain_oracle


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rel(a, b):
    r = np.linalg.norm(a - b, axis=1) / np.maximum(np.linalg.norm(b, axis=1), 1e-300)
    return float(np.sqrt(np.mean(r * r)))


def _rank_main(rank, world, port, local, phys, q, halo="aabb", force_only=False, pm="replicated"):
    import torch.distributed as dist
    from datetime import timedelta
    sys.path.insert(0, os.path.join(REPO, "gadget-ng_b200"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    try:
        from treepm.distributed import DomainTreePm
        d = DomainTreePm(NM, BOX, phys["r_split"], r_cut_factor=RCF, device=0, halo=halo, pm=pm)
        pos, vel, mass, gid = local
        d.set_particles(pos, mass, vel, gid=gid)
        d.compute_forces(phys["eps2"], phys["g"])
        _, _, _, acc = d.get_state()
        counts = d.interaction_counts()
        lr, sr = d.force_parts()
        n_halo = d.last_halo_count
        if force_only:
            q.put((rank, dict(acc=acc, counts=counts, sr=sr, n_halo=n_halo)))
            return
        d.kdk_step(phys["kh"], phys["drift"], phys["kh2"], phys["eps2"], phys["g"])
        _, p1, v1, a1 = d.get_state()
        d.redistribute(sample=64)
        d.compute_forces(phys["eps2"], phys["g"])
        g2, p2, _, a2 = d.get_state()
        q.put((rank, dict(acc=acc, counts=counts, sr=sr, n_halo=n_halo, p1=p1, v1=v1, a1=a1, g2=g2, p2=p2, a2=a2)))
    except BaseException as e:  # report instead of leaving the parent waiting
        q.put((rank, repr(e)))
        raise
    finally:
        dist.destroy_process_group()


def _run_ranks(parts, phys, halo="aabb", force_only=False, pm="replicated"):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, len(parts), port, parts[r], phys, q, halo, force_only, pm))
             for r in range(len(parts))]
    for p in procs:
        p.start()
    res = {}
    try:
        for _ in procs:
            r, out = q.get(timeout=600)
            assert isinstance(out, dict), out
            res[r] = out
    finally:
        for p in procs:
            p.join(120)
    assert all(p.exitcode == 0 for p in procs)
    return res


@pytest.fixture(scope="module")
def case():
    from treepm import ics
    b = ics.clustered_box(16, BOX, 0.3, 6, min_halo=20, max_halo=200, r_min=0.3, r_max=1.5, seed=23)
    pos, mass = b.positions(), b.mass
    n = pos.shape[0]
    rng = np.random.default_rng(4)
    vel = rng.normal(0.0, 0.3, (n, 3))
    phys = ics.physics(b, NM, 0.1)
    rs = phys["r_split"] = 1.25 * BOX / NM
    import treepm
    a0, a1 = 0.1, 0.102
    drift, kh, kh2 = treepm.drift_kick_factors(ics.OMEGA_M, ics.OMEGA_L, 1.0, a0, ics.time_between(a0, a1))
    phys.update(drift=drift, kh=kh, kh2=kh2)
    # Morton domains (the reference's Hilbert keys give domains spanning the
    # box, whose halos hold every particle)
    keys = dom().morton_keys(pos, dom().compute_aabb_3d(pos))
    cuts = dom().cutpoints(np.sort(keys), 2)
    owner = np.array([dom().rank_for(k, cuts, 2) for k in keys])
    gids = [np.nonzero(owner == r)[0] for r in range(2)]
    parts = [(pos[g], vel[g], mass[g], g) for g in gids]
    res = _run_ranks(parts, phys)
    cells = _run_ranks(parts, phys, halo="cells", force_only=True)
    slab = _run_ranks(parts, phys, pm="slab")
    return dict(pos=pos, vel=vel, mass=mass, owner=owner, gids=gids, phys=phys, res=res, cells=cells, slab=slab)


def test_domain_forces_and_interaction_sets_match_oracle(case):
    c = case
    ph = c["phys"]
    acc, sr, cnt, halos = dom().distributed_treepm(c["pos"], c["mass"], c["owner"], ph["eps2"], ph["g"], NM, BOX,
                                                   ph["r_split"], RCF)
    for r in range(2):
        out, g = c["res"][r], c["gids"][r]
        assert 0 < out["n_halo"] == halos[r].size < c["gids"][1 - r].size  # a partial halo
        np.testing.assert_array_equal(out["counts"], cnt[g])
        assert _rel(out["acc"], acc[g]) < 1e-5
        assert np.sqrt(np.sum((out["sr"] - sr[g]) ** 2) / np.sum(sr[g] ** 2)) < 1e-5


def test_domain_kdk_step_matches_oracle(case):
    c = case
    ph = c["phys"]
    args = (c["mass"], c["owner"], ph["eps2"], ph["g"], NM, BOX, ph["r_split"], RCF)
    a0 = dom().distributed_treepm(c["pos"], *args)[0]
    vh = c["vel"] + a0 * ph["kh"]
    x1 = np.mod(c["pos"] + vh * ph["drift"], BOX)
    a1 = dom().distributed_treepm(x1, *args)[0]
    v1 = vh + a1 * ph["kh2"]
    for r in range(2):
        out, g = c["res"][r], c["gids"][r]
        assert _rel(out["a1"], a1[g]) < 1e-4
        assert _rel(out["v1"], v1[g]) < 1e-4
        dp = (out["p1"] - x1[g] + 0.5 * BOX) % BOX - 0.5 * BOX
        assert np.max(np.abs(dp)) < 1e-6 * BOX


def test_redistribute_keeps_every_particle_once(case):
    c = case
    g = np.concatenate([c["res"][r]["g2"] for r in range(2)])
    assert np.array_equal(np.sort(g), np.arange(c["pos"].shape[0]))
    # the moved state is the stepped state
    p1 = np.zeros_like(c["pos"])
    for r in range(2):
        p1[c["gids"][r]] = c["res"][r]["p1"]
    for r in range(2):  # positions travel as float64 and are re-encoded: at most one fixed-point quantum
        dp = (c["res"][r]["p2"] - p1[c["res"][r]["g2"]] + 0.5 * BOX) % BOX - 0.5 * BOX
        assert np.max(np.abs(dp)) <= BOX * 2.0 ** -31
    # and the force after the move is the oracle's for the new decomposition
    owner = np.zeros(c["pos"].shape[0], dtype=int)
    for r in range(2):
        owner[c["res"][r]["g2"]] = r
    ph = c["phys"]
    acc = dom().distributed_treepm(p1, c["mass"], owner, ph["eps2"], ph["g"], NM, BOX, ph["r_split"], RCF)[0]
    for r in range(2):
        assert _rel(c["res"][r]["a2"], acc[c["res"][r]["g2"]]) < 1e-5


def test_sfc_keys_bit_exact():
    """tpm_sfc_keys: particle_hilbert over the positions' bounding box equals
    the oracle's Hilbert keys; particle_morton equals the restatement for that
    box and for a wider one."""
    import ctypes as C
    import treepm
    from treepm import ics
    b = ics.clustered_box(16, BOX, 0.3, 6, min_halo=20, max_halo=200, r_min=0.3, r_max=1.5, seed=31)
    pos = b.positions()
    s = treepm.TreePmSolver(NM, BOX, 1.25 * BOX / NM)
    s.set_particles(pos, b.mass)
    L = s._h._lib
    for bbox in (dom().compute_aabb_3d(pos), np.array([0.0, BOX, -1.0, BOX + 3.0, 0.5, BOX])):
        for kind in (0, 1):
            keys = np.empty(pos.shape[0], dtype=np.uint64)
            bb = np.ascontiguousarray(bbox, dtype=np.float64)
            assert L.tpm_sfc_keys(s._h.h, bb.ctypes.data_as(C.c_void_p), kind, keys.ctypes.data_as(C.c_void_p)) == 0
            if kind == 1:
                np.testing.assert_array_equal(keys, dom().morton_keys(pos, bbox))
            elif bbox[1] == pos[:, 0].max():
                np.testing.assert_array_equal(keys, oracle().hilbert_keys(pos)[0])


def test_cell_halo_rule_matches_oracle(case):
    """halo="cells": halo counts and interaction sets bit-exact with the
    restatement of the cell rule, accelerations within 1e-5 rms."""
    c = case
    ph = c["phys"]
    acc, sr, cnt, halos = dom().distributed_treepm(c["pos"], c["mass"], c["owner"], ph["eps2"], ph["g"], NM, BOX,
                                                   ph["r_split"], RCF, halo="cells")
    for r in range(2):
        out, g = c["cells"][r], c["gids"][r]
        assert out["n_halo"] == halos[r].size
        np.testing.assert_array_equal(out["counts"], cnt[g])
        assert _rel(out["acc"], acc[g]) < 1e-5


def test_domain_entry_points_report_misuse():
    """The staged force calls out of order return TPM_ERR_NOT_READY; a halo
    send buffer too small returns TPM_ERR_INVALID_ARGUMENT with the counts
    filled and nothing written; bad rank arguments are refused."""
    import ctypes as C
    import treepm
    from treepm import ics
    b = ics.clustered_box(8, BOX, 0.3, 3, min_halo=20, max_halo=60, r_min=0.3, r_max=1.5, seed=41)
    pos = b.positions()
    s = treepm.TreePmSolver(NM, BOX, 1.25 * BOX / NM, r_cut_factor=RCF)
    s.set_particles(pos, b.mass)
    L, h = s._h._lib, s._h.h
    assert L.tpm_force_short_range(h, 1e-4) == 7
    assert L.tpm_force_end(h, 1.0, 0.0) == 7
    assert L.tpm_force_begin(h) == 0
    assert L.tpm_force_end(h, 1.0, 0.0) == 7
    assert L.tpm_force_short_range(h, 1e-4) == 0
    assert L.tpm_force_end(h, 1.0, 0.0) == 0
    # rank 1 owns the whole box: every particle within r_cut of it goes there
    aabbs = np.ascontiguousarray(np.array([[np.inf, -np.inf] * 3, [0.0, BOX] * 3]).reshape(-1))
    counts = np.zeros(2, dtype=np.int64)
    p = lambda a: a.ctypes.data_as(C.c_void_p)
    assert L.tpm_halo_select(h, p(aabbs), 2, 0, 10.0, p(counts), None, 0) == 0
    assert counts[0] == 0 and counts[1] == b.n
    import torch
    buf = torch.zeros(24 * 4, dtype=torch.uint8, device="cuda")
    assert L.tpm_halo_select(h, p(aabbs), 2, 0, 10.0, p(counts), C.c_void_p(buf.data_ptr()), 4) == 1
    assert counts[1] == b.n and int(buf.sum()) == 0
    assert L.tpm_halo_select(h, p(aabbs), 2, 2, 10.0, p(counts), None, 0) == 1   # rank out of range
    assert L.tpm_halo_select(h, p(aabbs), 65, 0, 10.0, p(counts), None, 0) == 1  # too many ranks


def test_slab_pm_matches_replicated_and_oracle(case):
    """pm="slab": the PM solve split into z slabs with two all-to-all
    transposes (slab_fft.rs:209-330) gives the replicated solve's
    accelerations to float rounding and the restatement's within 1e-5 rms,
    through a KDK step and a redistribution as well."""
    c = case
    ph = c["phys"]
    acc = dom().distributed_treepm(c["pos"], c["mass"], c["owner"], ph["eps2"], ph["g"], NM, BOX, ph["r_split"],
                                   RCF)[0]
    for r in range(2):
        sl, rep, g = c["slab"][r], c["res"][r], c["gids"][r]
        np.testing.assert_array_equal(sl["counts"], rep["counts"])
        assert _rel(sl["acc"], rep["acc"]) < 1e-6
        assert _rel(sl["acc"], acc[g]) < 1e-5
        assert _rel(sl["a1"], rep["a1"]) < 1e-5
        assert _rel(sl["v1"], rep["v1"]) < 1e-5
        assert np.array_equal(np.sort(sl["g2"]), np.sort(rep["g2"]))
        assert _rel(sl["a2"], rep["a2"][np.argsort(rep["g2"])][np.searchsorted(np.sort(rep["g2"]), sl["g2"])]) < 1e-5


def test_slab_pm_refuses_a_mesh_not_divisible_by_the_ranks():
    import ctypes as C
    import treepm
    from treepm import _lib
    s = treepm.TreePmSolver(NM, BOX, 1.25 * BOX / NM, r_cut_factor=RCF)
    b = _lib.TpmSlabBuffers()
    assert s._h._lib.tpm_pm_slab_setup(s._h.h, 0, 3, C.byref(b)) == 1  # 64 planes over 3 ranks
    assert s._h._lib.tpm_pm_slab_setup(s._h.h, 2, 2, C.byref(b)) == 1  # rank out of range
    assert s._h._lib.tpm_pm_slab_forward(s._h.h) == 7                  # not set up
    assert s._h._lib.tpm_pm_slab_setup(s._h.h, 1, 4, C.byref(b)) == 0
    assert b.planes == NM // 4 and b.slab_cells == NM * NM * NM // 4 and b.mesh_cells == NM ** 3
    s.close()
