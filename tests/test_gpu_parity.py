"""Parity of the sm_100a library with the oracle, through the C ABI.

Bit-exact: CIC cell indices, Hilbert keys and their (key, index) order, the
octree node set with float64 mass and centre of mass, and the number of
short-range interactions (leaf pairs + monopoles) each walk evaluates.
Floating point: accelerations within 1e-5 rms relative force error (the
TreePM tolerance of the target) — FP32 pair arithmetic and FP32 FFTs against
the float64 reference restatement.
"""
import numpy as np
import pytest

from conftest import oracle

pytestmark = pytest.mark.gpu

RMS_TOL = 1e-5


def treepm():
    import treepm as t
    return t


def rel_err(a, b):
    """Per-particle |a - b| / |b| (rms and 99th percentile)."""
    d = np.linalg.norm(a - b, axis=1)
    n = np.linalg.norm(b, axis=1)
    r = d / np.maximum(n, 1e-300)
    return float(np.sqrt(np.mean(r * r))), float(np.percentile(r, 99))


def global_rel(a, b):
    return float(np.sqrt(np.sum((a - b) ** 2) / np.sum(b ** 2)))


def small_box(n_side=16, box=100.0, rms=1.0, seed=11):
    from treepm import ics
    return ics.lattice_box(n_side, box, rms, seed)


def clustered_small(n_side=16, box=100.0, seed=5):
    from treepm import ics
    return ics.clustered_box(n_side, box, 0.3, 6, min_halo=20, max_halo=200, r_min=0.3, r_max=1.5, seed=seed)


# ---------------------------------------------------------------------------
def test_cic_cells_bit_exact():
    t = treepm()
    b = small_box(32, 100.0, 1.0, seed=2)
    pos = b.positions()
    s = t.PmSolver(32, b.box_size)
    s.set_particles(pos, b.mass)
    assert np.array_equal(s.cic_cells(b.n), oracle().cic_cells(pos, b.box_size, 32))
    # a non power-of-two box length (inv_cell is not exact)
    s2 = t.PmSolver(64, 77.0)
    x = np.random.default_rng(3).uniform(0, 77.0, (5000, 3))
    s2.set_particles(x, np.ones(5000))
    got = s2.cic_cells(5000)
    p, _, _ = s2.get_state(5000, vel=False, acc=False)
    assert np.array_equal(got, oracle().cic_cells(p, 77.0, 64))


def test_hilbert_keys_and_order_bit_exact():
    t = treepm()
    for b in (small_box(16, 100.0, 1.0, 4), clustered_small(16, 200.0, 6)):
        s = t.TreePmSolver(32, b.box_size, 0.0)
        s.set_particles(b.positions(), b.mass)
        keys, order = s.hilbert_keys(b.n)
        rk, ro = oracle().hilbert_keys(b.positions())
        assert np.array_equal(keys, rk)
        assert np.array_equal(order, ro)


def _node_table(paths_hi, paths_lo, depth):
    return {(int(d), int(h), int(l)): i for i, (d, h, l) in enumerate(zip(depth, paths_hi, paths_lo))}


@pytest.mark.parametrize("kind", ["lattice", "clustered"])
def test_octree_nodes_bit_exact(kind):
    t = treepm()
    b = small_box(16, 100.0, 1.0, 8) if kind == "lattice" else clustered_small(16, 100.0, 9)
    pos = b.positions()
    s = t.TreePmSolver(32, b.box_size, 0.0)
    s.set_particles(pos, b.mass)
    s.compute_forces(1e-4, 1.0)
    dev = s.export_tree()
    ref = oracle().octree(pos, b.mass)
    keep, rh, rl = oracle().octree_paths(ref)
    # non-empty reference nodes: internal (particle_idx < 0) and leaves
    ridx = np.nonzero(keep)[0]
    assert len(ridx) == len(dev["depth"])
    dt = _node_table(dev["path_hi"], dev["path_lo"], dev["depth"])
    for i in ridx:
        key = (int(ref["depth"][i]), int(rh[i]), int(rl[i]))
        j = dt[key]
        assert dev["mass"][j] == ref["mass"][i]
        assert np.array_equal(dev["com"][j], ref["com"][i])
        np.testing.assert_array_equal(dev["quad"][j], ref["quad"][i])
        pi = int(ref["particle_idx"][i])
        assert int(dev["particle"][j]) == pi


def _sr_parity(b, nm, periodic=True, r_cut_factor=4.5, eps_frac=30.0):
    t = treepm()
    pos = b.positions()
    n_side = round(b.n ** (1 / 3))
    eps = b.box_size / n_side / eps_frac
    rs = 1.25 * b.box_size / nm
    s = t.TreePmSolver(nm, b.box_size, rs, r_cut_factor=r_cut_factor, periodic_walk=periodic)
    s.set_particles(pos, b.mass)
    g = 1.0
    s.compute_forces(eps * eps, g)
    lr, sr = s.force_parts(b.n)
    st = s.stats()
    ref_sr, cnt = oracle().short_range(pos, b.mass, eps * eps, g, rs, r_cut_factor * rs, b.box_size,
                                       periodic=periodic, counts=True)
    return s, sr, ref_sr, cnt, st


@pytest.mark.parametrize("kind", ["lattice", "clustered"])
def test_short_range_parity_and_interaction_set(kind):
    b = small_box(24, 100.0, 1.0, 12) if kind == "lattice" else clustered_small(24, 100.0, 13)
    s, sr, ref, cnt, st = _sr_parity(b, 32)
    per = s.interaction_counts(b.n)
    bad = np.nonzero(np.any(per != cnt, axis=1))[0]
    assert len(bad) == 0, (len(bad), bad[:8], per[bad[:8]], cnt[bad[:8]])
    assert st["leaf_pairs"] == int(cnt[:, 0].sum())
    assert st["monopoles"] == int(cnt[:, 1].sum())
    assert global_rel(sr, ref) < RMS_TOL
    rms, p99 = rel_err(sr, ref)
    assert rms < 1e-4, (rms, p99)


def test_monopole_with_centre_next_to_its_target_counts_once():
    """A terminal cell holding the target and one neighbour two fixed-point
    quanta away is a monopole whose centre of mass lies one quantum from the
    target (the reference takes it, short_range.rs:316-323).  Its float
    distance falls below the walk's coincidence threshold, so the float64
    test decides it, and it must enter the sum and the count exactly once."""
    import types
    t = treepm()
    L, ns, nm = 100.0, 16, 16
    g = (np.arange(ns) + 0.5) * (L / ns)
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    q = np.round(np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1) / L * 2.0 ** 32)
    k = 5 * ns * ns + 7 * ns + 9
    q = np.vstack([q, q[k] + np.array([2.0, 0.0, 0.0])])  # the neighbour: two quanta along x
    pos = q * (L / 2.0 ** 32)
    b = types.SimpleNamespace(positions=lambda: pos, mass=np.full(pos.shape[0], 1.0 / pos.shape[0]), n=pos.shape[0],
                              box_size=L)
    s, sr, ref, cnt, st = _sr_parity(b, nm)
    per = s.interaction_counts(b.n)
    for i in (k, b.n - 1):
        assert cnt[i, 1] >= 1, cnt[i]
        assert np.array_equal(per[i], cnt[i]), (i, per[i], cnt[i])
    assert np.array_equal(per, cnt)
    # an unperturbed lattice: each target's ~740 pair terms cancel to a net
    # force far below any one of them, so FP32 rounding of the sums weighs
    # more against the net force than in the perturbed boxes (RMS_TOL there)
    assert global_rel(sr, ref) < 5 * RMS_TOL


def test_short_range_aperiodic_parity():
    b = small_box(16, 100.0, 1.0, 21)
    s, sr, ref, cnt, st = _sr_parity(b, 32, periodic=False)
    assert st["leaf_pairs"] == int(cnt[:, 0].sum())
    assert st["monopoles"] == int(cnt[:, 1].sum())
    assert global_rel(sr, ref) < RMS_TOL


def test_pm_parity():
    t = treepm()
    b = small_box(32, 100.0, 0.2, 1)
    pos = b.positions()
    s = t.PmSolver(32, b.box_size)
    idx = np.arange(b.n)
    g = 3.7
    out = s.accelerations_for_indices(pos, b.mass, 0.0, g, idx)
    ref = oracle().pm(pos, b.mass, g, 32, b.box_size)
    rms, p99 = rel_err(out, ref)
    assert rms < RMS_TOL, (rms, p99)


@pytest.mark.parametrize("flags", [(False, False), (True, False), (False, True)])
def test_pm_extension_flags(flags):
    t = treepm()
    deconv, four = flags
    b = small_box(16, 64.0, 0.5, 31)
    pos = b.positions()
    s = t.PmSolver(16, b.box_size, deconvolve_cic=deconv, four_point_gradient=four)
    out = s.accelerations_for_indices(pos, b.mass, 0.0, 1.0, np.arange(b.n))
    of = (oracle().DECONVOLVE_CIC if deconv else 0) | (oracle().FOUR_POINT_GRADIENT if four else 0)
    ref = oracle().pm(pos, b.mass, 1.0, 16, b.box_size, pm_flags=of)
    assert rel_err(out, ref)[0] < RMS_TOL


def test_pm_mesh_matches_oracle_mesh():
    t = treepm()
    b = small_box(16, 32.0, 0.5, 41)
    pos = b.positions()
    s = t.PmSolver(16, b.box_size)
    s.accelerations_for_indices(pos, b.mass, 0.0, 1.0, [0])
    rho, fx, fy, fz = s.mesh()
    ref_rho = oracle().cic_assign(pos, b.mass, b.box_size, 16)
    assert np.max(np.abs(rho - ref_rho)) < 1e-6 * np.max(ref_rho)
    f = oracle().solve_forces(ref_rho, 1.0, 16, b.box_size)
    for got, want in zip((fx, fy, fz), f):
        assert np.sqrt(np.mean((got - want) ** 2)) < 2e-6 * np.sqrt(np.mean(want ** 2))


@pytest.mark.parametrize("layout", ["corner_clump", "sparse", "one_cell"])
def test_deposit_windows_match_oracle(layout):
    """The deposit sums neighbouring particles' corner nodes in a per-warp
    node window before the mesh atomics: a dense clump straddling the corner
    of the periodic box (windows that wrap on every axis), particles spread
    too far for one window (the direct path), and hundreds of particles in one
    cell (whole warps sharing a base cell).  The density equals the
    restatement's CIC (cic.rs:37-93) to float32 rounding."""
    t = treepm()
    rng = np.random.default_rng({"corner_clump": 3, "sparse": 4, "one_cell": 5}[layout])
    L, nm = 32.0, 32
    if layout == "corner_clump":
        pos = np.mod(rng.normal(0.0, 1.5, (6000, 3)), L)
    elif layout == "sparse":
        pos = rng.uniform(0.0, L, (3000, 3))
    else:
        pos = np.mod(np.array([7.3, 19.6, 30.9]) + rng.uniform(0.0, 0.9, (900, 3)), L)
    q = np.floor(pos / L * 2.0 ** 32) % 2.0 ** 32
    pos = q * (L / 2.0 ** 32)
    mass = rng.uniform(0.5, 1.5, pos.shape[0])
    s = t.PmSolver(nm, L)
    s.accelerations_for_indices(pos, mass, 0.0, 1.0, [0])
    rho = s.mesh()[0]
    ref = oracle().cic_assign(pos, mass, L, nm)
    assert np.max(np.abs(rho - ref)) < 2e-6 * np.max(ref), np.max(np.abs(rho - ref)) / np.max(ref)
    assert abs(float(np.sum(rho, dtype=np.float64)) - float(np.sum(ref))) < 1e-5 * float(np.sum(ref))


@pytest.mark.parametrize("kind", ["lattice", "clustered"])
def test_treepm_parity(kind):
    t = treepm()
    b = small_box(32, 100.0, 1.0, 51) if kind == "lattice" else clustered_small(32, 100.0, 52)
    pos = b.positions()
    nm = 32
    eps = b.box_size / 32 / 30
    rs = 1.25 * b.box_size / nm
    s = t.TreePmSolver(nm, b.box_size, rs, r_cut_factor=4.5)
    g = 2.5
    idx = np.arange(b.n)
    out = s.accelerations_for_indices(pos, b.mass, eps * eps, g, idx)
    ref = oracle().treepm(pos, b.mass, eps * eps, g, nm, b.box_size, rs, 4.5)["acc"]
    rms, p99 = rel_err(out, ref)
    assert rms < RMS_TOL, (rms, p99)


def test_index_subset_and_order():
    t = treepm()
    b = small_box(16, 100.0, 1.0, 61)
    pos = b.positions()
    s = t.TreePmSolver(16, b.box_size)
    full = s.accelerations_for_indices(pos, b.mass, 1e-3, 1.0, np.arange(b.n))
    idx = np.array([5, 0, 4095, 17, 5])
    sub = s.accelerations_for_indices(pos, b.mass, 1e-3, 1.0, idx)
    # float atomics in the mass deposit make repeated calls agree to rounding only
    np.testing.assert_allclose(sub, full[idx], rtol=1e-5, atol=0)
    assert np.array_equal(sub[0], sub[4])


def test_known_answer_pair_across_boundary():
    """minimum_image.rs:187-221 through the device path."""
    t = treepm()
    box, r_split, eps2, g = 1.0, 0.05, 1e-8, 1.0
    pos = np.array([[0.0, 0.0, 0.05], [0.0, 0.0, 0.95]])
    s = t.TreePmSolver(8, box, r_split)
    s.set_particles(pos, np.ones(2))
    s.compute_forces(eps2, g)
    _, sr = s.force_parts(2)
    ref = oracle().short_range(pos, np.ones(2), eps2, g, r_split, 5 * r_split, box)
    assert abs(sr[0, 2] - ref[0, 2]) <= 1e-6 * abs(ref[0, 2])
    assert abs(sr[0, 0]) < 1e-12 and abs(sr[0, 1]) < 1e-12


def test_single_and_two_particles():
    t = treepm()
    s = t.TreePmSolver(8, 1.0, 0.05)
    out = s.accelerations_for_indices(np.array([[0.5, 0.5, 0.5]]), np.ones(1), 1e-6, 1.0, [0])
    assert np.all(np.isfinite(out)) and np.linalg.norm(out) < 1e-6
    pos = np.array([[0.5, 0.5, 0.5], [0.5, 0.5, 0.55]])
    out = s.accelerations_for_indices(pos, np.ones(2), 1e-6, 1.0, [0, 1])
    ref = oracle().treepm(pos, np.ones(2), 1e-6, 1.0, 8, 1.0, 0.05, 5.0)["acc"]
    assert rel_err(out, ref)[0] < RMS_TOL


def test_coincident_positions_rejected():
    t = treepm()
    s = t.TreePmSolver(8, 1.0)
    pos = np.array([[0.25, 0.25, 0.25], [0.5, 0.5, 0.5], [0.5, 0.5, 0.5]])
    with pytest.raises(t.TreePmError) as e:
        s.accelerations_for_indices(pos, np.ones(3), 1e-6, 1.0, [0])
    assert e.value.code == 4


def test_nonfinite_rejected():
    t = treepm()
    s = t.TreePmSolver(8, 1.0)
    pos = np.array([[0.25, 0.25, np.nan], [0.5, 0.5, 0.5]])
    with pytest.raises(t.TreePmError) as e:
        s.accelerations_for_indices(pos, np.ones(2), 1e-6, 1.0, [0])
    assert e.value.code == 9


def test_memory_cap_refuses_cleanly():
    t = treepm()
    # the handle's fixed buffers (the walk's per-warp stacks: 66 MB at 7
    # resident blocks of 4 warps on 148 SMs) fit under the cap; the particle
    # buffers of 128^3 particles do not
    s = t.TreePmSolver(16, 100.0, memory_cap_bytes=128 << 20)
    b = small_box(128, 100.0, 1.0, 71)
    with pytest.raises(t.TreePmError) as e:
        s.accelerations_for_indices(b.positions(), b.mass, 1e-4, 1.0, [0])
    assert e.value.code == 3
    # the handle stays usable for a problem that fits
    small = small_box(8, 100.0, 1.0, 72)
    s2 = t.TreePmSolver(16, 100.0)
    out = s2.accelerations_for_indices(small.positions(), small.mass, 1e-4, 1.0, [0, 1])
    assert np.all(np.isfinite(out))


def test_kdk_step_matches_oracle_two_evaluations():
    """Fused step (cached opening kick) vs leapfrog_cosmo_kdk_step with two force evaluations."""
    t = treepm()
    from treepm import ics
    b = small_box(16, 100.0, 1.0, 81)
    pos = b.positions()
    nm = 16
    phys = ics.physics(b, nm, 0.1)
    a0, a1 = 0.1, 0.102
    dt = ics.time_between(a0, a1)
    drift, kh, kh2 = t.drift_kick_factors(ics.OMEGA_M, ics.OMEGA_L, 1.0, a0, dt)
    s = t.TreePmSolver(nm, b.box_size, phys["r_split"], r_cut_factor=4.5)
    s.set_particles(pos, b.mass)
    s.kdk_step(kh, drift, kh2, phys["eps2"], phys["g"])
    p_dev, v_dev, a_dev = s.get_state(b.n)
    p_ref, v_ref, a_ref = oracle().kdk_step_treepm(pos, np.zeros_like(pos), b.mass, drift, kh, kh2, phys["eps2"],
                                                   phys["g"], nm, b.box_size, phys["r_split"], 4.5)
    assert rel_err(a_dev, a_ref)[0] < 1e-4
    assert rel_err(v_dev, v_ref)[0] < 1e-4
    dp = (p_dev - p_ref + 0.5 * b.box_size) % b.box_size - 0.5 * b.box_size
    assert np.max(np.abs(dp)) < 1e-6 * b.box_size


def test_drift_kick_factors_match_oracle_bitwise():
    t = treepm()
    for a0, dt in ((0.02, 0.001), (0.1, 0.0037), (1.0, 0.05)):
        assert t.drift_kick_factors(0.31, 0.69, 1.0, a0, dt) == oracle().drift_kick_factors(0.31, 0.69, 1.0, a0, dt)


def test_host_kdk_steps_reuse_the_resident_acceleration():
    """Host-buffer steps that hand back the returned state reuse the resident
    closing acceleration: three such steps equal three device-resident steps,
    with one force evaluation per step after the first; a changed state is
    re-encoded and evaluated twice (after the evaluation of the resident
    state that ran while the inputs were checked, which is discarded)."""
    t = treepm()
    from treepm import ics
    b = small_box(16, 100.0, 1.0, 83)
    nm = 16
    phys = ics.physics(b, nm, 0.1)
    a = 0.1
    steps = []
    for _ in range(3):
        dt = ics.time_between(a, a + 0.002)
        steps.append(t.drift_kick_factors(ics.OMEGA_M, ics.OMEGA_L, 1.0, a, dt))
        a += 0.002
    dev = t.TreePmSolver(nm, b.box_size, phys["r_split"], r_cut_factor=4.5)
    dev.set_particles(b.positions(), b.mass)
    for d, k1, k2 in steps:
        dev.kdk_step(k1, d, k2, phys["eps2"], phys["g"])
    p_dev, v_dev, _ = dev.get_state(b.n)
    host = t.TreePmSolver(nm, b.box_size, phys["r_split"], r_cut_factor=4.5)
    pos = np.ascontiguousarray(b.positions())
    vel = np.zeros_like(pos)
    evals = []
    for d, k1, k2 in steps:
        host.kdk_step_host(pos, vel, b.mass, k1, d, k2, phys["eps2"], phys["g"])
        evals.append(host.stats()["force_evaluations"])
    assert evals == [2, 3, 4], evals
    # the same steps as on the device (float atomics of the deposit make the
    # two runs differ in the last bits only)
    assert rel_err(vel, v_dev)[0] < 1e-5
    dp = (pos - p_dev + 0.5 * b.box_size) % b.box_size - 0.5 * b.box_size
    assert np.max(np.abs(dp)) < 1e-6 * b.box_size
    # a perturbed state is not the returned one.  Particle 1 is not among the
    # 256 evenly spaced particles the host compares before it queues any work
    # (indices k n / 256: 0, 16, 32, ... here), so the step runs speculatively
    # on the resident state, the device check rejects it, and the step
    # evaluates twice more; particle 0 is compared on the host, so that state
    # is stepped from the upload at once (two evaluations, nothing discarded).
    # Both match a device step from the same state.
    d, k1, k2 = steps[0]
    before = host.stats()["force_evaluations"]
    for idx, extra in ((1, 3), (0, 2)):
        pos2 = pos.copy()
        vel2 = vel.copy()
        pos2[idx, 0] = (pos2[idx, 0] + 1e-3) % b.box_size
        ref = t.TreePmSolver(nm, b.box_size, phys["r_split"], r_cut_factor=4.5)
        ref.set_particles(pos2, b.mass, vel2)
        ref.kdk_step(k1, d, k2, phys["eps2"], phys["g"])
        p_ref, v_ref, _ = ref.get_state(b.n)
        host.kdk_step_host(pos2, vel2, b.mass, k1, d, k2, phys["eps2"], phys["g"])
        assert host.stats()["force_evaluations"] == before + extra, (idx, host.stats()["force_evaluations"])
        before += extra
        assert rel_err(vel2, v_ref)[0] < 1e-5
        dp = (pos2 - p_ref + 0.5 * b.box_size) % b.box_size - 0.5 * b.box_size
        assert np.max(np.abs(dp)) < 1e-6 * b.box_size
        pos, vel = pos2, vel2  # the next call hands back what this one returned, then perturbs it


def test_host_kdk_step_after_another_call_steps_the_inputs():
    """A device-resident step between two host-buffer steps changes the
    resident state: handing back the earlier outputs must then be stepped from
    those inputs (no speculation on the moved state)."""
    t = treepm()
    from treepm import ics
    b = small_box(16, 100.0, 1.0, 85)
    nm = 16
    phys = ics.physics(b, nm, 0.1)
    d, k1, k2 = t.drift_kick_factors(ics.OMEGA_M, ics.OMEGA_L, 1.0, 0.1, ics.time_between(0.1, 0.102))
    host = t.TreePmSolver(nm, b.box_size, phys["r_split"], r_cut_factor=4.5)
    pos = np.ascontiguousarray(b.positions())
    vel = np.zeros_like(pos)
    host.kdk_step_host(pos, vel, b.mass, k1, d, k2, phys["eps2"], phys["g"])
    p1, v1 = pos.copy(), vel.copy()
    host.kdk_step(k1, d, k2, phys["eps2"], phys["g"])  # the resident state moves on
    ref = t.TreePmSolver(nm, b.box_size, phys["r_split"], r_cut_factor=4.5)
    ref.set_particles(p1, b.mass, v1)
    ref.kdk_step(k1, d, k2, phys["eps2"], phys["g"])
    p_ref, v_ref, _ = ref.get_state(b.n)
    host.kdk_step_host(pos, vel, b.mass, k1, d, k2, phys["eps2"], phys["g"])
    assert rel_err(vel, v_ref)[0] < 1e-5
    dp = (pos - p_ref + 0.5 * b.box_size) % b.box_size - 0.5 * b.box_size
    assert np.max(np.abs(dp)) < 1e-6 * b.box_size


def test_accelerations_with_costs():
    """accelerations_with_costs: the accelerations of accelerations_for_indices
    and, per index, the interactions of its walk (the oracle's counts)."""
    t = treepm()
    b = clustered_small(16, 100.0, 57)
    pos = b.positions()
    nm = 32
    eps = b.box_size / 16 / 30
    rs = 1.25 * b.box_size / nm
    s = t.TreePmSolver(nm, b.box_size, rs, r_cut_factor=4.5)
    idx = np.arange(b.n)[::7][::-1].copy()
    out, costs = s.accelerations_with_costs(pos, b.mass, eps * eps, 1.0, idx)
    # (two evaluations differ in the last bits: the deposit sums with float32 atomics)
    np.testing.assert_allclose(out, s.accelerations_for_indices(pos, b.mass, eps * eps, 1.0, idx), rtol=1e-5,
                               atol=1e-6 * np.abs(out).max())
    ref = oracle().treepm(pos, b.mass, eps * eps, 1.0, nm, b.box_size, rs, 4.5, counts=True)
    np.testing.assert_array_equal(costs, ref["counts"][idx].sum(axis=1).astype(np.uint64))
    assert costs.dtype == np.uint64 and costs.shape == idx.shape
    _, none = s.accelerations_with_costs(pos, b.mass, eps * eps, 1.0, np.zeros(0, dtype=np.int64))
    assert none.size == 0
