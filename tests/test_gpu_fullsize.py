"""Parity at the workload sizes the benchmark uses.

At these sizes the oracle builds the full insertion octree and PM mesh but
walks a seeded subsample of targets: the device's accelerations at those
targets must be within 1e-5 rms relative error, and the device's per-particle
interaction counts must equal the oracle's exactly.  Size-independent checks
cover every particle: finite forces and the mass deposit's total.
"""
import numpy as np
import pytest

from conftest import oracle

pytestmark = pytest.mark.gpu


def _run(box, mesh, n_targets, seed):
    import treepm
    from treepm import accuracy, ics
    phys = ics.physics(box, mesh, 0.1)
    s = treepm.TreePmSolver(mesh, box.box_size, phys["r_split"], r_cut_factor=phys["r_cut_factor"])
    pos = box.positions()
    s.set_particles(pos, box.mass)
    s.compute_forces(phys["eps2"], phys["g"])
    _, _, acc = s.get_state(box.n, pos=False, vel=False)
    counts = s.interaction_counts(box.n)
    rho, _, _, _ = s.mesh()
    t = accuracy.seeded_targets(box.n, n_targets, seed)
    ref = oracle().treepm(pos, box.mass, phys["eps2"], phys["g"], mesh, box.box_size, phys["r_split"],
                          phys["r_cut_factor"], targets=t, counts=True)
    return acc, counts, rho, t, ref


def _check(box, mesh, n_targets, seed):
    acc, counts, rho, t, ref = _run(box, mesh, n_targets, seed)
    assert np.all(np.isfinite(acc))
    assert np.array_equal(counts[t], ref["counts"])
    rel = np.linalg.norm(acc[t] - ref["acc"], axis=1) / np.linalg.norm(ref["acc"], axis=1)
    rms = float(np.sqrt(np.mean(rel ** 2)))
    assert rms < 1e-5, rms
    assert abs(float(rho.astype(np.float64).sum()) - box.mass.sum()) < 1e-5 * box.mass.sum()
    return rms


def test_treepm_box_128_parity():
    from treepm import ics
    _check(ics.treepm_box_128(), 128, 4096, 1)


def test_clustered_box_256_parity():
    from treepm import ics
    _check(ics.clustered_box_256(), 256, 2048, 2)


def test_pm_box_64_parity():
    import treepm
    from treepm import ics
    b = ics.pm_box_64()
    pos = b.positions()
    g = ics.physics(b, 64, 0.02)["g"]
    s = treepm.PmSolver(64, b.box_size)
    acc = s.accelerations_for_indices(pos, b.mass, 0.0, g, np.arange(b.n))
    ref = oracle().pm(pos, b.mass, g, 64, b.box_size)
    rel = np.linalg.norm(acc - ref, axis=1) / np.linalg.norm(ref, axis=1)
    assert float(np.sqrt(np.mean(rel ** 2))) < 1e-5


def test_hilbert_keys_and_order_bit_exact_at_256():
    """Every particle's Hilbert key and the (key, index) sort order of the
    256³ clustered workload, bit for bit against the oracle (sfc.rs:95-204,
    :371-372)."""
    import treepm
    from treepm import ics
    box = ics.clustered_box_256()
    pos = box.positions()
    s = treepm.TreePmSolver(64, box.box_size, 0.0)
    s.set_particles(pos, box.mass)
    keys, order = s.hilbert_keys(box.n)
    s.close()
    rk, ro = oracle().hilbert_keys(pos)
    assert np.array_equal(keys, rk)
    assert np.array_equal(order, ro)
