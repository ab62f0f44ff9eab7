"""Momentum along the clustered workload's trajectory.

The reference's own momentum test (crates/gadget-ng-treepm/tests/
treepm_vs_direct.rs:75-113: eight particles, |Σ m·a| / max m|a| < 1e-3)
runs through the device's trait entry.

Then ten fused KDK steps with one global dt from a = 0.1 to 0.12 on a
clustered box (30 % of the particles in Plummer spheres, as the 256³
workload, at 64³).  On clustered boxes the reference's periodic walk does not
conserve momentum: a node below 0.1 r_cut is taken as a monopole even when it
holds the target (short_range.rs:316-323), so the target pulls on its own
mass and nothing pulls back.  The device must show the same residual
|Σ m·a| / max m|a| as the oracle on the same state (within 2 %, the FP32 pair
arithmetic against float64), and the residual of the accurate mode (no
self-monopole) must stay below the parity mode's.
"""
import numpy as np
import pytest

from conftest import oracle

pytestmark = pytest.mark.gpu


def test_reference_momentum_test_through_the_device():
    import treepm
    from treepm import diagnostics
    box = 2.0
    c = [(0.15, 0.15, 0.15), (0.25, 0.15, 0.15), (0.15, 0.25, 0.15), (0.25, 0.25, 0.15),
         (0.15, 0.15, 0.25), (0.25, 0.15, 0.25), (0.15, 0.25, 0.25), (0.25, 0.25, 0.25)]
    pos = np.array(c) * box
    mass = np.ones(8)
    s = treepm.TreePmSolver(16, box, 0.0, device=0)
    acc = s.accelerations_for_indices(pos, mass, 1e-4, 1.0, np.arange(8))
    s.close()
    assert diagnostics.force_momentum_residual(acc, mass) < 1e-3


def test_momentum_residual_along_the_trajectory_matches_the_oracle():
    import bench
    import treepm
    from treepm import diagnostics, ics
    box = ics.clustered_box(64, 50.0, 0.3, 40, min_halo=50, max_halo=5000, r_min=0.05, r_max=0.5, seed=11)
    nm = 64
    phys = ics.physics(box, nm, 0.1)
    factors, a_of = bench.trajectory(0.1, 0.12, phys["G"])
    s = treepm.TreePmSolver(nm, box.box_size, phys["r_split"], r_cut_factor=phys["r_cut_factor"], device=0)
    s.set_particles_fixed(box.q, box.mass)
    s.compute_forces(phys["eps2"], factors[0][3])
    checked = 0
    for i, (d, k1, k2, g) in enumerate(factors):
        s.kdk_step(k1, d, k2, phys["eps2"], g)
        if i not in (0, 9):
            continue
        pos, vel, acc = s.get_state(box.n)
        res = diagnostics.force_momentum_residual(acc, box.mass)
        ref = oracle().treepm(pos, box.mass, phys["eps2"], g, nm, box.box_size, phys["r_split"],
                              phys["r_cut_factor"])["acc"]
        res_ref = diagnostics.force_momentum_residual(ref, box.mass)
        assert abs(res - res_ref) <= 0.02 * res_ref, (i, res, res_ref)
        acc_s = treepm.TreePmSolver(nm, box.box_size, phys["r_split"], r_cut_factor=phys["r_cut_factor"],
                                    accurate=True, theta=0.5, device=0)
        acc_s.set_particles(pos, box.mass)
        acc_s.compute_forces(phys["eps2"], g)
        _, _, a_acc = acc_s.get_state(box.n, pos=False, vel=False)
        acc_s.close()
        assert diagnostics.force_momentum_residual(a_acc, box.mass) < res
        rec = diagnostics.record(pos, vel, box.mass, a_of[i + 1])
        assert np.isfinite(rec["kinetic_energy"]) and rec["kinetic_energy"] > 0.0
        checked += 1
    s.close()
    assert checked == 2
