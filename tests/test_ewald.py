"""The FP64 Ewald accuracy reference.

The reference has no Ewald code, so the Ewald sum is validated on its own
terms (CPU oracle): independence of the splitting parameter, translation
invariance, momentum conservation, the Newtonian limit of a close pair.  The
device checker must then agree with it, and TreePM forces are reported
against it.
"""
import math

import numpy as np
import pytest

from conftest import oracle


def _params(box, alpha_rc=4.6, rc_frac=0.25, kx=4.6):
    r_c = rc_frac * box
    alpha = alpha_rc / r_c
    n_max = int(math.ceil(2 * alpha * kx * box / (2 * math.pi)))
    return alpha, r_c, n_max


def _cloud(n=64, box=1.0, seed=3):
    rng = np.random.default_rng(seed)
    return rng.uniform(0, box, (n, 3)), rng.uniform(0.5, 1.5, n)


def test_ewald_independent_of_splitting():
    pos, m = _cloud()
    t = np.arange(len(m))
    a1 = oracle().ewald(pos, m, 1.0, 1.0, 0.0, 0.0, t, *_params(1.0, rc_frac=0.25))
    a2 = oracle().ewald(pos, m, 1.0, 1.0, 0.0, 0.0, t, *_params(1.0, rc_frac=0.35))
    assert np.max(np.abs(a1 - a2)) < 1e-7 * np.max(np.abs(a1))


def test_ewald_translation_invariant():
    pos, m = _cloud(seed=5)
    t = np.arange(len(m))
    p = _params(1.0)
    a1 = oracle().ewald(pos, m, 1.0, 1.0, 0.0, 0.0, t, *p)
    a2 = oracle().ewald((pos + np.array([0.37, 0.81, 0.13])) % 1.0, m, 1.0, 1.0, 0.0, 0.0, t, *p)
    assert np.max(np.abs(a1 - a2)) < 1e-8 * np.max(np.abs(a1))


def test_ewald_conserves_momentum():
    pos, m = _cloud(seed=7)
    a = oracle().ewald(pos, m, 1.0, 1.0, 0.0, 0.0, np.arange(len(m)), *_params(1.0))
    assert np.linalg.norm((a * m[:, None]).sum(0)) < 1e-9 * np.max(np.linalg.norm(a, axis=1) * m)


def test_ewald_close_pair_is_newtonian():
    d = 1e-3
    pos = np.array([[0.5, 0.5, 0.5], [0.5 + d, 0.5, 0.5]])
    a = oracle().ewald(pos, np.ones(2), 1.0, 1.0, 0.0, 0.0, np.array([0, 1]), *_params(1.0))
    assert abs(a[0, 0] - 1.0 / d ** 2) < 1e-6 / d ** 2
    assert np.allclose(a[0], -a[1], rtol=1e-12, atol=1e-6)


def test_ewald_plummer_softening_applies_to_near_images():
    d, eps = 1e-3, 2e-3
    pos = np.array([[0.5, 0.5, 0.5], [0.5 + d, 0.5, 0.5]])
    a = oracle().ewald(pos, np.ones(2), 1.0, 1.0, eps * eps, 0.1, np.array([0]), *_params(1.0))
    want = d / (d * d + eps * eps) ** 1.5
    assert abs(a[0, 0] - want) < 1e-6 * want


@pytest.mark.gpu
def test_device_ewald_matches_oracle():
    from treepm import accuracy
    pos, m = _cloud(n=500, box=50.0, seed=11)
    t = np.arange(0, 500, 7)
    p = _params(50.0)
    want = oracle().ewald(pos, m, 50.0, 2.0, 1e-4, 1.0, t, *p)
    got = accuracy.ewald_accelerations(pos, m, 50.0, 2.0, 1e-4, 1.0, t, *p)
    assert np.max(np.abs(got - want)) < 1e-10 * np.max(np.abs(want))


@pytest.mark.gpu
def test_reference_treepm_error_against_ewald_is_reported():
    """The reference TreePM (parity mode) is far from Newton: its short-range
    kernel is erfc(x)/r^2 without the Gaussian term that completes the split
    (short_range.rs:108-111) and it takes nodes holding the target as
    monopoles (short_range.rs:316-323).  The device reproduces the oracle's
    error against Ewald, which is what the bench reports."""
    import treepm
    from treepm import accuracy, ics
    b = ics.lattice_box(32, 50.0, 0.2, seed=17)
    phys = ics.physics(b, 32, 1.0)
    s = treepm.TreePmSolver(32, b.box_size, phys["r_split"], r_cut_factor=phys["r_cut_factor"])
    t = accuracy.seeded_targets(b.n, 256)
    acc = s.accelerations_for_indices(b.positions(), b.mass, phys["eps2"], phys["g"], t)
    ref = accuracy.ewald_accelerations(b.positions(), b.mass, b.box_size, phys["g"], phys["eps2"],
                                       phys["r_cut_factor"] * phys["r_split"], t)
    orc = oracle().treepm(b.positions(), b.mass, phys["eps2"], phys["g"], 32, b.box_size, phys["r_split"],
                          phys["r_cut_factor"], targets=t)["acc"]
    rms_dev, _ = accuracy.relative_errors(acc, ref)
    rms_orc, _ = accuracy.relative_errors(orc, ref)
    assert np.isfinite(rms_dev) and abs(rms_dev - rms_orc) < 1e-4 * rms_orc


def _accurate_error(box, mesh, n_targets, **opts):
    import treepm
    from treepm import accuracy, ics
    phys = ics.physics(box, mesh, 1.0)
    s = treepm.TreePmSolver(mesh, box.box_size, phys["r_split"], r_cut_factor=phys["r_cut_factor"], **opts)
    t = accuracy.seeded_targets(box.n, n_targets)
    acc = s.accelerations_for_indices(box.positions(), box.mass, phys["eps2"], phys["g"], t)
    ref = accuracy.ewald_accelerations(box.positions(), box.mass, box.box_size, phys["g"], phys["eps2"],
                                       phys["r_cut_factor"] * phys["r_split"], t)
    return accuracy.relative_errors(acc, ref)


@pytest.mark.gpu
@pytest.mark.parametrize("clustered", [False, True])
def test_accurate_mode_against_ewald(clustered):
    """The extension mode (complete split kernel, opening angle 0.5, CIC
    deconvolution) is checked against FP64 Ewald on a near-uniform and a
    clustered 32^3 box.  At r_split = 1.25 cells the mesh part sets the
    floor (rms 2.2 % near-uniform, 1.4 % clustered on a B200; opening angle
    0.2 changes it by < 20 %); the reference algorithm is at 130-150 %."""
    from treepm import ics
    b = (ics.clustered_box(32, 50.0, 0.3, 20, min_halo=50, max_halo=2000, seed=9) if clustered
         else ics.lattice_box(32, 50.0, 1.0, seed=17))
    rms, p99 = _accurate_error(b, 32, 512, accurate=True, theta=0.5, deconvolve_cic=True)
    assert rms < 3e-2 and p99 < 1e-1, (rms, p99)


@pytest.mark.gpu
def test_accurate_mode_converges_with_theta():
    from treepm import ics
    b = ics.clustered_box(32, 50.0, 0.3, 20, min_halo=50, max_halo=2000, seed=9)
    e5, _ = _accurate_error(b, 32, 512, accurate=True, theta=0.5, deconvolve_cic=True)
    e2, _ = _accurate_error(b, 32, 512, accurate=True, theta=0.2, deconvolve_cic=True)
    assert e2 < e5, (e2, e5)


def test_accurate_mode_rejects_wide_opening_angle():
    """theta >= 1/sqrt(3) could take a cell holding the target as a monopole;
    the argument check runs before any device query."""
    import treepm
    with pytest.raises(treepm.TreePmError) as e:
        treepm.TreePmSolver(32, 50.0, 0.0, accurate=True, theta=0.6)
    assert e.value.code == 1  # TPM_ERR_INVALID_ARGUMENT


@pytest.mark.gpu
def test_accurate_mode_relative_criterion_against_ewald():
    """The relative opening criterion (octree.rs:769-796: open a node while the
    quadrupole estimate g |Q|_F / d^5 is at least err_tol times the monopole
    g M / (d^2 + eps^2), or while the target lies in its cell) on the
    clustered 32^3 box: a tight tolerance reaches the mesh floor of the
    opening-angle mode, a loose one is less accurate."""
    from treepm import ics
    b = ics.clustered_box(32, 50.0, 0.3, 20, min_halo=50, max_halo=2000, seed=9)
    tight, p99 = _accurate_error(b, 32, 512, accurate=True, opening_criterion=1, err_tol_force_acc=1e-4,
                                 deconvolve_cic=True)
    loose, _ = _accurate_error(b, 32, 512, accurate=True, opening_criterion=1, err_tol_force_acc=0.5,
                               deconvolve_cic=True)
    geo, _ = _accurate_error(b, 32, 512, accurate=True, theta=0.5, deconvolve_cic=True)
    assert tight < 3e-2 and p99 < 1e-1, (tight, p99)
    assert tight <= 1.05 * geo, (tight, geo)
    assert loose > tight, (loose, tight)


def test_relative_criterion_needs_a_positive_tolerance():
    import treepm
    with pytest.raises(treepm.TreePmError) as e:
        treepm.TreePmSolver(32, 50.0, 0.0, accurate=True, opening_criterion=1, err_tol_force_acc=0.0)
    assert e.value.code == 1  # TPM_ERR_INVALID_ARGUMENT
