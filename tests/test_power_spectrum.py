"""In-situ power spectrum (crates/gadget-ng-analysis/src/power_spectrum.rs).

The CPU restatement (oracle/pk_oracle.py) is pinned by the reference's own
tests (uniform lattice -> P = 0, one particle -> finite) and by an analytic
case; the device estimator must match it shell by shell (mode counts exactly,
P(k) to float rounding) on lattice and clustered boxes.
"""
import numpy as np
import pytest

import pk_oracle as pko


def _lattice(n, box=1.0):
    cell = box / n
    g = (np.arange(n) + 0.5) * cell
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    return np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1), np.ones(n ** 3)


def test_oracle_uniform_lattice_is_zero():  # power_spectrum.rs:205-230
    pos, m = _lattice(4)
    _, pk, nm = pko.power_spectrum(pos, m, 1.0, 4)
    assert np.all(pk[nm > 0] < 1e-20)


def test_oracle_single_particle_is_finite():  # power_spectrum.rs:232-242
    _, pk, _ = pko.power_spectrum(np.array([[0.5, 0.5, 0.5]]), np.array([1.0]), 1.0, 8)
    assert np.all(np.isfinite(pk))


def test_oracle_plane_wave_lands_in_its_shell():
    """A density wave along x with wavenumber 3: all its power in shell 3
    (bin 2), P = (A/2)^2 V / W^2-corrected / modes, within CIC aliasing."""
    n, box, amp = 32, 1.0, 0.1
    cell = box / n
    g = (np.arange(n) + 0.5) * cell
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    m = 1.0 + amp * np.cos(2 * np.pi * 3 * X.ravel() / box)
    pos = np.stack([X.ravel(), Y.ravel(), Z.ravel()], 1)
    k, pk, nm = pko.power_spectrum(pos, m, box, n)
    assert np.argmax(pk) == 2
    assert pk[2] > 1e3 * max(pk[0], pk[1], pk[3])


def test_oracle_mode_counts_fill_the_shells():
    n = 16
    _, _, nm = pko.power_spectrum(*_lattice(n), 1.0, n)
    f = pko.freq(n)
    kx, ky, kz = np.meshgrid(f, f, f, indexing="ij")
    kk = np.sqrt(kx ** 2 + ky ** 2 + kz ** 2)
    assert nm.sum() == int(np.sum((kk >= 0.5) & (kk < n // 2 + 0.5)))


@pytest.mark.gpu
@pytest.mark.parametrize("mesh", [16, 32, 64])
def test_device_matches_oracle(mesh):
    import treepm
    from treepm import ics
    for box in (ics.lattice_box(32, 50.0, 1.0, seed=5), ics.clustered_box(32, 50.0, 0.3, 10, 50, 2000, seed=6)):
        pos = box.positions()
        k, pk, nm = treepm.power_spectrum(pos, box.mass, box.box_size, mesh)
        rk, rpk, rnm = pko.power_spectrum(pos, box.mass, box.box_size, mesh)
        keep = rnm > 0
        assert np.array_equal(nm, rnm[keep])
        assert np.allclose(k, rk[keep], rtol=1e-14)
        # float32 mesh and FFT: relative 1e-4 per shell, plus float round-off
        # against the largest shell for shells of tiny power
        ref = rpk[keep]
        assert np.all(np.abs(pk - ref) <= 1e-4 * ref + 1e-6 * ref.max())


@pytest.mark.gpu
def test_in_situ_spectrum_equals_standalone():
    import treepm
    from treepm import ics
    box = ics.clustered_box(32, 50.0, 0.3, 10, 50, 2000, seed=8)
    s = treepm.TreePmSolver(32, box.box_size, 0.0)
    s.set_particles(box.positions(), box.mass)
    k, pk, nm = s.power_spectrum()
    k2, pk2, nm2 = treepm.power_spectrum(box.positions(), box.mass, box.box_size, 32)
    assert np.array_equal(nm, nm2) and np.allclose(pk, pk2, rtol=1e-5)


@pytest.mark.gpu
def test_uniform_lattice_on_device_is_negligible():
    import treepm
    pos, m = _lattice(16)
    _, pk, _ = treepm.power_spectrum(pos, m, 1.0, 16)
    # float32 mesh and FFT: round-off only (the reference's float64 gives < 1e-20)
    assert np.all(pk < 1e-14)
