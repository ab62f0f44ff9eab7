"""Host-side checks that need no GPU: the C ABI library loads and exports every
entry point the header declares, fails loudly without a device, and the
host-side logic (cosmology factors, FFT indexing, workload generators)
matches the oracle."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import REPO, oracle

HEADER = os.path.join(REPO, "include", "treepm_b200.h")


def header_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(tpm_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    import treepm._lib as L
    lib = ctypes.CDLL(L.LIB_PATH)
    names = header_functions()
    assert len(names) >= 20
    for name in names:
        assert hasattr(lib, name), name
    # the Python binding declares exactly the header's functions
    assert sorted(L.SIGNATURES) == names


def test_library_is_sm100a_only():
    import treepm._lib as L
    out = os.popen(f"/usr/local/cuda/bin/cuobjdump --list-elf {L.LIB_PATH} 2>/dev/null").read()
    if not out:
        pytest.skip("cuobjdump unavailable")
    archs = set(re.findall(r"sm_(\d+a?)", out))
    assert archs == {"100a"}, archs


def test_create_without_device_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import treepm
    with pytest.raises(treepm.TreePmError) as e:
        treepm.TreePmSolver(32, 100.0)
    assert e.value.code == 8  # TPM_ERR_NO_DEVICE


def test_drift_kick_factors_bitwise_equal_to_oracle():
    import treepm
    for args in ((0.31, 0.69, 1.0, 0.02, 0.001), (0.31, 0.69, 1.0, 0.1, 0.004), (1.0, 0.0, 1.0, 1.0, 0.05)):
        assert treepm.drift_kick_factors(*args) == oracle().drift_kick_factors(*args)
        assert treepm.advance_a(*args) == oracle().advance_a(*args)


def test_gravity_coupling():
    import treepm
    assert treepm.gravity_coupling_qksl(2.0, 0.5) == 2.0 * 0.5 * 0.5 * 0.5


def _stockham_mirror(x, inverse=False):
    """The Stockham indexing of the device FFT (pm.cu fft_smem): radix-4
    passes, then one radix-2 pass when log2 n is odd."""
    n = len(x)
    logn = n.bit_length() - 1
    a = x.astype(complex).copy()
    b = np.empty_like(a)
    tw = np.exp(-2j * np.pi * np.arange(n // 2) / n)

    def twiddle(m):
        w = tw[m] if m < n // 2 else -tw[m - n // 2]
        return np.conj(w) if inverse else w

    Ns, lNs = 1, 0
    while logn - lNs >= 2:
        q = n // 4
        for j in range(q):
            k = j & (Ns - 1)
            v = [a[j + i * q] for i in range(4)]
            if k:
                sh = logn - lNs - 2
                v = [v[0]] + [v[i] * twiddle((i * k) << sh) for i in (1, 2, 3)]
            a0, a1, a2, d = v[0] + v[2], v[0] - v[2], v[1] + v[3], v[1] - v[3]
            a3 = d * (1j if inverse else -1j)
            o = ((j - k) << 2) + k
            b[o], b[o + Ns], b[o + 2 * Ns], b[o + 3 * Ns] = a0 + a2, a1 + a3, a0 - a2, a1 - a3
        a, b = b, a
        Ns, lNs = Ns * 4, lNs + 2
    if lNs < logn:
        for j in range(n // 2):
            k = j & (Ns - 1)
            w = twiddle(k << (logn - 1 - lNs))
            x0, x1 = a[j], a[j + n // 2] * w
            o = ((j - k) << 1) + k
            b[o], b[o + Ns] = x0 + x1, x0 - x1
        a, b = b, a
    return a


@pytest.mark.parametrize("n", [2, 4, 8, 16, 32, 128, 256])
def test_stockham_indexing_is_a_dft(n):
    x = np.random.default_rng(n).standard_normal(n) + 1j * np.random.default_rng(n + 1).standard_normal(n)
    assert np.max(np.abs(_stockham_mirror(x) - np.fft.fft(x))) < 1e-12 * n
    assert np.max(np.abs(_stockham_mirror(x, True) - n * np.fft.ifft(x))) < 1e-12 * n


def _packed_forward_mirror(x):
    """pm.cu k_fft_x_r2c: the real row as h = n/2 complex samples, a length-h
    transform, then the split into even and odd halves."""
    n = len(x)
    h = n // 2
    z = _stockham_mirror(x[0::2] + 1j * x[1::2])
    tw = np.exp(-2j * np.pi * np.arange(h) / n)
    out = np.empty(h + 1, dtype=complex)
    for k in range(h + 1):
        zk, zm = z[k % h], z[(h - k) % h]
        e = 0.5 * (zk + np.conj(zm))
        o = (zk - np.conj(zm)) / 2j
        w = tw[k] if k < h else -tw[0]
        out[k] = e + w * o
    return out


def _packed_inverse_mirror(spec):
    """pm.cu k_fft_x_c2r: the half spectrum (h + 1 values) to the real row of
    the unnormalised inverse, through one length-h transform."""
    h = len(spec) - 1
    n = 2 * h
    X = spec.astype(complex).copy()
    X[0], X[h] = X[0].real, X[h].real
    z = np.empty(h, dtype=complex)
    for k in range(h):
        w = np.exp(2j * np.pi * k / n)
        z[k] = X[k] * (1 + 1j * w) + np.conj(X[h - k]) * (1 - 1j * w)
    r = _stockham_mirror(z, inverse=True)
    out = np.empty(n)
    out[0::2], out[1::2] = r.real, r.imag
    return out


@pytest.mark.parametrize("n", [4, 8, 16, 64, 256])
def test_packed_real_row_transforms(n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n)
    assert np.max(np.abs(_packed_forward_mirror(x) - np.fft.rfft(x))) < 1e-12 * n
    spec = np.fft.rfft(rng.standard_normal(n))
    assert np.max(np.abs(_packed_inverse_mirror(spec) - n * np.fft.irfft(spec, n))) < 1e-12 * n
    # a row whose DC and Nyquist entries carry imaginary parts: the real part of
    # the full inverse, as the full-length transform gave it
    spec[0] += 0.7j
    spec[-1] -= 0.3j
    full = np.concatenate([spec, np.conj(spec[1:-1][::-1])])
    assert np.max(np.abs(_packed_inverse_mirror(spec) - np.real(n * np.fft.ifft(full)))) < 1e-12 * n


def test_half_spectrum_gradient_equals_real_part_of_full():
    """Zeroing the derivative's Nyquist plane reproduces Re(ifft(-i k phi)) of the
    reference's full complex transform (fft_poisson.rs:542-548, :466-473)."""
    nm = 8
    rng = np.random.default_rng(3)
    rho = rng.standard_normal((nm, nm, nm))
    k = 2 * np.pi * np.array([j if j <= nm // 2 else j - nm for j in range(nm)])
    K = np.meshgrid(k, k, k, indexing="ij")  # axes (z, y, x)
    k2 = K[0] ** 2 + K[1] ** 2 + K[2] ** 2
    rk = np.fft.fftn(rho)
    with np.errstate(divide="ignore", invalid="ignore"):
        phi = np.where(k2 > 0, -rk / k2, 0)
    for axis in range(3):
        full = np.real(np.fft.ifftn(-1j * K[axis] * phi))
        d = K[axis].copy()
        d[np.isclose(np.abs(d), np.pi * nm)] = 0.0
        half = np.fft.irfftn((-1j * d * phi)[:, :, : nm // 2 + 1], s=(nm, nm, nm), axes=(0, 1, 2))
        assert np.max(np.abs(full - half)) < 1e-12


def test_workloads_are_seeded_and_distinct():
    from treepm import ics
    a = ics.lattice_box(16, 100.0, 1.0, seed=3)
    b = ics.lattice_box(16, 100.0, 1.0, seed=3)
    assert np.array_equal(a.q, b.q)
    c = ics.clustered_box(16, 200.0, 0.3, 5, min_halo=10, max_halo=100, seed=4)
    for box in (a, c):
        u = np.unique(box.q.view([("x", np.uint32), ("y", np.uint32), ("z", np.uint32)]))
        assert len(u) == box.n
    x = a.positions()
    assert np.all(x >= 0) and np.all(x < 100.0)
    assert np.array_equal(ics.encode(x, 100.0), a.q)  # exact round trip


def test_rms_displacement_scaling():
    from treepm import ics
    disp = ics._displacement_field(16, 0.2, 1)
    assert abs(np.sqrt(np.mean(np.sum(disp ** 2, axis=1))) - 0.2) < 1e-12
