"""CPU restatement (numpy, float64) of gadget-ng's power spectrum estimator.

Test infrastructure only.  Follows
crates/gadget-ng-analysis/src/power_spectrum.rs:
  :146-166  CIC assignment, fx = x / cell, floor, weights (1 - t, t),
            indices rem_euclid(n), product m * wx * wy * wz;
  :45-57    delta = rho / (mean_rho * V_cell) - 1, mean_rho = M / L^3;
  :59-72    unnormalised 3D complex FFT;
  :74-110   per mode k != 0: |delta_k|^2 / (sinc(kx/n) sinc(ky/n) sinc(kz/n))^2
            * (V / n^3)^2, binned by floor(|k| - 1/2) into n/2 bins (|k| in
            units of the fundamental), bins without modes dropped;
  :112-119  bin label (bin + 1) * 2 pi / L;
  :124-145  freq(i) = i for i <= n/2 else i - n; sinc(x) = sin(pi x)/(pi x).
"""
from __future__ import annotations

import numpy as np


def cic_grid(pos, mass, box, n):
    """Mass grid indexed [jx, jy, jz] (the reference's x-major layout)."""
    cell = box / n
    f = np.asarray(pos, dtype=np.float64) / cell
    i0 = np.floor(f)
    t = f - i0
    i0 = i0.astype(np.int64)
    grid = np.zeros((n, n, n))
    m = np.asarray(mass, dtype=np.float64)
    for dx in (0, 1):
        wx = t[:, 0] if dx else 1.0 - t[:, 0]
        for dy in (0, 1):
            wy = t[:, 1] if dy else 1.0 - t[:, 1]
            for dz in (0, 1):
                wz = t[:, 2] if dz else 1.0 - t[:, 2]
                np.add.at(grid, ((i0[:, 0] + dx) % n, (i0[:, 1] + dy) % n, (i0[:, 2] + dz) % n), m * wx * wy * wz)
    return grid


def freq(n):
    i = np.arange(n)
    return np.where(i <= n // 2, i, i - n)


def sinc(x):
    x = np.asarray(x, dtype=np.float64)
    px = np.pi * x
    with np.errstate(invalid="ignore", divide="ignore"):
        return np.where(np.abs(x) < 1e-12, 1.0, np.sin(px) / px)


def power_spectrum(pos, mass, box, n):
    """All n/2 bins: (k, pk, n_modes) arrays; pk = 0 where n_modes = 0."""
    grid = cic_grid(pos, mass, box, n)
    mean_rho = np.sum(mass) / box ** 3
    cell = box / n
    delta = grid / (mean_rho * cell ** 3) - 1.0
    dk = np.fft.fftn(delta)
    f = freq(n).astype(np.float64)
    kx, ky, kz = np.meshgrid(f, f, f, indexing="ij")
    w = sinc(kx / n) * sinc(ky / n) * sinc(kz / n)
    k2 = kx * kx + ky * ky + kz * kz
    kmag = np.sqrt(k2)
    bin_f = kmag - 0.5
    nb = n // 2
    ok = (k2 != 0.0) & (bin_f >= 0.0) & (bin_f < nb)
    b = np.floor(bin_f[ok]).astype(np.int64)
    norm = ((box ** 3) / n ** 3) ** 2
    val = (np.abs(dk[ok]) ** 2) / (w[ok] ** 2) * norm
    pk = np.bincount(b, weights=val, minlength=nb)
    nm = np.bincount(b, minlength=nb).astype(np.int64)
    k = (np.arange(nb) + 1.0) * 2.0 * np.pi / box
    with np.errstate(invalid="ignore", divide="ignore"):
        pk = np.where(nm > 0, pk / np.maximum(nm, 1), 0.0)
    return k, pk, nm
