"""Force-accuracy reporting: FP64 Ewald reference and error statistics.

The reference has no Ewald code; `ewald_accelerations` calls the library's
float64 Ewald checker (tpm_ewald).  Every TreePM result is reported as the rms
and 99th percentile of |a - a_ewald| / |a_ewald| over a seeded subsample of
4096 particles.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from ._lib import check, load


def ewald_parameters(box: float, accuracy: float = 1e-9):
    """(alpha, r_c, n_max) with real- and k-space truncation below `accuracy`."""
    x = math.sqrt(-math.log(accuracy))          # erfc(x) ~ exp(-x^2)
    r_c = 0.25 * box
    alpha = x / r_c
    k_max = 2.0 * alpha * x                     # exp(-k^2 / 4 alpha^2) ~ accuracy
    n_max = int(math.ceil(k_max * box / (2.0 * math.pi)))
    return alpha, r_c, n_max


def ewald_accelerations(pos, mass, box, g, eps2, r_soft, targets, alpha=None, r_c=None, n_max=None, device=0):
    pos = np.ascontiguousarray(pos, dtype=np.float64)
    mass = np.ascontiguousarray(mass, dtype=np.float64)
    t = np.ascontiguousarray(targets, dtype=np.int64)
    if alpha is None:
        alpha, r_c, n_max = ewald_parameters(box)
    out = np.zeros((t.shape[0], 3))
    rc = load().tpm_ewald(pos.ctypes.data_as(C.c_void_p), mass.ctypes.data_as(C.c_void_p), pos.shape[0],
                          float(box), float(g), float(eps2), float(r_soft), t.ctypes.data_as(C.c_void_p),
                          t.shape[0], float(alpha), float(r_c), int(n_max), int(device),
                          out.ctypes.data_as(C.c_void_p))
    check(None, rc)
    return out


def relative_errors(a, ref):
    """rms and 99th percentile of the per-particle |a - ref| / |ref|."""
    r = np.linalg.norm(np.asarray(a) - np.asarray(ref), axis=1) / np.maximum(np.linalg.norm(ref, axis=1), 1e-300)
    return float(np.sqrt(np.mean(r * r))), float(np.percentile(r, 99))


def seeded_targets(n: int, k: int = 4096, seed: int = 4096):
    rng = np.random.default_rng(seed)
    return np.sort(rng.choice(n, size=min(k, n), replace=False)).astype(np.int64)
