"""ctypes binding of the TreePM oracle (test infrastructure only).

The oracle is a CPU restatement of gadget-ng's TreePM force path
(treepm_oracle.cpp in this directory).  Only the test-suite, the smoke check
and the CPU-baseline leg of the benchmark may import this module; the product
library never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "liboracle.so")
_lib = None

_d = C.c_double
_i64 = C.c_int64
_i32 = C.c_int
_p = C.c_void_p


def build() -> str:
    """Compile liboracle.so with the committed Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        sig = {
            "orc_num_threads": ([], _i32),
            "orc_set_threads": ([_i32], None),
            "orc_erfc_approx": ([_d], _d),
            "orc_minimum_image": ([_d, _d], _d),
            "orc_min_dist2_aabb_periodic": ([_p, _p, _d, _d], _d),
            "orc_pair_accel": ([_p, _d, _d, _d, _d, _p], None),
            "orc_cic_assign": ([_p, _p, _i64, _d, _i32, _p], None),
            "orc_cic_interpolate": ([_p, _p, _p, _p, _i64, _d, _i32, _p], None),
            "orc_solve_forces": ([_p, _d, _i32, _d, _d, _d, _i32, _p, _p, _p], None),
            "orc_fft3d_roundtrip": ([_p, _i32, _p, _p, _p], None),
            "orc_octree": ([_p, _p, _i64, _i64, _p, _p, _p, _p, _p, _p, _p], _i64),
            "orc_short_range": ([_p, _p, _i64, _d, _d, _d, _d, _d, _i32, _p, _i64, _p, _p], _i32),
            "orc_treepm": ([_p, _p, _i64, _d, _d, _i32, _d, _d, _d, _i32, _i32, _p, _i64, _p, _p, _p, _p, _p],
                           _i32),
            "orc_pm": ([_p, _p, _i64, _d, _i32, _d, _i32, _p, _i64, _p], None),
            "orc_cic_cells": ([_p, _i64, _d, _i32, _p], None),
            "orc_hilbert3": ([_d, _d, _d], C.c_uint64),
            "orc_morton3": ([_d, _d, _d], C.c_uint64),
            "orc_coords_to_hilbert": ([C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32], C.c_uint64),
            "orc_hilbert_keys": ([_p, _i64, _p, _p], None),
            "orc_drift_kick_factors": ([_d, _d, _d, _d, _d, _p], None),
            "orc_advance_a": ([_d, _d, _d, _d, _d], _d),
            "orc_kdk_step_treepm": ([_p, _p, _p, _i64, _d, _d, _d, _d, _d, _i32, _d, _d, _d, _p], _i32),
            "orc_direct_min_image": ([_p, _p, _i64, _d, _d, _d, _p, _i64, _p], None),
            "orc_ewald": ([_p, _p, _i64, _d, _d, _d, _d, _p, _i64, _d, _d, _i32, _p], None),
        }
        for name, (args, res) in sig.items():
            f = getattr(L, name)
            f.argtypes = args
            f.restype = res
        _lib = L
    return _lib


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


def num_threads() -> int:
    return int(lib().orc_num_threads())


def erfc_approx(x: float) -> float:
    return lib().orc_erfc_approx(float(x))


def minimum_image(dx: float, box: float) -> float:
    return lib().orc_minimum_image(float(dx), float(box))


def min_dist2_to_aabb_periodic(xi, com, half: float, box: float) -> float:
    xi, com = _f64(xi), _f64(com)
    return lib().orc_min_dist2_aabb_periodic(_ptr(xi), _ptr(com), float(half), float(box))


def pair_accel(r, mass, eps2, g, r_split):
    r = _f64(r)
    out = np.zeros(3)
    lib().orc_pair_accel(_ptr(r), float(mass), float(eps2), float(g), float(r_split), _ptr(out))
    return out


def cic_assign(pos, mass, box, nm):
    pos, mass = _f64(pos), _f64(mass)
    rho = np.zeros(nm ** 3)
    lib().orc_cic_assign(_ptr(pos), _ptr(mass), pos.shape[0], float(box), int(nm), _ptr(rho))
    return rho


def cic_interpolate(fx, fy, fz, pos, box, nm):
    fx, fy, fz, pos = _f64(fx), _f64(fy), _f64(fz), _f64(pos)
    out = np.zeros((pos.shape[0], 3))
    lib().orc_cic_interpolate(_ptr(fx), _ptr(fy), _ptr(fz), _ptr(pos), pos.shape[0], float(box), int(nm), _ptr(out))
    return out


DECONVOLVE_CIC = 1
FOUR_POINT_GRADIENT = 2


def solve_forces(density, g, nm, box, r_split=None, plummer_eps=None, flags=0):
    density = _f64(density)
    f = [np.zeros(nm ** 3) for _ in range(3)]
    lib().orc_solve_forces(_ptr(density), float(g), int(nm), float(box), float(r_split or 0.0),
                           float(plummer_eps or 0.0), int(flags), _ptr(f[0]), _ptr(f[1]), _ptr(f[2]))
    return f


def fft3d_roundtrip(x, nm):
    x = _f64(x)
    fr, fi, back = np.zeros(nm ** 3), np.zeros(nm ** 3), np.zeros(nm ** 3)
    lib().orc_fft3d_roundtrip(_ptr(x), int(nm), _ptr(fr), _ptr(fi), _ptr(back))
    return fr + 1j * fi, back


def octree(pos, mass):
    """Full insertion octree (including empty leaves) as numpy arrays."""
    pos, mass = _f64(pos), _f64(mass)
    n = pos.shape[0]
    root = np.zeros(4)
    nn = lib().orc_octree(_ptr(pos), _ptr(mass), n, 0, None, None, None, None, None, None, _ptr(root))
    if nn < 0:
        raise ValueError("coincident positions")
    ch = np.zeros((nn, 4))
    mc = np.zeros((nn, 4))
    qd = np.zeros((nn, 6))
    pidx = np.zeros(nn, dtype=np.int64)
    depth = np.zeros(nn, dtype=np.int32)
    kids = np.zeros((nn, 8), dtype=np.uint32)
    lib().orc_octree(_ptr(pos), _ptr(mass), n, nn, _ptr(ch), _ptr(mc), _ptr(qd), _ptr(pidx), _ptr(depth),
                     _ptr(kids), _ptr(root))
    return dict(center=ch[:, :3], half=ch[:, 3], mass=mc[:, 0], com=mc[:, 1:], quad=qd, particle_idx=pidx,
                depth=depth, children=kids, root_center=root[:3], root_half=root[3])


def short_range(pos, mass, eps2, g, r_split, r_cut, box, targets=None, periodic=True, counts=False):
    pos, mass = _f64(pos), _f64(mass)
    n = pos.shape[0]
    t = np.arange(n, dtype=np.int64) if targets is None else np.ascontiguousarray(targets, dtype=np.int64)
    out = np.zeros((t.shape[0], 3))
    cnt = np.zeros((t.shape[0], 2), dtype=np.int64) if counts else None
    rc = lib().orc_short_range(_ptr(pos), _ptr(mass), n, float(eps2), float(g), float(r_split), float(r_cut) ** 2,
                               float(box), 1 if periodic else 0, _ptr(t), t.shape[0], _ptr(out), _ptr(cnt))
    if rc != 0:
        raise ValueError("coincident positions")
    return (out, cnt) if counts else out


def treepm(pos, mass, eps2, g, nm, box, r_split=0.0, r_cut_factor=5.0, targets=None, periodic=True, pm_flags=0,
           parts=False, counts=False):
    """TreePmSolver::accelerations_for_indices restated (periodic walk by default)."""
    pos, mass = _f64(pos), _f64(mass)
    n = pos.shape[0]
    t = np.arange(n, dtype=np.int64) if targets is None else np.ascontiguousarray(targets, dtype=np.int64)
    out = np.zeros((t.shape[0], 3))
    lr = np.zeros_like(out) if parts else None
    sr = np.zeros_like(out) if parts else None
    cnt = np.zeros((t.shape[0], 2), dtype=np.int64) if counts else None
    times = np.zeros(4)
    rc = lib().orc_treepm(_ptr(pos), _ptr(mass), n, float(eps2), float(g), int(nm), float(box), float(r_split),
                          float(r_cut_factor), 1 if periodic else 0, int(pm_flags), _ptr(t), t.shape[0], _ptr(out),
                          _ptr(lr), _ptr(sr), _ptr(cnt), _ptr(times))
    if rc != 0:
        raise ValueError("coincident positions")
    res = dict(acc=out, times=times)
    if parts:
        res.update(lr=lr, sr=sr)
    if counts:
        res.update(counts=cnt)
    return res


def pm(pos, mass, g, nm, box, targets=None, pm_flags=0):
    pos, mass = _f64(pos), _f64(mass)
    n = pos.shape[0]
    t = np.arange(n, dtype=np.int64) if targets is None else np.ascontiguousarray(targets, dtype=np.int64)
    out = np.zeros((t.shape[0], 3))
    lib().orc_pm(_ptr(pos), _ptr(mass), n, float(g), int(nm), float(box), int(pm_flags), _ptr(t), t.shape[0],
                 _ptr(out))
    return out


def cic_cells(pos, box, nm):
    pos = _f64(pos)
    out = np.zeros((pos.shape[0], 3), dtype=np.int32)
    lib().orc_cic_cells(_ptr(pos), pos.shape[0], float(box), int(nm), _ptr(out))
    return out


def octree_paths(tree):
    """(depth, path_hi, path_lo) of every non-empty node, paths packed like the
    device export: 3 bits per level from bit 62 down, levels 22.. in path_lo."""
    ch = tree["children"]
    n = ch.shape[0]
    hi = np.zeros(n, dtype=np.uint64)
    lo = np.zeros(n, dtype=np.uint64)
    depth = tree["depth"]
    stack = [0]
    while stack:
        i = stack.pop()
        for o in range(8):
            c = int(ch[i, o])
            if c == 0xFFFFFFFF:
                continue
            d = int(depth[c])
            h, l = int(hi[i]), int(lo[i])
            if d <= 21:
                h |= o << (63 - 3 * d)
            else:
                l |= o << (63 - 3 * (d - 21))
            hi[c], lo[c] = h, l
            stack.append(c)
    keep = tree["mass"] > 0
    return keep, hi, lo


def hilbert3(x, y, z) -> int:
    return int(lib().orc_hilbert3(float(x), float(y), float(z)))


def morton3(x, y, z) -> int:
    return int(lib().orc_morton3(float(x), float(y), float(z)))


def coords_to_hilbert(ix, iy, iz, p) -> int:
    return int(lib().orc_coords_to_hilbert(int(ix), int(iy), int(iz), int(p)))


def hilbert_keys(pos):
    pos = _f64(pos)
    n = pos.shape[0]
    keys = np.zeros(n, dtype=np.uint64)
    order = np.zeros(n, dtype=np.int64)
    lib().orc_hilbert_keys(_ptr(pos), n, _ptr(keys), _ptr(order))
    return keys, order


def drift_kick_factors(omega_m, omega_lambda, h0, a0, dt):
    out = np.zeros(3)
    lib().orc_drift_kick_factors(float(omega_m), float(omega_lambda), float(h0), float(a0), float(dt), _ptr(out))
    return tuple(float(v) for v in out)


def advance_a(omega_m, omega_lambda, h0, a, dt):
    return float(lib().orc_advance_a(float(omega_m), float(omega_lambda), float(h0), float(a), float(dt)))


def kdk_step_treepm(pos, vel, mass, drift, kick_half, kick_half2, eps2, g, nm, box, r_split, r_cut_factor):
    pos, vel, mass = _f64(pos).copy(), _f64(vel).copy(), _f64(mass)
    acc = np.zeros_like(pos)
    rc = lib().orc_kdk_step_treepm(_ptr(pos), _ptr(vel), _ptr(mass), pos.shape[0], float(drift), float(kick_half),
                                   float(kick_half2), float(eps2), float(g), int(nm), float(box), float(r_split),
                                   float(r_cut_factor), _ptr(acc))
    if rc != 0:
        raise ValueError("coincident positions")
    return pos, vel, acc


def direct_min_image(pos, mass, eps2, g, box, targets=None):
    pos, mass = _f64(pos), _f64(mass)
    n = pos.shape[0]
    t = np.arange(n, dtype=np.int64) if targets is None else np.ascontiguousarray(targets, dtype=np.int64)
    out = np.zeros((t.shape[0], 3))
    lib().orc_direct_min_image(_ptr(pos), _ptr(mass), n, float(eps2), float(g), float(box), _ptr(t), t.shape[0],
                               _ptr(out))
    return out


def ewald(pos, mass, box, g, eps2, r_soft, targets, alpha, r_c, n_max):
    """FP64 Ewald accelerations at `targets` (nearest images within r_soft Plummer-softened)."""
    pos, mass = _f64(pos), _f64(mass)
    t = np.ascontiguousarray(targets, dtype=np.int64)
    out = np.zeros((t.shape[0], 3))
    lib().orc_ewald(_ptr(pos), _ptr(mass), pos.shape[0], float(box), float(g), float(eps2), float(r_soft), _ptr(t),
                    t.shape[0], float(alpha), float(r_c), int(n_max), _ptr(out))
    return out
