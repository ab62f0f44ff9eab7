"""Seeded synthetic boxes for the TreePM force path.

The reference publishes no input files for its TreePM benchmarks, so every
workload here is generated from a fixed seed:

* ``lattice_box`` — a uniform n³ lattice displaced by a Gaussian random field
  whose power spectrum is P(k) ∝ k⁻²·exp(-(k/k_Ny)²), rescaled to a given rms
  displacement (in units of the lattice spacing).  Velocities are zero.
* ``clustered_box`` — the same lattice field for a fraction of the particles,
  the rest drawn from seeded Plummer spheres (log-uniform particle counts and
  log-uniform scale radii, truncated at 10 scale radii).

Positions are returned as uint32 fixed point in box units
(x = q · L / 2³²), which is how the device stores them; ``decode`` gives the
exact float64 values that the CPU path sees, so both sides start from
bit-identical inputs.  Masses are equal, m = 1/N (total mass 1).
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

TWO32 = float(1 << 32)


@dataclass
class Box:
    """One synthetic workload: fixed-point positions plus the physical setup."""

    q: np.ndarray  # (N, 3) uint32 fixed-point positions
    box_size: float
    mass: np.ndarray  # (N,) float64
    name: str

    @property
    def n(self) -> int:
        return int(self.q.shape[0])

    def positions(self) -> np.ndarray:
        """Exact float64 positions (N, 3) that the fixed-point values encode."""
        return decode(self.q, self.box_size)


def decode(q: np.ndarray, box_size: float) -> np.ndarray:
    """x = q · (L·2⁻³²): exact in float64 whenever q·L needs ≤ 53 bits."""
    return q.astype(np.float64) * (box_size / TWO32)


def encode(x: np.ndarray, box_size: float) -> np.ndarray:
    """Wrap to [0, L) and quantise to uint32 fixed point (floor)."""
    u = np.mod(np.asarray(x, dtype=np.float64) / box_size, 1.0)
    q = np.floor(u * TWO32).astype(np.uint64) & np.uint64(0xFFFFFFFF)
    return q.astype(np.uint32)


def _dedupe(q: np.ndarray) -> np.ndarray:
    """Nudge coincident positions by one quantum in x until all are distinct.

    The reference's insertion octree recurses without bound on coincident
    positions (crates/gadget-ng-tree/src/octree.rs:501-540), so no workload
    may contain them.
    """
    q = q.copy()
    for _ in range(8):
        key = (q[:, 0].astype(np.uint64) << np.uint64(32)) | q[:, 1].astype(np.uint64)
        order = np.lexsort((q[:, 2], key))
        ks, zs = key[order], q[order, 2]
        dup = np.nonzero((ks[1:] == ks[:-1]) & (zs[1:] == zs[:-1]))[0] + 1
        if dup.size == 0:
            return q
        idx = order[dup]
        q[idx, 0] = (q[idx, 0].astype(np.uint64) + 1).astype(np.uint32)
    raise RuntimeError("could not separate coincident positions")


def _displacement_field(n: int, rms_cells: float, seed: int) -> np.ndarray:
    """Zel'dovich-style displacement (n³, 3) in lattice-spacing units."""
    rng = np.random.default_rng(seed)
    white = rng.standard_normal((n, n, n))
    wk = np.fft.rfftn(white)
    kx = np.fft.fftfreq(n) * n
    kz = np.fft.rfftfreq(n) * n
    k2 = kx[:, None, None] ** 2 + kx[None, :, None] ** 2 + kz[None, None, :] ** 2
    kny = n / 2.0
    with np.errstate(divide="ignore", invalid="ignore"):
        amp = np.where(k2 > 0, np.sqrt(k2 ** -1.0 * np.exp(-k2 / kny ** 2)), 0.0)
        dk = wk * amp
        inv_k2 = np.where(k2 > 0, 1.0 / k2, 0.0)
    disp = np.empty((n, n, n, 3), dtype=np.float64)
    for a, ka in enumerate((kx[:, None, None], kx[None, :, None], kz[None, None, :])):
        psi_k = 1j * ka * inv_k2 * dk
        disp[..., a] = np.fft.irfftn(psi_k, s=(n, n, n), axes=(0, 1, 2))
    rms = math.sqrt(float(np.mean(np.sum(disp * disp, axis=-1))))
    disp *= rms_cells / rms
    return disp.reshape(-1, 3)


def lattice_box(n: int, box_size: float, rms_cells: float, seed: int = 1, name: str = "lattice") -> Box:
    """n³ particles on a lattice displaced by the seeded Gaussian field."""
    cell = box_size / n
    g = (np.arange(n, dtype=np.float64) + 0.5) * cell
    # index order: axis 0 = x, 1 = y, 2 = z (matches the field's axes)
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    base = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
    disp = _displacement_field(n, rms_cells, seed) * cell
    q = _dedupe(encode(base + disp, box_size))
    N = q.shape[0]
    return Box(q=q, box_size=box_size, mass=np.full(N, 1.0 / N), name=name)


def clustered_box(n: int, box_size: float, halo_fraction: float = 0.3, n_halos: int = 200,
                  min_halo: float = 1e3, max_halo: float = 1e5, r_min: float = 0.05, r_max: float = 0.5,
                  rms_cells: float = 1.0, seed: int = 3, name: str = "clustered") -> Box:
    """n³ particles: (1-f) on the displaced lattice, f in seeded Plummer spheres."""
    N = n ** 3
    rng = np.random.default_rng(seed + 1000)
    n_halo_tot = int(round(halo_fraction * N))
    # log-uniform particle counts, rescaled to sum exactly to n_halo_tot
    raw = np.exp(rng.uniform(math.log(min_halo), math.log(max_halo), n_halos))
    counts = np.floor(raw * (n_halo_tot / raw.sum())).astype(np.int64)
    counts[: n_halo_tot - counts.sum()] += 1
    radii = np.exp(rng.uniform(math.log(r_min), math.log(r_max), n_halos))
    centers = rng.uniform(0.0, box_size, (n_halos, 3))
    halo_pos = []
    xmax = 1000.0 / 101.0 ** 1.5  # enclosed fraction at r = 10 a
    for c, a, m in zip(centers, radii, counts):
        X = rng.uniform(0.0, xmax, m)
        r = a / np.sqrt(X ** (-2.0 / 3.0) - 1.0)
        u = rng.uniform(-1.0, 1.0, m)
        phi = rng.uniform(0.0, 2 * math.pi, m)
        s = np.sqrt(1.0 - u * u)
        halo_pos.append(c + r[:, None] * np.stack([s * np.cos(phi), s * np.sin(phi), u], axis=1))
    halo_pos = np.concatenate(halo_pos, axis=0)
    # lattice part: keep a seeded (1-f) subset of the lattice sites
    cell = box_size / n
    g = (np.arange(n, dtype=np.float64) + 0.5) * cell
    X, Y, Z = np.meshgrid(g, g, g, indexing="ij")
    base = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
    disp = _displacement_field(n, rms_cells, seed) * cell
    keep = np.sort(rng.permutation(N)[: N - n_halo_tot])
    lat = base[keep] + disp[keep]
    q = _dedupe(encode(np.concatenate([lat, halo_pos], axis=0), box_size))
    return Box(q=q, box_size=box_size, mass=np.full(N, 1.0 / N), name=name)


# ---- the workloads, named by what they are ---------------------------------

def pm_box_64(seed: int = 1) -> Box:
    """64³ particles, L = 100 Mpc/h, 0.2-cell rms displacement (plain PM case)."""
    return lattice_box(64, 100.0, 0.2, seed, name="pm64_L100")


def treepm_box_64(seed: int = 1) -> Box:
    """64³ particles, L = 50 Mpc/h (the 128³ box's density), 1.0-cell rms displacement."""
    return lattice_box(64, 50.0, 1.0, seed, name="treepm64_L50")


def treepm_box_128(seed: int = 1) -> Box:
    """128³ particles, L = 100 Mpc/h, 1.0-cell rms displacement (TreePM case)."""
    return lattice_box(128, 100.0, 1.0, seed, name="treepm128_L100")


def clustered_box_256(seed: int = 3) -> Box:
    """256³ particles, L = 200 Mpc/h, 30 % in 200 Plummer spheres (stress case)."""
    return clustered_box(256, 200.0, 0.3, 200, seed=seed, name="clustered256_L200")


def clustered_box_512(seed: int = 5) -> Box:
    """512³ particles, L = 400 Mpc/h, 30 % in 512 Plummer spheres (scale-up case)."""
    return clustered_box(512, 400.0, 0.3, 512, seed=seed, name="clustered512_L400")


# ---- physical constants of the cosmological setup ---------------------------

OMEGA_M = 0.31
OMEGA_L = 0.69
H0_INTERNAL = 1.0  # 1/H0 is the internal time unit


def g_code_consistent(omega_m: float, h0: float, rho_bar: float) -> float:
    """G = 3 Ωm H0² / (8π ρ̄) (crates/gadget-ng-core/src/cosmology.rs:474-476)."""
    return 3.0 * omega_m * h0 * h0 / (8.0 * math.pi * max(rho_bar, 1e-300))


def physics(box: Box, mesh: int, a: float) -> dict:
    """Force-call parameters of a box at scale factor a (comoving softening)."""
    n_side = round(box.n ** (1.0 / 3.0))
    spacing = box.box_size / n_side
    eps = spacing / 30.0
    G = g_code_consistent(OMEGA_M, H0_INTERNAL, float(box.mass.sum()) / box.box_size ** 3)
    cell = box.box_size / mesh
    return dict(eps2=eps * eps, G=G, g=G * a ** 3, r_split=1.25 * cell, r_cut_factor=4.5,
                grid=mesh, box_size=box.box_size)


def time_between(a0: float, a1: float, omega_m: float = OMEGA_M, omega_l: float = OMEGA_L,
                 h0: float = H0_INTERNAL, n: int = 4096) -> float:
    """Cosmic time from a0 to a1 (ΛCDM, Simpson's rule on dt = da / (a H))."""
    a = np.linspace(a0, a1, n + 1)
    f = 1.0 / (a * h0 * np.sqrt(omega_m / a ** 3 + omega_l))
    h = (a1 - a0) / n
    return float(h / 3.0 * (f[0] + f[-1] + 4.0 * f[1:-1:2].sum() + 2.0 * f[2:-1:2].sum()))
