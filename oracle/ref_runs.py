"""Restatement of gadget-ng's stepping runs whose per-step diagnostics the
reference commits (test infrastructure only: the test-suite uses it to pin the
oracle's force path to the reference's own outputs; the product never imports
it).

Three pieces, each following the reference file it cites:

* ``perturbed_lattice`` — ``perturbed_lattice_ics``
  (crates/gadget-ng-core/src/ic.rs:389-462) with its LCG ``LcgState::next_f64``
  (ic.rs:467-476) and Box–Muller ``gauss_bm`` (ic.rs:284-288).  ``math.log`` and
  ``math.cos`` call the C library's ``log``/``cos``, the functions Rust's
  ``f64::ln``/``f64::cos`` lower to on Linux.
* ``diagnostics`` — ``kinetic_local`` and ``local_moments``
  (crates/gadget-ng-cli/src/engine/diagnostics.rs:28-53, :55-90),
  ``peculiar_vrms``, ``density_contrast_rms`` (16³ counting grid) and
  ``hubble_param`` (crates/gadget-ng-core/src/cosmology.rs:276-327, :509-520).
  Every sum runs left to right, as Rust's iterator ``sum`` does.
* ``run`` — the cosmological stepping loop of ``run_stepping`` on one rank
  (crates/gadget-ng-cli/src/engine/stepping/mod.rs:1011-1100, :1535-1576):
  coupling and ε² fixed at the start of each step, ``drift_kick_factors`` at
  the old a, ``advance_a`` by one RK4 step, ``leapfrog_cosmo_kdk_step`` with two
  TreePM force evaluations (the second on the drifted, not yet wrapped
  positions), then ``wrap_position``.  At one rank the TreePM SR-SFC path is the
  serial CIC + filtered FFT Poisson + CIC interpolation plus the periodic
  short-range walk over all particles (stepping/mod.rs:1088-1275;
  crates/gadget-ng-pm/src/slab_pm.rs:51-53, :272-275;
  crates/gadget-ng-pm/src/slab_fft.rs:441-452;
  crates/gadget-ng-treepm/src/distributed.rs:55-99, :134-145;
  crates/gadget-ng-parallel/src/serial.rs:107-115), i.e. the C oracle's
  ``orc_kdk_step_treepm`` with r_s = 2.5 cells (stepping/domain.rs:130-140).

The committed runs predate the reference's change of the cosmological force
coupling from G/a to G·a³ (docs/reports/2026-04-phase45-units-audit.md, "antes:
g / a"; docs/reports/2026-04-phase17a-cosmology-serial.md:74), so ``run`` takes
the coupling as an argument.  Softening is comoving and constant
(``physical_softening`` defaults to false: stepping/mod.rs:88-100).
"""
from __future__ import annotations

import math
import tomllib

import numpy as np

import oracle

_MASK64 = (1 << 64) - 1


class _Lcg:
    """LcgState (ic.rs:467-476): 64-bit LCG, 31 output bits over u32::MAX."""

    __slots__ = ("s",)

    def __init__(self, seed: int):
        self.s = seed & _MASK64

    def next_f64(self) -> float:
        self.s = (self.s * 6364136223846793005 + 1442695040888963407) & _MASK64
        return float(self.s >> 33) / 4294967295.0


def _gauss_bm(lcg: _Lcg) -> float:
    """gauss_bm (ic.rs:284-288)."""
    u1 = max(lcg.next_f64(), 1e-300)
    u2 = lcg.next_f64()
    return math.sqrt(-2.0 * math.log(u1)) * math.cos(2.0 * math.pi * u2)


def perturbed_lattice(n: int, box_size: float, amplitude: float, velocity_amplitude: float, seed: int,
                      a_init: float, h0: float):
    """Positions (n, 3), canonical momenta (n, 3) and masses (n,) of
    perturbed_lattice_ics (ic.rs:389-462), global ids 0..n in order."""
    side = int(math.ceil(n ** (1.0 / 3.0)))
    while side ** 3 < n:
        side += 1
    spacing = box_size / side
    vel_scale = a_init * velocity_amplitude * h0 * box_size
    pos = np.zeros((n, 3))
    vel = np.zeros((n, 3))
    for gid in range(n):
        ix = gid // (side * side)
        rem = gid % (side * side)
        iy = rem // side
        iz = rem % side
        x0 = (ix + 0.5) * spacing
        y0 = (iy + 0.5) * spacing
        z0 = (iz + 0.5) * spacing
        lcg = _Lcg(seed + gid * 0x9E3779B97F4A7C15)
        dx = amplitude * spacing * _gauss_bm(lcg)
        dy = amplitude * spacing * _gauss_bm(lcg)
        dz = amplitude * spacing * _gauss_bm(lcg)
        pos[gid] = (x0 + dx, y0 + dy, z0 + dz)
        if vel_scale > 0.0:
            vel[gid] = (vel_scale * _gauss_bm(lcg), vel_scale * _gauss_bm(lcg), vel_scale * _gauss_bm(lcg))
    mass = np.full(n, 1.0 / n)
    return pos, vel, mass


def _hubble(omega_m: float, omega_lambda: float, h0: float, a: float) -> float:
    """hubble_param (cosmology.rs:509-520), ΛCDM branch, no neutrinos."""
    return h0 * math.sqrt(max(omega_m / (a * a * a) + omega_lambda, 0.0))


def _rem_euclid(x: float, l: float) -> float:
    """f64::rem_euclid for a positive modulus."""
    r = math.fmod(x, l)
    return r + l if r < 0.0 else r


def _density_contrast_rms(pos, box_size: float, n_grid: int = 16) -> float:
    """density_contrast_rms (cosmology.rs:297-327): particle counts on n_grid³."""
    ng = n_grid
    inv_cell = ng / box_size
    counts = np.zeros(ng ** 3, dtype=np.int64)
    for x, y, z in pos:
        xi = min(int(_rem_euclid(x, box_size) * inv_cell), ng - 1)
        yi = min(int(_rem_euclid(y, box_size) * inv_cell), ng - 1)
        zi = min(int(_rem_euclid(z, box_size) * inv_cell), ng - 1)
        counts[xi * ng * ng + yi * ng + zi] += 1
    mean = len(pos) / float(ng ** 3)
    s = 0.0
    for c in counts:
        d = (float(c) - mean) / mean
        s += d * d
    return math.sqrt(s / float(ng ** 3))


def diagnostics(pos, vel, mass, box_size: float, a=None, cosmo=None) -> dict:
    """One diagnostics.jsonl record (diagnostics.rs:55-90, cosmology.rs:276-327)."""
    ke = 0.0
    p = [0.0, 0.0, 0.0]
    l = [0.0, 0.0, 0.0]
    mr = [0.0, 0.0, 0.0]
    mt = 0.0
    for (rx, ry, rz), (vx, vy, vz), w in zip(pos.tolist(), vel.tolist(), mass.tolist()):
        ke += 0.5 * w * (vx * vx + vy * vy + vz * vz)
        mt += w
        p[0] += w * vx
        p[1] += w * vy
        p[2] += w * vz
        l[0] += w * (ry * vz - rz * vy)
        l[1] += w * (rz * vx - rx * vz)
        l[2] += w * (rx * vy - ry * vx)
        mr[0] += w * rx
        mr[1] += w * ry
        mr[2] += w * rz
    com = [mr[0] / mt, mr[1] / mt, mr[2] / mt] if mt > 0.0 else [0.0, 0.0, 0.0]
    out = {"kinetic_energy": ke, "momentum": p, "angular_momentum": l, "com": com, "mass_total": mt}
    if a is not None:
        s = 0.0
        inv_a = 1.0 / a
        for vx, vy, vz in vel.tolist():
            ux, uy, uz = vx * inv_a, vy * inv_a, vz * inv_a
            s += ux * ux + uy * uy + uz * uz
        out["a"] = a
        out["z"] = 1.0 / a - 1.0
        out["v_rms"] = math.sqrt(s / len(vel))
        out["delta_rms"] = _density_contrast_rms(pos, box_size, 16)
        out["hubble"] = _hubble(cosmo["omega_m"], cosmo["omega_lambda"], cosmo["h0"], a)
    return out


def load_config(path: str) -> dict:
    """The [simulation], [initial_conditions], [cosmology], [gravity] keys a run needs."""
    with open(path, "rb") as f:
        c = tomllib.load(f)
    sim, cos, grav = c["simulation"], c["cosmology"], c["gravity"]
    ic = c["initial_conditions"]["kind"]["perturbed_lattice"]
    return {
        "n": int(sim["particle_count"]), "box_size": float(sim["box_size"]), "dt": float(sim["dt"]),
        "num_steps": int(sim["num_steps"]), "softening": float(sim["softening"]),
        "g": float(sim.get("gravitational_constant", 1.0)), "seed": int(sim["seed"]),
        "amplitude": float(ic["amplitude"]), "velocity_amplitude": float(ic.get("velocity_amplitude", 0.0)),
        "omega_m": float(cos["omega_m"]), "omega_lambda": float(cos["omega_lambda"]), "h0": float(cos["h0"]),
        "a_init": float(cos["a_init"]), "pm_grid": int(grav["pm_grid_size"]),
        "r_split": float(grav.get("r_split", 0.0)),
    }


def coupling(kind: str, g: float, a: float) -> float:
    """The force coupling passed to the solver: "g_over_a" (stepping before the
    units audit) or "g_a3" (gravity_coupling_qksl, cosmology.rs:354-356)."""
    if kind == "g_over_a":
        return g / a
    if kind == "g_a3":
        return g * a * a * a
    raise ValueError(kind)


def initial_state(cfg: dict):
    return perturbed_lattice(cfg["n"], cfg["box_size"], cfg["amplitude"], cfg["velocity_amplitude"], cfg["seed"],
                             cfg["a_init"], cfg["h0"])


def r_split_of(cfg: dict) -> float:
    """stepping/domain.rs:130-138: the configured r_split, else 2.5 cells."""
    return cfg["r_split"] if cfg["r_split"] > 0.0 else 2.5 * cfg["box_size"] / cfg["pm_grid"]


def wrapped_mid_step_stepper(cfg: dict):
    """The same KDK step with the drifted positions wrapped into the box
    before the second force evaluation.  The reference evaluates that force on
    the unwrapped positions (the wrap follows the step), and its periodic
    walk's monopole set depends on them (the octree is built over the
    coordinates as given), so the two differ once particles leave the box
    during a drift.  A solver that stores positions modulo the box (fixed
    point) can only take this form."""
    box = cfg["box_size"]
    r_s = r_split_of(cfg)

    def stepper(p, v, m, drift, kh, kh2, e2, g):
        acc = oracle.treepm(p, m, e2, g, cfg["pm_grid"], box, r_s, 5.0)["acc"]
        v = v + acc * kh
        p = np.mod(p + v * drift, box)
        acc = oracle.treepm(p, m, e2, g, cfg["pm_grid"], box, r_s, 5.0)["acc"]
        return p, v + acc * kh2

    return stepper


def run(cfg: dict, steps: int, coupling_kind: str = "g_over_a", stepper=None):
    """Diagnostics records of steps 0..steps.  ``stepper(pos, vel, mass, drift,
    kick_half, kick_half2, eps2, g)`` advances one KDK step (positions wrapped
    on return); the default is the C oracle's two-evaluation TreePM step."""
    pos, vel, mass = initial_state(cfg)
    box = cfg["box_size"]
    cosmo = {k: cfg[k] for k in ("omega_m", "omega_lambda", "h0")}
    r_s = r_split_of(cfg)
    eps2 = cfg["softening"] * cfg["softening"]
    if stepper is None:
        def stepper(p, v, m, drift, kh, kh2, e2, g):
            p2, v2, _ = oracle.kdk_step_treepm(p, v, m, drift, kh, kh2, e2, g, cfg["pm_grid"], box, r_s, 5.0)
            return p2, v2
    recs = [dict(diagnostics(pos, vel, mass, box), step=0)]
    a = cfg["a_init"]
    for step in range(1, steps + 1):
        g = coupling(coupling_kind, cfg["g"], a)
        drift, kh, kh2 = oracle.drift_kick_factors(cfg["omega_m"], cfg["omega_lambda"], cfg["h0"], a, cfg["dt"])
        a = oracle.advance_a(cfg["omega_m"], cfg["omega_lambda"], cfg["h0"], a, cfg["dt"])
        pos, vel = stepper(pos, vel, mass, drift, kh, kh2, eps2, g)
        recs.append(dict(diagnostics(pos, vel, mass, box, a, cosmo), step=step))
    return recs
