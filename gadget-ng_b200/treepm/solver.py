"""Host-side mirror of gadget-ng's gravity-solver interface for the B200 library.

`TreePmSolver` and `PmSolver` have the constructor fields and the
`accelerations_for_indices` call of the reference's `GravitySolver` trait
(crates/gadget-ng-core/src/gravity.rs:14-56; TreePmSolver
crates/gadget-ng-treepm/src/solver.rs:44-108; PmSolver
crates/gadget-ng-pm/src/solver.rs:23-140).  Where the reference panics on a
device failure (crates/gadget-ng-cuda/src/pm_solver.rs:137-151) these raise
`TreePmError`.  `make_solver` reads the same [gravity] keys as
crates/gadget-ng-cli/src/engine/gravity.rs:352-517.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import TpmConfig, TpmStats, TpmZeldovich, TreePmError, check, load


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


class _Handle:
    def __init__(self, cfg: TpmConfig):
        self._lib = load()
        h = C.c_void_p()
        rc = self._lib.tpm_create(C.byref(cfg), C.byref(h))
        if rc != 0:
            raise TreePmError(rc, "tpm_create failed")
        self.h = h
        self.cfg = cfg

    def close(self):
        if getattr(self, "h", None):
            self._lib.tpm_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class TreePmSolver:
    """TreePM: PM with the Gaussian long-range filter + erfc short-range tree walk.

    Parameters mirror `TreePmSolver { grid_size, box_size, r_split }`; r_split
    <= 0 selects 2.5 cells.  `r_cut_factor` is the extension key for r_cut / r_s
    (the reference hard-codes 5).  `periodic_walk` selects the periodic walk of
    the P=1 slab path (default) or the aperiodic walk of the trait-level solver.
    `accurate` selects the extension mode (complete split kernel, geometric
    opening angle `theta`); it is validated against Ewald, not the reference.
    `learned` keeps the long-range potential on the mesh so that a trained
    `treepm.learned.Network` can be attached (`set_learned`) to stand in for
    the walk outside dense cells, or boxes can be captured to train one.
    """

    def __init__(self, grid_size: int, box_size: float, r_split: float = 0.0, *, r_cut_factor: float = 5.0,
                 periodic_walk: bool = True, theta: float = 0.5, opening_criterion: int = 0,
                 err_tol_force_acc: float = 0.005, deconvolve_cic: bool = False, four_point_gradient: bool = False,
                 accurate: bool = False, learned: bool = False, device: int = 0, memory_cap_bytes: int = 0,
                 _pm_only: bool = False):
        flags = 0
        if accurate:
            flags |= _lib.FLAG_ACCURATE
        if learned:
            flags |= _lib.FLAG_LEARNED
        if not periodic_walk:
            flags |= _lib.FLAG_APERIODIC_WALK
        if deconvolve_cic:
            flags |= _lib.FLAG_DECONVOLVE_CIC
        if four_point_gradient:
            flags |= _lib.FLAG_FOUR_POINT_GRADIENT
        if _pm_only:
            flags |= _lib.FLAG_PM_ONLY
        cfg = TpmConfig(grid_size=int(grid_size), box_size=float(box_size), r_split=float(r_split),
                        r_cut_factor=float(r_cut_factor), theta=float(theta),
                        opening_criterion=int(opening_criterion), err_tol_force_acc=float(err_tol_force_acc),
                        flags=flags, device=int(device), memory_cap_bytes=int(memory_cap_bytes))
        self.grid_size = int(grid_size)
        self.box_size = float(box_size)
        self.r_split = float(r_split)
        self._h = _Handle(cfg)

    def power_spectrum(self):
        """P(k) of the resident particles on this solver's mesh (in-situ
        analysis, power_spectrum.rs estimator): (k, pk, n_modes) of the shells
        that hold modes."""
        nb = self.grid_size // 2
        k, pk, nm = np.empty(nb), np.empty(nb), np.empty(nb, dtype=np.uint64)
        check(self._h.h, self._h._lib.tpm_get_power_spectrum(self._h.h, _ptr(k), _ptr(pk), _ptr(nm)))
        keep = nm > 0
        return k[keep], pk[keep], nm[keep].astype(np.int64)

    def set_learned(self, network):
        """Attach a trained network (a copy is taken); None detaches it."""
        check(self._h.h, self._h._lib.tpm_set_learned(self._h.h, None if network is None else network.h))

    # ---- the GravitySolver call ------------------------------------------
    def accelerations_for_indices(self, global_positions, global_masses, eps2: float, g: float,
                                  global_indices, out=None):
        """Accelerations of `global_indices` from the global state (gravity.rs:16-24)."""
        pos = np.ascontiguousarray(global_positions, dtype=np.float64).reshape(-1, 3)
        mass = np.ascontiguousarray(global_masses, dtype=np.float64).reshape(-1)
        idx = np.ascontiguousarray(global_indices, dtype=np.uint64).reshape(-1)
        if pos.shape[0] != mass.shape[0]:
            raise ValueError("positions and masses differ in length")
        if out is None:
            out = np.empty((idx.shape[0], 3), dtype=np.float64)
        elif out.shape != (idx.shape[0], 3) or out.dtype != np.float64 or not out.flags.c_contiguous:
            raise ValueError("out must be a C-contiguous float64 array of shape (len(global_indices), 3)")
        rc = self._h._lib.tpm_accelerations_for_indices(self._h.h, _ptr(pos), _ptr(mass), pos.shape[0], float(eps2),
                                                        float(g), _ptr(idx), idx.shape[0], _ptr(out))
        check(self._h.h, rc)
        return out

    def accelerations_with_costs(self, global_positions, global_masses, eps2: float, g: float, global_indices,
                                 out=None):
        """accelerations_with_costs (gravity.rs:36-55): the accelerations and
        one uint64 work figure per index, the short-range interactions its walk
        made (leaf pairs + monopoles, the per-target counters of
        tpm_get_interaction_counts).  Empty costs, as the trait's default, when
        nothing was walked (no indices, plain PM)."""
        out = self.accelerations_for_indices(global_positions, global_masses, eps2, g, global_indices, out)
        idx = np.ascontiguousarray(global_indices, dtype=np.int64).reshape(-1)
        n = np.asarray(global_positions).reshape(-1, 3).shape[0]
        if idx.size == 0 or self._h.cfg.flags & _lib.FLAG_PM_ONLY or n < 2:
            return out, np.zeros(0, dtype=np.uint64)
        counts = self.interaction_counts(n)
        return out, counts[idx].sum(axis=1).astype(np.uint64)

    # ---- device-resident state (fused integrator path) --------------------
    def set_particles(self, pos, mass, vel=None):
        pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
        mass = np.ascontiguousarray(mass, dtype=np.float64).reshape(-1)
        v = None if vel is None else np.ascontiguousarray(vel, dtype=np.float64).reshape(-1, 3)
        check(self._h.h, self._h._lib.tpm_set_particles(self._h.h, _ptr(pos), _ptr(v), _ptr(mass), pos.shape[0]))

    def set_particles_zeldovich(self, n_side: int, seed: int = 42, **cfg):
        """Zel'dovich initial conditions (ic_zeldovich.rs:621-760) generated on
        the device into this solver: n_side^3 particles of mass 1/N, gid = ix n^2
        + iy n + iz.  Keywords as `zeldovich_config`."""
        c = zeldovich_config(n_side, seed, **cfg)
        check(self._h.h, self._h._lib.tpm_set_particles_zeldovich(self._h.h, C.byref(c)))
        return int(n_side) ** 3

    # ---- snapshots and checkpoints (crates/gadget-ng-io, engine/checkpoint.rs) --
    def write_snapshot(self, out_dir, fmt="jsonl", time=0.0, redshift=0.0, box_size=None, units=None,
                       provenance=None):
        """The resident particles as a gadget-ng snapshot ("jsonl" or "bincode")."""
        from . import snapshot
        snapshot.solver_write_snapshot(self._h, out_dir, fmt, time, redshift,
                                       self.box_size if box_size is None else box_size, units, provenance)

    def read_snapshot(self, path, fmt="jsonl") -> dict:
        """Load a snapshot's particles (global ids 0..n-1); returns meta.json's fields."""
        from . import snapshot
        return snapshot.solver_read_snapshot(self._h, path, fmt)

    def write_checkpoint(self, out_dir, completed_step, a_current, config_hash=""):
        from . import snapshot
        snapshot.solver_write_checkpoint(self._h, out_dir, completed_step, a_current, config_hash)

    def read_checkpoint(self, resume_dir):
        """(completed_step, a_current, config_hash); the particles become the state."""
        from . import snapshot
        return snapshot.solver_read_checkpoint(self._h, resume_dir)

    def set_particles_fixed(self, q, mass, vel=None):
        q = np.ascontiguousarray(q, dtype=np.uint32).reshape(-1, 3)
        mass = np.ascontiguousarray(mass, dtype=np.float64).reshape(-1)
        v = None if vel is None else np.ascontiguousarray(vel, dtype=np.float32).reshape(-1, 3)
        check(self._h.h, self._h._lib.tpm_set_particles_fixed(self._h.h, _ptr(q), _ptr(v), _ptr(mass), q.shape[0]))

    def compute_forces(self, eps2: float, g: float):
        check(self._h.h, self._h._lib.tpm_compute_forces(self._h.h, float(eps2), float(g)))

    def kdk_step(self, kick_half: float, drift: float, kick_half2: float, eps2: float, g: float):
        check(self._h.h, self._h._lib.tpm_kdk_step(self._h.h, float(kick_half), float(drift), float(kick_half2),
                                                   float(eps2), float(g)))

    def kdk_step_host(self, pos, vel, mass, kick_half, drift, kick_half2, eps2, g):
        """KDK step on host arrays (pos/vel float64 (N,3), updated in place)."""
        assert pos.dtype == np.float64 and vel.dtype == np.float64 and pos.flags.c_contiguous
        mass = np.ascontiguousarray(mass, dtype=np.float64)
        check(self._h.h, self._h._lib.tpm_kdk_step_host(self._h.h, _ptr(pos), _ptr(vel), _ptr(mass), pos.shape[0],
                                                        float(kick_half), float(drift), float(kick_half2),
                                                        float(eps2), float(g)))

    def get_state(self, n: int, pos=True, vel=True, acc=True):
        p = np.empty((n, 3)) if pos else None
        v = np.empty((n, 3)) if vel else None
        a = np.empty((n, 3)) if acc else None
        check(self._h.h, self._h._lib.tpm_get_state(self._h.h, _ptr(p), _ptr(v), _ptr(a)))
        return p, v, a

    def force_parts(self, n: int):
        lr, sr = np.empty((n, 3)), np.empty((n, 3))
        check(self._h.h, self._h._lib.tpm_get_force_parts(self._h.h, _ptr(lr), _ptr(sr)))
        return lr, sr

    def interaction_counts(self, n: int):
        """(n, 2) leaf pairs and monopoles of the last walk, per particle."""
        c = np.empty((n, 2), dtype=np.int64)
        check(self._h.h, self._h._lib.tpm_get_interaction_counts(self._h.h, _ptr(c)))
        return c

    def stats(self) -> dict:
        s = TpmStats()
        check(self._h.h, self._h._lib.tpm_get_stats(self._h.h, C.byref(s)))
        return s.as_dict()

    # ---- inspection of the hot-path stages ------------------------------
    def hilbert_keys(self, n: int):
        keys = np.empty(n, dtype=np.uint64)
        order = np.empty(n, dtype=np.int64)
        check(self._h.h, self._h._lib.tpm_hilbert_keys(self._h.h, _ptr(keys), _ptr(order)))
        return keys, order

    def cic_cells(self, n: int):
        cells = np.empty((n, 3), dtype=np.int32)
        check(self._h.h, self._h._lib.tpm_cic_cells(self._h.h, _ptr(cells)))
        return cells

    def export_tree(self):
        L = self._h._lib
        tot = int(L.tpm_export_tree(self._h.h, 0, None, None, None, None, None, None, None))
        if tot < 0:
            check(self._h.h, -tot)
        depth = np.empty(tot, dtype=np.int32)
        mass = np.empty(tot)
        com = np.empty((tot, 3))
        quad = np.empty((tot, 6))
        part = np.empty(tot, dtype=np.int64)
        ph = np.empty(tot, dtype=np.uint64)
        pl = np.empty(tot, dtype=np.uint64)
        r = int(L.tpm_export_tree(self._h.h, tot, _ptr(depth), _ptr(mass), _ptr(com), _ptr(quad), _ptr(part),
                                  _ptr(ph), _ptr(pl)))
        if r < 0:
            check(self._h.h, -r)
        return dict(depth=depth, mass=mass, com=com, quad=quad, particle=part, path_hi=ph, path_lo=pl)

    def mesh(self):
        nm = self.grid_size
        arrs = [np.empty(nm ** 3, dtype=np.float32) for _ in range(4)]
        check(self._h.h, self._h._lib.tpm_get_mesh(self._h.h, *[_ptr(a) for a in arrs]))
        return arrs

    @property
    def stream(self) -> int:
        return int(self._h._lib.tpm_get_stream(self._h.h) or 0)

    def set_stream(self, stream_ptr: int):
        check(self._h.h, self._h._lib.tpm_set_stream(self._h.h, C.c_void_p(stream_ptr)))

    def close(self):
        self._h.close()


class PmSolver(TreePmSolver):
    """Plain PM (`PmSolver`, crates/gadget-ng-pm/src/solver.rs:23-140): no filter, no short range."""

    def __init__(self, grid_size: int, box_size: float, *, four_point_gradient: bool = False,
                 deconvolve_cic: bool = False, device: int = 0):
        super().__init__(grid_size, box_size, 0.0, four_point_gradient=four_point_gradient,
                         deconvolve_cic=deconvolve_cic, device=device, _pm_only=True)


def make_solver(cfg: dict):
    """Solver factory over the reference's TOML keys (engine/gravity.rs:352-517).

    `cfg` is the parsed TOML document: [simulation] box_size, [gravity]
    solver / pm_grid_size / r_split / theta / opening_criterion /
    err_tol_force_acc and the extension keys r_cut_factor and
    treepm_accurate (the complete split kernel with the opening angle).
    """
    sim = cfg.get("simulation", {})
    grav = cfg.get("gravity", {})
    kind = grav.get("solver", "tree_pm")
    box = float(sim.get("box_size", 1.0))
    nm = int(grav.get("pm_grid_size", 64))
    if kind == "pm":
        return PmSolver(nm, box)
    if kind not in ("tree_pm", "treepm"):
        raise ValueError(f"solver {kind!r} is not provided by the B200 library (tree_pm and pm are)")
    crit = grav.get("opening_criterion", "geometric")
    return TreePmSolver(nm, box, float(grav.get("r_split", 0.0)),
                        r_cut_factor=float(grav.get("r_cut_factor", 5.0)),
                        periodic_walk=bool(grav.get("treepm_slab", True)),
                        theta=float(grav.get("theta", 0.5)),
                        opening_criterion=1 if crit in ("relative", 1) else 0,
                        err_tol_force_acc=float(grav.get("err_tol_force_acc", 0.005)),
                        accurate=bool(grav.get("treepm_accurate", False)))


def power_spectrum(positions, masses, box_size: float, mesh: int, device: int = 0):
    """power_spectrum(positions, masses, box_size, mesh)
    (crates/gadget-ng-analysis/src/power_spectrum.rs:35-120) on the GPU:
    (k, pk, n_modes) of the shells that hold modes, by increasing k."""
    pos = np.ascontiguousarray(positions, dtype=np.float64).reshape(-1, 3)
    m = np.ascontiguousarray(masses, dtype=np.float64).reshape(-1)
    nb = int(mesh) // 2
    k, pk, nm = np.empty(max(nb, 1)), np.empty(max(nb, 1)), np.empty(max(nb, 1), dtype=np.uint64)
    rc = load().tpm_power_spectrum(_ptr(pos), _ptr(m), pos.shape[0], float(box_size), int(mesh), int(device),
                                   _ptr(k), _ptr(pk), _ptr(nm))
    check(None, rc)
    keep = nm[:nb] > 0
    return k[:nb][keep], pk[:nb][keep], nm[:nb][keep].astype(np.int64)


def zeldovich_config(n_side: int, seed: int = 42, *, transfer: str = "power_law", amplitude: float = 1e-4,
                     spectral_index: float = -2.0, sigma8: float = 0.0, omega_m: float = 1.0,
                     omega_lambda: float = 0.0, omega_b: float = 0.049, h: float = 0.674,
                     box_size_mpc_h: float = 0.0, a_init: float = 1.0, h0: float = 1.0, cosmology: bool = False,
                     rescale_to_a_init: bool = False, use_2lpt: bool = False) -> "TpmZeldovich":
    """IcKind::Zeldovich fields with the defaults of
    crates/gadget-ng-core/src/config/sections/simulation_ic.rs:285-303 (seed
    42, amplitude 1e-4, spectral index -2, omega_b 0.049, h 0.674); transfer
    "power_law" or "eisenstein_hu"."""
    kinds = {"power_law": 0, "eisenstein_hu": 1}
    if transfer not in kinds:
        raise ValueError(f"transfer must be one of {sorted(kinds)}")
    return TpmZeldovich(n_side=int(n_side), transfer=kinds[transfer], seed=int(seed), amplitude=float(amplitude),
                        spectral_index=float(spectral_index), sigma8=float(sigma8), omega_m=float(omega_m),
                        omega_lambda=float(omega_lambda), omega_b=float(omega_b), h=float(h),
                        box_size_mpc_h=float(box_size_mpc_h), a_init=float(a_init), h0=float(h0),
                        cosmology=int(bool(cosmology)), rescale_to_a_init=int(bool(rescale_to_a_init)),
                        use_2lpt=int(bool(use_2lpt)), reserved=0)


def zeldovich_sigma(n_abs, n_side: int, **cfg):
    """sigma(|n|) of the IC spectrum and the factors (A, a^2 f1 H, D(a)/D(1),
    D2/D1^2, a^2 f2 H D2/D1^2)."""
    c = zeldovich_config(n_side, 0, **cfg)
    x = np.ascontiguousarray(n_abs, dtype=np.float64).reshape(-1)
    sig, fac = np.empty_like(x), np.empty(5)
    check(None, load().tpm_zeldovich_sigma(C.byref(c), _ptr(x), x.shape[0], _ptr(sig), _ptr(fac)))
    return sig, tuple(float(v) for v in fac)


def drift_kick_factors(omega_m: float, omega_lambda: float, h0: float, a0: float, dt: float):
    """CosmologyParams::drift_kick_factors (crates/gadget-ng-core/src/cosmology.rs:188-233)."""
    out = np.zeros(3)
    load().tpm_drift_kick_factors(float(omega_m), float(omega_lambda), float(h0), float(a0), float(dt), _ptr(out))
    return float(out[0]), float(out[1]), float(out[2])


def advance_a(omega_m: float, omega_lambda: float, h0: float, a: float, dt: float) -> float:
    """CosmologyParams::advance_a (cosmology.rs:172-178)."""
    return float(load().tpm_advance_a(float(omega_m), float(omega_lambda), float(h0), float(a), float(dt)))


def gravity_coupling_qksl(g: float, a: float) -> float:
    """G·a³ (cosmology.rs:354-356)."""
    return g * a * a * a
