"""Per-step run diagnostics: the quantities gadget-ng writes to
diagnostics.jsonl (crates/gadget-ng-cli/src/engine/diagnostics.rs:28-90 and
crates/gadget-ng-core/src/cosmology.rs:276-327), computed from host copies of
the state.  Velocities are the canonical momenta the solver stores
(p = a² dx/dt), as in the reference.

Sums here are numpy's (pairwise), not the reference's left-to-right order:
these are run reports, not parity checks.
"""
from __future__ import annotations

import numpy as np


def record(pos, vel, mass, a=None) -> dict:
    """kinetic_energy, momentum, angular_momentum, com, mass_total (and
    v_rms = sqrt(<|p/a|²>) when a is given)."""
    pos = np.asarray(pos, dtype=np.float64)
    vel = np.asarray(vel, dtype=np.float64)
    m = np.asarray(mass, dtype=np.float64)
    mt = float(m.sum())
    mv = vel * m[:, None]
    out = {
        "kinetic_energy": float(0.5 * np.sum(m * np.einsum("ij,ij->i", vel, vel))),
        "momentum": mv.sum(axis=0).tolist(),
        "angular_momentum": np.cross(pos, mv).sum(axis=0).tolist(),
        "com": (np.sum(pos * m[:, None], axis=0) / mt).tolist() if mt > 0 else [0.0, 0.0, 0.0],
        "mass_total": mt,
    }
    if a is not None:
        out["a"] = float(a)
        out["v_rms"] = float(np.sqrt(np.mean(np.einsum("ij,ij->i", vel, vel)) / (a * a)))
    return out


def force_momentum_residual(acc, mass) -> float:
    """|Σ m·a| / max_i m_i|a_i|: the momentum-conservation figure of the
    reference's treepm_momentum_conserved test
    (crates/gadget-ng-treepm/tests/treepm_vs_direct.rs:75-113, bound 1e-3)."""
    acc = np.asarray(acc, dtype=np.float64)
    m = np.asarray(mass, dtype=np.float64)
    s = np.linalg.norm((acc * m[:, None]).sum(axis=0))
    scale = max(float(np.max(np.linalg.norm(acc, axis=1) * m)), 1e-30)
    return float(s / scale)
