"""B200 (sm_100a) TreePM force path for gadget-ng.

Public surface: `TreePmSolver`, `PmSolver`, `make_solver` (the reference's
GravitySolver contract), cosmology helpers for the KDK integrator, and the
seeded workload generators in `treepm.ics`.
"""
from ._lib import TreePmError, load  # noqa: F401
from .solver import (PmSolver, TreePmSolver, advance_a, drift_kick_factors,  # noqa: F401
                     gravity_coupling_qksl, make_solver, power_spectrum, zeldovich_config,
                     zeldovich_sigma)

__all__ = ["TreePmSolver", "PmSolver", "make_solver", "drift_kick_factors", "advance_a", "gravity_coupling_qksl",
           "power_spectrum", "zeldovich_config", "zeldovich_sigma", "TreePmError", "load"]
