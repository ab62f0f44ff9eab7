"""Learned short-range network (extension; no counterpart in the reference).

A small 3D CNN maps the long-range mesh (density and potential) to the
short-range acceleration at each particle (optionally less the pairs closer
than `near_cells` cells, which the solver then sums exactly over the
neighbouring cells).  A solver created with
`learned=True` and given a trained `Network` (`TreePmSolver.set_learned`)
takes the short range from it for particles whose 8 CIC nodes all have
overdensity <= `delta_max`, and walks the tree only for the rest.

Training data are (long-range, short-range) pairs that the solver itself
produces: `capture` runs the accurate walk on seeded clustered boxes and
stores, for every particle outside dense cells, its short-range acceleration
as the target; `Network.train` runs forward, backward and Adam on the GPU
(BF16 tensor-core convolutions, FP32 accumulation) on random 14^3 patches.
The loss weights each particle by 1 / (|a|^2 + 0.01 <|a|^2>), so it measures
the error relative to the particle's total acceleration.
"""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import ics
from ._lib import TreePmError, load
from .solver import TreePmSolver

C_IN = 10  # ln(1 + rho / m_cell), phi * cell / m_cell, ln(1 + 8 m_octant / m_cell) for 8 octants


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def init_params(c_in: int = C_IN, seed: int = 0) -> np.ndarray:
    """He-normal convolution and head weights (std sqrt(2 / fan_in)), zero biases."""
    rng = np.random.default_rng(seed)
    parts = []
    for cin in (c_in, 16, 16):
        parts.append(rng.normal(0.0, math.sqrt(2.0 / (27 * cin)), 27 * 16 * cin))
        parts.append(np.zeros(16))
    parts.append(rng.normal(0.0, math.sqrt(2.0 / 16), 3 * 16) * 0.1)
    parts.append(np.zeros(3))
    return np.concatenate(parts).astype(np.float32)


class Network:
    """Device-resident network, Adam state and training set (tpm_cnn)."""

    def __init__(self, c_in: int = C_IN, device: int = 0, params=None, seed: int = 0):
        self._lib = load()
        h = C.c_void_p()
        rc = self._lib.tpm_cnn_create(int(c_in), int(device), C.byref(h))
        if rc != 0:
            raise TreePmError(rc, "tpm_cnn_create failed")
        self.h = h
        self.c_in = int(c_in)
        self.n_params = int(self._lib.tpm_cnn_param_count(self.c_in))
        self.set_params(init_params(self.c_in, seed) if params is None else params)

    def _check(self, rc):
        if rc != 0:
            msg = self._lib.tpm_cnn_last_error(self.h) or b""
            raise TreePmError(rc, msg.decode(errors="replace"))

    def close(self):
        if getattr(self, "h", None):
            self._lib.tpm_cnn_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- parameters --------------------------------------------------------
    def set_params(self, params):
        p = np.ascontiguousarray(params, dtype=np.float32).reshape(-1)
        if p.shape[0] != self.n_params:
            raise ValueError(f"expected {self.n_params} parameters, got {p.shape[0]}")
        self._check(self._lib.tpm_cnn_set_params(self.h, _ptr(p), p.shape[0]))

    def params(self) -> np.ndarray:
        p = np.empty(self.n_params, dtype=np.float32)
        self._check(self._lib.tpm_cnn_get_params(self.h, _ptr(p), p.shape[0]))
        return p

    def set_scales(self, shift, scale, out_scale: float, delta_max: float = 200.0):
        sh = np.ascontiguousarray(shift, dtype=np.float32)
        sc = np.ascontiguousarray(scale, dtype=np.float32)
        self._check(self._lib.tpm_cnn_set_scales(self.h, _ptr(sh), _ptr(sc), float(out_scale), float(delta_max)))

    def set_near(self, near_cells: float):
        """Radius (cells) of the exact near-field sum the network complements."""
        self._check(self._lib.tpm_cnn_set_near(self.h, float(near_cells)))

    def near(self) -> float:
        return float(self._lib.tpm_cnn_get_near(self.h))

    def scales(self):
        sh = np.zeros(16, dtype=np.float32)
        sc = np.zeros(16, dtype=np.float32)
        o = C.c_float()
        d = C.c_float()
        self._check(self._lib.tpm_cnn_get_scales(self.h, _ptr(sh), _ptr(sc), C.byref(o), C.byref(d)))
        return sh[: self.c_in].copy(), sc[: self.c_in].copy(), float(o.value), float(d.value)

    # ---- single batches (checks against the CPU restatement) ---------------
    def forward(self, x0):
        x = np.ascontiguousarray(x0, dtype=np.float32)
        B, D = x.shape[0], x.shape[1]
        out = np.empty((B, D - 6, D - 6, D - 6, 3), dtype=np.float32)
        self._check(self._lib.tpm_cnn_forward(self.h, _ptr(x), B, D, _ptr(out)))
        return out

    def loss_grad(self, x0, pb, ps, target, weight):
        x = np.ascontiguousarray(x0, dtype=np.float32)
        pb = np.ascontiguousarray(pb, dtype=np.int32)
        ps = np.ascontiguousarray(ps, dtype=np.float32)
        tg = np.ascontiguousarray(target, dtype=np.float32)
        w = np.ascontiguousarray(weight, dtype=np.float32)
        loss = np.zeros(1, dtype=np.float32)
        grad = np.empty(self.n_params, dtype=np.float32)
        self._check(self._lib.tpm_cnn_loss_grad(self.h, _ptr(x), x.shape[0], x.shape[1], pb.shape[0], _ptr(pb),
                                                _ptr(ps), _ptr(tg), _ptr(w), _ptr(loss), _ptr(grad)))
        return float(loss[0]), grad

    def adam_step(self, grad=None, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8):
        g = None if grad is None else np.ascontiguousarray(grad, dtype=np.float32)
        self._check(self._lib.tpm_cnn_adam_step(self.h, _ptr(g), float(lr), float(beta1), float(beta2), float(eps)))

    # ---- training set and training loop ------------------------------------
    def add_box(self, solver: TreePmSolver, held_out: bool = False):
        self._check(self._lib.tpm_cnn_add_box(self.h, solver._h.h, 1 if held_out else 0))

    def box_count(self, held_out: bool = False) -> int:
        return int(self._lib.tpm_cnn_box_count(self.h, 1 if held_out else 0))

    def train(self, steps: int, batch: int = 64, lr: float = 1e-3, seed: int = 1):
        hist = np.empty(int(steps), dtype=np.float32)
        self._check(self._lib.tpm_cnn_train(self.h, int(steps), int(batch), float(lr), int(seed), _ptr(hist)))
        return hist

    def evaluate(self, held_out: bool = True, batch: int = 64) -> float:
        out = np.zeros(1, dtype=np.float32)
        self._check(self._lib.tpm_cnn_evaluate(self.h, 1 if held_out else 0, int(batch), _ptr(out)))
        return float(out[0])

    # ---- persistence -----------------------------------------------------------
    def save(self, path: str):
        sh, sc, o, d = self.scales()
        np.savez(path, params=self.params(), shift=sh, scale=sc, out_scale=np.float32(o), delta_max=np.float32(d),
                 c_in=np.int32(self.c_in), near_cells=np.float32(self.near()))

    @classmethod
    def load(cls, path: str, device: int = 0) -> "Network":
        z = np.load(path)
        net = cls(int(z["c_in"]), device, params=z["params"])
        net.set_near(float(z["near_cells"]) if "near_cells" in z else 0.0)
        net.set_scales(z["shift"], z["scale"], float(z["out_scale"]), float(z["delta_max"]))
        return net


# ---- training data ------------------------------------------------------------
def training_box(seed: int, side: int = 64, box_size: float = 50.0) -> ics.Box:
    """A seeded clustered box at the benchmark's mean density (cell 0.78 Mpc/h):
    30 % of the particles in 8 Plummer spheres of 10^3 - 3 10^4 particles."""
    return ics.clustered_box(side, box_size, 0.3, 8, min_halo=1e3, max_halo=3e4, seed=seed,
                             name=f"train{side}_s{seed}")


def training_box_mixed(seed: int, side: int = 128) -> ics.Box:
    """A seeded box at the benchmark's cell size (0.78 Mpc/h, L = side * 100 /
    128): even seeds from the displaced-lattice generator at 1.0 cell rms, odd
    seeds from the clustered generator (30 % of the particles in Plummer
    spheres of 10^3 - 10^5 particles, scale radii 0.05 - 0.5 Mpc/h)."""
    box_size = side * 100.0 / 128.0
    if seed % 2 == 0:
        return ics.lattice_box(side, box_size, 1.0, seed=seed, name=f"train{side}_lattice_s{seed}")
    n_halos = max(8, int(200 * (side / 256.0) ** 3))
    return ics.clustered_box(side, box_size, 0.3, n_halos, min_halo=1e3, max_halo=1e5, seed=seed,
                             name=f"train{side}_clustered_s{seed}")


def solver_for(box: ics.Box, mesh: int, device: int = 0, theta: float = 0.5) -> TreePmSolver:
    """The solver configuration the network is trained for and used with
    (training targets with opening angle 0.5; the fallback walk of the
    learned solver may use a wider one)."""
    phys = ics.physics(box, mesh, 1.0)
    return TreePmSolver(mesh, box.box_size, phys["r_split"], r_cut_factor=phys["r_cut_factor"], accurate=True,
                        theta=theta, deconvolve_cic=True, learned=True, device=device)


def capture(net: Network, box: ics.Box, mesh: int, held_out: bool = False, device: int = 0):
    """Run the accurate walk on `box` and add it to the network's training set."""
    phys = ics.physics(box, mesh, 1.0)
    s = solver_for(box, mesh, device)
    s.set_particles(box.positions(), box.mass)
    s.compute_forces(phys["eps2"], phys["g"])
    net.add_box(s, held_out)
    s.close()
