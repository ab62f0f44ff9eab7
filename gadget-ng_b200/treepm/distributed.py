"""Domain-decomposed TreePM: one GPU (one solver handle) per rank.

The reference's distributed TreePM with SFC domains
(crates/gadget-ng-cli/src/engine/stepping/mod.rs:1044-1250, `treepm_sr_sfc`):

* domains: `SfcDecomposition::build_with_bbox_and_kind`
  (crates/gadget-ng-parallel/src/sfc.rs:336-393) -- Hilbert keys over the
  all-ranks bounding box, cut points at count quantiles, `rank_for`
  (sfc.rs:499-504); `exchange_domain_sfc` (src/mpi_rt.rs:426-450) moves each
  particle to its key's rank;
* short range: `exchange_halos_3d_periodic` (src/mpi_rt.rs:723-781) -- AABB of
  each rank's particles, allgather, every particle within r_cut
  (periodic, `min_dist2_to_aabb_3d_periodic`) of another rank's AABB sent
  there -- then `short_range_accels_sfc`
  (crates/gadget-ng-treepm/src/distributed.rs:119-145): a tree of owned + halo
  particles walked for the owned ones;
* long range: the PM of the all-ranks density; each rank deposits its own
  particles and the meshes are summed (`allreduce_sum_f64_slice`,
  crates/gadget-ng-parallel/src/lib.rs:200-210), so every rank solves the
  same global mesh and gathers for its own particles.

The device work is the library's (`tpm_halo_select`, `tpm_set_halos`,
`tpm_force_begin` / `_short_range` / `_end`, `tpm_kick_drift`); the exchanges
are torch.distributed collectives.  With NCCL the halo records and the density
stay on the device and the density all-reduce runs on a side stream while the
walk runs; with gloo (CPU tests, several ranks sharing one GPU) they are
staged through host memory.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._lib import check
from .solver import TreePmSolver, _ptr

class _DeviceArray:
    """A library-owned device buffer seen by torch without a copy
    (__cuda_array_interface__)."""

    def __init__(self, ptr: int, count: int, typestr: str):
        self.__cuda_array_interface__ = {"shape": (int(count),), "typestr": typestr, "data": (int(ptr), False),
                                         "version": 2}


def aabb_is_valid(a) -> bool:
    """Aabb3::is_valid (crates/gadget-ng-parallel/src/halo3d.rs)."""
    return bool(a[0] <= a[1] and a[2] <= a[3] and a[4] <= a[5])


def union_bbox(aabbs):
    """global_bbox (sfc.rs:570-620): min / max over the valid per-rank boxes;
    (0, 0, ...) when every rank is empty."""
    valid = [a for a in aabbs if aabb_is_valid(a)]
    if not valid:
        return np.zeros(6)
    v = np.asarray(valid)
    return np.array([v[:, 0].min(), v[:, 1].max(), v[:, 2].min(), v[:, 3].max(), v[:, 4].min(), v[:, 5].max()])


def cutpoints_from_keys(sorted_keys: np.ndarray, n_ranks: int) -> np.ndarray:
    """Cut points of build_with_bbox_and_kind (sfc.rs:370-377): key index
    r n / P for r = 1..P-1 of the sorted keys; u64::MAX / P each when empty."""
    n = sorted_keys.shape[0]
    if n == 0:
        return np.full(n_ranks - 1, np.iinfo(np.uint64).max // np.uint64(n_ranks), dtype=np.uint64)
    idx = np.minimum((np.arange(1, n_ranks, dtype=np.int64) * n) // n_ranks, n - 1)
    return sorted_keys[idx].astype(np.uint64)


def rank_for(keys: np.ndarray, cutpoints: np.ndarray, n_ranks: int) -> np.ndarray:
    """SfcDecomposition::rank_for (sfc.rs:499-504): binary search of the cut
    points, a key equal to cut point i going to rank i + 1, capped at P - 1."""
    r = np.searchsorted(cutpoints, keys, side="right")
    return np.minimum(r, n_ranks - 1).astype(np.int64)


class _Exchange:
    """The collectives of ParallelRuntime this path uses, over a
    torch.distributed process group."""

    def __init__(self, group, device):
        import torch
        import torch.distributed as dist
        self.torch, self.dist, self.group = torch, dist, group
        self.rank = dist.get_rank(group)
        self.size = dist.get_world_size(group)
        self.device = device
        self.on_device = dist.get_backend(group) == "nccl"

    def _home(self, t):
        return t.to(self.device) if self.on_device else t.cpu()

    def allgather_f64(self, local: np.ndarray) -> np.ndarray:
        """allgather_f64 (lib.rs:212-218): (size, len) array."""
        torch = self.torch
        t = self._home(torch.from_numpy(np.ascontiguousarray(local, dtype=np.float64)))
        out = [torch.empty_like(t) for _ in range(self.size)]
        self.dist.all_gather(out, t, group=self.group)
        return np.stack([o.cpu().numpy() for o in out])

    def allgather_u32(self, local: np.ndarray) -> np.ndarray:
        """allgather of uint32 words: (size, len) array."""
        torch = self.torch
        t = self._home(torch.from_numpy(np.ascontiguousarray(local, dtype=np.uint32).view(np.int32)))
        out = [torch.empty_like(t) for _ in range(self.size)]
        self.dist.all_gather(out, t, group=self.group)
        return np.stack([o.cpu().numpy().view(np.uint32) for o in out])

    def alltoall_counts(self, counts: np.ndarray) -> np.ndarray:
        torch = self.torch
        send = self._home(torch.from_numpy(np.ascontiguousarray(counts, dtype=np.int64)))
        recv = torch.empty_like(send)
        self.dist.all_to_all_single(recv, send, group=self.group)
        return recv.cpu().numpy()

    def alltoallv_bytes(self, send, send_bytes, recv_bytes):
        """alltoallv (lib.rs:220-226) of byte buffers: send (device tensor),
        per-rank byte counts; returns the receive tensor on the device."""
        torch = self.torch
        total = int(np.sum(recv_bytes))
        if self.on_device:
            recv = torch.empty(max(total, 1), dtype=torch.uint8, device=self.device)
            self.dist.all_to_all_single(recv[:total], send[:int(np.sum(send_bytes))], [int(x) for x in recv_bytes],
                                        [int(x) for x in send_bytes], group=self.group)
            return recv
        recv = torch.empty(max(total, 1), dtype=torch.uint8)
        self.dist.all_to_all_single(recv[:total], send[:int(np.sum(send_bytes))].cpu(), [int(x) for x in recv_bytes],
                                    [int(x) for x in send_bytes], group=self.group)
        return recv.to(self.device)

    def reduce_scatter_sum_(self, out, t) -> None:
        """reduce_scatter of t (equal contiguous chunks, rank order) into out:
        out = the sum over ranks of this rank's chunk (gloo: all-reduce, then
        the chunk)."""
        if self.on_device:
            self.dist.reduce_scatter_tensor(out, t, group=self.group)
            return
        c = t.cpu()
        self.dist.all_reduce(c, group=self.group)
        n = out.numel()
        out.copy_(c[self.rank * n:(self.rank + 1) * n])

    def alltoall_equal_(self, out, t) -> None:
        """all-to-all of equal contiguous chunks (rank order) from t into out."""
        if self.on_device:
            self.dist.all_to_all_single(out, t, group=self.group)
            return
        o = self.torch.empty_like(out, device="cpu")
        self.dist.all_to_all_single(o, t.cpu(), group=self.group)
        out.copy_(o)

    def allgather_into_(self, out, t) -> None:
        """all-gather of equal chunks t (rank order) into out."""
        if self.on_device:
            self.dist.all_gather_into_tensor(out, t, group=self.group)
            return
        parts = [self.torch.empty_like(t, device="cpu") for _ in range(self.size)]
        self.dist.all_gather(parts, t.cpu(), group=self.group)
        out.copy_(self.torch.cat(parts))

    def allreduce_sum_(self, t) -> None:
        """allreduce_sum_f64_slice (lib.rs:200-210) in place on a device tensor."""
        if self.on_device:
            self.dist.all_reduce(t, group=self.group)
        else:
            c = t.cpu()
            self.dist.all_reduce(c, group=self.group)
            t.copy_(c)


class DomainTreePm:
    """One rank of the domain-decomposed TreePM (constructor keys as
    `TreePmSolver`; the periodic walk).  `group` is the torch.distributed
    process group (default: the world).  `halo`: "aabb" selects halos by the
    reference's rule (within r_cut of another rank's particle AABB); "cells"
    by the cells that rank occupies on a grid at least r_cut wide, which keeps
    every pair within r_cut and sends far fewer particles once domains are
    not slabs (the short-range trees then differ from the reference's).
    `pm`: "replicated" sums the density mesh on every rank and solves it
    everywhere (allreduce_sum_f64_slice, lib.rs:200-210); "slab" splits the
    solve into z slabs with two all-to-all transposes (slab_fft.rs:209-330,
    the reference's pm_slab path; pm_grid_size a multiple of the rank count)
    and all-gathers the force meshes for the gather."""

    def __init__(self, grid_size: int, box_size: float, r_split: float = 0.0, *, r_cut_factor: float = 5.0,
                 device: int = 0, group=None, overlap: bool = True, halo: str = "aabb", pm: str = "replicated"):
        if halo not in ("aabb", "cells"):
            raise ValueError("halo is 'aabb' or 'cells'")
        if pm not in ("replicated", "slab"):
            raise ValueError("pm is 'replicated' or 'slab'")
        self.halo = halo
        self.pm = pm
        import torch
        import torch.distributed as dist
        if not dist.is_initialized():
            raise RuntimeError("DomainTreePm needs an initialised torch.distributed process group")
        self.torch = torch
        self.solver = TreePmSolver(grid_size, box_size, r_split, r_cut_factor=r_cut_factor, device=device)
        self.box_size = float(box_size)
        nm = int(grid_size)
        r_s = float(r_split) if r_split > 0 else 2.5 * self.box_size / nm
        self.r_cut = (float(r_cut_factor) if r_cut_factor > 0 else 5.0) * r_s
        self.device = torch.device("cuda", int(device))
        self.ex = _Exchange(group, self.device)
        if self.ex.size > _lib.MAX_RANKS:
            raise ValueError(f"at most {_lib.MAX_RANKS} ranks")
        self.overlap = overlap and self.ex.on_device
        self._h = self.solver._h
        self._L = self._h._lib
        self.gid = np.zeros(0, dtype=np.int64)  # global ids of the owned particles, owned order
        self.mass = np.zeros(0)
        self._forces = None
        self.last_halo_count = 0
        self.last_halo_sent = 0
        self._stream = None
        self._side = None
        self._slab = None

    # ---- particles -----------------------------------------------------------
    def set_particles(self, pos, mass, vel=None, gid=None):
        """This rank's owned particles (n x 3 float64 positions, momenta, masses)."""
        pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
        self.mass = np.ascontiguousarray(mass, dtype=np.float64).reshape(-1).copy()
        self.solver.set_particles(pos, self.mass, vel)
        self._forces = None  # (eps2, g) of the accelerations held, if any
        self.gid = (np.arange(pos.shape[0], dtype=np.int64) if gid is None else np.asarray(gid, dtype=np.int64))

    @property
    def n_owned(self) -> int:
        no, nr = C.c_int64(), C.c_int64()
        check(self._h.h, self._L.tpm_particle_counts(self._h.h, C.byref(no), C.byref(nr)))
        return no.value

    def get_state(self):
        """(gid, pos, vel, acc) of the owned particles."""
        n = self.n_owned
        p, v, a = self.solver.get_state(n, True, True, True)
        return self.gid.copy(), p, v, a

    # ---- exchanges -----------------------------------------------------------
    def owned_aabb(self) -> np.ndarray:
        out = np.empty(6)
        check(self._h.h, self._L.tpm_owned_aabb(self._h.h, _ptr(out)))
        return out

    def exchange_halos(self) -> int:
        """exchange_halos_3d_periodic: returns the number of halo particles
        received (now resident in the handle)."""
        torch = self.torch
        ex = self.ex
        h = self._h.h
        counts = np.zeros(ex.size, dtype=np.int64)
        if self.halo == "aabb":
            table = np.ascontiguousarray(ex.allgather_f64(self.owned_aabb()).reshape(-1))

            def select(send, cap):
                check(h, self._L.tpm_halo_select(h, _ptr(table), ex.size, ex.rank, float(self.r_cut), _ptr(counts),
                                                 send, cap))
        else:
            grid = C.c_int32()
            check(h, self._L.tpm_occupancy(h, float(self.r_cut), C.byref(grid), None))
            words = (grid.value ** 3 + 31) // 32
            mine = np.zeros(words, dtype=np.uint32)
            check(h, self._L.tpm_occupancy(h, float(self.r_cut), C.byref(grid), _ptr(mine)))
            table = np.ascontiguousarray(ex.allgather_u32(mine).reshape(-1))

            def select(send, cap):
                check(h, self._L.tpm_halo_select_cells(h, _ptr(table), grid.value, ex.size, ex.rank,
                                                       float(self.r_cut), _ptr(counts), send, cap))
        select(None, 0)
        total = int(counts.sum())
        rb = _lib.HALO_RECORD_BYTES
        send = torch.empty(max(total * rb, rb), dtype=torch.uint8, device=self.device)
        if total:
            select(C.c_void_p(send.data_ptr()), total)
        recv_counts = ex.alltoall_counts(counts)
        recv = ex.alltoallv_bytes(send, counts * rb, recv_counts * rb)
        if ex.on_device:
            torch.cuda.current_stream(self.device).synchronize()
        n_halo = int(recv_counts.sum())
        check(h, self._L.tpm_set_halos(h, C.c_void_p(recv.data_ptr()) if n_halo else None, n_halo))
        self.last_halo_count = n_halo
        self.last_halo_sent = total
        return n_halo

    def _mesh_tensor(self):
        ptr, cells = C.c_void_p(), C.c_int64()
        check(self._h.h, self._L.tpm_mesh_density(self._h.h, C.byref(ptr), C.byref(cells)))
        return self.torch.as_tensor(_DeviceArray(ptr.value, cells.value, "<f4"), device=self.device)

    def _streams(self):
        if self._stream is None:
            torch = self.torch
            self._stream = torch.cuda.ExternalStream(self._L.tpm_get_stream(self._h.h), device=self.device)
            self._side = torch.cuda.Stream(device=self.device)
        return self._stream, self._side

    def _slab_buffers(self):
        if self._slab is None:
            b = _lib.TpmSlabBuffers()
            check(self._h.h, self._L.tpm_pm_slab_setup(self._h.h, self.ex.rank, self.ex.size, C.byref(b)))
            dev = self.device
            t = lambda ptr, n, ts: self.torch.as_tensor(_DeviceArray(ptr, n, ts), device=dev)
            self._slab = dict(
                rho=t(b.density_slab, b.slab_cells, "<f4"),
                send=t(b.send, b.return_bytes, "|u1"), recv=t(b.recv, b.return_bytes, "|u1"),
                fwd=int(b.forward_bytes), ret=int(b.return_bytes),
                force_slab=t(b.force_slab, 3 * b.slab_cells, "<f4"), force=t(b.force_mesh, 3 * b.mesh_cells, "<f4"),
                slab_cells=int(b.slab_cells), mesh_cells=int(b.mesh_cells))
        return self._slab

    def _slab_solve(self) -> None:
        """The z-slab PM solve (tpm_pm_slab_*): reduce-scatter of the density,
        forward transpose, z passes, return transpose, all-gather of the force
        slabs into the meshes the gather reads."""
        h, L, ex = self._h.h, self._L, self.ex
        sb = self._slab_buffers()
        ext, _ = self._streams()
        sync = lambda: (ext.synchronize(), self.torch.cuda.synchronize(self.device))
        sync()
        ex.reduce_scatter_sum_(sb["rho"], self._mesh_tensor())
        sync()
        check(h, L.tpm_pm_slab_forward(h))
        sync()
        ex.alltoall_equal_(sb["recv"][:sb["fwd"]], sb["send"][:sb["fwd"]])
        sync()
        check(h, L.tpm_pm_slab_poisson(h))
        sync()
        ex.alltoall_equal_(sb["recv"][:sb["ret"]], sb["send"][:sb["ret"]])
        sync()
        check(h, L.tpm_pm_slab_inverse(h))
        sync()
        n, m = sb["slab_cells"], sb["mesh_cells"]
        for c in range(3):
            ex.allgather_into_(sb["force"][c * m:(c + 1) * m], sb["force_slab"][c * n:(c + 1) * n])
        sync()

    def _force(self, eps2: float, g: float, kick: float) -> None:
        """Force evaluation of the owned particles with the current halos:
        deposit -> density all-reduce (overlapped with the walk on NCCL) ->
        FFT solve -> gather (+ kick); with pm="slab" the solve is split over
        the ranks (_slab_solve) and runs before the walk."""
        h = self._h.h
        L = self._L
        check(h, L.tpm_force_begin(h))
        if self.pm == "slab":
            self._slab_solve()
            check(h, L.tpm_force_short_range(h, float(eps2)))
            check(h, L.tpm_force_end_solved(h, float(g), float(kick)))
            self._forces = (float(eps2), float(g))
            return
        mesh = self._mesh_tensor()
        if self.overlap:
            ext, side = self._streams()
            side.wait_stream(ext)
            with self.torch.cuda.stream(side):
                self.ex.allreduce_sum_(mesh)
            check(h, L.tpm_force_short_range(h, float(eps2)))
            ext.wait_stream(side)
        else:
            ext, _ = self._streams()
            ext.synchronize()
            self.ex.allreduce_sum_(mesh)
            self.torch.cuda.synchronize(self.device)
            check(h, L.tpm_force_short_range(h, float(eps2)))
        check(h, L.tpm_force_end(h, float(g), float(kick)))
        self._forces = (float(eps2), float(g))

    # ---- the solver calls ------------------------------------------------------
    def compute_forces(self, eps2: float, g: float) -> None:
        """Accelerations of the owned particles (kept on the device)."""
        self.exchange_halos()
        self._force(eps2, g, 0.0)

    def accelerations(self, eps2: float, g: float) -> np.ndarray:
        """Owned particles' accelerations (n x 3), owned order."""
        self.compute_forces(eps2, g)
        return self.get_state()[3]

    def force_parts(self):
        """(long range, short range) of the owned particles from the last evaluation."""
        return self.solver.force_parts(self.n_owned)

    def interaction_counts(self):
        return self.solver.interaction_counts(self.n_owned)

    def kdk_step(self, kick_half: float, drift: float, kick_half2: float, eps2: float, g: float) -> None:
        """leapfrog_cosmo_kdk_step over the decomposed domain: opening kick +
        drift (owned), halo exchange at the new positions, force evaluation
        with the closing kick fused into the gather."""
        if self._forces is None or self._forces[0] != float(eps2):
            self.compute_forces(eps2, g)
        check(self._h.h, self._L.tpm_kick_drift(self._h.h, float(kick_half), float(drift), float(g)))
        self.exchange_halos()
        self._force(eps2, g, kick_half2)

    # ---- SFC domains -----------------------------------------------------------
    def sfc_keys(self, bbox6, kind: str = "morton") -> np.ndarray:
        """SfcKind keys of the owned particles over bbox6 (owned order)."""
        keys = np.empty(self.n_owned, dtype=np.uint64)
        check(self._h.h, self._L.tpm_sfc_keys(self._h.h, _ptr(np.ascontiguousarray(bbox6, dtype=np.float64)),
                                              _lib.SFC_KINDS[kind], _ptr(keys)))
        return keys

    def redistribute(self, sample: int = 4096, kind: str = "morton") -> None:
        """exchange_domain_sfc with a fresh SfcDecomposition: keys of `kind`
        (the reference's SfcKind) over the all-ranks bounding box; cut points at
        the count quantiles of a regular sample of every rank's sorted keys
        (every key when a rank holds at most `sample`); particles move to
        rank_for(key).  Morton by default: the reference's Hilbert keys pack the
        finest coordinate bits first, so their domains span the whole box and
        the AABB halo rule then sends every particle to every rank.
        Accelerations are recomputed by the next force evaluation."""
        ex = self.ex
        bbox = union_bbox(ex.allgather_f64(self.owned_aabb()))
        keys = self.sfc_keys(bbox, kind)
        sk = np.sort(keys)
        m = sk.shape[0]
        take = sk if m <= sample else sk[(np.arange(sample, dtype=np.int64) * m) // sample]
        counts = ex.allgather_f64(np.array([float(take.shape[0])]))[:, 0].astype(np.int64)
        width = max(int(counts.max()), 1)
        pad = np.zeros(width, dtype=np.float64)
        pad[:take.shape[0]] = take.view(np.float64) if take.shape[0] else pad[:0]
        allk = ex.allgather_f64(pad)
        pooled = np.concatenate([allk[r, :counts[r]].view(np.uint64) for r in range(ex.size)])
        cut = cutpoints_from_keys(np.sort(pooled), ex.size)
        dest = rank_for(keys, cut, ex.size)
        gid, pos, vel, _ = self.get_state()
        mass = self.mass
        order = np.argsort(dest, kind="stable")
        send_counts = np.bincount(dest, minlength=ex.size).astype(np.int64)
        rec = np.empty((pos.shape[0], 8))
        rec[:, 0] = gid.view(np.float64)
        rec[:, 1] = mass
        rec[:, 2:5] = pos
        rec[:, 5:8] = vel
        rec = np.ascontiguousarray(rec[order])
        torch = self.torch
        send = torch.from_numpy(rec.view(np.uint8).reshape(-1)).to(self.device)
        recv_counts = ex.alltoall_counts(send_counts)
        recv = ex.alltoallv_bytes(send, send_counts * 64, recv_counts * 64).cpu().numpy()
        got = recv[:int(recv_counts.sum()) * 64].view(np.float64).reshape(-1, 8)
        self.set_particles(got[:, 2:5], got[:, 1], got[:, 5:8], gid=got[:, 0].copy().view(np.int64))

    def close(self):
        self.solver._h.close()
