"""Benchmark: TreePM particle-updates/s on the 256³ clustered box (one GPU per rank).

A step is one cosmological KDK step of every particle (leapfrog_cosmo_kdk_step
of the reference + the periodic wrap): opening half kick, drift, one TreePM
force evaluation (keys, sort, octree, short-range walk, PM), closing half kick.
The fused step reuses the previous step's closing acceleration for its opening
kick; the reference evaluates the force twice per step, and the JSON line also
reports the per-force-evaluation rate.  The workload is a trajectory of 10 KDK
steps with one global dt from a = 0.1 to 0.12; timed steps are steps of that
trajectory, and an untimed pass over it reports per-step diagnostics and FP64
Ewald errors.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--workload clustered256]
  python bench.py --impl reference ...   # the CPU restatement of the reference

Multi-GPU (N > 1): the domain-decomposed solver (SFC domains, periodic halos,
density all-reduce) on one box split over the ranks, "scaling": "strong";
``--replicas`` runs N independent copies instead ("scaling": "weak").
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
LEARNED_THETA = 0.57
sys.path.insert(0, os.path.join(REPO, "gadget-ng_b200"))

WORKLOADS = {
    # name: (generator, mesh, a_start, a_end over 10 steps)
    "clustered256": ("clustered_box_256", 256, 0.1, 0.12),
    "treepm128": ("treepm_box_128", 128, 0.1, 0.12),
    "treepm64": ("treepm_box_64", 64, 0.1, 0.12),
    "clustered512": ("clustered_box_512", 512, 0.1, 0.12),
    "pm64": ("pm_box_64", 64, 0.02, 0.0202),
    # profiling case for the mesh kernels: the 256^3 mesh (working set above
    # the 126 MB L2) with 128^3 particles
    "treepm128_mesh256": ("treepm_box_128", 256, 0.1, 0.12),
}
FLOP_PER_INTERACTION = 37  # FMA = 2, MUFU = 1: the pair-kernel convention of the cost model
TRAJ_STEPS = 10  # KDK steps from a_start to a_end, one global dt


def trajectory(a0, a1, G, steps=TRAJ_STEPS, total=None):
    """(drift, kick_half, kick_half2, coupling G·a³) of each of `steps` KDK
    steps with one global dt from a0 to a1 (continued with the same dt to
    `total` steps when given), and the scale factor after each step
    (a_of[i] = a after i steps)."""
    import treepm
    from treepm import ics
    dt = ics.time_between(a0, a1) / steps
    a, factors, a_of = a0, [], [a0]
    for _ in range(total or steps):
        d, k1, k2 = treepm.drift_kick_factors(ics.OMEGA_M, ics.OMEGA_L, ics.H0_INTERNAL, a, dt)
        factors.append((d, k1, k2, G * a ** 3))
        a = treepm.advance_a(ics.OMEGA_M, ics.OMEGA_L, ics.H0_INTERNAL, a, dt)
        a_of.append(a)
    return factors, a_of


def env_rank():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def max_over_ranks(x: float, device) -> float:
    """The maximum of a per-rank time over all ranks (barrier first); the
    value itself on one rank."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.barrier()
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def whole_job_rate(units_per_rank: int, steps: int, seconds: float, world: int) -> float:
    """Units processed by all ranks per second of the slowest rank (replicas:
    every rank processes the same workload)."""
    return world * units_per_rank * steps / seconds


def make_box(name):
    from treepm import ics
    gen, mesh, a0, a1 = WORKLOADS[name]
    return getattr(ics, gen)(), mesh, a0, a1


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = float(p[2])
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    try:
        with open(os.path.join(REPO, "MEASURED_PEAKS.json")) as f:
            return json.load(f)
    except OSError:
        return {}


# DRAM bytes (read + write) of one k_walk launch on these workloads, from
# single-pass ncu captures of dram__bytes_read.sum + dram__bytes_write.sum made
# outside the bench (ncu cannot run inside a timed bench); reported with that label.
WALK_DRAM_BYTES = {"clustered256_L200": 963312384 + 368289792, "treepm128_L100": 144405760 + 69206272}


def profile_traffic(workload):
    """DRAM bytes per walk launch measured by ncu for this workload, if captured."""
    return WALK_DRAM_BYTES.get(workload)


def stage_rooflines(stage_ms, n, mesh):
    """HBM rooflines of the memory-bound stages from their algorithmic bytes per
    evaluation (keys + radix sort 68 B per particle; PM deposit + forward +
    three inverse transforms 12 N + 36 N_c with the spectral step fused; gather
    + kick 12 N_c + 36 N) against the measured copy bandwidth."""
    peak = measured_peaks().get("hbm_gbs") or 6650.0
    nc = mesh ** 3
    out = {}
    for name, key, nbytes in (("keys_sort", ("ms_bbox_keys", "ms_sort"), 68 * n),
                              ("pm", ("ms_pm",), 12 * n + 36 * nc),
                              ("gather_kick", ("ms_gather_kick",), 12 * nc + 36 * n)):
        ms = sum(stage_ms.get(k, 0.0) for k in key)
        if ms > 0:
            gbs = nbytes / (ms * 1e-3) / 1e9
            out[name] = {"bytes": nbytes, "ms": ms, "achieved_gbs": gbs, "peak_gbs": peak, "frac": gbs / peak}
    out["peak_source"] = "MEASURED_PEAKS.json hbm_gbs (measured)" if measured_peaks().get("hbm_gbs") else "fallback"
    return out


def sample_targets(n, n_targets, blocks=64, seed=12345):
    """Walk targets of the CPU sample: one run of consecutive particle indices
    at a seeded offset in each of `blocks` equal strata of the index range.
    The workloads store particles in spatial order (lattice part, then the
    halos), so the strata cover both in proportion, and a run keeps the cache
    locality of the full walk (neighbouring targets share tree nodes);
    scattered single targets walk slower per target than the full evaluation."""
    n_targets = min(n_targets, n)
    blocks = max(1, min(blocks, n_targets))
    blk = n_targets // blocks
    stratum = n // blocks
    rng = np.random.default_rng(seed)
    starts = np.arange(blocks) * stratum + rng.integers(0, stratum - blk + 1, blocks)
    return (starts[:, None] + np.arange(blk)[None, :]).ravel().astype(np.int64)


def cpu_sample(box, mesh, phys, n_targets, threads):
    """The oracle restatement on a bounded sample: full PM + full tree build +
    the walk of n_targets seeded targets (runs of consecutive particles),
    extrapolated to all particles."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle
    oracle.build()
    oracle.set_threads(threads)
    pos = box.positions()
    tg = sample_targets(box.n, n_targets)
    r = oracle.treepm(pos, box.mass, phys["eps2"], phys["g"], mesh, box.box_size, phys["r_split"],
                      phys["r_cut_factor"], targets=tg)
    t_pm, t_build, t_walk, _ = (float(x) for x in r["times"])
    t_force = t_pm + t_build + t_walk * box.n / len(tg)
    return t_force, dict(pm_s=t_pm, build_s=t_build, walk_s=t_walk, targets=int(len(tg)), threads=threads)


def cpu_full(box, mesh, phys, threads):
    """One complete force evaluation by the oracle restatement: every
    particle's walk, nothing extrapolated.  Returns seconds and stage times."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import oracle
    oracle.build()
    oracle.set_threads(threads)
    pos = box.positions()
    r = oracle.treepm(pos, box.mass, phys["eps2"], phys["g"], mesh, box.box_size, phys["r_split"],
                      phys["r_cut_factor"], targets=np.arange(box.n, dtype=np.int64))
    t_pm, t_build, t_walk, _ = (float(x) for x in r["times"])
    return t_pm + t_build + t_walk, dict(pm_s=t_pm, build_s=t_build, walk_s=t_walk)


def cpu_kick_drift(box, threads):
    """The O(N) part of a KDK step on the host, timed over every particle:
    opening half kick, drift with the periodic wrap, closing half kick
    (leapfrog.rs:72-91), float64, split over `threads` numpy workers (the
    accelerations are stand-ins of the right shape: the arithmetic does not
    depend on their values).  Seconds."""
    from concurrent.futures import ThreadPoolExecutor
    x = box.positions()
    v = np.zeros_like(x)
    acc = np.random.default_rng(0).standard_normal(x.shape)
    L = box.box_size
    bounds = np.linspace(0, box.n, threads + 1).astype(np.int64)

    def part(i):
        s = slice(bounds[i], bounds[i + 1])
        xs, vs, a = x[s], v[s], acc[s]
        vs += 0.5 * a
        xs += 0.01 * vs
        np.mod(xs, L, out=xs)
        vs += 0.5 * a

    with ThreadPoolExecutor(max_workers=threads) as pool:
        t0 = time.perf_counter()
        list(pool.map(part, range(threads)))
        return time.perf_counter() - t0


def run_reference(args):
    rank, world, _ = env_rank()
    if rank != 0:
        return 0
    box, mesh, a0, a1 = make_box(args.workload)
    from treepm import ics
    phys = ics.physics(box, mesh, a0)
    threads = os.cpu_count() or 1
    times, kd = [], []
    for i in range(args.warmup + args.steps):
        t_force, info = cpu_sample(box, mesh, phys, args.cpu_targets, threads)
        t_kd = cpu_kick_drift(box, threads)
        if i >= args.warmup:
            times.append(2.0 * t_force + t_kd)  # the reference evaluates the force twice per KDK step
            kd.append(t_kd)
    step_s = float(np.mean(times))
    value = box.n / step_s
    full = None
    if not args.no_cpu_full:
        t_full, finfo = cpu_full(box, mesh, phys, threads)
        full = {"seconds": t_full, "extrapolated_seconds": step_s / 2.0, "ratio_full_over_extrapolated":
                t_full / (step_s / 2.0), **finfo,
                "note": "one force evaluation with every particle's walk (no extrapolation), after the timed steps"}
    kd_s = float(np.mean(kd)) if kd else 0.0
    line = {
        "impl": "reference", "metric": "particle-updates/s", "value": value, "unit": "particle-updates/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_s * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": box.name, "particles": box.n, "mesh": mesh, "box_mpc_h": box.box_size,
                   "r_s_cells": 1.25, "r_cut_over_r_s": 4.5},
        "cpu_baseline": {"value": value, "unit": "particle-updates/s", "cores": threads, "kind": "port",
                         "sample": (f"oracle restatement (C++/OpenMP, FP64) of the reference TreePM: full CIC+FFT PM "
                                    f"and full insertion-octree build over {box.n} particles, periodic walk of "
                                    f"{info['targets']} seeded targets (one run of consecutive particles in each of 64 strata) extrapolated "
                                    f"to all; 2 force evaluations "
                                    f"per KDK step as leapfrog.rs:79,86, plus the kick-drift-kick over all particles "
                                    f"(numpy float64, {threads} threads, {kd_s * 1e3:.1f} ms per step)")},
        "full_force_evaluation": full,
        "e2e": {"value": value, "unit": "particle-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def fp32_peak_tflops(lib_solver):
    """FFMA throughput of this GPU, measured live (no FP32 figure is in MEASURED_PEAKS.json)."""
    import torch
    from treepm import _lib
    L = _lib.load()
    import ctypes
    out = ctypes.c_double(0.0)
    if L.tpm_fp32_peak(int(torch.cuda.current_device()), ctypes.byref(out)) != 0:
        return None
    return out.value


def accurate_mode_report(box, mesh, phys, pos, g, targets, ref, device, reps=3):
    """Speed and Ewald error of the extension mode (complete split kernel,
    CIC deconvolution) on the bench's final state, with the opening angle 0.5
    and with the relative opening criterion at the reference's default
    tolerance (err_tol_force_acc = 0.005)."""
    import treepm
    from treepm import accuracy

    def one(**crit):
        s = treepm.TreePmSolver(mesh, box.box_size, phys["r_split"], r_cut_factor=phys["r_cut_factor"],
                                accurate=True, deconvolve_cic=True, device=device, **crit)
        s.set_particles(pos, box.mass)
        for _ in range(2):
            s.compute_forces(phys["eps2"], g)
        ms, inter = [], []
        for _ in range(reps):
            s.compute_forces(phys["eps2"], g)
            st = s.stats()
            ms.append(st["ms_total"])
            inter.append(st["leaf_pairs"] + st["monopoles"])
        _, _, acc = s.get_state(box.n, pos=False, vel=False)
        rms, p99 = accuracy.relative_errors(acc[targets], ref)
        s.close()
        m = float(np.mean(ms))
        return {"ms_per_force_evaluation": m, "particle_updates_per_s": box.n / (m * 1e-3),
                "interactions_per_particle": float(np.mean(inter)) / box.n,
                "force_error_vs_ewald": {"rms": rms, "p99": p99, "targets": int(len(targets))}}

    out = {"flags": "accurate | deconvolve_cic", "theta": 0.5}
    out.update(one(theta=0.5))
    out["relative_criterion"] = dict(err_tol_force_acc=0.005, **one(opening_criterion=1, err_tol_force_acc=0.005))
    return out


def learned_mode_report(box, mesh, phys, pos, g, targets, ref, device, plain_ms, reps=3, path=None, deltas=None):
    """Speed and Ewald error of the learned short range (network outside
    dense cells, accurate walk inside them) on the bench's final state; with
    `deltas`, once per overdensity threshold of the fallback (cells above it
    keep the walk)."""
    import treepm
    from treepm import accuracy, learned
    path = path or os.path.join(REPO, "gadget-ng_b200", "treepm", "weights", "learned_sr.npz")
    if not os.path.exists(path):
        return {"unavailable": "no trained weights file"}
    net = learned.Network.load(path, device)
    sh, sc, o, d0 = net.scales()
    runs = []
    for dmax in (deltas or [d0]):
        net.set_scales(sh, sc, o, dmax)
        # the network's error dominates this mode, so the fallback walk takes
        # the widest opening angle the accurate walk allows
        s = treepm.TreePmSolver(mesh, box.box_size, phys["r_split"], r_cut_factor=phys["r_cut_factor"],
                                accurate=True, theta=LEARNED_THETA, deconvolve_cic=True, learned=True, device=device)
        s.set_learned(net)
        s.set_particles(pos, box.mass)
        for _ in range(2):
            s.compute_forces(phys["eps2"], g)
        sts = []
        for _ in range(reps):
            s.compute_forces(phys["eps2"], g)
            sts.append(s.stats())
        _, _, acc = s.get_state(box.n, pos=False, vel=False)
        rms, p99 = accuracy.relative_errors(acc[targets], ref)
        s.close()
        m = float(np.mean([st["ms_total"] for st in sts]))
        st = sts[-1]
        runs.append({"delta_max": float(dmax), "ms_per_force_evaluation": m,
                     "particle_updates_per_s": box.n / (m * 1e-3), "speedup_vs_plain_step": plain_ms / m,
                     "network_fraction": st["learned_particles"] / box.n, "walk_groups": st["walk_groups"],
                     "groups": st["n_groups"],
                     "stage_ms": {k: float(np.mean([x[k] for x in sts])) for k in
                                  ("ms_bbox_keys", "ms_sort", "ms_build", "ms_pm", "ms_learned", "ms_walk",
                                   "ms_gather_kick")},
                     "force_error_vs_ewald": {"rms": rms, "p99": p99, "targets": int(len(targets))}})
    net.close()
    out = {"flags": "accurate | deconvolve_cic | learned", "theta": LEARNED_THETA,
           "weights": os.path.relpath(os.path.abspath(path), REPO)}
    out.update(runs[0])
    if len(runs) > 1:
        out["delta_max_sweep"] = runs
    return out


IC_CFG = dict(transfer="eisenstein_hu", sigma8=0.8, omega_m=0.315, omega_lambda=0.685, omega_b=0.049, h=0.674,
              box_size_mpc_h=100.0, spectral_index=0.965, cosmology=True, a_init=0.02, h0=0.1)


def zeldovich_report(device, n_side=256, reps=3):
    """Time tpm_set_particles_zeldovich for n_side^3 particles (EH spectrum,
    sigma_8 = 0.8, a_init = 0.02), first and second order, into a solver whose
    PM mesh is the IC lattice (no allocation inside the call); wall time of the
    synchronous call, median of `reps`, with CUDA-event stage times."""
    import treepm
    solver = treepm.TreePmSolver(n_side, 100.0, r_split=2.5 * 100.0 / n_side, device=device)
    out = {"particles": n_side ** 3, "spectrum": "Eisenstein-Hu no-wiggle, sigma_8 0.8, n_s 0.965, a_init 0.02",
           "path": "tpm_set_particles_zeldovich (ic_zeldovich.rs zeldovich_ics / ic_2lpt.rs zeldovich_2lpt_ics)"}
    for order, lpt2 in (("1lpt", False), ("2lpt", True)):
        solver.set_particles_zeldovich(n_side, 1, use_2lpt=lpt2, **IC_CFG)  # warm
        ts = []
        for r in range(reps):
            c0 = time.perf_counter()
            solver.set_particles_zeldovich(n_side, 2 + r, use_2lpt=lpt2, **IC_CFG)
            ts.append(time.perf_counter() - c0)
        ms = 1e3 * float(np.median(ts))
        out[order] = {"ms": ms, "particles_per_s": n_side ** 3 / (ms * 1e-3)}
    solver.close()
    return out


def zeldovich_cpu_sample(n_side=64):
    """The numpy restatement (float64, pocketfft) of the same ICs, first and
    second order, on n_side^3 particles: particles/s of one call each."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import ic_oracle as ico
    f = ico.mode_int(n_side)
    nx, ny, nz = np.meshgrid(f, f, f, indexing="ij")
    nabs = np.sqrt(nx * nx + ny * ny + nz * nz)
    c = IC_CFG
    sig = ico.sigma_of_n(nabs, n_side, "eisenstein_hu", 0.0, c["spectral_index"], omega_m=c["omega_m"],
                         omega_b=c["omega_b"], h=c["h"], box_mpc_h=c["box_size_mpc_h"], sigma8=c["sigma8"])
    v1, d21, v2 = ico.lpt_factors(c["a_init"], c["omega_m"], c["omega_lambda"], c["h0"], True)
    t0 = time.perf_counter()
    ico.zeldovich(n_side, 100.0, sig, seed=2, vel_factor=v1)
    t1 = time.perf_counter()
    ico.zeldovich_2lpt(n_side, 100.0, sig, seed=2, vel1=v1, d21=d21, vel2=v2)
    t2 = time.perf_counter()
    return {"1lpt": n_side ** 3 / (t1 - t0), "2lpt": n_side ** 3 / (t2 - t1), "particles": n_side ** 3,
            "kind": "port", "cores": 1,
            "sample": f"oracle/ic_oracle.py (numpy float64, single thread) at {n_side}^3"}


def snapshot_report(device, n_side=128, reps=3):
    """Time tpm_write_snapshot (JSONL and bincode) of n_side^3 Zel'dovich
    particles into a temporary directory on the local disk: wall time of the
    synchronous call (device decode, chunked copies, host formatting, file
    writes), median of `reps`; the files are removed."""
    import shutil
    import tempfile
    import treepm
    solver = treepm.TreePmSolver(n_side, 100.0, r_split=2.5 * 100.0 / n_side, device=device)
    solver.set_particles_zeldovich(n_side, 3, **IC_CFG)
    out = {"particles": n_side ** 3, "threads": os.cpu_count()}
    root = tempfile.mkdtemp(prefix="tpm_snapshot_")
    try:
        for fmt, name in (("bincode", "particles.bin"), ("jsonl", "particles.jsonl")):
            ts, size = [], 0
            for r in range(reps):
                d = os.path.join(root, f"{fmt}{r}")
                c0 = time.perf_counter()
                solver.write_snapshot(d, fmt, time=0.02, redshift=49.0)
                ts.append(time.perf_counter() - c0)
                size = os.path.getsize(os.path.join(d, name))
                shutil.rmtree(d)
            sec = float(np.median(ts))
            out[fmt] = {"ms": 1e3 * sec, "bytes": size, "gb_per_s": size / sec / 1e9,
                        "records_per_s": n_side ** 3 / sec}
    finally:
        shutil.rmtree(root, ignore_errors=True)
        solver.close()
    return out


def snapshot_cpu_sample(records=1 << 15):
    """The pure-Python restatement of both writers on a bounded sample."""
    sys.path.insert(0, os.path.join(REPO, "oracle"))
    import snapshot_oracle as so
    rng = np.random.default_rng(1)
    pos, vel = rng.uniform(0, 100, (records, 3)), rng.normal(0, 1e-3, (records, 3))
    m, ids = np.full(records, 1.0 / records), np.arange(records)
    t0 = time.perf_counter()
    so.jsonl(ids, m, pos, vel)
    t1 = time.perf_counter()
    so.bincode(ids, m, pos, vel)
    t2 = time.perf_counter()
    return {"jsonl_records_per_s": records / (t1 - t0), "bincode_records_per_s": records / (t2 - t1),
            "kind": "port", "cores": 1, "sample": f"oracle/snapshot_oracle.py (pure Python) on {records} records"}


def run_snapshot_only(args):
    import torch
    torch.cuda.set_device(0)
    rep = snapshot_report(0, n_side=args.snapshot_side, reps=max(1, args.steps))
    rep["cpu_baseline"] = None if args.no_cpu_baseline else snapshot_cpu_sample()
    print(json.dumps({"metric": "snapshot records/s", "snapshot": rep}), flush=True)
    return 0


def run_ics_only(args):
    """One JSON line for the IC generator alone (profiling and the IC row)."""
    import torch
    torch.cuda.set_device(0)
    rep = zeldovich_report(0, n_side=args.ics_side, reps=max(1, args.steps))
    rep["cpu_baseline"] = None if args.no_cpu_baseline else zeldovich_cpu_sample()
    print(json.dumps({"metric": "IC particles/s", "zeldovich_ics": rep}), flush=True)
    return 0


def run_b200(args):
    import torch
    import torch.distributed as dist
    import treepm
    from treepm import ics

    rank, world, local = env_rank()
    torch.cuda.set_device(local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    box, mesh, a0, a1 = make_box(args.workload)
    phys = ics.physics(box, mesh, a0)
    n = box.n
    solver = treepm.TreePmSolver(mesh, box.box_size, phys["r_split"], r_cut_factor=phys["r_cut_factor"],
                                 device=local)
    stream = torch.cuda.ExternalStream(solver.stream, device=torch.device("cuda", local))
    # the workload's trajectory: TRAJ_STEPS KDK steps with one global dt from
    # a0 to a1; the factors are float64 host integrals
    factors, a_of = trajectory(a0, a1, phys["G"])

    def restart():
        """Back to the initial state (zero momenta) with its forces evaluated,
        so every timed step is one steady-state KDK step."""
        solver.set_particles_fixed(box.q, box.mass)
        solver.compute_forces(phys["eps2"], factors[0][3])

    # ---- the trajectory once, untimed: per-step diagnostics (kinetic energy,
    # momentum and angular momentum drift) and per-step FP64 Ewald errors
    from treepm import accuracy, diagnostics
    traj_rep = None
    tg = accuracy.seeded_targets(n, args.ewald_targets)
    ewald = accurate = learned_rep = None
    p_now = ref = None
    if rank == 0 and not args.no_ewald:
        restart()
        rows = []
        p0, v0, a_first = solver.get_state(n)
        rows.append(dict(diagnostics.record(p0, v0, box.mass, a0), step=0,
                         force_momentum_residual=diagnostics.force_momentum_residual(a_first, box.mass)))
        t_e = 0.0
        for i, (d, k1, k2, g) in enumerate(factors):
            solver.kdk_step(k1, d, k2, phys["eps2"], g)
            p_now, v_now, a_now = solver.get_state(n)
            row = dict(diagnostics.record(p_now, v_now, box.mass, a_of[i + 1]), step=i + 1,
                       force_momentum_residual=diagnostics.force_momentum_residual(a_now, box.mass))
            c0 = time.perf_counter()
            ref = accuracy.ewald_accelerations(p_now, box.mass, box.box_size, g, phys["eps2"],
                                               phys["r_cut_factor"] * phys["r_split"], tg, device=local)
            t_e += time.perf_counter() - c0
            row["ewald_rms"], row["ewald_p99"] = accuracy.relative_errors(a_now[tg], ref)
            rows.append(row)
        p_scale = max(math.sqrt(2.0 * r["kinetic_energy"] * r["mass_total"]) for r in rows)
        traj_rep = {
            "steps": len(factors), "a": [a0, a1],
            "rows": rows,
            "max_momentum_drift_over_rms_momentum": max(
                float(np.linalg.norm(np.subtract(r["momentum"], rows[0]["momentum"]))) for r in rows) / p_scale,
            "max_force_momentum_residual": max(r["force_momentum_residual"] for r in rows),
            "momentum_note": "the reference's periodic walk takes a node below 0.1 r_cut as a monopole even when it "
                             "holds the target (short_range.rs:316-323), so momentum is not conserved on clustered "
                             "boxes; the device's residual |sum m a| / max m|a| equals the oracle's on the same state",
            "ewald_seconds": t_e,
            "note": "kinetic energy, momentum, angular momentum and com as diagnostics.rs:55-90 on the canonical "
                    "momenta; Ewald error of each step's closing force on 4096 seeded targets",
        }
        last = rows[-1]
        ewald = {"rms": last["ewald_rms"], "p99": last["ewald_p99"], "targets": int(len(tg)), "seconds": t_e,
                 "state": f"after the {len(factors)} steps a = {a0} -> {a1}",
                 "reference": "FP64 Ewald, Plummer-softened nearest images within r_cut"}
        g_last = factors[-1][3]
        if not args.no_accurate:
            accurate = accurate_mode_report(box, mesh, phys, p_now, g_last, tg, ref, local)

    # ---- device-resident loop (value): K steady-state steps of the trajectory,
    # timed in segments of at most TRAJ_STEPS steps; each segment starts from
    # the initial state (restart outside the timed brackets)
    for i in range(args.warmup):
        if i % len(factors) == 0:
            restart()
        d, k1, k2, g = factors[i % len(factors)]
        solver.kdk_step(k1, d, k2, phys["eps2"], g)
    torch.cuda.synchronize()
    walk_ms, stats = [], []
    dev_ms_rank = 0.0
    with ClockSampler(local) as clocks:
        done = 0
        while done < args.steps:
            seg = min(len(factors), args.steps - done)
            restart()
            torch.cuda.synchronize()
            if world > 1:
                dist.barrier()
            torch.cuda.synchronize()
            ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ev0.record(stream)
            for i in range(seg):
                d, k1, k2, g = factors[i]
                solver.kdk_step(k1, d, k2, phys["eps2"], g)
                st = solver.stats()
                stats.append(st)
                walk_ms.append(st["ms_walk"])
            ev1.record(stream)
            torch.cuda.synchronize()
            dev_ms_rank += ev0.elapsed_time(ev1)
            done += seg
    dev_ms = max_over_ranks(dev_ms_rank, "cuda")
    ms_per_step = dev_ms / args.steps
    value = whole_job_rate(n, args.steps, dev_ms * 1e-3, world)
    if rank == 0 and p_now is not None and not args.no_accurate:
        learned_rep = learned_mode_report(box, mesh, phys, p_now, factors[-1][3], tg, ref, local, ms_per_step,
                                          path=args.learned_weights,
                                          deltas=[float(x) for x in args.learned_deltas.split(",")] if
                                          args.learned_deltas else None)

    # ---- in-situ P(k) of the final state (analysis, not part of the step) --
    pk_rep = None
    if rank == 0:
        t_pk = []
        for _ in range(3):
            c0 = time.perf_counter()
            kk, pk, nmod = solver.power_spectrum()
            t_pk.append(time.perf_counter() - c0)
        pk_rep = {"ms": 1e3 * float(np.median(t_pk)), "shells": int(len(kk)),
                  "k_h_per_mpc": [float(kk[0]), float(kk[-1])], "pk_first_last": [float(pk[0]), float(pk[-1])],
                  "estimator": "power_spectrum.rs (CIC, |delta_k|^2 / W, shells floor(|k| - 1/2))"}

    # ---- Zel'dovich ICs generated on the device (not part of the step) -----
    ic_rep = None
    if rank == 0 and not args.no_ics:
        ic_rep = zeldovich_report(local)

    # ---- end to end through the host-buffer API (e2e): the whole trajectory
    # from the initial state, float64 host arrays in and out every step; the
    # first step meets a new state (upload, encode, two force evaluations)
    e2e_steps = 0 if args.no_e2e else max(1, min(len(factors), args.e2e_steps))
    pos = torch.empty((n, 3), dtype=torch.float64, pin_memory=True).numpy()
    vel = torch.empty((n, 3), dtype=torch.float64, pin_memory=True).numpy()
    mass = torch.empty((n,), dtype=torch.float64, pin_memory=True).numpy()
    p_ic = box.positions()
    mass[:] = box.mass

    def host_ic():
        pos[:] = p_ic
        vel[:] = 0.0

    if e2e_steps:
        host_ic()
        for i in range(2):  # warm: the first two steps of the trajectory
            d, k1, k2, g = factors[i]
            solver.kdk_step_host(pos, vel, mass, k1, d, k2, phys["eps2"], g)
        host_ic()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    t0 = time.perf_counter()
    for i in range(e2e_steps):
        d, k1, k2, g = factors[i]
        solver.kdk_step_host(pos, vel, mass, k1, d, k2, phys["eps2"], g)
    torch.cuda.synchronize()
    e2e_wall = max_over_ranks(time.perf_counter() - t0, "cuda")
    e2e_value = whole_job_rate(n, e2e_steps, e2e_wall, world) if e2e_steps else None
    del p_ic
    h2d = n * (24 + 24 + 8)
    d2h = n * (24 + 24)

    # ---- roofline of the dominant kernel (short-range walk) --------------
    inter = float(np.mean([s["leaf_pairs"] + s["monopoles"] for s in stats]))
    evaluated = float(np.mean([s["evaluated_pairs"] for s in stats]))
    wms = float(np.mean(walk_ms))
    achieved = inter * FLOP_PER_INTERACTION / (wms * 1e-3) / 1e12
    peak = None if args.no_peak else fp32_peak_tflops(solver)
    st = stats[-1]
    stage_ms = {k: float(np.mean([s[k] for s in stats])) for k in
                ("ms_bbox_keys", "ms_sort", "ms_build", "ms_walk", "ms_pm", "ms_gather_kick", "ms_total")}
    line = {
        "metric": "particle-updates/s", "value": value, "unit": "particle-updates/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 pair arithmetic, int32 fixed-point positions, f64 decisions",
        "data": "synthetic",
        "config": {"workload": box.name, "particles": n, "mesh": mesh, "box_mpc_h": box.box_size,
                   "r_s_cells": 1.25, "r_cut_over_r_s": 4.5, "softening": "mean spacing / 30",
                   "a": [a0, a1], "trajectory_steps": len(factors),
                   "timing": "K steady-state steps of the a0 -> a1 trajectory, timed in segments of at most "
                             f"{len(factors)} steps, each from the initial state with its forces evaluated "
                             "(outside the timed brackets)",
                   "parallelism": f"{world} independent replica(s)",
                   "l2": "inputs larger than L2 (>= 0.8 GB touched per step)"},
        "per_force_evaluation": {"value": value, "note": "one force evaluation per fused step; the reference "
                                                         "evaluates twice per step"},
        "stage_ms": stage_ms,
        "stage_roofline": stage_rooflines(stage_ms, n, mesh),
        "walk": {"interactions_per_step": inter, "evaluated_pairs_per_step": evaluated,
                 "interactions_per_particle": inter / n, "exact_fallbacks": st["exact_fallbacks"],
                 "tree_nodes": st["n_tree_nodes"], "groups": st["n_groups"], "max_depth": st["max_tree_depth"]},
        "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                     "frac": (achieved / peak) if peak else None, "traffic": profile_traffic(box.name),
                     "traffic_source": "ncu single-pass capture of this workload's walk, not of this run",
                     "kernel": "k_walk (short-range erfc walk)",
                     "note": f"{FLOP_PER_INTERACTION} FLOP per reference interaction (leaf pair or monopole); "
                             "peak = FFMA throughput measured live on this GPU"},
        "e2e": {"value": e2e_value, "unit": "particle-updates/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h,
                "steps": e2e_steps,
                "path": "tpm_kdk_step_host over the whole trajectory from the initial state (wall clock): float64 "
                        "positions, velocities and masses from pinned host memory, state back to host each step; the "
                        "first step meets a new state (upload, encode, two force evaluations); later steps get the "
                        "state the previous call returned, so they run on the resident state (one force evaluation) "
                        "while a copy stream uploads and checks the inputs and returns the drifted positions; the "
                        "momenta are copied after the closing kick"},
        "gpu_launches": int(sum(s["kernel_launches"] for s in stats)),
        "force_error_vs_ewald": ewald,
        "trajectory_diagnostics": traj_rep,
        "accurate_mode": accurate,
        "learned_mode": learned_rep,
        "power_spectrum": pk_rep,
        "zeldovich_ics": ic_rep,
        "clocks": clocks.summary(),
    }
    if rank == 0 and not args.no_cpu_baseline:
        t_force, info = cpu_sample(box, mesh, phys, args.cpu_targets, os.cpu_count() or 1)
        t_kd = cpu_kick_drift(box, info["threads"])
        cv = n / (2.0 * t_force + t_kd)
        line["cpu_baseline"] = {"value": cv, "unit": "particle-updates/s", "cores": info["threads"], "kind": "port",
                                "sample": (f"oracle restatement (C++/OpenMP, FP64): full PM + full octree build, "
                                           f"walk of {info['targets']} targets (one run of consecutive particles in each of 64 strata) "
                                           f"extrapolated; 2 force evaluations "
                                           f"per step + the host kick-drift-kick; stages s: pm {info['pm_s']:.2f}, "
                                           f"build {info['build_s']:.2f}, walk-sample {info['walk_s']:.2f}, "
                                           f"kick-drift {t_kd:.3f}")}
    if rank == 0:
        print(json.dumps(line), flush=True)
    del stream
    solver.close()
    if world > 1:
        dist.destroy_process_group()
    return 0


def run_domain(args):
    """Domain-decomposed steps (treepm.distributed): the workload's particles
    split into SFC domains over the ranks (untimed), then K KDK steps with
    the halo exchange and the density all-reduce inside each step.  Total work
    is fixed: strong scaling.  One rank runs the same stages and collectives."""
    import torch
    import torch.distributed as dist
    import treepm
    from datetime import timedelta
    from treepm import ics
    from treepm.distributed import DomainTreePm

    rank, world, local = env_rank()
    torch.cuda.set_device(local)
    if world == 1:
        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        if "MASTER_PORT" not in os.environ:
            import socket
            with socket.socket() as sk:
                sk.bind(("127.0.0.1", 0))
                os.environ["MASTER_PORT"] = str(sk.getsockname()[1])
        os.environ.setdefault("RANK", "0")
        os.environ.setdefault("WORLD_SIZE", "1")
    dist.init_process_group("nccl", timeout=timedelta(seconds=300), device_id=torch.device("cuda", local))
    box, mesh, a0, a1 = make_box(args.workload)
    phys = ics.physics(box, mesh, a0)
    n = box.n
    factors, _ = trajectory(a0, a1, phys["G"], total=args.warmup + args.steps + 1)
    dom = DomainTreePm(mesh, box.box_size, phys["r_split"], r_cut_factor=phys["r_cut_factor"], device=local,
                       pm="slab" if args.pm_slab else "replicated")
    lo, hi = rank * n // world, (rank + 1) * n // world
    pos = box.positions()[lo:hi]
    dom.set_particles(pos, box.mass[lo:hi], None, gid=np.arange(lo, hi))
    del pos
    if world > 1:
        dom.redistribute()
    d, k1, k2, g = factors[0]
    dom.compute_forces(phys["eps2"], g)
    for i in range(args.warmup):
        d, k1, k2, g = factors[i]
        dom.kdk_step(k1, d, k2, phys["eps2"], g)
    torch.cuda.synchronize()
    dist.barrier()
    torch.cuda.synchronize()
    stream = torch.cuda.ExternalStream(dom.solver.stream, device=torch.device("cuda", local))
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    halos, stats = [], []
    with ClockSampler(local) as clocks:
        ev0.record(stream)
        for i in range(args.steps):
            d, k1, k2, g = factors[args.warmup + i]
            dom.kdk_step(k1, d, k2, phys["eps2"], g)
            halos.append(dom.last_halo_count)
            stats.append(dom.solver.stats())
        ev1.record(stream)
        torch.cuda.synchronize()
        dist.barrier()
        torch.cuda.synchronize()
    dev_ms = max_over_ranks(ev0.elapsed_time(ev1), "cuda")
    owned = dom.n_owned
    max_owned = int(max_over_ranks(float(owned), "cuda"))
    max_halo = int(max_over_ranks(float(max(halos) if halos else 0), "cuda"))
    stage_ms = {k: float(np.mean([s[k] for s in stats])) for k in
                ("ms_bbox_keys", "ms_sort", "ms_build", "ms_walk", "ms_pm", "ms_gather_kick", "ms_total")}
    # the dominant kernel on rank 0's GPU: its walk over its own particles and halos
    inter0 = float(np.mean([s["leaf_pairs"] + s["monopoles"] for s in stats]))
    achieved0 = inter0 * FLOP_PER_INTERACTION / (stage_ms["ms_walk"] * 1e-3) / 1e12
    peak0 = None if args.no_peak else fp32_peak_tflops(dom.solver)
    line = {
        "metric": "particle-updates/s", "value": n * args.steps / (dev_ms * 1e-3), "unit": "particle-updates/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": dev_ms / args.steps,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
        "dtype": "f32 pair arithmetic, int32 fixed-point positions, f64 decisions", "data": "synthetic",
        "config": {"workload": box.name, "particles": n, "mesh": mesh, "box_mpc_h": box.box_size,
                   "parallelism": f"{world} SFC domain(s), periodic 3D halos of r_cut, " +
                                  ("z-slab PM (two all-to-all transposes)" if args.pm_slab else
                                   "density all-reduce (replicated PM)"),
                   "l2": "inputs larger than L2 (>= 0.8 GB touched per step)"},
        "domain": {"max_owned": max_owned, "max_halo_particles": max_halo,
                   "halo_fraction": max_halo / max(max_owned, 1), "stage_ms_rank0": stage_ms},
        "roofline": {"bound": "fp32", "achieved": achieved0, "peak": peak0, "unit": "TFLOP/s",
                     "frac": (achieved0 / peak0) if peak0 else None, "traffic": None,
                     "kernel": "k_walk (short-range erfc walk) on rank 0",
                     "note": f"{FLOP_PER_INTERACTION} FLOP per reference interaction of rank 0's walk / its "
                             "CUDA-event walk time; peak = FFMA throughput measured live on rank 0's GPU"},
        "e2e": None,
        "e2e_note": "the domain-decomposed path keeps its particles resident and has no host-buffer step",
        "gpu_launches": int(sum(s["kernel_launches"] for s in stats)),
        "clocks": clocks.summary(),
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    del stream
    dom.close()
    dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="clustered256", choices=sorted(WORKLOADS))
    ap.add_argument("--e2e-steps", type=int, default=TRAJ_STEPS)
    ap.add_argument("--cpu-targets", type=int, default=262144)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-cpu-full", action="store_true",
                    help="reference arm: skip the one complete (non-extrapolated) CPU force evaluation")
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer pass (profiling runs)")
    ap.add_argument("--no-ics", action="store_true", help="skip the Zel'dovich IC timing")
    ap.add_argument("--ics-only", action="store_true", help="time only the Zel'dovich IC generator")
    ap.add_argument("--ics-side", type=int, default=256, help="particles per side for the IC timing")
    ap.add_argument("--snapshot-only", action="store_true", help="time only the snapshot writers")
    ap.add_argument("--snapshot-side", type=int, default=128, help="particles per side for the snapshot timing")
    ap.add_argument("--no-peak", action="store_true", help="skip the FFMA peak measurement (profiling runs)")
    ap.add_argument("--no-ewald", action="store_true", help="skip the FP64 Ewald error report")
    ap.add_argument("--no-accurate", action="store_true", help="skip the accurate-mode report")
    ap.add_argument("--ewald-targets", type=int, default=4096)
    ap.add_argument("--learned-weights", default=None, help="weights file of the learned mode (default: committed)")
    ap.add_argument("--learned-deltas", default=None,
                    help="comma-separated fallback overdensity thresholds to sweep in the learned mode")
    ap.add_argument("--domain", action="store_true",
                    help="domain-decomposed steps over the ranks (SFC domains, halos, density all-reduce); "
                         "the default when --gpus > 1")
    ap.add_argument("--replicas", action="store_true", help="with --gpus > 1: independent copies, one per rank")
    ap.add_argument("--pm-slab", action="store_true", help="domain mode: the z-slab PM solve instead of the replicated one")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    if args.ics_only:
        return run_ics_only(args)
    if args.snapshot_only:
        return run_snapshot_only(args)
    if args.domain or (args.gpus > 1 and not args.replicas):
        return run_domain(args)
    return run_b200(args)


if __name__ == "__main__":
    sys.exit(main())
