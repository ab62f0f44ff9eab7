"""Snapshot and checkpoint files of gadget-ng (crates/gadget-ng-io,
crates/gadget-ng-cli/src/engine/checkpoint.rs) through the C ABI.

Formats: "jsonl" (JsonlWriter: meta.json, provenance.json, particles.jsonl)
and "bincode" (BincodeWriter: the same sidecars, particles.bin).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import SNAPSHOT_FORMATS, TpmProvenance, TpmSnapshotEnv, TreePmError, check, load

DEFAULT_PROVENANCE = {"crate_version": "0.1.0", "git_commit": None, "build_profile": "release",
                      "enabled_features": [], "command_line": [], "config_hash": ""}


def _ptr(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _format(fmt: str) -> int:
    if fmt not in SNAPSHOT_FORMATS:
        raise ValueError(f"format must be one of {sorted(SNAPSHOT_FORMATS)}")
    return SNAPSHOT_FORMATS[fmt]


def provenance_struct(prov: dict | None):
    """(TpmProvenance, objects to keep alive while it is used)."""
    p = dict(DEFAULT_PROVENANCE, **(prov or {}))
    enc = lambda s: None if s is None else str(s).encode()  # noqa: E731
    feats = (C.c_char_p * max(1, len(p["enabled_features"])))(*[enc(s) for s in p["enabled_features"]])
    cmd = (C.c_char_p * max(1, len(p["command_line"])))(*[enc(s) for s in p["command_line"]])
    st = TpmProvenance(crate_version=enc(p["crate_version"]), git_commit=enc(p["git_commit"]),
                       build_profile=enc(p["build_profile"]), enabled_features=feats,
                       n_enabled_features=len(p["enabled_features"]), n_command_line=len(p["command_line"]),
                       command_line=cmd, config_hash=enc(p["config_hash"]))
    return st, (feats, cmd)


def env_struct(time: float = 0.0, redshift: float = 0.0, box_size: float = 1.0, units=None) -> TpmSnapshotEnv:
    """units: None or (length_in_kpc, mass_in_msun, velocity_in_km_s, time_in_gyr, g_internal)."""
    e = TpmSnapshotEnv(time=float(time), redshift=float(redshift), box_size=float(box_size))
    if units is not None:
        e.has_units = 1
        (e.length_in_kpc, e.mass_in_msun, e.velocity_in_km_s, e.time_in_gyr, e.g_internal) = map(float, units)
    return e


def env_dict(e: TpmSnapshotEnv) -> dict:
    units = None
    if e.has_units:
        units = (e.length_in_kpc, e.mass_in_msun, e.velocity_in_km_s, e.time_in_gyr, e.g_internal)
    return {"time": e.time, "redshift": e.redshift, "box_size": e.box_size, "units": units}


def _host_check(rc: int) -> None:
    if rc != 0:
        raise TreePmError(rc, (load().tpm_snapshot_last_error() or b"").decode(errors="replace"))


def write_snapshot(out_dir: str, positions, velocities, masses, global_ids=None, fmt: str = "jsonl",
                   time: float = 0.0, redshift: float = 0.0, box_size: float = 1.0, units=None,
                   provenance: dict | None = None) -> None:
    """SnapshotWriter::write on host arrays (n x 3 positions and velocities)."""
    pos = np.ascontiguousarray(positions, dtype=np.float64).reshape(-1, 3)
    vel = np.ascontiguousarray(velocities, dtype=np.float64).reshape(-1, 3)
    m = np.ascontiguousarray(masses, dtype=np.float64).reshape(-1)
    ids = None if global_ids is None else np.ascontiguousarray(global_ids, dtype=np.uint64).reshape(-1)
    if not (pos.shape[0] == vel.shape[0] == m.shape[0]) or (ids is not None and ids.shape[0] != m.shape[0]):
        raise ValueError("positions, velocities, masses and ids differ in length")
    prov, keep = provenance_struct(provenance)
    env = env_struct(time, redshift, box_size, units)
    _host_check(load().tpm_write_snapshot_host(str(out_dir).encode(), _format(fmt), _ptr(pos), _ptr(vel), _ptr(m),
                                               _ptr(ids), m.shape[0], C.byref(env), C.byref(prov)))
    del keep


def read_snapshot(path: str, fmt: str = "jsonl") -> dict:
    """Records in file order: ids, positions, velocities, masses and meta.json's fields."""
    L = load()
    n = C.c_int64(0)
    env = TpmSnapshotEnv()
    _host_check(L.tpm_read_snapshot_host(str(path).encode(), _format(fmt), C.byref(n), None, None, None, None, 0,
                                         None))
    k = n.value
    pos, vel, m, ids = np.empty((k, 3)), np.empty((k, 3)), np.empty(k), np.empty(k, dtype=np.uint64)
    _host_check(L.tpm_read_snapshot_host(str(path).encode(), _format(fmt), C.byref(n), _ptr(pos), _ptr(vel), _ptr(m),
                                         _ptr(ids), k, C.byref(env)))
    return dict(env_dict(env), ids=ids, positions=pos, velocities=vel, masses=m)


def solver_write_snapshot(handle, out_dir: str, fmt: str, time: float, redshift: float, box_size: float, units,
                          provenance: dict | None) -> None:
    prov, keep = provenance_struct(provenance)
    env = env_struct(time, redshift, box_size, units)
    check(handle.h, handle._lib.tpm_write_snapshot(handle.h, str(out_dir).encode(), _format(fmt), C.byref(env),
                                                   C.byref(prov)))
    del keep


def solver_read_snapshot(handle, path: str, fmt: str) -> dict:
    env = TpmSnapshotEnv()
    check(handle.h, handle._lib.tpm_read_snapshot(handle.h, str(path).encode(), _format(fmt), C.byref(env)))
    return env_dict(env)


def solver_write_checkpoint(handle, out_dir: str, completed_step: int, a_current: float, config_hash: str) -> None:
    check(handle.h, handle._lib.tpm_write_checkpoint(handle.h, str(out_dir).encode(), int(completed_step),
                                                     float(a_current), str(config_hash).encode()))


def solver_read_checkpoint(handle, resume_dir: str):
    step, a = C.c_uint64(0), C.c_double(0.0)
    buf = C.create_string_buffer(4096)
    check(handle.h, handle._lib.tpm_read_checkpoint(handle.h, str(resume_dir).encode(), C.byref(step), C.byref(a), buf,
                                                    len(buf)))
    return int(step.value), float(a.value), buf.value.decode()
