"""CPU restatement (pure Python) of gadget-ng's snapshot and checkpoint files.

Test infrastructure only.  Follows
  crates/gadget-ng-io/src/snapshot.rs:17-54 (ParticleRecord: global_id, mass,
    px, py, pz, vx, vy, vz, internal_energy, smoothing_length, ptype),
    :72-120 (SnapshotMeta, meta.json / provenance.json sidecars, pretty JSON),
    :124-146 (JsonlWriter: one serde_json line per particle, '\\n' after each);
  crates/gadget-ng-io/src/bincode_writer.rs:16-31 (Vec<ParticleRecord> through
    bincode 2.0.1 `config::standard()`);
  crates/gadget-ng-io/src/provenance.rs:4-12 (Provenance fields);
  crates/gadget-ng-cli/src/engine/checkpoint.rs:15-110 (CheckpointMeta,
    checkpoint.json, JSONL particles).
Third-party encodings restated from their published specifications:
  serde_json 1.0.149 writes finite f64 through ryu's `format_finite` (shortest
    round-trip digits; decimal notation while the decimal point falls within
    17 digits of the first digit or at most 5 places before it, scientific
    `d.ddde-7` / `1e30` otherwise, `.0` after integral values), non-finite as
    null, strings with `\\" \\\\ \\b \\f \\n \\r \\t` and `\\u00XX` escapes for the other
    control characters, unit enum variants as their name, None as null; the
    pretty formatter indents by two spaces, writes `"key": value`, one array
    element per line and `[]` for an empty array, and no final newline;
  bincode 2.0.1 standard config: little endian, integers as varints (< 251 one
    byte; 251 then u16; 252 then u32; 253 then u64), f64 as 8 raw bytes, a
    sequence as its varint length then its elements, a unit enum variant as
    its index (u32 varint), a struct as its fields in order.
The shortest digits come from Python's repr (shortest round-trip, correctly
rounded), the same digit string ryu produces.
"""
from __future__ import annotations

import math
import struct

import numpy as np

RECORD_FIELDS = ("global_id", "mass", "px", "py", "pz", "vx", "vy", "vz", "internal_energy", "smoothing_length",
                 "ptype")


def format_f64(x: float) -> str:
    """serde_json / ryu layout of one f64."""
    x = float(x)
    if not math.isfinite(x):
        return "null"
    if x == 0.0:
        return "-0.0" if math.copysign(1.0, x) < 0 else "0.0"
    sign = "-" if x < 0 else ""
    r = repr(abs(x))
    # digits d1..dn and decimal exponent: value = 0.d1..dn * 10^kk
    if "e" in r:
        mant, e = r.split("e")
        e = int(e)
    else:
        mant, e = r, 0
    if "." in mant:
        ip, fp = mant.split(".")
    else:
        ip, fp = mant, ""
    digits = (ip + fp).lstrip("0")
    lead_zeros = len(ip + fp) - len((ip + fp).lstrip("0"))
    kk = len(ip) + e - lead_zeros  # position of the decimal point after the first digit
    digits = digits.rstrip("0") or "0"
    length = len(digits)
    k = kk - length
    if 0 <= k and kk <= 16:
        return sign + digits + "0" * k + ".0"
    if 0 < kk <= 16:
        return sign + digits[:kk] + "." + digits[kk:]
    if -5 < kk <= 0:
        return sign + "0." + "0" * (-kk) + digits
    if length == 1:
        return sign + digits + "e" + str(kk - 1)
    return sign + digits[0] + "." + digits[1:] + "e" + str(kk - 1)


def json_string(s: str) -> str:
    out = ['"']
    for ch in s:
        o = ord(ch)
        if ch == '"':
            out.append('\\"')
        elif ch == "\\":
            out.append("\\\\")
        elif ch == "\n":
            out.append("\\n")
        elif ch == "\r":
            out.append("\\r")
        elif ch == "\t":
            out.append("\\t")
        elif ch == "\b":
            out.append("\\b")
        elif ch == "\f":
            out.append("\\f")
        elif o < 0x20:
            out.append("\\u%04x" % o)
        else:
            out.append(ch)
    out.append('"')
    return "".join(out)


def _value(v) -> str:
    if v is None:
        return "null"
    if isinstance(v, bool):
        return "true" if v else "false"
    if isinstance(v, (int, np.integer)):
        return str(int(v))
    if isinstance(v, (float, np.floating)):
        return format_f64(float(v))
    if isinstance(v, str):
        return json_string(v)
    raise TypeError(type(v))


def pretty(obj, indent: int = 0) -> str:
    """serde_json::to_string_pretty of dicts (ordered), lists and scalars."""
    pad, inner = "  " * indent, "  " * (indent + 1)
    if isinstance(obj, dict):
        if not obj:
            return "{}"
        items = [inner + json_string(k) + ": " + pretty(v, indent + 1) for k, v in obj.items()]
        return "{\n" + ",\n".join(items) + "\n" + pad + "}"
    if isinstance(obj, (list, tuple)):
        if not obj:
            return "[]"
        return "[\n" + ",\n".join(inner + pretty(v, indent + 1) for v in obj) + "\n" + pad + "]"
    return _value(obj)


def record_line(gid, mass, pos, vel, extended=True) -> str:
    """One JSONL line (without the newline); `extended` adds the fields the
    current ParticleRecord carries (internal_energy, smoothing_length = 0,
    ptype DarkMatter)."""
    parts = ['"global_id":' + str(int(gid)), '"mass":' + format_f64(mass)]
    for name, v in zip(("px", "py", "pz", "vx", "vy", "vz"), (*pos, *vel)):
        parts.append('"%s":%s' % (name, format_f64(v)))
    if extended:
        parts += ['"internal_energy":0.0', '"smoothing_length":0.0', '"ptype":"DarkMatter"']
    return "{" + ",".join(parts) + "}"


def jsonl(ids, mass, pos, vel, extended=True) -> bytes:
    return "".join(record_line(g, m, p, v, extended) + "\n" for g, m, p, v in zip(ids, mass, pos, vel)).encode()


def parse_jsonl(data: bytes):
    """(ids, mass, pos, vel) of a JSONL snapshot, any field order."""
    import json
    ids, mass, pos, vel = [], [], [], []
    for line in data.decode().splitlines():
        if not line.strip():
            continue
        r = json.loads(line)
        ids.append(r["global_id"])
        mass.append(r["mass"])
        pos.append((r["px"], r["py"], r["pz"]))
        vel.append((r["vx"], r["vy"], r["vz"]))
    return (np.array(ids, dtype=np.int64), np.array(mass, dtype=np.float64), np.array(pos, dtype=np.float64),
            np.array(vel, dtype=np.float64))


def varint(u: int) -> bytes:
    if u < 251:
        return bytes([u])
    if u < 1 << 16:
        return b"\xfb" + struct.pack("<H", u)
    if u < 1 << 32:
        return b"\xfc" + struct.pack("<I", u)
    return b"\xfd" + struct.pack("<Q", u)


def bincode(ids, mass, pos, vel) -> bytes:
    """particles.bin of BincodeWriter for dark-matter records."""
    out = [varint(len(ids))]
    for g, m, p, v in zip(ids, mass, pos, vel):
        out.append(varint(int(g)))
        out.append(struct.pack("<9d", float(m), *map(float, p), *map(float, v), 0.0, 0.0))
        out.append(varint(0))  # ParticleType::DarkMatter
    return b"".join(out)


def parse_bincode(data: bytes):
    def rd_varint(off):
        b = data[off]
        if b < 251:
            return b, off + 1
        if b == 251:
            return struct.unpack_from("<H", data, off + 1)[0], off + 3
        if b == 252:
            return struct.unpack_from("<I", data, off + 1)[0], off + 5
        if b == 253:
            return struct.unpack_from("<Q", data, off + 1)[0], off + 9
        raise ValueError("bad varint")
    n, off = rd_varint(0)
    ids, mass, pos, vel, ptype = [], [], [], [], []
    for _ in range(n):
        g, off = rd_varint(off)
        f = struct.unpack_from("<9d", data, off)
        off += 72
        t, off = rd_varint(off)
        ids.append(g)
        mass.append(f[0])
        pos.append(f[1:4])
        vel.append(f[4:7])
        ptype.append(t)
    if off != len(data):
        raise ValueError("trailing bytes")
    return (np.array(ids, dtype=np.int64), np.array(mass), np.array(pos), np.array(vel), np.array(ptype))


def provenance(crate_version, git_commit, build_profile, features, command_line, config_hash) -> dict:
    return {"crate_version": crate_version, "git_commit": git_commit, "build_profile": build_profile,
            "enabled_features": list(features), "command_line": list(command_line), "config_hash": config_hash}


def snapshot_meta(prov: dict, count: int, time: float, redshift: float, box_size: float, units=None) -> dict:
    m = {"schema_version": 1, "provenance": prov, "particle_count": int(count), "time": float(time),
         "redshift": float(redshift), "box_size": float(box_size)}
    if units is not None:
        m["units"] = {"length_in_kpc": units[0], "mass_in_msun": units[1], "velocity_in_km_s": units[2],
                      "time_in_gyr": units[3], "g_internal": units[4]}
    return m


def checkpoint_meta(completed_step: int, a_current: float, config_hash: str, total: int) -> dict:
    return {"schema_version": 1, "completed_step": int(completed_step), "a_current": float(a_current),
            "config_hash": config_hash, "total_particles": int(total), "has_hierarchical_state": False,
            "sfc_state_saved": False, "has_agn_state": False, "has_chem_state": False}
