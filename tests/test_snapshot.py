"""Snapshot and checkpoint files (crates/gadget-ng-io, engine/checkpoint.rs).

The restatement (oracle/snapshot_oracle.py) is pinned by the reference's own
committed run outputs (tests/golden/snapshot_ref, copied by
tests/golden/make_snapshot_fixtures.py): 400 JSONL records written by
JsonlWriter (2,800 floats in serde_json/ryu layout) and the pretty-printed
meta.json, provenance.json and checkpoint.json of the same run, reproduced
byte for byte.  bincode has no committed output in the reference; its bytes
follow bincode 2.0.1's published encoding and round-trip through the readers.
The library's writers must equal the restatement byte for byte, from host
arrays (CPU) and from the device-resident state (GPU).
"""
import json
import math
import os
import re
import shutil

import numpy as np
import pytest

import snapshot_oracle as so

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "snapshot_ref")
EXTRA = ',"internal_energy":0.0,"smoothing_length":0.0,"ptype":"DarkMatter"}'


def _golden_lines():
    with open(os.path.join(GOLDEN, "particles_sample.jsonl")) as f:
        return f.read().splitlines()


def _golden_arrays():
    recs = [json.loads(line) for line in _golden_lines()]
    ids = np.array([r["global_id"] for r in recs], dtype=np.uint64)
    m = np.array([r["mass"] for r in recs])
    pos = np.array([[r["px"], r["py"], r["pz"]] for r in recs])
    vel = np.array([[r["vx"], r["vy"], r["vz"]] for r in recs])
    return ids, m, pos, vel


def _edge_arrays(n=2000, seed=3):
    """Values across every layout branch: random magnitudes 1e-320..1e300,
    zeros of both signs, integral values, 1e16 / 1e17 boundaries, subnormals."""
    rng = np.random.default_rng(seed)
    mant = rng.uniform(1.0, 10.0, (n, 7))
    expo = rng.integers(-320, 300, (n, 7))
    vals = mant * 10.0 ** expo.astype(np.float64)
    vals[rng.random((n, 7)) < 0.5] *= -1
    special = [0.0, -0.0, 1.0, 100.0, 1e15, 1e16, 1e17, 1.5e17, 123456789012345678.0, 1e-5, 0.00012345, 2.5e-5,
               1e-7, 5e-324, 2.2250738585072014e-308, 1.7976931348623157e308, 0.1, 1 / 3, 5.960464477539063e-08]
    vals.flat[:len(special)] = special
    vals[~np.isfinite(vals)] = 1.0
    return vals[:, 0].copy(), vals[:, 1:4].copy(), vals[:, 4:7].copy()


# ---- the restatement against the reference's committed files ---------------------------
def test_oracle_reproduces_reference_jsonl_records():
    lines = _golden_lines()
    floats = 0
    for line in lines:
        r = json.loads(line)
        for s in re.findall(r'":(-?[0-9][^,}]*)', line):
            if "." in s or "e" in s:
                assert so.format_f64(float(s)) == s
                floats += 1
        assert so.record_line(r["global_id"], r["mass"], (r["px"], r["py"], r["pz"]), (r["vx"], r["vy"], r["vz"]),
                              extended=False) == line
    assert floats == 400 * 7


@pytest.mark.parametrize("name", ["meta.json", "provenance.json", "checkpoint.json"])
def test_oracle_reproduces_reference_sidecars(name):
    with open(os.path.join(GOLDEN, name)) as f:
        text = f.read()
    assert so.pretty(json.loads(text)) == text


def test_oracle_ryu_layout_branches():
    cases = {1.0: "1.0", 0.1: "0.1", 1e-7: "1e-7", 1e16: "1e16", 1e15: "1000000000000000.0", 1.5e17: "1.5e17",
             1e-5: "0.00001", 2.5e-5: "0.000025", 1.25e-5: "0.0000125", 5e-324: "5e-324", -0.0: "-0.0",
             123.456: "123.456", 5.960464477539063e-08: "5.960464477539063e-8", 1e21: "1e21",
             float("nan"): "null", float("inf"): "null"}
    for v, s in cases.items():
        assert so.format_f64(v) == s


def test_oracle_bincode_round_trip_and_sizes():
    ids = np.array([0, 250, 251, 65535, 65536, 2 ** 32 - 1, 2 ** 32], dtype=np.uint64)
    m, pos, vel = np.arange(7.0), np.ones((7, 3)), -np.ones((7, 3))
    data = so.bincode(ids, m, pos, vel)
    assert len(data) == 1 + 74 * 2 + 76 * 2 + 78 * 2 + 82
    g, mm, p, v, t = so.parse_bincode(data)
    assert np.array_equal(g, ids.astype(np.int64)) and np.array_equal(mm, m) and np.all(t == 0)


# ---- the library on host arrays (no GPU) ------------------------------------------------
def test_host_writer_reproduces_reference_records(tmp_path):
    """The C++ formatter on the reference's own values: each line is the
    reference's line with the three fields of the current ParticleRecord."""
    from treepm import snapshot
    ids, m, pos, vel = _golden_arrays()
    snapshot.write_snapshot(tmp_path / "s", pos, vel, m, ids, fmt="jsonl", time=0.125, box_size=20.0)
    got = (tmp_path / "s" / "particles.jsonl").read_text().splitlines()
    assert got == [line[:-1] + EXTRA for line in _golden_lines()]


@pytest.mark.parametrize("fmt", ["jsonl", "bincode"])
def test_host_writer_matches_oracle_bytes(tmp_path, fmt):
    from treepm import snapshot
    m, pos, vel = _edge_arrays()
    ids = (np.arange(m.shape[0], dtype=np.uint64) * np.uint64(2654435761)) % np.uint64(2 ** 40)
    prov = dict(crate_version="0.1.0", git_commit='c0ffee"\\\n\t\x01', build_profile="release",
                enabled_features=["mpi", "simd"], command_line=["gadget-ng", "stepping", "--config", "a b.toml"],
                config_hash="abc")
    units = (1.0, 1e10, 1.0, 0.97779, 43007.1)
    snapshot.write_snapshot(tmp_path / "s", pos, vel, m, ids, fmt=fmt, time=0.75, redshift=0.33, box_size=100.0,
                            units=units, provenance=prov)
    d = tmp_path / "s"
    expected = so.jsonl(ids, m, pos, vel) if fmt == "jsonl" else so.bincode(ids, m, pos, vel)
    name = "particles.jsonl" if fmt == "jsonl" else "particles.bin"
    assert (d / name).read_bytes() == expected
    p = so.provenance(prov["crate_version"], prov["git_commit"], "release", prov["enabled_features"],
                      prov["command_line"], "abc")
    assert (d / "provenance.json").read_text() == so.pretty(p)
    assert (d / "meta.json").read_text() == so.pretty(so.snapshot_meta(p, m.shape[0], 0.75, 0.33, 100.0, units))
    back = snapshot.read_snapshot(d, fmt)
    assert np.array_equal(back["ids"], ids) and np.array_equal(back["masses"], m)
    assert np.array_equal(back["positions"], pos) and np.array_equal(back["velocities"], vel)
    assert back["time"] == 0.75 and back["redshift"] == 0.33 and back["box_size"] == 100.0
    assert back["units"] == pytest.approx(units, rel=0, abs=0)


def test_host_reader_takes_the_reference_files(tmp_path):
    """The reader accepts the reference's older records (no SPH fields) and
    its meta.json."""
    from treepm import snapshot
    d = tmp_path / "ref"
    d.mkdir()
    shutil.copy(os.path.join(GOLDEN, "particles_sample.jsonl"), d / "particles.jsonl")
    shutil.copy(os.path.join(GOLDEN, "meta.json"), d / "meta.json")
    back = snapshot.read_snapshot(d, "jsonl")
    ids, m, pos, vel = _golden_arrays()
    assert np.array_equal(back["ids"], ids) and np.array_equal(back["positions"], pos)
    assert np.array_equal(back["velocities"], vel) and np.array_equal(back["masses"], m)
    assert back["time"] == 0.125 and back["box_size"] == 20.0 and back["units"] is None


def test_host_empty_snapshot(tmp_path):
    from treepm import snapshot
    z = np.zeros((0, 3))
    snapshot.write_snapshot(tmp_path / "j", z, z, np.zeros(0), fmt="jsonl")
    snapshot.write_snapshot(tmp_path / "b", z, z, np.zeros(0), fmt="bincode")
    assert (tmp_path / "j" / "particles.jsonl").read_bytes() == b""
    assert (tmp_path / "b" / "particles.bin").read_bytes() == b"\x00"
    assert snapshot.read_snapshot(tmp_path / "b", "bincode")["ids"].shape == (0,)


def test_host_errors(tmp_path):
    import treepm
    from treepm import snapshot
    one = np.zeros((1, 3))
    (tmp_path / "file").write_text("x")
    with pytest.raises(treepm.TreePmError, match="TPM_ERR_IO"):
        snapshot.write_snapshot(tmp_path / "file" / "sub", one, one, np.ones(1))
    with pytest.raises(treepm.TreePmError, match="TPM_ERR_IO"):
        snapshot.read_snapshot(tmp_path / "missing")
    d = tmp_path / "bad"
    snapshot.write_snapshot(d, one, one, np.ones(1))
    (d / "particles.jsonl").write_text('{"global_id":0,"mass":1.0,"px":0.0}\n')
    with pytest.raises(treepm.TreePmError, match="line 1"):
        snapshot.read_snapshot(d)
    (d / "particles.bin").write_bytes(b"\x02\x00")
    with pytest.raises(treepm.TreePmError, match="TPM_ERR_IO"):
        snapshot.read_snapshot(d, "bincode")
    with pytest.raises(ValueError):
        snapshot.write_snapshot(d, one, one, np.ones(1), fmt="hdf5")


# ---- the device-resident writer ---------------------------------------------------------
def _ics(n_side, box=100.0):
    import treepm
    solver = treepm.TreePmSolver(n_side, box, r_split=2.5 * box / n_side)
    solver.set_particles_zeldovich(n_side, 7, transfer="eisenstein_hu", sigma8=0.8, omega_m=0.315,
                                   omega_lambda=0.685, box_size_mpc_h=box, spectral_index=0.965, cosmology=True,
                                   a_init=0.02, h0=0.1)
    return solver


@pytest.mark.gpu
@pytest.mark.parametrize("fmt", ["jsonl", "bincode"])
def test_device_writer_matches_oracle_bytes(tmp_path, fmt):
    """64^3 Zel'dovich particles (ids across the 1-, 3- and 5-byte varints):
    the files equal the restatement of the state read back by get_state."""
    n = 64 ** 3
    solver = _ics(64)
    pos, vel, _ = solver.get_state(n, acc=False)
    mass = np.full(n, 1.0 / n)
    prov = dict(git_commit=None, command_line=["bench"], config_hash="h")
    solver.write_snapshot(tmp_path / "s", fmt, time=0.02, redshift=49.0, provenance=prov)
    ids = np.arange(n, dtype=np.uint64)
    if fmt == "jsonl":
        assert (tmp_path / "s" / "particles.jsonl").read_bytes() == so.jsonl(ids, mass, pos, vel)
    else:
        assert (tmp_path / "s" / "particles.bin").read_bytes() == so.bincode(ids, mass, pos, vel)
    p = so.provenance("0.1.0", None, "release", [], ["bench"], "h")
    assert (tmp_path / "s" / "meta.json").read_text() == so.pretty(so.snapshot_meta(p, n, 0.02, 49.0, 100.0))


@pytest.mark.gpu
def test_device_writer_streams_chunks_like_host_writer(tmp_path):
    """128^3 particles (two chunks of 2^20 and a remainder): the streamed
    device files equal the host writer's on the same state."""
    from treepm import snapshot
    n = 128 ** 3
    solver = _ics(128)
    pos, vel, _ = solver.get_state(n, acc=False)
    mass = np.full(n, 1.0 / n)
    for fmt, name in (("jsonl", "particles.jsonl"), ("bincode", "particles.bin")):
        solver.write_snapshot(tmp_path / ("d" + fmt), fmt)
        snapshot.write_snapshot(tmp_path / ("h" + fmt), pos, vel, mass, fmt=fmt, box_size=100.0)
        assert (tmp_path / ("d" + fmt) / name).read_bytes() == (tmp_path / ("h" + fmt) / name).read_bytes()
        os.remove(tmp_path / ("d" + fmt) / name)
        os.remove(tmp_path / ("h" + fmt) / name)


@pytest.mark.gpu
@pytest.mark.parametrize("fmt", ["jsonl", "bincode"])
def test_device_snapshot_round_trip(tmp_path, fmt):
    import treepm
    n = 32 ** 3
    solver = _ics(32)
    solver.write_snapshot(tmp_path / "s", fmt)
    other = treepm.TreePmSolver(32, 100.0, r_split=2.5 * 100.0 / 32)
    env = other.read_snapshot(tmp_path / "s", fmt)
    assert env["box_size"] == 100.0
    a = solver.get_state(n, acc=False)
    b = other.get_state(n, acc=False)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])


@pytest.mark.gpu
def test_device_checkpoint_resume(tmp_path):
    """save_checkpoint after two steps, load into a fresh solver: identical
    state, checkpoint.json as the restatement, and the resumed step matches
    the uninterrupted one (forces within float rounding of the deposit)."""
    import treepm
    n, box = 32 ** 3, 100.0
    solver = _ics(32, box)
    for _ in range(2):
        solver.kdk_step(1e-3, 2e-3, 1e-3, 1e-4, 1.0)
    solver.write_checkpoint(tmp_path, 2, 0.0213, config_hash="214658da")
    ck = tmp_path / "checkpoint"
    assert (ck / "checkpoint.json").read_text() == so.pretty(so.checkpoint_meta(2, 0.0213, "214658da", n))
    p = so.provenance("checkpoint", None, "release", [], [], "214658da")
    assert (ck / "meta.json").read_text() == so.pretty(so.snapshot_meta(p, n, 0.0, 0.0, 1.0))
    other = treepm.TreePmSolver(32, box, r_split=2.5 * box / 32)
    step, a, h = other.read_checkpoint(tmp_path)
    assert (step, a, h) == (2, 0.0213, "214658da")
    s0, s1 = solver.get_state(n, acc=False), other.get_state(n, acc=False)
    assert np.array_equal(s0[0], s1[0]) and np.array_equal(s0[1], s1[1])
    solver.kdk_step(1e-3, 2e-3, 1e-3, 1e-4, 1.0)
    other.kdk_step(1e-3, 2e-3, 1e-3, 1e-4, 1.0)
    p0, v0, _ = solver.get_state(n, acc=False)
    p1, v1, _ = other.get_state(n, acc=False)
    d = p1 - p0
    d -= box * np.round(d / box)
    v_rms = math.sqrt(np.mean(v0 ** 2))
    assert np.max(np.abs(d)) < 1e-9 * box and np.max(np.abs(v1 - v0)) < 1e-4 * v_rms
