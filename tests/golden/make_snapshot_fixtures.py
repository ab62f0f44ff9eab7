"""Copy a small sample of the reference's own committed run outputs into
tests/golden/snapshot_ref/: the first 400 records of a JSONL snapshot and the
meta.json / provenance.json / checkpoint.json sidecars of the same run
(experiments/nbody/phase16_tiled_simd/results/p14/validation_N2000_P2, written
by gadget-ng's JsonlWriter and checkpoint code).  They pin the float layout
and the pretty-printed JSON of the snapshot writer.  Run once in a checkout
that has the reference tree:
    python tests/golden/make_snapshot_fixtures.py <gadget-ng checkout root>
"""
import os
import sys

RUN = "experiments/nbody/phase16_tiled_simd/results/p14/validation_N2000_P2"
DST = os.path.join(os.path.dirname(os.path.abspath(__file__)), "snapshot_ref")


def main():
    if len(sys.argv) != 2:
        sys.exit("usage: make_snapshot_fixtures.py <gadget-ng checkout root>")
    SRC = os.path.join(sys.argv[1], RUN)
    os.makedirs(DST, exist_ok=True)
    with open(os.path.join(SRC, "frames/snap_000005/particles.jsonl"), "rb") as f:
        lines = f.read().split(b"\n")[:400]
    with open(os.path.join(DST, "particles_sample.jsonl"), "wb") as f:
        f.write(b"\n".join(lines) + b"\n")
    for rel, name in (("frames/snap_000005/meta.json", "meta.json"),
                      ("frames/snap_000005/provenance.json", "provenance.json"),
                      ("checkpoint/checkpoint.json", "checkpoint.json")):
        with open(os.path.join(SRC, rel), "rb") as f:
            data = f.read()
        with open(os.path.join(DST, name), "wb") as f:
            f.write(data)


if __name__ == "__main__":
    main()
