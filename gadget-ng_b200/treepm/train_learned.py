"""Train the learned short-range network on solver-generated boxes.

Usage (on a machine with a B200):
    python gadget-ng_b200/treepm/train_learned.py --out gadget-ng_b200/treepm/weights/learned_sr.npz
    python gadget-ng_b200/treepm/train_learned.py --spec128 --out ...   # the 128^3 training set below

Each seeded box is run through the accurate TreePM once; its mesh features
and the walk's short-range accelerations become training data on the device.
Adam runs on random patches of 8^3 output cells (14^3 input nodes: three
valid 3^3 convolutions), batch 64; the held-out boxes' loss is printed after
every stage.  The weights file holds the parameters and the feature / output
normalisation.

Default set: 24 + 4 held-out clustered boxes of 64^3 particles (L = 50 Mpc/h,
the benchmark's cell size), 6000 / 3000 / 1500 steps at lr 1e-3 / 3e-4 / 1e-4.
--spec128: 64 training + 8 held-out boxes of 128^3 particles at L = 100 Mpc/h
(the same cell size), half from the displaced-lattice generator at 1.0 cell
rms and half from the clustered generator (30 % of the particles in Plummer
spheres), 20,000 Adam steps at lr 1e-3, batch 64.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

if __package__ in (None, ""):
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))

from treepm import learned  # noqa: E402

DEFAULT_OUT = os.path.join(os.path.dirname(os.path.abspath(__file__)), "weights", "learned_sr.npz")


def train(n_train=24, n_held=4, steps=(6000, 3000, 1500), lrs=(1e-3, 3e-4, 1e-4), batch=64, seed=7,
          delta_max=200.0, c_in=learned.C_IN, near_cells=0.0, log=print, side=64):
    net = learned.Network(c_in, params=learned.init_params(c_in, seed))
    net.set_near(near_cells)
    t0 = time.time()
    if side == 64:
        for k in range(n_train):
            learned.capture(net, learned.training_box(1000 + k), 64)
        for k in range(n_held):
            learned.capture(net, learned.training_box(9000 + k), 64, held_out=True)
    else:
        for k in range(n_train):
            learned.capture(net, learned.training_box_mixed(1000 + k, side), side)
        for k in range(n_held):
            learned.capture(net, learned.training_box_mixed(9000 + k, side), side, held_out=True)
    sh, sc, o, _ = net.scales()
    net.set_scales(sh, sc, o, delta_max)
    p0 = net.params()
    net.set_params(0.0 * p0)
    zero = net.evaluate(True)
    net.set_params(p0)
    log(json.dumps({"captured_boxes": n_train + n_held, "seconds": round(time.time() - t0, 2),
                    "held_out_loss_of_zero_prediction": zero, "held_out_loss": net.evaluate(True)}))
    for st, lr in zip(steps, lrs):
        t0 = time.time()
        hist = net.train(st, batch, lr, seed=seed + st)
        log(json.dumps({"steps": st, "lr": lr, "seconds": round(time.time() - t0, 2),
                        "train_loss_last100": float(hist[-100:].mean()), "held_out_loss": net.evaluate(True)}))
    return net


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--out", default=DEFAULT_OUT)
    ap.add_argument("--boxes", type=int, default=24)
    ap.add_argument("--held-out", type=int, default=4)
    ap.add_argument("--steps", type=int, nargs=3, default=[6000, 3000, 1500])
    ap.add_argument("--batch", type=int, default=64)
    ap.add_argument("--seed", type=int, default=7)
    ap.add_argument("--channels", type=int, default=learned.C_IN, help="input features (2: density and potential)")
    ap.add_argument("--near", type=float, default=0.0, help="exact near-field radius in cells (0: network alone)")
    ap.add_argument("--spec128", action="store_true",
                    help="64 + 8 boxes of 128^3 (lattice and clustered generators), 20000 steps at lr 1e-3")
    args = ap.parse_args()
    if args.spec128:
        net = train(64, 8, (20000,), (1e-3,), batch=64, seed=args.seed, c_in=args.channels, near_cells=args.near,
                    side=128)
    else:
        net = train(args.boxes, args.held_out, tuple(args.steps), batch=args.batch, seed=args.seed,
                    c_in=args.channels, near_cells=args.near)
    os.makedirs(os.path.dirname(os.path.abspath(args.out)), exist_ok=True)
    net.save(args.out)
    print(json.dumps({"saved": args.out}))


if __name__ == "__main__":
    main()
