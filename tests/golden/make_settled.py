"""Generates the settled plain-scene fixture.

Steps the plain at-scale workload -- 131,072 bodies (70% boxes, 20% spheres,
10% box+sphere compounds, 2% distance-joined pairs), seed 1, 200 x 50 x 200 m
above a floor -- through its full 600 steps at dt = 1/120 s and stores the
state every actor ends in:

  plain_131k_step600.npz
    state    (n_actors, 13) float32: position(3) linear velocity(3)
             orientation xyzw(4) angular velocity(3); the floor first
    sleeping (n_actors,) uint8: asleep at the end of the run
    steps, seed, bodies: the run's parameters; engine: which step made it

bench.py starts its settled-pile legs (the B200 arm and the reference arm)
from this state, so both time the same settled pile.  The committed
fixture was made with --engine b200 (the B200 step, one GPU, under a
second); --engine reference steps the reference's NativeCpu scene instead
(oracle/_ref), which takes hours on its two threads as the pile forms.

Usage:  python tests/golden/make_settled.py [--engine b200|reference] [--steps 600] [--out PATH]
"""
from __future__ import annotations

import argparse
import importlib
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import refscene  # noqa: E402

scenes = importlib.import_module("fyzzxyzzy-sdk_b200.scenes")

N_BODIES = 131072
SEED = 1
DT = 1.0 / 120.0
OUT = os.path.join(HERE, "plain_131k_step600.npz")


def plain_spec():
    return scenes.mixed_scale(N_BODIES, seed=SEED, region=(200.0, 50.0, 200.0))


def save(states: np.ndarray, steps: int, engine: str, path: str = OUT) -> None:
    """states: (n_actors, 14) body states (the 13 floats and the sleeping
    flag), as World.read_bodies and the reference harness return them."""
    st = np.asarray(states, np.float32)
    np.savez_compressed(path, state=np.ascontiguousarray(st[:, :13]), sleeping=(st[:, 13] != 0).astype(np.uint8),
                        steps=np.int64(steps), seed=np.int64(SEED), bodies=np.int64(N_BODIES),
                        engine=np.array(engine))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--engine", choices=["b200", "reference"], default="b200")
    ap.add_argument("--steps", type=int, default=600)
    ap.add_argument("--out", default=OUT)
    args = ap.parse_args()
    t0 = time.time()
    if args.engine == "b200":
        pkg = importlib.import_module("fyzzxyzzy-sdk_b200")
        w = pkg.World(0)
        w.add_scene(plain_spec())
        w.step(DT, args.steps)
        states = w.read_bodies()
        print(f"{args.steps} steps on the B200 step: {time.time() - t0:.1f} s, {w.counts()}", flush=True)
    else:
        if not refscene.available():
            raise SystemExit("reference harness not built (make -C oracle ref)")
        r = refscene.RefScene(plain_spec())
        for k in range(args.steps):
            r.step(DT, 1)
            if k % 50 == 0:
                print(f"step {k}: {time.time() - t0:.0f} s, {r.counts()}", flush=True)
        states = r.body_states()
    save(states, args.steps, args.engine, args.out)
    print("wrote", args.out)


if __name__ == "__main__":
    main()
