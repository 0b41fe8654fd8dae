"""Autotuner of the step's performance parameters (fyzz_b200_tuning_t).

Sweeps, on a B200, the parameters that change how a step runs but not what
it computes (every setting gives bit-identical results):

  island_thread   islands of at most this many descriptors: one thread each
  island_warp     ... up to this many: one warp each
  island_cta      ... up to this many: one 128-thread CTA (larger: 384 threads)
  radix_bits      digit width of the device-wide radix sorts (endpoint sort of
                  large scenes, island sort of the descriptors)
  elem_block      threads a block of the elementwise kernels
  work_queue      warp / CTA solvers take islands round-robin (0) or from a
                  device work queue, a per-step counter each worker draws
                  the next island from (1)

for each world class the library distinguishes -- "large_scene" (some scene
above 2,048 finite shapes: the 131,072-body plain scene from its settled
state, timed over steps 6-25 like the bench's headline) and "many_scenes"
(the 4,096-scene batched world, timed over steps 61-80).  Every setting
computes the same trajectory, so each candidate is timed on a fresh world
over exactly the same steps (CUDA events on the world's stream, the better
of two worlds); one round of coordinate descent keeps a candidate when it
is at least 1% faster than the incumbent.  It writes the table the library
reads when a world's device state is built (fyzzxyzzy-sdk_b200/tuning.txt:
one line per class, the defaults' and the tuned step times in its header).

  python fyzzxyzzy-sdk_b200/autotune.py [--out PATH] [--steps N]
"""
from __future__ import annotations

import argparse
import datetime
import importlib
import os
import statistics
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
DT = 1.0 / 120.0
DEFAULTS = {"island_thread": 8, "island_warp": 96, "island_cta": 512, "radix_bits": 8, "elem_block": 256,
            "work_queue": 0}
CANDIDATES = {
    "radix_bits": [8, 9, 10, 11],
    "island_thread": [0, 4, 8],
    "island_warp": [32, 64, 96],
    "island_cta": [128, 256, 512],
    "elem_block": [128, 256, 512],
    "work_queue": [0, 1],
}
FIELDS = ["island_thread", "island_warp", "island_cta", "radix_bits", "elem_block", "work_queue"]


def _pkg():
    if ROOT not in sys.path:
        sys.path.insert(0, ROOT)
    return importlib.import_module("fyzzxyzzy-sdk_b200"), importlib.import_module("fyzzxyzzy-sdk_b200.scenes")


def large_scene_specs(scenes):
    """The plain 131,072-body scene from its settled state (the bench's
    headline workload)."""
    spec = scenes.mixed_scale(131072, seed=1, region=(200.0, 50.0, 200.0))
    path = os.path.join(ROOT, "tests", "golden", "plain_131k_step600.npz")
    with np.load(path) as f:
        st = np.asarray(f["state"], np.float32)
    rec = np.zeros((st.shape[0], 14), np.float32)
    rec[:, :13] = st
    return [scenes.with_state(spec, rec)], 5


def many_scenes_specs(scenes):
    """The batched 4,096-scene world, timed after 60 steps (first impacts)."""
    return scenes.batched_scenes(4096), 60


def measure(torch, pkg, specs, settle: int, params: dict, steps: int) -> float:
    """ms per step of a fresh world under `params`, over steps settle+1 ..
    settle+steps.  Every setting computes the same trajectory, so every
    candidate is timed on exactly the same steps."""
    w = pkg.World(0)
    for s in specs:
        w.add_scene(s)
    w.set_tuning(**params)
    w.step(DT, settle)
    stream = torch.cuda.ExternalStream(w.device_view().stream)
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    w.synchronize()
    start.record(stream)
    w.step(DT, steps)
    end.record(stream)
    end.synchronize()
    ms = start.elapsed_time(end) / steps
    w.close()
    return ms


def tune(torch, pkg, specs, settle, steps: int, log) -> tuple[dict, float, float]:
    """One round of coordinate descent: each parameter's candidates timed on
    fresh worlds (the better of two), the fastest kept when at least 1%
    ahead of the incumbent."""
    def timed(params):
        return min(measure(torch, pkg, specs, settle, params, steps) for _ in range(2))
    best = dict(DEFAULTS)
    base = best_ms = timed(best)
    log(f"  defaults {best}: {base:.4f} ms/step")
    for name in ["work_queue", "radix_bits", "island_thread", "island_warp", "island_cta", "elem_block"]:
        for v in CANDIDATES[name]:
            if v == best[name]:
                continue
            trial = dict(best, **{name: v})
            ms = timed(trial)
            log(f"  {name}={v}: {ms:.4f} ms/step (incumbent {best_ms:.4f})")
            if ms < best_ms * 0.99:
                best, best_ms = trial, ms
    return best, best_ms, base


def main():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--out", default=os.path.join(HERE, "tuning.txt"))
    ap.add_argument("--steps", type=int, default=20)
    args = ap.parse_args()
    import torch
    pkg, scenes = _pkg()
    os.environ["FYZZ_B200_TUNING"] = "none"      # start every world from the defaults
    lines, notes = [], []

    def log(msg):
        print(msg, flush=True)

    for cls, make in (("large_scene", large_scene_specs), ("many_scenes", many_scenes_specs)):
        log(f"{cls}:")
        specs, settle = make(scenes)
        best, best_ms, base = tune(torch, pkg, specs, settle, args.steps, log)
        lines.append(f"{cls} " + " ".join(str(best[f]) for f in FIELDS))
        notes.append(f"# {cls}: defaults {base:.4f} ms/step, tuned {best_ms:.4f} ms/step")
        log(f"  -> {best} ({base:.4f} -> {best_ms:.4f} ms/step)")
    gpu = torch.cuda.get_device_name(0)
    with open(args.out, "w") as f:
        f.write(f"# Step tuning table (fyzz_b200_tuning_t per world class), written by autotune.py on {gpu},\n")
        f.write(f"# {datetime.date.today().isoformat()}; one round of coordinate descent, each candidate the better of\n")
        f.write(f"# two fresh worlds timed over the same {args.steps} steps (the bench's window).\n")
        f.write("# class island_thread island_warp island_cta radix_bits elem_block work_queue\n")
        for n in notes:
            f.write(n + "\n")
        for line in lines:
            f.write(line + "\n")
    log(f"wrote {args.out}")


if __name__ == "__main__":
    main()
