#!/usr/bin/env python3
"""Rigid-body step benchmark: body-steps/s of the B200 step.

Headline workload: the plain at-scale scene -- 131,072 dynamic bodies (70%
boxes, 20% spheres, 10% box+sphere compounds, 2% in distance-joined pairs)
in a 200 x 50 x 200 m region above a floor; dt = 1/120 s, 4 position + 1
velocity iteration -- taken from the state it reaches after its 600 steps in
its run (tests/golden/plain_131k_step600.npz: a settled pile of ~270k
contact managers, where the solver dominates).  W untimed warm-up
steps, then K timed steps.  The same line carries the run from the seeded
start (600 steps), the batched forward (4,096 independent scenes, one launch
per stage), the differentiable rollouts (1,024 x 64 boxes, 128 steps; and at
scale: 16,384 mixed scenes, 64 steps), the cooked-hull leg, the end-to-end
loop through the C ABI with host buffers, the whole-step HBM roofline and the
reference NativeCpu scene timed on the host cores.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

For N > 1 (torchrun, one rank per GPU) every rank steps its own replica of
the plain scene and its own shard of the batched scenes (weak scaling, no
data-path collective); times are the maximum over ranks.  --impl reference
times the reference SDK's NativeCpu scene (built from the reference sources
by oracle/Makefile) on the host cores, from the same settled state.
"""
from __future__ import annotations

import argparse
import datetime
import importlib
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
PKG = "fyzzxyzzy-sdk_b200"
DT = 1.0 / 120.0
METRIC = "body-steps/s on 1 B200: batched vs plain GPU step; backward/forward ratio"
UNIT = "body-steps/s"
PLAIN_WORKLOAD = ("plain method at scale, one scene: 131,072 bodies (70% boxes, 20% spheres, "
                  "10% box+sphere compounds, 2% distance-joined pairs), 200x50x200 m above a floor, "
                  "dt=1/120 s, 4 position + 1 velocity iterations")
SETTLED_FIXTURE = os.path.join(ROOT, "tests", "golden", "plain_131k_step600.npz")
SETTLED_START = ("settled: every body's pose and velocity after the workload's 600 steps from its seeded start "
                 "(tests/golden/plain_131k_step600.npz, made by tests/golden/make_settled.py), all bodies awake, "
                 "contact history rebuilt by the warm-up steps; both arms start from it")
BATCHED_WORKLOAD = ("batched forward: 4,096 independent scenes, body count log-uniform in [16,512] "
                    "(random piles and 5-20 high unit-cube stacks), own floor each, one launch per stage, "
                    "step captured as a CUDA graph")
CONVEX_WORKLOAD = ("cooked convex hulls: one scene of 32,768 bodies (75% cooked hulls of 6 shared meshes: "
                   "prisms, frustums, bipyramids, a box hull, random ellipsoid hulls; 25% boxes and spheres), "
                   "size U[0.12,0.3] m, dropped from 0.5-20 m over 120x120 m onto a floor, steps 121..360")
L2_BYTES = 126 * 1024 * 1024


def parse_args():
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=600)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["b200", "reference"], default="b200")
    ap.add_argument("--batched-steps", type=int, default=256)
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=60)
    ap.add_argument("--profile-steps", type=int, default=6)
    ap.add_argument("--cpu-seconds", type=float, default=20.0)
    ap.add_argument("--bodies", type=int, default=131072, help="plain-scene body count")
    ap.add_argument("--scenes", type=int, default=4096, help="batched scene count per rank")
    ap.add_argument("--same-scenes", type=int, default=64,
                    help="batched scenes sampled for the plain-path-on-the-same-bodies comparison")
    ap.add_argument("--same-steps", type=int, default=32)
    ap.add_argument("--no-diff", action="store_true", help="skip the differentiable rollout leg")
    ap.add_argument("--diff-only", action="store_true", help="time the differentiable rollout leg only")
    ap.add_argument("--diff-scenes", type=int, default=1024)
    ap.add_argument("--diff-boxes", type=int, default=64)
    ap.add_argument("--diff-steps", type=int, default=128)
    ap.add_argument("--diff-every", type=int, default=16)
    ap.add_argument("--diff-settle", type=int, default=120)
    ap.add_argument("--diff4", action="store_true",
                    help="also run the differentiable rollout at scale (16,384 mixed scenes, 64 steps)")
    ap.add_argument("--diff4-scenes", type=int, default=16384)
    ap.add_argument("--diff4-steps", type=int, default=64)
    ap.add_argument("--diff4-every", type=int, default=8)
    ap.add_argument("--settle", type=int, default=0,
                    help="untimed steps of the plain scene before warm-up (profiling a settled pile)")
    ap.add_argument("--convex-bodies", type=int, default=32768)
    ap.add_argument("--convex-steps", type=int, default=240)
    ap.add_argument("--convex-settle", type=int, default=120)
    ap.add_argument("--no-convex", action="store_true", help="skip the cooked-hull leg")
    ap.add_argument("--plain-only", action="store_true",
                    help="time the plain scene only (no e2e, batched or CPU legs; for profiler runs)")
    ap.add_argument("--fresh", action="store_true",
                    help="start the plain scene from its seeded initial state instead of the settled fixture")
    ap.add_argument("--run-steps", type=int, default=600,
                    help="steps of the plain run from the seeded start (0 skips the leg)")
    ap.add_argument("--no-diff4", action="store_true", help="skip the differentiable rollout at scale")
    ap.add_argument("--ref-budget", type=float, default=120.0,
                    help="seconds the reference arm may spend on timed steps")
    return ap.parse_args()


def scenes_mod():
    return importlib.import_module(PKG + ".scenes")


def plain_spec(n):
    """The plain at-scale scene; a smaller body count keeps the scene's
    density (the 200 x 200 m footprint shrinks with sqrt(n / 131,072))."""
    side = 200.0 * (n / 131072.0) ** 0.5
    return scenes_mod().mixed_scale(n, seed=1, region=(side, 50.0, side))


def headline_spec(args):
    """The headline scene and a description of its start: the settled
    fixture for the full-size scene, else the seeded start (smaller
    profiling cases settle on the device with --settle)."""
    spec = plain_spec(args.bodies)
    if args.fresh or args.bodies != 131072:
        return spec, "seeded initial state" + (f", then {args.settle} untimed steps" if args.settle else "")
    if not os.path.exists(SETTLED_FIXTURE):
        raise SystemExit(f"settled fixture missing: {SETTLED_FIXTURE} (tests/golden/make_settled.py)")
    with np.load(SETTLED_FIXTURE) as f:
        st = np.asarray(f["state"], np.float32)
    rec = np.zeros((st.shape[0], 14), np.float32)
    rec[:, :13] = st
    return scenes_mod().with_state(spec, rec), SETTLED_START


def plain_config(spec, start, world):
    """The config object both arms print (identical for the same scene)."""
    return {"workload": PLAIN_WORKLOAD, "start": start, "bodies": spec.n_bodies, "shapes": spec.n_shapes,
            "joints": int(spec.joints.shape[0]), "dt": DT, "position_iterations": 4, "velocity_iterations": 1,
            "l2": "resident working set (~200-400 MB) > 126 MB L2; not flushed between steps",
            "parallelism": f"replicas x{world}" if world > 1 else "single scene"}


def batched_specs(n, rank):
    return scenes_mod().batched_scenes(n, base_seed=rank * n)


# --------------------------------------------------------------- clocks
class ClockSampler:
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, local_rank: int):
        vis = os.environ.get("CUDA_VISIBLE_DEVICES")
        idx = vis.split(",")[local_rank] if vis else str(local_rank)
        self.proc = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", idx, f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, smax, power, reasons = [], [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in out.strip().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
                power.append(float(parts[2]))
            except ValueError:
                continue
            for name, val in zip(names, parts[4:8]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        # samples under load: power above the idle floor (the sampler runs
        # from before the warm-up through the plain legs)
        floor = min(power) + 0.25 * (max(power) - min(power))
        loaded = [c for c, w in zip(sm, power) if w >= floor] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm), "samples_under_load": len(loaded), "power_w_max": max(power),
                "window": "from before the warm-up through the timed, profiled and end-to-end plain steps"}


def clocks_bad(c: dict) -> bool:
    bad = {"hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown"}
    if bad & set(c.get("reasons", [])):
        return True
    sm, smax = c.get("sm_mhz"), c.get("sm_max_mhz")
    return bool(sm and smax and sm < 0.5 * smax and not c.get("reasons"))


# --------------------------------------------------------------- roofline
# Algorithmic bytes per step: the fixed per-unit accounting constants of the
# hot path (bytes per body / shape / pair / contact point / friction row /
# joint row), independent of tuning.  PGS runs I = 4 + 1 passes.
def step_bytes(c: dict, iters: int = 5) -> dict:
    nb, ns, npair = c["bodies"], c["shapes"], c["pairs"]
    nc, nf, nj = c["points"], c["friction_rows"], c["joints"]
    return {
        "bounds": 68.0 * ns,                                        # pose + geometry in, encoded bounds out
        "sort": 384.0 * ns,                                         # 3 axes x 2 endpoints x 8 B x r+w x 4 passes
        "pairs": 48.0 * ns + 8.0 * c["found_lost"],                 # sweep of sorted endpoints, publication
        "narrowphase": 212.0 * npair,                               # 2 x 64 B shape records + 84 B result
        "prep": 92.0 * nc + 56.0 * nf + 64.0 * nj,                  # contact / friction / joint rows
        "pgs": iters * (68.0 * nc + 60.0 * nf + 68.0 * nj + 48.0 * nb),
        "integrate": 120.0 * nb,                                    # body state: read 68 B, write 52 B
    }


def roofline_of(counts: dict, ms_per_step: float, stages: dict, peak: float, peak_kind: str) -> dict:
    """Whole-step roofline (all algorithmic bytes of a step / device time of
    a step) plus per-stage fractions for the stages the accounting covers;
    the island / partition stage has no algorithmic bytes (latency-bound
    integer work) and is listed with its time only."""
    per = step_bytes(counts)
    total = sum(per.values())
    achieved = total / (ms_per_step / 1e3) / 1e9
    tr = ncu_traffic()
    traffic = None
    if tr and tr.get("step_bytes_per_body"):
        traffic = round(tr["step_bytes_per_body"] * counts["bodies"])
    st = {}
    for k, ms in stages.items():
        if k in per and ms > 0:
            a = per[k] / (ms / 1e3) / 1e9
            st[k] = {"ms": round(ms, 4), "algorithmic_bytes": per[k], "achieved": round(a, 1),
                     "frac": round(a / peak, 4)}
        else:
            st[k] = {"ms": round(ms, 4), "algorithmic_bytes": None,
                     "bound": "latency (partition rounds, union-find; no algorithmic bytes)"}
    dom = max((k for k in stages if k in per), key=lambda k: stages[k], default=None)
    out = {"bound": "hbm", "kernel_stage": "whole step (one CUDA graph)", "achieved": round(achieved, 1),
           "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4), "peak_kind": peak_kind,
           "traffic": traffic, "algorithmic_bytes": total, "ms_per_step": round(ms_per_step, 4),
           "traffic_source": (tr or {}).get("_source"), "stages": st, "dominant_stage": dom}
    if dom and tr and tr.get(dom + "_bytes_per_manager"):
        out["dominant_stage_traffic"] = round(tr[dom + "_bytes_per_manager"] * counts["managers"])
    return out


def measured_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic():
    """Per-unit DRAM traffic from the committed ncu summary
    (profiles/ncu_traffic.json), or None."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if not os.path.exists(path):
        return None
    with open(path) as f:
        return json.load(f)


# --------------------------------------------------------------- ranks
class RankReducer:
    """Cross-rank reductions of the timing (max of device times, sum of
    work units).  Single process: identity.  Under torch.distributed the
    reductions run on `device` ("cuda" with NCCL, "cpu" with gloo)."""

    def __init__(self, dist=None, device: str = "cuda"):
        self.dist = dist
        self.device = device

    def _reduce(self, x: float, op) -> float:
        if self.dist is None:
            return x
        import torch
        t = torch.tensor([x], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=op)
        return float(t.item())

    def max(self, x: float) -> float:
        return self._reduce(x, self.dist.ReduceOp.MAX if self.dist else None)

    def sum(self, x: float) -> float:
        return self._reduce(x, self.dist.ReduceOp.SUM if self.dist else None)

    def barrier(self):
        if self.dist is not None:
            self.dist.barrier()


# --------------------------------------------------------------- b200 arm
DIFF_WORKLOAD = ("differentiable batched rollout: 1,024 scenes of 64 boxes (half extents U[0.1,0.3]) settled "
                 "into loose piles, v0 and w0 ~ N(0, 0.5), masses log-uniform [0.5,5] kg, per-scene friction "
                 "U[0.2,1.0]; 128-step horizon, checkpoint every 16 steps; loss = mean squared distance of "
                 "the final centres to targets uniform within 2 m; gradients w.r.t. v0, w0, masses, friction")


def differentiable_leg(torch, pkg, local_rank, args):
    """Forward and backward time of the differentiable rollout; the forward
    includes its checkpoints, the backward the segment recompute, the taped
    re-run of each step and its adjoint."""
    specs = scenes_mod().loose_piles(args.diff_scenes, args.diff_boxes)
    w = pkg.World(local_rank)
    for s in specs:
        w.add_scene(s)
    w.step(DT, args.diff_settle)                      # settled piles: the shared input state
    w.fit_pair_budget(1.5)                            # checkpoints and frames sized by the live pairs
    nb = w.counts()["bodies"]
    v6 = np.zeros((nb, 6), np.float32)
    dyn = np.zeros(nb, bool)
    at = 0
    for s in specs:
        n = s.n_bodies
        v6[at + 1: at + 1 + n, 0:3] = s.bodies[:, 7:10]
        v6[at + 1: at + 1 + n, 3:6] = s.bodies[:, 10:13]
        dyn[at + 1: at + 1 + n] = True
        at += s.n_actors
    w.write_velocities(v6)
    c_start, _ = w.read_mass_frames()
    rng = np.random.default_rng(0)
    d = rng.normal(size=(nb, 3))
    d *= (2.0 * rng.uniform(0, 1, (nb, 1)) ** (1.0 / 3.0)) / np.linalg.norm(d, axis=1, keepdims=True)
    target = c_start + d
    # one untimed rollout (graph capture, first-use costs), then back to the
    # same start state; the timed rollout reuses its buffers and graphs
    w.rollout_begin(args.diff_steps, args.diff_every)
    w.rollout_forward(DT)
    w.rollout_backward(grad_center=np.zeros((nb, 3)))
    w.rollout_rewind()
    w.rollout_begin(args.diff_steps, args.diff_every)
    w.synchronize()
    t0 = time.perf_counter()
    w.rollout_forward(DT)
    w.synchronize()
    fwd = time.perf_counter() - t0
    c, _ = w.read_mass_frames()
    n_dyn = int(dyn.sum())
    loss = float(np.sum((c - target)[dyn] ** 2) / n_dyn)
    grad = (2.0 * (c - target) / n_dyn) * dyn[:, None]
    t0 = time.perf_counter()
    torch.cuda.nvtx.range_push("diff_backward")
    g = w.rollout_backward(grad_center=grad)
    w.synchronize()
    torch.cuda.nvtx.range_pop()
    bwd = time.perf_counter() - t0
    w.close()
    return {"workload": DIFF_WORKLOAD, "scenes": len(specs), "bodies": n_dyn, "steps": args.diff_steps,
            "checkpoint_every": args.diff_every, "forward_ms": fwd * 1e3, "backward_ms": bwd * 1e3,
            "backward_forward_ratio": bwd / fwd,
            "forward_value": n_dyn * args.diff_steps / fwd, "unit": UNIT, "loss": loss,
            "grad_norm_v0": float(np.linalg.norm(g["v0"])),
            "timing": "host clock around the synchronised rollout_forward / rollout_backward calls, after one "
                      "untimed rollout of the same shape from the same start state"}


DIFF4_WORKLOAD = ("batched and differentiable at scale: 16,384 scenes, body count log-uniform in [8,256] (60% "
                  "boxes, 25% spheres, 15% box+sphere compounds, 5% distance-joined pairs), friction U[0.2,1.0]; "
                  "64-step horizon, checkpoint every 8 steps; loss = mean over scenes of the final centre-of-mass "
                  "height plus translational kinetic energy; gradients w.r.t. initial velocities and masses")


def differentiable_leg_at_scale(torch, pkg, local_rank, args):
    specs = scenes_mod().mixed_batched(args.diff4_scenes)
    w = pkg.World(local_rank)
    first = [w.add_scene(s) for s in specs]
    w.step(DT, 1)
    budget = w.fit_pair_budget(1.5)
    nb = w.counts()["bodies"]
    mass = np.zeros(nb)
    scene_of = np.full(nb, -1)
    for k, (s, f) in enumerate(zip(specs, first)):
        for i in range(s.n_bodies):
            mass[f + i] = 1.0 / w.body_mass_properties(f + i)[0]
            scene_of[f + i] = k
    dyn = scene_of >= 0
    free0, total = torch.cuda.mem_get_info()
    w.rollout_begin(args.diff4_steps, args.diff4_every)
    free1, _ = torch.cuda.mem_get_info()
    # one untimed rollout (graph capture, first-use costs), then back to the
    # same start state; the timed rollout reuses its buffers and graphs
    w.rollout_forward(DT)
    w.rollout_backward(grad_center=np.zeros((nb, 3)))
    w.rollout_rewind()
    w.rollout_begin(args.diff4_steps, args.diff4_every)
    w.synchronize()
    t0 = time.perf_counter()
    w.rollout_forward(DT)
    w.synchronize()
    fwd = time.perf_counter() - t0
    c, _ = w.read_mass_frames()
    v = w.read_bodies()[:, 3:6].astype(np.float64)
    S = len(specs)
    M = np.bincount(scene_of[dyn], weights=mass[dyn], minlength=S)
    gc = np.zeros((nb, 3))
    gc[dyn, 1] = mass[dyn] / M[scene_of[dyn]] / S
    gv = np.zeros((nb, 3))
    gv[dyn] = mass[dyn, None] * v[dyn] / S
    height = np.bincount(scene_of[dyn], weights=mass[dyn] * c[dyn, 1], minlength=S) / M
    ke = np.bincount(scene_of[dyn], weights=0.5 * mass[dyn] * (v[dyn] ** 2).sum(1), minlength=S)
    t0 = time.perf_counter()
    g = w.rollout_backward(grad_center=gc, grad_velocity=gv)
    w.synchronize()
    bwd = time.perf_counter() - t0
    w.close()
    return {"workload": DIFF4_WORKLOAD, "scenes": S, "bodies": int(dyn.sum()), "steps": args.diff4_steps,
            "checkpoint_every": args.diff4_every, "pair_budget": budget,
            "rollout_device_bytes": int(free0 - free1), "device_bytes_total": int(total),
            "forward_ms": fwd * 1e3, "backward_ms": bwd * 1e3, "backward_forward_ratio": bwd / fwd,
            "forward_value": int(dyn.sum()) * args.diff4_steps / fwd, "unit": UNIT,
            "loss": float(np.mean(height + ke)), "grad_norm_mass": float(np.linalg.norm(g["mass"])),
            "timing": "host clock around the synchronised rollout_forward / rollout_backward calls, after one "
                      "untimed rollout of the same shape from the same start state"}


def convex_spec(n):
    return scenes_mod().convex_pile(n, seed=11, xz=60.0, y=(0.5, 20.0))


def convex_leg(torch, pkg, local_rank, rank, world, args, barrier, max_over_ranks, sum_over_ranks):
    """The cooked-hull path: a convex pile stepped past its first impacts,
    then timed with CUDA events; on rank 0 of a one-GPU run the reference
    NativeCpu scene steps the same scene on the host for a bounded sample."""
    spec = convex_spec(args.convex_bodies)
    w = pkg.World(local_rank)
    w.add_scene(spec)
    w.step(DT, args.convex_settle)
    stream = torch.cuda.ExternalStream(w.device_view().stream)
    barrier()
    ms = timed_steps(torch, w, args.convex_steps, stream)
    ms_max = max_over_ranks(ms)
    value = sum_over_ranks(spec.n_bodies * args.convex_steps) / (ms_max / 1e3)
    prof = w.profile_step(DT)
    counts = w.counts()
    sc = w.step_counters()
    w.close()
    out = {"workload": CONVEX_WORKLOAD, "bodies": spec.n_bodies * world, "steps": args.convex_steps,
           "value": value, "unit": UNIT, "ms_per_step": ms_max / args.convex_steps,
           "stages_ms": {k: round(v, 4) for k, v in prof.items()}, "counts": counts,
           "convex_pairs": sc["convex_pairs"], "convex_regenerated": sc["convex_regenerated"],
           "cpu_reference": None}
    if rank == 0 and world == 1:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import refscene
        if refscene.available():
            r = refscene.RefScene(spec)
            r.step(DT, args.convex_settle)
            n, t0 = 0, time.perf_counter()
            while n < args.convex_steps and time.perf_counter() - t0 < 10.0:
                r.step(DT, 1)
                n += 1
            el = time.perf_counter() - t0
            r.close()
            out["cpu_reference"] = {"value": spec.n_bodies * n / el, "unit": UNIT, "cores": 2, "kind": "reference",
                                    "sample": f"steps {args.convex_settle + 1}..{args.convex_settle + n} of the same "
                                              f"scene ({el:.1f} s)"}
            out["vs_cpu_reference"] = value / out["cpu_reference"]["value"]
    return out


def plain_same_bodies(torch, pkg, specs, local_rank, n_sample, steps):
    """The plain single-scene path on the batched workload's own bodies: a
    sample of the scenes (evenly spaced over the list, so over the size
    distribution), each stepped as its own one-scene world, timed with CUDA
    events on that world's stream.  Returns body-steps/s over the sample."""
    if n_sample <= 0:
        return None
    idx = np.unique(np.linspace(0, len(specs) - 1, min(n_sample, len(specs))).astype(int))
    total_ms, total_bs = 0.0, 0
    for i in idx:
        w = pkg.World(local_rank)
        w.add_scene(specs[i])
        w.step(DT, 3)
        st = torch.cuda.ExternalStream(w.device_view().stream)
        total_ms += timed_steps(torch, w, steps, st)
        total_bs += specs[i].n_bodies * steps
        w.close()
    return {"value": total_bs / (total_ms / 1e3), "unit": UNIT, "scenes_sampled": int(len(idx)),
            "bodies_sampled": int(sum(specs[i].n_bodies for i in idx)), "steps": steps,
            "how": "each sampled scene stepped alone as a one-scene world (the plain path), "
                   "device time summed over scenes"}


def timed_steps(torch, w, steps, stream):
    start = torch.cuda.Event(enable_timing=True)
    end = torch.cuda.Event(enable_timing=True)
    w.synchronize()
    start.record(stream)
    w.step(DT, steps)
    end.record(stream)
    end.synchronize()
    return start.elapsed_time(end)


def plain_run_leg(torch, pkg, local_rank, args, max_over_ranks, sum_over_ranks, barrier):
    """The plain scene's full run from its seeded start (the workload's 600
    steps: free fall, impacts, settling), one timed region."""
    spec = plain_spec(args.bodies)
    w = pkg.World(local_rank)
    w.add_scene(spec)
    w.step(DT, 1)                      # device state built, graphs captured
    stream = torch.cuda.ExternalStream(w.device_view().stream)
    barrier()
    ms = max_over_ranks(timed_steps(torch, w, args.run_steps, stream))
    counts = w.counts()
    w.close()
    return {"start": "seeded initial state (step 1 untimed)", "steps": args.run_steps,
            "value": sum_over_ranks(spec.n_bodies * args.run_steps) / (ms / 1e3), "unit": UNIT,
            "ms_per_step": ms / args.run_steps, "counts_at_end": counts}


def run_b200(args, rank, world, local_rank):
    import torch
    if args.diff_only:
        torch.cuda.set_device(local_rank)
        pkg = importlib.import_module(PKG)
        out = {"metric": METRIC, "differentiable": differentiable_leg(torch, pkg, local_rank, args)}
        if args.diff4:
            out["differentiable_at_scale"] = differentiable_leg_at_scale(torch, pkg, local_rank, args)
        if rank == 0:
            print(json.dumps(out), flush=True)
        return
    pkg = importlib.import_module(PKG)
    dist = None
    if world > 1:
        import torch.distributed as dist
    torch.cuda.set_device(local_rank)

    red = RankReducer(dist, "cuda")
    barrier, max_over_ranks, sum_over_ranks = red.barrier, red.max, red.sum

    # ---- plain scene (replica per rank), settled ----
    spec, start = headline_spec(args)
    n_dyn = spec.n_bodies
    for attempt in range(2):
        sampler = ClockSampler(local_rank)      # from before the warm-up
        w = pkg.World(local_rank)
        w.add_scene(spec)
        if args.settle:
            w.step(DT, args.settle)
        if args.warmup:
            w.step(DT, args.warmup)
        stream = torch.cuda.ExternalStream(w.device_view().stream)
        barrier()
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_push("timed")
        ms = timed_steps(torch, w, args.steps, stream)
        torch.cuda.nvtx.range_pop()
        barrier()
        ms_max = max_over_ranks(ms)
        counts = w.counts()
        kernels = w.kernels_per_step()
        tuning = w.tuning()

        # ---- per-stage device times (CUDA events at stage boundaries) ----
        prof = {}
        for _ in range(max(1, args.profile_steps)):
            st = w.profile_step(DT)
            for k, v in st.items():
                prof[k] = prof.get(k, 0.0) + v / max(1, args.profile_steps)

        # ---- end to end through the C ABI with host buffers ----
        e2e = None
        if not args.plain_only:
            e2e_steps = max(1, min(args.e2e_steps, args.steps))
            # host buffers in pinned (page-locked) memory, as a host loop that
            # streams state every step would keep them
            buf = torch.empty((spec.n_actors, 14), dtype=torch.float32, pin_memory=True).numpy()
            barrier()
            t0 = time.perf_counter()
            for _ in range(e2e_steps):
                w.read_bodies(buf)
                w.write_states(buf)
                w.step(DT)
            w.synchronize()
            e2e_s = max_over_ranks(time.perf_counter() - t0)
            e2e = {"value": sum_over_ranks(n_dyn * e2e_steps) / e2e_s, "unit": UNIT,
                   "h2d_bytes_per_step": 56 * spec.n_actors, "d2h_bytes_per_step": 56 * spec.n_actors,
                   "steps": e2e_steps,
                   "loop": "read_bodies (D2H of the 14-float records) -> write_states (H2D of the same records, "
                           "velocities unpacked on the device) -> step, one pinned host buffer, host clock"}
        clocks = sampler.stop()
        if not clocks_bad(clocks) or attempt == 1:
            break
        w.close()
    value = sum_over_ranks(n_dyn * args.steps) / (ms_max / 1e3)
    ms_step = ms_max / args.steps
    peak, peak_kind = measured_peaks()
    roofline = roofline_of(counts, ms_step, prof, peak, peak_kind)
    w.close()

    # ---- the plain run from its seeded start ----
    plain_run = None
    if args.run_steps and not args.plain_only:
        plain_run = plain_run_leg(torch, pkg, local_rank, args, max_over_ranks, sum_over_ranks, barrier)

    # ---- batched forward ----
    batched = None
    if not args.no_batched and not args.plain_only:
        specs = batched_specs(args.scenes, rank)
        wb = pkg.World(local_rank)
        for s in specs:
            wb.add_scene(s)
        nb_dyn = sum(s.n_bodies for s in specs)
        if args.warmup:
            wb.step(DT, args.warmup)
        bstream = torch.cuda.ExternalStream(wb.device_view().stream)
        barrier()
        sampler = ClockSampler(local_rank)
        bms = timed_steps(torch, wb, args.batched_steps, bstream)
        bclocks = sampler.stop()
        bms_max = max_over_ranks(bms)
        bvalue = sum_over_ranks(nb_dyn * args.batched_steps) / (bms_max / 1e3)
        bprof = wb.profile_step(DT)
        bcounts = wb.counts()
        bkernels = wb.kernels_per_step()
        btuning = wb.tuning()
        wb.close()
        same = plain_same_bodies(torch, pkg, specs, local_rank, args.same_scenes, args.same_steps)
        batched = {"workload": BATCHED_WORKLOAD, "scenes": len(specs) * world, "bodies": nb_dyn * world,
                   "steps": args.batched_steps, "value": bvalue, "unit": UNIT,
                   "ms_per_step": bms_max / args.batched_steps, "clocks": bclocks,
                   "stages_ms": {k: round(v, 4) for k, v in bprof.items()},
                   "counts": bcounts, "gpu_launches": bkernels * args.batched_steps,
                   "tuning": dict(btuning, table_class="many_scenes"),
                   "plain_same_bodies": same,
                   "vs_plain_same_bodies": bvalue / world / same["value"] if same else None}

    # ---- differentiable rollouts (forward + adjoint) ----
    diff = None
    if not args.no_diff and not args.plain_only:
        diff = differentiable_leg(torch, pkg, local_rank, args)
    diff4 = None
    if not args.no_diff4 and not args.no_diff and not args.plain_only:
        diff4 = differentiable_leg_at_scale(torch, pkg, local_rank, args)

    # ---- cooked convex hulls ----
    convex = None
    if not args.no_convex and not args.plain_only:
        convex = convex_leg(torch, pkg, local_rank, rank, world, args, barrier, max_over_ranks, sum_over_ranks)

    # ---- CPU baseline: the reference NativeCpu scene on this host ----
    cpu = None
    if rank == 0 and world == 1 and not args.plain_only:
        cpu = cpu_baseline(spec, start, args.cpu_seconds)

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic: seeded generator with the workload's distributions (no dataset); settled "
                    "start state committed as a fixture (the workload's own 600-step run)",
            "config": plain_config(spec, start, world),
            "gpu_launches": kernels * args.steps,
            "kernels_per_step": kernels,
            "tuning": dict(tuning, table_class="large_scene",
                           source="fyzzxyzzy-sdk_b200/tuning.txt (fyzzxyzzy-sdk_b200/autotune.py)"),
            "clocks": clocks,
            "counts": counts,
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "plain_run": plain_run,
            "convex": convex,
            "differentiable": diff,
            "differentiable_at_scale": diff4,
            "batched": batched,
            "summary": {
                "settled_value": value, "settled_ms_per_step": ms_step,
                "settled_vs_cpu_baseline": (value / cpu["value"]) if cpu and cpu.get("value") else None,
                "e2e_value": e2e["value"] if e2e else None,
                "plain_run_value": plain_run["value"] if plain_run else None,
                "batched_value": batched["value"] if batched else None,
                "batched_vs_plain_same_bodies": batched["vs_plain_same_bodies"] if batched else None,
                "batched_vs_plain_scene_run": (batched["value"] / plain_run["value"])
                if batched and plain_run else None,
                "backward_forward_ratio": diff["backward_forward_ratio"] if diff else None,
                "backward_forward_ratio_at_scale": diff4["backward_forward_ratio"] if diff4 else None,
                "roofline_frac": roofline["frac"],
            },
        }
        print(json.dumps(line), flush=True)


def ref_settled_sample(spec, warmup, max_steps, budget_s, warmup_budget_s=None):
    """The reference NativeCpu scene from the same start: `warmup` untimed
    steps (bounded by warmup_budget_s), then up to `max_steps` timed steps
    within `budget_s` seconds.  Returns (steps, seconds, warm-up steps)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import refscene
    r = refscene.RefScene(spec)
    t0 = time.perf_counter()
    done_w = 0
    while done_w < warmup and (warmup_budget_s is None or time.perf_counter() - t0 < warmup_budget_s):
        r.step(DT, 1)
        done_w += 1
    n = 0
    t0 = time.perf_counter()
    while n < max_steps and (n == 0 or time.perf_counter() - t0 < budget_s):
        r.step(DT, 1)
        n += 1
    el = time.perf_counter() - t0
    r.close()
    return n, el, done_w


def cpu_baseline(spec, start, seconds):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import refscene
    if not refscene.available():
        return {"value": None, "unit": UNIT, "cores": 0, "kind": "reference",
                "sample": "reference harness not built"}
    n, el, wu = ref_settled_sample(spec, 1, 200, seconds)
    return {"value": spec.n_bodies * n / el, "unit": UNIT, "cores": 2, "kind": "reference",
            "sample": f"{n} steps after {wu} untimed step of the same {spec.n_bodies}-body scene from the same "
                      f"start ({el:.1f} s; NativeCpu uses the caller plus one worker thread)"}


# --------------------------------------------------------------- reference arm
def run_reference(args):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import refscene
    if not refscene.available():
        print(json.dumps({"impl": "reference", "unavailable": "reference NativeCpu harness not built (oracle/_ref)"}))
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    spec, start = headline_spec(args)
    # warm-up aligned with the B200 arm's (W steps), bounded in time
    n, el, wu = ref_settled_sample(spec, args.warmup, args.steps, args.ref_budget, warmup_budget_s=90.0)
    value = spec.n_bodies * n / el
    cores = os.cpu_count() or 1
    batched = None
    if not args.no_batched:
        specs = batched_specs(args.scenes, 0)[:512]
        refs = [refscene.RefScene(s) for s in specs]
        refscene.step_many(refs, DT, 1, cores)
        bsteps = 16
        t0 = time.perf_counter()
        refscene.step_many(refs, DT, bsteps, cores)
        bel = time.perf_counter() - t0
        nb = sum(s.n_bodies for s in specs)
        batched = {"value": nb * bsteps / bel, "unit": UNIT, "scenes": len(specs),
                   "sample": f"{len(specs)} of the 4,096 batched scenes x {bsteps} steps, "
                             f"one NativeCpu scene per batched scene over {cores} host threads"}
    sample = (f"{n} timed steps after {wu} untimed warm-up steps of the {spec.n_bodies}-body scene from the same "
              f"start as the B200 arm ({el:.1f} s; {n} of the requested {args.steps} steps within a "
              f"{args.ref_budget:.0f} s budget; NativeCpu runs on the caller plus one worker thread)")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 0,
            "steps": args.steps, "timed_steps": n, "warmup": args.warmup, "warmup_done": wu,
            "ms_per_step": el / max(n, 1) * 1e3, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32",
            "data": "synthetic: seeded generator with the workload's distributions (no dataset); settled "
                    "start state committed as a fixture (the workload's own 600-step run)",
            "config": plain_config(spec, start, world),
            "cpu_baseline": {"value": value, "unit": UNIT, "kind": "reference", "cores": 2, "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "batched": batched}
    print(json.dumps(line), flush=True)


def main():
    args = parse_args()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            run_reference(args)
        return
    if world > 1:
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=180))
    try:
        run_b200(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
