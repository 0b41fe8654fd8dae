"""Gauss-Seidel order replay (fyzz_b200_set_descriptor_order): the B200
step run in lockstep with the reference's own NativeCpu scene, each step
taking the solver order the reference used for that step (its
partition_constraints input: joints, then touching managers in island-edge
order, scene.cpp:7153-7216).

On a fresh scene's first step the two orders coincide and the velocities
are bit-identical.  From the second step on, the reference's order follows
its island graph's insertion history; replaying it, the B200 step solves
the same rows in the same sequence: one step from the same state (the same
bodies and contact history; orientations can differ by an ulp through the
quaternion integration's sinf / cosf, which are not correctly rounded in
either libm) matches the reference's velocities within 1e-4 relative
(components below 1 cm/s compared absolutely), where the canonical pair
order is off by orders of magnitude.  Piles are chaotic: the ulp-level
differences grow over later steps (a contact appearing on one side only
after a few steps), so the multi-step checks are made where contacts stay
put: unit-cube stacks stay bit-identical for all 30 steps, a mixed scene
with joints within 1e-3.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DT = 1.0 / 120.0
STEPS = 30


def rel_err(a, b, floor=1e-3):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), floor))) if a.size else 0.0


def golden_like(scenes, name):
    return {"boxes": scenes.random_boxes(120, seed=3, xz=2.0, y=(0.3, 4.0)),
            "mixed": scenes.mixed_scale(160, seed=2, region=(5.0, 3.0, 5.0), joint_frac=0.05),
            "stack": scenes.box_stack_scene(24, seed=7),
            "pile": scenes.random_boxes(400, seed=3, xz=4.0, y=(0.3, 6.0))}[name]


def run(pkg, ref, spec, replay, floor=1e-3):
    w = pkg.World(0)
    w.add_scene(spec)
    r = ref.RefScene(spec)
    errs = []
    for k in range(STEPS):
        r.step(DT)
        if replay:
            w.set_descriptor_order(r.manager_order_pairs(), r.joint_order())
        w.step(DT)
        ws, rs = w.read_bodies(), r.body_states()
        errs.append(max(rel_err(ws[:, 3:6], rs[:, 3:6], floor), rel_err(ws[:, 10:13], rs[:, 10:13], floor)))
    return np.array(errs), w, r


@pytest.mark.parametrize("name", ["boxes", "mixed", "stack", "pile"])
def test_replayed_order_matches_reference(pkg, ref, scenes, name):
    spec = golden_like(scenes, name)
    errs, w, r = run(pkg, ref, spec, replay=True, floor=1e-2)
    print(name, "replayed order: max rel err per step", np.array2string(errs, precision=2))
    assert r.counts()["manifolds"] > 10
    assert errs[0] <= 1e-6                   # fresh scene: bit-identical first step
    assert errs[1] <= 1e-4, errs             # one solve with contact history, the reference's order
    if name == "stack":
        assert errs.max() == 0.0, errs       # contacts stay put: bit-identical for all steps
    if name == "mixed":
        assert errs.max() <= 1e-3, errs


def test_replay_changes_the_sweep(pkg, ref, scenes):
    # in a dense pile the canonical order differs from the reference's
    # insertion order from the second step on: replaying it is what matches
    spec = golden_like(scenes, "pile")
    replayed, _, _ = run(pkg, ref, spec, replay=True, floor=1e-2)
    canonical, _, _ = run(pkg, ref, spec, replay=False, floor=1e-2)
    print("canonical order: max rel err per step", np.array2string(canonical, precision=2))
    assert canonical[1] > 100 * max(replayed[1], 1e-7)
