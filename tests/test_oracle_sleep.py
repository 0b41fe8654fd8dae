"""The sleep restatement in the C oracle (Dy sleepCheck, activation and
deactivation of islands) against the reference's own NativeCpu scene,
replaying the reference's Dy order: trajectories, sleeping flags, wake
counters, readiness, counted interactions and sleep filters agree bit for
bit through hundreds of sleep / wake transitions."""
import numpy as np
import pytest

DT = 1.0 / 120.0


def _run(oracle, ref, spec, steps):
    r = ref.RefScene(spec)
    o = oracle.OracleScene(spec)
    transitions, prev = 0, None
    for k in range(steps):
        r.step(DT)
        o.step(DT, r.manager_order(), r.joint_order())
        rs, os_ = r.body_states(), o.body_states()
        np.testing.assert_array_equal(os_, rs, err_msg=f"step {k}")
        a, b = o.sleep_state(), r.sleep_state()
        for key in ("wake", "sleeping", "ready", "counted", "motion"):
            np.testing.assert_array_equal(a[key], b[key], err_msg=f"step {k} {key}")
        if prev is not None:
            transitions += int(np.sum(prev != rs[:, 13]))
        prev = rs[:, 13].copy()
    return transitions, int(prev.sum())


def test_sleep_pile_matches_reference(oracle, ref, scenes):
    spec = scenes.random_boxes(40, seed=4, xz=1.5, y=(0.5, 3.0))
    transitions, asleep = _run(oracle, ref, spec, 400)
    assert transitions >= 30 and asleep >= 20


def test_sleep_mixed_joints_matches_reference(oracle, ref, scenes):
    # spheres, compounds and distance joints; a body resting near an awake
    # one wakes when their overlap pair is lost while a new one is found
    spec = scenes.mixed_scale(200, seed=3, region=(10.0, 3.0, 10.0), joint_frac=0.1)
    transitions, asleep = _run(oracle, ref, spec, 360)
    assert transitions >= 200 and asleep >= 50


def test_sleep_off_never_sleeps(oracle, scenes):
    spec = scenes.random_boxes(6, seed=11, xz=6.0, y=(0.6, 1.5))
    o = oracle.OracleScene(spec)
    o.set_sleeping(False)
    for _ in range(200):
        o.step(DT)
    assert not o.body_states()[:, 13].any()
