"""Force-threshold stream of the B200 step (World::set_body_contact_report_
threshold / force_threshold_changes) against the reference and the
restatement (oracle/thresholds.py, itself pinned to the reference in
test_oracle_thresholds).

Keys, change kinds and thresholds are exact; against the reference the
impulses are within 1e-4 relative (the one-step velocity tolerance of the
solver they come from); against the restatement fed with the device's own
manifolds and point impulses they are bit-exact."""
import numpy as np
import pytest

import thresholds as th_mod

pytestmark = pytest.mark.gpu

DT = 1.0 / 120.0
FLT_MAX = float(np.finfo(np.float32).max)


def rel_err(a, b, floor=1e-3):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), floor))) if a.size else 0.0


def as_rows(ch):
    return np.stack([ch["actor0"], ch["actor1"], ch["static_world"], ch["change"]], 1).astype(np.uint32)


def threshold_pile(scenes, n=60, seed=11):
    spec = scenes.random_boxes(n, seed=seed, xz=2.0, y=(0.3, 2.5))
    spec.shape_mat[:, 2] = 0.4
    thr = np.array([[60.0, 1500.0, FLT_MAX][i % 3] for i in range(spec.n_bodies)], np.float32)
    return spec, thr


def make_world(pkg, spec, thr, notify=False):
    w = pkg.World(0)
    if notify:
        w.set_contact_notifications(True)
    first = w.add_scene(spec)
    for i, t in enumerate(thr):
        if t != FLT_MAX:
            w.set_body_contact_report_threshold(first + i, float(t))
    return w


def test_off_by_default_and_validation(pkg, scenes):
    spec, thr = threshold_pile(scenes)
    w = pkg.World(0)
    first = w.add_scene(spec)
    w.step(DT, steps=3)
    assert w.force_threshold_changes().size == 0
    with pytest.raises(ValueError):
        w.set_body_contact_report_threshold(first, -1.0)
    with pytest.raises(ValueError):
        w.set_body_contact_report_threshold(first, float("nan"))
    with pytest.raises(RuntimeError):           # the floor is static
        w.set_body_contact_report_threshold(0, 10.0)


def test_first_step_matches_reference(pkg, ref, scenes):
    spec, thr = threshold_pile(scenes)
    w = make_world(pkg, spec, thr)
    r = ref.RefScene(spec)
    for i, t in enumerate(thr):
        if t != FLT_MAX:
            r.set_contact_report_threshold(i + 1, float(t))
    w.step(DT)
    r.step(DT)
    got = w.force_threshold_changes()
    rows, imp, tr = r.force_threshold_changes()
    assert len(rows) > 0
    np.testing.assert_array_equal(as_rows(got), rows)
    np.testing.assert_array_equal(got["threshold"], tr)
    assert rel_err(got["normal_impulse"], imp) <= 1e-4


def test_stream_over_a_settling_pile(pkg, scenes):
    # 180 steps: impacts (Found), resting contacts above a low threshold
    # (Persists), bounces and islands falling asleep (Lost)
    spec, thr = threshold_pile(scenes)
    w = make_world(pkg, spec, thr, notify=True)
    sb = np.concatenate([[0], np.asarray(spec.shape_body, np.int64) + 1])
    motion = np.concatenate([[th_mod.STATIC], np.full(spec.n_bodies, th_mod.DYNAMIC)])
    actor_thr = np.concatenate([[FLT_MAX], thr]).astype(np.float32)
    builder = th_mod.ThresholdBuilder(sb, motion)
    seen = set()
    for k in range(180):
        w.step(DT)
        ev, pts = w.contact_events()
        touching = ev[ev["kind"] != 2]
        pairs = np.stack([np.minimum(touching["shape0"], touching["shape1"]),
                          np.maximum(touching["shape0"], touching["shape1"])], 1)
        imp = np.concatenate([pts["normal_impulse"][e["point_offset"]:e["point_offset"] + e["contact_count"]]
                              for e in touching]) if len(touching) else np.zeros(0)
        sleeping = np.concatenate([[False], (w.sleep_state()["flags"][1:] & 1) != 0])
        rows, want_imp, want_thr = builder.step(pairs, touching["contact_count"], imp, sleeping, actor_thr, DT)
        got = w.force_threshold_changes()
        np.testing.assert_array_equal(as_rows(got), rows, err_msg=f"step {k}")
        np.testing.assert_array_equal(got["normal_impulse"], want_imp, err_msg=f"step {k}")
        np.testing.assert_array_equal(got["threshold"], want_thr, err_msg=f"step {k}")
        seen |= set(rows[:, 3].tolist())
    assert seen == {0, 1, 2}


def test_kinematic_pairs_keep_both_ids(pkg, scenes):
    # boxes riding a kinematic platform: their pairs with the platform keep
    # both actor ids (not the world key) and the smaller threshold
    spec = scenes.kinematic_platform(12, seed=0)
    w = pkg.World(0)
    first = w.add_scene(spec)
    w.set_body_kinematic(first, True)
    for i in range(spec.n_bodies):
        w.set_body_contact_report_threshold(first + i, 5.0 if i == 0 else 40.0)
    plat = []
    for k in range(150):
        w.step(DT)
        got = w.force_threshold_changes()
        plat += [r for r in got if first in (r["actor0"], r["actor1"]) and not r["static_world"]]
        assert all(r["actor0"] != first for r in got if r["static_world"])
    assert plat, "some box must press on the platform above its threshold"
    for r in plat:
        assert r["actor0"] < r["actor1"]
        assert r["threshold"] == np.float32(5.0)


def test_rollback_keeps_the_previous_generation(pkg, scenes):
    # a failed step (non-finite velocity) leaves the stream where it was:
    # after the fix the run reports exactly what an undisturbed run reports
    spec, thr = threshold_pile(scenes)
    w, ref_w = make_world(pkg, spec, thr), make_world(pkg, spec, thr)
    w.step(DT, steps=30)
    ref_w.step(DT, steps=30)
    good = w.read_bodies()
    bad = good.copy()
    bad[5, 4] = np.inf
    w.write_states(np.ascontiguousarray(bad))
    with pytest.raises(OverflowError):
        w.step(DT)
    assert w.force_threshold_changes().size == 0
    w.write_states(np.ascontiguousarray(good))
    ref_w.write_states(np.ascontiguousarray(good))
    for k in range(5):
        w.step(DT)
        ref_w.step(DT)
        a, b = w.force_threshold_changes(), ref_w.force_threshold_changes()
        np.testing.assert_array_equal(a, b)
