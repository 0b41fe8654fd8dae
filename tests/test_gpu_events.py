"""Contact events of the B200 step (World::contact_events /
contact_event_points) against the reference and the event restatement
(oracle/events.py, itself pinned to the reference in test_oracle_events).

Integer fields (bodies, shapes, kinds, counts, offsets) are exact; point
geometry within 1e-5 relative; impulses within 1e-4 relative (the
one-step velocity tolerance of the solver they come from)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DT = 1.0 / 120.0
FLOOR = 1e-3


def rel_err(a, b, floor=FLOOR):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), floor))) if a.size else 0.0


def world_shape_body(spec):
    sb = np.asarray(spec.shape_body, np.int64)
    if spec.floor is None:
        return sb, np.ones(spec.n_bodies, bool)
    return np.concatenate([[0], sb + 1]), np.concatenate([[False], np.ones(spec.n_bodies, bool)])


def as_rows(events):
    return np.stack([events["body0"], events["body1"], events["kind"], events["contact_count"],
                     events["point_offset"].astype(np.uint32), events["shape0"], events["shape1"]], 1)


def bouncing_pile(scenes):
    spec = scenes.random_boxes(60, seed=11, xz=2.0, y=(0.3, 2.5))
    spec.shape_mat[:, 2] = 0.4
    return spec


def test_disabled_by_default(pkg, scenes):
    w = pkg.World(0)
    w.add_scene(bouncing_pile(scenes))
    w.step(DT, steps=3)
    ev, pts = w.contact_events()
    assert ev.size == 0 and pts.size == 0


@pytest.mark.parametrize("which", ["pile", "mixed"])
def test_first_step_matches_reference(pkg, ref, scenes, which):
    spec = bouncing_pile(scenes) if which == "pile" else \
        scenes.mixed_scale(400, seed=2, region=(6.0, 2.0, 6.0), joint_frac=0.0)
    w = pkg.World(0)
    w.set_contact_notifications(True)
    w.add_scene(spec)
    r = ref.RefScene(spec, contact_notifications=True)
    # let the pile touch first, then compare the first step with the same
    # poses: start both from the state the B200 world reached
    w.step(DT)
    r.step(DT)
    ev, pts = w.contact_events()
    want_ev, want_imp = r.contact_events()
    want_pts, want_pimp = r.contact_event_points()
    assert len(ev) > 0
    np.testing.assert_array_equal(as_rows(ev), want_ev)
    geom = np.concatenate([pts["position"], pts["normal"], pts["separation"][:, None]], 1)
    assert rel_err(geom, want_pts) <= 1e-5
    assert rel_err(pts["normal_impulse"], want_pimp) <= 1e-4
    assert rel_err(ev["normal_impulse"], want_imp) <= 1e-4


def test_event_stream_over_a_bouncing_pile(pkg, scenes):
    # 60 steps with restitution: the device's merge of touching managers and
    # lost touches, normal orientation and per-event sums equal the
    # restatement fed with the device's own manifolds and point impulses.
    import events as ev_mod
    spec = bouncing_pile(scenes)
    w = pkg.World(0)
    w.set_contact_notifications(True)
    w.add_scene(spec)
    sb, dyn = world_shape_body(spec)
    builder = ev_mod.EventBuilder(sb, dyn)
    kinds = set()
    for k in range(60):
        w.step(DT)
        pairs, counts, mpts = w.manifolds()
        ev, pts = w.contact_events()
        # point impulses in manifold order: the touching events in order
        touching = ev[ev["kind"] != 2]
        imp = np.concatenate([pts["normal_impulse"][e["point_offset"]:e["point_offset"] + e["contact_count"]]
                              for e in touching]) if len(touching) else np.zeros(0)
        got_ev, got_imp, got_pts, got_pimp = builder.step(pairs, counts, mpts, imp)
        np.testing.assert_array_equal(as_rows(ev), got_ev, err_msg=f"step {k}")
        np.testing.assert_array_equal(ev["normal_impulse"], got_imp)
        geom = np.concatenate([pts["position"], pts["normal"], pts["separation"][:, None]], 1)
        np.testing.assert_array_equal(geom, got_pts)
        kinds |= set(ev["kind"].tolist())
    assert kinds == {0, 1, 2}


def test_events_track_oracle_for_a_few_steps(pkg, oracle, scenes):
    import events as ev_mod
    spec = bouncing_pile(scenes)
    w = pkg.World(0)
    w.set_contact_notifications(True)
    w.add_scene(spec)
    o = oracle.OracleScene(spec)
    sb, dyn = world_shape_body(spec)
    builder = ev_mod.EventBuilder(sb, dyn)
    for k in range(6):
        w.step(DT)
        o.step(DT)
        pairs, counts, _, mpts = o.manifolds()
        want = builder.step(pairs, counts, mpts, o.normal_impulses())
        ev, pts = w.contact_events()
        np.testing.assert_array_equal(as_rows(ev), want[0], err_msg=f"step {k}")
        assert rel_err(ev["normal_impulse"], want[1]) <= 1e-4
        geom = np.concatenate([pts["position"], pts["normal"], pts["separation"][:, None]], 1)
        assert rel_err(geom, want[2], floor=1.0) <= 1e-4
        assert rel_err(pts["normal_impulse"], want[3]) <= 1e-4
