"""The contact-event restatement (oracle/events.py), fed by the C oracle
replaying the reference's Dy order, reproduces the reference's own
World::contact_events / contact_event_points step by step, bit for bit."""
import numpy as np
import pytest


def world_shape_body(spec):
    """World body id of every world shape (floor = body 0, shape 0)."""
    sb = np.asarray(spec.shape_body, np.int64)
    if spec.floor is None:
        return sb, np.ones(spec.n_bodies, bool)
    return np.concatenate([[0], sb + 1]), np.concatenate([[False], np.ones(spec.n_bodies, bool)])


def test_events_match_reference(oracle, ref, scenes):
    import events as ev_mod
    spec = scenes.random_boxes(60, seed=11, xz=2.0, y=(0.3, 2.5))
    spec.shape_mat[:, 2] = 0.4          # restitution: bounces produce lost touches
    r = ref.RefScene(spec, contact_notifications=True)
    o = oracle.OracleScene(spec)
    sb, dyn = world_shape_body(spec)
    builder = ev_mod.EventBuilder(sb, dyn)
    kinds = set()
    for k in range(60):
        r.step(1.0 / 120.0)
        o.step(1.0 / 120.0, r.manager_order(), r.joint_order())
        pairs, counts, _, pts = o.manifolds()
        got = builder.step(pairs, counts, pts, o.normal_impulses())
        want_ev, want_imp = r.contact_events()
        want_pts, want_pimp = r.contact_event_points()
        np.testing.assert_array_equal(got[0], want_ev, err_msg=f"step {k}")
        np.testing.assert_array_equal(got[1], want_imp)
        np.testing.assert_array_equal(got[2], want_pts)
        np.testing.assert_array_equal(got[3], want_pimp)
        kinds |= set(want_ev[:, 2].tolist())
    assert kinds == {0, 1, 2}, "scene must produce found, persists and lost events"
