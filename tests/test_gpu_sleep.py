"""Sleeping on the B200 path (sleep check after integration, deactivation of
touch-graph islands, waking through the overlap graph and on authored
velocities) against the reference's NativeCpu scene and the C oracle, whose
sleep restatement is pinned bit for bit to the reference in
test_oracle_sleep.

Where the B200 trajectory equals the reference's bit for bit (bodies that
only touch the floor) the sleep state is compared exactly, step by step.
In piles the trajectories part after some steps (sqrtf / trig rounding),
so sleep flags are compared exactly up to that point and by counts after.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DT = 1.0 / 120.0


def make_world(pkg, spec):
    w = pkg.World(0)
    w.add_scene(spec)
    return w


def separated(scenes):
    # six boxes dropped onto the floor far apart: each settles and sleeps
    return scenes.random_boxes(6, seed=11, xz=6.0, y=(0.6, 1.5))


def test_separated_bodies_sleep_like_the_reference(pkg, ref, scenes):
    spec = separated(scenes)
    w = make_world(pkg, spec)
    r = ref.RefScene(spec)
    slept_at = {}
    for k in range(300):
        w.step(DT)
        r.step(DT)
        ws, rs = w.read_bodies(), r.body_states()
        np.testing.assert_allclose(ws, rs, rtol=0, atol=1e-6, err_msg=f"step {k}")
        np.testing.assert_array_equal(ws[:, 13], rs[:, 13], err_msg=f"step {k}")
        g, e = w.sleep_state(), r.sleep_state()
        np.testing.assert_array_equal(g["wake"], e["wake"], err_msg=f"step {k}")
        np.testing.assert_array_equal((g["flags"] & 1) != 0, e["sleeping"])
        np.testing.assert_array_equal((g["flags"] & 2) != 0, e["ready"])
        np.testing.assert_array_equal(g["counted"], e["counted"])
        for b in np.nonzero(rs[:, 13])[0]:
            slept_at.setdefault(int(b), k)
    assert len(slept_at) == spec.n_bodies, slept_at
    # a sleeping body reports zero velocity and keeps its pose
    st = w.read_bodies()
    assert np.all(st[1:, 3:6] == 0.0) and np.all(st[1:, 10:13] == 0.0)
    before = st.copy()
    w.step(DT, steps=10)
    np.testing.assert_array_equal(w.read_bodies(), before)
    assert w.body_state(1).sleeping == 1


def test_falling_box_wakes_a_sleeping_box_like_the_reference(pkg, ref, scenes):
    # box 1 rests on the floor and falls asleep; box 2, dropped from high
    # above it, wakes it when their bounds first overlap
    spec = scenes.random_boxes(2, seed=0, xz=0.0, y=(0.0, 0.0))
    spec.bodies[:, 3:7] = [0, 0, 0, 1]
    spec.shape_geom[:, :3] = 0.25
    spec.bodies[0, 0:3] = [0.0, 0.26, 0.0]
    spec.bodies[1, 0:3] = [0.05, 12.0, 0.0]
    w = make_world(pkg, spec)
    r = ref.RefScene(spec)
    flags_w, flags_r = [], []
    for k in range(260):
        w.step(DT)
        r.step(DT)
        flags_w.append(w.read_bodies()[1:, 13].copy())
        flags_r.append(r.body_states()[1:, 13].copy())
    fw, fr = np.array(flags_w), np.array(flags_r)
    np.testing.assert_array_equal(fw, fr)
    asleep = np.nonzero(fr[:, 0])[0]
    assert asleep.size and asleep[0] < 150, "the resting box must fall asleep before the drop arrives"
    woke = [k for k in range(1, len(fr)) if fr[k - 1, 0] and not fr[k, 0]]
    assert woke, "the falling box must wake the sleeping one"


def test_pile_sleep_tracks_the_oracle(pkg, oracle, scenes):
    spec = scenes.random_boxes(40, seed=4, xz=1.5, y=(0.5, 3.0))
    w = make_world(pkg, spec)
    o = oracle.OracleScene(spec)
    for k in range(400):
        w.step(DT)
        o.step(DT)
        if k < 150:
            np.testing.assert_array_equal(w.read_bodies()[:, 13], o.body_states()[:, 13], err_msg=f"step {k}")
    nw, no = int(w.read_bodies()[:, 13].sum()), int(o.body_states()[:, 13].sum())
    assert no >= 20 and abs(nw - no) <= max(4, no // 5), (nw, no)


def test_sleep_statistics_vs_reference(pkg, ref, scenes):
    # 1,000 boxes, 600 steps: sleeping counts and kinetic energy over time
    spec = scenes.random_boxes(1000, seed=0)
    w = make_world(pkg, spec)
    r = ref.RefScene(spec)
    for k in range(20):
        w.step(DT, steps=30)
        r.step(DT, 30)
        ws, rs = w.read_bodies()[1:], r.body_states()[1:]
        nw, nr = int(ws[:, 13].sum()), int(rs[:, 13].sum())
        assert abs(nw - nr) <= max(15, nr // 2), (k, nw, nr)
    assert nr >= 30 and nw >= 30
    # sleeping bodies are at rest on something: floor or pile
    asleep = ws[:, 13] > 0
    assert np.all(ws[asleep, 3:6] == 0.0)


def test_authored_velocity_wakes(pkg, scenes):
    spec = separated(scenes)
    w = make_world(pkg, spec)
    w.step(DT, steps=300)
    assert w.read_bodies()[1:, 13].all()
    w.set_body_velocity(1, (0.0, 2.0, 0.0))
    assert w.body_state(1).sleeping == 0
    st = w.sleep_state()
    assert st["wake"][1] == np.float32(0.4) and st["flags"][1] == 0
    assert w.read_bodies()[2, 13] == 1.0
    w.step(DT)
    assert w.body_state(1).velocity[1] > 1.0
    # the bulk write wakes every body it writes
    v6 = np.zeros((spec.n_actors, 6), np.float32)
    w.write_velocities(v6)
    assert not w.read_bodies()[:, 13].any()


def test_sleeping_off(pkg, scenes):
    spec = separated(scenes)
    w = make_world(pkg, spec)
    w.step(DT, steps=300)
    assert w.read_bodies()[1:, 13].all()
    w.set_sleeping(False)
    assert not w.read_bodies()[:, 13].any()
    w.step(DT, steps=200)
    assert not w.read_bodies()[:, 13].any()
    w.set_sleeping(True)
    w.step(DT, steps=200)
    assert w.read_bodies()[1:, 13].all()


def test_persisting_touches_of_sleeping_bodies_report_no_event(pkg, ref, scenes):
    spec = separated(scenes)
    w = pkg.World(0)
    w.set_contact_notifications(True)
    w.add_scene(spec)
    r = ref.RefScene(spec, contact_notifications=True)
    counts = []
    for k in range(300):
        w.step(DT)
        r.step(DT)
        ev, _ = w.contact_events()
        rev, _ = r.contact_events()
        got = np.stack([ev["body0"], ev["body1"], ev["kind"], ev["contact_count"]], 1) if ev.size else \
            np.zeros((0, 4), np.uint32)
        np.testing.assert_array_equal(got, rev[:, :4], err_msg=f"step {k}")
        counts.append(len(ev))
    assert counts[-1] == 0 and max(counts) >= spec.n_bodies
