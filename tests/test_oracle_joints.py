"""The joint families of the reference's NativeCpu scene (center and
anchored distance, fixed, spherical, revolute, prismatic; scene.cpp:
3046-3141 authoring, 7615-7767 row preparation, 8895-8945 PGS rows), as
restated in the C oracle, against the reference itself replaying its Dy
order: chains of boxes joined by each kind, some hung from the floor,
moving, colliding and sleeping, agree bit for bit."""
import numpy as np
import pytest

DT = 1.0 / 120.0


@pytest.mark.parametrize("kind", range(6))
def test_joint_kind_matches_reference(oracle, ref, scenes, kind):
    spec = scenes.joint_mechanisms(6, seed=kind, kinds=[kind])
    r = ref.RefScene(spec)
    o = oracle.OracleScene(spec)
    for k in range(160):
        r.step(DT)
        o.step(DT, r.manager_order(), r.joint_order())
        np.testing.assert_array_equal(o.body_states(), r.body_states(), err_msg=f"step {k}")


def test_mixed_joint_kinds_match_reference(oracle, ref, scenes):
    spec = scenes.joint_mechanisms(12, seed=9, links=5)
    r = ref.RefScene(spec)
    o = oracle.OracleScene(spec)
    for k in range(120):
        r.step(DT)
        o.step(DT, r.manager_order(), r.joint_order())
        np.testing.assert_array_equal(o.body_states(), r.body_states(), err_msg=f"step {k}")


def test_joints_hold_their_frames(oracle, scenes):
    # a fixed joint keeps the two local frames together: after a second of
    # motion and collisions the anchor points are typically within a few
    # millimetres (4 position iterations do not converge a chain exactly)
    spec = scenes.joint_mechanisms(4, seed=3, kinds=[scenes.JOINT_FIXED], floor_every=0)
    o = oracle.OracleScene(spec)
    for _ in range(120):
        o.step(DT)
    st = o.body_states()
    loc = spec.joint_locals()

    def rot(q, v):
        u = q[:3]
        t = 2.0 * np.cross(u, v)
        return v + q[3] * t + np.cross(u, t)
    gaps = []
    for j, (a, b) in enumerate(spec.joints):
        pa, qa = st[a + 1, 0:3], st[a + 1, 6:10]
        pb, qb = st[b + 1, 0:3], st[b + 1, 6:10]
        gaps.append(np.linalg.norm(pa + rot(qa, loc[j, 0:3]) - pb - rot(qb, loc[j, 7:10])))
    assert np.median(gaps) < 3e-3 and max(gaps) < 0.1, gaps
