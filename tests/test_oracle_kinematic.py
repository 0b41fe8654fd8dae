"""Kinematic bodies (Scene::set_kinematic / set_kinematic_target,
scene.cpp:858-1003; target velocities 2005-2043; publication 2045-2065;
their hold on sleep 893-911 and 6430-6463) as restated in the C oracle,
against the reference replaying its Dy order: boxes riding a moving,
turning kinematic platform, then settling and sleeping on it after it
stops, agree bit for bit."""
import numpy as np

DT = 1.0 / 120.0


def test_platform_riders_match_reference(oracle, ref, scenes):
    spec = scenes.kinematic_platform(16, seed=3)
    r = ref.RefScene(spec)
    o = oracle.OracleScene(spec)
    r.set_kinematic(0)
    o.set_kinematic(0)
    for k in range(420):
        if k < 150:
            tg = scenes.platform_target(k)
            r.set_kinematic_target(0, tg)
            o.set_kinematic_target(0, tg)
        r.step(DT)
        o.step(DT, r.manager_order(), r.joint_order())
        np.testing.assert_array_equal(o.body_states(), r.body_states(), err_msg=f"step {k}")
    st = r.body_states()
    np.testing.assert_allclose(st[1, 0:3], scenes.platform_target(149)[0:3], atol=1e-6)
    assert st[2:, 13].sum() >= 12   # the riders sleep once the platform stops
