"""Kinematic bodies on the B200 path against the C oracle (pinned bit for
bit to the reference in test_oracle_kinematic) and the reference: the
platform follows its targets, riders move with it and fall asleep after it
stops; authoring errors map to the reference's exception types."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DT = 1.0 / 120.0


def rel_err(a, b, floor):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), floor)))


def test_platform_tracks_oracle(pkg, oracle, scenes):
    spec = scenes.kinematic_platform(16, seed=3)
    w = pkg.World(0)
    first = w.add_scene(spec)
    o = oracle.OracleScene(spec)
    w.set_body_kinematic(first)
    o.set_kinematic(0)
    for k in range(40):
        tg = scenes.platform_target(k)
        w.set_body_kinematic_target(first, tg)
        o.set_kinematic_target(0, tg)
        w.step(DT)
        o.step(DT)
        ws, os_ = w.read_bodies(), o.body_states()
        assert rel_err(ws[:, 0:3], os_[:, 0:3], 1.0) <= 1e-4, k
        assert rel_err(ws[:, 3:6], os_[:, 3:6], 0.1) <= 1e-2, k
    np.testing.assert_allclose(w.read_bodies()[first, 0:3], scenes.platform_target(39)[0:3], atol=1e-6)


def test_riders_settle_like_the_reference(pkg, ref, scenes):
    spec = scenes.kinematic_platform(16, seed=3)
    w = pkg.World(0)
    first = w.add_scene(spec)
    r = ref.RefScene(spec)
    w.set_body_kinematic(first)
    r.set_kinematic(0)
    for k in range(420):
        if k < 150:
            tg = scenes.platform_target(k)
            w.set_body_kinematic_target(first, tg)
            r.set_kinematic_target(0, tg)
        w.step(DT)
        r.step(DT)
    ws, rs = w.read_bodies(), r.body_states()
    # the riders came along: same mean position as the reference's, at rest
    assert np.linalg.norm(ws[2:, 0:3].mean(0) - rs[2:, 0:3].mean(0)) < 0.1
    assert ws[2:, 13].sum() >= 12 and rs[2:, 13].sum() >= 12
    np.testing.assert_allclose(ws[first, 0:3], rs[1, 0:3], atol=1e-5)


def test_kinematic_authoring_errors(pkg, scenes):
    spec = scenes.kinematic_platform(2, seed=1)
    w = pkg.World(0)
    first = w.add_scene(spec)
    with pytest.raises(RuntimeError):      # logic_error: not kinematic
        w.set_body_kinematic_target(first, scenes.platform_target(0))
    w.set_body_kinematic(first)
    with pytest.raises(ValueError):        # invalid_argument: insane orientation
        w.set_body_kinematic_target(first, (0, 0, 0, 0, 0, 0, 2.0))
    with pytest.raises(RuntimeError):      # logic_error: kinematic bodies take no velocity
        w.set_body_velocity(first, (1.0, 0.0, 0.0))
    w.set_body_kinematic_target(first, scenes.platform_target(0))
    w.step(DT)
    np.testing.assert_allclose(w.read_bodies()[first, 0:3], scenes.platform_target(0)[0:3], atol=1e-6)
    w.set_body_kinematic(first, False)     # dynamic again: falls under gravity
    w.step(DT, steps=5)
    assert w.read_bodies()[first, 4] < 0.0


def test_hull_riders_on_a_hull_platform_track_oracle(pkg, oracle, scenes):
    # the platform is a cooked box hull and the riders cooked hulls: the
    # convex generators against an infinite-mass kinematic partner
    spec = scenes.kinematic_platform(12, seed=5)
    spec.convex_meshes = [scenes.hull_box((1.5, 0.1, 1.5)), scenes.hull_prism(6, 0.15, 0.1),
                          scenes.hull_bipyramid(5, 0.12, 0.15)]
    spec.shape_type[:] = scenes.CONVEX
    spec.shape_geom[:, 0] = [0] + [1 + (i % 2) for i in range(12)]
    w = pkg.World(0)
    first = w.add_scene(spec)
    o = oracle.OracleScene(spec)
    w.set_body_kinematic(first)
    o.set_kinematic(0)
    for k in range(40):
        tg = scenes.platform_target(k)
        w.set_body_kinematic_target(first, tg)
        o.set_kinematic_target(0, tg)
        w.step(DT)
        o.step(DT)
    ws, os_ = w.read_bodies(), o.body_states()
    assert rel_err(ws[:, 0:3], os_[:, 0:3], 1.0) <= 1e-4
    assert rel_err(ws[:, 3:6], os_[:, 3:6], 0.1) <= 1e-2
    assert w.step_counters()["convex_pairs"] > 0
