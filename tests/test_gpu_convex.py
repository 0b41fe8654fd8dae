"""Cooked convex hulls on the B200 path against the C oracle, whose convex
restatement is pinned bit for bit to the reference in test_oracle_convex,
and against the reference itself for fresh manifolds and long runs.

  integer work (encoded bounds, pair sets)                    bit-exact
  fresh manifolds from identical poses                        1e-5 relative
  one step from identical state (velocities)                  1e-4 relative
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DT = 1.0 / 120.0
CONTACT_RTOL = 1e-5
VEL_RTOL = 1e-4
FLOOR = 1e-3


def rel_err(a, b, floor=FLOOR):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), floor))) if a.size else 0.0


def world_of(pkg, spec):
    w = pkg.World(0)
    w.add_scene(spec)
    return w


def resting_pile(scenes, seed, n=48):
    # hulls, boxes and spheres dropped close together just above the floor:
    # contacts against the floor and between shapes from the first step on
    return scenes.convex_pile(n, seed=seed, xz=0.9, y=(0.15, 1.2))


@pytest.mark.parametrize("seed", [0, 1])
def test_bounds_and_pairs_bitexact(pkg, oracle, scenes, seed):
    spec = resting_pile(scenes, seed)
    w = world_of(pkg, spec)
    o = oracle.OracleScene(spec)
    w.collide()
    o.advance_collision()
    np.testing.assert_array_equal(w.encoded_bounds(), o.encoded_bounds())
    np.testing.assert_array_equal(w.pairs(0), o.pairs(0))
    assert w.step_counters()["convex_pairs"] > 0


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_fresh_manifolds_match_reference(pkg, ref, scenes, seed):
    spec = resting_pile(scenes, seed)
    w = world_of(pkg, spec)
    w.collide()
    r = ref.RefScene(spec)
    r.advance_collision()
    wp, wc, wpts = w.manifolds()
    rp, rc, _, rpts = r.manifolds()
    np.testing.assert_array_equal(wp, rp)
    np.testing.assert_array_equal(wc, rc)
    assert rel_err(wpts, rpts) <= CONTACT_RTOL


@pytest.mark.parametrize("seed", [0, 1])
def test_one_step_matches_oracle(pkg, oracle, scenes, seed):
    spec = resting_pile(scenes, seed)
    w = world_of(pkg, spec)
    o = oracle.OracleScene(spec)
    w.step(DT)
    o.step(DT)
    np.testing.assert_array_equal(w.pairs(0), o.pairs(0))
    ws, os_ = w.read_bodies(), o.body_states()
    assert rel_err(ws[:, 3:6], os_[:, 3:6]) <= VEL_RTOL
    assert rel_err(ws[:, 10:13], os_[:, 10:13]) <= VEL_RTOL
    assert rel_err(ws[:, 0:3], os_[:, 0:3]) <= VEL_RTOL


def test_mass_properties_match_reference(pkg, ref, scenes):
    spec = scenes.convex_pile(40, seed=3, offset_frac=0.6)
    w = world_of(pkg, spec)
    r = ref.RefScene(spec)
    got = np.stack([w.body_mass_properties(b + 1) for b in range(spec.n_bodies)])
    want = r.mass_props()[1:]
    np.testing.assert_array_equal(got, want)


def test_short_run_tracks_oracle(pkg, oracle, scenes):
    spec = resting_pile(scenes, 4)
    w = world_of(pkg, spec)
    o = oracle.OracleScene(spec)
    for k in range(20):
        w.step(DT)
        o.step(DT)
    ws, os_ = w.read_bodies(), o.body_states()
    assert rel_err(ws[:, 0:3], os_[:, 0:3], floor=1.0) <= 1e-3
    assert rel_err(ws[:, 3:6], os_[:, 3:6], floor=0.1) <= 5e-2


def test_pile_settles_like_reference(pkg, ref, scenes):
    # 300 hulls, boxes and spheres dropped from 0.5-4 m: heights, kinetic
    # energy and sleeping counts over the run agree statistically
    spec = scenes.convex_pile(300, seed=8, xz=3.0)
    w = world_of(pkg, spec)
    r = ref.RefScene(spec)
    for k in range(12):
        w.step(DT, steps=30)
        r.step(DT, 30)
        ws, rs = w.read_bodies()[1:], r.body_states()[1:]
        hw, hr = ws[:, 1].mean(), rs[:, 1].mean()
        assert abs(hw - hr) <= 0.05 * hr + 0.03, (k, hw, hr)
    # spheres keep rolling on both sides: kinetic energy (unit mass) is
    # compared within a factor of two
    ke_w, ke_r = 0.5 * np.sum(ws[:, 3:6] ** 2), 0.5 * np.sum(rs[:, 3:6] ** 2)
    assert ke_w <= 2.0 * ke_r + 1.0 and ke_r <= 2.0 * ke_w + 1.0, (ke_w, ke_r)
    assert abs(int(ws[:, 13].sum()) - int(rs[:, 13].sum())) <= 60
    _, _, pts = w.manifolds()
    assert -pts[..., 6].min() < 0.05
    assert np.all(np.isfinite(ws))


def test_hull_on_floor_rests_on_a_face(pkg, scenes):
    # a hexagonal prism dropped flat settles on its cap: its lowest vertex
    # rests at the floor and it falls asleep
    v, t = scenes.hull_prism(6, 0.3, 0.15)
    w = pkg.World(0)
    w.add_static_floor(0.0)
    mesh = pkg.ConvexMesh(v, t)
    b = w.create_dynamic_body((0, 0.5, 0, 0, 0, 0, 1))
    w.attach_convex_shape(b, mesh)
    del mesh                      # the world keeps its own reference
    w.update_mass_properties(b, 500.0)
    w.step(DT, steps=240)
    st = w.body_state(b)
    assert abs(st.position[1] - 0.15) < 0.02, st.position[1]
    assert st.sleeping == 1


def test_convex_validation(pkg, scenes):
    w = pkg.World(0)
    b = w.create_dynamic_body((0, 1, 0, 0, 0, 0, 1))
    mesh = pkg.ConvexMesh(*scenes.hull_box((0.2, 0.2, 0.2)))
    with pytest.raises(ValueError):
        w.attach_convex_shape(b, mesh, (np.nan, 0, 0, 0, 0, 0, 1))
    with pytest.raises(ValueError):
        w.attach_convex_shape(b, mesh, (0, 0, 0, 0, 0, 0, 2.0))
    s = w.attach_convex_shape(b, mesh)
    assert s == 0


def test_many_sided_faces_take_the_lane_zero_clipping(pkg, ref, scenes):
    # 70-sided prisms stacked flat: their caps have more vertices than the
    # warp clipping stages, so the lane-0 clipping runs; fresh manifolds
    # still match the reference
    spec = scenes.convex_pile(6, seed=1, xz=0.0, frac_other=0.0)
    spec.convex_meshes = [scenes.hull_prism(70, 0.3, 0.1)]
    spec.shape_geom[:, 0] = 0
    spec.shape_local[:] = [0, 0, 0, 0, 0, 0, 1]
    spec.bodies[:, 3:7] = [0, 0, 0, 1]
    for i in range(6):
        spec.bodies[i, 0:3] = [0.01 * i, 0.099 + 0.199 * i, 0.0]
    w = world_of(pkg, spec)
    w.collide()
    r = ref.RefScene(spec)
    r.advance_collision()
    wp, wc, wpts = w.manifolds()
    rp, rc, _, rpts = r.manifolds()
    np.testing.assert_array_equal(wp, rp)
    np.testing.assert_array_equal(wc, rc)
    assert wc.sum() >= 20
    assert rel_err(wpts, rpts) <= CONTACT_RTOL
