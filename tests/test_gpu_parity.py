"""B200 kernels against the oracle and the reference, through the C ABI.

Tolerances (from the step's parity targets):
  integer work (encoded bounds, sorted endpoints, pair sets)   bit-exact
  contact points / normals / depths from identical poses      1e-5 relative
  one PGS step from identical state (velocities)               1e-4 relative
Relative errors use max(|ref|, FLOOR) as the denominator so near-zero
components are compared absolutely.
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


def make_world(pkg, specs):
    w = pkg.World(0)
    firsts = [w.add_scene(s) for s in specs]
    return w, firsts


@pytest.fixture(scope="module")
def cases(scenes):
    return {
        "boxes": scenes.random_boxes(400, seed=3, xz=4.0, y=(0.3, 6.0)),
        "mixed": scenes.mixed_scale(600, seed=2, region=(8.0, 4.0, 8.0), joint_frac=0.05),
        "stack": scenes.box_stack_scene(60, seed=7),
    }


@pytest.mark.parametrize("name", ["boxes", "mixed", "stack"])
def test_bounds_sort_pairs_bitexact(pkg, oracle, cases, name):
    spec = cases[name]
    w, _ = make_world(pkg, [spec])
    o = oracle.OracleScene(spec)
    w.collide()
    o.advance_collision()
    np.testing.assert_array_equal(w.encoded_bounds(), o.encoded_bounds())
    v, i = w.sorted_min_x(0)
    ov, oi = o.sorted_min_x()
    np.testing.assert_array_equal(v, ov)
    np.testing.assert_array_equal(i, oi)
    np.testing.assert_array_equal(w.pairs(0), o.pairs(0))
    np.testing.assert_array_equal(w.pairs(1), o.pairs(1))


@pytest.mark.parametrize("name", ["boxes", "mixed", "stack"])
def test_fresh_manifolds_match_reference(pkg, oracle, ref, cases, name):
    spec = cases[name]
    w, _ = make_world(pkg, [spec])
    w.collide()
    r = ref.RefScene(spec)
    r.advance_collision()
    wp, wc, wpts = w.manifolds()
    rp, rc, _, rpts = r.manifolds()
    np.testing.assert_array_equal(wp, rp)
    np.testing.assert_array_equal(wc, rc)
    assert rel_err(wpts, rpts) <= CONTACT_RTOL


@pytest.mark.parametrize("name", ["boxes", "mixed", "stack"])
def test_one_step_matches_oracle(pkg, oracle, cases, name):
    spec = cases[name]
    w, _ = make_world(pkg, [spec])
    o = oracle.OracleScene(spec)
    w.step(DT)
    o.step(DT)
    np.testing.assert_array_equal(w.pairs(0), o.pairs(0))
    ws, os_ = w.read_bodies(), o.body_states()
    assert rel_err(ws[:, 3:6], os_[:, 3:6]) <= VEL_RTOL
    assert rel_err(ws[:, 10:13], os_[:, 10:13]) <= VEL_RTOL
    assert rel_err(ws[:, 0:3], os_[:, 0:3]) <= VEL_RTOL


def oracle_levels(o, n_joints):
    """Per-descriptor partition in canonical order (joints, then managers)."""
    desc, ends = o.partitions()
    man = o.counts()["manifolds"]
    levels = np.zeros(n_joints + man, np.uint32)
    start = 0
    for p, e in enumerate(ends):
        for d in desc[start:int(e)]:
            idx = int(d[0]) if d[3] else n_joints + int(d[0])
            levels[idx] = p
        start = int(e)
    return levels


def wave_scene(scenes):
    # One 10 x 0.2 x 10 m slab carrying 40 small boxes: the slab's 40
    # dynamic contacts overflow the 32-bit partition mask into a second wave.
    n_small = 40
    nb = 1 + n_small
    bodies = np.zeros((nb, 14), np.float32)
    bodies[:, 6] = 1.0
    bodies[:, 13] = 1000.0
    bodies[0, :3] = (0.0, 0.1, 0.0)
    geom = np.zeros((nb, 4), np.float32)
    geom[0, :3] = (5.0, 0.1, 5.0)
    for i in range(n_small):
        gx, gz = divmod(i, 7)
        bodies[1 + i, :3] = (-4.0 + 1.3 * gx, 0.2 + 0.25, -4.0 + 1.3 * gz)
        geom[1 + i, :3] = (0.25, 0.25, 0.25)
    local = np.tile(np.array([0, 0, 0, 0, 0, 0, 1], np.float32), (nb, 1))
    mat = np.tile(np.array([0.5, 0.5, 0.0], np.float32), (nb, 1))
    return scenes.SceneSpec(bodies=bodies, shape_body=np.arange(nb, dtype=np.uint32),
                            shape_type=np.zeros(nb, np.uint32), shape_geom=geom,
                            shape_local=local, shape_mat=mat, floor=0.0)


@pytest.mark.parametrize("name", ["dense", "wave", "mixed"])
def test_partition_levels_match_oracle(pkg, oracle, scenes, cases, name):
    spec = {"dense": scenes.random_boxes(1200, seed=4, xz=3.0, y=(0.3, 9.0)),
            "wave": wave_scene(scenes), "mixed": cases["mixed"]}[name]
    w, _ = make_world(pkg, [spec])
    o = oracle.OracleScene(spec)
    w.step(DT)
    o.step(DT)
    want = oracle_levels(o, spec.joints.shape[0])
    got = w.levels()
    np.testing.assert_array_equal(got, want)
    if name == "wave":
        assert want.max() >= 32, "scene must exercise a second partition wave"


def test_one_step_matches_reference_sparse(pkg, ref, scenes):
    # Bodies touch only the floor or one partner, so every island's
    # descriptor order is forced and the reference's order coincides.
    spec = scenes.mixed_scale(300, seed=5, region=(40.0, 0.6, 40.0), joint_frac=0.0)
    spec.bodies[:, 1] = 0.32
    w, _ = make_world(pkg, [spec])
    r = ref.RefScene(spec)
    w.step(DT)
    r.step(DT)
    ws, rs = w.read_bodies(), r.body_states()
    assert rel_err(ws[:, 3:6], rs[:, 3:6]) <= VEL_RTOL
    assert rel_err(ws[:, 10:13], rs[:, 10:13]) <= VEL_RTOL


def test_multi_step_tracks_oracle(pkg, oracle, cases):
    spec = cases["mixed"]
    w, _ = make_world(pkg, [spec])
    o = oracle.OracleScene(spec)
    for k in range(8):
        w.step(DT)
        o.step(DT)
    ws, os_ = w.read_bodies(), o.body_states()
    assert rel_err(ws[:, 0:3], os_[:, 0:3], floor=1.0) <= 1e-4


def test_pairs_found_lost_consistency(pkg, oracle, cases):
    spec = cases["boxes"]
    w, _ = make_world(pkg, [spec])
    prev = np.zeros((0, 2), np.uint32)
    for k in range(20):
        before = w.read_bodies()
        w.step(DT)
        cur = w.pairs(0)
        # the step's pair set equals the oracle's set on the same poses
        o = oracle.OracleScene(spec)
        o.set_body_states(before)
        o.advance_collision()
        np.testing.assert_array_equal(cur, o.pairs(0))
        key = lambda a: set(map(tuple, a.tolist()))
        assert key(w.pairs(1)) == key(cur) - key(prev)
        assert key(w.pairs(2)) == key(prev) - key(cur)
        prev = cur


def test_batched_equals_single_scene_worlds(pkg, scenes):
    specs = scenes.batched_scenes(12, low=16, high=200, base_seed=100)
    wb, firsts = make_world(pkg, specs)
    wb.step(DT, steps=5)
    sb = wb.read_bodies()
    for spec, first in zip(specs, firsts):
        ws, (f1,) = make_world(pkg, [spec])
        ws.step(DT, steps=5)
        s1 = ws.read_bodies()
        n = spec.n_actors
        np.testing.assert_array_equal(sb[first - 1: first - 1 + n], s1[f1 - 1: f1 - 1 + n])


def test_batched_one_step_matches_oracle(pkg, oracle, scenes):
    specs = scenes.batched_scenes(8, low=16, high=120, base_seed=7)
    wb, firsts = make_world(pkg, specs)
    wb.step(DT)
    sb = wb.read_bodies()
    for spec, first in zip(specs, firsts):
        o = oracle.OracleScene(spec)
        o.step(DT)
        n = spec.n_actors
        assert rel_err(sb[first - 1: first - 1 + n, 3:6], o.body_states()[:, 3:6]) <= VEL_RTOL


def test_pair_capacity_growth(pkg, scenes):
    # 256 boxes at one spot overlap pairwise: far beyond the initial budget.
    spec = scenes.random_boxes(256, seed=1, xz=0.05, y=(2.0, 2.1))
    w, _ = make_world(pkg, [spec])
    w.collide()
    n = w.counts()["pairs"]
    assert n >= 256 * 255 // 2
    w.step(DT)
    assert np.all(np.isfinite(w.read_bodies()))


def test_empty_and_floor_only_worlds(pkg, scenes):
    w = pkg.World(0)
    w.add_static_floor(0.0)
    w.step(DT)
    assert w.counts()["pairs"] == 0
    spec = scenes.random_boxes(5, seed=2)
    spec.floor = None
    w2, _ = make_world(pkg, [spec])
    w2.step(DT, steps=3)
    st = w2.read_bodies()
    # free fall: v_y = -9.81 * 3 dt exactly as the reference accumulates it
    assert np.allclose(st[:, 4], -9.81 * 3 * DT, rtol=1e-5)


def test_long_run_statistics_vs_reference(pkg, ref, scenes):
    # Plain single scene (1,000 boxes, 300 steps): trajectories are chaotic,
    # so long runs are compared by kinetic-energy, height and penetration
    # statistics.  Reference vs C oracle on this workload agree to ~2% in
    # mean height and ~15% in kinetic energy at the settling stage.
    spec = scenes.random_boxes(1000, seed=0)
    w, _ = make_world(pkg, [spec])
    r = ref.RefScene(spec)
    for k in range(10):
        w.step(DT, steps=30)
        r.step(DT, 30)
        ws, rs = w.read_bodies()[1:], r.body_states()[1:]
        hw, hr = ws[:, 1].mean(), rs[:, 1].mean()
        assert abs(hw - hr) <= 0.05 * hr + 0.02, (k, hw, hr)
        ke_w, ke_r = 0.5 * np.sum(ws[:, 3:6] ** 2), 0.5 * np.sum(rs[:, 3:6] ** 2)
        assert abs(ke_w - ke_r) <= 0.35 * ke_r + 50.0, (k, ke_w, ke_r)
    _, _, pts = w.manifolds()
    assert -pts[..., 6].min() < 0.25
    assert np.all(np.isfinite(ws))


def test_gjk_epa_manifolds_match_reference(pkg, ref, scenes):
    # Densely overlapping rotated boxes: many pairs have no face contact and
    # finish through GJK/EPA (the warp-cooperative continuation).
    spec = scenes.random_boxes(500, seed=9, xz=2.5, y=(0.3, 3.0))
    w, _ = make_world(pkg, [spec])
    w.collide()
    assert w.step_counters()["gjk_pairs"] > 0
    r = ref.RefScene(spec)
    r.advance_collision()
    wp, wc, wpts = w.manifolds()
    rp, rc, _, rpts = r.manifolds()
    np.testing.assert_array_equal(wp, rp)
    np.testing.assert_array_equal(wc, rc)
    assert rel_err(wpts, rpts) <= CONTACT_RTOL


def test_fit_pair_budget_keeps_the_trajectory(pkg, scenes):
    # Shrinking the pair budget keeps the contact-manager history: the run
    # continues bit for bit as without it.
    spec = scenes.random_boxes(300, seed=12, xz=2.0, y=(0.3, 4.0))
    wa, _ = make_world(pkg, [spec])
    wb, _ = make_world(pkg, [spec])
    wa.step(DT, steps=20)
    wb.step(DT, steps=20)
    before = wa.counts()["pairs"]
    budget = wa.fit_pair_budget(1.2)
    # both generations stay: the budget covers the larger one
    assert before <= budget <= int(1.5 * before) + 4097
    wa.step(DT, steps=20)
    wb.step(DT, steps=20)
    np.testing.assert_array_equal(wa.read_bodies(), wb.read_bodies())
    np.testing.assert_array_equal(wa.pairs(0), wb.pairs(0))


def test_write_states_equals_write_velocities(pkg, scenes):
    # the 14-float records written back as they are give the same state as
    # the 6-float velocity records
    spec = scenes.random_boxes(300, seed=12, xz=3.0, y=(0.3, 4.0))
    wa, _ = make_world(pkg, [spec])
    wb, _ = make_world(pkg, [spec])
    wa.step(DT, steps=20)
    wb.step(DT, steps=20)
    st = wa.read_bodies()
    rng = np.random.default_rng(0)
    st[:, 3:6] += rng.normal(0, 0.5, (st.shape[0], 3)).astype(np.float32)
    st[:, 10:13] += rng.normal(0, 0.5, (st.shape[0], 3)).astype(np.float32)
    wa.write_states(np.ascontiguousarray(st))
    wb.write_velocities(np.concatenate([st[:, 3:6], st[:, 10:13]], 1))
    np.testing.assert_array_equal(wa.read_bodies(), wb.read_bodies())
    wa.step(DT, steps=5)
    wb.step(DT, steps=5)
    np.testing.assert_array_equal(wa.read_bodies(), wb.read_bodies())
