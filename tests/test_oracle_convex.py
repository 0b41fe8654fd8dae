"""Cooked convex hulls as restated in the C oracle, pinned to the reference:
cooking (cooked_convex.cpp:41-330: bounds, planar face polygons, density-one
mass properties), the convex Gu functions (GuPCMGjkEpa.cpp:528-804:
GJK/EPA with extreme-vertex supports and sphere point cores, face
clipping) on seeded random poses, and whole scenes of hulls, boxes and
spheres on a floor (scene.cpp:1258-1298 bounds, 3655-3772 convex
manifolds, 3774-3972 hull vertices against the plane, compound.cpp
convex mass) stepped side by side, all bit for bit."""
import numpy as np
import pytest

DT = 1.0 / 120.0


def meshes_under_test(scenes):
    rng = np.random.Generator(np.random.PCG64(7))
    return [scenes.hull_prism(6, 0.3, 0.2), scenes.hull_prism(5, 0.25, 0.2, taper=0.5, phase=0.3),
            scenes.hull_bipyramid(5, 0.2, 0.3), scenes.hull_box((0.3, 0.2, 0.25)),
            scenes.hull_random(rng, 30, (0.3, 0.2, 0.25)), scenes.hull_random(rng, 12, (0.15, 0.3, 0.2))]


def test_cooking_matches_reference(ref, oracle, scenes):
    for k, (v, t) in enumerate(meshes_under_test(scenes)):
        r = ref.cook_convex(v, t)
        o = oracle.cook_convex(v, t)
        for key in ("faces", "idx", "center", "inertia", "lo", "hi"):
            np.testing.assert_array_equal(o[key], r[key], err_msg=f"mesh {k} {key}")
        assert o["volume"] == r["volume"]
    # the prism's caps are fans of 4 triangles each, cooked to one hexagon
    r = ref.cook_convex(*scenes.hull_prism(6, 0.3, 0.2))
    assert sorted(r["faces"][:, 5].astype(int).tolist()) == [4] * 6 + [6, 6]


def test_cooking_rejects_what_the_reference_rejects(ref, scenes):
    v, t = scenes.hull_box((0.2, 0.2, 0.2))
    with pytest.raises(ValueError):
        ref.cook_convex(v, t[:-1])                  # open surface
    with pytest.raises(ValueError):
        ref.cook_convex(v, t[:, ::-1])              # inward wound


def random_shape(rng, mesh_count, kind):
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    d = np.zeros(11, np.float32)
    d[3:6] = rng.uniform(-0.25, 0.25, 3)
    d[6:10] = q
    if kind == "sphere":
        r = rng.uniform(0.1, 0.3)
        d[0:3] = r
        d[10] = r
        return d, -1
    if kind == "box":
        d[0:3] = rng.uniform(0.1, 0.3, 3)
        return d, -1
    return d, int(rng.integers(0, mesh_count))


def half_of(cooked, d, m):
    if m < 0:
        return d
    d = d.copy()
    d[0:3] = 0.5 * (cooked[m]["hi"] - cooked[m]["lo"])
    return d


@pytest.mark.parametrize("kinds", [("hull", "hull"), ("hull", "box"), ("box", "hull"), ("hull", "sphere"),
                                   ("sphere", "hull")])
def test_convex_gu_functions_match_reference(ref, oracle, scenes, kinds):
    meshes = meshes_under_test(scenes)
    cooked = [ref.cook_convex(v, t) for v, t in meshes]
    R = ref.RefConvexGu(meshes)
    O = oracle.OracleConvexGu(meshes)
    rng = np.random.Generator(np.random.PCG64(sum(map(ord, "".join(kinds)))))
    hits = faces = 0
    for it in range(400):
        a, ma = random_shape(rng, len(meshes), kinds[0])
        b, mb = random_shape(rng, len(meshes), kinds[1])
        a, b = half_of(cooked, a, ma), half_of(cooked, b, mb)
        ok_r, wr = R.gjk_epa(a, ma, b, mb, 0.04)
        ok_o, wo = O.gjk_epa(a, ma, b, mb, 0.04)
        assert ok_r == ok_o, it
        np.testing.assert_array_equal(wo, wr, err_msg=f"pair {it}")
        if ok_r:
            hits += 1
            cr = R.face_contacts(a, ma, b, mb, 0.04, wr)
            co = O.face_contacts(a, ma, b, mb, 0.04, wr)
            np.testing.assert_array_equal(co, cr, err_msg=f"pair {it}")
            faces += len(cr) > 0
    assert hits >= 100, hits
    if "sphere" not in kinds:
        assert faces >= 20, faces


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_convex_pile_matches_reference(ref, oracle, scenes, seed):
    spec = scenes.convex_pile(40, seed=seed)
    r = ref.RefScene(spec)
    o = oracle.OracleScene(spec)
    np.testing.assert_array_equal(o.mass_props(), r.mass_props())
    np.testing.assert_array_equal(o.encoded_bounds(), r.encoded_bounds())
    for k in range(300):
        r.step(DT)
        o.step(DT, r.manager_order(), r.joint_order())
        np.testing.assert_array_equal(o.body_states(), r.body_states(), err_msg=f"step {k}")
    st = r.body_states()
    assert np.all(st[1:, 1] > -0.05) and np.all(st[1:, 1] < 1.0)    # at rest on the floor


def test_convex_pile_sleeps_like_reference(ref, oracle, scenes):
    spec = scenes.convex_pile(24, seed=5, xz=1.0, frac_other=0.0)
    r = ref.RefScene(spec)
    o = oracle.OracleScene(spec)
    for k in range(500):
        r.step(DT)
        o.step(DT, r.manager_order(), r.joint_order())
    np.testing.assert_array_equal(o.body_states(), r.body_states())
    assert r.body_states()[1:, 13].sum() >= 12


def test_product_cooking_matches_reference(pkg, ref, scenes):
    """The product's cooking (host code behind fyzz_b200_cook_convex_mesh)
    gives the reference's faces, loops, volume, centre, inertia and bounds
    bit for bit, and rejects what the reference rejects."""
    for k, (v, t) in enumerate(meshes_under_test(scenes)):
        got = pkg.ConvexMesh(v, t).info()
        want = ref.cook_convex(v, t)
        for key in ("faces", "idx", "center", "inertia", "lo", "hi"):
            np.testing.assert_array_equal(got[key], want[key], err_msg=f"mesh {k} {key}")
        assert got["volume"] == want["volume"]
    v, t = scenes.hull_box((0.2, 0.2, 0.2))
    bad = [(v, t[:-1]),                                     # open
           (v, t[:, ::-1]),                                 # inward
           (v[:3], t[:4] % 3),                              # too few vertices
           (np.vstack([v, [[0.0, 0.0, 0.0]]]), t),          # unused (interior) vertex
           (v * np.float32(np.nan), t),                     # not finite
           (v, np.vstack([t, t[:1]]))]                      # duplicated triangle
    for i, (bv, bt) in enumerate(bad):
        with pytest.raises(ValueError):
            ref.cook_convex(bv, bt)
        with pytest.raises(ValueError):
            pkg.ConvexMesh(bv, bt)


@pytest.mark.parametrize("scale", [0.02, 25.0])
def test_convex_gu_functions_match_reference_at_scale(ref, oracle, scenes, scale):
    # tiny and large hulls: the scale-relative facet admission and witness
    # tolerance of the hull EPA (GuPCMGjkEpa.cpp:210-213, 296-302)
    meshes = [(v * np.float32(scale), t) for v, t in meshes_under_test(scenes)]
    cooked = [ref.cook_convex(v, t) for v, t in meshes]
    R = ref.RefConvexGu(meshes)
    O = oracle.OracleConvexGu(meshes)
    rng = np.random.Generator(np.random.PCG64(int(scale * 100)))
    hits = 0
    for it in range(300):
        a, ma = random_shape(rng, len(meshes), "hull")
        b, mb = random_shape(rng, len(meshes), "hull")
        a[3:6] *= scale
        b[3:6] *= scale
        a, b = half_of(cooked, a, ma), half_of(cooked, b, mb)
        cd = 0.04 * scale
        ok_r, wr = R.gjk_epa(a, ma, b, mb, cd)
        ok_o, wo = O.gjk_epa(a, ma, b, mb, cd)
        assert ok_r == ok_o, it
        np.testing.assert_array_equal(wo, wr, err_msg=f"pair {it}")
        if ok_r:
            hits += 1
            np.testing.assert_array_equal(O.face_contacts(a, ma, b, mb, cd, wr), R.face_contacts(a, ma, b, mb, cd, wr))
    assert hits >= 80, hits


def test_hull_riders_on_a_kinematic_hull_platform(ref, oracle, scenes):
    spec = scenes.kinematic_platform(12, seed=5)
    spec.convex_meshes = [scenes.hull_box((1.5, 0.1, 1.5)), scenes.hull_prism(6, 0.15, 0.1),
                          scenes.hull_bipyramid(5, 0.12, 0.15)]
    spec.shape_type[:] = scenes.CONVEX
    spec.shape_geom[:, 0] = [0] + [1 + (i % 2) for i in range(12)]
    r = ref.RefScene(spec)
    o = oracle.OracleScene(spec)
    r.set_kinematic(0)
    o.set_kinematic(0)
    for k in range(200):
        if k < 120:
            tg = scenes.platform_target(k)
            r.set_kinematic_target(0, tg)
            o.set_kinematic_target(0, tg)
        r.step(DT)
        o.step(DT, r.manager_order(), r.joint_order())
        np.testing.assert_array_equal(o.body_states(), r.body_states(), err_msg=f"step {k}")
    assert r.counts()["manifolds"] >= 8
