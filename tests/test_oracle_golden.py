"""The C restatement oracle against golden vectors produced by the reference
itself (tests/golden/make_golden.py).  Integer work must be bit-exact; the
float work is also bit-exact because the oracle evaluates every expression
in the reference's order without FMA contraction."""
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")


def _golden_specs():
    import sys
    sys.path.insert(0, GOLDEN)
    import make_golden
    return make_golden.golden_scenes(), make_golden.STEPS, make_golden.DT


def test_gu_candidates_selection_gjk(oracle):
    g = np.load(os.path.join(GOLDEN, "golden_gu.npz"))
    assert g["a"].shape[0] >= 400
    n_gjk = 0
    for i in range(g["a"].shape[0]):
        ok, c = oracle.pcm_box_box_candidates(g["a"][i], g["b"][i], 0.04)
        assert ok == bool(g["ok"][i])
        assert c.shape[0] == g["counts"][i]
        np.testing.assert_array_equal(c, g["cands"][i][: c.shape[0]])
        if c.shape[0] > 4:
            np.testing.assert_array_equal(oracle.pcm_batch_selection(c), g["sel"][i])
        if ok and c.shape[0] == 0:
            n_gjk += 1
            gok, w = oracle.pcm_box_box_gjk_epa(g["a"][i], g["b"][i], 0.04)
            assert gok == bool(g["gjk_ok"][i])
            if gok:
                np.testing.assert_array_equal(w, g["gjk"][i])
    assert n_gjk > 0, "fixture must exercise the GJK/EPA continuation"


@pytest.mark.parametrize("name", ["boxes", "mixed", "stack"])
def test_scene_collision_and_steps(oracle, name):
    specs, steps, dt = _golden_specs()
    spec = specs[name]
    g = np.load(os.path.join(GOLDEN, f"golden_{name}.npz"))
    o = oracle.OracleScene(spec)
    np.testing.assert_array_equal(o.mass_props(), g["mass"])
    o.advance_collision()
    np.testing.assert_array_equal(o.encoded_bounds(), g["bounds"])
    np.testing.assert_array_equal(o.pairs(), g["pairs"])
    p, c, r, pts = o.manifolds()
    np.testing.assert_array_equal(p, g["man_pairs"])
    np.testing.assert_array_equal(c, g["man_counts"])
    np.testing.assert_array_equal(r, g["man_rev"])
    np.testing.assert_array_equal(pts, g["man_pts"])
    v, i = o.sorted_min_x()
    np.testing.assert_array_equal(v, g["minx_vals"])
    np.testing.assert_array_equal(i, g["minx_ids"])
    o2 = oracle.OracleScene(spec)
    for k in range(steps):
        o2.step(dt, g[f"order_{k}"], g[f"jorder_{k}"])
        np.testing.assert_array_equal(o2.pairs(1), g[f"found_{k}"])
        np.testing.assert_array_equal(o2.pairs(2), g[f"lost_{k}"])
        np.testing.assert_array_equal(o2.body_states(), g["states"][k])


def test_edge_cases_empty_and_floor_only(oracle, scenes):
    empty = scenes.SceneSpec(bodies=np.zeros((0, 14), np.float32),
                             shape_body=np.zeros(0, np.uint32), shape_type=np.zeros(0, np.uint32),
                             shape_geom=np.zeros((0, 4), np.float32), shape_local=np.zeros((0, 7), np.float32),
                             shape_mat=np.zeros((0, 3), np.float32), floor=None)
    o = oracle.OracleScene(empty)
    o.step()
    assert o.counts()["pairs"] == 0
    floor_only = scenes.SceneSpec(bodies=np.zeros((0, 14), np.float32),
                                  shape_body=np.zeros(0, np.uint32), shape_type=np.zeros(0, np.uint32),
                                  shape_geom=np.zeros((0, 4), np.float32), shape_local=np.zeros((0, 7), np.float32),
                                  shape_mat=np.zeros((0, 3), np.float32), floor=0.0)
    o = oracle.OracleScene(floor_only)
    o.step()
    assert o.counts()["pairs"] == 0 and o.counts()["actors"] == 1


def test_encoding_known_answers(oracle):
    L = oracle.lib()
    # order preservation across the sign boundary and the 4-bit expansion
    vals = np.array([-1e30, -2.5, -1e-30, -0.0, 0.0, 1e-30, 2.5, 1e30], np.float32)
    mins = [L.fo_encode_min(float(v)) for v in vals]
    maxs = [L.fo_encode_max(float(v)) for v in vals]
    assert all(a <= b for a, b in zip(mins, mins[1:]))
    assert all(a <= b for a, b in zip(maxs, maxs[1:]))
    assert all(m & 0xF == 0 for m in mins) and all(m & 0xF == 4 for m in maxs)
    for lo, hi in zip(mins, maxs):
        assert lo < hi
