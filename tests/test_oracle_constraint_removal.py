"""World::remove_constraint and joints added after stepping
(scene.cpp:3088-3140 slot reuse with generations, 3195-3228 edge
retirement), as restated in the C oracle, against the reference replaying
its Dy order: chains lose links and gain new ones mid-run, with sleeping on,
and stay bit for bit equal."""
import numpy as np
import pytest

DT = 1.0 / 120.0


def run_pair(ref, oracle, spec, plan, steps):
    r = ref.RefScene(spec)
    o = oracle.OracleScene(spec)
    ids_r, ids_o = {}, {}
    for k in range(steps):
        for (at, op, key, args) in plan:
            if at != k:
                continue
            if op == "remove":
                r.remove_joint(ids_r.get(key, key))
                o.remove_joint(ids_o.get(key, key))
            else:
                ids_r[key] = r.add_joint(*args)
                ids_o[key] = o.add_joint(*args)
                assert ids_r[key] == ids_o[key], (key, ids_r[key], ids_o[key])
        r.step(DT)
        o.step(DT, r.manager_order(), r.joint_order())
        np.testing.assert_array_equal(o.body_states(), r.body_states(), err_msg=f"step {k}")
        # the reference's Dy joint order is the live slots, descending, less
        # joints of sleeping islands: the canonical order the oracle and the
        # device use
        jo = [int(x) for x in r.joint_order()]
        assert jo == sorted(jo, reverse=True), (k, jo)
    return r, o


def test_removed_and_added_joints_match_reference(ref, oracle, scenes):
    spec = scenes.joint_mechanisms(12, seed=41, links=4)
    nj = spec.joints.shape[0]
    first = [(1 << 32) | s for s in range(nj)]     # ids of the authored joints
    ident = np.array([0, 0, 0, 0, 0, 0, 1], np.float32)
    plan = [(40, "remove", first[3], None), (40, "remove", first[7], None),
            (60, "add", "x", (3, 0, 5, ident, ident, 0.0)),          # reuses slot 7, generation 2
            (80, "remove", first[1], None),
            (90, "add", "y", (0, 2, 9, None, None, 0.6)),            # reuses slot 1
            (100, "add", "z", (2, 0xFFFFFFFF, 11, ident, ident, 0.0)),  # reuses slot 3
            (150, "remove", "x", None)]
    r, o = run_pair(ref, oracle, spec, plan, 240)


def test_stale_and_unknown_ids_are_rejected(ref, oracle, scenes):
    spec = scenes.joint_mechanisms(4, seed=2, links=3)
    for s in (ref.RefScene(spec), oracle.OracleScene(spec)):
        s.step(DT)
        s.remove_joint((1 << 32) | 0)
        with pytest.raises(RuntimeError):
            s.remove_joint((1 << 32) | 0)          # already retired
        new = s.add_joint(0, 0, 1, None, None, 0.5)
        assert new == (2 << 32) | 0
        with pytest.raises(RuntimeError):
            s.remove_joint((1 << 32) | 0)          # stale generation
        with pytest.raises(RuntimeError):
            s.remove_joint((1 << 32) | 999)        # unknown slot
