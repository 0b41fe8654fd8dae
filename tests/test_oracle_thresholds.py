"""The force-threshold restatement (oracle/thresholds.py), fed by the C
oracle replaying the reference's Dy order, reproduces the reference's own
World::force_threshold_changes step by step, bit for bit (keys, changes,
double impulses, thresholds)."""
import numpy as np

import thresholds as th_mod

FLT_MAX = float(np.finfo(np.float32).max)
DT = 1.0 / 120.0


def actor_tables(spec):
    sb = np.asarray(spec.shape_body, np.int64)
    if spec.floor is None:
        return sb, np.full(spec.n_bodies, th_mod.DYNAMIC)
    return np.concatenate([[0], sb + 1]), np.concatenate([[th_mod.STATIC], np.full(spec.n_bodies, th_mod.DYNAMIC)])


def threshold_pile(scenes):
    spec = scenes.random_boxes(60, seed=11, xz=2.0, y=(0.3, 2.5))
    spec.shape_mat[:, 2] = 0.4          # restitution: impacts come and go
    # per body: a low threshold (resting contact exceeds), a high one
    # (impacts only) or none
    thr = np.array([[60.0, 1500.0, FLT_MAX][i % 3] for i in range(spec.n_bodies)], np.float32)
    return spec, thr


def test_threshold_stream_matches_reference(oracle, ref, scenes):
    spec, thr = threshold_pile(scenes)
    r = ref.RefScene(spec)
    o = oracle.OracleScene(spec)
    actor_thr = np.concatenate([[FLT_MAX], thr]).astype(np.float32)
    for i, t in enumerate(thr):
        if t != FLT_MAX:
            r.set_contact_report_threshold(i + 1, float(t))
    sb, motion = actor_tables(spec)
    builder = th_mod.ThresholdBuilder(sb, motion)
    changes = set()
    for k in range(180):
        r.step(DT)
        o.step(DT, r.manager_order(), r.joint_order())
        pairs, counts, _, _ = o.manifolds()
        sleeping = o.sleep_state()["sleeping"]
        got = builder.step(pairs, counts, o.normal_impulses(), sleeping, actor_thr, DT)
        want = r.force_threshold_changes()
        np.testing.assert_array_equal(got[0], want[0], err_msg=f"step {k}")
        np.testing.assert_array_equal(got[1], want[1], err_msg=f"step {k}")
        np.testing.assert_array_equal(got[2], want[2], err_msg=f"step {k}")
        changes |= set(want[0][:, 3].tolist())
    assert changes == {0, 1, 2}, "scene must produce found, persists and lost changes"
    assert np.any(sleeping), "the pile must fall asleep within the run"
