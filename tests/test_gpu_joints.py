"""Joint families on the B200 path (center and anchored distance, fixed,
spherical, revolute, prismatic) against the C oracle, whose joints are
pinned bit for bit to the reference's NativeCpu scene in test_oracle_joints.

One step from identical state: velocities within 1e-4 relative (the PGS
parity tolerance).  Both sides use the canonical descriptor order (joints
by constraint slot descending, then touching managers in pair order), so
short runs are compared step by step as well."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DT = 1.0 / 120.0
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


@pytest.mark.parametrize("kind", range(6))
def test_one_step_matches_oracle(pkg, oracle, scenes, kind):
    spec = scenes.joint_mechanisms(8, seed=10 + kind, kinds=[kind])
    w = world_of(pkg, spec)
    o = oracle.OracleScene(spec)
    w.step(DT)
    o.step(DT)
    ws, os_ = w.read_bodies(), o.body_states()
    assert rel_err(ws[:, 3:6], os_[:, 3:6]) <= VEL_RTOL
    assert rel_err(ws[:, 10:13], os_[:, 10:13]) <= VEL_RTOL


@pytest.mark.parametrize("kind", range(6))
def test_short_run_tracks_oracle(pkg, oracle, scenes, kind):
    spec = scenes.joint_mechanisms(8, seed=20 + kind, kinds=[kind])
    w = world_of(pkg, spec)
    o = oracle.OracleScene(spec)
    for k in range(24):
        w.step(DT)
        o.step(DT)
    ws, os_ = w.read_bodies(), o.body_states()
    assert rel_err(ws[:, 0:3], os_[:, 0:3], floor=1.0) <= 1e-4
    assert rel_err(ws[:, 3:6], os_[:, 3:6], floor=0.1) <= 1e-2


def test_mixed_kinds_statistics_vs_reference(pkg, ref, scenes):
    # 200 steps of every kind together: chains fall, swing and collide; the
    # joint frames stay together on both sides to the same degree
    spec = scenes.joint_mechanisms(24, seed=31, links=5)
    w = world_of(pkg, spec)
    r = ref.RefScene(spec)
    w.step(DT, steps=200)
    r.step(DT, 200)
    loc = spec.joint_locals()

    def rot(q, v):
        u = q[:3]
        t = 2.0 * np.cross(u, v)
        return v + q[3] * t + np.cross(u, t)

    def gaps(st):
        out = []
        for j, (a, b) in enumerate(spec.joints):
            if spec.joint_kinds()[j] < 2:
                continue
            ia = 0 if a == scenes.FLOOR_BODY else a + 1
            ib = 0 if b == scenes.FLOOR_BODY else b + 1
            pa = st[ia, 0:3] + rot(st[ia, 6:10], loc[j, 0:3])
            pb = st[ib, 0:3] + rot(st[ib, 6:10], loc[j, 7:10])
            out.append(np.linalg.norm(pa - pb))
        return np.array(out)
    gw, gr = gaps(w.read_bodies()), gaps(r.body_states())
    assert np.median(gw) < 5e-3 and np.median(gr) < 5e-3, (np.median(gw), np.median(gr))
    assert abs(np.mean(w.read_bodies()[1:, 1]) - np.mean(r.body_states()[1:, 1])) < 0.1


def test_joint_validation(pkg, scenes):
    w = pkg.World(0)
    floor = w.add_static_floor(0.0)
    a = w.create_dynamic_body((0, 1, 0, 0, 0, 0, 1))
    w.attach_box_shape(a, (0.2, 0.2, 0.2))
    b = w.create_dynamic_body((1, 1, 0, 0, 0, 0, 1))
    w.attach_box_shape(b, (0.2, 0.2, 0.2))
    ident = (0, 0, 0, 0, 0, 0, 1)
    with pytest.raises(ValueError):
        w.add_fixed_constraint(a, a, ident, ident)
    with pytest.raises(ValueError):
        w.add_revolute_constraint(a, b, (np.inf, 0, 0, 0, 0, 0, 1), ident)
    with pytest.raises(ValueError):
        w.add_spherical_constraint(a, b, (0, 0, 0, 0, 0, 0, 2.0), ident)
    with pytest.raises(ValueError):
        w.add_anchored_distance_constraint(a, b, (0, 0, 0), (0, 0, 0), -1.0)
    ids = [w.add_fixed_constraint(a, b, ident, ident), w.add_prismatic_constraint(floor, b, ident, ident),
           w.add_anchored_distance_constraint(b, a, (0.1, 0, 0), (0, 0.1, 0), 0.5)]
    assert [i & 0xFFFFFFFF for i in ids] == [0, 1, 2]
    w.step(DT, steps=3)
    assert np.all(np.isfinite(w.read_bodies()))
    with pytest.raises(RuntimeError):
        w.rollout_begin(4, 2)


def test_removed_and_added_joints_track_oracle(pkg, oracle, scenes):
    # a pile settling onto the floor with eight center distance joints: at
    # step 10 (19 touching managers) two joints are retired and two new ones
    # take their slots; the run goes on from the same contact history and
    # tracks the oracle (which keeps it, like the reference) as closely as
    # an unedited short run does
    spec = scenes.random_boxes(30, seed=5, xz=2.0, y=(0.4, 2.0))
    pairs = np.array([[2 * i, 2 * i + 1] for i in range(8)], np.uint32)
    spec.joints = pairs
    spec.joint_dist = np.linalg.norm(spec.bodies[pairs[:, 0], 0:3] - spec.bodies[pairs[:, 1], 0:3],
                                     axis=1).astype(np.float32)
    w = pkg.World(0)
    first = w.add_scene(spec)
    o = oracle.OracleScene(spec)
    for k in range(10):
        w.step(DT)
        o.step(DT)
    assert w.counts()["managers"] > 10
    for cid in ((1 << 32) | 3, (1 << 32) | 6):
        w.remove_constraint(cid)
        o.remove_joint(cid)
    st = o.body_states()
    da = float(np.linalg.norm(st[21, 0:3] - st[22, 0:3]))
    db = float(np.linalg.norm(st[7, 0:3] - st[10, 0:3]))
    got = [w.add_center_distance_constraint(first + 20, first + 21, da),
           w.add_center_distance_constraint(first + 6, first + 9, db)]
    want = [o.add_joint(0, 20, 21, None, None, da), o.add_joint(0, 6, 9, None, None, db)]
    assert got == want == [(2 << 32) | 6, (2 << 32) | 3]
    assert w.counts()["joints"] == 8
    for k in range(14):
        w.step(DT)
        o.step(DT)
    ws, os_ = w.read_bodies(), o.body_states()
    assert rel_err(ws[:, 0:3], os_[:, 0:3], floor=1.0) <= 1e-4
    assert rel_err(ws[:, 3:6], os_[:, 3:6], floor=0.1) <= 1e-2
    with pytest.raises((ValueError, RuntimeError)):
        w.remove_constraint((1 << 32) | 3)       # expired generation
    with pytest.raises((ValueError, RuntimeError)):
        w.remove_constraint((1 << 32) | 9999)    # unknown slot


def test_joint_edits_keep_device_memory_flat(pkg, scenes):
    # grab-and-release between steps: 200 add / remove edits reuse the
    # device joint tables instead of allocating new ones
    import torch
    spec = scenes.random_boxes(40, seed=8, xz=2.0, y=(0.4, 2.0))
    w = pkg.World(0)
    first = w.add_scene(spec)
    w.step(DT)
    held = w.add_center_distance_constraint(first, first + 1, 0.7)
    w.step(DT)
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for k in range(200):
        w.remove_constraint(held)
        held = w.add_center_distance_constraint(first + (k % 20), first + 20 + (k % 20), 0.7)
        w.step(DT)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free0 - free1 < 4 << 20, (free0, free1)
    assert np.all(np.isfinite(w.read_bodies()))
