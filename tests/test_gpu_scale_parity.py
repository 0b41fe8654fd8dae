"""The plain at-scale scene's own code paths against the oracle, through the
C ABI.

The 131,072-body scene runs paths the small parity scenes never reach: the
device-wide radix sort of the endpoints (scenes above 2,048 finite shapes),
the sweep and pair matching at ~150k-400k pairs, and the CTA-per-island
solvers with shared-memory deltas.  A block of touching cubes adds one
island above 4,096 descriptors, which takes the global-memory partition
rounds and PGS.

Tolerances (the step's parity targets):
  integer work (encoded bounds, sorted endpoints, pair sets,
  found / lost sets, partition levels)                         bit-exact
  one step from identical state (velocities, poses)             1e-4 relative
Relative errors use max(|ref|, 1e-3) as the denominator.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DT = 1.0 / 120.0
VEL_RTOL = 1e-4
FLOOR = 1e-3
N_PLAIN = 131072


def rel_err(a, b, floor=FLOOR):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), floor))) if a.size else 0.0


def plain_spec(scenes, n=N_PLAIN):
    side = 200.0 * (n / 131072.0) ** 0.5
    return scenes.mixed_scale(n, seed=1, region=(side, 50.0, side))


def as_set(a):
    return set(map(tuple, np.asarray(a).tolist()))


def oracle_levels(o, n_joints):
    desc, ends = o.partitions()
    levels = np.zeros(n_joints + o.counts()["manifolds"], np.uint32)
    start = 0
    for p, e in enumerate(ends):
        for d in desc[start:int(e)]:
            levels[int(d[0]) if d[3] else n_joints + int(d[0])] = p
        start = int(e)
    return levels


def test_plain_scene_collide_bitexact(pkg, oracle, scenes):
    """Bounds, the radix-sorted min-x endpoints and the fresh pair set of the
    131,072-body scene."""
    spec = plain_spec(scenes)
    w = pkg.World(0)
    w.add_scene(spec)
    w.collide()
    o = oracle.OracleScene(spec)
    o.advance_collision()
    assert spec.n_shapes > 2048            # above the per-CTA sort: the radix path
    np.testing.assert_array_equal(w.encoded_bounds(), o.encoded_bounds())
    v, i = w.sorted_min_x(0)
    ov, oi = o.sorted_min_x()
    assert v.shape[0] == spec.n_shapes
    np.testing.assert_array_equal(v, ov)
    np.testing.assert_array_equal(i, oi)
    got, want = w.pairs(0), o.pairs(0)
    assert want.shape[0] > 100000
    np.testing.assert_array_equal(got, want)
    np.testing.assert_array_equal(w.pairs(1), want)     # every pair of a fresh scene is found
    assert w.pairs(2).shape[0] == 0


def test_plain_scene_found_lost_while_landing(pkg, oracle, scenes):
    """Ten consecutive steps while the pile lands (steps 241-250): each step's
    endpoints and pair set equal the oracle's on the same poses, and the
    device's found / lost lists equal the differences of consecutive sets."""
    spec = plain_spec(scenes)
    w = pkg.World(0)
    w.add_scene(spec)
    w.step(DT, steps=240)
    prev = w.pairs(0)
    o = oracle.OracleScene(spec)
    total_found = total_lost = 0
    for k in range(10):
        before = w.read_bodies()
        w.step(DT)
        o.set_body_states(before)
        o.advance_collision()
        np.testing.assert_array_equal(w.encoded_bounds(), o.encoded_bounds())
        v, i = w.sorted_min_x(0)
        ov, oi = o.sorted_min_x()
        np.testing.assert_array_equal(v, ov)
        np.testing.assert_array_equal(i, oi)
        cur = w.pairs(0)
        np.testing.assert_array_equal(cur, o.pairs(0))
        found, lost = w.pairs(1), w.pairs(2)
        assert as_set(found) == as_set(cur) - as_set(prev)
        assert as_set(lost) == as_set(prev) - as_set(cur)
        # both lists come out in canonical (shape a, shape b) order
        assert np.all(np.diff(found[:, 0].astype(np.int64) * 2**32 + found[:, 1]) > 0) if len(found) > 1 else True
        total_found += len(found)
        total_lost += len(lost)
        prev = cur
    assert total_found > 0 and total_lost > 0


def test_plain_scene_one_step_from_landed_state(pkg, oracle, scenes):
    """One step of the landed 131,072-body pile (its state after 360 steps),
    started fresh on both sides: pairs and partition levels bit-exact,
    velocities and poses within 1e-4, with the CTA-per-island solvers in
    use."""
    spec = plain_spec(scenes)
    w0 = pkg.World(0)
    w0.add_scene(spec)
    w0.step(DT, steps=360)
    start = scenes.with_state(spec, w0.read_bodies())
    w0.close()
    w = pkg.World(0)
    w.add_scene(start)
    w.set_sleeping(False)
    o = oracle.OracleScene(start)
    o.set_sleeping(False)
    w.step(DT)
    o.step(DT)
    np.testing.assert_array_equal(w.pairs(0), o.pairs(0))
    sc = w.step_counters()
    assert sc["managers"] > 100000
    assert sc["islands_512_4096"] + sc["islands_96_512"] > 0
    np.testing.assert_array_equal(w.levels(), oracle_levels(o, start.joints.shape[0]))
    ws, os_ = w.read_bodies(), o.body_states()
    assert rel_err(ws[:, 3:6], os_[:, 3:6]) <= VEL_RTOL
    assert rel_err(ws[:, 10:13], os_[:, 10:13]) <= VEL_RTOL
    assert rel_err(ws[:, 0:3], os_[:, 0:3], floor=1.0) <= VEL_RTOL


def test_island_above_4096_descriptors(pkg, oracle, scenes):
    """A 12 x 30 x 12 block of touching cubes is one island of more than
    4,096 descriptors: partition rounds and PGS in global memory.  Levels
    equal the oracle's sequential greedy; one step within 1e-4."""
    spec = scenes.cube_block(12, 30, 12)
    w = pkg.World(0)
    w.add_scene(spec)
    o = oracle.OracleScene(spec)
    w.step(DT)
    o.step(DT)
    sc = w.step_counters()
    assert sc["islands_4096_up"] == 1
    assert sc["descriptors"] > 4096
    np.testing.assert_array_equal(w.pairs(0), o.pairs(0))
    want = oracle_levels(o, 0)
    np.testing.assert_array_equal(w.levels(), want)
    ws, os_ = w.read_bodies(), o.body_states()
    assert rel_err(ws[:, 3:6], os_[:, 3:6]) <= VEL_RTOL
    assert rel_err(ws[:, 10:13], os_[:, 10:13]) <= VEL_RTOL
    assert rel_err(ws[:, 0:3], os_[:, 0:3], floor=1.0) <= VEL_RTOL
    # a second step keeps the island in the large class and stays finite
    w.step(DT)
    assert w.step_counters()["islands_4096_up"] == 1
    assert np.all(np.isfinite(w.read_bodies()))
