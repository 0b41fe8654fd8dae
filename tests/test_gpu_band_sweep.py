"""The z-band sweep of large scenes (above 2,048 finite shapes) against the
oracle's one-axis sweep, through the C ABI.

A large scene is swept per band of z: bands at least as wide as its widest
shape, a shape entered in each band its z extent touches, a pair kept only
in the band of the larger of the two min z.  The published pair set must be
the one-axis sweep's exactly, whatever the shapes: these scenes put one long
shape across the whole scene (two wide bands), every shape in one thin slab
(one band), shapes across a long z range (bands at the 1/250 floor), and two
large scenes beside a small one in one world (band keys over two scenes).

Tolerance: pair sets and found / lost sets bit-exact.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DT = 1.0 / 120.0


def boxes(scenes, n, seed, region, half=(0.1, 0.4)):
    """n random boxes: centres uniform in +-region/2 (x, z) and
    [0.5, 0.5 + region y] (y), random orientations."""
    rng = np.random.Generator(np.random.PCG64(seed))
    rx, ry, rz = region
    h = rng.uniform(half[0], half[1], (n, 3)).astype(np.float32)
    pos = np.stack([rng.uniform(-rx / 2, rx / 2, n), rng.uniform(0.5, 0.5 + ry, n),
                    rng.uniform(-rz / 2, rz / 2, n)], 1).astype(np.float32)
    quat = scenes.random_quaternions(rng, n)
    z = np.zeros((n, 3), np.float32)
    mats = np.tile(np.array([0.5, 0.5, 0.0], np.float32), (n, 1))
    return pos, quat, z, mats, [[scenes._box(h[i])] for i in range(n)]


def long_box_scene(scenes):
    """3,000 boxes over 40 x 40 m and one dynamic rod 25 m long in z: the
    band width follows the rod (two bands for the whole scene)."""
    pos, quat, z, mats, shapes = boxes(scenes, 3000, 11, (40.0, 4.0, 40.0))
    quat[0] = (0.0, 0.0, 0.0, 1.0)
    pos[0] = (0.0, 1.0, 0.0)
    shapes[0] = [scenes._box((0.1, 0.1, 12.5))]
    return scenes._assemble(pos, quat, z, z, 1000.0, shapes, mats)


def slab_scene(scenes):
    """3,000 spheres (r 0.05-0.15) with centres in a 2 mm slab of z and
    40 m of x: the z range is about one shape wide (one or two bands)."""
    rng = np.random.Generator(np.random.PCG64(12))
    n = 3000
    r = rng.uniform(0.05, 0.15, n).astype(np.float32)
    pos = np.stack([rng.uniform(-20, 20, n), rng.uniform(0.2, 2.0, n), rng.uniform(0.0, 0.002, n)],
                   1).astype(np.float32)
    quat = np.tile(np.array([0, 0, 0, 1], np.float32), (n, 1))
    z = np.zeros((n, 3), np.float32)
    mats = np.tile(np.array([0.5, 0.5, 0.0], np.float32), (n, 1))
    return scenes._assemble(pos, quat, z, z, 1000.0, [[scenes._sphere(r[i])] for i in range(n)], mats)


def long_range_scene(scenes):
    """6,000 small boxes along 400 m of z and 6 m of x: bands at the floor
    of 1/250 of the z range (wider than any box)."""
    pos, quat, z, mats, shapes = boxes(scenes, 6000, 13, (6.0, 3.0, 400.0), half=(0.05, 0.3))
    return scenes._assemble(pos, quat, z, z, 1000.0, shapes, mats)


def as_set(a):
    return set(map(tuple, np.asarray(a).tolist()))


@pytest.mark.parametrize("make", [long_box_scene, slab_scene, long_range_scene],
                         ids=["long_box", "slab", "long_range"])
def test_band_sweep_pairs_equal_oracle(pkg, oracle, scenes, make):
    spec = make(scenes)
    assert spec.n_shapes > 2048
    w = pkg.World(0)
    w.add_scene(spec)
    o = oracle.OracleScene(spec)
    w.collide()
    o.advance_collision()
    want = o.pairs(0)
    assert want.shape[0] > 1000
    np.testing.assert_array_equal(w.pairs(0), want)
    np.testing.assert_array_equal(w.pairs(1), want)
    # steps while the boxes fall: each step's pair set equals the oracle's
    # on the same poses, and the found / lost lists are the differences of
    # consecutive sets
    w.step(DT, 40)
    prev = w.pairs(0)
    for _ in range(4):
        before = w.read_bodies()
        w.step(DT)
        o.set_body_states(before)
        o.advance_collision()
        cur = w.pairs(0)
        np.testing.assert_array_equal(cur, o.pairs(0))
        assert as_set(w.pairs(1)) == as_set(cur) - as_set(prev)
        assert as_set(w.pairs(2)) == as_set(prev) - as_set(cur)
        prev = cur


def test_band_sweep_two_large_scenes_and_a_small_one(pkg, oracle, scenes):
    """Band keys of two large scenes in one world, with a small scene (the
    per-CTA sort and the plain sweep) between them."""
    specs = [long_box_scene(scenes), scenes.random_boxes(300, seed=5, xz=3.0, y=(0.3, 3.0)),
             long_range_scene(scenes)]
    w = pkg.World(0)
    firsts = [w.add_scene(s) for s in specs]
    w.collide()
    got = w.pairs(0)
    off = 0
    total = 0
    for spec in specs:
        n = spec.n_shapes + (1 if spec.floor is not None else 0)
        o = oracle.OracleScene(spec)
        o.advance_collision()
        want = o.pairs(0)
        mine = got[(got[:, 0] >= off) & (got[:, 0] < off + n)]
        assert np.all((mine[:, 1] >= off) & (mine[:, 1] < off + n))
        np.testing.assert_array_equal(mine - off, want)
        total += want.shape[0]
        off += n
    assert got.shape[0] == total
    assert firsts[0] == 1
