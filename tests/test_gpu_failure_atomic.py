"""Failure atomicity of the step (Scene::step's checkpoint and rollback,
src/native/scene.cpp:9706-10020, 11013-11016 of the reference), through the
C ABI.  Failures are made on the host (a pair budget too small for the
scene, a non-finite velocity written in bulk) or through the scan's test
hook; none of them faults the device.

  * a rollback keeps the contact-manager history, so a world that outgrows
    its pair budget mid-run ends bit-identical to one that had room;
  * a non-finite state raises OverflowError with the pre-step state intact,
    and the world steps on normally once the input is fixed;
  * the look-back scan's bounded wait gives up, reports a logic error, and
    later scans and steps run clean.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DT = 1.0 / 120.0
K_ERR_LOGIC = 1 << 7


def world(pkg, spec):
    w = pkg.World(0)
    w.add_scene(spec)
    return w


def test_tiny_pair_budget_ends_bit_identical(pkg, scenes):
    # a 600-box pile lands: its pairs outgrow a 64-pair budget several times,
    # inside one 30-step batch (wa) and between single steps (wc)
    spec = scenes.random_boxes(600, seed=31, xz=3.0, y=(0.3, 8.0))
    wa, wb, wc = world(pkg, spec), world(pkg, spec), world(pkg, spec)
    assert wa.set_pair_budget(64) == 64
    assert wc.set_pair_budget(64) == 64
    wa.step(DT, steps=30)
    wb.step(DT, steps=30)
    for _ in range(30):
        wc.step(DT)
    assert wb.counts()["pairs"] > 256
    assert wb.counts()["managers"] > 100
    want = wb.read_bodies()
    np.testing.assert_array_equal(wa.read_bodies(), want)
    np.testing.assert_array_equal(wc.read_bodies(), want)
    np.testing.assert_array_equal(wa.pairs(0), wb.pairs(0))
    np.testing.assert_array_equal(wc.pairs(0), wb.pairs(0))
    # the histories themselves: friction anchors of the last step
    for w in (wa, wc):
        got, ref = w.friction_anchors(), wb.friction_anchors()
        for g, r in zip(got, ref):
            np.testing.assert_array_equal(g, r)


def test_nonfinite_velocity_rolls_back(pkg, scenes):
    spec = scenes.random_boxes(300, seed=32, xz=2.0, y=(0.3, 4.0))
    w, ref = world(pkg, spec), world(pkg, spec)
    w.step(DT, steps=20)
    ref.step(DT, steps=20)
    good = w.read_bodies()
    bad = good.copy()
    bad[17, 3] = np.nan
    w.write_states(np.ascontiguousarray(bad))
    pre = w.read_bodies()
    assert np.isnan(pre[17, 3])
    with pytest.raises(OverflowError):
        w.step(DT)
    np.testing.assert_array_equal(w.read_bodies(), pre)
    # fixed: the run continues exactly as one that never saw the bad input
    w.write_states(np.ascontiguousarray(good))
    ref.write_states(np.ascontiguousarray(good))
    w.step(DT, steps=10)
    ref.step(DT, steps=10)
    np.testing.assert_array_equal(w.read_bodies(), ref.read_bodies())
    np.testing.assert_array_equal(w.pairs(0), ref.pairs(0))


def test_scan_wait_gives_up_then_recovers(pkg, scenes):
    spec = scenes.random_boxes(200, seed=33, xz=2.0, y=(0.3, 3.0))
    w, ref = world(pkg, spec), world(pkg, spec)
    w.step(DT, steps=5)
    ref.step(DT, steps=5)
    n = 3 * 2048 + 5                     # four tiles: tile 0 is never taken
    with pytest.raises(pkg.LogicError):
        w.test_scan(n, skip_first_tile=True)
    bits, bad = w.last_scan
    assert bits & K_ERR_LOGIC
    assert bad > 0
    assert w.test_scan(n) == (0, 0)
    w.step(DT, steps=5)
    ref.step(DT, steps=5)
    np.testing.assert_array_equal(w.read_bodies(), ref.read_bodies())
    assert w.error_bits() == 0
