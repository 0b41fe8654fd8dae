"""Allocation-free sweep-and-prune (fyzz_b200_sap_pairs_static_scratch)
against the world's broadphase, through the C ABI.

The entry point keeps its working set in one fixed device array instead of
allocated buffers.  On the same encoded bounds its pair list must equal the
world's current pair list (fyzz_b200_read_pairs, which = 0) bit for bit
(integer work: exact), on consecutive calls that reuse the array.  Device
buffers for inputs and outputs are the caller's (allocated here by torch).
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DT = 1.0 / 120.0
MAX_SHAPES = 8192
DYNAMIC = np.uint32(1 << 31)


def static_pairs(pkg, bounds, body_flags, cap=None):
    import torch
    dev = torch.device("cuda:0")
    n = int(bounds.shape[0])
    cap = max(1, 64 * n) if cap is None else cap
    b = torch.from_numpy(np.ascontiguousarray(bounds, np.uint32).reshape(-1).view(np.int32)).to(dev)
    f = torch.from_numpy(np.ascontiguousarray(body_flags, np.uint32).view(np.int32)).to(dev)
    p = torch.full((2 * cap,), -1, dtype=torch.int32, device=dev)
    c = torch.full((1,), -1, dtype=torch.int32, device=dev)
    torch.cuda.synchronize()
    msg = C.create_string_buffer(256)
    rc = pkg.lib().fyzz_b200_sap_pairs_static_scratch(
        b.data_ptr() if n else None, f.data_ptr() if n else None, n, p.data_ptr(), cap,
        c.data_ptr(), None, msg, len(msg))
    assert rc == 0, msg.value
    torch.cuda.synchronize()
    total = int(c.cpu().numpy().view(np.uint32)[0])
    got = p.cpu().numpy().view(np.uint32).reshape(-1, 2)[: min(total, cap)]
    return total, got


def world_of(pkg, spec):
    spec.floor = None          # finite shapes only: shape id == row of the bounds
    w = pkg.World(0)
    w.add_scene(spec)
    return w


def test_two_calls_match_world_pairs(pkg, scenes):
    spec = scenes.mixed_scale(2500, seed=21, region=(14.0, 6.0, 14.0), joint_frac=0.0)
    w = world_of(pkg, spec)
    flags = spec.shape_body.astype(np.uint32) | DYNAMIC
    w.collide()
    want1 = w.pairs(0)
    total1, got1 = static_pairs(pkg, w.encoded_bounds(), flags)
    assert total1 == len(want1) > 0
    np.testing.assert_array_equal(got1, want1)
    # second call in a row, on the bounds of a later step of the same scene
    w.step(DT, steps=40)
    want2 = w.pairs(0)
    total2, got2 = static_pairs(pkg, w.encoded_bounds(), flags)
    assert total2 == len(want2) > 0
    np.testing.assert_array_equal(got2, want2)


def test_largest_scene_and_static_filter(pkg, scenes):
    spec = scenes.random_boxes(MAX_SHAPES, seed=22, xz=7.0, y=(0.3, 14.0))
    w = world_of(pkg, spec)
    w.collide()
    want = w.pairs(0)
    bounds = w.encoded_bounds()
    assert bounds.shape[0] == MAX_SHAPES
    body = spec.shape_body.astype(np.uint32)
    total, got = static_pairs(pkg, bounds, body | DYNAMIC)
    assert total == len(want) > 0
    np.testing.assert_array_equal(got, want)
    # every third body static: pairs of two static bodies drop out
    dyn = (body % 3) != 0
    total_s, got_s = static_pairs(pkg, bounds, np.where(dyn, body | DYNAMIC, body))
    keep = dyn[body[want[:, 0]]] | dyn[body[want[:, 1]]]
    assert total_s == int(keep.sum()) < len(want)
    np.testing.assert_array_equal(got_s, want[keep])


def test_capacity_and_empty(pkg, scenes):
    spec = scenes.random_boxes(600, seed=23, xz=2.0, y=(0.3, 4.0))
    w = world_of(pkg, spec)
    w.collide()
    want = w.pairs(0)
    flags = spec.shape_body.astype(np.uint32) | DYNAMIC
    cap = len(want) // 3
    total, got = static_pairs(pkg, w.encoded_bounds(), flags, cap=cap)
    assert total == len(want)             # the full total, list truncated
    # only whole owner buckets that fit are written: a prefix of the full
    # list ending at a bucket boundary, the rest of the buffer untouched
    written = got[:, 0] != 0xFFFFFFFF
    k = int(written.sum())
    assert 0 < k <= cap and np.all(written[:k])
    np.testing.assert_array_equal(got[:k], want[:k])
    assert want[k, 0] != want[k - 1, 0]
    assert np.all(got[k:] == 0xFFFFFFFF)
    total0, got0 = static_pairs(pkg, np.zeros((0, 6), np.uint32), np.zeros(0, np.uint32))
    assert total0 == 0 and got0.shape[0] == 0


def test_oversize_rejected_before_launch(pkg):
    import torch
    c = torch.full((1,), -1, dtype=torch.int32, device="cuda:0")
    msg = C.create_string_buffer(256)
    # pointers are never dereferenced: the size check comes first
    rc = pkg.lib().fyzz_b200_sap_pairs_static_scratch(
        c.data_ptr(), c.data_ptr(), MAX_SHAPES + 1, c.data_ptr(), 1, c.data_ptr(), None, msg,
        len(msg))
    assert rc == 1
    assert b"FYZZ_B200_STATIC_SAP_MAX_SHAPES" in msg.value
    torch.cuda.synchronize()
    assert int(c.cpu()[0]) == -1
