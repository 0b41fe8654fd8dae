"""The z-band rule of the large-scene sweep, restated on the host.

The device sweeps a large scene per band of z: a shape enters every band
its encoded z extent touches (bands at least as wide as the widest
extent, so one or two), the band entries keep the x order, and a pair
found in a band is kept only in the band of the larger of the two min z.
Because the band index is monotone in the encoded bound, that band holds
both shapes, so every overlapping pair is reported exactly once.  These
tests check that invariant on random encoded bounds (float32 arithmetic as
on the device), against all-pairs overlap: narrow and wide shapes, a
single shape as wide as the scene, and bands at the 1/250 floor.
"""
import numpy as np

BANDS = 256


def encode(v):
    """Order-preserving float32 -> uint32 encoding, quantised down (min) or
    up (max) to 16 ulps as the endpoint encoding does."""
    bits = np.asarray(v, np.float32).view(np.uint32).astype(np.uint64)
    enc = np.where(bits & 0x80000000, (~bits) & 0xFFFFFFFF, bits | 0x80000000)
    return enc.astype(np.uint64)


def enc_min(v):
    return (((encode(v) >> 4) - 1) << 4) & 0xFFFFFFFF


def enc_max(v):
    return ((((encode(v) >> 4) + 1) << 4) | 4) & 0xFFFFFFFF


def decode(e):
    e = np.asarray(e, np.uint64)
    bits = np.where(e & 0x80000000, e & 0x7FFFFFFF, (~e) & 0xFFFFFFFF).astype(np.uint32)
    return bits.view(np.float32)


def band_params(zlo, zhi):
    ext = np.max(decode(zhi) - decode(zlo)).astype(np.float32)
    z0, z1 = decode(np.min(zlo)), decode(np.max(zhi))
    width = np.float32(ext * np.float32(1.001))
    floor_w = np.float32((z1 - z0) / np.float32(250.0))
    width = max(width, floor_w)
    return np.float32(z0), np.float32(np.float32(1.0) / width)


def band_of(e, z0, inv):
    t = (decode(e) - z0).astype(np.float32) * inv
    t = np.asarray(t, np.float32)
    b = np.where(t > 0, np.minimum(np.floor(t), BANDS - 1), 0)
    return b.astype(np.int64)


def band_pairs(lo, hi):
    """Pairs (i < j) the band rule reports, with multiplicity."""
    z0, inv = band_params(lo[:, 2], hi[:, 2])
    b0, b1 = band_of(lo[:, 2], z0, inv), band_of(hi[:, 2], z0, inv)
    assert np.all(b1 - b0 <= 1), "a shape spans more than two bands"
    out = []
    for band in np.unique(np.concatenate([b0, b1])):
        members = np.nonzero((b0 <= band) & (b1 >= band))[0]
        for ii, i in enumerate(members):
            for j in members[ii + 1:]:
                if np.all(lo[i] <= hi[j]) and np.all(lo[j] <= hi[i]):
                    if band_of(max(lo[i, 2], lo[j, 2]), z0, inv) == band:
                        out.append((min(i, j), max(i, j)))
    return out


def all_pairs(lo, hi):
    n = lo.shape[0]
    ov = np.all(lo[:, None, :] <= hi[None, :, :], axis=2) & np.all(lo[None, :, :] <= hi[:, None, :], axis=2)
    i, j = np.nonzero(np.triu(ov, 1))
    return set(zip(i.tolist(), j.tolist()))


def bounds(rng, n, region, half):
    c = rng.uniform(-0.5, 0.5, (n, 3)) * np.asarray(region)
    h = rng.uniform(half[0], half[1], (n, 3))
    lo = np.stack([enc_min(np.float32(c[:, k] - h[:, k])) for k in range(3)], 1)
    hi = np.stack([enc_max(np.float32(c[:, k] + h[:, k])) for k in range(3)], 1)
    return lo, hi


def check(lo, hi):
    got = band_pairs(lo, hi)
    assert len(got) == len(set(got)), "a pair was reported in two bands"
    assert set(got) == all_pairs(lo, hi)


def test_band_rule_narrow_shapes():
    rng = np.random.default_rng(1)
    lo, hi = bounds(rng, 400, (20.0, 2.0, 20.0), (0.05, 0.6))
    check(lo, hi)


def test_band_rule_one_shape_across_the_scene():
    rng = np.random.default_rng(2)
    lo, hi = bounds(rng, 300, (10.0, 2.0, 30.0), (0.05, 0.5))
    lo[0, 2] = enc_min(np.float32(-15.0))
    hi[0, 2] = enc_max(np.float32(15.0))
    check(lo, hi)


def test_band_rule_bands_at_the_range_floor():
    rng = np.random.default_rng(3)
    lo, hi = bounds(rng, 500, (3.0, 2.0, 600.0), (0.05, 0.3))
    check(lo, hi)


def test_band_rule_negative_and_straddling_z():
    rng = np.random.default_rng(4)
    lo, hi = bounds(rng, 300, (4.0, 1.0, 4.0), (0.01, 0.4))
    check(lo, hi)
