"""Performance parameters (fyzz_b200_tuning_t) change how the step runs,
not what it computes: worlds stepped under different island size classes,
radix digit widths and block sizes stay bit-identical (bodies, pairs,
partition levels), and a world takes its class's line of the tuning table
when its device state is built."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DT = 1.0 / 120.0
SETTINGS = [
    {"island_thread": 8, "island_warp": 96, "island_cta": 512, "radix_bits": 8, "elem_block": 256, "work_queue": 0},
    {"island_thread": 0, "island_warp": 32, "island_cta": 128, "radix_bits": 11, "elem_block": 128, "work_queue": 1},
    {"island_thread": 4, "island_warp": 64, "island_cta": 256, "radix_bits": 9, "elem_block": 512, "work_queue": 1},
    {"island_thread": 8, "island_warp": 96, "island_cta": 512, "radix_bits": 10, "elem_block": 1024, "work_queue": 0},
]


def build(pkg, specs, tuning):
    w = pkg.World(0)
    for s in specs:
        w.add_scene(s)
    w.set_tuning(**tuning)
    return w


@pytest.mark.parametrize("kind", ["large_scene", "many_scenes"])
def test_settings_give_identical_steps(pkg, scenes, kind):
    if kind == "large_scene":
        # above 2,048 shapes: the device-wide radix sort of the endpoints
        specs = [scenes.mixed_scale(6000, seed=4, region=(18.0, 8.0, 18.0), joint_frac=0.02)]
    else:
        specs = scenes.batched_scenes(48, low=16, high=512, base_seed=5)
    worlds = [build(pkg, specs, t) for t in SETTINGS]
    for w, t in zip(worlds, SETTINGS):
        assert w.tuning() == t
    for w in worlds:
        w.step(DT, steps=40)
    ref = worlds[0]
    assert ref.counts()["managers"] > 100
    for w in worlds[1:]:
        np.testing.assert_array_equal(w.read_bodies(), ref.read_bodies())
        np.testing.assert_array_equal(w.pairs(0), ref.pairs(0))
        np.testing.assert_array_equal(w.levels(), ref.levels())


def test_invalid_settings_are_rejected(pkg, scenes):
    w = build(pkg, [scenes.random_boxes(20, seed=1)], SETTINGS[0])
    for bad in ({"radix_bits": 12}, {"island_warp": 16}, {"island_cta": 1024}, {"elem_block": 100},
                {"island_thread": 9}, {"work_queue": 2}):
        with pytest.raises(ValueError):
            w.set_tuning(**bad)
    assert w.tuning() == SETTINGS[0]


def test_world_reads_its_class_line(pkg, scenes, tmp_path):
    table = tmp_path / "tuning.txt"
    table.write_text("# test table\nlarge_scene 4 64 256 11 128 1\nmany_scenes 0 32 128 9 512 0\n")
    old = os.environ.get("FYZZ_B200_TUNING")
    os.environ["FYZZ_B200_TUNING"] = str(table)
    try:
        small = pkg.World(0)
        small.add_scene(scenes.random_boxes(50, seed=2))
        large = pkg.World(0)
        large.add_scene(scenes.random_boxes(3000, seed=2))
        assert small.tuning() == {"island_thread": 0, "island_warp": 32, "island_cta": 128, "radix_bits": 9,
                                  "elem_block": 512, "work_queue": 0}
        assert large.tuning() == {"island_thread": 4, "island_warp": 64, "island_cta": 256, "radix_bits": 11,
                                  "elem_block": 128, "work_queue": 1}
    finally:
        if old is None:
            del os.environ["FYZZ_B200_TUNING"]
        else:
            os.environ["FYZZ_B200_TUNING"] = old
