"""Generates the committed golden fixtures from the reference itself.

Runs the reference SDK's NativeCpu scene (oracle/_ref/libfyzz_ref.so, built
from the reference sources by oracle/Makefile) on small seeded scenes and
stores its outputs:

  golden_gu.npz     box/box PCM candidates, batch selection and GJK/EPA
                    witnesses for seeded random box pairs
                    (src/native/GuPCMContactBoxBox.cpp, GuPCMGjkEpa.cpp)
  golden_<scene>.npz for each scene: mass properties, encoded bounds, pair
                    set and manifolds after advance_collision, and for
                    N steps the body states, found/lost pairs and the Dy
                    descriptor input order the reference used
                    (src/native/scene.cpp)

Usage:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import importlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import refscene  # noqa: E402

scenes = importlib.import_module("fyzzxyzzy-sdk_b200.scenes")

STEPS = 12
DT = 1.0 / 120.0


def golden_scenes():
    return {
        "boxes": scenes.random_boxes(120, seed=3, xz=2.0, y=(0.3, 4.0)),
        "mixed": scenes.mixed_scale(160, seed=2, region=(5.0, 3.0, 5.0), joint_frac=0.05),
        "stack": scenes.box_stack_scene(24, seed=7),
    }


def gu_vectors(n=400, seed=11):
    rng = np.random.default_rng(seed)
    recs_a, recs_b, ok, counts, cands, sel, gjk_ok, gjk = [], [], [], [], [], [], [], []
    for _ in range(n):
        def rec():
            h = rng.uniform(0.1, 0.5, 3)
            p = rng.uniform(-0.5, 0.5, 3)
            q = rng.standard_normal(4)
            q /= np.linalg.norm(q)
            return np.concatenate([h, p, q]).astype(np.float32)
        a, b = rec(), rec()
        o, c = refscene.pcm_box_box_candidates(a, b, 0.04)
        pad = np.zeros((64, 10), np.float32)
        pad[: c.shape[0]] = c
        s = refscene.pcm_batch_selection(c) if c.shape[0] > 4 else np.zeros(4, np.uint8)
        g_ok, g = refscene.pcm_box_box_gjk_epa(a, b, 0.04) if (o and c.shape[0] == 0) else (False, np.zeros(10, np.float32))
        recs_a.append(a); recs_b.append(b); ok.append(o); counts.append(c.shape[0])
        cands.append(pad); sel.append(s); gjk_ok.append(g_ok); gjk.append(g)
    np.savez_compressed(os.path.join(HERE, "golden_gu.npz"), a=np.stack(recs_a), b=np.stack(recs_b),
                        ok=np.array(ok), counts=np.array(counts, np.int32), cands=np.stack(cands),
                        sel=np.stack(sel), gjk_ok=np.array(gjk_ok), gjk=np.stack(gjk))


def scene_fixture(name, spec):
    r = refscene.RefScene(spec)
    out = {"mass": r.mass_props()}
    r.advance_collision()
    out["bounds"] = r.encoded_bounds()
    out["pairs"] = r.pairs()
    mp, mc, mr, mpts = r.manifolds()
    out.update(man_pairs=mp, man_counts=mc, man_rev=mr, man_pts=mpts)
    v, i, m = r.endpoints(0)
    out["minx_vals"], out["minx_ids"] = v[m == 0], i[m == 0]
    # stepping from a fresh scene (advance_collision above is a query only on
    # another scene instance)
    r2 = refscene.RefScene(spec)
    states, orders, jorders, found, lost = [], [], [], [], []
    for _ in range(STEPS):
        r2.step(DT)
        states.append(r2.body_states())
        orders.append(r2.manager_order())
        jorders.append(r2.joint_order())
        found.append(r2.pairs(1))
        lost.append(r2.pairs(2))
    out["states"] = np.stack(states)
    for k in range(STEPS):
        out[f"order_{k}"] = orders[k]
        out[f"jorder_{k}"] = jorders[k]
        out[f"found_{k}"] = found[k]
        out[f"lost_{k}"] = lost[k]
    np.savez_compressed(os.path.join(HERE, f"golden_{name}.npz"), **out)


def main():
    gu_vectors()
    for name, spec in golden_scenes().items():
        scene_fixture(name, spec)
    print("wrote", sorted(f for f in os.listdir(HERE) if f.endswith(".npz")))


if __name__ == "__main__":
    main()
