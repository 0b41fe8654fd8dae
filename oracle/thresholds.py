"""Force-threshold stream restated from scene outputs (test infrastructure:
the checker for the B200 threshold kernels, never part of the product).

Follows the reference's Scene::update_threshold_stream
(src/native/scene.cpp:9391-9508) after its force writeback (9293-9330) and
the dormant-manager rule of contact preparation (7804-7820):

* a touching manager counts only when one of its bodies is dynamic and
  awake (dormant managers are not solved and write zero impulses);
* its key is (dynamic body, world) against a static body, else the ordered
  body pair (kinematic bodies are rigid nodes with their own id), with the
  dynamic body's report threshold or the smaller of the two;
* a threshold of FLT_MAX disables the row; the row's impulse is the double
  sum of the manager's final per-contact normal impulses and zero sums are
  dropped;
* rows are grouped by key in key order (actor0, static world, actor1);
  within a key the impulses are added in manager order and the thresholds
  reduced by min; a key exceeds when impulse > threshold * dt (double);
* exceeded keys merge with the previous step's in key order: Found (this
  step's impulse and threshold), Persists (the previous step's impulse and
  threshold), Lost (zero impulse, previous threshold).

The reference sorts its rows with std::sort (not stable) before adding
equal keys; impulses of one key are then added in an unspecified order.
This restatement adds them in manager (shape-pair) order, which gives the
same double sum whenever the per-manager sums add exactly (they are sums of
a few floats), and is the order the B200 kernels use.
"""
from __future__ import annotations

import numpy as np

FOUND, PERSISTS, LOST = 0, 1, 2
FLT_MAX = float(np.finfo(np.float32).max)
STATIC, DYNAMIC, KINEMATIC = 0, 1, 2


class ThresholdBuilder:
    """Feeds on each step's touching managers and final point impulses."""

    def __init__(self, shape_body: np.ndarray, motion: np.ndarray):
        """shape_body: actor of each shape; motion: per actor STATIC,
        DYNAMIC or KINEMATIC."""
        self.shape_body = np.asarray(shape_body, np.int64)
        self.motion = np.asarray(motion, np.int64)
        self.prev = []          # [(key, impulse, threshold)] sorted by key

    def step(self, pairs, counts, impulses, sleeping, thresholds, seconds: float):
        """pairs (n, 2) shape pairs of the touching managers (in the order
        their impulses are to be added), counts (n,), impulses: per point in
        the same order; sleeping / thresholds per actor.  Returns (rows
        (m, 4) u32: actor0 actor1 static_world change, impulse (m,) f64,
        threshold (m,) f32)."""
        thr_all = np.asarray(thresholds, np.float32)
        rows = []
        off = 0
        for (sa, sb), c in zip(np.asarray(pairs, np.int64), np.asarray(counts, np.int64)):
            imp = impulses[off: off + int(c)]
            off += int(c)
            b0, b1 = int(self.shape_body[sa]), int(self.shape_body[sb])
            a, b = min(b0, b1), max(b0, b1)
            dyn_a, dyn_b = self.motion[a] == DYNAMIC, self.motion[b] == DYNAMIC
            if not dyn_a and not dyn_b:
                continue
            if not ((dyn_a and not sleeping[a]) or (dyn_b and not sleeping[b])):
                continue                      # dormant: not solved, zero impulses
            world = self.motion[a] == STATIC or self.motion[b] == STATIC
            if world:
                key = ((a if dyn_a else b), 1, 0)
                thr = np.float32(thr_all[key[0]])
            else:
                key = (a, 0, b)
                ta, tb = thr_all[a], thr_all[b]
                thr = np.float32(tb if tb < ta else ta)
            if float(thr) == FLT_MAX:
                continue
            total = 0.0
            for x in imp:
                total += float(x)
            if not np.isfinite(total):
                raise OverflowError("threshold stream: non-finite impulse sum")
            if total == 0.0:
                continue
            rows.append((key, total, thr))
        rows.sort(key=lambda r: r[0])        # stable: manager order within a key
        cur = []
        for key, total, thr in rows:
            if cur and cur[-1][0] == key:
                k, s, t = cur[-1]
                cur[-1] = (k, s + total, thr if thr < t else t)
            else:
                cur.append((key, total, thr))
        dt = float(np.float32(seconds))
        cur = [r for r in cur if r[1] > float(r[2]) * dt]
        out, imp, thr = [], [], []
        i = j = 0
        while i < len(self.prev) or j < len(cur):
            if i < len(self.prev) and (j >= len(cur) or self.prev[i][0] < cur[j][0]):
                k, _, t = self.prev[i]
                out.append((k[0], k[2], k[1], LOST)); imp.append(0.0); thr.append(t)
                i += 1
            elif j < len(cur) and (i >= len(self.prev) or cur[j][0] < self.prev[i][0]):
                k, s, t = cur[j]
                out.append((k[0], k[2], k[1], FOUND)); imp.append(s); thr.append(t)
                j += 1
            else:
                k, s, t = self.prev[i]
                out.append((k[0], k[2], k[1], PERSISTS)); imp.append(s); thr.append(t)
                i += 1
                j += 1
        self.prev = cur
        return (np.array(out, np.uint32).reshape(-1, 4), np.array(imp, np.float64),
                np.array(thr, np.float32))
