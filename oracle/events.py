"""Contact-event publication restated from scene outputs (test
infrastructure: the checker for the B200 event kernels, never part of the
product).

Follows the reference's Scene::update_contacts touch transitions
(src/native/scene.cpp:4655-4700: a pair starts touching when its manifold
has contacts and had none the previous step; it stops touching when a
previously touching pair has no contacts or left the broadphase) and
Scene::publish_contact_events (scene.cpp:9149-9264): every touching manager
in pair order reports Found (new touch) or Persists, lost touches are
merged in pair order with no points, points carry the manifold point with
its normal flipped when the manager's solver orientation
(gu_order_reversed, scene.cpp:3276-3287) disagrees with body order, event
bodies are ordered body0 < body1, and impulses are the solver's final
per-point normal impulses summed in double precision.  Sleeping is not
modelled: every touching manager has an active dynamic body.
"""
from __future__ import annotations

import numpy as np

FOUND, PERSISTS, LOST = 0, 1, 2


class EventBuilder:
    """Feeds on (manifolds, impulses) after each step of one scene."""

    def __init__(self, shape_body: np.ndarray, body_dynamic: np.ndarray):
        self.shape_body = np.asarray(shape_body, np.int64)
        self.body_dynamic = np.asarray(body_dynamic, bool)
        self.prev = set()

    def _reversed(self, a: int, b: int) -> bool:
        ba, bb = self.shape_body[a], self.shape_body[b]
        da, db = self.body_dynamic[ba], self.body_dynamic[bb]
        return (not da) or (da and db and ba < bb)

    def step(self, pairs, counts, pts, impulses):
        """pairs (n,2), counts (n,), pts (n,4,7) of the touching managers in
        pair order; impulses: per point, in the same order.  Returns
        (events (m,7) u32: body0 body1 kind count offset shape0 shape1,
        event impulses (m,) f64, points (p,7) f32, point impulses (p,) f64)."""
        cur = [(int(a), int(b)) for a, b in pairs]
        cur_set = set(cur)
        lost = sorted(self.prev - cur_set)
        events, ev_imp, points, pt_imp = [], [], [], []
        off = np.concatenate([[0], np.cumsum(counts)]).astype(np.int64)
        li = 0

        def event(pair, kind, count, offset, imp):
            a, b = pair
            ba, bb = int(self.shape_body[a]), int(self.shape_body[b])
            rev = ba > bb
            events.append((bb if rev else ba, ba if rev else bb, kind, count, offset,
                           b if rev else a, a if rev else b))
            ev_imp.append(imp)

        for m, pair in enumerate(cur):
            while li < len(lost) and lost[li] < pair:
                event(lost[li], LOST, 0, len(points), 0.0)
                li += 1
            kind = PERSISTS if pair in self.prev else FOUND
            a, b = pair
            flip = self._reversed(a, b) != (self.shape_body[a] > self.shape_body[b])
            offset = len(points)
            total = 0.0
            for j in range(int(counts[m])):
                p = pts[m, j].astype(np.float32).copy()
                if flip:
                    p[3:6] = -p[3:6]
                imp = float(impulses[off[m] + j])
                total += imp
                points.append(p)
                pt_imp.append(imp)
            event(pair, kind, int(counts[m]), offset, total)
        for pair in lost[li:]:
            event(pair, LOST, 0, len(points), 0.0)
        self.prev = cur_set
        return (np.array(events, np.uint32).reshape(-1, 7), np.array(ev_imp, np.float64),
                np.array(points, np.float32).reshape(-1, 7), np.array(pt_imp, np.float64))
