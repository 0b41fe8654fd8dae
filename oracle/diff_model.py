"""FP64 reference for the B200 step adjoint (test infrastructure: the checker
of fyzz_b200_rollout_backward, never part of the product).

An independent restatement, in torch float64 with autograd, of the
differentiable model the adjoint kernels implement: the rigid-body step
(pre-integration, sqrt-inverse-inertia tensor, contact / friction / joint
rows -- centre and anchored distance, fixed, spherical, revolute and
prismatic joints, their rows orthogonalised in the inverse-mass metric --,
4 + 1 Gauss-Seidel passes in partition order, integration; reference
src/native/scene.cpp:114-143, 7490-8510, 7615-7767, 8853-9148,
10383-10707) with its
discrete structure frozen from a recorded forward run of the B200 world:
touching managers and their contact points, friction anchors (carried ones
body-local, ones taken from the step's own contact points at those points),
partition levels.  Contact points move rigidly with their bodies, as the
persistent PCM manifold keeps them: point j is the material point of
shape1's body B (fixed in the world when B is static) that coincided with
the recorded point at the step's start, the normal turns with B, and the
separation changes by n0 . (Pa - Pb) with Pa the coinciding material point
of shape0's body A.  Branch
decisions (separated / closing / bouncing, PGS clamps) are taken from this
model's own values.

Gradients come from torch.autograd, so nothing here shares code with the
hand-written adjoint it checks.
"""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

GRAVITY = -9.81
FLT_MAX = 3.4028234663852886e38


def _t(x):
    return torch.as_tensor(np.asarray(x, np.float64), dtype=torch.float64)


def _f(x) -> float:
    """Value of a scalar tensor for a branch decision."""
    return float(x.detach()) if isinstance(x, torch.Tensor) else float(x)


def cross(a, b):
    return torch.stack([a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]])


def rot(q, v):
    u = q[:3]
    t = 2.0 * cross(u, v)
    return v + q[3] * t + cross(u, t)


def conj(q):
    return torch.stack([-q[0], -q[1], -q[2], q[3]])


def rotinv(q, v):
    return rot(conj(q), v)


def qmul(a, b):
    return torch.stack([a[3] * b[0] + b[3] * a[0] + a[1] * b[2] - a[2] * b[1],
                        a[3] * b[1] + b[3] * a[1] + a[2] * b[0] - a[0] * b[2],
                        a[3] * b[2] + b[3] * a[2] + a[0] * b[1] - a[1] * b[0],
                        a[3] * b[3] - a[0] * b[0] - a[1] * b[1] - a[2] * b[2]])


def integrate_q(pose, w, dt):
    m2 = (w * w).sum()
    if _f(m2) == 0.0:
        return pose
    m = torch.sqrt(m2)
    half = dt * m * 0.5
    sn = torch.sin(half) / m
    dq = qmul(torch.cat([w * sn, torch.zeros(1, dtype=torch.float64)]), pose)
    nx = dq + pose * torch.cos(half)
    return nx / torch.sqrt((nx * nx).sum())


@dataclass
class StepRecord:
    """Frozen structure of one recorded step."""
    frames_c: np.ndarray      # (nb, 3) mass-frame centres at the step's start
    frames_q: np.ndarray      # (nb, 4)
    pairs: np.ndarray         # (m, 2) touching managers, pair order
    counts: np.ndarray        # (m,)
    pts: np.ndarray           # (m, 4, 7) point, normal, separation
    anchors: np.ndarray       # (m,) anchor word (count | fresh bits << 10 | sources << 12)
    a0: np.ndarray            # (m, 2, 3)
    a1: np.ndarray            # (m, 2, 3)
    levels: np.ndarray        # (joints + m,) partition of every descriptor


def record(world, steps: int, dt: float):
    """Steps a B200 world one step at a time and records each step's
    structure (the world must match the one being differentiated)."""
    recs = []
    for _ in range(steps):
        c, q = world.read_mass_frames()
        world.step(dt)
        pairs, counts, pts = world.manifolds()
        cnt, a0, a1 = world.friction_anchors()
        recs.append(StepRecord(c, q, pairs, counts, pts, cnt, a0, a1, world.levels()))
    return recs


class Model:
    """The differentiable step over recorded structure.

    bodies: per world body, dynamic flag, inverse mass, inverse principal
    inertia, mass-frame offset u of the body origin (for joint anchors),
    damping; shapes: owning body, restitution, rest offset; joints: in the
    step's canonical order, (a, b, rest length) for a centre distance joint
    or (a, b, rest length, kind, local frame a (7), local frame b (7)) for
    the other kinds (kind numbers of scenes.JOINT_*)."""

    def __init__(self, dynamic, inv_mass, inv_inertia, origin_offset, shape_body, restitution,
                 rest_offset, joints, lin_damp=0.0, ang_damp=0.05, mass_local_q=None):
        self.dyn = np.asarray(dynamic, bool)
        # per body, the mass frame's orientation in the body frame (body
        # orientation = mass-frame orientation * conj(mass_local_q))
        self.mlq = (np.tile([0.0, 0.0, 0.0, 1.0], (len(self.dyn), 1)) if mass_local_q is None
                    else np.asarray(mass_local_q, np.float64))
        self.im0 = np.asarray(inv_mass, np.float64)
        self.iI0 = np.asarray(inv_inertia, np.float64)
        self.u = np.asarray(origin_offset, np.float64)
        self.shape_body = np.asarray(shape_body, np.int64)
        self.rest = np.asarray(restitution, np.float64)
        self.rest_off = np.asarray(rest_offset, np.float64)
        self.joints = list(joints)
        self.lin_damp, self.ang_damp = lin_damp, ang_damp

    def rollout(self, recs, dt, c0, q0, v0, w0, mass, mu_s, mu_d):
        """Runs the recorded steps from (c0, q0, v0, w0) with masses and
        per-shape friction as tensors; returns the final (c, q, v, w) lists."""
        nb = len(self.dyn)
        c = [c0[i] for i in range(nb)]
        q = [q0[i] for i in range(nb)]
        v = [v0[i] for i in range(nb)]
        w = [w0[i] for i in range(nb)]
        m0 = np.where(self.im0 > 0, 1.0 / np.where(self.im0 > 0, self.im0, 1.0), 0.0)
        im, iI = [], []
        for i in range(nb):
            if self.dyn[i]:
                scale = _t(m0[i]) / mass[i]
                im.append(_t(self.im0[i]) * scale)
                iI.append(_t(self.iI0[i]) * scale)
            else:
                im.append(_t(0.0))
                iI.append(_t([0.0, 0.0, 0.0]))
        for rec in recs:
            c, q, v, w = self.step(rec, dt, c, q, v, w, im, iI, mu_s, mu_d)
        return c, q, v, w

    def step(self, rec, dt, c, q, v, w, im, iI, mu_s, mu_d):
        nb = len(self.dyn)
        zero3 = _t([0.0, 0.0, 0.0])
        lm = max(1.0 - self.lin_damp * dt, 0.0)
        am = max(1.0 - self.ang_damp * dt, 0.0)
        v1, w1, C = [], [], []
        for i in range(nb):
            if not self.dyn[i]:
                v1.append(zero3); w1.append(zero3); C.append(torch.zeros(3, 3, dtype=torch.float64))
                continue
            v1.append(lm * (v[i] + _t([0.0, GRAVITY * dt, 0.0])))
            w1.append(am * w[i])
            l = torch.sqrt(iI[i])
            cols = [rot(q[i], _t(e)) for e in ([1, 0, 0], [0, 1, 0], [0, 0, 1])]
            C.append(sum(l[k] * torch.outer(cols[k], cols[k]) for k in range(3)))
        # ---- rows
        nj = len(self.joints)
        desc = []
        for jt in self.joints:
            a, b, length = jt[0], jt[1], jt[2]
            if len(jt) == 3 or jt[3] == 0:
                row = self._joint_row(a, b, length, c, q, v1, w1, C, im, dt)
                desc.append(("joint", row[0], row[1], [row[2:]]))
            else:
                desc.append(("joint",) + self._frame_joint_rows(a, b, length, jt[3], jt[4], jt[5], c, q, v1, w1,
                                                                C, im, dt))
        for k in range(len(rec.pairs)):
            desc.append(("contact",) + self._contact_rows(rec, k, c, q, v1, w1, C, im, mu_s, mu_d, dt))
        # ---- Gauss-Seidel in partition order, islands independent
        order = self._order(rec, nj)
        dv = [zero3] * nb
        dw = [zero3] * nb
        applied = [None] * len(desc)
        for d, item in enumerate(desc):
            applied[d] = [_t(0.0)] * (len(item[3]) if item[0] == "joint" else 8)
        pos, passes = 4, 5
        dvm = dwm = None
        for it in range(passes):
            for d in order:
                self._solve(desc[d], applied[d], dv, dw, it, pos)
            if it + 1 == pos:
                dvm, dwm = list(dv), list(dw)
        # ---- integration
        nc, nq, nv, nw = [], [], [], []
        for i in range(nb):
            if not self.dyn[i]:
                nc.append(c[i]); nq.append(q[i]); nv.append(v[i]); nw.append(w[i])
                continue
            nc.append(c[i] + (v1[i] + dvm[i]) * dt)
            nq.append(integrate_q(q[i], w1[i] + C[i] @ dwm[i], dt))
            nv.append(v1[i] + dv[i])
            nw.append(w1[i] + C[i] @ dw[i])
        return nc, nq, nv, nw

    def _order(self, rec, nj):
        """Descriptors island by island, partitions ascending."""
        bodies = []
        for jt in self.joints:
            a, b = jt[0], jt[1]
            bodies.append((a if self.dyn[a] else -1, b if self.dyn[b] else -1))
        for (sa, sb) in rec.pairs:
            ba, bb = self.shape_body[sa], self.shape_body[sb]
            bodies.append((ba if self.dyn[ba] else -1, bb if self.dyn[bb] else -1))
        parent = list(range(len(self.dyn)))

        def find(x):
            while parent[x] != x:
                parent[x] = parent[parent[x]]
                x = parent[x]
            return x
        for a, b in bodies:
            if a >= 0 and b >= 0:
                ra, rb = find(a), find(b)
                if ra != rb:
                    parent[max(ra, rb)] = min(ra, rb)
        key = [(find(a if a >= 0 else b), int(rec.levels[d]), d) for d, (a, b) in enumerate(bodies)]
        return [d for _, _, d in sorted(key)]

    def _joint_row(self, a, b, length, c, q, v1, w1, C, im, dt):
        da, db = self.dyn[a], self.dyn[b]
        ra = -rot(q[a], _t(self.u[a]))
        rb = -rot(q[b], _t(self.u[b]))
        off = (c[a] + ra) - (c[b] + rb)
        dist = torch.sqrt((off * off).sum())
        axis = off / dist if _f(dist) >= 1.192092896e-07 else _t([1.0, 0.0, 0.0])
        an0, an1 = cross(ra, axis), cross(rb, axis)
        ja = C[a] @ an0 if da else _t([0.0, 0.0, 0.0])
        jb = C[b] @ an1 if db else _t([0.0, 0.0, 0.0])
        response = im[a] + im[b] + (ja * ja).sum() + (jb * jb).sum()
        rcp = 1.0 / response
        speed = (axis * (v1[a] - v1[b])).sum() + (an0 * w1[a]).sum() - (an1 * w1[b]).sum()
        err = dist - length
        return (a if da else -1, b if db else -1, axis, ja, jb, im[a], im[b], -rcp,
                -rcp * (err / dt + speed), -rcp * speed)

    def _frame_joint_rows(self, a, b, length, kind, la, lb, c, q, v1, w1, C, im, dt):
        """Rows of an anchored distance, fixed, spherical, revolute or
        prismatic joint (scene.cpp:7615-7767): anchors and frames from the
        bodies' poses, translation locked along frame A's axes (prismatic:
        not X), rotation through the relative quaternion's vector part
        (spherical: none; revolute: not X), each row orthogonalised against
        the earlier ones in the inverse-mass metric."""
        da, db = self.dyn[a], self.dyn[b]
        zero3 = _t([0.0, 0.0, 0.0])
        qa0 = qmul(q[a], conj(_t(self.mlq[a])))
        qb0 = qmul(q[b], conj(_t(self.mlq[b])))
        pa0 = c[a] - rot(q[a], _t(self.u[a]))
        pb0 = c[b] - rot(q[b], _t(self.u[b]))
        la, lb = np.asarray(la, np.float64), np.asarray(lb, np.float64)
        world0 = pa0 + rot(qa0, _t(la[:3]))
        world1 = pb0 + rot(qb0, _t(lb[:3]))
        ra, rb = world0 - c[a], world1 - c[b]
        m0 = im[a] if da else _t(0.0)
        m1 = im[b] if db else _t(0.0)
        rel = v1[a] - v1[b]
        wa, wb = w1[a], w1[b]
        rows = []

        def emit(axis, a0, a1, ja, jb, error, response):
            rcp = 1.0 / response
            speed = (axis * rel).sum() + (a0 * wa).sum() - (a1 * wb).sum()
            rows.append((axis, ja, jb, m0, m1, -rcp, -rcp * (error / dt + speed), -rcp * speed))

        if kind == 1:   # anchored distance: one row along the anchors' separation
            off = world0 - world1
            dist = torch.sqrt((off * off).sum())
            axis = off / dist if _f(dist) >= 1.192092896e-07 else _t([1.0, 0.0, 0.0])
            an0, an1 = cross(ra, axis), cross(rb, axis)
            ja = C[a] @ an0 if da else zero3
            jb = C[b] @ an1 if db else zero3
            emit(axis, an0, an1, ja, jb, dist - length, m0 + m1 + (ja * ja).sum() + (jb * jb).sum())
            return (a if da else -1, b if db else -1, rows)
        qa = qmul(qa0, _t(la[3:7]))
        error_p = rotinv(qa, world0 - world1)
        ea = va = vb = cc = zero3
        dd = overlap = _t(0.0)
        if kind != 3:   # not spherical
            qb = qmul(qb0, _t(lb[3:7]))
            if _f((qa * qb).sum()) < 0.0:
                qb = -qb
            eq = qmul(conj(qa), qb)
            ea, va, vb = eq[:3], qa[:3], qb[:3]
            dd = qa[3] * qb[3] - (va * vb).sum()
            overlap = qa[3] * qb[3] + (va * vb).sum()
            cc = qa[3] * vb + qb[3] * va
        errors = [error_p[0], error_p[1], error_p[2], -ea[0], -ea[1], -ea[2]]
        diag = [torch.stack([dd, cc[2], -cc[1]]), torch.stack([-cc[2], dd, cc[0]]), torch.stack([cc[1], -cc[0], dd])]
        count = {2: 6, 3: 3, 4: 5, 5: 5}[kind]
        done = []   # (lin, a0, a1, ja, jb, err, inv) of the rows so far
        for k in range(count):
            comp = k + (1 if kind == 5 else 0) + (1 if kind == 4 and k >= 3 else 0)
            err = errors[comp]
            if comp < 3:
                basis = _t([1.0 if comp == i else 0.0 for i in range(3)])
                lin = rot(qa, basis)
                arm = (world1 - c[a]) if kind == 5 else ra
                a0, a1 = cross(arm, lin), cross(rb, lin)
            else:
                qq = comp - 3
                lin = zero3
                a0 = 0.5 * (va * vb[qq] + vb * va[qq] + diag[qq])
                if _f(overlap) == 0.0:
                    # the relative quaternion's Jacobian is singular at 180 degrees
                    a0 = a0 + _t([1.0 if qq == i else 0.0 for i in range(3)]) * 1.1920928955078125e-07
                a1 = a0
            ja = C[a] @ a0 if da else zero3
            jb = C[b] @ a1 if db else zero3
            for (flin, fa0, fa1, fja, fjb, ferr, finv) in done:
                t = ((m0 + m1) * (lin * flin).sum() + (ja * fja).sum() + (jb * fjb).sum()) * finv
                lin, a0, a1 = lin - flin * t, a0 - fa0 * t, a1 - fa1 * t
                ja, jb = ja - fja * t, jb - fjb * t
                err = err - ferr * t
            response = (m0 + m1) * (lin * lin).sum() + (ja * ja).sum() + (jb * jb).sum()
            inv = 1.0 / response if _f(response) > 0.0 else _t(0.0)
            done.append((lin, a0, a1, ja, jb, err, inv))
            emit(lin, a0, a1, ja, jb, err, response)
        return (a if da else -1, b if db else -1, rows)

    def _contact_rows(self, rec, k, c, q, v1, w1, C, im, mu_s, mu_d, dt):
        sa, sb = (int(x) for x in rec.pairs[k])
        ba, bb = self.shape_body[sa], self.shape_body[sb]
        da, db = self.dyn[ba], self.dyn[bb]
        reversed_ = (not da) or (da and db and ba < bb)
        sh0, sh1 = (sb, sa) if reversed_ else (sa, sb)
        A, B = self.shape_body[sh0], self.shape_body[sh1]
        Bdyn = bool(self.dyn[B])
        cnt = int(rec.counts[k])
        P0 = rec.pts[k, :cnt, 0:3].astype(np.float64)
        n0 = _t(rec.pts[k, 0, 3:6])
        s0 = rec.pts[k, :cnt, 6].astype(np.float64)
        cA0, qA0 = _t(rec.frames_c[A]), _t(rec.frames_q[A])
        cB0, qB0 = _t(rec.frames_c[B]), _t(rec.frames_q[B])
        nb_local = rotinv(qB0, n0)
        n = rot(q[B], nb_local) if Bdyn else n0
        rest_d = self.rest_off[sh0] + self.rest_off[sh1]
        e = 0.5 * (self.rest[sh0] + self.rest[sh1])
        rows = []
        for j in range(cnt):
            P0j = _t(P0[j])
            la = rotinv(qA0, P0j - cA0)
            lb = rotinv(qB0, P0j - cB0)
            Pa = c[A] + rot(q[A], la)
            Pb = (c[B] + rot(q[B], lb)) if Bdyn else P0j
            P = Pb
            sep = _t(s0[j]) + (n0 * (Pa - Pb)).sum()
            rA, rB = P - c[A], P - c[B]
            raxn, rbxn = cross(rA, n), cross(rB, n)
            ra, rb = C[A] @ raxn, C[B] @ rbxn
            vrel = (n * (v1[A] - v1[B])).sum() + ((raxn * w1[A]).sum() - (rbxn * w1[B]).sum())
            response = (im[A] + (ra * ra).sum()) + (im[B] + (rb * rb).sum())
            vm = 1.0 / response
            pen = sep - rest_d
            pen_dt = pen / dt
            separated = _f(pen) >= 0.0
            closing = -_f(vrel) > _f(pen_dt)
            bouncing = e > 0.0 and -2.0 > _f(vrel) and closing
            pds = pen_dt if separated else pen * (0.8 / dt)
            sbias = _t(0.0) if bouncing else vm * pds
            target = (-vrel * e if bouncing else 0.0) - vrel
            biased = target * vm - sbias
            unbiased = target * vm - (0.0 if bouncing else torch.clamp(sbias, min=0.0))
            rows.append((n, ra, rb, vm, biased, unbiased))
        dfr = torch.clamp(0.5 * (mu_d[sh0] + mu_d[sh1]), min=0.0)
        ssum = 0.5 * (mu_s[sh0] + mu_s[sh1])
        sfr = ssum if _f(dfr) < _f(ssum) else dfr
        frows = []
        K = int(rec.anchors[k]) & 255
        word = int(rec.anchors[k])
        if K:
            rel = v1[A] - v1[B]
            u = rel - n * (n * rel).sum()
            if _f((u * u).sum()) <= 0.0001:
                u = torch.stack([0.0 * n[0], -n[2], n[1]]) if abs(_f(n[0])) < 0.70710678 \
                    else torch.stack([-n[1], n[0], 0.0 * n[2]])
            t0 = u / torch.sqrt((u * u).sum())
            t1 = cross(n, t0)
            for a in range(K):
                if (word >> (10 + a)) & 1:
                    # taken from this step's point: at that point on both bodies
                    src = (word >> (12 + 2 * a)) & 3
                    Psrc = _t(P0[src])
                    lbs = rotinv(qB0, Psrc - cB0)
                    Pk = (c[B] + rot(q[B], lbs)) if Bdyn else Psrc
                    raK, rbK = Pk - c[A], Pk - c[B]
                else:
                    raK = rot(q[A], _t(rec.a0[k, a]))
                    rbK = rot(q[B], _t(rec.a1[k, a]))
                err = (raK + c[A]) - (rbK + c[B])
                for tg in (t0, t1):
                    ax0, ax1 = cross(raK, tg), cross(rbK, tg)
                    j0, j1 = C[A] @ ax0, C[B] @ ax1
                    resp = (im[A] + (j0 * j0).sum()) + (im[B] + (j1 * j1).sum())
                    frows.append((tg, j0, j1, 0.8 / resp, (tg * err).sum() / dt,
                                  -((tg * rel).sum() + (ax0 * w1[A]).sum() - (ax1 * w1[B]).sum())))
        return (A if self.dyn[A] else -1, B if Bdyn else -1, rows, frows, K, sfr, dfr, im[A], im[B])

    @staticmethod
    def _solve(item, applied, dv, dw, it, pos):
        zero3 = torch.zeros(3, dtype=torch.float64)

        def get(b):
            return (dv[b], dw[b]) if b >= 0 else (zero3, zero3)
        if item[0] == "joint":
            _, a, b, rows = item
            av, aw = get(a)
            bv, bw = get(b)
            for r, (axis, ja, jb, ima, imb, vm, const, unb) in enumerate(rows):
                nd = (axis * (av - bv)).sum() + (ja * aw).sum() - (jb * bw).sum()
                nx = applied[r] + nd * vm + (const if it < pos else unb)
                dl = nx - applied[r]
                applied[r] = nx
                av = av + axis * (dl * ima); aw = aw + ja * dl
                bv = bv - axis * (dl * imb); bw = bw - jb * dl
            if a >= 0:
                dv[a], dw[a] = av, aw
            if b >= 0:
                dv[b], dw[b] = bv, bw
            return
        _, a, b, rows, frows, K, sf, df, ima, imb = item
        av, aw = get(a)
        bv, bw = get(b)
        nsum = torch.zeros((), dtype=torch.float64)
        for j, (n, ra, rb, vm, biased, unbiased) in enumerate(rows):
            nvel = (n * (av - bv)).sum() + (aw * ra).sum() - (bw * rb).sum()
            err = biased if it < pos else unbiased
            dc_a, dc_b = -nvel * vm + err, -applied[j]
            dc = dc_b if _f(dc_a) < _f(dc_b) else dc_a
            ni = applied[j] + dc
            dl = ni - applied[j]
            av = av + n * (dl * ima); bv = bv - n * (dl * imb)
            aw = aw + ra * dl; bw = bw - rb * dl
            applied[j] = ni
            nsum = nsum + ni
        if (it >= pos or pos - it <= 3) and K:
            coeff = 0.5 if K == 2 else 1.0
            ms, md = sf * coeff * nsum, df * coeff * nsum
            for k, (t, ra, rb, vm, bias, target) in enumerate(frows):
                td = (t * (av - bv)).sum() + (aw * ra).sum() - (bw * rb).sum()
                y = applied[4 + k]
                cand = y + (target - (bias if it < pos else 0.0) - td) * vm
                if abs(_f(cand)) > _f(ms):
                    nx = -md if _f(cand) < -_f(md) else (md if _f(md) < _f(cand) else cand)
                else:
                    nx = cand
                dl = nx - y
                av = av + t * (dl * ima); bv = bv - t * (dl * imb)
                aw = aw + ra * dl; bw = bw - rb * dl
                applied[4 + k] = nx
        if a >= 0:
            dv[a], dw[a] = av, aw
        if b >= 0:
            dv[b], dw[b] = bv, bw


def model_for(pkg_world, spec):
    """Model constants of a one-scene world built from a SceneSpec."""
    nb = pkg_world.counts()["bodies"]
    dyn = np.zeros(nb, bool)
    im = np.zeros(nb)
    iI = np.zeros((nb, 3))
    u = np.zeros((nb, 3))
    first = 1 if spec.floor is not None else 0
    for i in range(nb):
        mp = pkg_world.body_mass_properties(i)
        dyn[i] = i >= first
        im[i], iI[i] = mp[0], mp[1:4]
        mlp = _t(mp[4:7])
        mlq = _t(mp[7:11])
        u[i] = rotinv(mlq, mlp).numpy()
    shape_body = np.asarray(spec.shape_body, np.int64) + first
    rest = np.asarray(spec.shape_mat[:, 2], np.float64)
    if spec.floor is not None:
        shape_body = np.concatenate([[0], shape_body])
        rest = np.concatenate([[spec.floor_mat[2]], rest])
    mlq = np.tile([0.0, 0.0, 0.0, 1.0], (nb, 1))
    for i in range(first, nb):
        mlq[i] = pkg_world.body_mass_properties(i)[7:11]
    return Model(dyn, im, iI, u, shape_body, rest, np.zeros(len(shape_body)), spec_joints(spec),
                 mass_local_q=mlq)


def spec_joints(spec):
    """The model's joints of a SceneSpec, in the step's canonical order
    (constraint slot descending); FLOOR_BODY endpoints are the floor actor."""
    first = 1 if spec.floor is not None else 0
    kinds = spec.joint_kinds()
    local = spec.joint_locals()

    def actor(i):
        return 0 if int(i) == 0xFFFFFFFF else int(i) + first
    joints = []
    for j, ((a, b), d) in enumerate(zip(spec.joints, spec.joint_dist)):
        if int(kinds[j]) == 0:
            joints.append((actor(a), actor(b), float(d)))
        else:
            joints.append((actor(a), actor(b), float(d), int(kinds[j]), local[j, :7].astype(np.float64),
                           local[j, 7:].astype(np.float64)))
    return joints[::-1]
