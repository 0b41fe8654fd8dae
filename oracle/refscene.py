"""Test infrastructure: ctypes access to the reference SDK's NativeCpu scene.

Loads ``oracle/_ref/libfyzz_ref.so`` (built by ``oracle/Makefile`` from the
reference sources plus ``ref_harness.cpp``).  Only tests, ``smoke()`` and the
CPU-baseline leg of ``bench.py`` use this module; the product never does.
"""
from __future__ import annotations

import ctypes as C
import os
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_ref", "libfyzz_ref.so")
_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise RuntimeError(f"reference harness not built: {LIB_PATH}")
        L = C.CDLL(LIB_PATH)
        vp, u32, u64, f32, i32 = C.c_void_p, C.c_uint32, C.c_uint64, C.c_float, C.c_int
        P = C.POINTER
        L.fz_ref_error.restype = C.c_char_p
        L.fz_ref_create.restype = vp
        L.fz_ref_create.argtypes = [i32]
        L.fz_ref_destroy.argtypes = [vp]
        L.fz_ref_build.argtypes = [vp, u32, vp, u32, vp, vp, vp, vp, vp, u32, vp, vp, i32, f32, vp]
        L.fz_ref_step.argtypes = [vp, f32, i32]
        L.fz_ref_advance_collision.argtypes = [vp]
        L.fz_ref_counts.argtypes = [vp, vp]
        L.fz_ref_body_states.argtypes = [vp, vp]
        L.fz_ref_mass_props.argtypes = [vp, vp]
        L.fz_ref_sleep_state.argtypes = [vp, vp]
        L.fz_ref_add_joint.argtypes = [vp, i32, u32, u32, vp, vp, f32, vp]
        L.fz_ref_remove_joint.argtypes = [vp, u64]
        L.fz_ref_set_kinematic.argtypes = [vp, u32, i32]
        L.fz_ref_set_kinematic_target.argtypes = [vp, u32, vp]
        L.fz_ref_encoded_bounds.argtypes = [vp, vp]
        L.fz_ref_set_meshes.argtypes = [vp, u32, vp, vp, vp, vp]
        L.fz_ref_cook_convex.argtypes = [vp, u32, vp, u32, vp, vp, vp, vp, vp]
        L.fz_ref_pcm_convex_gjk_epa.argtypes = [vp, vp, i32, vp, i32, f32, vp]
        L.fz_ref_pcm_convex_face_contacts.argtypes = [vp, vp, i32, vp, i32, f32, vp, vp]
        for name in ("fz_ref_endpoints",):
            getattr(L, name).restype = u64
        L.fz_ref_endpoints.argtypes = [vp, i32, vp, vp, vp]
        L.fz_ref_pairs.restype = u64
        L.fz_ref_pairs.argtypes = [vp, i32, vp]
        L.fz_ref_manifolds.restype = u64
        L.fz_ref_manifolds.argtypes = [vp, vp, vp, vp, vp]
        L.fz_ref_manager_order.restype = u64
        L.fz_ref_manager_order.argtypes = [vp, vp]
        L.fz_ref_joint_order.restype = u64
        L.fz_ref_joint_order.argtypes = [vp, vp]
        L.fz_ref_partitions.restype = u64
        L.fz_ref_partitions.argtypes = [vp, vp, vp]
        L.fz_ref_normal_impulses.restype = u64
        L.fz_ref_normal_impulses.argtypes = [vp, vp]
        L.fz_ref_contact_events.restype = u64
        L.fz_ref_contact_events.argtypes = [vp, vp, vp]
        L.fz_ref_contact_event_points.restype = u64
        L.fz_ref_contact_event_points.argtypes = [vp, vp, vp]
        L.fz_ref_pcm_box_box_candidates.argtypes = [vp, vp, f32, vp, vp]
        L.fz_ref_pcm_batch_selection.argtypes = [vp, u32, vp]
        L.fz_ref_pcm_box_box_gjk_epa.argtypes = [vp, vp, f32, vp]
        L.fz_ref_pcm_sphere_sphere.argtypes = [vp, f32, vp, f32, f32, vp]
        L.fz_ref_pcm_sphere_box.argtypes = [vp, f32, vp, f32, vp]
        L.fz_ref_step_many.argtypes = [P(vp), u32, f32, i32, i32]
        L.fz_ref_manager_order_pairs.restype = C.c_uint64
        L.fz_ref_manager_order_pairs.argtypes = [C.c_void_p, C.c_void_p]
        L.fz_ref_set_contact_report_threshold.argtypes = [C.c_void_p, C.c_uint32, C.c_float]
        L.fz_ref_force_threshold_changes.restype = C.c_uint64
        L.fz_ref_force_threshold_changes.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None and a.size else None


class RefScene:
    """One reference NativeCpu scene built from a SceneSpec."""

    def __init__(self, spec, contact_notifications: bool = False):
        L = lib()
        self.spec = spec
        self.h = L.fz_ref_create(1 if contact_notifications else 0)
        arrs = [np.ascontiguousarray(x) for x in (
            spec.bodies, spec.shape_body, spec.shape_type, spec.shape_geom,
            spec.shape_local, spec.shape_mat, spec.joints, spec.joint_dist)]
        self._keep = arrs
        self._floor_mat = np.asarray(spec.floor_mat, np.float32)
        kinds = spec.has_joint_kinds()
        if spec.convex_meshes:
            self._meshes = spec.mesh_arrays()
            nv, v, nt, t = self._meshes
            self._check(L.fz_ref_set_meshes(self.h, len(spec.convex_meshes), _p(nv), _p(v), _p(nt), _p(t)))
        rc = L.fz_ref_build(self.h, spec.n_bodies, _p(arrs[0]), spec.n_shapes,
                            _p(arrs[1]), _p(arrs[2]), _p(arrs[3]), _p(arrs[4]),
                            _p(arrs[5]), 0 if kinds else arrs[6].shape[0], _p(arrs[6]), _p(arrs[7]),
                            0 if spec.floor is None else 1,
                            0.0 if spec.floor is None else float(spec.floor),
                            _p(self._floor_mat))
        self._check(rc)
        if kinds:   # every joint in authoring order, each with its kind
            jk, local = spec.joint_kinds(), spec.joint_locals()
            for j in range(spec.joints.shape[0]):
                la, lb = np.ascontiguousarray(local[j, :7]), np.ascontiguousarray(local[j, 7:])
                self._check(L.fz_ref_add_joint(self.h, int(jk[j]), int(spec.joints[j, 0]), int(spec.joints[j, 1]),
                                               _p(la), _p(lb), float(spec.joint_dist[j]), None))

    def _check(self, rc):
        if rc:
            raise RuntimeError(f"reference error {rc}: {lib().fz_ref_error().decode()}")

    def close(self):
        if self.h:
            lib().fz_ref_destroy(self.h)
            self.h = None

    __del__ = close

    def step(self, dt: float = 1.0 / 120.0, steps: int = 1):
        self._check(lib().fz_ref_step(self.h, dt, steps))

    def advance_collision(self):
        self._check(lib().fz_ref_advance_collision(self.h))

    def counts(self) -> dict:
        out = np.zeros(10, np.uint64)
        lib().fz_ref_counts(self.h, _p(out))
        keys = ["actors", "shapes", "pairs", "found", "lost", "manifolds",
                "points", "partitions", "ordered", "tasks"]
        return {k: int(v) for k, v in zip(keys, out)}

    def body_states(self) -> np.ndarray:
        n = self.counts()["actors"]
        out = np.zeros((n, 14), np.float32)
        lib().fz_ref_body_states(self.h, _p(out))
        return out

    def add_joint(self, kind, a, b, local_a=None, local_b=None, distance=0.0) -> int:
        """A joint between 0-based dynamic bodies (0xffffffff: the floor);
        returns its ConstraintId."""
        ident = np.array([0, 0, 0, 0, 0, 0, 1], np.float32)
        la = np.ascontiguousarray(ident if local_a is None else local_a, np.float32).reshape(7)
        lb = np.ascontiguousarray(ident if local_b is None else local_b, np.float32).reshape(7)
        out = np.zeros(1, np.uint64)
        self._check(lib().fz_ref_add_joint(self.h, int(kind), int(a), int(b), _p(la), _p(lb), float(distance),
                                           _p(out)))
        return int(out[0])

    def remove_joint(self, cid: int):
        self._check(lib().fz_ref_remove_joint(self.h, int(cid)))

    def set_kinematic(self, body: int, on: bool = True):
        """Kinematic mode of dynamic body `body` (0-based index in the spec)."""
        self._check(lib().fz_ref_set_kinematic(self.h, body, 1 if on else 0))

    def set_kinematic_target(self, body: int, pose):
        p = np.ascontiguousarray(pose, np.float32).reshape(7)
        self._check(lib().fz_ref_set_kinematic_target(self.h, body, _p(p)))

    def sleep_state(self) -> dict:
        """Per actor: wake counter, sleeping, ready, counted interactions and
        the sleep filter's linear / local angular motion."""
        out = np.zeros((self.counts()["actors"], 10), np.float32)
        lib().fz_ref_sleep_state(self.h, _p(out))
        return {"wake": out[:, 0], "sleeping": out[:, 1].astype(bool), "ready": out[:, 2].astype(bool),
                "counted": out[:, 3].astype(np.uint32), "motion": out[:, 4:10]}

    def mass_props(self) -> np.ndarray:
        n = self.counts()["actors"]
        out = np.zeros((n, 11), np.float32)
        lib().fz_ref_mass_props(self.h, _p(out))
        return out

    def encoded_bounds(self) -> np.ndarray:
        n = self.counts()["shapes"]
        out = np.zeros((n, 6), np.uint32)
        lib().fz_ref_encoded_bounds(self.h, _p(out))
        return out

    def endpoints(self, axis: int = 0):
        n = lib().fz_ref_endpoints(self.h, axis, None, None, None)
        v = np.zeros(n, np.uint32); i = np.zeros(n, np.uint32); m = np.zeros(n, np.uint8)
        lib().fz_ref_endpoints(self.h, axis, _p(v), _p(i), _p(m))
        return v, i, m

    def pairs(self, which: int = 0) -> np.ndarray:
        n = lib().fz_ref_pairs(self.h, which, None)
        out = np.zeros((n, 2), np.uint32)
        lib().fz_ref_pairs(self.h, which, _p(out))
        return out

    def manifolds(self):
        n = lib().fz_ref_manifolds(self.h, None, None, None, None)
        pairs = np.zeros((n, 2), np.uint32)
        counts = np.zeros(n, np.uint32)
        rev = np.zeros(n, np.uint32)
        pts = np.zeros((n, 4, 7), np.float32)
        lib().fz_ref_manifolds(self.h, _p(pairs), _p(counts), _p(rev), _p(pts))
        return pairs, counts, rev, pts

    def manager_order(self) -> np.ndarray:
        n = lib().fz_ref_manager_order(self.h, None)
        out = np.zeros(n, np.uint64)
        lib().fz_ref_manager_order(self.h, _p(out))
        return out

    def manager_order_pairs(self) -> np.ndarray:
        """The last step's manager order as shape pairs (n, 2)."""
        n = lib().fz_ref_manager_order_pairs(self.h, None)
        out = np.zeros((n, 2), np.uint32)
        lib().fz_ref_manager_order_pairs(self.h, _p(out))
        return out

    def joint_order(self) -> np.ndarray:
        n = lib().fz_ref_joint_order(self.h, None)
        out = np.zeros(n, np.uint64)
        lib().fz_ref_joint_order(self.h, _p(out))
        return out

    def partitions(self):
        c = self.counts()
        d = np.zeros((c["ordered"], 4), np.uint32)
        e = np.zeros(c["partitions"], np.uint64)
        lib().fz_ref_partitions(self.h, _p(d), _p(e))
        return d, e

    def normal_impulses(self) -> np.ndarray:
        n = lib().fz_ref_normal_impulses(self.h, None)
        out = np.zeros(n, np.float64)
        lib().fz_ref_normal_impulses(self.h, _p(out))
        return out

    def set_contact_report_threshold(self, actor: int, force: float):
        """Scene::set_contact_report_threshold on BodyId `actor`."""
        self._check(lib().fz_ref_set_contact_report_threshold(self.h, int(actor), float(force)))

    def force_threshold_changes(self):
        """(rows (n, 4) u32: actor0, actor1, static_world, change; impulse
        (n,) f64; threshold (n,) f32) of the last step."""
        n = lib().fz_ref_force_threshold_changes(self.h, None, None, None)
        rows = np.zeros((n, 4), np.uint32)
        imp = np.zeros(n, np.float64)
        thr = np.zeros(n, np.float32)
        lib().fz_ref_force_threshold_changes(self.h, _p(rows), _p(imp), _p(thr))
        return rows, imp, thr

    def contact_events(self):
        """Events as (n, 7) u32: body0, body1, kind, count, point offset,
        shape0, shape1; and their summed normal impulses."""
        n = lib().fz_ref_contact_events(self.h, None, None)
        ev = np.zeros((n, 7), np.uint32)
        imp = np.zeros(n, np.float64)
        lib().fz_ref_contact_events(self.h, _p(ev), _p(imp))
        return ev, imp

    def contact_event_points(self):
        """Points as (n, 7) f32: position, normal, separation; and impulses."""
        n = lib().fz_ref_contact_event_points(self.h, None, None)
        pts = np.zeros((n, 7), np.float32)
        imp = np.zeros(n, np.float64)
        lib().fz_ref_contact_event_points(self.h, _p(pts), _p(imp))
        return pts, imp


def step_many(scenes, dt: float, steps: int, threads: int) -> None:
    arr = (C.c_void_p * len(scenes))(*[s.h for s in scenes])
    rc = lib().fz_ref_step_many(arr, len(scenes), dt, steps, threads)
    if rc:
        raise RuntimeError(f"reference error {rc}: {lib().fz_ref_error().decode()}")


def box_record(h, p, q):
    return np.array([*h, *p, *q], np.float32)


def pcm_box_box_candidates(a, b, cd):
    out = np.zeros((64, 10), np.float32)
    cnt = np.zeros(1, np.uint32)
    ok = lib().fz_ref_pcm_box_box_candidates(_p(a), _p(b), cd, _p(out), _p(cnt))
    if ok < 0:
        raise RuntimeError(lib().fz_ref_error().decode())
    return bool(ok), out[: int(cnt[0])]


def pcm_batch_selection(cands):
    out = np.zeros(4, np.uint8)
    c = np.ascontiguousarray(cands, np.float32)
    rc = lib().fz_ref_pcm_batch_selection(_p(c), c.shape[0], _p(out))
    if rc:
        raise RuntimeError(lib().fz_ref_error().decode())
    return out


def pcm_box_box_gjk_epa(a, b, cd):
    out = np.zeros(10, np.float32)
    ok = lib().fz_ref_pcm_box_box_gjk_epa(_p(a), _p(b), cd, _p(out))
    if ok < 0:
        raise RuntimeError(lib().fz_ref_error().decode())
    return bool(ok), out


def cook_convex(verts, tris):
    """fyzz::cook_convex_mesh: dict of faces (nf, 6: normal, distance, first,
    count), idx, volume (float64), center (3), inertia (3x3, column j =
    inertia[:, j]), lo, hi.  Raises ValueError when cooking rejects the mesh."""
    L = lib()
    v = np.ascontiguousarray(verts, np.float32).reshape(-1, 3)
    t = np.ascontiguousarray(tris, np.uint32).reshape(-1, 3)
    cap = 3 * t.shape[0]
    faces = np.zeros((cap, 6), np.float32)
    idx = np.zeros(cap, np.uint32)
    counts = np.zeros(2, np.uint32)
    vol = np.zeros(1, np.float64)
    m = np.zeros(18, np.float32)
    rc = L.fz_ref_cook_convex(_p(v), v.shape[0], _p(t), t.shape[0], _p(faces), _p(idx), _p(counts), _p(vol), _p(m))
    if rc:
        raise ValueError(L.fz_ref_error().decode())
    return {"faces": faces[:counts[0]], "idx": idx[:counts[1]], "volume": float(vol[0]), "center": m[0:3],
            "inertia": m[3:12].reshape(3, 3).T.copy(), "lo": m[12:15], "hi": m[15:18]}


class RefConvexGu:
    """The reference's free convex Gu functions (source_pcm_convex_gjk_epa,
    source_pcm_convex_face_contacts) over a fixed list of cooked meshes.
    Shapes are 11 floats: half extents, position, quaternion xyzw, radius."""

    def __init__(self, meshes):
        L = lib()
        self.h = L.fz_ref_create(0)
        self.spec_meshes = SceneMeshes(meshes)
        nv, v, nt, t = self.spec_meshes.arrays
        rc = L.fz_ref_set_meshes(self.h, len(meshes), _p(nv), _p(v), _p(nt), _p(t))
        if rc:
            raise ValueError(L.fz_ref_error().decode())

    def __del__(self):
        if getattr(self, "h", None):
            lib().fz_ref_destroy(self.h)
            self.h = None

    def gjk_epa(self, a, ma, b, mb, cd):
        out = np.zeros(10, np.float32)
        a = np.ascontiguousarray(a, np.float32)
        b = np.ascontiguousarray(b, np.float32)
        rc = lib().fz_ref_pcm_convex_gjk_epa(self.h, _p(a), ma, _p(b), mb, cd, _p(out))
        if rc < 0:
            raise RuntimeError(lib().fz_ref_error().decode())
        return bool(rc), out

    def face_contacts(self, a, ma, b, mb, cd, witness):
        out = np.zeros((4, 10), np.float32)
        a = np.ascontiguousarray(a, np.float32)
        b = np.ascontiguousarray(b, np.float32)
        w = np.ascontiguousarray(witness, np.float32)
        n = lib().fz_ref_pcm_convex_face_contacts(self.h, _p(a), ma, _p(b), mb, cd, _p(w), _p(out))
        if n < 0:
            raise RuntimeError(lib().fz_ref_error().decode())
        return out[:n]


class SceneMeshes:
    """Concatenated mesh arrays for the C ABIs."""

    def __init__(self, meshes):
        nv = np.asarray([m[0].shape[0] for m in meshes], np.uint32)
        nt = np.asarray([m[1].shape[0] for m in meshes], np.uint32)
        v = np.ascontiguousarray(np.concatenate([np.asarray(m[0], np.float32).reshape(-1, 3) for m in meshes]))
        t = np.ascontiguousarray(np.concatenate([np.asarray(m[1], np.uint32).reshape(-1, 3) for m in meshes]))
        self.arrays = (nv, v, nt, t)
