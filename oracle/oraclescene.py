"""Test infrastructure: ctypes access to the C restatement oracle
(``oracle/_build/liboracle.so``, built by ``oracle/Makefile``).

Only tests, ``smoke()`` and ``bench.py``'s CPU-baseline leg use this module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")
_lib = None


def build() -> None:
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        vp, u32, u64, f32, i32 = C.c_void_p, C.c_uint32, C.c_uint64, C.c_float, C.c_int
        L.fo_error.restype = C.c_char_p
        L.fo_scene_create.restype = vp
        L.fo_scene_create.argtypes = [u32, vp, u32, vp, vp, vp, vp, vp, u32, vp, vp, i32, f32, vp]
        L.fo_scene_create_ex.restype = vp
        L.fo_scene_create_ex.argtypes = [u32, vp, u32, vp, vp, vp, vp, vp, u32, vp, vp, i32, f32, vp,
                                         u32, vp, vp, vp, vp]
        L.fo_scene_destroy.argtypes = [vp]
        L.fo_scene_step.argtypes = [vp, f32, vp, u64, vp, u64]
        L.fo_scene_advance_collision.argtypes = [vp]
        for n in ("fo_scene_counts", "fo_scene_body_states", "fo_scene_set_body_states",
                  "fo_scene_mass_props", "fo_scene_encoded_bounds"):
            getattr(L, n).argtypes = [vp, vp]
        L.fo_scene_pairs.restype = u64
        L.fo_scene_pairs.argtypes = [vp, i32, vp]
        L.fo_scene_manifolds.restype = u64
        L.fo_scene_manifolds.argtypes = [vp, vp, vp, vp, vp]
        L.fo_scene_partitions.restype = u64
        L.fo_scene_partitions.argtypes = [vp, vp, vp]
        L.fo_scene_normal_impulses.restype = u64
        L.fo_scene_normal_impulses.argtypes = [vp, vp]
        L.fo_scene_set_sleeping.argtypes = [vp, i32]
        L.fo_scene_set_joint.argtypes = [vp, u32, u32, vp, vp]
        L.fo_scene_add_joint.argtypes = [vp, u32, u32, u32, vp, vp, f32, vp]
        L.fo_scene_remove_joint.argtypes = [vp, u64]
        L.fo_scene_set_kinematic.argtypes = [vp, u32, i32]
        L.fo_scene_set_kinematic_target.argtypes = [vp, u32, vp]
        L.fo_scene_sleep_state.argtypes = [vp, vp]
        L.fo_scene_sorted_min_x.restype = u64
        L.fo_scene_sorted_min_x.argtypes = [vp, vp, vp]
        L.fo_encode_min.restype = u32
        L.fo_encode_min.argtypes = [f32]
        L.fo_encode_max.restype = u32
        L.fo_encode_max.argtypes = [f32]
        L.fo_pcm_box_box_candidates.argtypes = [vp, vp, f32, vp, i32, vp]
        L.fo_pcm_batch_selection.argtypes = [vp, i32, f32, vp]
        L.fo_pcm_box_box_gjk_epa.argtypes = [vp, vp, f32, vp]
        L.fo_pcm_sphere_sphere.argtypes = [vp, f32, vp, f32, f32, vp]
        L.fo_pcm_sphere_plane.argtypes = [vp, f32, f32, f32, vp]
        L.fo_pcm_sphere_box.argtypes = [vp, f32, vp, f32, vp]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None and a.size else None


class OracleScene:
    def __init__(self, spec):
        L = lib()
        self.spec = spec
        arrs = [np.ascontiguousarray(x) for x in (
            spec.bodies, spec.shape_body, spec.shape_type, spec.shape_geom,
            spec.shape_local, spec.shape_mat, spec.joints, spec.joint_dist)]
        self._keep = arrs
        self._floor_mat = np.asarray(spec.floor_mat, np.float32)
        self._meshes = spec.mesh_arrays()
        nv, v, nt, t = self._meshes
        self.h = L.fo_scene_create_ex(spec.n_bodies, _p(arrs[0]), spec.n_shapes, _p(arrs[1]),
                                      _p(arrs[2]), _p(arrs[3]), _p(arrs[4]), _p(arrs[5]),
                                      arrs[6].shape[0], _p(arrs[6]), _p(arrs[7]),
                                      0 if spec.floor is None else 1,
                                      0.0 if spec.floor is None else float(spec.floor),
                                      _p(self._floor_mat), len(spec.convex_meshes), _p(nv), _p(v), _p(nt), _p(t))
        if not self.h:
            raise RuntimeError(L.fo_error().decode())
        if spec.has_joint_kinds():
            kinds, local = spec.joint_kinds(), spec.joint_locals()
            for j in range(spec.joints.shape[0]):
                la, lb = np.ascontiguousarray(local[j, :7]), np.ascontiguousarray(local[j, 7:])
                self._check(L.fo_scene_set_joint(self.h, j, int(kinds[j]), _p(la), _p(lb)))

    def close(self):
        if getattr(self, "h", None):
            lib().fo_scene_destroy(self.h)
            self.h = None

    __del__ = close

    def _check(self, rc):
        if rc:
            raise RuntimeError(f"oracle error {rc}: {lib().fo_error().decode()}")

    def step(self, dt: float = 1.0 / 120.0, manager_order=None, joint_order=None):
        mo = None if manager_order is None else np.ascontiguousarray(manager_order, np.uint64)
        jo = None if joint_order is None else np.ascontiguousarray(joint_order, np.uint64)
        rc = lib().fo_scene_step(self.h, dt, None if mo is None else mo.ctypes.data_as(C.c_void_p),
                                 0 if mo is None else mo.size,
                                 None if jo is None else jo.ctypes.data_as(C.c_void_p),
                                 0 if jo is None else jo.size)
        self._check(rc)

    def advance_collision(self):
        self._check(lib().fo_scene_advance_collision(self.h))

    def counts(self) -> dict:
        out = np.zeros(10, np.uint64)
        lib().fo_scene_counts(self.h, _p(out))
        keys = ["actors", "shapes", "pairs", "found", "lost", "manifolds",
                "points", "partitions", "ordered", "tasks"]
        return {k: int(v) for k, v in zip(keys, out)}

    def body_states(self) -> np.ndarray:
        out = np.zeros((self.counts()["actors"], 14), np.float32)
        lib().fo_scene_body_states(self.h, _p(out))
        return out

    def _actor(self, body: int) -> int:
        return body + (0 if self.spec.floor is None else 1)

    def add_joint(self, kind, a, b, local_a=None, local_b=None, distance=0.0) -> int:
        ident = np.array([0, 0, 0, 0, 0, 0, 1], np.float32)
        la = np.ascontiguousarray(ident if local_a is None else local_a, np.float32).reshape(7)
        lb = np.ascontiguousarray(ident if local_b is None else local_b, np.float32).reshape(7)
        out = np.zeros(1, np.uint64)
        self._check(lib().fo_scene_add_joint(self.h, int(kind), int(a), int(b), _p(la), _p(lb), float(distance),
                                             _p(out)))
        return int(out[0])

    def remove_joint(self, cid: int):
        self._check(lib().fo_scene_remove_joint(self.h, int(cid)))

    def set_kinematic(self, body: int, on: bool = True):
        """Kinematic mode of dynamic body `body` (0-based index in the spec)."""
        self._check(lib().fo_scene_set_kinematic(self.h, self._actor(body), 1 if on else 0))

    def set_kinematic_target(self, body: int, pose):
        p = np.ascontiguousarray(pose, np.float32).reshape(7)
        self._check(lib().fo_scene_set_kinematic_target(self.h, self._actor(body), _p(p)))

    def set_sleeping(self, on: bool):
        lib().fo_scene_set_sleeping(self.h, 1 if on else 0)

    def sleep_state(self) -> dict:
        """Per actor: wake counter, sleeping, ready, counted interactions and
        the sleep filter's linear / local angular motion."""
        out = np.zeros((self.counts()["actors"], 10), np.float32)
        lib().fo_scene_sleep_state(self.h, _p(out))
        return {"wake": out[:, 0], "sleeping": out[:, 1].astype(bool), "ready": out[:, 2].astype(bool),
                "counted": out[:, 3].astype(np.uint32), "motion": out[:, 4:10]}

    def set_body_states(self, st: np.ndarray):
        st = np.ascontiguousarray(st, np.float32)
        lib().fo_scene_set_body_states(self.h, _p(st))

    def mass_props(self) -> np.ndarray:
        out = np.zeros((self.counts()["actors"], 11), np.float32)
        lib().fo_scene_mass_props(self.h, _p(out))
        return out

    def encoded_bounds(self) -> np.ndarray:
        out = np.zeros((self.counts()["shapes"], 6), np.uint32)
        lib().fo_scene_encoded_bounds(self.h, _p(out))
        return out

    def pairs(self, which: int = 0) -> np.ndarray:
        n = lib().fo_scene_pairs(self.h, which, None)
        out = np.zeros((n, 2), np.uint32)
        lib().fo_scene_pairs(self.h, which, _p(out))
        return out

    def manifolds(self):
        n = lib().fo_scene_manifolds(self.h, None, None, None, None)
        pairs = np.zeros((n, 2), np.uint32)
        counts = np.zeros(n, np.uint32)
        rev = np.zeros(n, np.uint32)
        pts = np.zeros((n, 4, 7), np.float32)
        lib().fo_scene_manifolds(self.h, _p(pairs), _p(counts), _p(rev), _p(pts))
        return pairs, counts, rev, pts

    def partitions(self):
        c = self.counts()
        d = np.zeros((c["ordered"], 4), np.uint32)
        e = np.zeros(c["partitions"], np.uint64)
        lib().fo_scene_partitions(self.h, _p(d), _p(e))
        return d, e

    def normal_impulses(self) -> np.ndarray:
        n = lib().fo_scene_normal_impulses(self.h, None)
        out = np.zeros(n, np.float64)
        lib().fo_scene_normal_impulses(self.h, _p(out))
        return out

    def sorted_min_x(self):
        n = lib().fo_scene_sorted_min_x(self.h, None, None)
        v = np.zeros(n, np.uint32); i = np.zeros(n, np.uint32)
        lib().fo_scene_sorted_min_x(self.h, _p(v), _p(i))
        return v, i


def pcm_box_box_candidates(a, b, cd):
    out = np.zeros((64, 10), np.float32)
    cnt = np.zeros(1, np.int32)
    ok = lib().fo_pcm_box_box_candidates(_p(np.asarray(a, np.float32)), _p(np.asarray(b, np.float32)),
                                         cd, _p(out), 64, _p(cnt))
    if ok < 0:
        raise RuntimeError("oracle candidate overflow")
    return bool(ok), out[: int(cnt[0])]


def pcm_batch_selection(cands):
    out = np.zeros(4, np.uint8)
    c = np.ascontiguousarray(cands, np.float32)
    lib().fo_pcm_batch_selection(_p(c), c.shape[0], 1.0, _p(out))
    return out


def pcm_box_box_gjk_epa(a, b, cd):
    out = np.zeros(10, np.float32)
    ok = lib().fo_pcm_box_box_gjk_epa(_p(np.asarray(a, np.float32)), _p(np.asarray(b, np.float32)), cd, _p(out))
    return bool(ok), out


# ---------------- cooked convex hulls ----------------
class _Face(C.Structure):
    _fields_ = [("n", C.c_float * 3), ("d", C.c_float), ("first", C.c_uint32), ("count", C.c_uint32)]


class _Mesh(C.Structure):
    _fields_ = [("nv", C.c_uint32), ("nf", C.c_uint32), ("ni", C.c_uint32),
                ("verts", C.POINTER(C.c_float)), ("faces", C.POINTER(_Face)), ("idx", C.POINTER(C.c_uint32)),
                ("volume", C.c_double), ("center", C.c_float * 3), ("inertia", C.c_float * 9),
                ("lo", C.c_float * 3), ("hi", C.c_float * 3)]


class _Finite(C.Structure):
    _fields_ = [("half", C.c_float * 3), ("p", C.c_float * 3), ("q", C.c_float * 4), ("radius", C.c_float),
                ("hull", C.POINTER(_Mesh))]


def _cook(verts, tris):
    L = lib()
    L.fo_cook_convex.argtypes = [C.c_void_p, C.c_uint32, C.c_void_p, C.c_uint32, C.POINTER(_Mesh)]
    v = np.ascontiguousarray(verts, np.float32).reshape(-1, 3)
    t = np.ascontiguousarray(tris, np.uint32).reshape(-1, 3)
    m = _Mesh()
    if L.fo_cook_convex(_p(v), v.shape[0], _p(t), t.shape[0], C.byref(m)):
        raise ValueError("oracle cooking rejected the mesh")
    return m


def cook_convex(verts, tris):
    """The oracle's cooking, in the format of refscene.cook_convex."""
    m = _cook(verts, tris)
    faces = np.array([[*m.faces[i].n, m.faces[i].d, m.faces[i].first, m.faces[i].count] for i in range(m.nf)],
                     np.float32).reshape(-1, 6)
    out = {"faces": faces, "idx": np.array([m.idx[i] for i in range(m.ni)], np.uint32), "volume": m.volume,
           "center": np.array(m.center, np.float32), "inertia": np.array(m.inertia, np.float32).reshape(3, 3).T.copy(),
           "lo": np.array(m.lo, np.float32), "hi": np.array(m.hi, np.float32)}
    lib().fo_mesh_free(C.byref(m))
    return out


class OracleConvexGu:
    """fo_pcm_convex_gjk_epa / fo_pcm_convex_face_contacts over cooked
    meshes, with the argument format of refscene.RefConvexGu."""

    def __init__(self, meshes):
        self.meshes = [_cook(v, t) for (v, t) in meshes]
        L = lib()
        L.fo_pcm_convex_gjk_epa.argtypes = [C.POINTER(_Finite), C.POINTER(_Finite), C.c_float, C.c_void_p]
        L.fo_pcm_convex_face_contacts.argtypes = [C.POINTER(_Finite), C.POINTER(_Finite), C.c_float, C.c_void_p,
                                                  C.c_void_p]

    def __del__(self):
        for m in getattr(self, "meshes", []):
            lib().fo_mesh_free(C.byref(m))

    def _finite(self, d, mesh):
        f = _Finite()
        d = np.asarray(d, np.float32)
        f.half[:] = d[0:3].tolist()
        f.p[:] = d[3:6].tolist()
        f.q[:] = d[6:10].tolist()
        f.radius = float(d[10])
        if mesh >= 0:
            f.hull = C.pointer(self.meshes[mesh])
        return f

    def gjk_epa(self, a, ma, b, mb, cd):
        out = np.zeros(10, np.float32)
        ok = lib().fo_pcm_convex_gjk_epa(C.byref(self._finite(a, ma)), C.byref(self._finite(b, mb)), cd, _p(out))
        return bool(ok), out

    def face_contacts(self, a, ma, b, mb, cd, witness):
        out = np.zeros((4, 10), np.float32)
        w = np.ascontiguousarray(witness, np.float32)
        n = lib().fo_pcm_convex_face_contacts(C.byref(self._finite(a, ma)), C.byref(self._finite(b, mb)), cd,
                                             _p(w), _p(out))
        return out[:n]
