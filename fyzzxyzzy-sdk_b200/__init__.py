"""B200 rigid-body step: Python mirror of fyzz::World over the C ABI.

The product is ``lib/libfyzz_b200.so`` (CUDA kernels for sm_100a + the C++23
host engine); this module only binds its ``extern "C"`` entry points
(``include/fyzz_b200.h``).  There is no CPU fallback: creating a world raises
when the library or a CUDA device is missing.

Errors follow the reference's exception types (status 1 ValueError for
std::invalid_argument, 2 RuntimeError for std::logic_error, 3 OverflowError
for std::overflow_error, 4 RuntimeError for std::runtime_error).
"""
from __future__ import annotations

import ctypes as C
import os
import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libfyzz_b200.so")
_lib = None

# Every entry point declared in include/fyzz_b200.h.
EXPORTS = (
    "fyzz_b200_create", "fyzz_b200_destroy", "fyzz_b200_last_error", "fyzz_b200_error_bits",
    "fyzz_b200_begin_scene", "fyzz_b200_add_static_floor", "fyzz_b200_create_dynamic_body",
    "fyzz_b200_attach_box_shape", "fyzz_b200_attach_sphere_shape",
    "fyzz_b200_update_mass_properties", "fyzz_b200_body_mass_properties",
    "fyzz_b200_set_shape_material", "fyzz_b200_set_body_velocity",
    "fyzz_b200_set_body_angular_velocity", "fyzz_b200_add_center_distance_constraint",
    "fyzz_b200_add_anchored_distance_constraint", "fyzz_b200_add_fixed_constraint",
    "fyzz_b200_add_spherical_constraint", "fyzz_b200_add_revolute_constraint",
    "fyzz_b200_add_prismatic_constraint",
    "fyzz_b200_add_scene", "fyzz_b200_step", "fyzz_b200_step_n", "fyzz_b200_collide",
    "fyzz_b200_synchronize", "fyzz_b200_body_state", "fyzz_b200_read_bodies",
    "fyzz_b200_write_velocities", "fyzz_b200_counts", "fyzz_b200_device_view",
    "fyzz_b200_read_pairs", "fyzz_b200_read_manifolds", "fyzz_b200_read_encoded_bounds",
    "fyzz_b200_read_sorted_min_x", "fyzz_b200_read_levels", "fyzz_b200_profile_step",
    "fyzz_b200_kernels_per_step", "fyzz_b200_sap_pairs_static_scratch",
    "fyzz_b200_read_step_counters", "fyzz_b200_set_contact_notifications",
    "fyzz_b200_contact_events", "fyzz_b200_rollout_begin", "fyzz_b200_rollout_forward",
    "fyzz_b200_rollout_backward", "fyzz_b200_read_mass_frames", "fyzz_b200_read_friction_anchors",
    "fyzz_b200_fit_pair_budget", "fyzz_b200_set_sleeping", "fyzz_b200_read_sleep_state", "fyzz_b200_set_body_kinematic",
    "fyzz_b200_set_body_kinematic_target", "fyzz_b200_rollout_rewind",
    "fyzz_b200_cook_convex_mesh", "fyzz_b200_convex_mesh_release", "fyzz_b200_cook_error",
    "fyzz_b200_convex_mesh_info", "fyzz_b200_attach_convex_shape", "fyzz_b200_add_scene_ex",
    "fyzz_b200_write_velocities_strided", "fyzz_b200_remove_constraint",
    "fyzz_b200_set_pair_budget", "fyzz_b200_test_scan",
    "fyzz_b200_set_body_contact_report_threshold", "fyzz_b200_force_threshold_changes",
    "fyzz_b200_read_islands", "fyzz_b200_set_caller_validated_transforms",
    "fyzz_b200_set_descriptor_order", "fyzz_b200_set_tuning", "fyzz_b200_get_tuning",
)
STAGES = ("bounds", "sort", "pairs", "narrowphase", "islands", "prep", "pgs", "integrate")


def build() -> str:
    from importlib import import_module
    return import_module(__name__ + ".build").build()


class BodyState(C.Structure):
    _fields_ = [("position", C.c_float * 3), ("velocity", C.c_float * 3),
                ("orientation", C.c_float * 4), ("angular_velocity", C.c_float * 3),
                ("sleeping", C.c_uint32)]


class Material(C.Structure):
    _fields_ = [("static_friction", C.c_float), ("dynamic_friction", C.c_float),
                ("restitution", C.c_float)]


class ContactEvent(C.Structure):
    """fyzz_b200_contact_event_t (reference ContactEvent, world.h:176-190)."""
    _fields_ = [("body0", C.c_uint32), ("body1", C.c_uint32), ("shape0", C.c_uint32),
                ("shape1", C.c_uint32), ("kind", C.c_uint32), ("contact_count", C.c_uint32),
                ("point_offset", C.c_uint64), ("normal_impulse", C.c_double)]


class ContactEventPoint(C.Structure):
    """fyzz_b200_contact_event_point_t (reference ContactEventPoint, world.h:194-199)."""
    _fields_ = [("position", C.c_float * 3), ("normal", C.c_float * 3), ("separation", C.c_float),
                ("reserved", C.c_uint32), ("normal_impulse", C.c_double)]


EVENT_DTYPE = np.dtype([("body0", "<u4"), ("body1", "<u4"), ("shape0", "<u4"), ("shape1", "<u4"),
                        ("kind", "<u4"), ("contact_count", "<u4"), ("point_offset", "<u8"),
                        ("normal_impulse", "<f8")])
EVENT_POINT_DTYPE = np.dtype([("position", "<f4", 3), ("normal", "<f4", 3), ("separation", "<f4"),
                              ("reserved", "<u4"), ("normal_impulse", "<f8")])
FOUND, PERSISTS, LOST = 0, 1, 2


class ForceThresholdReport(C.Structure):
    _fields_ = [("actor0", C.c_uint32), ("actor1", C.c_uint32), ("static_world", C.c_uint32),
                ("change", C.c_uint32), ("normal_impulse", C.c_double), ("threshold", C.c_float),
                ("reserved", C.c_uint32)]


THRESHOLD_DTYPE = np.dtype([("actor0", "<u4"), ("actor1", "<u4"), ("static_world", "<u4"), ("change", "<u4"),
                            ("normal_impulse", "<f8"), ("threshold", "<f4"), ("reserved", "<u4")])


class Tuning(C.Structure):
    _fields_ = [("island_thread", C.c_uint32), ("island_warp", C.c_uint32), ("island_cta", C.c_uint32),
                ("radix_bits", C.c_uint32), ("elem_block", C.c_uint32), ("work_queue", C.c_uint32)]

    def as_dict(self) -> dict:
        return {k: int(getattr(self, k)) for k, _ in self._fields_}


class DeviceView(C.Structure):
    _fields_ = [("position", C.c_void_p), ("orientation", C.c_void_p),
                ("velocity", C.c_void_p), ("angular_velocity", C.c_void_p),
                ("n_bodies", C.c_uint32), ("n_shapes", C.c_uint32), ("stream", C.c_void_p)]


def lib():
    """Load the in-tree library (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(f"B200 library missing: {LIB_PATH} (run build())")
        L = C.CDLL(LIB_PATH)
        vp, u32, u64, f32, i32 = C.c_void_p, C.c_uint32, C.c_uint64, C.c_float, C.c_int
        P = C.POINTER
        L.fyzz_b200_create.argtypes = [i32, P(vp)]
        L.fyzz_b200_destroy.argtypes = [vp]
        L.fyzz_b200_last_error.argtypes = [vp]
        L.fyzz_b200_last_error.restype = C.c_char_p
        L.fyzz_b200_error_bits.argtypes = [vp, P(u32)]
        L.fyzz_b200_begin_scene.argtypes = [vp, P(u32)]
        L.fyzz_b200_add_static_floor.argtypes = [vp, f32, P(u32)]
        L.fyzz_b200_create_dynamic_body.argtypes = [vp, vp, P(u32)]
        L.fyzz_b200_attach_box_shape.argtypes = [vp, u32, vp, vp, P(u32)]
        L.fyzz_b200_attach_sphere_shape.argtypes = [vp, u32, f32, vp, P(u32)]
        L.fyzz_b200_update_mass_properties.argtypes = [vp, u32, f32]
        L.fyzz_b200_body_mass_properties.argtypes = [vp, u32, vp]
        L.fyzz_b200_set_shape_material.argtypes = [vp, u32, P(Material)]
        L.fyzz_b200_set_body_velocity.argtypes = [vp, u32, vp]
        L.fyzz_b200_set_body_angular_velocity.argtypes = [vp, u32, vp]
        L.fyzz_b200_add_center_distance_constraint.argtypes = [vp, u32, u32, f32, P(u64)]
        L.fyzz_b200_add_anchored_distance_constraint.argtypes = [vp, u32, u32, vp, vp, f32, P(u64)]
        for name in ("fixed", "spherical", "revolute", "prismatic"):
            getattr(L, f"fyzz_b200_add_{name}_constraint").argtypes = [vp, u32, u32, vp, vp, P(u64)]
        L.fyzz_b200_add_scene.argtypes = [vp, u32, vp, u32, vp, vp, vp, vp, vp, u32, vp, vp, i32, f32, vp, P(u32)]
        L.fyzz_b200_add_scene_ex.argtypes = [vp, u32, vp, u32, vp, vp, vp, vp, vp, u32, vp, vp, i32, f32, vp,
                                             u32, P(vp), P(u32)]
        L.fyzz_b200_cook_convex_mesh.argtypes = [vp, u32, vp, u32, P(vp)]
        L.fyzz_b200_convex_mesh_release.argtypes = [vp]
        L.fyzz_b200_convex_mesh_release.restype = None
        L.fyzz_b200_cook_error.argtypes = []
        L.fyzz_b200_cook_error.restype = C.c_char_p
        L.fyzz_b200_convex_mesh_info.argtypes = [vp, vp, vp, vp, vp, vp]
        L.fyzz_b200_attach_convex_shape.argtypes = [vp, u32, vp, vp, P(u32)]
        L.fyzz_b200_step.argtypes = [vp, f32]
        L.fyzz_b200_step_n.argtypes = [vp, f32, u32]
        L.fyzz_b200_collide.argtypes = [vp]
        L.fyzz_b200_synchronize.argtypes = [vp]
        L.fyzz_b200_body_state.argtypes = [vp, u32, P(BodyState)]
        L.fyzz_b200_read_bodies.argtypes = [vp, vp, u32]
        L.fyzz_b200_write_velocities.argtypes = [vp, vp, u32]
        L.fyzz_b200_write_velocities_strided.argtypes = [vp, vp, u32, u32, u32, u32]
        L.fyzz_b200_remove_constraint.argtypes = [vp, u64]
        L.fyzz_b200_counts.argtypes = [vp, vp]
        L.fyzz_b200_device_view.argtypes = [vp, P(DeviceView)]
        L.fyzz_b200_read_pairs.argtypes = [vp, i32, vp, u64]
        L.fyzz_b200_read_pairs.restype = u64
        L.fyzz_b200_read_manifolds.argtypes = [vp, vp, vp, vp, u64]
        L.fyzz_b200_read_manifolds.restype = u64
        L.fyzz_b200_read_encoded_bounds.argtypes = [vp, vp, u32]
        L.fyzz_b200_read_sorted_min_x.argtypes = [vp, u32, vp, vp, u64]
        L.fyzz_b200_read_sorted_min_x.restype = u64
        L.fyzz_b200_read_levels.argtypes = [vp, vp, u64]
        L.fyzz_b200_read_islands.argtypes = [vp, vp, vp, u64]
        L.fyzz_b200_read_islands.restype = u64
        L.fyzz_b200_read_levels.restype = u64
        L.fyzz_b200_profile_step.argtypes = [vp, f32, vp, u32]
        L.fyzz_b200_kernels_per_step.argtypes = [vp, P(u32)]
        L.fyzz_b200_read_step_counters.argtypes = [vp, vp, u32]
        L.fyzz_b200_set_contact_notifications.argtypes = [vp, i32]
        L.fyzz_b200_set_sleeping.argtypes = [vp, i32]
        L.fyzz_b200_set_body_kinematic.argtypes = [vp, u32, i32]
        L.fyzz_b200_set_body_kinematic_target.argtypes = [vp, u32, vp]
        L.fyzz_b200_read_sleep_state.argtypes = [vp, vp, vp, vp, vp, u32]
        L.fyzz_b200_rollout_begin.argtypes = [vp, u32, u32]
        L.fyzz_b200_rollout_rewind.argtypes = [vp]
        L.fyzz_b200_fit_pair_budget.argtypes = [vp, f32, P(u32)]
        L.fyzz_b200_set_pair_budget.argtypes = [vp, u32, P(u32)]
        L.fyzz_b200_set_descriptor_order.argtypes = [vp, vp, u64, vp, u64]
        L.fyzz_b200_set_tuning.argtypes = [vp, P(Tuning)]
        L.fyzz_b200_get_tuning.argtypes = [vp, P(Tuning)]
        L.fyzz_b200_set_body_contact_report_threshold.argtypes = [vp, u32, f32]
        L.fyzz_b200_force_threshold_changes.argtypes = [vp, P(P(ForceThresholdReport)), P(u64)]
        L.fyzz_b200_test_scan.argtypes = [vp, u32, i32, P(u32), P(u64)]
        L.fyzz_b200_rollout_forward.argtypes = [vp, f32]
        L.fyzz_b200_rollout_backward.argtypes = [vp] + [vp] * 9
        L.fyzz_b200_read_mass_frames.argtypes = [vp, vp, vp]
        L.fyzz_b200_read_friction_anchors.argtypes = [vp, vp, vp, vp, u64]
        L.fyzz_b200_read_friction_anchors.restype = u64
        L.fyzz_b200_contact_events.argtypes = [vp, P(P(ContactEvent)), P(u64), P(P(ContactEventPoint)),
                                               P(u64)]
        L.fyzz_b200_sap_pairs_static_scratch.argtypes = [vp, vp, u32, vp, u32, vp, vp, C.c_char_p,
                                                         C.c_size_t]
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None and a.size else None


def _f32(x, n):
    a = np.ascontiguousarray(np.asarray(x, np.float32).reshape(-1))
    if a.size != n:
        raise ValueError(f"expected {n} floats")
    return a


_IDENTITY = np.array([0, 0, 0, 0, 0, 0, 1], np.float32)


class LogicError(RuntimeError):
    """FYZZ_B200_LOGIC_ERROR: the reference's std::logic_error (an operation
    the world's state does not allow, or a bounded device wait that gave
    up)."""


class World:
    """One B200 world: a batch of independent scenes stepped together.

    Mirrors fyzz::World (reference include/fyzzxyzzy/world.h:396-510) for the
    operations the rigid-body step supports."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        rc = lib().fyzz_b200_create(device, C.byref(h))
        if rc:
            raise RuntimeError(f"fyzz_b200_create failed ({rc}): no CUDA device or context")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().fyzz_b200_destroy(self.h)
            self.h = None

    __del__ = close

    def _check(self, rc):
        if rc == 0:
            return
        msg = lib().fyzz_b200_last_error(self.h).decode()
        if rc == 1:
            raise ValueError(msg)
        if rc == 3:
            raise OverflowError(msg)
        if rc == 2:
            raise LogicError(msg)
        raise RuntimeError(msg)

    # ---- authoring ----
    def begin_scene(self) -> int:
        out = C.c_uint32()
        self._check(lib().fyzz_b200_begin_scene(self.h, C.byref(out)))
        return out.value

    def add_static_floor(self, height: float) -> int:
        out = C.c_uint32()
        self._check(lib().fyzz_b200_add_static_floor(self.h, height, C.byref(out)))
        return out.value

    def create_dynamic_body(self, pose=_IDENTITY) -> int:
        p = _f32(pose, 7)
        out = C.c_uint32()
        self._check(lib().fyzz_b200_create_dynamic_body(self.h, _p(p), C.byref(out)))
        return out.value

    def attach_box_shape(self, body: int, half_extents, local_pose=_IDENTITY) -> int:
        h, l = _f32(half_extents, 3), _f32(local_pose, 7)
        out = C.c_uint32()
        self._check(lib().fyzz_b200_attach_box_shape(self.h, body, _p(h), _p(l), C.byref(out)))
        return out.value

    def attach_sphere_shape(self, body: int, radius: float, local_pose=_IDENTITY) -> int:
        l = _f32(local_pose, 7)
        out = C.c_uint32()
        self._check(lib().fyzz_b200_attach_sphere_shape(self.h, body, radius, _p(l), C.byref(out)))
        return out.value

    def attach_convex_shape(self, body: int, mesh: "ConvexMesh", local_pose=_IDENTITY) -> int:
        """World::attach_convex_shape (reference world.h:412)."""
        l = _f32(local_pose, 7)
        out = C.c_uint32()
        self._check(lib().fyzz_b200_attach_convex_shape(self.h, body, mesh.h, _p(l), C.byref(out)))
        return out.value

    def update_mass_properties(self, body: int, density: float):
        self._check(lib().fyzz_b200_update_mass_properties(self.h, body, density))

    def body_mass_properties(self, body: int) -> np.ndarray:
        out = np.zeros(11, np.float32)
        self._check(lib().fyzz_b200_body_mass_properties(self.h, body, _p(out)))
        return out

    def set_shape_material(self, shape: int, static_friction=0.5, dynamic_friction=0.5, restitution=0.2):
        m = Material(static_friction, dynamic_friction, restitution)
        self._check(lib().fyzz_b200_set_shape_material(self.h, shape, C.byref(m)))

    def set_body_velocity(self, body: int, v):
        a = _f32(v, 3)
        self._check(lib().fyzz_b200_set_body_velocity(self.h, body, _p(a)))

    def set_body_angular_velocity(self, body: int, v):
        a = _f32(v, 3)
        self._check(lib().fyzz_b200_set_body_angular_velocity(self.h, body, _p(a)))

    def add_center_distance_constraint(self, a: int, b: int, distance: float) -> int:
        out = C.c_uint64()
        self._check(lib().fyzz_b200_add_center_distance_constraint(self.h, a, b, distance, C.byref(out)))
        return out.value

    def add_anchored_distance_constraint(self, a: int, b: int, local_a, local_b, distance: float) -> int:
        """World::add_anchored_distance_constraint (reference world.h:441)."""
        la, lb = np.asarray(local_a, np.float32)[:3].copy(), np.asarray(local_b, np.float32)[:3].copy()
        out = C.c_uint64()
        self._check(lib().fyzz_b200_add_anchored_distance_constraint(self.h, a, b, _p(la), _p(lb), distance,
                                                                     C.byref(out)))
        return out.value

    def _frame_joint(self, name: str, a: int, b: int, local_a, local_b) -> int:
        la, lb = np.asarray(local_a, np.float32).reshape(7).copy(), np.asarray(local_b, np.float32).reshape(7).copy()
        out = C.c_uint64()
        self._check(getattr(lib(), f"fyzz_b200_add_{name}_constraint")(self.h, a, b, _p(la), _p(lb), C.byref(out)))
        return out.value

    def remove_constraint(self, cid: int):
        """World::remove_constraint (reference world.h:458)."""
        self._check(lib().fyzz_b200_remove_constraint(self.h, int(cid)))

    def add_fixed_constraint(self, a: int, b: int, local_a, local_b) -> int:
        """World::add_fixed_constraint: local frames are position(3) + xyzw(4)."""
        return self._frame_joint("fixed", a, b, local_a, local_b)

    def add_spherical_constraint(self, a: int, b: int, local_a, local_b) -> int:
        return self._frame_joint("spherical", a, b, local_a, local_b)

    def add_revolute_constraint(self, a: int, b: int, local_a, local_b) -> int:
        return self._frame_joint("revolute", a, b, local_a, local_b)

    def add_prismatic_constraint(self, a: int, b: int, local_a, local_b) -> int:
        return self._frame_joint("prismatic", a, b, local_a, local_b)

    def add_scene(self, spec) -> int:
        """Author one seeded scene (fyzzxyzzy-sdk_b200.scenes.SceneSpec);
        returns the BodyId of its first dynamic body."""
        arrs = [np.ascontiguousarray(x) for x in (
            spec.bodies, spec.shape_body, spec.shape_type, spec.shape_geom,
            spec.shape_local, spec.shape_mat, spec.joints, spec.joint_dist)]
        fm = np.asarray(spec.floor_mat, np.float32)
        out = C.c_uint32()
        kinds = spec.has_joint_kinds()
        meshes = [ConvexMesh(v, t) for (v, t) in getattr(spec, "convex_meshes", [])]
        handles = (C.c_void_p * max(1, len(meshes)))(*[m.h for m in meshes])
        self._check(lib().fyzz_b200_add_scene_ex(
            self.h, spec.n_bodies, _p(arrs[0]), spec.n_shapes, _p(arrs[1]), _p(arrs[2]),
            _p(arrs[3]), _p(arrs[4]), _p(arrs[5]), 0 if kinds else arrs[6].shape[0], _p(arrs[6]), _p(arrs[7]),
            0 if spec.floor is None else 1, 0.0 if spec.floor is None else float(spec.floor),
            _p(fm), len(meshes), handles, C.byref(out)))
        first = out.value
        if kinds:   # every joint in authoring order, each with its kind
            from .scenes import FLOOR_BODY
            jk, local = spec.joint_kinds(), spec.joint_locals()
            body = lambda i: first - 1 if int(i) == FLOOR_BODY else first + int(i)
            names = {2: "fixed", 3: "spherical", 4: "revolute", 5: "prismatic"}
            for j in range(spec.joints.shape[0]):
                a, b, k = body(spec.joints[j, 0]), body(spec.joints[j, 1]), int(jk[j])
                if k == 0:
                    self.add_center_distance_constraint(a, b, float(spec.joint_dist[j]))
                elif k == 1:
                    self.add_anchored_distance_constraint(a, b, local[j, :3], local[j, 7:10],
                                                          float(spec.joint_dist[j]))
                else:
                    self._frame_joint(names[k], a, b, local[j, :7], local[j, 7:])
        return first

    # ---- stepping ----
    def step(self, seconds: float = 1.0 / 120.0, steps: int = 1):
        if steps == 1:
            self._check(lib().fyzz_b200_step(self.h, seconds))
        else:
            self._check(lib().fyzz_b200_step_n(self.h, seconds, steps))

    def collide(self):
        self._check(lib().fyzz_b200_collide(self.h))

    def profile_step(self, seconds: float = 1.0 / 120.0) -> dict:
        """One eagerly launched step; per-stage device milliseconds from CUDA
        events the library records on its stream."""
        out = np.zeros(len(STAGES), np.float32)
        self._check(lib().fyzz_b200_profile_step(self.h, seconds, _p(out), out.size))
        return dict(zip(STAGES, out.tolist()))

    def kernels_per_step(self) -> int:
        out = C.c_uint32()
        self._check(lib().fyzz_b200_kernels_per_step(self.h, C.byref(out)))
        return out.value

    def synchronize(self):
        self._check(lib().fyzz_b200_synchronize(self.h))

    # ---- results ----
    def counts(self) -> dict:
        out = np.zeros(12, np.uint64)
        self._check(lib().fyzz_b200_counts(self.h, _p(out)))
        keys = ["bodies", "shapes", "scenes", "pairs", "managers", "points",
                "descriptors", "islands", "joints", "steps", "friction_rows", "found_lost"]
        return {k: int(v) for k, v in zip(keys, out)}

    def body_state(self, body: int) -> BodyState:
        out = BodyState()
        self._check(lib().fyzz_b200_body_state(self.h, body, C.byref(out)))
        return out

    def read_bodies(self, out: np.ndarray | None = None) -> np.ndarray:
        n = self.counts()["bodies"] if out is None else out.shape[0]
        if out is None:
            out = np.zeros((n, 14), np.float32)
        self._check(lib().fyzz_b200_read_bodies(self.h, _p(out), n))
        return out

    def write_velocities(self, v6: np.ndarray):
        v6 = np.ascontiguousarray(v6, np.float32)
        self._check(lib().fyzz_b200_write_velocities(self.h, _p(v6), v6.shape[0]))

    def write_states(self, states: np.ndarray):
        """Writes back the velocities of (n, 14) body records as read_bodies
        returns them (one host-to-device copy of the records as they are)."""
        if states.dtype != np.float32 or states.ndim != 2 or states.shape[1] != 14 or not states.flags.c_contiguous:
            raise ValueError("states must be a contiguous (n, 14) float32 array")
        self._check(lib().fyzz_b200_write_velocities_strided(self.h, _p(states), states.shape[0], 14, 3, 10))

    def device_view(self) -> DeviceView:
        out = DeviceView()
        self._check(lib().fyzz_b200_device_view(self.h, C.byref(out)))
        return out

    def pairs(self, which: int = 0) -> np.ndarray:
        n = lib().fyzz_b200_read_pairs(self.h, which, None, 0)
        out = np.zeros((n, 2), np.uint32)
        lib().fyzz_b200_read_pairs(self.h, which, _p(out), n)
        return out

    def manifolds(self):
        n = lib().fyzz_b200_read_manifolds(self.h, None, None, None, 0)
        pairs = np.zeros((n, 2), np.uint32)
        counts = np.zeros(n, np.uint32)
        pts = np.zeros((n, 4, 7), np.float32)
        lib().fyzz_b200_read_manifolds(self.h, _p(pairs), _p(counts), _p(pts), n)
        return pairs, counts, pts

    def encoded_bounds(self) -> np.ndarray:
        n = self.counts()["shapes"]
        out = np.zeros((n, 6), np.uint32)
        self._check(lib().fyzz_b200_read_encoded_bounds(self.h, _p(out), n))
        return out

    def sorted_min_x(self, scene: int = 0):
        n = lib().fyzz_b200_read_sorted_min_x(self.h, scene, None, None, 0)
        v = np.zeros(n, np.uint32)
        i = np.zeros(n, np.uint32)
        lib().fyzz_b200_read_sorted_min_x(self.h, scene, _p(v), _p(i), n)
        return v, i

    def levels(self) -> np.ndarray:
        n = lib().fyzz_b200_read_levels(self.h, None, 0)
        out = np.zeros(n, np.uint32)
        lib().fyzz_b200_read_levels(self.h, _p(out), n)
        return out

    def islands(self):
        """Awake islands of the last step: (descriptors, levels) per island."""
        n = lib().fyzz_b200_read_islands(self.h, None, None, 0)
        d = np.zeros(n, np.uint32)
        lv = np.zeros(n, np.uint32)
        lib().fyzz_b200_read_islands(self.h, _p(d), _p(lv), n)
        return d, lv

    def set_body_kinematic(self, body: int, enabled: bool = True):
        """World::set_body_kinematic (reference world.h:505)."""
        self._check(lib().fyzz_b200_set_body_kinematic(self.h, body, 1 if enabled else 0))

    def set_body_kinematic_target(self, body: int, pose):
        """World::set_body_kinematic_target: position(3) + quaternion xyzw(4)."""
        p = np.asarray(pose, np.float32).reshape(7).copy()
        self._check(lib().fyzz_b200_set_body_kinematic_target(self.h, body, _p(p)))

    def set_sleeping(self, enabled: bool = True):
        """Sleeping on (default, as in the reference scene) or off (wakes every body)."""
        self._check(lib().fyzz_b200_set_sleeping(self.h, 1 if enabled else 0))

    def sleep_state(self) -> dict:
        """Per body: wake counter, flags (1 asleep, 2 ready), sleep-filter motion
        (accumulated linear, body-local angular) and counted interactions."""
        n = self.counts()["bodies"]
        wake = np.zeros(n, np.float32)
        flags = np.zeros(n, np.uint32)
        motion = np.zeros((n, 6), np.float32)
        counted = np.zeros(n, np.uint32)
        self._check(lib().fyzz_b200_read_sleep_state(self.h, _p(wake), _p(flags), _p(motion), _p(counted), n))
        return {"wake": wake, "flags": flags, "motion": motion, "counted": counted}

    def set_contact_notifications(self, enabled: bool = True):
        """WorldOptions::contact_notifications (reference world.h:61)."""
        self._check(lib().fyzz_b200_set_contact_notifications(self.h, 1 if enabled else 0))

    def contact_events(self):
        """Events and points of the last step as numpy structured arrays
        (EVENT_DTYPE, EVENT_POINT_DTYPE), copied out of the world's buffers."""
        ev, pt = C.POINTER(ContactEvent)(), C.POINTER(ContactEventPoint)()
        nev, npt = C.c_uint64(), C.c_uint64()
        self._check(lib().fyzz_b200_contact_events(self.h, C.byref(ev), C.byref(nev), C.byref(pt),
                                                   C.byref(npt)))
        events = np.zeros(nev.value, EVENT_DTYPE)
        points = np.zeros(npt.value, EVENT_POINT_DTYPE)
        if nev.value:
            C.memmove(events.ctypes.data, ev, nev.value * EVENT_DTYPE.itemsize)
        if npt.value:
            C.memmove(points.ctypes.data, pt, npt.value * EVENT_POINT_DTYPE.itemsize)
        return events, points

    # ---- force-threshold stream ----
    def set_body_contact_report_threshold(self, body: int, force: float):
        """World::set_body_contact_report_threshold (FLT_MAX disables)."""
        self._check(lib().fyzz_b200_set_body_contact_report_threshold(self.h, body, force))

    def force_threshold_changes(self) -> np.ndarray:
        """The last step's force-threshold changes (structured array:
        actor0, actor1, static_world, change 0 Found / 1 Persists / 2 Lost,
        normal_impulse, threshold), in key order."""
        ptr = C.POINTER(ForceThresholdReport)()
        n = C.c_uint64()
        self._check(lib().fyzz_b200_force_threshold_changes(self.h, C.byref(ptr), C.byref(n)))
        if not n.value:
            return np.zeros(0, THRESHOLD_DTYPE)
        raw = C.string_at(ptr, n.value * THRESHOLD_DTYPE.itemsize)
        return np.frombuffer(raw, THRESHOLD_DTYPE).copy()

    # ---- differentiable rollouts ----
    def fit_pair_budget(self, headroom: float = 1.5) -> int:
        """Shrinks the pair budget to the live pairs x headroom (history kept)."""
        out = C.c_uint32()
        self._check(lib().fyzz_b200_fit_pair_budget(self.h, headroom, C.byref(out)))
        return out.value

    def set_descriptor_order(self, pairs, joint_ids=None):
        """Gauss-Seidel order of the next step: touching-manager shape pairs
        (n, 2) in order, joint constraint ids in order."""
        p = np.ascontiguousarray(np.asarray(pairs, np.uint32).reshape(-1, 2))
        j = np.ascontiguousarray(np.zeros(0, np.uint64) if joint_ids is None else np.asarray(joint_ids, np.uint64))
        self._check(lib().fyzz_b200_set_descriptor_order(self.h, _p(p), p.shape[0], _p(j), j.size))

    def set_tuning(self, **params):
        """Performance parameters (fyzz_b200_tuning_t fields); unnamed ones
        keep their current values.  Results are unchanged by any setting."""
        t = self.tuning()
        for k, v in params.items():
            t[k] = int(v)
        self._check(lib().fyzz_b200_set_tuning(self.h, C.byref(Tuning(**t))))

    def tuning(self) -> dict:
        t = Tuning()
        self._check(lib().fyzz_b200_get_tuning(self.h, C.byref(t)))
        return t.as_dict()

    def set_pair_budget(self, pairs: int) -> int:
        """Sets the pair budget (at least the live pairs; history kept)."""
        out = C.c_uint32()
        self._check(lib().fyzz_b200_set_pair_budget(self.h, pairs, C.byref(out)))
        return out.value

    def test_scan(self, n: int, skip_first_tile: bool = False):
        """Test hook of the step's look-back scan: (error bits, mismatches).
        Raises LogicError when the scan's bounded wait gave up."""
        bits, bad = C.c_uint32(), C.c_uint64()
        rc = lib().fyzz_b200_test_scan(self.h, n, 1 if skip_first_tile else 0, C.byref(bits), C.byref(bad))
        self.last_scan = (bits.value, bad.value)
        self._check(rc)
        return bits.value, bad.value

    def rollout_begin(self, steps: int, checkpoint_every: int):
        self._check(lib().fyzz_b200_rollout_begin(self.h, steps, checkpoint_every))

    def rollout_rewind(self):
        """Back to the state the last rollout_forward started from."""
        self._check(lib().fyzz_b200_rollout_rewind(self.h))

    def rollout_forward(self, seconds: float = 1.0 / 120.0):
        self._check(lib().fyzz_b200_rollout_forward(self.h, seconds))

    def rollout_backward(self, grad_center, grad_orientation=None, grad_velocity=None, grad_angular=None):
        """Gradients of a loss on the final state with respect to the initial
        velocities, body masses and shape friction coefficients."""
        nb, ns = self.counts()["bodies"], self.counts()["shapes"]

        def arr(x, k):
            return None if x is None else np.ascontiguousarray(np.asarray(x, np.float32).reshape(nb, k))
        gc, gq, gv, gw = arr(grad_center, 3), arr(grad_orientation, 4), arr(grad_velocity, 3), arr(grad_angular, 3)
        out = {"v0": np.zeros((nb, 3), np.float32), "w0": np.zeros((nb, 3), np.float32),
               "mass": np.zeros(nb, np.float32), "static_friction": np.zeros(ns, np.float32),
               "dynamic_friction": np.zeros(ns, np.float32)}
        self._check(lib().fyzz_b200_rollout_backward(
            self.h, _p(gc), _p(gq), _p(gv), _p(gw), _p(out["v0"]), _p(out["w0"]), _p(out["mass"]),
            _p(out["static_friction"]), _p(out["dynamic_friction"])))
        return out

    def friction_anchors(self):
        """Per touching manager (pair order): anchor word (count in bits 0-7,
        bit 10 + k: anchor k taken from this step's contact point, whose
        index is in bits 12 + 2k..13 + 2k) and the anchors in the shape0 /
        shape1 bodies' mass frames, (n, 2, 3) each."""
        n = lib().fyzz_b200_read_friction_anchors(self.h, None, None, None, 0)
        cnt = np.zeros(n, np.uint32)
        a0 = np.zeros((n, 2, 3), np.float32)
        a1 = np.zeros((n, 2, 3), np.float32)
        lib().fyzz_b200_read_friction_anchors(self.h, _p(cnt), _p(a0), _p(a1), n)
        return cnt, a0, a1

    def read_mass_frames(self):
        nb = self.counts()["bodies"]
        c = np.zeros((nb, 3), np.float32)
        q = np.zeros((nb, 4), np.float32)
        self._check(lib().fyzz_b200_read_mass_frames(self.h, _p(c), _p(q)))
        return c, q

    def step_counters(self) -> dict:
        """Device counters of the last step (see fyzz_b200_read_step_counters)."""
        out = np.zeros(18, np.uint32)
        self._check(lib().fyzz_b200_read_step_counters(self.h, _p(out), 18))
        return {"managers": int(out[0]), "descriptors": int(out[1]), "gjk_pairs": int(out[5]),
                "convex_pairs": int(out[16]), "convex_regenerated": int(out[17]),
                "islands_32_512": int(out[8]), "islands_96_512": int(out[9]),
                "islands_512_4096": int(out[10]), "islands_4096_up": int(out[11])}

    def error_bits(self) -> int:
        out = C.c_uint32()
        lib().fyzz_b200_error_bits(self.h, C.byref(out))
        return out.value


class ConvexMesh:
    """fyzz::cook_convex_mesh (reference include/fyzzxyzzy/convex.h:56-60):
    a cooked, reference-counted convex hull.  Host code only; usable
    without a GPU.  Raises ValueError for meshes the reference rejects."""

    def __init__(self, vertices, triangles):
        v = np.ascontiguousarray(vertices, np.float32).reshape(-1, 3)
        t = np.ascontiguousarray(triangles, np.uint32).reshape(-1, 3)
        h = C.c_void_p()
        rc = lib().fyzz_b200_cook_convex_mesh(_p(v), v.shape[0], _p(t), t.shape[0], C.byref(h))
        if rc:
            raise (ValueError if rc == 1 else RuntimeError)(lib().fyzz_b200_cook_error().decode())
        self.h = h.value

    def __del__(self):
        if getattr(self, "h", None):
            lib().fyzz_b200_convex_mesh_release(self.h)
            self.h = None

    def info(self) -> dict:
        """Faces (n, 6: normal, distance, first, count), face indices,
        volume, centre, inertia (3x3, columns), bounds lo / hi."""
        counts = np.zeros(3, np.uint32)
        self._info(counts, None, None, None, None)
        faces = np.zeros((counts[1], 6), np.float32)
        idx = np.zeros(counts[2], np.uint32)
        vol = np.zeros(1, np.float64)
        m = np.zeros(18, np.float32)
        self._info(counts, faces, idx, vol, m)
        return {"faces": faces, "idx": idx, "volume": float(vol[0]), "center": m[0:3],
                "inertia": m[3:12].reshape(3, 3).T.copy(), "lo": m[12:15], "hi": m[15:18]}

    def _info(self, counts, faces, idx, vol, m):
        rc = lib().fyzz_b200_convex_mesh_info(self.h, _p(counts), _p(faces), _p(idx), _p(vol), _p(m))
        if rc:
            raise RuntimeError("invalid convex mesh handle")
