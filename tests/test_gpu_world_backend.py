"""The drop-in at the C++ level: the reference SDK's own fyzz::World driven
over the B200 WorldBackend (fyzzxyzzy-sdk_b200/integration/
b200_world_backend.cpp) and over its NativeCpu backend, authored through the
same public World calls (tests/world_backend_check.cpp, built with the
reference sources into oracle/_ref/libfyzz_backend_check.so).

Both worlds start fresh from the same authored state.  Where every
island's Gauss-Seidel order is forced (each body touches the floor or one
partner) the two solve the same rows in the same order and the body
velocities match within the one-step tolerance (1e-4 relative).  In dense
piles the reference orders a fresh island's descriptors by the insertion
history of its island graph, the B200 step by pair key; both orders are
valid Gauss-Seidel sweeps, so there the check is the contact-event counts,
the poses within 1e-4 and the velocities within 1e-2."""
import ctypes as C
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "oracle", "_ref", "libfyzz_backend_check.so")
DT = 1.0 / 120.0


def rel_err(a, b, floor=1e-3):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), floor))) if a.size else 0.0


@pytest.fixture(scope="module")
def check(pkg):
    if not os.path.exists(LIB):
        pytest.skip("backend check library not built (make -C oracle backend)")
    pkg.lib()
    L = C.CDLL(LIB)
    vp = C.c_void_p
    L.fz_backend_compare.argtypes = [C.c_uint32, vp, C.c_uint32, vp, vp, vp, vp, vp, C.c_uint32, vp, vp, C.c_int,
                                     C.c_float, vp, C.c_float, C.c_uint32, vp, vp, vp, C.c_char_p, C.c_size_t]
    L.fz_backend_rejects.argtypes = [C.c_char_p, C.c_size_t]
    return L


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None and a.size else None


def compare(L, spec, steps=1):
    arrs = [np.ascontiguousarray(x) for x in (spec.bodies, spec.shape_body, spec.shape_type, spec.shape_geom,
                                               spec.shape_local, spec.shape_mat, spec.joints, spec.joint_dist)]
    fm = np.asarray(spec.floor_mat, np.float32)
    n = spec.n_actors
    a = np.zeros((n, 14), np.float32)
    b = np.zeros((n, 14), np.float32)
    ev = np.zeros(4, np.uint32)
    msg = C.create_string_buffer(512)
    rc = L.fz_backend_compare(spec.n_bodies, _p(arrs[0]), spec.n_shapes, _p(arrs[1]), _p(arrs[2]), _p(arrs[3]),
                              _p(arrs[4]), _p(arrs[5]), arrs[6].shape[0], _p(arrs[6]), _p(arrs[7]),
                              0 if spec.floor is None else 1, 0.0 if spec.floor is None else float(spec.floor),
                              _p(fm), DT, steps, _p(a), _p(b), _p(ev), msg, len(msg))
    assert rc == 0, msg.value.decode()
    return a, b, ev


def landed(oracle, spec, steps):
    # the state a pile reaches, from the oracle (the scene is then authored
    # fresh from it on both backends)
    o = oracle.OracleScene(spec)
    for _ in range(steps):
        o.step(DT)
    return o.body_states()


def test_forced_order_scene_matches(check, scenes):
    # mixed shapes resting on the floor, spread out: every island's order
    # is forced, so both backends run the same sweep
    spec = scenes.mixed_scale(300, seed=5, region=(40.0, 0.6, 40.0), joint_frac=0.0)
    spec.bodies[:, 1] = 0.32
    got, want, ev = compare(check, spec)
    assert ev[1] > 100
    assert ev[0] == ev[1] and ev[2] == ev[3]
    assert rel_err(got[:, 3:6], want[:, 3:6]) <= 1e-4
    assert rel_err(got[:, 10:13], want[:, 10:13]) <= 1e-4
    assert rel_err(got[:, 0:3], want[:, 0:3], floor=1.0) <= 1e-4


@pytest.mark.parametrize("which", ["config0_pile", "mixed_with_joints"])
def test_dense_pile_first_step(check, oracle, scenes, which):
    if which == "config0_pile":
        spec = scenes.random_boxes(1000, seed=0)
        start = scenes.with_state(spec, landed(oracle, spec, 240))
    else:
        spec = scenes.mixed_scale(400, seed=2, region=(6.0, 2.0, 6.0), joint_frac=0.05)
        start = scenes.with_state(spec, landed(oracle, spec, 60))
    got, want, ev = compare(check, start)
    assert ev[1] > 50, "the pile must touch"
    assert ev[0] == ev[1] and ev[2] == ev[3]
    assert rel_err(got[:, 0:3], want[:, 0:3], floor=1.0) <= 1e-4
    assert rel_err(got[:, 3:6], want[:, 3:6], floor=1e-2) <= 1e-2
    assert rel_err(got[:, 10:13], want[:, 10:13], floor=1e-2) <= 1e-2


def test_unsupported_members_are_rejected(check):
    msg = C.create_string_buffer(64)
    assert check.fz_backend_rejects(msg, len(msg)) == 4
