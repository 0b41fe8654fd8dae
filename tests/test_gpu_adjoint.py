"""Differentiable rollouts (fyzz_b200_rollout_*) against an independent FP64
reference (oracle/diff_model.py: the same model in torch float64 with
autograd) and against central finite differences of the B200 forward.

Tolerances: gradients within 1e-3 (norm-relative, per parameter group) of
the FP64 reference; the model's own forward within 1e-4 m of the B200
trajectory; finite differences (eps 1e-3, short horizon so the contact
structure does not change) within 2e-2."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DT = 1.0 / 120.0


def slab_scene(scenes, n_side=10):
    """A dynamic 10 x 0.2 x 10 m slab carrying n_side^2 boxes: all boxes touch
    the slab, so the island holds more than 96 descriptors."""
    n = n_side * n_side
    nb = 1 + n
    bodies = np.zeros((nb, 14), np.float32)
    bodies[:, 6] = 1.0
    bodies[:, 13] = 500.0
    bodies[0, :3] = (0.0, 0.1, 0.0)
    geom = np.zeros((nb, 4), np.float32)
    geom[0, :3] = (5.0, 0.1, 5.0)
    for i in range(n):
        gx, gz = divmod(i, n_side)
        bodies[1 + i, :3] = (-4.5 + 0.95 * gx, 0.4, -4.5 + 0.95 * gz)
        geom[1 + i, :3] = (0.2, 0.2, 0.2)
    local = np.tile(np.array([0, 0, 0, 0, 0, 0, 1], np.float32), (nb, 1))
    mat = np.tile(np.array([0.6, 0.6, 0.0], np.float32), (nb, 1))
    return scenes.SceneSpec(bodies=bodies, shape_body=np.arange(nb, dtype=np.uint32),
                            shape_type=np.zeros(nb, np.uint32), shape_geom=geom, shape_local=local,
                            shape_mat=mat, floor=0.0, floor_mat=(0.6, 0.6, 0.0))


def settled_piles(pkg, scenes, n_scenes=2, n_boxes=10, settle=90, seed=3, dense=False):
    if dense:
        specs = [slab_scene(scenes)]
    else:
        specs = scenes.loose_piles(n_scenes, n_boxes, base_seed=seed)
    w = pkg.World(0)
    for s in specs:
        w.add_scene(s)
    w.step(DT, steps=settle)
    return w, specs


def set_velocities(w, v0, w0):
    w.write_velocities(np.ascontiguousarray(np.concatenate([v0, w0], 1), np.float32))


def initial_velocities(nb, dynamic, seed=1):
    rng = np.random.default_rng(seed)
    v0 = rng.normal(0, 0.5, (nb, 3)).astype(np.float32)
    w0 = rng.normal(0, 0.5, (nb, 3)).astype(np.float32)
    v0[~dynamic] = 0
    w0[~dynamic] = 0
    return v0, w0


def body_props(w):
    """Mass properties per body (zeros for the static floors)."""
    nb = w.counts()["bodies"]
    out = np.zeros((nb, 11), np.float64)
    out[:, 10] = 1.0
    for i in range(nb):
        try:
            out[i] = w.body_mass_properties(i)
        except RuntimeError:
            pass
    return out


def dynamic_mask(w):
    return body_props(w)[:, 0] > 0


def rel_norm(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-12))


def one_scene_model(dm, w, specs):
    """Model constants for a world of several scenes built from specs."""
    nb = w.counts()["bodies"]
    dyn = dynamic_mask(w)
    props = body_props(w)
    import torch
    u = np.zeros((nb, 3))
    for i in range(nb):
        u[i] = dm.rotinv(torch.as_tensor(props[i, 7:11]), torch.as_tensor(props[i, 4:7])).numpy()
    shape_body, rest = [], []
    first = 0
    for s in specs:
        shape_body.append([first])                       # floor shape
        rest.append([s.floor_mat[2]])
        shape_body.append(np.asarray(s.shape_body, np.int64) + first + 1)
        rest.append(np.asarray(s.shape_mat[:, 2], np.float64))
        first += s.n_actors
    shape_body = np.concatenate(shape_body)
    rest = np.concatenate(rest)
    return dm.Model(dyn, props[:, 0], props[:, 1:4], u, shape_body, rest, np.zeros(len(shape_body)), [])


def shape_friction(specs):
    fs, fd = [], []
    for s in specs:
        fs.append([s.floor_mat[0]]); fd.append([s.floor_mat[1]])
        fs.append(s.shape_mat[:, 0]); fd.append(s.shape_mat[:, 1])
    return np.concatenate(fs).astype(np.float64), np.concatenate(fd).astype(np.float64)


@pytest.mark.parametrize("steps,every,pile", [(12, 4, "small"), (16, 16, "small"), (10, 5, "dense")])
def test_gradients_match_fp64_model(pkg, scenes, steps, every, pile):
    import torch
    import diff_model as dm
    kw = {} if pile == "small" else dict(settle=30, dense=True)
    wa, specs = settled_piles(pkg, scenes, **kw)
    wb, _ = settled_piles(pkg, scenes, **kw)
    if pile == "dense":
        wa.step(DT)
        wb.step(DT)
        assert wa.step_counters()["islands_96_512"] > 0, "the dense pile must reach the CTA island class"
    nb = wa.counts()["bodies"]
    dyn = dynamic_mask(wa)
    v0, w0 = initial_velocities(nb, dyn)
    set_velocities(wa, v0, w0)
    set_velocities(wb, v0, w0)
    rng = np.random.default_rng(7)
    a = rng.normal(size=(nb, 3)) * dyn[:, None]
    b = rng.normal(size=(nb, 3)) * dyn[:, None]
    # B200 rollout and its adjoint
    wa.rollout_begin(steps, every)
    wa.rollout_forward(DT)
    cK, _ = wa.read_mass_frames()
    vK = wa.read_bodies()[:, 3:6]
    g = wa.rollout_backward(grad_center=a, grad_velocity=b)
    # FP64 model over the recorded structure of an identical world
    c0, q0 = wb.read_mass_frames()
    recs = dm.record(wb, steps, DT)
    model = one_scene_model(dm, wb, specs)
    props = body_props(wb)
    T = lambda x, grad=False: torch.tensor(np.asarray(x, np.float64), requires_grad=grad)
    v0t, w0t = T(v0, True), T(w0, True)
    mass = T(np.where(dyn, 1.0 / np.where(props[:, 0] > 0, props[:, 0], 1.0), 1.0), True)
    fs, fd = shape_friction(specs)
    mus, mud = T(fs, True), T(fd, True)
    c, q, v, w = model.rollout(recs, DT, T(c0), T(q0), v0t, w0t, mass, mus, mud)
    cm = torch.stack(c).detach().numpy()
    assert np.max(np.abs(cm - cK)[dyn]) < 1e-4, "model forward must follow the B200 trajectory"
    L = (torch.stack(c) * T(a)).sum() + (torch.stack(v) * T(b)).sum()
    L.backward()
    assert rel_norm(g["v0"][dyn], v0t.grad.numpy()[dyn]) <= 1e-3
    assert rel_norm(g["w0"][dyn], w0t.grad.numpy()[dyn]) <= 1e-3
    assert rel_norm(g["mass"][dyn], mass.grad.numpy()[dyn]) <= 1e-3
    # static friction only enters when it exceeds the dynamic one
    ref_mu = sum(x.grad.numpy() for x in (mus, mud) if x.grad is not None)
    assert rel_norm(g["static_friction"] + g["dynamic_friction"], ref_mu) <= 1e-3
    # the world is left at the end of the rollout
    np.testing.assert_array_equal(wa.read_mass_frames()[0], cK)


def sliding_box(scenes, density=1000.0, friction=0.5):
    bodies = np.zeros((1, 14), np.float32)
    bodies[0, :3] = (0.0, 0.25, 0.0)
    bodies[0, 6] = 1.0
    bodies[0, 13] = density
    return scenes.SceneSpec(bodies=bodies, shape_body=np.zeros(1, np.uint32),
                            shape_type=np.zeros(1, np.uint32),
                            shape_geom=np.array([[0.25, 0.25, 0.25, 0.0]], np.float32),
                            shape_local=np.array([[0, 0, 0, 0, 0, 0, 1]], np.float32),
                            shape_mat=np.array([[friction, friction, 0.0]], np.float32), floor=0.0,
                            floor_mat=(friction, friction, 0.0))


def jointed_pair(scenes, density=1000.0):
    bodies = np.zeros((2, 14), np.float32)
    bodies[:, 6] = 1.0
    bodies[0, :3] = (0.0, 5.0, 0.0)
    bodies[1, :3] = (0.8, 5.3, 0.1)
    bodies[:, 13] = density
    return scenes.SceneSpec(bodies=bodies, shape_body=np.arange(2, dtype=np.uint32),
                            shape_type=np.zeros(2, np.uint32),
                            shape_geom=np.array([[0.2, 0.1, 0.15, 0], [0.1, 0.2, 0.1, 0]], np.float32),
                            shape_local=np.tile(np.array([0, 0, 0, 0, 0, 0, 1], np.float32), (2, 1)),
                            shape_mat=np.tile(np.array([0.5, 0.5, 0.0], np.float32), (2, 1)),
                            joints=np.array([[0, 1]], np.uint32),
                            joint_dist=np.array([0.7], np.float32), floor=None)


def rollout_loss(pkg, spec, v0, w0, steps, weights, settle):
    w = pkg.World(0)
    w.add_scene(spec)
    w.step(DT, steps=settle)
    set_velocities(w, v0, w0)
    w.step(DT, steps=steps)
    c, _ = w.read_mass_frames()
    return float(np.sum(np.asarray(c, np.float64) * weights))


@pytest.mark.parametrize("case", ["sliding", "jointed"])
def test_gradients_match_finite_differences(pkg, scenes, case):
    # Smooth cases (no contact appears or vanishes, no stick/slip switch
    # inside the perturbation): central differences of the B200 forward.
    steps, eps = 8, 1e-3
    make = sliding_box if case == "sliding" else jointed_pair
    settle = 30 if case == "sliding" else 1
    spec = make(scenes)
    nb = spec.n_actors
    v0 = np.zeros((nb, 3), np.float32)
    w0 = np.zeros((nb, 3), np.float32)
    if case == "sliding":
        v0[1] = (1.5, 0.0, 0.4)                 # slides: friction at its dynamic bound
        weights = np.zeros((nb, 3)); weights[1] = (1.0, 0.3, 0.5)
    else:
        v0[:] = ((0.3, -0.2, 0.5), (-0.4, 0.1, 0.2))
        w0[:] = ((0.5, 0.2, -0.3), (0.1, -0.6, 0.2))
        weights = np.array([[1.0, 0.5, -0.7], [0.2, 1.0, 0.4]])
    w = pkg.World(0)
    w.add_scene(spec)
    w.step(DT, steps=settle)
    set_velocities(w, v0, w0)
    w.rollout_begin(steps, 4)
    w.rollout_forward(DT)
    g = w.rollout_backward(grad_center=weights)
    dyn = dynamic_mask(w)
    checked = 0
    for body in np.flatnonzero(dyn):
        for axis in range(3):
            dv = np.zeros((nb, 3), np.float32)
            dv[body, axis] = eps
            fd = (rollout_loss(pkg, spec, v0 + dv, w0, steps, weights, settle) -
                  rollout_loss(pkg, spec, v0 - dv, w0, steps, weights, settle)) / (2 * eps)
            assert abs(fd - g["v0"][body, axis]) <= 2e-2 * max(abs(fd), 1e-2), (body, axis, fd, g["v0"][body, axis])
            checked += 1
    # masses: density scales the mass of every body of the scene alike
    d = 1e-3
    hi, lo = make(scenes, density=1000.0 * (1 + d)), make(scenes, density=1000.0 * (1 - d))
    fd_m = (rollout_loss(pkg, hi, v0, w0, steps, weights, settle) -
            rollout_loss(pkg, lo, v0, w0, steps, weights, settle)) / (2 * d)
    props = body_props(w)
    mass = np.where(dyn, 1.0 / np.where(props[:, 0] > 0, props[:, 0], 1.0), 0.0)
    adj_m = float(np.sum(g["mass"] * mass))   # dL/dlog(density) = sum_i m_i dL/dm_i
    assert abs(fd_m - adj_m) <= 2e-2 * max(abs(fd_m), 1e-3), (fd_m, adj_m)
    if case == "sliding":
        # friction of the box and the floor (static = dynamic, combined as their mean)
        mu = 0.5
        fd_f = (rollout_loss(pkg, sliding_box(scenes, friction=mu + eps), v0, w0, steps, weights, settle) -
                rollout_loss(pkg, sliding_box(scenes, friction=mu - eps), v0, w0, steps, weights, settle)) / (2 * eps)
        adj_f = float(np.sum(g["static_friction"] + g["dynamic_friction"]))
        assert abs(fd_f - adj_f) <= 2e-2 * max(abs(fd_f), 1e-3), (fd_f, adj_f)
    assert checked == 3 * int(dyn.sum())


def test_rewind_reruns_the_same_rollout(pkg, scenes):
    # rollout_rewind restores the start state; a second rollout of the same
    # shape reuses the checkpoints, frames and captured segment graphs and
    # reproduces the first bit for bit
    spec = scenes.random_boxes(40, seed=6, xz=1.5, y=(0.3, 2.0))
    w = pkg.World(0)
    w.add_scene(spec)
    w.step(1.0 / 120.0, steps=30)
    w.fit_pair_budget(1.5)
    nb = w.counts()["bodies"]
    grad = np.zeros((nb, 3), np.float32)
    grad[1:, 1] = 1.0
    runs = []
    for _ in range(2):
        w.rollout_begin(24, 8)
        w.rollout_forward(1.0 / 120.0)
        c, _ = w.read_mass_frames()
        g = w.rollout_backward(grad_center=grad)
        runs.append((c, g["v0"], g["mass"]))
        w.rollout_rewind()
    for a, b in zip(runs[0], runs[1]):
        np.testing.assert_array_equal(a, b)
    assert np.abs(runs[0][1]).max() > 0


def sliding_hull(scenes, density=1000.0, friction=0.5):
    """The sliding box as a cooked hull (8 vertices, 6 quad faces), so its
    floor contacts come from the hull-vertex generator.  A face of exactly
    four vertices keeps the forward smooth: with more vertices on the
    resting face the four kept witnesses change with the tilt, and finite
    differences straddle those switches."""
    spec = sliding_box(scenes, density, friction)
    spec.shape_type[:] = scenes.CONVEX
    spec.shape_geom[0] = (0.0, 0.0, 0.0, 0.0)
    spec.convex_meshes = [scenes.hull_box((0.25, 0.25, 0.25))]
    return spec


def test_gradients_through_a_sliding_hull(pkg, scenes):
    # the adjoint moves hull contacts with the body like any other
    # persistent manifold
    steps, eps, settle = 8, 1e-3, 30
    spec = sliding_hull(scenes)
    nb = spec.n_actors
    v0 = np.zeros((nb, 3), np.float32)
    w0 = np.zeros((nb, 3), np.float32)
    v0[1] = (1.5, 0.0, 0.4)
    weights = np.zeros((nb, 3))
    weights[1] = (1.0, 0.3, 0.5)
    w = pkg.World(0)
    w.add_scene(spec)
    w.step(DT, steps=settle)
    assert w.counts()["points"] >= 4
    set_velocities(w, v0, w0)
    w.rollout_begin(steps, 4)
    w.rollout_forward(DT)
    g = w.rollout_backward(grad_center=weights)
    for axis in range(3):
        dv = np.zeros((nb, 3), np.float32)
        dv[1, axis] = eps
        fd = (rollout_loss(pkg, spec, v0 + dv, w0, steps, weights, settle) -
              rollout_loss(pkg, spec, v0 - dv, w0, steps, weights, settle)) / (2 * eps)
        assert abs(fd - g["v0"][1, axis]) <= 2e-2 * max(abs(fd), 1e-2), (axis, fd, g["v0"][1, axis])
    mu = 0.5
    fd_f = (rollout_loss(pkg, sliding_hull(scenes, friction=mu + eps), v0, w0, steps, weights, settle) -
            rollout_loss(pkg, sliding_hull(scenes, friction=mu - eps), v0, w0, steps, weights, settle)) / (2 * eps)
    adj_f = float(np.sum(g["static_friction"] + g["dynamic_friction"]))
    assert abs(fd_f - adj_f) <= 2e-2 * max(abs(fd_f), 1e-3), (fd_f, adj_f)
