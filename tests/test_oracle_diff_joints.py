"""The FP64 differentiable model's joint rows (oracle/diff_model.py) against
the C oracle's step, on the host.

The model is the checker of differentiable rollouts; these tests pin its
restatement of the joint families (anchored distance, fixed, spherical,
revolute, prismatic: scene.cpp:7615-7767 rows, 8895-8945 PGS) to the
oracle, which is itself bit-exact against the reference for every kind:
chains of spheres joined by one kind, moving in free flight, one step from
identical state, the model's velocities against the oracle's float32 ones;
and the model's autograd gradient of a velocity loss against its own
central differences.  The joints' frames start a few millimetres and
milliradians apart and their anchors off the line of the centres, so
every row's error and arm are well above float32 rounding.

Tolerance: velocities within 1e-4 of the joints' velocity change (the
float32 oracle and the float64 model part by rounding in the Gauss-Seidel
chains); gradients within 1e-6 of central differences (eps 1e-6, float64).
"""
import numpy as np
import pytest
import torch

DT = 1.0 / 120.0


def rot(q, v):
    u = q[:3]
    t = 2.0 * np.cross(u, v)
    return v + q[3] * t + np.cross(u, t)


def qmul(a, b):
    return np.array([a[3] * b[0] + b[3] * a[0] + a[1] * b[2] - a[2] * b[1],
                     a[3] * b[1] + b[3] * a[1] + a[2] * b[0] - a[0] * b[2],
                     a[3] * b[2] + b[3] * a[2] + a[0] * b[1] - a[1] * b[0],
                     a[3] * b[3] - a[0] * b[0] - a[1] * b[1] - a[2] * b[2]])


def chains(scenes, kind, n_chains=4, links=4, seed=0):
    """Chains of spheres (radius 0.1, 0.6 m apart) high above the floor,
    joined by `kind` with random joint frames, random velocities."""
    rng = np.random.Generator(np.random.PCG64(seed + 10 * kind))
    pos, quat, vel, ang, shapes, joints, dist, jl = [], [], [], [], [], [], [], []
    for c in range(n_chains):
        origin = np.array([3.0 * c, 6.0, 0.0])
        direction = rng.normal(size=3)
        direction /= np.linalg.norm(direction)
        first = len(pos)
        for k in range(links):
            pos.append(origin + direction * 0.6 * k)
            quat.append(scenes.random_quaternions(rng, 1)[0].astype(np.float64))
            vel.append(rng.normal(0.0, 0.5, 3))
            ang.append(rng.normal(0.0, 0.5, 3))
            shapes.append([scenes._sphere(0.1)])
        for k in range(1, links):
            a, b = first + k - 1, first + k
            mid = 0.5 * (pos[a] + pos[b])
            # Frames a few millimetres and milliradians apart, so every row
            # carries an error well above float32 rounding; the anchored
            # distance joint's anchors 0.2 m apart (a distance row's axis
            # is undefined while its anchors coincide), rest length 2 mm
            # off their distance.
            gap = 0.1 * direction if kind == 1 else np.zeros(3)
            # off the line of the centres, so the anchors' arms are not
            # parallel to the chain (the angular rows are well conditioned)
            side = np.cross(direction, rng.normal(size=3))
            mid = mid + 0.08 * side / np.linalg.norm(side)
            qj = scenes.random_quaternions(rng, 1)[0].astype(np.float64)
            tilt = rng.normal(0.0, 2e-3, 3)
            qt = np.concatenate([0.5 * tilt, [1.0]])
            qt /= np.linalg.norm(qt)
            shift = rng.normal(0.0, 2e-3, 3) if kind != 1 else np.zeros(3)
            ca = quat[a] * np.array([-1, -1, -1, 1])
            cb = quat[b] * np.array([-1, -1, -1, 1])
            la = np.concatenate([rot(ca, mid - gap - pos[a]), qmul(ca, qj)])
            lb = np.concatenate([rot(cb, mid + gap + shift - pos[b]), qmul(cb, qmul(qt, qj))])
            joints.append((a, b))
            dist.append(0.2 + 2e-3 if kind == 1 else 0.05)
            jl.append(np.concatenate([la, lb]))
    n = len(pos)
    mats = np.tile(np.array([0.5, 0.5, 0.0], np.float32), (n, 1))
    spec = scenes._assemble(np.asarray(pos, np.float32), np.asarray(quat, np.float32),
                            np.asarray(vel, np.float32), np.asarray(ang, np.float32), 700.0, shapes, mats,
                            joints=np.asarray(joints, np.uint32).reshape(-1, 2),
                            joint_dist=np.asarray(dist, np.float32))
    spec.joint_kind = np.full(len(joints), kind, np.uint32)
    spec.joint_local = np.asarray(jl, np.float32).reshape(-1, 14)
    return spec


def model_and_state(diff_model, oracle, spec):
    o = oracle.OracleScene(spec)
    mp = o.mass_props().astype(np.float64)
    st = o.body_states().astype(np.float64)
    na = st.shape[0]
    dyn = np.zeros(na, bool)
    dyn[1:] = True
    u = np.zeros((na, 3))
    c0, q0 = np.zeros((na, 3)), np.zeros((na, 4))
    for i in range(na):
        qb = st[i, 6:10]
        mlp, mlq = mp[i, 4:7], mp[i, 7:11]
        qm = qmul(qb, mlq)
        u[i] = rot(mlq * np.array([-1, -1, -1, 1]), mlp)
        c0[i] = st[i, 0:3] + rot(qb, mlp)
        q0[i] = qm
    shape_body = np.concatenate([[0], np.asarray(spec.shape_body, np.int64) + 1])
    model = diff_model.Model(dyn, mp[:, 0], mp[:, 1:4], u, shape_body, np.zeros(len(shape_body)),
                             np.zeros(len(shape_body)), diff_model.spec_joints(spec), mass_local_q=mp[:, 7:11])
    return o, model, st, c0, q0, mp


ROWS = {0: 1, 1: 1, 2: 6, 3: 3, 4: 5, 5: 5}


def oracle_levels(o, spec):
    """Partition of every descriptor (joints in canonical order, then
    managers).  The oracle lists a joint by its first row and row count."""
    kinds = spec.joint_kinds()[::-1]               # canonical: slot descending
    first_row = np.concatenate([[0], np.cumsum([ROWS[int(k)] for k in kinds])])
    joint_of_row = {int(r): j for j, r in enumerate(first_row[:-1])}
    n_joints = len(kinds)
    desc, ends = o.partitions()
    levels = np.zeros(n_joints + o.counts()["manifolds"], np.uint32)
    start = 0
    for p, e in enumerate(ends):
        for d in desc[start:int(e)]:
            levels[joint_of_row[int(d[0])] if d[3] else n_joints + int(d[0])] = p
        start = int(e)
    return levels


def run_model(diff_model, model, rec, c0, q0, v0, w0, mp):
    t = diff_model._t
    nb = len(model.dyn)
    c = [t(c0[i]) for i in range(nb)]
    q = [t(q0[i]) for i in range(nb)]
    v = [v0[i] for i in range(nb)]
    w = [w0[i] for i in range(nb)]
    im = [t(mp[i, 0]) for i in range(nb)]
    iI = [t(mp[i, 1:4]) for i in range(nb)]
    zero = torch.zeros(len(model.shape_body), dtype=torch.float64)
    return model.step(rec, DT, c, q, v, w, im, iI, zero, zero)


def empty_record(diff_model, levels, c0, q0):
    return diff_model.StepRecord(c0, q0, np.zeros((0, 2), np.uint32), np.zeros(0, np.uint32),
                                 np.zeros((0, 4, 7), np.float32), np.zeros(0, np.uint32),
                                 np.zeros((0, 2, 3)), np.zeros((0, 2, 3)), levels)


@pytest.mark.parametrize("kind", [1, 2, 3, 4, 5], ids=["anchored", "fixed", "spherical", "revolute", "prismatic"])
def test_model_joint_step_matches_oracle(oracle, scenes, kind):
    import diff_model
    spec = chains(scenes, kind)
    o, model, st, c0, q0, mp = model_and_state(diff_model, oracle, spec)
    o.step(DT)
    assert o.counts()["manifolds"] == 0          # free flight: joints only
    st1 = o.body_states().astype(np.float64)
    rec = empty_record(diff_model, oracle_levels(o, spec), c0, q0)
    t = diff_model._t
    v0 = [t(st[i, 3:6]) for i in range(st.shape[0])]
    w0 = [t(st[i, 10:13]) for i in range(st.shape[0])]
    _, _, nv, nw = run_model(diff_model, model, rec, c0, q0, v0, w0, mp)
    got = np.concatenate([np.stack([x.detach().numpy() for x in nv])[1:],
                          np.stack([x.detach().numpy() for x in nw])[1:]], 1)
    want = np.concatenate([st1[1:, 3:6], st1[1:, 10:13]], 1)
    # the joints' velocity change (against free flight) sets the scale: the
    # float32 oracle and the float64 model part by rounding in the
    # Gauss-Seidel chains of the corrections
    free = np.concatenate([st[1:, 3:6] + np.array([0.0, -9.81 * DT, 0.0]), st[1:, 10:13]], 1)
    scale = np.max(np.abs(want - free))
    assert scale > 0.1
    err = np.max(np.abs(got - want)) / scale
    assert err < 1e-4, err


@pytest.mark.parametrize("kind", [2, 4, 5], ids=["fixed", "revolute", "prismatic"])
def test_model_joint_gradient_matches_central_differences(oracle, scenes, kind):
    import diff_model
    spec = chains(scenes, kind, n_chains=2, links=3)
    o, model, st, c0, q0, mp = model_and_state(diff_model, oracle, spec)
    o.step(DT)
    rec = empty_record(diff_model, oracle_levels(o, spec), c0, q0)
    t = diff_model._t
    nb = st.shape[0]
    target = torch.linspace(-1.0, 1.0, 3 * (nb - 1), dtype=torch.float64).reshape(nb - 1, 3)

    def loss(v0_flat):
        v0 = [t(st[0, 3:6])] + [v0_flat[3 * (i - 1):3 * i] for i in range(1, nb)]
        w0 = [t(st[i, 10:13]) for i in range(nb)]
        _, _, nv, nw = run_model(diff_model, model, rec, c0, q0, v0, w0, mp)
        v = torch.stack(nv[1:])
        w = torch.stack(nw[1:])
        return ((v - target) ** 2).sum() + (w ** 2).sum()

    x = torch.tensor(st[1:, 3:6].reshape(-1), dtype=torch.float64, requires_grad=True)
    l = loss(x)
    (g,) = torch.autograd.grad(l, x)
    eps = 1e-6
    fd = np.zeros(x.shape[0])
    for i in range(x.shape[0]):
        e = torch.zeros_like(x)
        e[i] = eps
        fd[i] = (loss(x.detach() + e).item() - loss(x.detach() - e).item()) / (2 * eps)
    err = np.max(np.abs(g.numpy() - fd) / np.maximum(np.abs(fd), 1e-3))
    assert err < 1e-6, err
