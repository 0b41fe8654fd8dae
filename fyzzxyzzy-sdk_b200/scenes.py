"""Seeded synthetic rigid-body workloads.

Every workload is produced on the host from a numpy ``Generator(PCG64(seed))``
and fed identically to the B200 world and to the NativeCpu reference.  The
record layout is the one both C ABIs consume:

* ``bodies``   (nb, 14) float32: position(3) orientation xyzw(4) linear
  velocity(3) angular velocity(3) density(1)
* ``shape_body`` (ns,) uint32: owning dynamic-body index (grouped, ascending)
* ``shape_type`` (ns,) uint32: 0 = box, 1 = sphere, 3 = cooked convex hull
* ``shape_geom`` (ns, 4) float32: half extents (box), radius (sphere) or the
  index into ``convex_meshes`` (hull)
* ``shape_local`` (ns, 7) float32: shape pose in the body frame
* ``shape_mat``  (ns, 3) float32: static friction, dynamic friction, restitution
* ``joints`` (nj, 2) uint32 and ``joint_dist`` (nj,) float32: centre-anchored
  distance constraints (``World::add_center_distance_constraint``)
* ``convex_meshes``: list of (vertices (nv, 3) float32, outward triangles
  (nt, 3) uint32) for ``cook_convex_mesh`` / ``World::attach_convex_shape``
* ``floor``: static floor height or ``None``.  When present the floor is the
  first actor (BodyId 0, ShapeId 0), so dynamic body ``i`` is BodyId ``i+1``;
  ``floor_mat`` is its (static friction, dynamic friction, restitution).

The workloads follow the five benchmark configurations of the rigid-body step
(plain single scene, plain at scale, batched forward, differentiable rollout,
batched differentiable at scale); sizes are parameters so tests can run the
same distributions small.
"""
from __future__ import annotations

from dataclasses import dataclass, field
import numpy as np

BOX, SPHERE, CONVEX = 0, 1, 3
# Joint kinds: World::add_center_distance_constraint, add_anchored_distance_
# constraint, add_fixed / spherical / revolute / prismatic_constraint.
JOINT_CENTER, JOINT_ANCHORED, JOINT_FIXED, JOINT_SPHERICAL, JOINT_REVOLUTE, JOINT_PRISMATIC = range(6)
FLOOR_BODY = 0xFFFFFFFF


@dataclass
class SceneSpec:
    bodies: np.ndarray
    shape_body: np.ndarray
    shape_type: np.ndarray
    shape_geom: np.ndarray
    shape_local: np.ndarray
    shape_mat: np.ndarray
    joints: np.ndarray = field(default_factory=lambda: np.zeros((0, 2), np.uint32))
    joint_dist: np.ndarray = field(default_factory=lambda: np.zeros((0,), np.float32))
    # Per joint: kind (JOINT_* below; default center distance) and the local
    # frames of its two bodies (position 3 + quaternion xyzw 4 each).  A
    # joint endpoint of FLOOR_BODY is the scene's static floor.
    joint_kind: np.ndarray | None = None
    joint_local: np.ndarray | None = None
    floor: float | None = 0.0
    floor_mat: tuple = (0.5, 0.5, 0.0)
    convex_meshes: list = field(default_factory=list)

    @property
    def n_bodies(self) -> int:
        return int(self.bodies.shape[0])

    @property
    def n_shapes(self) -> int:
        return int(self.shape_body.shape[0])

    @property
    def n_actors(self) -> int:
        return self.n_bodies + (1 if self.floor is not None else 0)

    def joint_kinds(self) -> np.ndarray:
        n = self.joints.shape[0]
        return np.zeros(n, np.uint32) if self.joint_kind is None else np.asarray(self.joint_kind, np.uint32)

    def joint_locals(self) -> np.ndarray:
        n = self.joints.shape[0]
        if self.joint_local is not None:
            return np.ascontiguousarray(self.joint_local, np.float32).reshape(n, 14)
        out = np.zeros((n, 14), np.float32)
        out[:, 6] = out[:, 13] = 1.0
        return out

    def has_joint_kinds(self) -> bool:
        """True when some joint is not a plain center distance joint."""
        return bool(self.joints.shape[0]) and (bool(np.any(self.joint_kinds() != JOINT_CENTER)) or
                                               bool(np.any(self.joints == FLOOR_BODY)))

    def mesh_arrays(self):
        """Meshes concatenated for the C ABIs: (vertex counts, vertices,
        triangle counts, triangles), indices local to each mesh."""
        nv = np.asarray([m[0].shape[0] for m in self.convex_meshes], np.uint32)
        nt = np.asarray([m[1].shape[0] for m in self.convex_meshes], np.uint32)
        v = np.ascontiguousarray(np.concatenate([np.asarray(m[0], np.float32).reshape(-1, 3)
                                                 for m in self.convex_meshes]) if self.convex_meshes
                                 else np.zeros((0, 3), np.float32))
        t = np.ascontiguousarray(np.concatenate([np.asarray(m[1], np.uint32).reshape(-1, 3)
                                                 for m in self.convex_meshes]) if self.convex_meshes
                                 else np.zeros((0, 3), np.uint32))
        return nv, v, nt, t

    def validate(self) -> "SceneSpec":
        assert self.bodies.dtype == np.float32 and self.bodies.shape[1] == 14
        assert self.shape_body.dtype == np.uint32
        assert np.all(np.diff(self.shape_body.astype(np.int64)) >= 0)
        assert self.shape_geom.shape == (self.n_shapes, 4)
        assert self.shape_local.shape == (self.n_shapes, 7)
        assert self.shape_mat.shape == (self.n_shapes, 3)
        return self


IDENTITY = np.array([0, 0, 0, 0, 0, 0, 1], np.float32)


def random_quaternions(rng: np.random.Generator, n: int) -> np.ndarray:
    """Uniform unit quaternions: normalised 4-vectors of i.i.d. N(0,1)."""
    q = rng.standard_normal((n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    return q.astype(np.float32)


def _assemble(pos, quat, vel, ang, density, shapes, mat_per_body, joints=None,
              joint_dist=None, floor=0.0) -> SceneSpec:
    """shapes: list per body of (type, geom4, local7)."""
    nb = pos.shape[0]
    bodies = np.zeros((nb, 14), np.float32)
    bodies[:, 0:3] = pos
    bodies[:, 3:7] = quat
    bodies[:, 7:10] = vel
    bodies[:, 10:13] = ang
    bodies[:, 13] = density
    sb, st, sg, sl, sm = [], [], [], [], []
    for b, lst in enumerate(shapes):
        for (t, g, l) in lst:
            sb.append(b); st.append(t); sg.append(g); sl.append(l)
            sm.append(mat_per_body[b])
    spec = SceneSpec(
        bodies=bodies,
        shape_body=np.asarray(sb, np.uint32),
        shape_type=np.asarray(st, np.uint32),
        shape_geom=np.asarray(sg, np.float32).reshape(-1, 4),
        shape_local=np.asarray(sl, np.float32).reshape(-1, 7),
        shape_mat=np.asarray(sm, np.float32).reshape(-1, 3),
        joints=np.zeros((0, 2), np.uint32) if joints is None else np.asarray(joints, np.uint32).reshape(-1, 2),
        joint_dist=np.zeros((0,), np.float32) if joint_dist is None else np.asarray(joint_dist, np.float32),
        floor=floor,
    )
    return spec.validate()


def _box(h):
    return (BOX, np.array([h[0], h[1], h[2], 0.0], np.float32), IDENTITY)


def _sphere(r, local=IDENTITY):
    return (SPHERE, np.array([r, 0.0, 0.0, 0.0], np.float32), local)


def random_boxes(n: int = 1000, seed: int = 0, half=(0.1, 0.5), xz=10.0,
                 y=(1.0, 21.0), density=1000.0, friction=0.5) -> SceneSpec:
    """Plain single scene: n random dynamic boxes above a floor at y=0
    (half extents U[0.1,0.5] per axis, centres x,z in U[-10,10], y in U[1,21],
    random orientations, zero velocity, density 1000, friction 0.5,
    restitution 0)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    h = rng.uniform(half[0], half[1], (n, 3)).astype(np.float32)
    pos = np.stack([rng.uniform(-xz, xz, n), rng.uniform(y[0], y[1], n),
                    rng.uniform(-xz, xz, n)], 1).astype(np.float32)
    quat = random_quaternions(rng, n)
    z = np.zeros((n, 3), np.float32)
    mats = np.tile(np.array([friction, friction, 0.0], np.float32), (n, 1))
    return _assemble(pos, quat, z, z, density, [[_box(h[i])] for i in range(n)], mats)


def mixed_scale(n: int = 131072, seed: int = 1, region=(200.0, 50.0, 200.0),
                frac_box=0.7, frac_sphere=0.2, joint_frac=0.02,
                size=(0.05, 0.3), density=1000.0) -> SceneSpec:
    """Plain method at scale: 70% boxes, 20% spheres, 10% box+sphere
    compounds (sphere at a local offset in a 0.5 m cube), random
    orientations, v0 ~ N(0,1) per axis, friction U[0.3,0.8] per body, and
    2% of bodies in pairs joined by distance constraints whose rest length is
    the initial separation.  Bodies fill a 200 x 50 x 200 m region above the
    floor."""
    rng = np.random.Generator(np.random.PCG64(seed))
    kind = rng.uniform(0, 1, n)
    pos = np.stack([rng.uniform(-region[0] / 2, region[0] / 2, n),
                    rng.uniform(1.0, 1.0 + region[1], n),
                    rng.uniform(-region[2] / 2, region[2] / 2, n)], 1)
    n_pairs = int(round(n * joint_frac / 2))
    perm = rng.permutation(n)[: 2 * n_pairs].reshape(-1, 2)
    # The partner of each constrained pair starts 0.8-1.5 m from its anchor.
    d = rng.standard_normal((n_pairs, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    d *= rng.uniform(0.8, 1.5, (n_pairs, 1))
    pos[perm[:, 1]] = pos[perm[:, 0]] + d
    pos = pos.astype(np.float32)
    quat = random_quaternions(rng, n)
    vel = rng.standard_normal((n, 3)).astype(np.float32)
    ang = np.zeros((n, 3), np.float32)
    mu = rng.uniform(0.3, 0.8, n).astype(np.float32)
    mats = np.stack([mu, mu, np.zeros(n, np.float32)], 1)
    shapes = []
    for i in range(n):
        if kind[i] < frac_box:
            shapes.append([_box(rng.uniform(size[0], size[1], 3))])
        elif kind[i] < frac_box + frac_sphere:
            shapes.append([_sphere(rng.uniform(size[0], size[1]))])
        else:
            off = rng.uniform(-0.25, 0.25, 3)
            local = np.array([off[0], off[1], off[2], 0, 0, 0, 1], np.float32)
            shapes.append([_box(rng.uniform(size[0], size[1], 3)),
                           _sphere(rng.uniform(size[0], size[1]), local)])
    dist = np.linalg.norm(pos[perm[:, 0]] - pos[perm[:, 1]], axis=1).astype(np.float32)
    return _assemble(pos, quat, vel, ang, density, shapes, mats,
                     joints=perm.astype(np.uint32), joint_dist=dist)


def box_stack_scene(n: int, seed: int, height_range=(5, 20), jitter=1.0e-3,
                    density=1000.0, friction=0.5) -> SceneSpec:
    """Towers of unit cubes 5-20 high, resting on the floor, with N(0, 1 mm)
    placement jitter; towers stand on a 2 m grid."""
    rng = np.random.Generator(np.random.PCG64(seed))
    hgt = int(rng.integers(height_range[0], height_range[1] + 1))
    towers = (n + hgt - 1) // hgt
    side = int(np.ceil(np.sqrt(towers)))
    pos = np.zeros((n, 3), np.float32)
    for i in range(n):
        t, k = divmod(i, hgt)
        gx, gz = divmod(t, side)
        pos[i] = (2.0 * gx, 0.5 + 1.0 * k, 2.0 * gz)
    pos += rng.normal(0.0, jitter, (n, 3)).astype(np.float32)
    pos[:, 1] = np.maximum(pos[:, 1], 0.5)
    quat = np.tile(np.array([0, 0, 0, 1], np.float32), (n, 1))
    z = np.zeros((n, 3), np.float32)
    mats = np.tile(np.array([friction, friction, 0.0], np.float32), (n, 1))
    return _assemble(pos, quat, z, z, density,
                     [[_box((0.5, 0.5, 0.5))] for _ in range(n)], mats)


def cube_block(nx: int, ny: int, nz: int, half: float = 0.25, jitter: float = 1.0e-4, seed: int = 0,
               density: float = 1000.0, friction: float = 0.5) -> SceneSpec:
    """One block of nx x ny x nz touching cubes (half extent `half`) resting
    on the floor, with N(0, jitter) placement noise: every cube touches its
    neighbours, so the block is a single island with several contact
    managers per cube."""
    rng = np.random.Generator(np.random.PCG64(seed))
    g = np.stack(np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij"), -1).reshape(-1, 3)
    pos = (g * (2.0 * half) + np.array([-(nx - 1) * half, half, -(nz - 1) * half])).astype(np.float32)
    pos += rng.normal(0.0, jitter, pos.shape).astype(np.float32)
    pos[:, 1] = np.maximum(pos[:, 1], half)
    n = pos.shape[0]
    quat = np.tile(np.array([0, 0, 0, 1], np.float32), (n, 1))
    z = np.zeros((n, 3), np.float32)
    mats = np.tile(np.array([friction, friction, 0.0], np.float32), (n, 1))
    return _assemble(pos, quat, z, z, density, [[_box((half, half, half))] for _ in range(n)], mats)


def with_state(spec: SceneSpec, states: np.ndarray) -> SceneSpec:
    """A copy of `spec` whose dynamic bodies start from `states`: per actor
    (the floor first when the scene has one) the 14-float records of
    World.read_bodies / the reference's body states (position 3, linear
    velocity 3, orientation xyzw 4, angular velocity 3, sleeping 1).
    Shapes, materials, densities and joints are kept."""
    st = np.asarray(states, np.float32)
    first = 1 if spec.floor is not None else 0
    st = st[first: first + spec.n_bodies]
    bodies = spec.bodies.copy()
    bodies[:, 0:3] = st[:, 0:3]
    bodies[:, 3:7] = st[:, 6:10]
    bodies[:, 7:10] = st[:, 3:6]
    bodies[:, 10:13] = st[:, 10:13]
    out = SceneSpec(**{k: getattr(spec, k) for k in spec.__dataclass_fields__})
    out.bodies = bodies
    return out


def batched_scenes(n_scenes: int = 4096, low: int = 16, high: int = 512,
                   base_seed: int = 0) -> list[SceneSpec]:
    """Batched forward: per-scene body count log-uniform in [low, high];
    even scenes are random piles (the plain scene scaled so the region side
    grows as n^(1/3)), odd scenes are unit-cube stacks.  Scene i uses seed
    base_seed + i and its own floor."""
    out = []
    for s in range(n_scenes):
        rng = np.random.Generator(np.random.PCG64(base_seed + s))
        n = int(np.exp(rng.uniform(np.log(low), np.log(high + 1))))
        n = max(low, min(high, n))
        if s % 2 == 0:
            scale = (n / 1000.0) ** (1.0 / 3.0)
            out.append(random_boxes(n, seed=base_seed + s, xz=10.0 * scale,
                                    y=(1.0, 1.0 + 20.0 * scale)))
        else:
            out.append(box_stack_scene(n, seed=base_seed + s))
    return out


def loose_piles(n_scenes: int = 1024, n_boxes: int = 64, base_seed: int = 0) -> list[SceneSpec]:
    """Differentiable rollout scenes: 64 boxes (half extents U[0.1,0.3]) in a
    loose pile, v0 and w0 ~ N(0, 0.5), per-body mass log-uniform in [0.5, 5]
    kg (density = mass / volume), per-scene friction U[0.2, 1.0]."""
    out = []
    for s in range(n_scenes):
        rng = np.random.Generator(np.random.PCG64(base_seed + s))
        h = rng.uniform(0.1, 0.3, (n_boxes, 3)).astype(np.float32)
        side = 1.2
        pos = np.stack([rng.uniform(-side, side, n_boxes),
                        rng.uniform(0.4, 2.4, n_boxes),
                        rng.uniform(-side, side, n_boxes)], 1).astype(np.float32)
        quat = random_quaternions(rng, n_boxes)
        vel = rng.normal(0, 0.5, (n_boxes, 3)).astype(np.float32)
        ang = rng.normal(0, 0.5, (n_boxes, 3)).astype(np.float32)
        mass = np.exp(rng.uniform(np.log(0.5), np.log(5.0), n_boxes))
        dens = (mass / (8.0 * h.prod(1))).astype(np.float32)
        mu = np.float32(rng.uniform(0.2, 1.0))
        mats = np.tile(np.array([mu, mu, 0.0], np.float32), (n_boxes, 1))
        spec = _assemble(pos, quat, vel, ang, 1.0,
                         [[_box(h[i])] for i in range(n_boxes)], mats)
        spec.bodies[:, 13] = dens
        out.append(spec)
    return out


def mixed_batched(n_scenes: int = 16384, low: int = 8, high: int = 256,
                  base_seed: int = 0) -> list[SceneSpec]:
    """Batched and differentiable at scale: per-scene counts log-uniform in
    [8, 256]; 60% boxes, 25% spheres, 15% compounds, 5% distance pairs,
    friction U[0.2, 1.0]."""
    out = []
    for s in range(n_scenes):
        rng = np.random.Generator(np.random.PCG64(base_seed + s))
        n = int(np.exp(rng.uniform(np.log(low), np.log(high + 1))))
        n = max(low, min(high, n))
        scale = (n / 1000.0) ** (1.0 / 3.0)
        out.append(mixed_scale(n, seed=base_seed + s,
                               region=(20.0 * scale, 20.0 * scale, 20.0 * scale),
                               frac_box=0.6, frac_sphere=0.25, joint_frac=0.05,
                               size=(0.05, 0.3)))
    return out


def _qmul(a, b):
    ax, ay, az, aw = a
    bx, by, bz, bw = b
    return np.array([aw * bx + bw * ax + ay * bz - az * by, aw * by + bw * ay + az * bx - ax * bz,
                     aw * bz + bw * az + ax * by - ay * bx, aw * bw - ax * bx - ay * by - az * bz])


def _qrot(q, v):
    u = np.asarray(q[:3], np.float64)
    t = 2.0 * np.cross(u, v)
    return v + q[3] * t + np.cross(u, t)


def joint_mechanisms(n_chains: int = 24, seed: int = 0, links: int = 4, kinds=None, floor_every: int = 3,
                     spacing: float = 4.0, height: float = 2.5, density: float = 500.0,
                     speed: float = 1.0) -> SceneSpec:
    """Chains of boxes joined end to end by the joint kinds in `kinds`
    (cycled over the chains; default: every kind), at rest or moving with
    N(0, speed) velocities.  Each joint's two local frames coincide in the
    world at creation: the joint sits halfway between the linked boxes with
    a random orientation (the hinge / slider axis is its local X).  Every
    `floor_every`-th chain hangs its first box from the floor by a joint of
    the same kind."""
    rng = np.random.Generator(np.random.PCG64(seed))
    kinds = list(range(6)) if kinds is None else list(kinds)
    side = int(np.ceil(np.sqrt(n_chains)))
    pos, quat, vel, ang, shapes, joints, dist, jk, jl = [], [], [], [], [], [], [], [], []
    body = 0
    for c in range(n_chains):
        kind = kinds[c % len(kinds)]
        gx, gz = divmod(c, side)
        origin = np.array([spacing * gx, height, spacing * gz])
        direction = rng.normal(size=3)
        direction[1] = abs(direction[1]) * 0.3
        direction /= np.linalg.norm(direction)
        half = rng.uniform(0.1, 0.25, (links, 3))
        step = 2.0 * half[:, 0].max() + 0.1
        first = body
        for k in range(links):
            p = origin + direction * step * k
            q = random_quaternions(rng, 1)[0].astype(np.float64)
            pos.append(p); quat.append(q)
            vel.append(rng.normal(0.0, speed, 3)); ang.append(rng.normal(0.0, speed, 3))
            shapes.append([_box(half[k])])
            body += 1
        def frames(pa, qa, pb, qb, mid):
            qj = random_quaternions(rng, 1)[0].astype(np.float64)
            ca, cb = qa * np.array([-1, -1, -1, 1]), qb * np.array([-1, -1, -1, 1])
            la = np.concatenate([_qrot(ca, mid - pa), _qmul(ca, qj)])
            lb = np.concatenate([_qrot(cb, mid - pb), _qmul(cb, qj)])
            return np.concatenate([la, lb])
        def length(kind, pa, pb):
            # center distance: the centres' separation; anchored: a short rope
            return float(np.linalg.norm(pa - pb)) if kind == JOINT_CENTER else 0.05
        for k in range(1, links):
            a, b = first + k - 1, first + k
            joints.append((a, b)); dist.append(length(kind, pos[a], pos[b])); jk.append(kind)
            jl.append(frames(pos[a], quat[a], pos[b], quat[b], 0.5 * (pos[a] + pos[b])))
        if floor_every and c % floor_every == 0:
            # hung from the floor actor (at the origin: floor height 0)
            anchor = pos[first] - direction * step * 0.5
            floor_p, floor_q = np.zeros(3), np.array([0, 0, 0, 1.0])
            joints.append((FLOOR_BODY, first)); jk.append(kind)
            dist.append(float(np.linalg.norm(floor_p - pos[first])) if kind == JOINT_CENTER else 0.05)
            jl.append(frames(floor_p, floor_q, pos[first], quat[first], anchor))
    n = len(pos)
    mats = np.tile(np.array([0.5, 0.5, 0.0], np.float32), (n, 1))
    spec = _assemble(np.asarray(pos, np.float32), np.asarray(quat, np.float32), np.asarray(vel, np.float32),
                     np.asarray(ang, np.float32), density, shapes, mats,
                     joints=np.asarray(joints, np.uint32).reshape(-1, 2), joint_dist=np.asarray(dist, np.float32))
    spec.joint_kind = np.asarray(jk, np.uint32)
    spec.joint_local = np.asarray(jl, np.float32).reshape(-1, 14)
    return spec


def kinematic_platform(n: int = 12, seed: int = 0) -> SceneSpec:
    """A 3 x 0.2 x 3 m platform (body 0, to be made kinematic) at 0.6 m with
    n random boxes (half extents U[0.1,0.2]) dropped onto it from 1-3 m."""
    spec = random_boxes(n + 1, seed=seed, xz=0.8, y=(1.0, 3.0), half=(0.1, 0.2))
    spec.bodies[0, 0:3] = [0, 0.6, 0]
    spec.bodies[0, 3:7] = [0, 0, 0, 1]
    spec.shape_geom[0, :3] = [1.5, 0.1, 1.5]
    return spec


def platform_target(step: int, dt: float = 1.0 / 120.0) -> np.ndarray:
    """Target pose of the platform after `step`: drifting along x at 0.4 m/s,
    bobbing 0.2 m in y and turning about y at 0.3 rad/s."""
    t = (step + 1) * dt
    ang = 0.3 * t
    return np.array([0.4 * t, 0.6 + 0.2 * np.sin(2 * t), 0.0, 0.0, np.sin(ang / 2), 0.0, np.cos(ang / 2)],
                    np.float32)


# ---------------- cooked convex hulls ----------------
def _outward(verts: np.ndarray, tris: np.ndarray) -> np.ndarray:
    """Winds every triangle of a convex surface outward (about the vertex
    mean, which lies inside)."""
    c = verts.mean(0)
    t = np.asarray(tris, np.int64).copy()
    a, b, d = verts[t[:, 0]], verts[t[:, 1]], verts[t[:, 2]]
    flip = np.einsum("ij,ij->i", np.cross(b - a, d - a), a - c) < 0
    t[flip, 1], t[flip, 2] = t[flip, 2].copy(), t[flip, 1].copy()
    return t.astype(np.uint32)


def hull_prism(sides: int, radius: float, half_height: float, taper: float = 1.0, phase: float = 0.0):
    """An n-sided prism (taper 1) or frustum along y: two n-gon caps, each
    a triangle fan that cooks to one planar face, and quad sides."""
    ang = phase + 2 * np.pi * np.arange(sides) / sides
    bot = np.stack([radius * np.cos(ang), np.full(sides, -half_height), radius * np.sin(ang)], 1)
    top = np.stack([taper * radius * np.cos(ang), np.full(sides, half_height), taper * radius * np.sin(ang)], 1)
    v = np.concatenate([bot, top]).astype(np.float32)
    tris = [(0, i, i + 1) for i in range(1, sides - 1)]
    tris += [(sides, sides + i, sides + i + 1) for i in range(1, sides - 1)]
    for i in range(sides):
        j = (i + 1) % sides
        tris += [(i, j, sides + j), (i, sides + j, sides + i)]
    return v, _outward(v.astype(np.float64), np.asarray(tris))


def hull_bipyramid(sides: int, radius: float, half_height: float):
    """Two n-gon pyramids joined at their base (apexes on +-y)."""
    ang = 2 * np.pi * np.arange(sides) / sides
    ring = np.stack([radius * np.cos(ang), np.zeros(sides), radius * np.sin(ang)], 1)
    v = np.concatenate([ring, [[0, half_height, 0], [0, -half_height, 0]]]).astype(np.float32)
    tris = []
    for i in range(sides):
        j = (i + 1) % sides
        tris += [(i, j, sides), (i, j, sides + 1)]
    return v, _outward(v.astype(np.float64), np.asarray(tris))


def hull_box(h):
    """A box as a cooked hull: 8 vertices, 12 triangles, 6 quad faces."""
    v = np.array([[sx * h[0], sy * h[1], sz * h[2]] for sx in (-1, 1) for sy in (-1, 1) for sz in (-1, 1)],
                 np.float32)
    quads = [(0, 1, 3, 2), (4, 5, 7, 6), (0, 1, 5, 4), (2, 3, 7, 6), (0, 2, 6, 4), (1, 3, 7, 5)]
    tris = [t for a, b, c, d in quads for t in ((a, b, c), (a, c, d))]
    return v, _outward(v.astype(np.float64), np.asarray(tris))


def hull_random(rng: np.random.Generator, n_points: int, radii=(0.2, 0.2, 0.2)):
    """The convex hull of n points on an ellipsoid with the given radii
    (scipy's Quickhull; only hull vertices are kept)."""
    from scipy.spatial import ConvexHull
    p = rng.normal(size=(n_points, 3))
    p /= np.linalg.norm(p, axis=1, keepdims=True)
    p *= np.asarray(radii)
    h = ConvexHull(p)
    keep = np.asarray(h.vertices)
    remap = np.full(n_points, -1, np.int64)
    remap[keep] = np.arange(keep.size)
    v = p[keep].astype(np.float32)
    return v, _outward(v.astype(np.float64), remap[h.simplices])


def convex_pile(n: int = 48, seed: int = 0, xz: float = 2.0, y=(0.5, 4.0), frac_other: float = 0.25,
                size=(0.12, 0.3), density: float = 1000.0, friction: float = 0.5, offset_frac: float = 0.2,
                n_meshes: int = 6) -> SceneSpec:
    """Cooked hulls dropped onto the floor: a few shared meshes (prisms,
    frustums, bipyramids, a box-shaped hull and random ellipsoid hulls),
    some attached with an off-centre local pose, mixed with frac_other boxes
    and spheres."""
    rng = np.random.Generator(np.random.PCG64(seed))
    meshes = []
    for m in range(n_meshes):
        r = float(rng.uniform(*size))
        kind = m % 5
        if kind == 0:
            meshes.append(hull_prism(int(rng.integers(5, 9)), r, 0.6 * r))
        elif kind == 1:
            meshes.append(hull_prism(int(rng.integers(4, 7)), r, 0.7 * r, taper=0.55))
        elif kind == 2:
            meshes.append(hull_bipyramid(int(rng.integers(4, 7)), r, 0.9 * r))
        elif kind == 3:
            meshes.append(hull_box(rng.uniform(0.6, 1.0, 3) * r))
        else:
            meshes.append(hull_random(rng, int(rng.integers(12, 40)), rng.uniform(0.6, 1.0, 3) * r))
    pos = np.stack([rng.uniform(-xz, xz, n), rng.uniform(y[0], y[1], n), rng.uniform(-xz, xz, n)], 1)
    quat = random_quaternions(rng, n)
    z = np.zeros((n, 3), np.float32)
    mats = np.tile(np.array([friction, friction, 0.0], np.float32), (n, 1))
    shapes = []
    for i in range(n):
        u = rng.uniform()
        if u < frac_other / 2:
            shapes.append([_box(rng.uniform(*size, 3))])
        elif u < frac_other:
            shapes.append([_sphere(float(rng.uniform(*size)))])
        else:
            local = IDENTITY.copy()
            if rng.uniform() < offset_frac:
                local[:3] = rng.uniform(-0.05, 0.05, 3)
                local[3:] = random_quaternions(rng, 1)[0]
            shapes.append([(CONVEX, np.array([float(rng.integers(0, n_meshes)), 0, 0, 0], np.float32), local)])
    spec = _assemble(pos.astype(np.float32), quat, z, z, density, shapes, mats)
    spec.convex_meshes = meshes
    return spec
