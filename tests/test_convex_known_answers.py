"""Known-answer checks of convex cooking (the analytic cases the reference's
own cooking test covers, tests/cooked_convex.cpp): volume, centre of mass
and density-one inertia of a right tetrahedron, a cube and a triangular
wedge from the closed-form integrals; planar polygon merging; and the
meshes cooking must reject.  Run on the product's cooking (host code of the
C ABI, no GPU needed) and on the oracle's restatement.
"""
import numpy as np
import pytest

TETRA_V = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], np.float32)
TETRA_T = np.array([[0, 2, 1], [0, 1, 3], [0, 3, 2], [1, 2, 3]], np.uint32)
CUBE_V = np.array([[x, y, z] for x in (-1, 1) for y in (-1, 1) for z in (-1, 1)], np.float32)
CUBE_T = np.array([[0, 1, 3], [0, 3, 2], [4, 6, 7], [4, 7, 5], [0, 4, 5], [0, 5, 1],
                   [2, 3, 7], [2, 7, 6], [0, 2, 6], [0, 6, 4], [1, 5, 7], [1, 7, 3]], np.uint32)
# right triangle legs 1, 1 in xy, extruded 2 along z
WEDGE_V = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 2], [1, 0, 2], [0, 1, 2]], np.float32)
WEDGE_T = np.array([[0, 2, 1], [3, 4, 5], [0, 1, 4], [0, 4, 3], [0, 3, 5], [0, 5, 2], [1, 2, 5], [1, 5, 4]],
                   np.uint32)
# pyramid over a pentagon in y = 0 with its apex at y = 1
PENTA_V = np.array([[-1, 0, -1], [-1, 0, 1], [0, 0, 1.5], [1, 0, 1], [1, 0, -1], [0, 1, 0]], np.float32)
PENTA_T = np.array([[0, 2, 1], [0, 3, 2], [0, 4, 3], [0, 1, 5], [1, 2, 5], [2, 3, 5], [3, 4, 5], [4, 0, 5]],
                   np.uint32)


@pytest.fixture(params=["product", "oracle"])
def cook(request, pkg, oracle):
    if request.param == "product":
        return lambda v, t: pkg.ConvexMesh(v, t).info()

    def via_oracle(v, t):
        return oracle.cook_convex(v, t)
    return via_oracle


def test_tetrahedron(cook):
    m = cook(TETRA_V, TETRA_T)
    assert abs(m["volume"] - 1.0 / 6.0) < 1e-8
    np.testing.assert_allclose(m["center"], [0.25, 0.25, 0.25], atol=1e-6)
    # about the centre: second moments 1/60 and 1/120 less V * c^2
    np.testing.assert_allclose(np.diag(m["inertia"]), [1 / 80] * 3, atol=1e-7)
    np.testing.assert_allclose([m["inertia"][0, 1], m["inertia"][0, 2], m["inertia"][1, 2]], [1 / 480] * 3,
                               atol=1e-7)
    assert m["faces"].shape[0] == 4
    # translated far from the origin: same volume and inertia, shifted centre
    t = cook(TETRA_V + np.float32([10000, -20000, 30000]), TETRA_T)
    assert abs(t["volume"] - m["volume"]) < 1e-8
    np.testing.assert_allclose(t["center"], [10000.25, -19999.75, 30000.25], atol=1e-3)
    assert abs(t["inertia"][0, 0] - m["inertia"][0, 0]) < 1e-7


def test_cube(cook):
    m = cook(CUBE_V, CUBE_T)
    assert abs(m["volume"] - 8.0) < 1e-7
    np.testing.assert_allclose(m["center"], 0, atol=1e-7)
    np.testing.assert_allclose(m["inertia"], np.eye(3) * 16 / 3, atol=1e-6)
    assert m["faces"].shape[0] == 6 and np.all(m["faces"][:, 5] == 4)   # quads, not triangles


def test_wedge(cook):
    m = cook(WEDGE_V, WEDGE_T)
    assert abs(m["volume"] - 1.0) < 1e-8
    np.testing.assert_allclose(m["center"], [1 / 3, 1 / 3, 1.0], atol=1e-6)
    np.testing.assert_allclose(np.diag(m["inertia"]), [7 / 18, 7 / 18, 1 / 9], atol=1e-6)
    assert abs(m["inertia"][0, 1] - 1 / 36) < 1e-6
    assert m["faces"].shape[0] == 5


def test_pentagon_merges(cook):
    m = cook(PENTA_V, PENTA_T)
    assert m["faces"].shape[0] == 6
    assert 5 in m["faces"][:, 5].astype(int).tolist()


def test_rejected_meshes(pkg, ref):
    pinched_v = np.array([[-1, -1, 0], [1, -1, 0], [1, 1, 0], [-1, 1, 0], [0, 0, -0.25]], np.float32)
    pinched_t = np.array([[0, 3, 2], [0, 2, 1], [0, 1, 4], [1, 2, 4], [2, 3, 4], [3, 0, 4]], np.uint32)
    bad_v = TETRA_V.copy()
    bad_v[3, 2] = np.inf
    doubled_v = np.vstack([TETRA_V, TETRA_V])
    doubled_t = np.vstack([TETRA_T, TETRA_T + 4])
    cases = {"open": (TETRA_V, TETRA_T[:3]),
             "inward": (TETRA_V, np.vstack([TETRA_T[:3], [[1, 3, 2]]])),
             "nonfinite": (bad_v, TETRA_T),
             "degenerate": (TETRA_V, np.vstack([[[0, 2, 2]], TETRA_T[1:]])),
             "concave": (pinched_v, pinched_t),
             "two shells": (doubled_v, doubled_t)}
    for name, (v, t) in cases.items():
        with pytest.raises(ValueError):
            pkg.ConvexMesh(v, t)
        with pytest.raises(ValueError):
            ref.cook_convex(v, t)
