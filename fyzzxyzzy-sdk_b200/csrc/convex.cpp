// Convex hull cooking (src/native/cooked_convex.cpp:41-330).
//
// What a reference user sees is reproduced exactly: the same admission rules
// (finite, closed, manifold, outward, convex, connected, positive volume and
// inertia), the same planar face polygons in the same order, and mass
// properties from the same double-precision signed-tetrahedron sums, so the
// cooked floats are bit-identical.  The bookkeeping is this file's own:
// half-edges are sorted by undirected key instead of hashed, face
// connectivity is a union-find over the sorted pairs, and each planar
// group's boundary is found from the same sorted half-edge list.
#include "convex.h"

#include <algorithm>
#include <cmath>
#include <limits>
#include <numeric>
#include <stdexcept>

namespace fyzz::b200 {
namespace {

struct D3 {
    double x[3];
};
D3 dsub(const D3& a, const D3& b) { return {{a.x[0] - b.x[0], a.x[1] - b.x[1], a.x[2] - b.x[2]}}; }
D3 dcross(const D3& a, const D3& b) {
    return {{a.x[1] * b.x[2] - a.x[2] * b.x[1], a.x[2] * b.x[0] - a.x[0] * b.x[2], a.x[0] * b.x[1] - a.x[1] * b.x[0]}};
}
double ddot(const D3& a, const D3& b) { return a.x[0] * b.x[0] + a.x[1] * b.x[1] + a.x[2] * b.x[2]; }

float to_float(double v) {
    if (!std::isfinite(v) || std::abs(v) > std::numeric_limits<float>::max())
        throw std::invalid_argument("Convex mass property outside float range");
    return static_cast<float>(v);
}

// One directed triangle edge: its undirected key, direction and face.
struct HalfEdge {
    uint64_t key;
    uint32_t from, to, face;
};

uint32_t find_root(std::vector<uint32_t>& parent, uint32_t i) {
    while (parent[i] != i) {
        parent[i] = parent[parent[i]];
        i = parent[i];
    }
    return i;
}

}  // namespace

std::shared_ptr<const CookedMesh> cook_convex(const float* verts, uint32_t nv, const uint32_t* tris, uint32_t nt) {
    if (nv < 4u || nt < 4u || !verts || !tris) throw std::invalid_argument("Convex hull requires a closed volume");
    auto mesh = std::make_shared<CookedMesh>();
    mesh->verts.resize(nv);
    mesh->tris.resize(nt);
    std::vector<D3> p(nv);
    for (uint32_t i = 0; i < nv; ++i) {
        for (int k = 0; k < 3; ++k) {
            mesh->verts[i][k] = verts[3 * size_t(i) + k];
            if (!std::isfinite(mesh->verts[i][k])) throw std::invalid_argument("Convex vertex must be finite");
            p[i].x[k] = mesh->verts[i][k];
        }
    }
    for (uint32_t f = 0; f < nt; ++f)
        for (int k = 0; k < 3; ++k) mesh->tris[f][k] = tris[3 * size_t(f) + k];

    // bounds and the vertex mean, each term divided before it is summed
    D3 lo = p[0], hi = p[0], origin{{0, 0, 0}};
    for (uint32_t i = 0; i < nv; ++i)
        for (int k = 0; k < 3; ++k) {
            lo.x[k] = std::min(lo.x[k], p[i].x[k]);
            hi.x[k] = std::max(hi.x[k], p[i].x[k]);
            origin.x[k] += p[i].x[k] / static_cast<double>(nv);
        }
    const D3 extent = dsub(hi, lo);
    const double scale = std::max({extent.x[0], extent.x[1], extent.x[2]});
    if (!(scale > 0.0) || !std::isfinite(scale)) throw std::invalid_argument("Convex hull has no spatial extent");
    for (int k = 0; k < 3; ++k) {
        mesh->lo[k] = to_float(lo.x[k]);
        mesh->hi[k] = to_float(hi.x[k]);
    }

    // per triangle: indices, area, the supporting-plane test and the
    // signed tetrahedron about the vertex mean
    std::vector<HalfEdge> half(3 * size_t(nt));
    std::vector<uint8_t> used(nv, 0u);
    double volume = 0.0, first[3] = {0, 0, 0}, second[3][3] = {};
    for (uint32_t f = 0; f < nt; ++f) {
        const auto& t = mesh->tris[f];
        for (int k = 0; k < 3; ++k)
            if (t[k] >= nv || t[k] == t[(k + 1) % 3] || t[k] == t[(k + 2) % 3])
                throw std::invalid_argument("Convex face has invalid indices");
        const D3 a = dsub(p[t[0]], origin), b = dsub(p[t[1]], origin), c = dsub(p[t[2]], origin);
        const D3 n = dcross(dsub(b, a), dsub(c, a));
        const double len = std::sqrt(ddot(n, n));
        if (!(len > scale * scale * 1.e-12) || !std::isfinite(len))
            throw std::invalid_argument("Convex hull has degenerate triangles");
        const double tol = scale * len * 1.e-6;
        for (uint32_t i = 0; i < nv; ++i)
            if (ddot(n, dsub(p[i], p[t[0]])) > tol) throw std::invalid_argument("Convex hull is nonconvex or inward-wound");
        for (int k = 0; k < 3; ++k) {
            const uint32_t u = t[k], v = t[(k + 1) % 3];
            used[u] = 1u;
            half[3 * size_t(f) + k] = {(uint64_t(std::min(u, v)) << 32) | std::max(u, v), u, v, f};
        }
        const double tetra = ddot(a, dcross(b, c)) / 6.0;
        volume += tetra;
        for (int i = 0; i < 3; ++i) first[i] += tetra * (a.x[i] + b.x[i] + c.x[i]) * 0.25;
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                const double si = a.x[i] + b.x[i] + c.x[i];
                const double sj = a.x[j] + b.x[j] + c.x[j];
                second[i][j] += tetra * 0.05 * (si * sj + a.x[i] * a.x[j] + b.x[i] * b.x[j] + c.x[i] * c.x[j]);
            }
    }
    // every undirected edge exactly once in each direction; faces that share
    // an edge belong to one shell
    std::vector<HalfEdge> sorted = half;
    std::sort(sorted.begin(), sorted.end(), [](const HalfEdge& x, const HalfEdge& y) {
        return x.key != y.key ? x.key < y.key : x.from < y.from;
    });
    std::vector<uint32_t> parent(nt);
    std::iota(parent.begin(), parent.end(), 0u);
    for (size_t i = 0; i < sorted.size();) {
        size_t j = i;
        while (j < sorted.size() && sorted[j].key == sorted[i].key) ++j;
        if (j - i != 2 || sorted[i].from == sorted[i + 1].from) {
            if (j - i > 2 || (j - i == 2 && sorted[i].from == sorted[i + 1].from))
                throw std::invalid_argument("Convex surface has nonmanifold edges");
            throw std::invalid_argument("Convex surface must be closed and use every vertex");
        }
        parent[find_root(parent, sorted[i].face)] = find_root(parent, sorted[i + 1].face);
        i = j;
    }
    if (std::find(used.begin(), used.end(), uint8_t(0)) != used.end())
        throw std::invalid_argument("Convex surface must be closed and use every vertex");
    const uint32_t shell = find_root(parent, 0);
    for (uint32_t f = 1; f < nt; ++f)
        if (find_root(parent, f) != shell) throw std::invalid_argument("Convex surface has disconnected shells");

    // planar groups in triangle order (first matching group wins)
    struct Group {
        D3 n, point;
        std::vector<uint32_t> tris;
    };
    std::vector<Group> groups;
    const double plane_tol = scale * 1.e-6;
    for (uint32_t f = 0; f < nt; ++f) {
        const auto& t = mesh->tris[f];
        const D3 p0 = p[t[0]], p1 = p[t[1]], p2 = p[t[2]];
        D3 n = dcross(dsub(p1, p0), dsub(p2, p0));
        const double len = std::sqrt(ddot(n, n));
        for (double& c : n.x) c /= len;
        auto g = std::find_if(groups.begin(), groups.end(), [&](const Group& c) {
            return ddot(n, c.n) > 1.0 - 1.e-7 && std::abs(ddot(c.n, dsub(p0, c.point))) <= plane_tol &&
                   std::abs(ddot(c.n, dsub(p1, c.point))) <= plane_tol &&
                   std::abs(ddot(c.n, dsub(p2, c.point))) <= plane_tol;
        });
        if (g == groups.end()) groups.push_back({n, p0, {f}});
        else g->tris.push_back(f);
    }
    // each group's boundary: its half-edges whose twin lies outside the
    // group, walked from the smallest vertex
    constexpr uint32_t kNone = std::numeric_limits<uint32_t>::max();
    std::vector<uint32_t> next(nv, kNone);
    for (const Group& g : groups) {
        std::vector<HalfEdge> e;
        for (uint32_t f : g.tris)
            for (int k = 0; k < 3; ++k) e.push_back(half[3 * size_t(f) + k]);
        std::sort(e.begin(), e.end(), [](const HalfEdge& x, const HalfEdge& y) {
            return x.key != y.key ? x.key < y.key : x.from < y.from;
        });
        std::vector<HalfEdge> boundary;
        for (size_t i = 0; i < e.size();) {
            size_t j = i;
            while (j < e.size() && e[j].key == e[i].key) ++j;
            if (j - i == 1) boundary.push_back(e[i]);
            else if (j - i != 2 || e[i].from == e[i + 1].from)
                throw std::invalid_argument("Convex polygon has inconsistent triangulation");
            i = j;
        }
        if (boundary.size() < 3) throw std::invalid_argument("Convex polygon has no boundary");
        uint32_t start = kNone;
        for (const HalfEdge& h : boundary) {
            if (next[h.from] != kNone) throw std::invalid_argument("Convex planar facet has branching boundary");
            next[h.from] = h.to;
            start = std::min(start, h.from);
        }
        if (mesh->idx.size() > std::numeric_limits<uint32_t>::max() - boundary.size())
            throw std::overflow_error("Convex face index stream too large");
        const uint32_t off = uint32_t(mesh->idx.size());
        uint32_t cur = start;
        for (size_t i = 0; i < boundary.size(); ++i) {
            if (cur == kNone || next[cur] == kNone || (i > 0 && cur == start))
                throw std::invalid_argument("Convex planar facet is not a single boundary loop");
            mesh->idx.push_back(cur);
            cur = next[cur];
        }
        if (cur != start) throw std::invalid_argument("Convex planar facet has disconnected boundary loops");
        for (const HalfEdge& h : boundary) next[h.from] = kNone;
        const double dist = ddot(g.n, g.point);
        if (!std::isfinite(dist) || std::abs(dist) > std::numeric_limits<float>::max())
            throw std::invalid_argument("Convex facet plane outside float range");
        CookedMesh::Face face;
        for (int k = 0; k < 3; ++k) face.n[k] = to_float(g.n.x[k]);
        face.d = static_cast<float>(dist);
        face.first = off;
        face.count = uint32_t(boundary.size());
        mesh->faces.push_back(face);
    }
    if (!std::isfinite(volume) || !(volume > 0.0)) throw std::invalid_argument("Convex mesh has nonpositive volume");

    // centroid, and the second moment moved to it and turned into inertia
    double center[3], inertia[3][3];
    for (int i = 0; i < 3; ++i) center[i] = first[i] / volume;
    double cov[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) cov[i][j] = second[i][j] - volume * center[i] * center[j];
    const double trace = cov[0][0] + cov[1][1] + cov[2][2];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) inertia[i][j] = (i == j ? trace : 0.0) - cov[i][j];
    const double m2 = inertia[0][0] * inertia[1][1] - inertia[0][1] * inertia[1][0];
    const double det = inertia[0][0] * (inertia[1][1] * inertia[2][2] - inertia[1][2] * inertia[2][1]) -
                       inertia[0][1] * (inertia[1][0] * inertia[2][2] - inertia[1][2] * inertia[2][0]) +
                       inertia[0][2] * (inertia[1][0] * inertia[2][1] - inertia[1][1] * inertia[2][0]);
    if (!(inertia[0][0] > 0.0) || !(m2 > 0.0) || !(det > 0.0) || !std::isfinite(det))
        throw std::invalid_argument("Convex hull has invalid rigid-body inertia");
    mesh->volume = volume;
    for (int i = 0; i < 3; ++i) mesh->center[i] = to_float(center[i] + origin.x[i]);
    for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i) mesh->inertia[j][i] = to_float(inertia[i][j]);
    return mesh;
}

}  // namespace fyzz::b200
