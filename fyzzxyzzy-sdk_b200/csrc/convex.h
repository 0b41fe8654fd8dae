// Cooked convex hulls: the host-side cooking of fyzz::cook_convex_mesh
// (include/fyzzxyzzy/convex.h:56-60, src/native/cooked_convex.cpp:41-330).
#pragma once
#include <array>
#include <cstdint>
#include <memory>
#include <vector>

namespace fyzz::b200 {

// An immutable cooked hull.  Faces are the hull's planar polygons (coplanar
// input triangles merged), each an outward normal, plane distance and a
// boundary loop idx[first, first + count) starting at its smallest vertex.
// Mass properties are for density one in the authoring frame: volume,
// centre of mass and the inertia tensor about it (columns).
struct CookedMesh {
    struct Face {
        std::array<float, 3> n;
        float d;
        uint32_t first, count;
    };
    std::vector<std::array<float, 3>> verts;
    std::vector<std::array<uint32_t, 3>> tris;
    std::vector<Face> faces;
    std::vector<uint32_t> idx;
    double volume = 0.0;
    std::array<float, 3> center{}, lo{}, hi{};
    std::array<std::array<float, 3>, 3> inertia{};   // columns
};

// Validates and cooks an outward-wound, closed, convex, manifold triangle
// surface.  Throws std::invalid_argument for the meshes the reference
// rejects and std::overflow_error past 32-bit indexing.
std::shared_ptr<const CookedMesh> cook_convex(const float* verts, uint32_t nv, const uint32_t* tris,
                                              uint32_t nt);

}  // namespace fyzz::b200
