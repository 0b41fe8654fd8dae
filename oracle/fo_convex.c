/* Test infrastructure: C restatement of the reference's convex mesh cooking
 * (src/native/cooked_convex.cpp:41-330, cook_convex_mesh) for the rigid-body
 * step oracle.  Only the published results are computed: the vertex bounds,
 * the planar face polygons (ConvexFace, include/fyzzxyzzy/convex.h:19-24)
 * and the density-one mass properties.  Input validation is the product's
 * and the reference's job; this assumes a mesh the reference accepts.
 *
 * Double arithmetic follows the reference expression by expression (x86-64
 * SSE2, no contraction), so the cooked floats are bit-identical. */
#include "fyzz_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

typedef struct { double x[3]; } dv;
static dv dsub(dv a, dv b) { dv r = {{a.x[0] - b.x[0], a.x[1] - b.x[1], a.x[2] - b.x[2]}}; return r; }
static dv dcross(dv a, dv b) {
    dv r = {{a.x[1] * b.x[2] - a.x[2] * b.x[1], a.x[2] * b.x[0] - a.x[0] * b.x[2],
             a.x[0] * b.x[1] - a.x[1] * b.x[0]}};
    return r;
}
static double ddot(dv a, dv b) { return a.x[0] * b.x[0] + a.x[1] * b.x[1] + a.x[2] * b.x[2]; }
static dv dvert(const float* v, uint32_t i) {
    dv r = {{v[3 * i], v[3 * i + 1], v[3 * i + 2]}};
    return r;
}

void fo_mesh_free(fo_mesh* m) {
    free(m->verts);
    free(m->faces);
    free(m->idx);
    memset(m, 0, sizeof *m);
}

int fo_cook_convex(const float* verts, uint32_t nv, const uint32_t* tris, uint32_t nt, fo_mesh* m) {
    memset(m, 0, sizeof *m);
    if (nv < 4 || nt < 4) return FO_INVALID;
    /* cooked_convex.cpp:52-68: bounds and the vertex mean (each term
     * divided by the count before it is summed) */
    dv lo = dvert(verts, 0), hi = lo, origin = {{0, 0, 0}};
    for (uint32_t i = 0; i < nv; ++i) {
        const dv p = dvert(verts, i);
        for (int k = 0; k < 3; ++k) {
            lo.x[k] = p.x[k] < lo.x[k] ? p.x[k] : lo.x[k];
            hi.x[k] = hi.x[k] < p.x[k] ? p.x[k] : hi.x[k];
            origin.x[k] += p.x[k] / (double)nv;
        }
    }
    const dv extent = dsub(hi, lo);
    double scale = extent.x[0];
    if (scale < extent.x[1]) scale = extent.x[1];
    if (scale < extent.x[2]) scale = extent.x[2];
    if (!(scale > 0.0)) return FO_INVALID;
    for (int k = 0; k < 3; ++k) {
        m->lo[k] = (float)lo.x[k];
        m->hi[k] = (float)hi.x[k];
    }
    /* cooked_convex.cpp:134-147: signed tetrahedra about the vertex mean */
    double volume = 0.0, first[3] = {0, 0, 0}, second[3][3];
    memset(second, 0, sizeof second);
    for (uint32_t f = 0; f < nt; ++f) {
        const uint32_t* t = tris + 3ull * f;
        if (t[0] >= nv || t[1] >= nv || t[2] >= nv) return FO_INVALID;
        const dv a = dsub(dvert(verts, t[0]), origin);
        const dv b = dsub(dvert(verts, t[1]), origin);
        const dv c = dsub(dvert(verts, t[2]), origin);
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
    /* cooked_convex.cpp:160-246: coplanar triangles grouped in triangle
     * order; each group's boundary loop starts at its smallest vertex */
    const double plane_tol = scale * 1.e-6;
    dv* gn = (dv*)malloc(sizeof(dv) * nt);
    dv* gp = (dv*)malloc(sizeof(dv) * nt);
    uint32_t* tri_group = (uint32_t*)malloc(4ull * nt);
    uint32_t ng = 0;
    for (uint32_t i = 0; i < nt; ++i) {
        const uint32_t* t = tris + 3ull * i;
        const dv p0 = dvert(verts, t[0]), p1 = dvert(verts, t[1]), p2 = dvert(verts, t[2]);
        dv n = dcross(dsub(p1, p0), dsub(p2, p0));
        const double len = sqrt(ddot(n, n));
        for (int k = 0; k < 3; ++k) n.x[k] /= len;
        uint32_t g = 0;
        for (; g < ng; ++g)
            if (ddot(n, gn[g]) > 1.0 - 1.e-7 && fabs(ddot(gn[g], dsub(p0, gp[g]))) <= plane_tol &&
                fabs(ddot(gn[g], dsub(p1, gp[g]))) <= plane_tol && fabs(ddot(gn[g], dsub(p2, gp[g]))) <= plane_tol)
                break;
        if (g == ng) {
            gn[ng] = n;
            gp[ng] = p0;
            ++ng;
        }
        tri_group[i] = g;
    }
    m->faces = (fo_face*)calloc(ng, sizeof(fo_face));
    m->idx = (uint32_t*)malloc(4ull * 3 * nt);
    uint32_t* efrom = (uint32_t*)malloc(4ull * 3 * nt);
    uint32_t* eto = (uint32_t*)malloc(4ull * 3 * nt);
    uint32_t* next = (uint32_t*)malloc(4ull * nv);
    int rc = FO_OK;
    for (uint32_t g = 0; g < ng && rc == FO_OK; ++g) {
        uint32_t ne = 0;
        for (uint32_t i = 0; i < nt; ++i) {
            if (tri_group[i] != g) continue;
            const uint32_t* t = tris + 3ull * i;
            for (int k = 0; k < 3; ++k) {
                const uint32_t from = t[k], to = t[(k + 1) % 3];
                uint32_t e = 0;
                while (e < ne && !(efrom[e] == to && eto[e] == from)) ++e;
                if (e < ne) {            /* interior edge: both windings seen */
                    efrom[e] = efrom[ne - 1];
                    eto[e] = eto[ne - 1];
                    --ne;
                } else {
                    efrom[ne] = from;
                    eto[ne] = to;
                    ++ne;
                }
            }
        }
        if (ne < 3) { rc = FO_INVALID; break; }
        uint32_t start = 0xffffffffu;
        for (uint32_t e = 0; e < ne; ++e) {
            next[efrom[e]] = eto[e];
            if (efrom[e] < start) start = efrom[e];
        }
        const uint32_t off = m->ni;
        uint32_t cur = start;
        for (uint32_t e = 0; e < ne; ++e) {
            m->idx[m->ni++] = cur;
            cur = next[cur];
        }
        const double dist = ddot(gn[g], gp[g]);
        fo_face* F = &m->faces[g];
        for (int k = 0; k < 3; ++k) F->n[k] = (float)gn[g].x[k];
        F->d = (float)dist;
        F->first = off;
        F->count = ne;
    }
    m->nf = ng;
    free(gn); free(gp); free(tri_group); free(efrom); free(eto); free(next);
    if (rc != FO_OK || !(volume > 0.0)) {
        fo_mesh_free(m);
        return FO_INVALID;
    }
    /* cooked_convex.cpp:257-300: centroid and inertia about it */
    double center[3];
    for (int i = 0; i < 3; ++i) center[i] = first[i] / volume;
    double cov[3][3];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) cov[i][j] = second[i][j] - volume * center[i] * center[j];
    const double trace = cov[0][0] + cov[1][1] + cov[2][2];
    m->volume = volume;
    for (int i = 0; i < 3; ++i) m->center[i] = (float)(center[i] + origin.x[i]);
    for (int j = 0; j < 3; ++j)
        for (int i = 0; i < 3; ++i) m->inertia[3 * j + i] = (float)((i == j ? trace : 0.0) - cov[i][j]);
    m->nv = nv;
    m->verts = (float*)malloc(12ull * nv);
    memcpy(m->verts, verts, 12ull * nv);
    return FO_OK;
}
