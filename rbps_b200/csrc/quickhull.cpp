// quickhull.cpp - host convex hull builder (setup only).
//
// The reference ships no hull builder: ConvexHullData takes caller-provided
// CCW triangles (rbc/shapes/ConvexHull.hpp:29-33, 126-420).  This
// incremental hull (initial tetrahedron, then each point added by deleting
// the faces it sees and fanning the horizon) produces those triangles with
// outward normals for the synthetic hull scenes.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "rbps_gpu.h"

int rbps_internal_fail(int code, const char *msg);

namespace
{
    struct V
    {
        double x, y, z;
    };
    V sub(V a, V b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
    V crs(V a, V b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
    double dt(V a, V b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
    double nrm(V a) { return std::sqrt(dt(a, a)); }

    struct Face
    {
        uint32_t a, b, c;
        V n;
        double d;
    };

    Face make_face(const std::vector<V> &p, uint32_t a, uint32_t b, uint32_t c)
    {
        Face f{a, b, c, crs(sub(p[b], p[a]), sub(p[c], p[a])), 0.0};
        const double l = nrm(f.n);
        if (l > 0)
            f.n = {f.n.x / l, f.n.y / l, f.n.z / l};
        f.d = dt(f.n, p[a]);
        return f;
    }
} // namespace

extern "C" int rbps_quickhull(const double *points, uint32_t n, uint32_t *tris, uint32_t cap, uint32_t *n_tris)
{
    if (!points || n < 4 || !n_tris)
        return rbps_internal_fail(RBPS_ERR_INVALID, "rbps_quickhull: need at least 4 points");
    std::vector<V> p(n);
    double scale = 0;
    for (uint32_t i = 0; i < n; ++i)
    {
        p[i] = {points[3 * i], points[3 * i + 1], points[3 * i + 2]};
        scale = std::max(scale, std::fabs(p[i].x) + std::fabs(p[i].y) + std::fabs(p[i].z));
    }
    const double eps = 1e-9 * std::max(scale, 1.0);
    // initial simplex: extreme x pair, farthest from their line, farthest from the plane
    uint32_t i0 = 0, i1 = 0;
    for (uint32_t i = 1; i < n; ++i)
    {
        if (p[i].x < p[i0].x)
            i0 = i;
        if (p[i].x > p[i1].x)
            i1 = i;
    }
    if (i0 == i1)
        return rbps_internal_fail(RBPS_ERR_INVALID, "rbps_quickhull: degenerate point set");
    uint32_t i2 = n;
    double best = eps;
    for (uint32_t i = 0; i < n; ++i)
    {
        const double d = nrm(crs(sub(p[i], p[i0]), sub(p[i1], p[i0])));
        if (d > best)
        {
            best = d;
            i2 = i;
        }
    }
    if (i2 == n)
        return rbps_internal_fail(RBPS_ERR_INVALID, "rbps_quickhull: collinear points");
    Face base = make_face(p, i0, i1, i2);
    uint32_t i3 = n;
    best = eps;
    for (uint32_t i = 0; i < n; ++i)
    {
        const double d = std::fabs(dt(base.n, p[i]) - base.d);
        if (d > best)
        {
            best = d;
            i3 = i;
        }
    }
    if (i3 == n)
        return rbps_internal_fail(RBPS_ERR_INVALID, "rbps_quickhull: coplanar points");
    std::vector<Face> faces;
    if (dt(base.n, p[i3]) - base.d > 0)
        std::swap(i1, i2);
    faces.push_back(make_face(p, i0, i1, i2));
    faces.push_back(make_face(p, i0, i3, i1));
    faces.push_back(make_face(p, i1, i3, i2));
    faces.push_back(make_face(p, i2, i3, i0));
    for (uint32_t q = 0; q < n; ++q)
    {
        if (q == i0 || q == i1 || q == i2 || q == i3)
            continue;
        std::vector<char> vis(faces.size(), 0);
        bool any = false;
        for (size_t f = 0; f < faces.size(); ++f)
            if (dt(faces[f].n, p[q]) - faces[f].d > eps)
            {
                vis[f] = 1;
                any = true;
            }
        if (!any)
            continue;
        std::vector<std::pair<uint32_t, uint32_t>> edges;
        for (size_t f = 0; f < faces.size(); ++f)
            if (vis[f])
            {
                edges.push_back({faces[f].a, faces[f].b});
                edges.push_back({faces[f].b, faces[f].c});
                edges.push_back({faces[f].c, faces[f].a});
            }
        std::vector<Face> keep;
        for (size_t f = 0; f < faces.size(); ++f)
            if (!vis[f])
                keep.push_back(faces[f]);
        for (const auto &e : edges)
        {
            bool interior = false;
            for (const auto &g : edges)
                if (g.first == e.second && g.second == e.first)
                {
                    interior = true;
                    break;
                }
            if (!interior)
                keep.push_back(make_face(p, e.first, e.second, q));
        }
        faces.swap(keep);
    }
    *n_tris = (uint32_t)faces.size();
    if (tris)
        for (uint32_t f = 0; f < faces.size() && f < cap; ++f)
        {
            tris[3 * f] = faces[f].a;
            tris[3 * f + 1] = faces[f].b;
            tris[3 * f + 2] = faces[f].c;
        }
    return RBPS_OK;
}
