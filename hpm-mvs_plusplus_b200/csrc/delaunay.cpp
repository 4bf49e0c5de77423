// Delaunay triangulation of the planar-prior support points (the role of
// cv::Subdiv2D in HPM::DelaunayTriangulation, HPM.cpp:1075-1097).
//
// Incremental Bowyer-Watson: points are inserted in the given order; the
// triangle containing the new point is found by walking across adjacencies from
// the last created triangle (support points arrive in block order, so walks are
// short); the cavity of triangles whose circumcircle strictly contains the point
// is re-triangulated as a fan.  Coordinates are integers, so orientation and
// in-circle are evaluated exactly in 128-bit integers.  A duplicate point is
// skipped (Subdiv2D::insert returns the existing vertex).  Triangles touching the
// three enclosing vertices are not reported, like getTriangleList with the
// image rectangle.
#include "hpm_types.h"

#include <cstdint>
#include <unordered_map>
#include <vector>

namespace hpm {

namespace {

typedef __int128 i128;

struct Tri {
    int v[3];   // counter-clockwise (in a y-down image frame: orient > 0)
    int n[3];   // n[k] = triangle across the edge opposite v[k], -1 for none
    bool alive;
};

struct Mesh {
    std::vector<long long> x, y;
    std::vector<Tri> tris;

    long long orient(int a, int b, int c) const {
        return (x[b] - x[a]) * (y[c] - y[a]) - (y[b] - y[a]) * (x[c] - x[a]);
    }
    // > 0 when d is strictly inside the circumcircle of the ccw triangle (a, b, c)
    i128 incircle(int a, int b, int c, int d) const {
        const i128 adx = x[a] - x[d], ady = y[a] - y[d];
        const i128 bdx = x[b] - x[d], bdy = y[b] - y[d];
        const i128 cdx = x[c] - x[d], cdy = y[c] - y[d];
        const i128 ad = adx * adx + ady * ady, bd = bdx * bdx + bdy * bdy, cd = cdx * cdx + cdy * cdy;
        return adx * (bdy * cd - bd * cdy) - ady * (bdx * cd - bd * cdx) + ad * (bdx * cdy - bdy * cdx);
    }
};

}  // namespace

int delaunay_triangulate(const int32_t* xy, int n, int width, int height, std::vector<hpm_triangle>& out) {
    out.clear();
    if (n <= 0) return 0;
    Mesh m;
    const long long big = 64LL * (long long)(width > height ? width : height) + 1024;
    // enclosing triangle, counter-clockwise for orient() (x right, y down)
    m.x = { -big, 3 * big, -big };
    m.y = { -big, -big, 3 * big };
    if (m.orient(0, 1, 2) < 0) { std::swap(m.x[1], m.x[2]); std::swap(m.y[1], m.y[2]); }
    m.tris.push_back({ { 0, 1, 2 }, { -1, -1, -1 }, true });
    std::unordered_map<long long, int> seen;
    seen.reserve((size_t)n * 2);
    int last = 0;
    std::vector<int> cavity, stack;
    std::vector<char> in_cavity;
    struct Edge { int a, b, outer; };
    std::vector<Edge> boundary;
    for (int i = 0; i < n; ++i) {
        const long long px = xy[2 * i], py = xy[2 * i + 1];
        const long long key = (px << 32) ^ (py & 0xffffffffLL);
        if (seen.count(key)) continue;
        const int p = (int)m.x.size();
        m.x.push_back(px);
        m.y.push_back(py);
        seen[key] = p;
        // locate: walk towards the point
        int t = last;
        if (!m.tris[t].alive) {
            for (t = (int)m.tris.size() - 1; t >= 0 && !m.tris[t].alive; --t) {}
        }
        for (size_t guard = 0; guard < m.tris.size() + 16; ++guard) {
            const Tri& T = m.tris[t];
            int next = -1;
            for (int k = 0; k < 3; ++k) {
                const int a = T.v[(k + 1) % 3], b = T.v[(k + 2) % 3];
                if (m.orient(a, b, p) < 0) { next = T.n[k]; break; }
            }
            if (next < 0) break;
            t = next;
        }
        // cavity: triangles whose circumcircle strictly contains p (connected from t)
        cavity.clear();
        stack.clear();
        in_cavity.resize(m.tris.size(), 0);
        stack.push_back(t);
        in_cavity[t] = 1;
        while (!stack.empty()) {
            const int c = stack.back();
            stack.pop_back();
            cavity.push_back(c);
            for (int k = 0; k < 3; ++k) {
                const int nb = m.tris[c].n[k];
                if (nb < 0 || in_cavity[nb]) continue;
                const Tri& N = m.tris[nb];
                if (m.incircle(N.v[0], N.v[1], N.v[2], p) > 0) {
                    in_cavity[nb] = 1;
                    stack.push_back(nb);
                }
            }
        }
        // boundary edges of the cavity (directed ccw), with the outside neighbour
        boundary.clear();
        for (int c : cavity) {
            const Tri& T = m.tris[c];
            for (int k = 0; k < 3; ++k) {
                const int nb = T.n[k];
                if (nb >= 0 && in_cavity[nb]) continue;
                boundary.push_back({ T.v[(k + 1) % 3], T.v[(k + 2) % 3], nb });
            }
        }
        for (int c : cavity) { m.tris[c].alive = false; in_cavity[c] = 0; }
        // fan of new triangles (p, a, b) for each boundary edge a->b
        const int first = (int)m.tris.size();
        std::unordered_map<int, int> start_of;  // boundary vertex a -> new triangle (p, a, b)
        start_of.reserve(boundary.size() * 2);
        for (size_t e = 0; e < boundary.size(); ++e) {
            const Edge& E = boundary[e];
            Tri T;
            T.v[0] = p; T.v[1] = E.a; T.v[2] = E.b;
            T.n[0] = E.outer;  // across edge (a, b)
            T.n[1] = -1; T.n[2] = -1;
            T.alive = true;
            const int id = first + (int)e;
            m.tris.push_back(T);
            start_of[E.a] = id;
            if (E.outer >= 0) {
                Tri& O = m.tris[E.outer];
                for (int k = 0; k < 3; ++k) {
                    const int oa = O.v[(k + 1) % 3], ob = O.v[(k + 2) % 3];
                    if (oa == E.b && ob == E.a) O.n[k] = id;
                }
            }
        }
        for (size_t e = 0; e < boundary.size(); ++e) {
            const int id = first + (int)e;
            Tri& T = m.tris[id];
            // edge opposite v[1]=a is (b, p): neighbour is the triangle starting at b
            auto it = start_of.find(T.v[2]);
            T.n[1] = it == start_of.end() ? -1 : it->second;
            // edge opposite v[2]=b is (p, a): neighbour is the triangle ending at a
            for (size_t f = 0; f < boundary.size(); ++f)
                if (boundary[f].b == T.v[1]) { T.n[2] = first + (int)f; break; }
        }
        last = first;
        in_cavity.resize(m.tris.size(), 0);
    }
    for (const Tri& T : m.tris) {
        if (!T.alive || T.v[0] < 3 || T.v[1] < 3 || T.v[2] < 3) continue;
        hpm_triangle o;
        o.x1 = (int32_t)m.x[T.v[0]]; o.y1 = (int32_t)m.y[T.v[0]];
        o.x2 = (int32_t)m.x[T.v[1]]; o.y2 = (int32_t)m.y[T.v[1]];
        o.x3 = (int32_t)m.x[T.v[2]]; o.y3 = (int32_t)m.y[T.v[2]];
        out.push_back(o);
    }
    return (int)out.size();
}

}  // namespace hpm
