// Delaunay triangulation of the planar-prior support points (the role of
// cv::Subdiv2D in HPM::DelaunayTriangulation, HPM.cpp:1075-1097), producing the
// same triangle LIST as Subdiv2D -- same triangles, same order, same first
// vertex -- because the prior raster lets the last triangle win on shared
// edges (main.cpp:398-404) and the plane fit rounds by vertex order.
//
// Algorithm: incremental Delaunay on a quad-edge structure, Guibas & Stolfi,
// "Primitives for the manipulation of general subdivisions and the computation
// of Voronoi diagrams", ACM TOG 4(2), 1985 (MakeEdge, Splice, Connect, Swap,
// DeleteEdge, the Locate walk and InsertSite).  The triangle list depends on
// how edges are numbered, which the paper leaves open; the conventions below
// were established by comparing this structure, edge by edge and after every
// insertion, with what Subdiv2D's public interface reports (edge origins,
// destinations and next-around-origin links), on random, grid-aligned and
// dense point sets up to 1600 x 1200:
//   * quad-edge 0 and vertex 0 are unused; vertices 1-3 enclose the image at
//     (B, 0), (0, B), (-B, -B) with B = 6 * max(width, height); quad-edges 1-3
//     are their edges 1->2, 2->3, 3->1, joined by Splice(e12, sym e31),
//     Splice(e23, sym e12), Splice(e31, sym e23);
//   * a new quad-edge takes the slot of the last deleted one, else the next
//     slot; an insertion makes its base edge first, then its Connect edges;
//   * each walk starts from the edge the previous walk ended on (for a point
//     already present, the edge whose origin or destination it is, not
//     reversed); when the point lies on that edge it is deleted and the walk's
//     start becomes its Oprev, the edge the insertion continues from;
//   * triangles are listed by scanning primal edges in increasing id and
//     taking each unvisited edge's left face (edge, Lnext, Lnext Lnext), first
//     vertex the scanned edge's origin, faces touching an enclosing vertex
//     skipped.
// Coordinates are integers, so the orientation and in-circle tests are exact
// (128-bit).  A point equal to an inserted one is skipped, as Subdiv2D::insert
// returns the existing vertex; points outside [0, width) x [0, height), which
// Subdiv2D rejects, are skipped.
#include "hpm_types.h"

#include <cstdint>
#include <vector>

namespace hpm {

namespace {

typedef __int128 i128;

class QuadEdges {
public:
    QuadEdges(int width, int height) {
        const long long big = 6LL * (width > height ? width : height);
        vx_ = { 0, big, 0, -big };
        vy_ = { 0, 0, big, -big };
        next_.assign(4, 0);
        org_.assign(4, 0);
        for (int i = 0; i < 4; ++i) next_[i] = i;
        const int ab = make(1, 2), bc = make(2, 3), ca = make(3, 1);
        splice(ab, ca ^ 2);
        splice(bc, ab ^ 2);
        splice(ca, bc ^ 2);
        recent_ = ab;
    }

    // Inserts (x, y); returns false for a point already present.
    bool insert(long long x, long long y) {
        int e = recent_;
        const int where = locate(x, y, e);
        recent_ = e;
        if (where == kVertex) return false;
        if (where == kEdge) {
            const int t = oprev(e);
            remove(e);
            e = t;
            recent_ = e;
        }
        vx_.push_back(x);
        vy_.push_back(y);
        const int v = (int)vx_.size() - 1;
        const int first = org_[e];
        int base = make(first, v);
        splice(base, e);
        const int start = base;
        do {
            base = connect(e, base ^ 2);
            e = oprev(base);
        } while (dst(e) != first);
        e = oprev(base);
        for (;;) {
            const int t = oprev(e);
            const int tv = dst(t);
            if (right_of(vx_[tv], vy_[tv], e) > 0 && in_circle(org_[e], tv, dst(e), v) > 0) {
                swap(e);
                e = oprev(e);
            } else if (next_[e] == start) {
                break;
            } else {
                e = lprev(next_[e]);
            }
        }
        return true;
    }

    void triangles(int width, int height, std::vector<hpm_triangle>& out) const {
        std::vector<char> seen(next_.size(), 0);
        auto inside = [&](int v) { return vx_[v] >= 0 && vx_[v] < width && vy_[v] >= 0 && vy_[v] < height; };
        for (int e = 4; e < (int)next_.size(); e += 2) {
            if (seen[e] || free_has(e >> 2)) continue;
            const int b = lnext(e), c = lnext(b);
            seen[e] = seen[b] = seen[c] = 1;
            const int va = org_[e], vb = org_[b], vc = org_[c];
            if (va < 4 || vb < 4 || vc < 4 || !inside(va) || !inside(vb) || !inside(vc)) continue;
            hpm_triangle t;
            t.x1 = (int32_t)vx_[va]; t.y1 = (int32_t)vy_[va];
            t.x2 = (int32_t)vx_[vb]; t.y2 = (int32_t)vy_[vb];
            t.x3 = (int32_t)vx_[vc]; t.y3 = (int32_t)vy_[vc];
            out.push_back(t);
        }
    }

private:
    enum { kInside, kEdge, kVertex };
    std::vector<long long> vx_, vy_;
    std::vector<int> next_, org_;
    std::vector<int> free_;
    int recent_ = 0;

    static int rot(int e) { return (e & ~3) | ((e + 1) & 3); }
    static int irot(int e) { return (e & ~3) | ((e + 3) & 3); }
    int oprev(int e) const { return rot(next_[rot(e)]); }
    int lnext(int e) const { return rot(next_[irot(e)]); }
    int lprev(int e) const { return next_[e] ^ 2; }
    int dprev(int e) const { return irot(next_[irot(e)]); }
    int dst(int e) const { return org_[e ^ 2]; }
    bool free_has(int q) const {
        for (int f : free_) if (f == q) return true;
        return false;
    }

    int make(int a, int b) {
        int q;
        if (!free_.empty()) {
            q = free_.back();
            free_.pop_back();
        } else {
            q = (int)(next_.size() / 4);
            next_.resize(next_.size() + 4);
            org_.resize(org_.size() + 4);
        }
        const int e = 4 * q;
        next_[e] = e; next_[e + 1] = e + 3; next_[e + 2] = e + 2; next_[e + 3] = e + 1;
        org_[e] = a; org_[e + 1] = 0; org_[e + 2] = b; org_[e + 3] = 0;
        return e;
    }

    void splice(int a, int b) {
        const int al = rot(next_[a]), be = rot(next_[b]);
        std::swap(next_[a], next_[b]);
        std::swap(next_[al], next_[be]);
    }

    int connect(int a, int b) {
        const int e = make(dst(a), org_[b]);
        splice(e, lnext(a));
        splice(e ^ 2, b);
        return e;
    }

    void swap(int e) {
        const int a = oprev(e), b = oprev(e ^ 2);
        splice(e, a);
        splice(e ^ 2, b);
        splice(e, lnext(a));
        splice(e ^ 2, lnext(b));
        org_[e] = dst(a);
        org_[e ^ 2] = dst(b);
    }

    void remove(int e) {
        splice(e, oprev(e));
        splice(e ^ 2, oprev(e ^ 2));
        free_.push_back(e >> 2);
    }

    // sign of the orientation of (p, dst(e), org(e)): > 0 when p lies right of e
    int right_of(long long px, long long py, int e) const {
        const int d = dst(e), o = org_[e];
        const i128 v = (i128)(vx_[d] - px) * (vy_[o] - py) - (i128)(vy_[d] - py) * (vx_[o] - px);
        return (v > 0) - (v < 0);
    }

    // sign of the in-circle determinant of (a, b, c) and d
    int in_circle(int a, int b, int c, int d) const {
        const i128 adx = vx_[a] - vx_[d], ady = vy_[a] - vy_[d];
        const i128 bdx = vx_[b] - vx_[d], bdy = vy_[b] - vy_[d];
        const i128 cdx = vx_[c] - vx_[d], cdy = vy_[c] - vy_[d];
        const i128 ad = adx * adx + ady * ady, bd = bdx * bdx + bdy * bdy, cd = cdx * cdx + cdy * cdy;
        const i128 v = adx * (bdy * cd - bd * cdy) - ady * (bdx * cd - bd * cdx) + ad * (bdx * cdy - bdy * cdx);
        return (v > 0) - (v < 0);
    }

    // The Locate walk from e; leaves in e the edge with p on its left (or on it).
    int locate(long long px, long long py, int& e) const {
        for (size_t guard = 0; guard < 4 * next_.size() + 64; ++guard) {
            if (vx_[org_[e]] == px && vy_[org_[e]] == py) return kVertex;
            if (vx_[dst(e)] == px && vy_[dst(e)] == py) return kVertex;  // the walk keeps e, not its reverse
            const int r = right_of(px, py, e);
            if (r > 0) { e ^= 2; continue; }
            const int on = next_[e];
            if (right_of(px, py, on) <= 0) { e = on; continue; }
            const int dp = dprev(e);
            if (right_of(px, py, dp) <= 0) { e = dp; continue; }
            return r == 0 ? kEdge : kInside;
        }
        return kInside;
    }
};

}  // namespace

int delaunay_triangulate(const int32_t* xy, int n, int width, int height, std::vector<hpm_triangle>& out) {
    out.clear();
    if (n <= 0 || width <= 0 || height <= 0) return 0;
    QuadEdges q(width, height);
    for (int i = 0; i < n; ++i) {
        const long long x = xy[2 * i], y = xy[2 * i + 1];
        if (x < 0 || x >= width || y < 0 || y >= height) continue;
        q.insert(x, y);
    }
    q.triangles(width, height, out);
    return (int)out.size();
}

}  // namespace hpm
