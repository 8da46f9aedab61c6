// Octree builder with the reference's linearized layout; see octree.h.
#include "octree.h"

#include <cmath>
#include <fstream>
#include <queue>
#include <sstream>
#include <stdexcept>

namespace nbx {

namespace {
constexpr int kMaxDepth = 21;    // octree_builder.h:157
constexpr int kSplitCount = 16;  // octree_builder.h:158

inline Vec3 add(Vec3 a, Vec3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline Vec3 sub(Vec3 a, Vec3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline Vec3 scale(float s, Vec3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline bool eq(Vec3 a, Vec3 b) { return a.x == b.x && a.y == b.y && a.z == b.z; }
inline float fmin_ref(float a, float b) { return (b < a) ? b : a; }   // std::min
inline float fmax_ref(float a, float b) { return (a < b) ? b : a; }   // std::max

Vec3 vert(const Triangle& t, int i) {
    if (i == 0) return t.r0;
    return add(t.r0, i == 1 ? t.e1 : t.e2);
}

// triangle::perfect_overlap (source/core/triangle.inl:94-111): same vertex
// set in any cyclic or reversed order, materials ignored.
bool perfect_overlap(const Triangle& a, const Triangle& b) {
    const Vec3 a0 = vert(a, 0), a1 = vert(a, 1), a2 = vert(a, 2);
    const Vec3 b0 = vert(b, 0), b1 = vert(b, 1), b2 = vert(b, 2);
    return (eq(a0, b0) && eq(a1, b1) && eq(a2, b2)) || (eq(a0, b1) && eq(a1, b2) && eq(a2, b0)) ||
           (eq(a0, b2) && eq(a1, b0) && eq(a2, b1)) || (eq(a0, b0) && eq(a1, b2) && eq(a2, b1)) ||
           (eq(a0, b1) && eq(a1, b0) && eq(a2, b2)) || (eq(a0, b2) && eq(a1, b1) && eq(a2, b0));
}

// Separating-axis triangle/box overlap test of T. Akenine-Moeller ("Fast 3D
// Triangle-Box Overlap Testing", 2001), in double precision, with every
// projection evaluated as in the reference's tribox.cc so borderline cells
// (faces lying on cell planes are common in CAD-like geometry) are decided
// identically.
struct SepAxis {
    const double* v0;
    const double* v1;
    const double* v2;
    const double* h;

    // axis = edge x unit-x; uses components (y, z)
    static bool outside(double p_a, double p_b, double rad) {
        const double mn = p_a < p_b ? p_a : p_b;
        const double mx = p_a < p_b ? p_b : p_a;
        return mn > rad || mx < -rad;
    }
    bool x_axis(double a, double b, double fa, double fb, const double* va, const double* vb) const {
        const double pa = a * va[1] - b * va[2];
        const double pb = a * vb[1] - b * vb[2];
        return outside(pa, pb, fa * h[1] + fb * h[2]);
    }
    bool y_axis(double a, double b, double fa, double fb, const double* va, const double* vb) const {
        const double pa = -a * va[0] + b * va[2];
        const double pb = -a * vb[0] + b * vb[2];
        return outside(pa, pb, fa * h[0] + fb * h[2]);
    }
    bool z_axis(double a, double b, double fa, double fb, const double* va, const double* vb) const {
        const double pa = a * va[0] - b * va[1];
        const double pb = a * vb[0] - b * vb[1];
        return outside(pa, pb, fa * h[0] + fb * h[1]);
    }
};

bool plane_box_overlap(const double n[3], const double v[3], const double maxbox[3]) {
    double vmin[3], vmax[3];
    for (int q = 0; q < 3; ++q) {
        if (n[q] > 0) {
            vmin[q] = -maxbox[q] - v[q];
            vmax[q] = maxbox[q] - v[q];
        } else {
            vmin[q] = maxbox[q] - v[q];
            vmax[q] = -maxbox[q] - v[q];
        }
    }
    if (n[0] * vmin[0] + n[1] * vmin[1] + n[2] * vmin[2] > 0) return false;
    if (n[0] * vmax[0] + n[1] * vmax[1] + n[2] * vmax[2] >= 0) return true;
    return false;
}

bool tri_box_overlap(const double c[3], const double h[3], const double tv[3][3]) {
    double v0[3], v1[3], v2[3], e0[3], e1[3], e2[3];
    for (int i = 0; i < 3; ++i) {
        v0[i] = tv[0][i] - c[i];
        v1[i] = tv[1][i] - c[i];
        v2[i] = tv[2][i] - c[i];
    }
    for (int i = 0; i < 3; ++i) {
        e0[i] = v1[i] - v0[i];
        e1[i] = v2[i] - v1[i];
        e2[i] = v0[i] - v2[i];
    }
    // Box axes: the triangle's AABB against the box.
    for (int ax = 0; ax < 3; ++ax) {
        double mn = v0[ax], mx = v0[ax];
        if (v1[ax] < mn) mn = v1[ax];
        if (v1[ax] > mx) mx = v1[ax];
        if (v2[ax] < mn) mn = v2[ax];
        if (v2[ax] > mx) mx = v2[ax];
        if (mn > h[ax] || mx < -h[ax]) return false;
    }
    // Triangle plane.
    double n[3];
    n[0] = e0[1] * e1[2] - e0[2] * e1[1];
    n[1] = e0[2] * e1[0] - e0[0] * e1[2];
    n[2] = e0[0] * e1[1] - e0[1] * e1[0];
    if (!plane_box_overlap(n, v0, h)) return false;
    // Nine edge x axis cross products; each edge is projected with the two
    // vertices that differ on it.
    const SepAxis s{v0, v1, v2, h};
    double fx = std::fabs(e0[0]), fy = std::fabs(e0[1]), fz = std::fabs(e0[2]);
    if (s.x_axis(e0[2], e0[1], fz, fy, v0, v2)) return false;
    if (s.y_axis(e0[2], e0[0], fz, fx, v0, v2)) return false;
    if (s.z_axis(e0[1], e0[0], fy, fx, v1, v2)) return false;
    fx = std::fabs(e1[0]); fy = std::fabs(e1[1]); fz = std::fabs(e1[2]);
    if (s.x_axis(e1[2], e1[1], fz, fy, v0, v2)) return false;
    if (s.y_axis(e1[2], e1[0], fz, fx, v0, v2)) return false;
    if (s.z_axis(e1[1], e1[0], fy, fx, v0, v1)) return false;
    fx = std::fabs(e2[0]); fy = std::fabs(e2[1]); fz = std::fabs(e2[2]);
    if (s.x_axis(e2[2], e2[1], fz, fy, v0, v1)) return false;
    if (s.y_axis(e2[2], e2[0], fz, fx, v0, v1)) return false;
    if (s.z_axis(e2[1], e2[0], fy, fx, v1, v2)) return false;
    return true;
}

// octree_node::overlap (octree_builder.cpp:30-39): the cell grown by 1%.
bool overlap(const Triangle& t, Vec3 c, Vec3 h) {
    const double center[3] = {c.x, c.y, c.z};
    const double half[3] = {1.01 * h.x, 1.01 * h.y, 1.01 * h.z};
    double tv[3][3];
    for (int i = 0; i < 3; ++i) {
        const Vec3 v = vert(t, i);
        tv[i][0] = v.x;
        tv[i][1] = v.y;
        tv[i][2] = v.z;
    }
    return tri_box_overlap(center, half, tv);
}

struct Builder {
    struct Node {
        int32_t first_child = -1;     // -1: leaf
        std::vector<uint32_t> tris;
    };
    const std::vector<Triangle>& all;
    std::vector<Node> nodes;
    uint64_t duplicates = 0;
    int max_depth = 0;

    explicit Builder(const std::vector<Triangle>& t) : all(t) {}

    static void octant(int o, Vec3 c, Vec3 h, Vec3* oc, Vec3* oh) {
        *oh = scale(0.5f, h);
        oc->x = c.x + float(((o & 1) << 1) - 1) * oh->x;
        oc->y = c.y + float((o & 2) - 1) * oh->y;
        oc->z = c.z + float(((o & 4) >> 1) - 1) * oh->z;
    }

    bool insert(int32_t node, uint32_t ti, Vec3 c, Vec3 h, int depth) {
        const Triangle& t = all[ti];
        if (!overlap(t, c, h)) return false;
        if (depth > max_depth) max_depth = depth;
        if (nodes[node].first_child < 0) {
            for (uint32_t j : nodes[node].tris) {
                if (perfect_overlap(t, all[j])) {
                    ++duplicates;
                    return false;
                }
            }
            nodes[node].tris.push_back(ti);
            if (int(nodes[node].tris.size()) > kSplitCount && depth < kMaxDepth) split(node, c, h, depth);
        } else {
            const int32_t fc = nodes[node].first_child;
            for (int o = 0; o < 8; ++o) {
                Vec3 oc, oh;
                octant(o, c, h, &oc, &oh);
                insert(fc + o, ti, oc, oh, depth + 1);
            }
        }
        return true;
    }

    void split(int32_t node, Vec3 c, Vec3 h, int depth) {
        const int32_t fc = int32_t(nodes.size());
        nodes.resize(nodes.size() + 8);
        nodes[node].first_child = fc;
        const std::vector<uint32_t> tris = nodes[node].tris;
        for (int o = 0; o < 8; ++o) {
            Vec3 oc, oh;
            octant(o, c, h, &oc, &oh);
            for (uint32_t ti : tris) insert(fc + o, ti, oc, oh, depth + 1);
        }
        std::vector<uint32_t>().swap(nodes[node].tris);
    }
};
}  // namespace

Triangle make_triangle(Vec3 a, Vec3 b, Vec3 c, int mat_in, int mat_out) {
    Triangle t;
    t.r0 = a;
    t.e1 = sub(b, a);
    t.e2 = sub(c, a);
    t.mat_in = mat_in;
    t.mat_out = mat_out;
    return t;
}

LinearOctree build_octree(const std::vector<Triangle>& input) {
    if (input.empty()) throw std::runtime_error("no triangles");
    if (input.size() > uint64_t(INT32_MAX)) throw std::runtime_error("Too many triangles for linearized octree.");
    LinearOctree out;

    // Root box: union of triangle AABBs plus 1 nm (octree_builder.cpp:171-209).
    Vec3 mn, mx;
    for (size_t i = 0; i < input.size(); ++i) {
        const Vec3 A = vert(input[i], 0), B = vert(input[i], 1), C = vert(input[i], 2);
        const Vec3 tmin{fmin_ref(fmin_ref(A.x, B.x), C.x), fmin_ref(fmin_ref(A.y, B.y), C.y), fmin_ref(fmin_ref(A.z, B.z), C.z)};
        const Vec3 tmax{fmax_ref(fmax_ref(A.x, B.x), C.x), fmax_ref(fmax_ref(A.y, B.y), C.y), fmax_ref(fmax_ref(A.z, B.z), C.z)};
        if (i == 0) {
            mn = tmin;
            mx = tmax;
        } else {
            mn = {fmin_ref(mn.x, tmin.x), fmin_ref(mn.y, tmin.y), fmin_ref(mn.z, tmin.z)};
            mx = {fmax_ref(mx.x, tmax.x), fmax_ref(mx.y, tmax.y), fmax_ref(mx.z, tmax.z)};
        }
    }
    out.center = scale(0.5f, add(mn, mx));
    out.halfsize = add(scale(0.5f, sub(mx, mn)), Vec3{1, 1, 1});

    // Insert (octree_root::insert): triangles outside the root are skipped and
    // the kept ones are renumbered in insertion order.
    std::vector<Triangle> kept;
    kept.reserve(input.size());
    for (const Triangle& t : input)
        if (overlap(t, out.center, out.halfsize)) kept.push_back(t);
    Builder b(kept);
    b.nodes.resize(9);
    b.nodes[0].first_child = 1;
    for (uint32_t ti = 0; ti < kept.size(); ++ti) {
        for (int o = 0; o < 8; ++o) {
            Vec3 oc, oh;
            Builder::octant(o, out.center, out.halfsize, &oc, &oh);
            b.insert(1 + o, ti, oc, oh, 1);
        }
    }
    out.duplicates_dropped = b.duplicates;
    out.max_depth = b.max_depth;

    // Breadth-first (Morton) order of nodes.
    std::vector<int32_t> order;
    order.reserve(b.nodes.size());
    {
        std::queue<int32_t> q;
        q.push(0);
        while (!q.empty()) {
            const int32_t n = q.front();
            q.pop();
            order.push_back(n);
            if (b.nodes[n].first_child >= 0)
                for (int o = 0; o < 8; ++o) q.push(b.nodes[n].first_child + o);
        }
    }
    // Triangles in first-visit order over the leaves.
    std::vector<int32_t> tri_map(kept.size(), -1);
    out.triangles.reserve(kept.size());
    for (int32_t n : order) {
        if (b.nodes[n].first_child >= 0) continue;
        for (uint32_t ti : b.nodes[n].tris) {
            if (tri_map[ti] >= 0) continue;
            tri_map[ti] = int32_t(out.triangles.size());
            out.triangles.push_back(kept[ti]);
        }
    }
    // Node table: 8 child slots for inner nodes, -1-terminated lists for leaves.
    std::vector<int64_t> start(b.nodes.size(), -1);
    for (int32_t n : order) {
        start[n] = int64_t(out.octree_data.size());
        if (b.nodes[n].first_child < 0) {
            for (uint32_t ti : b.nodes[n].tris) out.octree_data.push_back(tri_map[ti]);
            out.octree_data.push_back(-1);
        } else {
            for (int o = 0; o < 8; ++o) out.octree_data.push_back(0);
        }
        if (out.octree_data.size() > size_t(INT32_MAX)) throw std::runtime_error("Octree is too large.");
    }
    for (int32_t n : order) {
        if (b.nodes[n].first_child < 0) continue;
        for (int o = 0; o < 8; ++o) {
            const int32_t c = b.nodes[n].first_child + o;
            int32_t v = int32_t(start[c]);
            if (b.nodes[c].first_child < 0) v = -v;
            out.octree_data[size_t(start[n]) + o] = v;
        }
    }
    return out;
}

std::vector<Triangle> load_tri_file(const std::string& filename) {
    std::vector<Triangle> tris;
    std::ifstream ifs(filename);
    if (!ifs.is_open()) return tris;
    size_t line_num = 1;
    std::string line;
    while (std::getline(ifs, line)) {
        line_num++;
        if (line.empty()) continue;
        const size_t i = line.find_first_not_of(" \t");
        if (i < line.size() && line[i] == '#') continue;
        std::istringstream ss(line);
        std::vector<std::string> cols;
        std::string tok;
        while (ss >> tok) cols.push_back(tok);
        if (cols.empty()) continue;
        if (cols.size() != 11)
            throw std::runtime_error("invalid number of columns in line '" + std::to_string(line_num) + "'");
        const int in = std::stoi(cols[0]);
        const int out = std::stoi(cols[1]);
        float v[9];
        for (int k = 0; k < 9; ++k) v[k] = float(std::stod(cols[2 + k]));
        tris.push_back(make_triangle({v[0], v[1], v[2]}, {v[3], v[4], v[5]}, {v[6], v[7], v[8]}, in, out));
    }
    return tris;
}

}  // namespace nbx
