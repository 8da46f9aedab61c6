// Octree builder with the reference's linearized layout; see octree.h.
#include "octree.h"

#include <algorithm>
#include <array>
#include <atomic>
#include <cmath>
#include <cstring>
#include <fstream>
#include <sstream>
#include <stdexcept>
#include <thread>
#include <unordered_map>

namespace nbx {

namespace {
constexpr int kMaxDepth = 21;    // octree_builder.h:157
constexpr int kSplitCount = 16;  // octree_builder.h:158

inline Vec3 add(Vec3 a, Vec3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline Vec3 sub(Vec3 a, Vec3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline Vec3 scale(float s, Vec3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline float fmin_ref(float a, float b) { return (b < a) ? b : a; }   // std::min
inline float fmax_ref(float a, float b) { return (a < b) ? b : a; }   // std::max

Vec3 vert(const Triangle& t, int i) {
    if (i == 0) return t.r0;
    return add(t.r0, i == 1 ? t.e1 : t.e2);
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

// Children of a cell (octree_builder.cpp: octree_node octants).
void octant(int o, Vec3 c, Vec3 h, Vec3* oc, Vec3* oh) {
    *oh = scale(0.5f, h);
    oc->x = c.x + float(((o & 1) << 1) - 1) * oh->x;
    oc->y = c.y + float((o & 2) - 1) * oh->y;
    oc->z = c.z + float(((o & 4) >> 1) - 1) * oh->z;
}

// Runs fn(task) for task in [0, n) on all host cores.
template <typename Fn>
void parallel_for(size_t n, Fn fn) {
    const size_t hw = std::max<unsigned>(1u, std::thread::hardware_concurrency());
    const size_t nt = std::min(hw, n);
    if (nt <= 1) {
        for (size_t i = 0; i < n; ++i) fn(i);
        return;
    }
    std::atomic<size_t> next{0};
    std::vector<std::thread> th;
    th.reserve(nt);
    for (size_t t = 0; t < nt; ++t)
        th.emplace_back([&] {
            for (size_t i; (i = next.fetch_add(1)) < n;) fn(i);
        });
    for (auto& t : th) t.join();
}

// Perfect-overlap class key (triangle::perfect_overlap, core/triangle.inl:
// 94-111): the three vertices compared with ==, in any order.  -0 is folded
// into +0 (they compare equal); a vertex with a NaN never equals anything.
struct TriKey {
    uint32_t w[9];
    bool operator==(const TriKey& o) const { return std::memcmp(w, o.w, sizeof w) == 0; }
};
struct TriKeyHash {
    size_t operator()(const TriKey& k) const {
        uint64_t h = 1469598103934665603ull;
        for (uint32_t x : k.w) h = (h ^ x) * 1099511628211ull;
        return size_t(h);
    }
};
bool tri_key(const Triangle& t, TriKey* k) {
    std::array<std::array<uint32_t, 3>, 3> v;
    for (int i = 0; i < 3; ++i) {
        const Vec3 p = vert(t, i);
        const float c[3] = {p.x, p.y, p.z};
        for (int j = 0; j < 3; ++j) {
            if (std::isnan(c[j])) return false;
            const float f = c[j] == 0.0f ? 0.0f : c[j];
            std::memcpy(&v[i][j], &f, 4);
        }
    }
    std::sort(v.begin(), v.end());
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) k->w[3 * i + j] = v[i][j];
    return true;
}

// Top-down, level-synchronous construction of the tree the reference's
// incremental octree_root::insert produces (octree_builder.cpp:93-169):
//  * a triangle that perfectly overlaps an earlier one has the same geometry,
//    so it reaches exactly the cells of the earlier one and is rejected in
//    every leaf it reaches: dropping it up front changes no cell;
//  * a cell is split as soon as its leaf list exceeds 16 distinct triangles
//    below depth 21, and the set reaching a cell only grows, so the final
//    tree splits exactly the cells whose final distinct count exceeds 16;
//  * each list keeps insertion (= input) order, as splitting redistributes a
//    leaf's list in order and later triangles are appended.
// Cells are created level by level with children in octant order, which is
// the breadth-first order of the linearized layout.  Each level's overlap
// tests run in parallel over (cell, chunk of its list) tasks whose outputs
// are concatenated in chunk order.
struct Cell {
    Vec3 c, h;
    int depth;
    int32_t first_child = -1;   // -1: leaf
    std::vector<uint32_t> tris;
};

std::vector<Cell> build_cells(const std::vector<Triangle>& all, const std::vector<uint32_t>& ids, Vec3 c, Vec3 h,
                              int* max_depth) {
    std::vector<Cell> cells;
    cells.push_back(Cell{c, h, 0, 1, {}});   // the root is always split
    for (int o = 0; o < 8; ++o) {
        Cell ch;
        octant(o, c, h, &ch.c, &ch.h);
        ch.depth = 1;
        cells.push_back(std::move(ch));
    }
    // level 1 lists from the whole (deduplicated) triangle set
    struct Task {
        size_t parent;   // cell whose children receive the output
        size_t lo, hi;   // range of the parent's list (or of `ids` for the root)
        std::array<std::vector<uint32_t>, 8> out;
    };
    constexpr size_t kChunk = 4096;
    auto run_level = [&](std::vector<Task>& tasks, auto source) {
        parallel_for(tasks.size(), [&](size_t i) {
            Task& t = tasks[i];
            const Cell& p = cells[t.parent];
            const std::vector<uint32_t>& src = source(t.parent);
            Vec3 oc[8], oh[8];
            for (int o = 0; o < 8; ++o) octant(o, p.c, p.h, &oc[o], &oh[o]);
            for (size_t k = t.lo; k < t.hi; ++k) {
                const uint32_t ti = src[k];
                for (int o = 0; o < 8; ++o)
                    if (overlap(all[ti], oc[o], oh[o])) t.out[o].push_back(ti);
            }
        });
        // concatenate per child in chunk order
        for (Task& t : tasks) {
            const int32_t fc = cells[t.parent].first_child;
            for (int o = 0; o < 8; ++o) {
                auto& dst = cells[size_t(fc) + o].tris;
                dst.insert(dst.end(), t.out[o].begin(), t.out[o].end());
                std::vector<uint32_t>().swap(t.out[o]);
            }
        }
    };
    {
        std::vector<Task> tasks;
        for (size_t lo = 0; lo < ids.size(); lo += kChunk) tasks.push_back(Task{0, lo, std::min(ids.size(), lo + kChunk), {}});
        run_level(tasks, [&](size_t) -> const std::vector<uint32_t>& { return ids; });
    }
    size_t level_begin = 1, level_end = cells.size();
    while (level_begin < level_end) {
        std::vector<Task> tasks;
        for (size_t n = level_begin; n < level_end; ++n) {
            Cell& cell = cells[n];
            if (!cell.tris.empty() && cell.depth > *max_depth) *max_depth = cell.depth;
            if (int(cell.tris.size()) > kSplitCount && cell.depth < kMaxDepth) {
                cell.first_child = int32_t(cells.size());
                const Vec3 pc = cell.c, ph = cell.h;
                const int d = cell.depth + 1;
                const size_t m = cell.tris.size();
                for (int o = 0; o < 8; ++o) {
                    Cell ch;
                    octant(o, pc, ph, &ch.c, &ch.h);
                    ch.depth = d;
                    cells.push_back(std::move(ch));   // invalidates `cell`
                }
                for (size_t lo = 0; lo < m; lo += kChunk) tasks.push_back(Task{n, lo, std::min(m, lo + kChunk), {}});
            }
        }
        run_level(tasks, [&](size_t parent) -> const std::vector<uint32_t>& { return cells[parent].tris; });
        for (size_t n = level_begin; n < level_end; ++n)
            if (cells[n].first_child >= 0) std::vector<uint32_t>().swap(cells[n].tris);
        level_begin = level_end;
        level_end = cells.size();
    }
    return cells;
}
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
    Vec3 mn{}, mx{};   // set from the first triangle below
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
    {
        std::vector<uint8_t> keep(input.size());
        parallel_for((input.size() + 4095) / 4096, [&](size_t c) {
            const size_t hi = std::min(input.size(), (c + 1) * 4096);
            for (size_t i = c * 4096; i < hi; ++i) keep[i] = overlap(input[i], out.center, out.halfsize) ? 1 : 0;
        });
        kept.reserve(input.size());
        for (size_t i = 0; i < input.size(); ++i)
            if (keep[i]) kept.push_back(input[i]);
    }
    // Perfect-overlap duplicates (rejected in every leaf they reach).
    std::vector<uint32_t> ids;
    ids.reserve(kept.size());
    {
        std::unordered_map<TriKey, uint32_t, TriKeyHash> seen;
        seen.reserve(kept.size() * 2);
        for (uint32_t i = 0; i < kept.size(); ++i) {
            TriKey k;
            if (tri_key(kept[i], &k) && !seen.emplace(k, i).second) {
                ++out.duplicates_dropped;
                continue;
            }
            ids.push_back(i);
        }
    }
    int max_depth = 0;
    const std::vector<Cell> cells = build_cells(kept, ids, out.center, out.halfsize, &max_depth);
    out.max_depth = max_depth;

    // Triangles in first-visit order over the leaves (cells are breadth-first).
    std::vector<int32_t> tri_map(kept.size(), -1);
    out.triangles.reserve(ids.size());
    for (const Cell& cell : cells) {
        if (cell.first_child >= 0) continue;
        for (uint32_t ti : cell.tris) {
            if (tri_map[ti] >= 0) continue;
            tri_map[ti] = int32_t(out.triangles.size());
            out.triangles.push_back(kept[ti]);
        }
    }
    // Node table: 8 child slots for inner nodes, -1-terminated lists for leaves.
    std::vector<int64_t> start(cells.size(), -1);
    for (size_t n = 0; n < cells.size(); ++n) {
        start[n] = int64_t(out.octree_data.size());
        if (cells[n].first_child < 0) {
            for (uint32_t ti : cells[n].tris) out.octree_data.push_back(tri_map[ti]);
            out.octree_data.push_back(-1);
        } else {
            for (int o = 0; o < 8; ++o) out.octree_data.push_back(0);
        }
        if (out.octree_data.size() > size_t(INT32_MAX)) throw std::runtime_error("Octree is too large.");
    }
    for (size_t n = 0; n < cells.size(); ++n) {
        if (cells[n].first_child < 0) continue;
        for (int o = 0; o < 8; ++o) {
            const size_t c = size_t(cells[n].first_child) + o;
            int32_t v = int32_t(start[c]);
            if (cells[c].first_child < 0) v = -v;
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
