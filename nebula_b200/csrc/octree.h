// Host-side octree builder producing the linearized layout the transport
// kernels traverse.
//
// The layout is identical, word for word, to the reference's
// octree_builder::linearized_octree (source/geometry/octree/octree_builder.cpp
// :171-352): same root box (triangle AABB + 1 nm), same insertion rule
// (triangle/box overlap on the cell grown by 1%, split above 16 triangles up
// to depth 21, duplicate triangles dropped), breadth-first node order, leaf
// triangle lists in first-visit order terminated by -1, leaf children stored
// as negated offsets.  Bit-exact ray queries depend on this: the traversal
// order of leaf triangles decides ties.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace nbx {

struct Vec3 {
    float x, y, z;
};

// core/triangle.h: r0, e1 = r1 - r0, e2 = r2 - r0, material_in, material_out.
struct Triangle {
    Vec3 r0, e1, e2;
    int32_t mat_in, mat_out;
};
static_assert(sizeof(Triangle) == 44, "Triangle must match the 44-byte reference record");

Triangle make_triangle(Vec3 a, Vec3 b, Vec3 c, int mat_in, int mat_out);

struct LinearOctree {
    std::vector<int32_t> octree_data;
    std::vector<Triangle> triangles;      // Morton (first-visit) order
    Vec3 center{0, 0, 0};
    Vec3 halfsize{0, 0, 0};
    uint64_t duplicates_dropped = 0;
    int max_depth = 0;
};

LinearOctree build_octree(const std::vector<Triangle>& tris);

// .tri loader with the reference's rules (source/io/load_tri_file.cpp:8-60).
std::vector<Triangle> load_tri_file(const std::string& filename);

}  // namespace nbx
