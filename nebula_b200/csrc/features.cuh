// Input features of the escape-probability network (no reference
// counterpart): log energy, distance to the nearest surface, direction
// cosine toward that surface, material one-hot.
//
// The nearest surface comes from a surface map: a regular grid over a region
// of interest whose cells store, for the cell centre c, the distance d_c to
// the nearest point q of any material triangle and the unit vector
// g = (c - q) / d_c from that point to the centre (the gradient of the
// distance field), or d_c < 0 when no triangle lies within d_max.  At a point
// p of the cell the distance is taken to first order, d_c + g . (p - c):
// exact where p and c see the same face of the nearest triangle, and within
// the cell's extent of the true distance elsewhere (both lie between
// d_c - |p - c| and |p - q|).  The cosine toward the surface is -g . dir.  A
// feature lookup is one 16-byte gather.
#pragma once

#include <cstdint>

#include "dev_types.h"

namespace nbx {
namespace dev {

struct SurfaceMap {
    const float4* cell;   // per cell (g.x, g.y, g.z, d_c); nullptr: no map (distance feature saturates)
    float lox, loy, loz;
    float cell_size, inv_cell;
    int nx, ny, nz;
    float d_max;
};

#ifdef __CUDACC__
// Closest point of triangle (a, a + e1, a + e2) to p, by the Voronoi-region
// classification of C. Ericson, "Real-Time Collision Detection" (2005), 5.1.5.
__device__ __forceinline__ void closest_point_on_triangle(float px, float py, float pz, const float4& A, const float4& E1,
                                                          const float4& E2, float* qx, float* qy, float* qz) {
    const float abx = E1.x, aby = E1.y, abz = E1.z;
    const float acx = E2.x, acy = E2.y, acz = E2.z;
    const float apx = px - A.x, apy = py - A.y, apz = pz - A.z;
    const float d1 = abx * apx + aby * apy + abz * apz;
    const float d2 = acx * apx + acy * apy + acz * apz;
    if (d1 <= 0 && d2 <= 0) {
        *qx = A.x; *qy = A.y; *qz = A.z;
        return;
    }
    const float bx = A.x + abx, by = A.y + aby, bz = A.z + abz;
    const float bpx = px - bx, bpy = py - by, bpz = pz - bz;
    const float d3 = abx * bpx + aby * bpy + abz * bpz;
    const float d4 = acx * bpx + acy * bpy + acz * bpz;
    if (d3 >= 0 && d4 <= d3) {
        *qx = bx; *qy = by; *qz = bz;
        return;
    }
    const float vc = d1 * d4 - d3 * d2;
    if (vc <= 0 && d1 >= 0 && d3 <= 0) {
        const float v = d1 / (d1 - d3);
        *qx = A.x + v * abx; *qy = A.y + v * aby; *qz = A.z + v * abz;
        return;
    }
    const float cx = A.x + acx, cy = A.y + acy, cz = A.z + acz;
    const float cpx = px - cx, cpy = py - cy, cpz = pz - cz;
    const float d5 = abx * cpx + aby * cpy + abz * cpz;
    const float d6 = acx * cpx + acy * cpy + acz * cpz;
    if (d6 >= 0 && d5 <= d6) {
        *qx = cx; *qy = cy; *qz = cz;
        return;
    }
    const float vb = d5 * d2 - d1 * d6;
    if (vb <= 0 && d2 >= 0 && d6 <= 0) {
        const float w = d2 / (d2 - d6);
        *qx = A.x + w * acx; *qy = A.y + w * acy; *qz = A.z + w * acz;
        return;
    }
    const float va = d3 * d6 - d5 * d4;
    if (va <= 0 && (d4 - d3) >= 0 && (d5 - d6) >= 0) {
        const float w = (d4 - d3) / ((d4 - d3) + (d5 - d6));
        *qx = bx + w * (cx - bx); *qy = by + w * (cy - by); *qz = bz + w * (cz - bz);
        return;
    }
    const float denom = 1.0f / (va + vb + vc);
    const float v = vb * denom, w = vc * denom;
    *qx = A.x + abx * v + acx * w;
    *qy = A.y + aby * v + acy * w;
    *qz = A.z + abz * v + acz * w;
}

__device__ __forceinline__ float dist2_to_triangle(const float4* tri, int ti, float px, float py, float pz) {
    const float4 a = tri[3 * ti], b = tri[3 * ti + 1], c = tri[3 * ti + 2];
    float qx, qy, qz;
    closest_point_on_triangle(px, py, pz, a, b, c, &qx, &qy, &qz);
    return (px - qx) * (px - qx) + (py - qy) * (py - qy) + (pz - qz) * (pz - qz);
}

// The surface-map cell of p: its record, and the offset of p from the cell
// centre; false when p lies outside the map or the cell has no surface within
// d_max.
__device__ __forceinline__ bool surface_cell(const SurfaceMap& S, float px, float py, float pz, float4* rec,
                                             float* ox, float* oy, float* oz) {
    if (!S.cell) return false;
    const int ix = int(floorf((px - S.lox) * S.inv_cell));
    const int iy = int(floorf((py - S.loy) * S.inv_cell));
    const int iz = int(floorf((pz - S.loz) * S.inv_cell));
    if (ix < 0 || iy < 0 || iz < 0 || ix >= S.nx || iy >= S.ny || iz >= S.nz) return false;
    *rec = __ldg(S.cell + (size_t(iz) * S.ny + iy) * S.nx + ix);
    if (!(rec->w >= 0.0f)) return false;
    *ox = px - (S.lox + (float(ix) + 0.5f) * S.cell_size);
    *oy = py - (S.loy + (float(iy) + 0.5f) * S.cell_size);
    *oz = pz - (S.loz + (float(iz) + 0.5f) * S.cell_size);
    return true;
}

// Distance from p to the nearest surface (first order in the map cell),
// clamped to [0, d_max]; d_max outside the map or with no surface within d_max.
__device__ __forceinline__ float surface_distance(const SurfaceMap& S, float px, float py, float pz) {
    float4 r;
    float ox, oy, oz;
    if (!surface_cell(S, px, py, pz, &r, &ox, &oy, &oz)) return S.d_max;
    return fminf(fmaxf(r.w + r.x * ox + r.y * oy + r.z * oz, 0.0f), S.d_max);
}

// Feature scaling: log E over [log 12 eV, log 8 keV] -> about [0, 1]; the
// distance over [0, d_max] -> [0, 1].
constexpr float kLogEOffset = 2.5f;
constexpr float kLogEScale = 1.0f / 6.5f;

// f[6] for an electron at p with unit direction d in material `mat` (>= 0).
__device__ __forceinline__ void electron_features(const SurfaceMap& S, float px, float py, float pz, float dx,
                                                  float dy, float dz, float logE, int mat, float f[6]) {
    f[0] = (logE - kLogEOffset) * kLogEScale;
    f[1] = 1.0f;
    f[2] = 0.0f;
    f[3] = mat == 0 ? 1.0f : 0.0f;
    f[4] = mat == 1 ? 1.0f : 0.0f;
    f[5] = mat == 2 ? 1.0f : 0.0f;
    float4 r;
    float ox, oy, oz;
    if (!surface_cell(S, px, py, pz, &r, &ox, &oy, &oz)) return;
    const float dist = fminf(fmaxf(r.w + r.x * ox + r.y * oy + r.z * oz, 0.0f), S.d_max);
    f[1] = dist / S.d_max;
    f[2] = -(r.x * dx + r.y * dy + r.z * dz);
}
#endif

}  // namespace dev
}  // namespace nbx
