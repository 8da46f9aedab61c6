// Device-side electron transport for sm_100a.
//
// Single-precision arithmetic follows the reference's order and grouping
// operation by operation; the translation unit is compiled with
// -fmad=false and IEEE division/square root, so octree ray queries and table
// lookups are bit-identical to the reference CPU path.  The physics that is
// compared only statistically (free-path sampling, the scattering and
// boundary tails) uses the hardware's approximate forms (namespace approx,
// __logf, __expf), except expm1f, which stays accurate.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "dev_types.h"

namespace nbx {
namespace dev {

// ---------------------------------------------------------------------------
// Random numbers: Philox4x32-10 (Salmon et al., SC'11)
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k) {
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t lo0 = 0xD2511F53u * c.x;
        const uint32_t hi0 = __umulhi(0xD2511F53u, c.x);
        const uint32_t lo1 = 0xCD9E8D57u * c.z;
        const uint32_t hi1 = __umulhi(0xCD9E8D57u, c.z);
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
        k.x += 0x9E3779B9u;
        k.y += 0xBB67AE85u;
    }
    return c;
}
// (k + 1/2) / 2^23 with k the top 23 bits: exact, in (0, 1).
__device__ __forceinline__ float u01(uint32_t x) {
    return __fadd_rn(__fmul_rn(float(x >> 9), 1.1920928955078125e-07f), 5.9604644775390625e-08f);
}
__device__ __forceinline__ uint64_t secondary_uid(uint64_t parent, uint32_t step) {
    uint64_t z = parent + 0x9E3779B97F4A7C15ull * (uint64_t(step) + 1u);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z = z ^ (z >> 31);
    return z | (1ull << 63);
}
__device__ __forceinline__ uint4 draw(uint32_t seed, const Electron& e, uint32_t block) {
    return philox4x32_10(make_uint4(e.step, block, uint32_t(e.uid), uint32_t(e.uid >> 32)), make_uint2(seed, 0u));
}

// ---------------------------------------------------------------------------
// Scalar helpers with the reference CPU semantics
// ---------------------------------------------------------------------------
// (int)std::floor(x) as an x86-64 host evaluates it: out-of-range and NaN
// give INT_MIN (scalar_math.h:44-56, CPU branch).
__device__ __forceinline__ int floor_to_int(float x) {
    const float f = floorf(x);
    return (fabsf(f) < 2147483648.0f) ? int(f) : int(0x80000000u);
}
__device__ __forceinline__ int clampi(int i, int lo, int hi) { return i < lo ? lo : (i > hi ? hi : i); }
__device__ __forceinline__ float clampr(float i, float lo, float hi) { return i < lo ? lo : (i > hi ? hi : i); }
__device__ __forceinline__ float min_ref(float a, float b) { return (b < a) ? b : a; }
__device__ __forceinline__ float max_ref(float a, float b) { return (a < b) ? b : a; }

// ---------------------------------------------------------------------------
// Tables (common/util/table_1D.inl:66-80, table_2D.inl:74-104)
// ---------------------------------------------------------------------------
__device__ __forceinline__ float table1d_get(const Table1D& t, float x) {
    const float xi = (x - t.x_min) * t.x_step;
    const int lo = clampi(floor_to_int(xi), 0, t.n - 2);
    const float a = __ldg(t.data + lo);
    const float b = __ldg(t.data + lo + 1);
    const float f = xi - float(lo);
    return (1 - f) * a + f * b;
}
__device__ __forceinline__ float table2d_get(const Table2D& t, float x, float y) {
    const float xi = (x - t.x_min) * t.x_step;
    const float yi = (y - t.y_min) * t.y_step;
    const int lx = clampi(floor_to_int(xi), 0, t.w - 2);
    const int ly = clampi(floor_to_int(yi), 0, t.h - 2);
    const float* r0 = t.data + size_t(lx) * t.h + ly;
    const float* r1 = r0 + t.h;
    const float v00 = __ldg(r0), v01 = __ldg(r0 + 1);
    const float v10 = __ldg(r1), v11 = __ldg(r1 + 1);
    const float fx = xi - float(lx);
    const float fy = yi - float(ly);
    return (1 - fx) * (1 - fy) * v00 + fx * (1 - fy) * v10 + (1 - fx) * fy * v01 + fx * fy * v11;
}
__device__ __forceinline__ float table2d_rounddown(const Table2D& t, float x, float y) {
    const float xi = (x - t.x_min) * t.x_step;
    const float yi = (y - t.y_min) * t.y_step;
    const int lx = clampi(floor_to_int(xi), 0, t.w - 1);
    const int ly = clampi(floor_to_int(yi), 0, t.h - 1);
    return __ldg(t.data + size_t(lx) * t.h + ly);
}

// table_3D::get / get_rounddown (common/util/table_3D.inl:79-122); element
// (i, j, k) at data[(j + i * height) * depth + k] (table_3D.inl:66-70).
__device__ __forceinline__ float table3d_get(const Table3D& t, float x, float y, float z) {
    const float xi = (x - t.x_min) * t.x_step;
    const float yi = (y - t.y_min) * t.y_step;
    const float zi = (z - t.z_min) * t.z_step;
    const int lx = clampi(floor_to_int(xi), 0, t.w - 2);
    const int ly = clampi(floor_to_int(yi), 0, t.h - 2);
    const int lz = clampi(floor_to_int(zi), 0, t.d - 2);
    const float* p00 = t.data + (size_t(lx) * t.h + ly) * t.d + lz;   // (lx,   ly)
    const float* p10 = p00 + size_t(t.h) * t.d;                        // (lx+1, ly)
    const float* p01 = p00 + t.d;                                      // (lx,   ly+1)
    const float* p11 = p10 + t.d;                                      // (lx+1, ly+1)
    const float v000 = __ldg(p00), v001 = __ldg(p00 + 1);
    const float v100 = __ldg(p10), v101 = __ldg(p10 + 1);
    const float v010 = __ldg(p01), v011 = __ldg(p01 + 1);
    const float v110 = __ldg(p11), v111 = __ldg(p11 + 1);
    const float fx = xi - float(lx);
    const float fy = yi - float(ly);
    const float fz = zi - float(lz);
    return (1 - fx) * (1 - fy) * (1 - fz) * v000 + fx * (1 - fy) * (1 - fz) * v100 + (1 - fx) * fy * (1 - fz) * v010 +
           fx * fy * (1 - fz) * v110 + (1 - fx) * (1 - fy) * fz * v001 + fx * (1 - fy) * fz * v101 +
           (1 - fx) * fy * fz * v011 + fx * fy * fz * v111;
}
__device__ __forceinline__ float table3d_rounddown(const Table3D& t, float x, float y, float z) {
    const float xi = (x - t.x_min) * t.x_step;
    const float yi = (y - t.y_min) * t.y_step;
    const float zi = (z - t.z_min) * t.z_step;
    const int lx = clampi(floor_to_int(xi), 0, t.w - 1);
    const int ly = clampi(floor_to_int(yi), 0, t.h - 1);
    const int lz = clampi(floor_to_int(zi), 0, t.d - 1);
    return __ldg(t.data + (size_t(lx) * t.h + ly) * t.d + lz);
}

// ---------------------------------------------------------------------------
// Vector helpers (common/vector_math.h, CPU branches)
// ---------------------------------------------------------------------------
struct V3 {
    float x, y, z;
};
__device__ __forceinline__ float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ V3 cross(V3 a, V3 b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
// normalised(a) = a * (1 / sqrt(a.a))   (vector_math.h:37-40,128-140)
__device__ __forceinline__ V3 normalised(V3 a) {
    const float inv = 1.0f / sqrtf(a.x * a.x + a.y * a.y + a.z * a.z);
    return {a.x * inv, a.y * inv, a.z * inv};
}
// ---------------------------------------------------------------------------
// Approximate forms for the statistical-only physics: the scattering and
// boundary tails are compared with the reference by their statistics, not
// bit for bit, so they use the hardware's approximate reciprocal square
// root, quotient, exponential, logarithm and sine/cosine (a few ulp) instead
// of the correctly rounded or accurate library forms.  Nothing that feeds
// octree::propagate or a table index comparison with the reference goes
// through these.
// ---------------------------------------------------------------------------
namespace approx {
// sqrt(x) for x >= 0 as x / sqrt(x) with the hardware reciprocal square root
__device__ __forceinline__ float sqrt(float x) { return x > 0.0f ? x * rsqrtf(x) : 0.0f; }
__device__ __forceinline__ float div(float a, float b) { return __fdividef(a, b); }
__device__ __forceinline__ V3 normalised(V3 a) {
    const float inv = rsqrtf(a.x * a.x + a.y * a.y + a.z * a.z);
    return {a.x * inv, a.y * inv, a.z * inv};
}
// sin and cos of 2 pi u for u in [0, 1): the angle is shifted into
// [-pi, pi) where the hardware sine and cosine are accurate, and the signs
// restored (sin(x + pi) = -sin(x), cos(x + pi) = -cos(x)).
__device__ __forceinline__ void sincos_2pi(float u, float* s, float* c) {
    __sincosf(6.28318530717958648f * u - 3.14159265358979324f, s, c);
    *s = -*s;
    *c = -*c;
}
// make_normal_vec (vector_math.h:171-186) with the rotation angle given as a
// uniform u (phi = 2 pi u).  The reference takes cos and sin of
// atan2(dir.y, dir.x); here they are dir.x / r and dir.y / r with
// r = |(dir.x, dir.y)| (azimuth 0 when r = 0), the same values without the
// two transcendental calls.
__device__ __forceinline__ V3 make_normal_vec(V3 dir, float u_phi) {
    const float r2 = dir.x * dir.x + dir.y * dir.y;
    float sin_az = 0.0f, cos_az = 1.0f, r = 0.0f;
    if (r2 > 0.0f) {
        const float inv = rsqrtf(r2);
        cos_az = dir.x * inv;
        sin_az = dir.y * inv;
        r = r2 * inv;
    }
    const V3 v{dir.z * cos_az, dir.z * sin_az, -r};
    const V3 u = cross(v, dir);
    float sp, cp;
    sincos_2pi(u_phi, &sp, &cp);
    return {u.x * cp + v.x * sp, u.y * cp + v.y * sp, u.z * cp + v.z * sp};
}
// make_unit_vec (vector_math.h:194-206), phi = 2 pi u_phi
__device__ __forceinline__ V3 make_unit_vec(float cos_theta, float u_phi) {
    float sp, cp;
    sincos_2pi(u_phi, &sp, &cp);
    cos_theta = clampr(cos_theta, -1, 1);
    const float st = approx::sqrt(1 - cos_theta * cos_theta);
    return {st * cp, st * sp, cos_theta};
}
}  // namespace approx

// ---------------------------------------------------------------------------
// Geometry
// ---------------------------------------------------------------------------
__device__ __forceinline__ void load_tri_vertices(const Geometry& g, int ti, V3& r0, V3& e1, V3& e2) {
    const float4 a = __ldg(g.tri + 3 * ti);
    const float4 b = __ldg(g.tri + 3 * ti + 1);
    const float4 c = __ldg(g.tri + 3 * ti + 2);
    r0 = {a.x, a.y, a.z};
    e1 = {b.x, b.y, b.z};
    e2 = {c.x, c.y, c.z};
}

// Unnormalised normal e1 x e2 (triangle::get_normal, core/triangle.inl:71-74)
// and the two materials, from the triangle's 16-byte face record.
__device__ __forceinline__ V3 load_face(const Geometry& g, int ti, int& mi, int& mo) {
    const float4 f = __ldg(g.tri_face + ti);
    const int w = __float_as_int(f.w);
    mi = int(int16_t(w & 0xFFFF));
    mo = w >> 16;
    return V3{f.x, f.y, f.z};
}

// triangle::intersect_ray (core/triangle.inl:7-29)
__device__ __forceinline__ float intersect_ray(V3 r0, V3 e1, V3 e2, V3 start, V3 dir) {
    const V3 pvec = cross(dir, e2);
    const float det = dot(e1, pvec);
    if (fabsf(det) < kEps) return -1;
    const V3 s{start.x - r0.x, start.y - r0.y, start.z - r0.z};
    const float u = dot(s, pvec) / det;
    if ((u < -kEps) || (u > 1 + kEps)) return -1;
    const V3 qvec = cross(s, e1);
    const float v = dot(dir, qvec) / det;
    if ((v < -kEps) || (u + v > 1 + kEps)) return -1;
    const float t = dot(e2, qvec) / det;
    if (t < 0) return -1;
    return t;
}

// octree::in_domain (geometry/octree.inl:25-31)
__device__ __forceinline__ bool in_domain(const Geometry& g, V3 p) {
    return (p.x > g.cx - g.hx) && (p.x < g.cx + g.hx) && (p.y > g.cy - g.hy) && (p.y < g.cy + g.hy) &&
           (p.z > g.cz - g.hz) && (p.z < g.cz + g.hz);
}

// The octant offset (bit - 0.5) of geometry/octree.inl:65-67,79-81, as a
// select: exactly +-0.5, without an integer-to-float conversion.
__device__ __forceinline__ float half_step(unsigned bit) { return bit ? 0.5f : -0.5f; }

// Per-thread memo of the last octree leaf a descent reached, kept in shared
// memory as 13 words strided by the block size: location code (2 words), raw
// leaf value, the leaf's AABB centre and scale (ax, ay, az, aw) exactly as the
// descent computed them, and per-axis bounds (lo, hi].  A position p with
// lo < p <= hi on every axis gives the same octant at every level of a descent
// from the root (octant bit = p > centre), so it lands in the same leaf with
// the same float AABB: reusing the memo is bit-identical to descending.
struct LeafCache {
    float* base;   // nullptr: no cache
    int stride;
    __device__ __forceinline__ float& f(int i) const { return base[i * stride]; }
};

// octree::propagate (geometry/octree.inl:33-192).  Returns the travelled
// distance; *hit receives the triangle index or -1.
__device__ __forceinline__ float propagate(const Geometry& g, V3 start, V3 dir, float distance, int ignore_tri,
                                           int ignore_mat, int* hit, LeafCache cache = LeafCache{nullptr, 0}) {
    const int32_t* od = g.octree;
    V3 cur = start;
    float to_go = distance;
    uint64_t location = 1;
    bool first = true;
    do {
        float ax, ay, az, aw;
        int index;
        bool cached = false;
        if (first && cache.base) {
            const uint64_t cl = uint64_t(__float_as_uint(cache.f(0))) | (uint64_t(__float_as_uint(cache.f(1))) << 32);
            if (cl > 1 && cur.x > cache.f(7) && cur.x <= cache.f(10) && cur.y > cache.f(8) && cur.y <= cache.f(11) &&
                cur.z > cache.f(9) && cur.z <= cache.f(12)) {
                location = cl;
                index = __float_as_int(cache.f(2));
                ax = cache.f(3);
                ay = cache.f(4);
                az = cache.f(5);
                aw = cache.f(6);
                cached = true;
            }
        }
        if (!cached) {
            const float inf = __int_as_float(0x7f800000);
            float lox = -inf, loy = -inf, loz = -inf, hix = inf, hiy = inf, hiz = inf;
            ax = g.cx;
            ay = g.cy;
            az = g.cz;
            aw = 1;
            index = 0;
            for (int i = 60 - __clzll(location); i >= 0; i -= 3) {
                const unsigned octant = unsigned(location >> i) & 7u;
                index = __ldg(od + index + octant);
                if (octant & 1) lox = ax; else hix = ax;
                if (octant & 2) loy = ay; else hiy = ay;
                if (octant & 4) loz = az; else hiz = az;
                ax += aw * g.hx * half_step(octant & 1);
                ay += aw * g.hy * half_step(octant & 2);
                az += aw * g.hz * half_step(octant & 4);
                aw *= 0.5f;
            }
            while (index >= 0) {
                unsigned octant = 0;
                octant ^= (cur.x > ax) ? 1u : 0u;
                octant ^= (cur.y > ay) ? 2u : 0u;
                octant ^= (cur.z > az) ? 4u : 0u;
                location = (location << 3) | octant;
                index = __ldg(od + index + octant);
                if (octant & 1) lox = ax; else hix = ax;
                if (octant & 2) loy = ay; else hiy = ay;
                if (octant & 4) loz = az; else hiz = az;
                ax += aw * g.hx * half_step(octant & 1);
                ay += aw * g.hy * half_step(octant & 2);
                az += aw * g.hz * half_step(octant & 4);
                aw *= 0.5f;
            }
            if (cache.base) {
                cache.f(0) = __uint_as_float(uint32_t(location));
                cache.f(1) = __uint_as_float(uint32_t(location >> 32));
                cache.f(2) = __int_as_float(index);
                cache.f(3) = ax;
                cache.f(4) = ay;
                cache.f(5) = az;
                cache.f(6) = aw;
                cache.f(7) = lox;
                cache.f(8) = loy;
                cache.f(9) = loz;
                cache.f(10) = hix;
                cache.f(11) = hiy;
                cache.f(12) = hiz;
            }
        }
        first = false;
        index = -index;

        float intersect;
        int target;
        {
            const float bx = aw * g.hx, by = aw * g.hy, bz = aw * g.hz;
            const float tx = (ax + copysignf(bx + kEps, dir.x) - cur.x) / dir.x;
            const float ty = (ay + copysignf(by + kEps, dir.y) - cur.y) / dir.y;
            const float tz = (az + copysignf(bz + kEps, dir.z) - cur.z) / dir.z;
            if ((tx < ty) && (tx < tz)) {
                intersect = tx;
                target = -1;
            } else if ((ty < tx) && (ty < tz)) {
                intersect = ty;
                target = -2;
            } else {
                intersect = tz;
                target = -4;
            }
        }
        for (;;) {
            const int ti = __ldg(od + index);
            ++index;
            if (ti < 0) break;
            if (ti == ignore_tri) continue;
            // The face record alone decides the exit material (the normal is
            // e1 x e2 as computed on the device, so the sign is the
            // reference's); only candidates that survive load the vertices.
            int mi, mo;
            const V3 nrm = load_face(g, ti, mi, mo);
            const int mat_out = (dot(nrm, dir) < 0) ? mi : mo;
            if (mat_out == ignore_mat) continue;
            V3 r0, e1, e2;
            load_tri_vertices(g, ti, r0, e1, e2);
            const float t = intersect_ray(r0, e1, e2, cur, dir);
            if ((t > 0) && (t <= intersect + kEps)) {
                intersect = t;
                target = ti;
            }
        }
        if (intersect >= to_go) {
            *hit = -1;
            return distance;
        } else if (target >= 0) {
            *hit = target;
            return distance - to_go + intersect;
        }
        to_go -= intersect;
        cur.x += dir.x * intersect;
        cur.y += dir.y * intersect;
        cur.z += dir.z * intersect;
        const unsigned mask = unsigned(-target);
        unsigned value;
        if (mask == 1)
            value = (dir.x >= 0) ? 0u : 1u;
        else if (mask == 2)
            value = (dir.y >= 0) ? 0u : 2u;
        else
            value = (dir.z >= 0) ? 0u : 4u;
        while (location > 1) {
            if ((location & mask) == value) {
                location ^= mask;
                break;
            }
            location >>= 3;
        }
    } while (location > 1);
    *hit = -1;
    return distance;
}

// ---------------------------------------------------------------------------
// Physics
// ---------------------------------------------------------------------------
// The two scattering mechanisms share their first half: a 2D ICDF lookup at
// (log E, U) and the random normal to the current direction.  step() runs
// that half once for every lane that scatters (the warp stays converged) and
// then branches into the mechanism-specific remainder below.

// kieft_elastic<acoustic phonon loss, atomic recoil>::execute (physics/kieft/elastic.h:68-115)
// after the ICDF lookup (icdf_value) and with d = normalised(dir),
// n = normalised(make_normal_vec(d, phi)).
__device__ __forceinline__ void elastic_finish(const Material& m, Electron& e, float icdf_value, V3 d, V3 n) {
    const float cos_theta = clampr(icdf_value, -1, 1);
    const float sin_theta = approx::sqrt(1 - cos_theta * cos_theta);
    e.dx = d.x * cos_theta + n.x * sin_theta;
    e.dy = d.y * cos_theta + n.y * sin_theta;
    e.dz = d.z * cos_theta + n.z * sin_theta;
    if (e.E < 200)
        e.E -= min_ref(50e-3f, m.phonon_loss);
    else
        e.E -= m.recoil_const * (1 - cos_theta) * e.E;
}

// kieft_inelastic<all options>::execute (physics/kieft/inelastic.h:69-206)
// after the log-omega' ICDF lookup (log_omega0), with d and n as above.
// u_bind, u_omega: binding-energy and energy-loss draws; u_v1, u_v2: the
// instantaneous-momentum unit vector.  Returns true and fills *se when a
// secondary is created.
__device__ __forceinline__ bool inelastic_finish(const Material& m, Electron& e, float log_omega0, V3 d, V3 n,
                                                 float u_bind, float u_omega, float u_v1, float u_v2, Electron* se) {
    const float K = e.E;
    const float omega0 = __expf(log_omega0);
    // log(omega0) is the ICDF value itself (the reference takes the log of
    // its exponential); the rounddown lookup sees the same coordinate.
    float binding = table2d_rounddown(m.ion, log_omega0, u_bind);
    float omega;
    {
        const float omega_max = 0.5f * (K + omega0 - m.fermi);
        float omega_min = omega0;
        float w0 = min_ref(omega0 - 1, max_ref(0, binding) - m.fermi);
        if (K > 2 * omega0) {
            omega_min = 0.5f * (K + omega0 - approx::sqrt(K * (K - 2 * omega0)));
            w0 = omega0;
        }
        const float U = u_omega;
        if ((w0 > 0) && (omega_min > w0) && (omega_min < omega_max)) {
            const float inv_w0 = approx::div(1.0f, w0);
            const float f_min = inv_w0 * __logf(approx::div(omega_min - w0, omega_min));
            const float f_max = inv_w0 * __logf(approx::div(omega_max - w0, omega_max));
            omega = approx::div(-w0, expm1f(w0 * (f_min * (1 - U) + f_max * U)));
        } else {
            omega = approx::div(omega0 * omega_max, omega0 * (1 - U) + omega_max * U);
        }
    }
    if (binding < 0) {
        if (m.band_gap < 0) {
            // metals: no special treatment
        } else if (omega0 > m.band_gap) {
            binding = m.band_gap;
        } else {
            e.E -= omega0;   // optical phonon: direction untouched, no secondary
            return false;
        }
    }
    binding = max_ref(0, binding);

    const float Kp = e.E - m.fermi + 2 * binding;
    const float dK = binding + omega;
    const float cos_theta = approx::sqrt(approx::div(dK, Kp));
    const float sin_theta = approx::sqrt(1 - clampr(cos_theta * cos_theta, 0, 1));
    V3 s{d.x * cos_theta + n.x * sin_theta, d.y * cos_theta + n.y * sin_theta, d.z * cos_theta + n.z * sin_theta};
    s = approx::normalised(s);
    {
        const V3 uv = approx::make_unit_vec(2 * u_v1 - 1, u_v2);
        const float a = approx::sqrt(approx::div(binding, dK));
        s.x += a * uv.x;
        s.y += a * uv.y;
        s.z += a * uv.z;
    }
    s = approx::normalised(s);

    se->px = e.px;
    se->py = e.py;
    se->pz = e.pz;
    se->dx = s.x;
    se->dy = s.y;
    se->dz = s.z;
    se->E = m.fermi + omega - binding;
    se->mat = e.mat;
    se->last_tri = -1;
    se->tag = e.tag;
    se->uid = secondary_uid(e.uid, e.step);
    se->step = 0;

    e.E -= omega;
    e.dx = d.x - cos_theta * s.x;
    e.dy = d.y - cos_theta * s.y;
    e.dz = d.z - cos_theta * s.z;
    return true;
}

// Plasmon-decay rejection loop: at most this many rounds (the acceptance
// ratio sqrt(x^2 + x) / (x + 1/2) is above 1/2 for x > 0.08, so 64 rounds
// fail with probability far below one in 2^40); the last draw is kept then.
constexpr uint32_t kMaxPlasmonRounds = 64;

// full_penn<gpu, true>::execute (physics/full_penn.h:63-289) after the
// log-omega ICDF lookup (log_omega), with d = normalised(dir) and
// n = normalised(make_normal_vec(d, phi)) from the shared half.  Uniforms:
// block 1 x binding, y q, z q-normal azimuth, w single-excitation radius or
// the f < 0.1 plasmon draw; block 3 x, y the secondary's uniform_vector;
// blocks 4, 5, ... the plasmon rejection rounds (U1, U2, U3).
__device__ __forceinline__ bool penn_finish(const Physics& P, const Material& m, Electron& e, float log_omega,
                                            float logE, V3 d, V3 n, uint4 r1, Electron* se) {
    const float K = e.E;
    const float omega = __expf(log_omega);
    // ionisation table at (log K, log(omega / K), P)
    const float binding = table3d_rounddown(m.ion3, logE, __logf(approx::div(omega, K)), u01(r1.x));
    V3 sdir;
    float se_E;
    if (binding <= 0) {
        if (!(omega > m.band_gap)) {
            // sub-band-gap loss (longitudinal optical phonon): energy only; the
            // reference stores the direction it normalised
            e.dx = d.x;
            e.dy = d.y;
            e.dz = d.z;
            e.E = K - omega;
            return false;
        }
        // Fermi-sea excitation; q = hbar q / sqrt(2m) in eV^1/2
        const float q = table3d_get(m.q, logE, approx::div(omega, K), u01(r1.y));
        const float c1 = clampr(approx::div(omega + q * q, 2 * approx::sqrt(K) * q), -1, 1);
        const float s1 = approx::sqrt(1 - c1 * c1);
        const V3 q_dir = approx::normalised(V3{d.x * c1 + n.x * s1, d.y * c1 + n.y * s1, d.z * c1 + n.z * s1});
        const V3 q_normal = approx::normalised(approx::make_normal_vec(q_dir, u01(r1.z)));
        const float c2 = clampr(approx::div(2 * K - omega - q * q, 2 * approx::sqrt(K * (K - omega))), -1, 1);
        const float s2 = approx::sqrt(1 - c2 * c2);
        e.E = K - omega;
        e.dx = d.x * c2 + n.x * s2;
        e.dy = d.y * c2 + n.y * s2;
        e.dz = d.z * c2 + n.z * s2;
        const float k_fermi = approx::sqrt(m.fermi);
        const float k_fermi_omega = approx::sqrt(m.fermi + omega);
        if (q < k_fermi_omega - k_fermi) {
            // plasmon decay: x = E_i / omega from p(x) ~ sqrt(x (x + 1)) on [0, f]
            const float f = approx::div(m.fermi, omega);
            float x;
            if (f < 0.1f) {
                const float U = cbrtf(u01(r1.w));
                x = f * U * U;
            } else {
                const float lower = max_ref(0, f - 1);
                const float upper = f;
                const float d1 = upper - lower;
                const float d2 = upper * upper - lower * lower;
                const float alpha = approx::div(d2, d1 + d2);
                for (uint32_t k = 0;; ++k) {
                    const uint4 rk = draw(P.seed, e, 4 + k);
                    const float U1 = u01(rk.x);
                    const float U2 = u01(rk.y);
                    x = (U1 < alpha) ? approx::sqrt(d2 * U2 + lower * lower) : d1 * U2 + lower;
                    if (!(u01(rk.z) > approx::div(approx::sqrt(x * x + x), x + 0.5f)) || k + 1 == kMaxPlasmonRounds)
                        break;
                }
            }
            se_E = x * omega + omega;
            const uint4 r3 = draw(P.seed, e, 3);
            sdir = approx::make_unit_vec(2 * u01(r3.x) - 1, u01(r3.y));
        } else if (q < k_fermi_omega + k_fermi) {
            // single excitation from the annulus of allowed initial k around q
            const float ki_parr = approx::div(omega - q * q, 2 * q);
            const float kf_parr = ki_parr + q;
            const float ki_perp_min_sq = max_ref(0, m.fermi - kf_parr * kf_parr);
            const float ki_perp_max_sq = m.fermi - ki_parr * ki_parr;
            const float ki_perp_sq = max_ref(0, ki_perp_min_sq + (ki_perp_max_sq - ki_perp_min_sq) * u01(r1.w));
            const float kp = approx::sqrt(ki_perp_sq);
            const V3 ki{ki_parr * q_dir.x + kp * q_normal.x, ki_parr * q_dir.y + kp * q_normal.y,
                        ki_parr * q_dir.z + kp * q_normal.z};
            se_E = (ki.x * ki.x + ki.y * ki.y + ki.z * ki.z) + omega;
            sdir = V3{ki.x + q * q_dir.x, ki.y + q * q_dir.y, ki.z + q * q_dir.z};
        } else {
            return false;   // q too large for either: no secondary
        }
    } else {
        // inner-shell excitation (Ivanchenko angles, as kieft_inelastic)
        const float Kp = K - m.fermi + 2 * binding;
        const float dK = binding + omega;
        const float cos_theta = approx::sqrt(approx::div(dK, Kp));
        const float sin_theta = approx::sqrt(1 - clampr(cos_theta * cos_theta, 0, 1));
        V3 s{d.x * cos_theta + n.x * sin_theta, d.y * cos_theta + n.y * sin_theta, d.z * cos_theta + n.z * sin_theta};
        s = approx::normalised(s);
        const uint4 r3 = draw(P.seed, e, 3);
        const V3 uv = approx::make_unit_vec(2 * u01(r3.x) - 1, u01(r3.y));
        const float a = approx::sqrt(approx::div(binding, dK));
        s.x += a * uv.x;
        s.y += a * uv.y;
        s.z += a * uv.z;
        s = approx::normalised(s);
        se_E = m.fermi + omega - binding;
        sdir = s;
        e.E = K - omega;
        e.dx = d.x - cos_theta * s.x;
        e.dy = d.y - cos_theta * s.y;
        e.dz = d.z - cos_theta * s.z;
    }
    se->px = e.px;
    se->py = e.py;
    se->pz = e.pz;
    se->dx = sdir.x;
    se->dy = sdir.y;
    se->dz = sdir.z;
    se->E = se_E;
    se->mat = e.mat;
    se->last_tri = -1;
    se->tag = e.tag;
    se->uid = secondary_uid(e.uid, e.step);
    se->step = 0;
    return true;
}

// boundary_intersect<quantum transmission, refraction, no absorption>::execute
// (physics/boundary_intersect.h:40-156)
__device__ __forceinline__ int boundary(const Physics& P, Electron& e, float u) {
    int mi, mo;
    const V3 face = load_face(P.geo, e.last_tri, mi, mo);
    const V3 nd = approx::normalised(V3{e.dx, e.dy, e.dz});
    const V3 n = approx::normalised(face);
    const float cos_theta = dot(n, nd);
    int in, out;
    if (cos_theta > 0) {
        in = mi;
        out = mo;
    } else {
        in = mo;
        out = mi;
    }
    switch (out) {
    case kDetector:
        return kDetected;
    case kDetectorLT50:
        return e.E < 50 ? kDetected : kAlive;
    case kDetectorGE50:
        return e.E >= 50 ? kDetected : kAlive;
    case kTerminator:
        return kTerminated;
    case kMirror:
        e.dx = nd.x - 2 * n.x * cos_theta;
        e.dy = nd.y - 2 * n.y * cos_theta;
        e.dz = nd.z - 2 * n.z * cos_theta;
        return kAlive;
    case kNop:
        return kAlive;
    default:
        break;
    }
    float dU = 0;
    if (in >= 0) dU -= P.mat[in].barrier;
    if (out >= 0) dU += P.mat[out].barrier;
    if (e.E * cos_theta * cos_theta + dU > 0) {
        const float s = approx::sqrt(1 + approx::div(dU, e.E * cos_theta * cos_theta));
        const float T = approx::div(4 * s, (1 + s) * (1 + s));
        if (u < T) {
            e.dx = (nd.x - n.x * cos_theta) + s * n.x * cos_theta;
            e.dy = (nd.y - n.y * cos_theta) + s * n.y * cos_theta;
            e.dz = (nd.z - n.z * cos_theta) + s * n.z * cos_theta;
            e.E += dU;
            e.mat = out;
            return kAlive;
        }
    }
    e.dx = nd.x - 2 * n.x * cos_theta;
    e.dy = nd.y - 2 * n.y * cos_theta;
    e.dz = nd.z - 2 * n.z * cos_theta;
    return kAlive;
}

// A step's two log-IMFP lookups (table_1D::get, common/util/table_1D.inl:
// 66-80): from the interleaved pair table when both tables share one axis --
// the same index, fraction and lerps as two table1d_get calls, so the same
// values -- else one table1d_get each.
__device__ __forceinline__ void imfp_pair_get(const Material& m, float logE, float& in_v, float& el_v) {
    if (m.imfp_pair) {
        const Table1D& t = m.in_imfp;
        const float xi = (logE - t.x_min) * t.x_step;
        const int lo = clampi(floor_to_int(xi), 0, t.n - 2);
        const float4 v = __ldg(m.imfp_pair + lo);
        const float f = xi - float(lo);
        in_v = (1 - f) * v.x + f * v.y;
        el_v = (1 - f) * v.z + f * v.w;
    } else {
        in_v = table1d_get(m.in_imfp, logE);
        el_v = table1d_get(m.el_imfp, logE);
    }
}

// The init pass's termination test (drivers/cpu/cpu_driver.inl:73-92): outside
// the simulation domain, or inside a material with an energy outside
// [barrier + min_energy, barrier + max_energy].  A step that ends here draws no
// random numbers and changes nothing, so callers may apply it early.
__device__ __forceinline__ bool ends_at_init(const Physics& P, const Electron& e) {
    if (!in_domain(P.geo, V3{e.px, e.py, e.pz})) return true;
    if (e.mat >= 0) {
        const Material& m = P.mat[e.mat];
        if (e.E < m.barrier + P.min_energy || e.E > m.barrier + P.max_energy) return true;
    }
    return false;
}

// One pass of init -> intersect -> scatter (drivers/cpu/cpu_driver.inl:73-161,
// cpu_particle_manager.inl:214-235).  Uniforms of step k come from Philox
// blocks (k, 0) and (k, 1) of the electron's stream: block 0 x/y feed the
// inelastic/elastic free paths, z the ICDF probability (or the boundary
// transmission draw), w the scattering azimuth; block 1 the remaining four
// inelastic draws.  The mechanisms' log(E) is the init pass's log(E): the
// energy has not changed in between, so the value is the same.  kPenn
// selects the inelastic model at compile time (P.penn must agree), as the
// reference's physics_config.h does.
template <bool kPenn>
__device__ __forceinline__ int step(const Physics& P, Electron& e, int* event, Electron* se, bool* has_se,
                                    LeafCache cache = LeafCache{nullptr, 0}) {
    *event = kEvNone;
    *has_se = false;
    if (ends_at_init(P, e)) return kTerminated;
    const uint4 r0 = draw(P.seed, e, 0);
    int type = 0;
    float dist = P.geo.max_extent;
    float logE = 0;
    if (e.mat >= 0) {
        const Material& m = P.mat[e.mat];
        // The free-path sampling uses the hardware log2/exp2 approximations
        // (__logf / __expf: a few ulp, 2^-21 absolute for log near 1): the
        // paths only enter the statistics, and the table lookups that follow
        // are exact functions of the log E they are given.  A path that the
        // approximation would make slightly negative (U within 2^-21 of 1) is
        // taken as 0.
        logE = __logf(e.E);
        dist = __int_as_float(0x7f800000);
        // Mean free path exp(-log imfp) rather than 1 / exp(log imfp): the
        // same exponential sampling (scatter_list.h:106-132, random.h
        // exponential) without a division per mechanism.
        float in_lg, el_lg;
        imfp_pair_get(m, logE, in_lg, el_lg);
        {
            const float mfp = __expf(-in_lg);
            const float path = fmaxf(-mfp * __logf(u01(r0.x)), 0.0f);
            if (path < dist) {
                type = 1;
                dist = path;
            }
        }
        {
            const float mfp = __expf(-el_lg);
            const float path = fmaxf(-mfp * __logf(u01(r0.y)), 0.0f);
            if (path < dist) {
                type = 2;
                dist = path;
            }
        }
    }
    const V3 nd = normalised(V3{e.dx, e.dy, e.dz});
    int hit;
    const float tdist = propagate(P.geo, V3{e.px, e.py, e.pz}, nd, dist, e.last_tri, e.mat, &hit, cache);
    int status = kAlive;
    if (hit < 0) {
        e.px += nd.x * dist;
        e.py += nd.y * dist;
        e.pz += nd.z * dist;
        if (type != 0) {
            // Shared first half of both mechanisms (see elastic_finish).
            // Uniforms: block 0 z -> ICDF probability, w -> azimuth; block 1
            // -> binding, energy loss and the two unit-vector draws.
            e.last_tri = -1;
            const Material& m = P.mat[e.mat];
            const bool inel = (type == 1);
            const float tv = table2d_get(inel ? m.in_icdf : m.el_icdf, logE, u01(r0.z));
            const V3 n = approx::normalised(approx::make_normal_vec(nd, u01(r0.w)));
            if (!inel) {
                elastic_finish(m, e, tv, nd, n);
                *event = kEvElastic;
            } else {
                const uint4 r1 = draw(P.seed, e, 1);
                if constexpr (kPenn)
                    *has_se = penn_finish(P, m, e, tv, logE, nd, n, r1, se);
                else
                    *has_se = inelastic_finish(m, e, tv, nd, n, u01(r1.x), u01(r1.y), u01(r1.z), u01(r1.w), se);
                *event = kEvInelastic;
            }
        }
    } else {
        e.px += nd.x * tdist;
        e.py += nd.y * tdist;
        e.pz += nd.z * tdist;
        e.last_tri = hit;
        status = boundary(P, e, u01(r0.z));
        *event = kEvBoundary;
    }
    e.step += 1;
    return status;
}

}  // namespace dev
}  // namespace nbx
