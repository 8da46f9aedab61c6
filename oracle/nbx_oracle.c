/* CPU restatement of Nebula's electron-transport hot path (test infrastructure;
 * see nbx_oracle.h).  Compiled as C99 without -ffast-math and without FMA. */
#include "nbx_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define NBO_EPS (10.0f * 1.1920928955078125e-07f) /* config/data_types.h:55 */
#define NBO_PI 3.1415926535897932f                 /* config/config.h:32 */

/* ---------------------------------------------------------------------------
 * Philox4x32-10 (Salmon et al. SC'11): 10 rounds of two 32x32->64 multiplies
 * with the Weyl key schedule.
 * ------------------------------------------------------------------------- */
void nbo_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]) {
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        c0 = hi1 ^ c1 ^ k0;
        c1 = lo1;
        c2 = hi0 ^ c3 ^ k1;
        c3 = lo0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0;
    out[1] = c1;
    out[2] = c2;
    out[3] = c3;
}

/* Uniform in the open interval (0, 1): (k + 1/2) / 2^23 with k the top 23
 * bits; every step is exact in single precision. */
float nbo_u01(uint32_t x) { return (float)(x >> 9) * 1.1920928955078125e-07f + 5.9604644775390625e-08f; }

/* splitmix64 finaliser (S. Vigna) of (parent uid, parent step); top bit set
 * so secondaries never collide with primary uids (< 2^63). */
uint64_t nbo_secondary_uid(uint64_t parent_uid, uint32_t parent_step) {
    uint64_t z = parent_uid + 0x9E3779B97F4A7C15ull * ((uint64_t)parent_step + 1u);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z = z ^ (z >> 31);
    return z | (1ull << 63);
}

/* ---------------------------------------------------------------------------
 * Vector helpers (common/vector_math.h:9-206, CPU branches)
 * ------------------------------------------------------------------------- */
static float dot3(const float a[3], const float b[3]) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
static void cross3(const float a[3], const float b[3], float out[3]) {
    const float x = a[1] * b[2] - a[2] * b[1];
    const float y = a[2] * b[0] - a[0] * b[2];
    const float z = a[0] * b[1] - a[1] * b[0];
    out[0] = x;
    out[1] = y;
    out[2] = z;
}
/* normalise(a): a /= sqrt(a.a), where vec/real is vec * (1/real)
 * (vector_math.h:37-40,147-157) */
static void normalise3(float a[3]) {
    const float inv = 1.0f / sqrtf(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
    a[0] *= inv;
    a[1] *= inv;
    a[2] *= inv;
}
static float clampf_ref(float i, float lo, float hi) { return i < lo ? lo : (i > hi ? hi : i); } /* scalar_math.h:24 */
static int clampi_ref(int i, int lo, int hi) { return i < lo ? lo : (i > hi ? hi : i); }          /* scalar_math.h:19 */
static float minf_ref(float a, float b) { return (b < a) ? b : a; }                              /* std::min */
static float maxf_ref(float a, float b) { return (a < b) ? b : a; }                              /* std::max */

/* make_normal_vec (vector_math.h:171-186) */
static void make_normal_vec(const float dir[3], float phi, float out[3]) {
    const float az = atan2f(dir[1], dir[0]);
    const float sin_az = sinf(az), cos_az = cosf(az);
    const float unit_v[3] = {dir[2] * cos_az, dir[2] * sin_az, -sqrtf(dir[0] * dir[0] + dir[1] * dir[1])};
    float unit_u[3];
    cross3(unit_v, dir, unit_u);
    const float sin_phi = sinf(phi), cos_phi = cosf(phi);
    for (int i = 0; i < 3; ++i) out[i] = unit_u[i] * cos_phi + unit_v[i] * sin_phi;
}

/* make_unit_vec (vector_math.h:194-206) */
static void make_unit_vec(float cos_theta, float phi, float out[3]) {
    const float sin_phi = sinf(phi), cos_phi = cosf(phi);
    cos_theta = clampf_ref(cos_theta, -1.0f, 1.0f);
    const float sin_theta = sqrtf(1.0f - cos_theta * cos_theta);
    out[0] = sin_theta * cos_phi;
    out[1] = sin_theta * sin_phi;
    out[2] = cos_theta;
}

/* ---------------------------------------------------------------------------
 * Geometry
 * ------------------------------------------------------------------------- */
/* triangle::intersect_ray (core/triangle.inl:7-29) */
float nbo_triangle_intersect(const float tri[9], const float pos[3], const float dir[3]) {
    const float* r0 = tri;
    const float* e1 = tri + 3;
    const float* e2 = tri + 6;
    float pvec[3];
    cross3(dir, e2, pvec);
    const float det = dot3(e1, pvec);
    if (fabsf(det) < NBO_EPS) return -1;
    const float s[3] = {pos[0] - r0[0], pos[1] - r0[1], pos[2] - r0[2]};
    const float u = dot3(s, pvec) / det;
    if ((u < -NBO_EPS) || (u > 1 + NBO_EPS)) return -1;
    float qvec[3];
    cross3(s, e1, qvec);
    const float v = dot3(dir, qvec) / det;
    if ((v < -NBO_EPS) || (u + v > 1 + NBO_EPS)) return -1;
    const float t = dot3(e2, qvec) / det;
    if (t < 0) return -1;
    return t;
}

/* octree::in_domain (geometry/octree.inl:25-31) */
int nbo_in_domain(const nbo_geometry* g, const float p[3]) {
    return (p[0] > g->center[0] - g->half[0]) && (p[0] < g->center[0] + g->half[0]) &&
           (p[1] > g->center[1] - g->half[1]) && (p[1] < g->center[1] + g->half[1]) &&
           (p[2] > g->center[2] - g->half[2]) && (p[2] < g->center[2] + g->half[2]);
}

static int clz64(uint64_t x) { return __builtin_clzll(x); }

/* Instrumentation for the roofline's algorithmic bytes: octree words and
 * triangle records read by propagate (not thread-safe; single-threaded use). */
static uint64_t g_words_read = 0, g_tris_read = 0;
void nbo_geom_counters(uint64_t out[2]) {
    out[0] = g_words_read;
    out[1] = g_tris_read;
}
void nbo_geom_counters_reset(void) { g_words_read = g_tris_read = 0; }

/* octree::propagate (geometry/octree.inl:33-192) with AABB_intersect
 * (:212-220).  Triangles are identified by index; -1 is "none". */
void nbo_propagate(const nbo_geometry* g, const float start[3], const float dir[3], float distance,
                   int32_t ignore_tri, int32_t ignore_mat, float* out_dist, int32_t* out_tri) {
    const int32_t* od = g->octree_data;
    float cur[3] = {start[0], start[1], start[2]};
    float to_go = distance;
    uint64_t location = 1;
    do {
        float ax = g->center[0], ay = g->center[1], az = g->center[2], aw = 1;
        int index = 0;
        for (int i = 60 - clz64(location); i >= 0; i -= 3) {
            const unsigned octant = (unsigned)(location >> i) & 7u;
            index = od[index + (int)octant];
            ++g_words_read;
            ax += aw * g->half[0] * ((float)(octant & 1) - 0.5f);
            ay += aw * g->half[1] * ((float)((octant & 2) >> 1) - 0.5f);
            az += aw * g->half[2] * ((float)((octant & 4) >> 2) - 0.5f);
            aw *= 0.5f;
        }
        while (index >= 0) {
            unsigned octant = 0;
            octant ^= (cur[0] > ax) ? 1u : 0u;
            octant ^= (cur[1] > ay) ? 2u : 0u;
            octant ^= (cur[2] > az) ? 4u : 0u;
            location = (location << 3) | octant;
            index = od[index + (int)octant];
            ++g_words_read;
            ax += aw * g->half[0] * ((float)(octant & 1) - 0.5f);
            ay += aw * g->half[1] * ((float)((octant & 2) >> 1) - 0.5f);
            az += aw * g->half[2] * ((float)((octant & 4) >> 2) - 0.5f);
            aw *= 0.5f;
        }
        index = -index;

        float intersect;
        int target;
        {
            const float hx = aw * g->half[0], hy = aw * g->half[1], hz = aw * g->half[2];
            const float tx = (ax + copysignf(hx + NBO_EPS, dir[0]) - cur[0]) / dir[0];
            const float ty = (ay + copysignf(hy + NBO_EPS, dir[1]) - cur[1]) / dir[1];
            const float tz = (az + copysignf(hz + NBO_EPS, dir[2]) - cur[2]) / dir[2];
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
            const int ti = od[index++];
            ++g_words_read;
            if (ti < 0) break;
            if (ti == ignore_tri) continue;
            ++g_tris_read;
            const float* tri = g->tri + 9 * (size_t)ti;
            float n[3];
            cross3(tri + 3, tri + 6, n);
            const int mat_out = (dot3(n, dir) < 0) ? g->tri_mat[2 * ti] : g->tri_mat[2 * ti + 1];
            if (mat_out == ignore_mat) continue;
            const float t = nbo_triangle_intersect(tri, cur, dir);
            if ((t > 0) && (t <= intersect + NBO_EPS)) {
                intersect = t;
                target = ti;
            }
        }
        if (intersect >= to_go) {
            *out_dist = distance;
            *out_tri = -1;
            return;
        } else if (target >= 0) {
            *out_dist = distance - to_go + intersect;
            *out_tri = target;
            return;
        }
        to_go -= intersect;
        cur[0] += dir[0] * intersect;
        cur[1] += dir[1] * intersect;
        cur[2] += dir[2] * intersect;

        const unsigned mask = (unsigned)(-target);
        unsigned value;
        if (mask == 1)
            value = (dir[0] >= 0) ? 0u : 1u;
        else if (mask == 2)
            value = (dir[1] >= 0) ? 0u : 2u;
        else
            value = (dir[2] >= 0) ? 0u : 4u;
        while (location > 1) {
            if ((location & mask) == value) {
                location ^= mask;
                break;
            }
            location >>= 3;
        }
    } while (location > 1);
    *out_dist = distance;
    *out_tri = -1;
}

void nbo_propagate_batch(const nbo_geometry* g, const float* pos, const float* dir, const float* dist,
                         const int32_t* ignore_tri, const int32_t* ignore_mat, int64_t n, float* out_dist,
                         int32_t* out_tri) {
    for (int64_t i = 0; i < n; ++i)
        nbo_propagate(g, pos + 3 * i, dir + 3 * i, dist[i], ignore_tri[i], ignore_mat[i], out_dist + i, out_tri + i);
}

/* ---------------------------------------------------------------------------
 * Tables (common/util/table_1D.inl:66-80, table_2D.inl:74-104)
 * ------------------------------------------------------------------------- */
float nbo_table1d_get(const nbo_table1d* t, float x) {
    const float x_index = (x - t->x_min) * t->x_step;
    const int low = clampi_ref((int)floorf(x_index), 0, t->n - 2);
    const float lo = t->data[low];
    const float hi = t->data[low + 1];
    const float f = x_index - (float)low;
    return (1 - f) * lo + f * hi;
}

float nbo_table2d_get(const nbo_table2d* t, float x, float y) {
    const float xi = (x - t->x_min) * t->x_step;
    const float yi = (y - t->y_min) * t->y_step;
    const int lx = clampi_ref((int)floorf(xi), 0, t->w - 2);
    const int ly = clampi_ref((int)floorf(yi), 0, t->h - 2);
    const float v00 = t->data[(size_t)lx * t->h + ly];
    const float v10 = t->data[(size_t)(lx + 1) * t->h + ly];
    const float v01 = t->data[(size_t)lx * t->h + ly + 1];
    const float v11 = t->data[(size_t)(lx + 1) * t->h + ly + 1];
    const float fx = xi - (float)lx;
    const float fy = yi - (float)ly;
    return (1 - fx) * (1 - fy) * v00 + fx * (1 - fy) * v10 + (1 - fx) * fy * v01 + fx * fy * v11;
}

float nbo_table2d_get_rounddown(const nbo_table2d* t, float x, float y) {
    const float xi = (x - t->x_min) * t->x_step;
    const float yi = (y - t->y_min) * t->y_step;
    const int lx = clampi_ref((int)floorf(xi), 0, t->w - 1);
    const int ly = clampi_ref((int)floorf(yi), 0, t->h - 1);
    return t->data[(size_t)lx * t->h + ly];
}

/* table_3D::get / get_rounddown (common/util/table_3D.inl:79-122) */
static float t3at(const nbo_table3d* t, int i, int j, int k) { return t->data[((size_t)i * t->h + j) * t->d + k]; }

float nbo_table3d_get(const nbo_table3d* t, float x, float y, float z) {
    const float x_index = (x - t->x_min) * t->x_step;
    const float y_index = (y - t->y_min) * t->y_step;
    const float z_index = (z - t->z_min) * t->z_step;
    const int low_x = clampi_ref((int)floorf(x_index), 0, t->w - 2);
    const int low_y = clampi_ref((int)floorf(y_index), 0, t->h - 2);
    const int low_z = clampi_ref((int)floorf(z_index), 0, t->d - 2);
    const float v000 = t3at(t, low_x, low_y, low_z);
    const float v100 = t3at(t, low_x + 1, low_y, low_z);
    const float v010 = t3at(t, low_x, low_y + 1, low_z);
    const float v110 = t3at(t, low_x + 1, low_y + 1, low_z);
    const float v001 = t3at(t, low_x, low_y, low_z + 1);
    const float v101 = t3at(t, low_x + 1, low_y, low_z + 1);
    const float v011 = t3at(t, low_x, low_y + 1, low_z + 1);
    const float v111 = t3at(t, low_x + 1, low_y + 1, low_z + 1);
    const float frac_x = x_index - (float)low_x;
    const float frac_y = y_index - (float)low_y;
    const float frac_z = z_index - (float)low_z;
    return (1 - frac_x) * (1 - frac_y) * (1 - frac_z) * v000 + frac_x * (1 - frac_y) * (1 - frac_z) * v100 +
           (1 - frac_x) * frac_y * (1 - frac_z) * v010 + frac_x * frac_y * (1 - frac_z) * v110 +
           (1 - frac_x) * (1 - frac_y) * frac_z * v001 + frac_x * (1 - frac_y) * frac_z * v101 +
           (1 - frac_x) * frac_y * frac_z * v011 + frac_x * frac_y * frac_z * v111;
}

float nbo_table3d_get_rounddown(const nbo_table3d* t, float x, float y, float z) {
    const float x_index = (x - t->x_min) * t->x_step;
    const float y_index = (y - t->y_min) * t->y_step;
    const float z_index = (z - t->z_min) * t->z_step;
    const int low_x = clampi_ref((int)floorf(x_index), 0, t->w - 1);
    const int low_y = clampi_ref((int)floorf(y_index), 0, t->h - 1);
    const int low_z = clampi_ref((int)floorf(z_index), 0, t->d - 1);
    return t3at(t, low_x, low_y, low_z);
}

/* ---------------------------------------------------------------------------
 * Physics
 * ------------------------------------------------------------------------- */
/* kieft_elastic::execute (physics/kieft/elastic.h:68-115) */
void nbo_elastic(const nbo_material* m, nbo_electron* e, float u_cos, float u_phi) {
    const float x = logf(e->E);
    const float cos_theta = clampf_ref(nbo_table2d_get(&m->el_icdf, x, u_cos), -1, 1);
    const float sin_theta = sqrtf(1 - cos_theta * cos_theta);
    normalise3(e->dir);
    float nd[3];
    make_normal_vec(e->dir, (2 * NBO_PI) * u_phi, nd);
    normalise3(nd);
    for (int i = 0; i < 3; ++i) e->dir[i] = e->dir[i] * cos_theta + nd[i] * sin_theta;
    if (e->E < 200)
        e->E -= minf_ref(50e-3f, m->phonon_loss);
    else
        e->E -= m->recoil_const * (1 - cos_theta) * e->E;
}

/* kieft_inelastic::execute (physics/kieft/inelastic.h:69-206), all options on */
int nbo_inelastic(const nbo_material* m, nbo_electron* e, const float u[6], nbo_electron* se) {
    const float K = e->E;
    const float omega0 = expf(nbo_table2d_get(&m->in_icdf, logf(K), u[0]));
    float binding = nbo_table2d_get_rounddown(&m->ion, logf(omega0), u[1]);
    float omega;
    {
        const float omega_max = 0.5f * (K + omega0 - m->fermi);
        float omega_min = omega0;
        float w0 = minf_ref(omega0 - 1, maxf_ref(0, binding) - m->fermi);
        if (K > 2 * omega0) {
            omega_min = 0.5f * (K + omega0 - sqrtf(K * (K - 2 * omega0)));
            w0 = omega0;
        }
        const float U = u[2];
        if ((w0 > 0) && (omega_min > w0) && (omega_min < omega_max)) {
            const float f_min = 1 / w0 * logf((omega_min - w0) / omega_min);
            const float f_max = 1 / w0 * logf((omega_max - w0) / omega_max);
            omega = -w0 / expm1f(w0 * (f_min * (1 - U) + f_max * U));
        } else {
            omega = omega0 * omega_max / (omega0 * (1 - U) + omega_max * U);
        }
    }
    if (binding < 0) {
        if (m->band_gap < 0) {
            /* metals: no special treatment */
        } else if (omega0 > m->band_gap) {
            binding = m->band_gap;
        } else {
            e->E -= omega0;
            return 0;
        }
    }
    binding = maxf_ref(0, binding);

    normalise3(e->dir);
    float nd[3];
    make_normal_vec(e->dir, (2 * NBO_PI) * u[3], nd);
    normalise3(nd);
    const float _K = e->E - m->fermi + 2 * binding;
    const float dK = binding + omega;
    const float cos_theta = sqrtf(dK / _K);
    const float sin_theta = sqrtf(1 - clampf_ref(cos_theta * cos_theta, 0, 1));
    float sd[3];
    for (int i = 0; i < 3; ++i) sd[i] = e->dir[i] * cos_theta + nd[i] * sin_theta;
    normalise3(sd);
    {
        float uv[3];
        make_unit_vec(2 * u[4] - 1, (2 * NBO_PI) * u[5], uv);
        const float a = sqrtf(binding / dK);
        for (int i = 0; i < 3; ++i) sd[i] += a * uv[i];
    }
    normalise3(sd);

    se->E = m->fermi + omega - binding;
    memcpy(se->pos, e->pos, sizeof se->pos);
    memcpy(se->dir, sd, sizeof se->dir);
    se->mat = e->mat;
    se->last_tri = -1;
    se->tag = e->tag;
    se->uid = nbo_secondary_uid(e->uid, e->step);
    se->step = 0;

    e->E -= omega;
    for (int i = 0; i < 3; ++i) e->dir[i] -= cos_theta * sd[i];
    return 1;
}

static void philox_block(const nbo_params* p, const nbo_electron* e, uint32_t block, uint32_t out[4]) {
    const uint32_t key[2] = {p->seed, 0u};
    const uint32_t c[4] = {e->step, block, (uint32_t)e->uid, (uint32_t)(e->uid >> 32)};
    nbo_philox4x32_10(c, key, out);
}

/* full_penn<cpu, true>::execute (physics/full_penn.h:63-289).  Uniform slots
 * (shared with the GPU): omega ICDF <- block 0 z (done by the caller),
 * primary normal azimuth <- block 0 w (u_phi), binding <- block 1 x, q <-
 * block 1 y, q-normal azimuth <- block 1 z, single-excitation radius or the
 * f < 0.1 plasmon draw <- block 1 w, secondary uniform_vector <- block 3 x, y,
 * plasmon rejection round k <- block 4 + k (x, y, z), at most 64 rounds. */
int nbo_penn_inelastic(const nbo_material* m, const nbo_params* p, nbo_electron* e, float log_omega, float u_phi,
                       const uint32_t r1[4], nbo_electron* se) {
    const float K = e->E;
    const float omega = expf(log_omega);
    const float binding = nbo_table3d_get_rounddown(&m->ion3, logf(K), logf(omega / K), nbo_u01(r1[0]));
    normalise3(e->dir);
    float sdir[3];
    float se_E;
    if (binding <= 0) {
        if (!(omega > m->band_gap)) {
            e->E -= omega; /* sub-band-gap loss: energy only */
            return 0;
        }
        const float q = nbo_table3d_get(&m->q, logf(K), omega / K, nbo_u01(r1[1]));
        float prim_normal[3];
        make_normal_vec(e->dir, (2 * NBO_PI) * u_phi, prim_normal);
        normalise3(prim_normal);
        float q_dir[3], q_normal[3];
        {
            const float c = clampf_ref((omega + q * q) / (2 * sqrtf(K) * q), -1, 1);
            const float sn = sqrtf(1 - c * c);
            for (int i = 0; i < 3; ++i) q_dir[i] = e->dir[i] * c + prim_normal[i] * sn;
            normalise3(q_dir);
            make_normal_vec(q_dir, (2 * NBO_PI) * nbo_u01(r1[2]), q_normal);
            normalise3(q_normal);
        }
        const float c2 = clampf_ref((2 * K - omega - q * q) / (2 * sqrtf(K * (K - omega))), -1, 1);
        const float s2 = sqrtf(1 - c2 * c2);
        e->E -= omega;
        for (int i = 0; i < 3; ++i) e->dir[i] = e->dir[i] * c2 + prim_normal[i] * s2;
        const float k_fermi = sqrtf(m->fermi);
        const float k_fermi_omega = sqrtf(m->fermi + omega);
        if (q < k_fermi_omega - k_fermi) {
            /* plasmon decay */
            const float f = m->fermi / omega;
            float x;
            if (f < 0.1f) {
                const float U = cbrtf(nbo_u01(r1[3]));
                x = f * U * U;
            } else {
                const float lower = maxf_ref(0, f - 1);
                const float upper = f;
                const float d1 = upper - lower;
                const float d2 = upper * upper - lower * lower;
                const float alpha = d2 / (d1 + d2);
                for (uint32_t k = 0;; ++k) {
                    uint32_t rk[4];
                    philox_block(p, e, 4 + k, rk);
                    const float U1 = nbo_u01(rk[0]);
                    const float U2 = nbo_u01(rk[1]);
                    x = (U1 < alpha) ? sqrtf(d2 * U2 + lower * lower) : d1 * U2 + lower;
                    if (!(nbo_u01(rk[2]) > sqrtf(x * x + x) / (x + 0.5f)) || k + 1 == 64) break;
                }
            }
            se_E = x * omega + omega;
            uint32_t r3[4];
            philox_block(p, e, 3, r3);
            make_unit_vec(2 * nbo_u01(r3[0]) - 1, (2 * NBO_PI) * nbo_u01(r3[1]), sdir);
        } else if (q < k_fermi_omega + k_fermi) {
            /* single excitation */
            const float ki_parr = (omega - q * q) / (2 * q);
            const float kf_parr = ki_parr + q;
            const float ki_perp_min_sq = maxf_ref(0, m->fermi - kf_parr * kf_parr);
            const float ki_perp_max_sq = m->fermi - ki_parr * ki_parr;
            const float ki_perp_sq =
                maxf_ref(0, ki_perp_min_sq + (ki_perp_max_sq - ki_perp_min_sq) * nbo_u01(r1[3]));
            float ki[3];
            for (int i = 0; i < 3; ++i) ki[i] = ki_parr * q_dir[i] + sqrtf(ki_perp_sq) * q_normal[i];
            se_E = (ki[0] * ki[0] + ki[1] * ki[1] + ki[2] * ki[2]) + omega;
            for (int i = 0; i < 3; ++i) sdir[i] = ki[i] + q * q_dir[i];
        } else {
            return 0;
        }
    } else {
        /* inner-shell excitation */
        float nd[3];
        make_normal_vec(e->dir, (2 * NBO_PI) * u_phi, nd);
        normalise3(nd);
        const float _K = K - m->fermi + 2 * binding;
        const float dK = binding + omega;
        const float cos_theta = sqrtf(dK / _K);
        const float sin_theta = sqrtf(1 - clampf_ref(cos_theta * cos_theta, 0, 1));
        for (int i = 0; i < 3; ++i) sdir[i] = e->dir[i] * cos_theta + nd[i] * sin_theta;
        normalise3(sdir);
        {
            uint32_t r3[4];
            philox_block(p, e, 3, r3);
            float uv[3];
            make_unit_vec(2 * nbo_u01(r3[0]) - 1, (2 * NBO_PI) * nbo_u01(r3[1]), uv);
            const float a = sqrtf(binding / dK);
            for (int i = 0; i < 3; ++i) sdir[i] += a * uv[i];
        }
        normalise3(sdir);
        se_E = m->fermi + omega - binding;
        e->E -= omega;
        for (int i = 0; i < 3; ++i) e->dir[i] -= cos_theta * sdir[i];
    }
    se->E = se_E;
    memcpy(se->pos, e->pos, sizeof se->pos);
    memcpy(se->dir, sdir, sizeof se->dir);
    se->mat = e->mat;
    se->last_tri = -1;
    se->tag = e->tag;
    se->uid = nbo_secondary_uid(e->uid, e->step);
    se->step = 0;
    return 1;
}

/* special_materials (core/cpu_material_manager.h:82-91) */
enum { SM_NOP = -128, SM_TERMINATOR = -127, SM_DETECTOR = -126, SM_DETECTOR_LT50 = -125, SM_DETECTOR_GE50 = -124,
       SM_VACUUM = -123, SM_MIRROR = -122 };

/* boundary_intersect<true, true, false>::execute (physics/boundary_intersect.h:40-156) */
int nbo_boundary(const nbo_geometry* g, const nbo_material* mats, nbo_electron* e, float u) {
    const int32_t ti = e->last_tri;
    const float* tri = g->tri + 9 * (size_t)ti;
    float nd[3] = {e->dir[0], e->dir[1], e->dir[2]};
    normalise3(nd);
    float n[3];
    cross3(tri + 3, tri + 6, n);
    normalise3(n);
    const float cos_theta = dot3(n, nd);
    int in, out;
    if (cos_theta > 0) {
        in = g->tri_mat[2 * ti];
        out = g->tri_mat[2 * ti + 1];
    } else {
        in = g->tri_mat[2 * ti + 1];
        out = g->tri_mat[2 * ti];
    }
    switch (out) {
    case SM_DETECTOR:
        return NBO_DETECTED;
    case SM_DETECTOR_LT50:
        return e->E < 50 ? NBO_DETECTED : NBO_ALIVE;
    case SM_DETECTOR_GE50:
        return e->E >= 50 ? NBO_DETECTED : NBO_ALIVE;
    case SM_TERMINATOR:
        return NBO_TERMINATED;
    case SM_MIRROR:
        for (int i = 0; i < 3; ++i) e->dir[i] = nd[i] - 2 * n[i] * cos_theta;
        return NBO_ALIVE;
    case SM_NOP:
        return NBO_ALIVE;
    default:
        break;
    }
    float dU = 0;
    if (in >= 0) dU -= mats[in].barrier;
    if (out >= 0) dU += mats[out].barrier;
    if (e->E * cos_theta * cos_theta + dU > 0) {
        const float s = sqrtf(1 + dU / (e->E * cos_theta * cos_theta));
        const float T = 4 * s / ((1 + s) * (1 + s));
        if (u < T) {
            for (int i = 0; i < 3; ++i) e->dir[i] = (nd[i] - n[i] * cos_theta) + s * n[i] * cos_theta;
            e->E += dU;
            e->mat = out;
            return NBO_ALIVE;
        }
    }
    for (int i = 0; i < 3; ++i) e->dir[i] = nd[i] - 2 * n[i] * cos_theta;
    return NBO_ALIVE;
}

/* ---------------------------------------------------------------------------
 * Driver step (drivers/cpu/cpu_driver.inl:73-161, cpu_particle_manager.inl:214-235)
 * ------------------------------------------------------------------------- */
int nbo_step(const nbo_geometry* g, const nbo_material* mats, const nbo_params* p, nbo_electron* e, int* event,
             nbo_electron* se, int* has_se) {
    *event = NBO_EV_NONE;
    *has_se = 0;
    if (!nbo_in_domain(g, e->pos)) return NBO_TERMINATED;

    uint32_t r0[4], r1[4];
    {
        const uint32_t key[2] = {p->seed, 0u};
        const uint32_t c0[4] = {e->step, 0u, (uint32_t)e->uid, (uint32_t)(e->uid >> 32)};
        nbo_philox4x32_10(c0, key, r0);
    }
    int type = 0;
    float dist = g->max_extent;
    if (e->mat >= 0) {
        const nbo_material* m = &mats[e->mat];
        if (e->E < m->barrier + p->min_energy || e->E > m->barrier + p->max_energy) return NBO_TERMINATED;
        /* scatter_list::sample_path (core/scatter_list.h:106-112,148-162):
         * inelastic first, then elastic; exponential(tau) = -tau*log(U)
         * (common/util/random.h:80-83) */
        const float logE = logf(e->E);
        dist = INFINITY;
        {
            const float imfp = expf(nbo_table1d_get(&m->in_imfp, logE));
            const float path = -(1 / imfp) * logf(nbo_u01(r0[0]));
            if (path < dist) {
                type = 1;
                dist = path;
            }
        }
        {
            const float imfp = expf(nbo_table1d_get(&m->el_imfp, logE));
            const float path = -(1 / imfp) * logf(nbo_u01(r0[1]));
            if (path < dist) {
                type = 2;
                dist = path;
            }
        }
    }
    float nd[3] = {e->dir[0], e->dir[1], e->dir[2]};
    normalise3(nd);
    float t_dist;
    int32_t t_idx;
    nbo_propagate(g, e->pos, nd, dist, e->last_tri, e->mat, &t_dist, &t_idx);
    int status = NBO_ALIVE;
    if (t_idx < 0) {
        for (int i = 0; i < 3; ++i) e->pos[i] += nd[i] * dist;
        if (type == 2) {
            e->last_tri = -1;
            nbo_elastic(&mats[e->mat], e, nbo_u01(r0[2]), nbo_u01(r0[3]));
            *event = NBO_EV_ELASTIC;
        } else if (type == 1) {
            e->last_tri = -1;
            uint32_t r1c[4] = {e->step, 1u, (uint32_t)e->uid, (uint32_t)(e->uid >> 32)};
            const uint32_t key[2] = {p->seed, 0u};
            nbo_philox4x32_10(r1c, key, r1);
            if (p->penn) {
                /* full_penn: log omega ICDF <- block 0 z, the rest as listed
                 * at nbo_penn_inelastic */
                const float log_omega = nbo_table2d_get(&mats[e->mat].in_icdf, logf(e->E), nbo_u01(r0[2]));
                *has_se = nbo_penn_inelastic(&mats[e->mat], p, e, log_omega, nbo_u01(r0[3]), r1, se);
            } else {
                /* slots: omega' ICDF <- block 0 z, binding <- block 1 x, energy
                 * loss <- block 1 y, azimuth <- block 0 w, unit vector <- block
                 * 1 z, w */
                const float u[6] = {nbo_u01(r0[2]), nbo_u01(r1[0]), nbo_u01(r1[1]),
                                    nbo_u01(r0[3]), nbo_u01(r1[2]), nbo_u01(r1[3])};
                *has_se = nbo_inelastic(&mats[e->mat], e, u, se);
            }
            *event = NBO_EV_INELASTIC;
        }
    } else {
        for (int i = 0; i < 3; ++i) e->pos[i] += nd[i] * t_dist;
        e->last_tri = t_idx;
        status = nbo_boundary(g, mats, e, nbo_u01(r0[2]));
        *event = NBO_EV_BOUNDARY;
    }
    e->step += 1;
    return status;
}

/* Whole cascades, one primary at a time (simple_cpu_driver.h:54-62 order:
 * the primary first, then its secondaries in creation order). */
int nbo_run(const nbo_geometry* g, const nbo_material* mats, const nbo_params* p, const float* primaries,
            const uint32_t* tags, uint64_t uid_base, uint64_t n, void* records, uint64_t capacity,
            uint32_t* se_count, uint32_t* bse_count, nbo_counts* c) {
    memset(c, 0, sizeof *c);
    size_t cap = 64, len = 0;
    nbo_electron* stack = (nbo_electron*)malloc(cap * sizeof *stack);
    if (!stack) return -1;
    for (uint64_t i = 0; i < n; ++i) {
        nbo_electron e;
        memcpy(e.pos, primaries + 7 * i, 12);
        memcpy(e.dir, primaries + 7 * i + 3, 12);
        e.E = primaries[7 * i + 6];
        e.mat = SM_VACUUM;
        e.last_tri = -1;
        e.tag = tags[i];
        e.uid = uid_base + i;
        e.step = 0;
        len = 0;
        stack[len++] = e;
        size_t head = 0;
        c->n_primaries++;
        while (head < len) {
            nbo_electron cur = stack[head++];
            for (;;) {
                int ev, has_se;
                nbo_electron se;
                const int st = nbo_step(g, mats, p, &cur, &ev, &se, &has_se);
                c->n_steps++;
                if (ev == NBO_EV_ELASTIC) c->n_elastic++;
                if (ev == NBO_EV_INELASTIC) c->n_inelastic++;
                if (ev == NBO_EV_BOUNDARY) c->n_boundary++;
                if (has_se) {
                    if (len == cap) {
                        cap *= 2;
                        nbo_electron* ns = (nbo_electron*)realloc(stack, cap * sizeof *stack);
                        if (!ns) {
                            free(stack);
                            return -1;
                        }
                        stack = ns;
                    }
                    stack[len++] = se;
                    c->n_secondaries++;
                }
                if (st == NBO_ALIVE) continue;
                if (st == NBO_DETECTED) {
                    c->n_detected++;
                    if (cur.E < 50) {
                        if (se_count) se_count[i]++;
                    } else {
                        if (bse_count) bse_count[i]++;
                    }
                    if (records && c->n_detected - c->n_dropped_records <= capacity) {
                        float* r = (float*)((char*)records + 36 * (c->n_detected - c->n_dropped_records - 1));
                        r[0] = cur.pos[0];
                        r[1] = cur.pos[1];
                        r[2] = cur.pos[2];
                        r[3] = cur.dir[0];
                        r[4] = cur.dir[1];
                        r[5] = cur.dir[2];
                        r[6] = cur.E;
                        memcpy(r + 7, &cur.tag, 4);
                        memset(r + 8, 0, 4);
                    } else if (records) {
                        c->n_dropped_records++;
                    }
                }
                break;
            }
        }
    }
    free(stack);
    return 0;
}
