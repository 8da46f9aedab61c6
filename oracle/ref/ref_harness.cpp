// Test infrastructure: C-ABI entry points into the reference's own CPU code,
// compiled unmodified from its source tree (see oracle/Makefile).  Used only
// by tests/ and by bench.py's CPU-baseline leg to check and time the product.
//
//   nbref_build_octree   octree_builder::linearized_octree (octree_builder.cpp:252-352)
//   nbref_propagate      octree<false>::propagate (geometry/octree.inl:33-192)
//   nbref_material_*     material<scatter_list<inelastic, kieft_elastic>>::create
//                        and the reference table lookups (table_1D.inl:66, table_2D.inl:74,97,
//                        table_3D.inl:79,114)
//
// Built twice: with the Kieft inelastic model (kieft_physics_config.h, the
// commented block of physics_config.h:27-33) as libnbref.so, and with
// -DNBREF_PENN against the reference's own physics_config.h (full Penn, the
// stock build) as libnbref_penn.so.
//   nbref_run            cpu_mt_main.cpp:158-203 (one simple_cpu_driver per thread pulling
//                        one primary at a time), optionally counting events
#include <atomic>
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <random>
#include <thread>
#include <vector>

#ifdef NBREF_PENN
#include "config/config.h"   // as cpu_mt_main.cpp includes it before physics_config.h
#include "physics_config.h"
#else
#include "kieft_physics_config.h"
#endif
#include "common/work_pool.h"
#include "drivers/cpu/simple_cpu_driver.h"
#include "geometry/octree.h"
#include "io/load_pri_file.h"
#include "io/load_tri_file.h"

using geometry_t = nbl::geometry::octree<false>;
using material_t = material<scatter_physics<false>>;
using elastic_t = nbl::scatter::kieft_elastic<false, true, true>;
#ifdef NBREF_PENN
using inelastic_t = nbl::scatter::full_penn<false, true>;
#else
using inelastic_t = nbl::scatter::kieft_inelastic<false, true, true, true, true>;
#endif

// The reference classes keep their tables private and befriend every
// specialisation of their own template; these two explicit specialisations
// (never used as physics) read the tables through that friendship.
namespace nbl { namespace scatter {
template<>
class kieft_elastic<true, false, false> {
public:
    static util::table_1D<real, false> const& imfp(elastic_t const& e) { return e._log_imfp_table; }
    static util::table_2D<real, false> const& icdf(elastic_t const& e) { return e._icdf_table; }
    static real phonon(elastic_t const& e) { return e._phonon_loss; }
    static real recoil(elastic_t const& e) { return e._recoil_const; }
};
#ifdef NBREF_PENN
template<>
class full_penn<true, false> {
public:
    static util::table_1D<real, false> const& imfp(inelastic_t const& e) { return e._log_imfp_table; }
    static util::table_2D<real, false> const& icdf(inelastic_t const& e) { return e._log_omega_icdf_table; }
    static util::table_3D<real, false> const& q(inelastic_t const& e) { return e._q_icdf_table; }
    static util::table_3D<real, false> const& ion3(inelastic_t const& e) { return e._ionisation_table; }
    static real fermi(inelastic_t const& e) { return e._fermi; }
    static real gap(inelastic_t const& e) { return e._band_gap; }
};
#else
template<>
class kieft_inelastic<true, false, false, false, false> {
public:
    static util::table_1D<real, false> const& imfp(inelastic_t const& e) { return e._log_imfp_table; }
    static util::table_2D<real, false> const& icdf(inelastic_t const& e) { return e._log_icdf_table; }
    static util::table_2D<real, false> const& ion(inelastic_t const& e) { return e._ionisation_table; }
    static real fermi(inelastic_t const& e) { return e._fermi; }
    static real gap(inelastic_t const& e) { return e._band_gap; }
};
#endif
}}  // namespace nbl::scatter
// The table classes befriend their other-device counterpart; these
// specialisations (never instantiated on a device in this CPU build) read
// the axis parameters x_min/x_step/y_min/y_step through that friendship.
namespace nbl { namespace util {
template<>
class table_1D<real, true> {
public:
    static void scales(table_1D<real, false> const& t, float out[4]) {
        out[0] = t._x_min; out[1] = t._x_step; out[2] = 0; out[3] = 0;
    }
};
template<>
class table_2D<real, true> {
public:
    static void scales(table_2D<real, false> const& t, float out[4]) {
        out[0] = t._x_min; out[1] = t._x_step; out[2] = t._y_min; out[3] = t._y_step;
    }
};
template<>
class table_3D<real, true> {
public:
    static void scales(table_3D<real, false> const& t, float out[6]) {
        out[0] = t._x_min; out[1] = t._x_step; out[2] = t._y_min; out[3] = t._y_step;
        out[4] = t._z_min; out[5] = t._z_step;
    }
};
}}  // namespace nbl::util
using el_spy = nbl::scatter::kieft_elastic<true, false, false>;
#ifdef NBREF_PENN
using in_spy = nbl::scatter::full_penn<true, false>;
#else
using in_spy = nbl::scatter::kieft_inelastic<true, false, false, false, false>;
#endif

namespace {
// Byte-layout mirrors of two reference classes, read with memcpy.
struct triangle_bytes {
    int32_t mat_in, mat_out;
    float r0[3], e1[3], e2[3];
};
static_assert(sizeof(triangle_bytes) == sizeof(triangle), "triangle layout");
struct octree_bytes {
    int* data;
    triangle* tris;
    float c[3], h[3], max_extent;
};
static_assert(sizeof(octree_bytes) == sizeof(geometry_t), "octree layout");

std::vector<triangle> make_tris(const float* verts, const int32_t* mats, int64_t n) {
    std::vector<triangle> t;
    t.reserve(size_t(n));
    for (int64_t i = 0; i < n; ++i) {
        const float* v = verts + 9 * i;
        t.push_back(triangle({v[0], v[1], v[2]}, {v[3], v[4], v[5]}, {v[6], v[7], v[8]}, mats[2 * i], mats[2 * i + 1]));
    }
    return t;
}

template<typename S, typename I, typename G>
class counting_driver : public nbl::drivers::cpu_driver<S, I, G> {
public:
    using base_t = nbl::drivers::cpu_driver<S, I, G>;
    counting_driver(I inter, typename base_t::material_manager_t const& m, G const& g, real mn, real mx,
                    typename base_t::seed_t seed)
        : base_t(inter, m, g, mn, mx, seed) {}
    uint64_t n_isect = 0, n_elastic = 0, n_inelastic = 0;
    // simple_cpu_driver::simulate_to_end (simple_cpu_driver.h:54-62) with
    // the event type recorded between init and the event handlers.
    void simulate_to_end() {
        for (typename base_t::particle_index_t idx = 0; idx < this->_particles.get_total_count(); ++idx) {
            while (this->_particles.active(idx)) {
                this->init(idx);
                if (this->_particles.next_intersect(idx))
                    ++n_isect;
                else if (this->_particles.next_scatter(idx))
                    (this->_particles.get_next_scatter(idx) == 1 ? n_inelastic : n_elastic)++;
                this->intersect(idx);
                this->scatter(idx);
            }
        }
    }
};
}  // namespace

extern "C" {

void nbref_free(void* p) { std::free(p); }

// Linearized octree of the reference builder.  Outputs are malloc'd.
int nbref_build_octree(const float* verts, const int32_t* mats, int64_t n, int32_t** data, int64_t* n_data,
                       float** tri_geom, int32_t** tri_mats, int64_t* n_tri, float center[3], float half[3]) {
    try {
        auto tris = make_tris(verts, mats, n);
        nbl::geometry::octree_builder::linearized_octree lin{nbl::geometry::octree_builder::octree_root(tris)};
        *n_data = int64_t(lin.octree_data.size());
        *data = static_cast<int32_t*>(std::malloc(sizeof(int32_t) * lin.octree_data.size()));
        std::memcpy(*data, lin.octree_data.data(), sizeof(int32_t) * lin.octree_data.size());
        *n_tri = int64_t(lin.triangle_data.size());
        *tri_geom = static_cast<float*>(std::malloc(sizeof(float) * 9 * lin.triangle_data.size() + 4));
        *tri_mats = static_cast<int32_t*>(std::malloc(sizeof(int32_t) * 2 * lin.triangle_data.size() + 4));
        for (size_t i = 0; i < lin.triangle_data.size(); ++i) {
            triangle_bytes b;
            std::memcpy(&b, &lin.triangle_data[i], sizeof(b));
            std::memcpy(*tri_geom + 9 * i, b.r0, 36);
            (*tri_mats)[2 * i] = b.mat_in;
            (*tri_mats)[2 * i + 1] = b.mat_out;
        }
        center[0] = lin.center.x; center[1] = lin.center.y; center[2] = lin.center.z;
        half[0] = lin.halfsize.x; half[1] = lin.halfsize.y; half[2] = lin.halfsize.z;
        return 0;
    } catch (...) {
        return -1;
    }
}

// Geometry handle for ray queries.
void* nbref_geometry_create(const float* verts, const int32_t* mats, int64_t n) {
    try {
        auto tris = make_tris(verts, mats, n);
        return new geometry_t(geometry_t::create(tris));
    } catch (...) {
        return nullptr;
    }
}

void nbref_geometry_destroy(void* g) {
    if (!g) return;
    auto* geo = static_cast<geometry_t*>(g);
    geometry_t::destroy(*geo);
    delete geo;
}

void nbref_geometry_info(void* g, float aabb_min[3], float aabb_max[3], float* max_extent) {
    auto* geo = static_cast<geometry_t*>(g);
    const vec3 mn = geo->AABB_min(), mx = geo->AABB_max();
    aabb_min[0] = mn.x; aabb_min[1] = mn.y; aabb_min[2] = mn.z;
    aabb_max[0] = mx.x; aabb_max[1] = mx.y; aabb_max[2] = mx.z;
    *max_extent = geo->get_max_extent();
}

// Batched octree<false>::propagate.  ignore_tri / out_tri index the
// linearized (Morton-ordered) triangle array; -1 means none.
void nbref_propagate(void* g, const float* pos, const float* dir, const float* dist, const int32_t* ignore_tri,
                     const int32_t* ignore_mat, int64_t n, float* out_dist, int32_t* out_tri) {
    auto* geo = static_cast<geometry_t*>(g);
    octree_bytes ob;
    std::memcpy(&ob, geo, sizeof(ob));
    for (int64_t i = 0; i < n; ++i) {
        const triangle* ign = ignore_tri[i] >= 0 ? ob.tris + ignore_tri[i] : nullptr;
        const intersect_event ev = geo->propagate({pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]},
                                                  {dir[3 * i], dir[3 * i + 1], dir[3 * i + 2]}, dist[i], ign,
                                                  ignore_mat[i]);
        out_dist[i] = ev.isect_distance;
        out_tri[i] = ev.isect_triangle ? int32_t(ev.isect_triangle - ob.tris) : -1;
    }
}

int nbref_in_domain(void* g, const float* pos, int64_t n, int32_t* out) {
    auto* geo = static_cast<geometry_t*>(g);
    for (int64_t i = 0; i < n; ++i) out[i] = geo->in_domain({pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]}) ? 1 : 0;
    return 0;
}

// Material loaded by the reference loaders (kieft_inelastic + kieft_elastic).
void* nbref_material_load(const char* path) {
    try {
        nbl::hdf5_file f(path);
        return new material_t(material_t::create(f));
    } catch (std::exception const& e) {
        std::fprintf(stderr, "nbref_material_load: %s\n", e.what());
        return nullptr;
    }
}

void nbref_material_destroy(void* m) {
    if (!m) return;
    auto* mat = static_cast<material_t*>(m);
    material_t::destroy(*mat);
    delete mat;
}

// barrier, fermi, band_gap, phonon_loss, recoil_const, max_energy
void nbref_material_info(void* m, float out[6]) {
    auto* mat = static_cast<material_t*>(m);
    auto const& inel = nbl::tuple::get<0>(*mat);
    auto const& el = nbl::tuple::get<1>(*mat);
    out[0] = mat->barrier;
    out[1] = in_spy::fermi(inel);
    out[2] = in_spy::gap(inel);
    out[3] = el_spy::phonon(el);
    out[4] = el_spy::recoil(el);
    out[5] = mat->get_max_energy();
}

// which: 0 elastic log-IMFP, 1 elastic cos-theta ICDF, 2 inelastic log-IMFP,
//        3 inelastic log-omega' ICDF, 4 ionisation (get_rounddown)
void nbref_material_eval(void* m, int which, const float* x, const float* y, int64_t n, float* out) {
    auto* mat = static_cast<material_t*>(m);
    auto const& inel = nbl::tuple::get<0>(*mat);
    auto const& el = nbl::tuple::get<1>(*mat);
    for (int64_t i = 0; i < n; ++i) {
        switch (which) {
        case 0: out[i] = el_spy::imfp(el).get(x[i]); break;
        case 1: out[i] = el_spy::icdf(el).get(x[i], y[i]); break;
        case 2: out[i] = in_spy::imfp(inel).get(x[i]); break;
        case 3: out[i] = in_spy::icdf(inel).get(x[i], y[i]); break;
#ifdef NBREF_PENN
        default: out[i] = 0; break;
#else
        default: out[i] = in_spy::ion(inel).get_rounddown(x[i], y[i]); break;
#endif
        }
    }
}

// Full table contents: copies width*height values (height=1 for 1D) into
// `out` (may be null to query sizes) and the axis {x_min, x_step, y_min, y_step}.
int nbref_material_table(void* m, int which, float* out, int32_t dims[2], float scales[4]) {
    auto* mat = static_cast<material_t*>(m);
    auto const& inel = nbl::tuple::get<0>(*mat);
    auto const& el = nbl::tuple::get<1>(*mat);
    if (which == 0 || which == 2) {
        auto const& t = which == 0 ? el_spy::imfp(el) : in_spy::imfp(inel);
        dims[0] = t.width();
        dims[1] = 1;
        nbl::util::table_1D<real, true>::scales(t, scales);
        if (out)
            for (int i = 0; i < t.width(); ++i) out[i] = t(i);
        return 0;
    }
#ifdef NBREF_PENN
    if (which == 4) return -1;
    auto const& t = which == 1 ? el_spy::icdf(el) : in_spy::icdf(inel);
#else
    auto const& t = which == 1 ? el_spy::icdf(el) : which == 3 ? in_spy::icdf(inel) : in_spy::ion(inel);
#endif
    dims[0] = t.width();
    dims[1] = t.height();
    nbl::util::table_2D<real, true>::scales(t, scales);
    if (out)
        for (int i = 0; i < t.width(); ++i)
            for (int j = 0; j < t.height(); ++j) out[size_t(i) * t.height() + j] = t(i, j);
    return 0;
}

// Full Penn 3-D tables (libnbref_penn.so only; the Kieft build returns -1):
// which 0 = q ICDF (table_3D::get), 1 = ionisation (table_3D::get_rounddown).
int nbref_material_eval3(void* m, int which, const float* x, const float* y, const float* z, int64_t n, float* out) {
#ifdef NBREF_PENN
    auto* mat = static_cast<material_t*>(m);
    auto const& inel = nbl::tuple::get<0>(*mat);
    for (int64_t i = 0; i < n; ++i)
        out[i] = which == 0 ? in_spy::q(inel).get(x[i], y[i], z[i]) : in_spy::ion3(inel).get_rounddown(x[i], y[i], z[i]);
    return 0;
#else
    (void)m; (void)which; (void)x; (void)y; (void)z; (void)n; (void)out;
    return -1;
#endif
}

// Full contents of a Penn 3-D table: data[(x * height + y) * depth + z] (out
// may be null to query sizes) and {x_min, x_step, y_min, y_step, z_min, z_step}.
int nbref_material_table3(void* m, int which, float* out, int32_t dims[3], float scales[6]) {
#ifdef NBREF_PENN
    auto* mat = static_cast<material_t*>(m);
    auto const& inel = nbl::tuple::get<0>(*mat);
    auto const& t = which == 0 ? in_spy::q(inel) : in_spy::ion3(inel);
    dims[0] = t.width();
    dims[1] = t.height();
    dims[2] = t.depth();
    nbl::util::table_3D<real, true>::scales(t, scales);
    if (out)
        for (int i = 0; i < t.width(); ++i)
            for (int j = 0; j < t.height(); ++j)
                for (int k = 0; k < t.depth(); ++k) out[(size_t(i) * t.height() + j) * t.depth() + k] = t(i, j, k);
    return 0;
#else
    (void)m; (void)which; (void)out; (void)dims; (void)scales;
    return -1;
#endif
}

// cpu_mt_main-style run.  Writes detected 36-byte records (malloc'd) and
// stats = {n_primaries, n_detected, n_intersect, n_elastic, n_inelastic};
// *seconds = wall time of the simulation phase (cpu_mt_main.cpp:201-219).
// max_primaries < 0 runs them all.
int nbref_run(const char* tri_path, const char* pri_path, const char* const* mat_paths, int n_mats, uint32_t seed,
              float energy_threshold, int n_threads, int count_events, int64_t max_primaries, void** records,
              int64_t* n_records, uint64_t stats[5], double* seconds) {
    try {
        std::vector<triangle> triangles = nbl::load_tri_file(tri_path);
        if (triangles.empty()) return -1;
        geometry_t geometry = geometry_t::create(triangles);
        nbl::cpu_material_manager<material_t> materials;
        for (int i = 0; i < n_mats; ++i) {
            nbl::hdf5_file f(mat_paths[i]);
            materials.add(f);
        }
        std::vector<particle> primaries;
        std::vector<int2> pixels;
        std::tie(primaries, pixels) =
            nbl::load_pri_file(pri_path, geometry.AABB_min(), geometry.AABB_max(), materials.get_max_energy());
        if (max_primaries >= 0 && size_t(max_primaries) < primaries.size()) {
            primaries.resize(size_t(max_primaries));
            pixels.resize(size_t(max_primaries));
        }
        std::vector<uint32_t> tags(primaries.size());
        for (size_t i = 0; i < tags.size(); ++i) tags[i] = uint32_t(i);
        work_pool pool(primaries.data(), tags.data(), primaries.size());
        intersect_t inter;
        if (n_threads <= 0) n_threads = int(std::thread::hardware_concurrency());

        std::mutex out_mutex;
        std::vector<float> out;   // 9 words per record
        std::atomic<uint64_t> n_isect{0}, n_el{0}, n_inel{0};
        std::mt19937 master(seed);
        std::vector<uint32_t> seeds;
        for (int i = 0; i < n_threads; ++i) seeds.push_back(master());

        auto loop = [&](uint32_t s) {
            std::vector<float> local;
            auto flush = [&](particle p, uint32_t t) {
                float rec[9] = {p.pos.x, p.pos.y, p.pos.z, p.dir.x, p.dir.y, p.dir.z, p.kin_energy, 0, 0};
                int32_t px[2] = {pixels[t].x, pixels[t].y};
                std::memcpy(rec + 7, px, 8);
                local.insert(local.end(), rec, rec + 9);
            };
            if (count_events) {
                counting_driver<scatter_physics<false>, intersect_t, geometry_t> d(
                    inter, materials, geometry, energy_threshold, materials.get_max_energy(), s);
                for (;;) {
                    auto w = pool.get_work(1);
                    if (std::get<2>(w) == 0) break;
                    d.push(std::get<0>(w), std::get<1>(w), std::get<2>(w));
                    d.simulate_to_end();
                    d.flush_detected(flush);
                }
                n_isect += d.n_isect;
                n_el += d.n_elastic;
                n_inel += d.n_inelastic;
            } else {
                nbl::drivers::simple_cpu_driver<scatter_physics<false>, intersect_t, geometry_t> d(
                    inter, materials, geometry, energy_threshold, materials.get_max_energy(), s);
                for (;;) {
                    auto w = pool.get_work(1);
                    if (std::get<2>(w) == 0) break;
                    d.push(std::get<0>(w), std::get<1>(w), std::get<2>(w));
                    d.simulate_to_end();
                    d.flush_detected(flush);
                }
            }
            std::lock_guard<std::mutex> lk(out_mutex);
            out.insert(out.end(), local.begin(), local.end());
        };
        const auto t0 = std::chrono::steady_clock::now();
        std::vector<std::thread> threads;
        for (int i = 0; i < n_threads; ++i) threads.emplace_back(loop, seeds[size_t(i)]);
        for (auto& t : threads) t.join();
        const auto t1 = std::chrono::steady_clock::now();
        *seconds = std::chrono::duration<double>(t1 - t0).count();

        *n_records = int64_t(out.size() / 9);
        *records = std::malloc(out.size() * sizeof(float) + 4);
        std::memcpy(*records, out.data(), out.size() * sizeof(float));
        stats[0] = primaries.size();
        stats[1] = uint64_t(*n_records);
        stats[2] = n_isect;
        stats[3] = n_el;
        stats[4] = n_inel;
        geometry_t::destroy(geometry);
        return 0;
    } catch (std::exception const& e) {
        std::fprintf(stderr, "nbref_run: %s\n", e.what());
        return -2;
    }
}

}  // extern "C"
