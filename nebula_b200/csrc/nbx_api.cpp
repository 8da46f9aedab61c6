// Host runtime behind the C ABI declared in include/nbx.h.
//
// One nbx_ctx owns one CUDA device's share of the simulation: the uploaded
// octree and material tables, the primary queue, two generation queues for
// secondaries, per-tag detection tallies, optional detected records and the
// energy histogram.  nbx_run launches the persistent transport kernel once per
// secondary generation, all on one stream, reading each generation's size on
// the device; the host only checks after each chunk of launches whether the
// last generation produced further secondaries.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

#include "kernels.h"
#include "material.h"
#include "mlp.cuh"
#include "mlp_kernels.h"
#include "nbx.h"
#include "octree.h"

namespace {

struct CudaError : std::runtime_error {
    explicit CudaError(const std::string& s) : std::runtime_error(s) {}
};
struct ApiError : std::runtime_error {
    int code;
    ApiError(int c, const std::string& s) : std::runtime_error(s), code(c) {}
};

void ck(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw CudaError(std::string(what) + ": " + cudaGetErrorString(e));
}

template <typename T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    void alloc(size_t count) {
        release();
        if (count == 0) return;
        if (cudaMalloc(&p, count * sizeof(T)) != cudaSuccess) {
            cudaGetLastError();
            p = nullptr;
            throw ApiError(NBX_ERR_OOM, "cudaMalloc of " + std::to_string(count * sizeof(T)) + " bytes failed");
        }
        n = count;
    }
    void ensure(size_t count) {
        if (count > n) alloc(count);
    }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    ~DevBuf() { release(); }
};

struct QueueBuf {
    DevBuf<float4> a, b;
    DevBuf<uint4> c;
    size_t cap = 0;
    void ensure(size_t n) {
        if (n <= cap) return;
        a.alloc(n);
        b.alloc(n);
        c.alloc(n);
        cap = n;
    }
    nbx::Queue q() const { return nbx::Queue{a.p, b.p, c.p}; }
};

constexpr int kMaxGenerations = 4096;
constexpr int kHistBins = 20000;
constexpr float kHistWidth = 0.5f;

}  // namespace

struct nbx_ctx {
    nbx_config cfg{};
    std::string err;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    int sms = 0;

    // geometry
    DevBuf<int32_t> octree;
    DevBuf<float4> tris;
    DevBuf<float4> tri_faces;
    // energy-deposit records (kDepositWords floats each) and the device cursor
    DevBuf<float> dep;
    DevBuf<unsigned long long> dep_cursor;
    uint64_t dep_cap = 0, dep_flushed = 0;
    bool have_geometry = false;
    // materials
    std::vector<DevBuf<float>*> tables;
    int n_mat = 0;
    float max_energy = std::numeric_limits<float>::infinity();
    nbx::dev::Physics phys{};

    // queues
    QueueBuf prim, qa, qb;
    uint64_t n_queued = 0;      // primaries waiting in `prim`
    uint64_t uid_next = 0;
    DevBuf<float> stage_p;
    DevBuf<uint32_t> stage_t;
    // staged batch (nbx_stage): copied on its own stream while a run may be
    // in flight, queued by nbx_push_staged
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t staged_ev = nullptr;
    DevBuf<float> staged_p;
    DevBuf<uint32_t> staged_t;
    DevBuf<uint32_t> staged_max;
    uint64_t staged_n = 0;
    bool staged_pending = false;
    DevBuf<uint32_t> ctl;       // head[G], tail[G], n_primary
    // tallies
    DevBuf<uint32_t> se_count, bse_count;
    uint64_t n_tags = 0;
    DevBuf<unsigned long long> counters;
    DevBuf<unsigned long long> hist;
    DevBuf<float4> rec;   // detected records, two float4 each in nbx_detected's layout
    DevBuf<uint32_t> rec_count;
    // escape-probability network: FP32 master parameters, Adam moments, gradient
    DevBuf<float> mlp_params, mlp_m, mlp_v, mlp_grad, mlp_loss;
    DevBuf<float> mlp_feat, mlp_lab, mlp_out;
    DevBuf<uint32_t> mlp_index;
    bool mlp_ready = false;
    int mlp_step = 0;
    // transport mode (plain / sample / learned) and its buffers
    int mode = nbx::kModePlain;
    float rr_threshold = 0.05f, split_threshold = 0.5f;
    int max_roulette_exp = 6;
    float birth_min_distance = 0.0f, birth_max_energy = 0.0f, birth_survival = 0.0f;   // off
    // importance table (nbx_set_importance_table): the network's escape
    // probability on a grid over its inputs, rebuilt when the parameters change
    DevBuf<float> imp_table;
    int imp_ne = 0, imp_nd = 0, imp_nc = 0, imp_materials = 0;
    uint64_t imp_version = ~0ull;  // mlp_version the table was built from
    uint64_t mlp_version = 0;      // bumped by every parameter change
    DevBuf<float> cost_table;      // cost-aware survival (nbx_set_learned_cost)
    int cost_bins = 0, cost_materials = 0;
    float cost_log_e_min = 0, cost_inv_width = 0, value_per_cost = 0;
    DevBuf<float4> smap_cells;
    nbx::dev::SurfaceMap smap{};
    DevBuf<float> sample_feat, sample_label, sample_cost;
    DevBuf<uint32_t> sample_count;
    uint64_t sample_cap = 0;
    DevBuf<float> se_w, bse_w;
    DevBuf<float4> stack_mem;     // transport parked-ancestor stacks (grow-only)
    DevBuf<uint32_t> range_cursor; // per-SM pop cursors of the primary generation (grow-only)
    DevBuf<uint32_t> yield_map;   // nbx_pixel_yields work buffers (grow-only)
    uint64_t pixel_map_len = 0;    // tags covered by a map from nbx_set_pixel_map
    DevBuf<float> pix_spec;        // per-pixel exit spectra (nbx_enable_pixel_spectra)
    uint64_t spec_pixels = 0;
    int spec_bins = 0;
    float spec_width = 0;
    DevBuf<double> yield_out;
    uint64_t rec_cap = 0;
    uint64_t rec_read = 0;   // records [0, rec_read) already flushed
    // stats
    uint64_t pushed = 0, generations = 0;
    double last_run_ms = 0, last_kernel_ms = 0;
    int block = 256, bpsm = 0, variant = 3;
    int stack_depth = 16;   // parked ancestors per thread before a secondary goes to the next generation
    int chunk = 8;          // generation launches queued between two 4-byte host reads
    uint64_t queue_capacity = 0;   // overflow-queue entries of the last run
    // device address of the allocation-free transport's scratch array,
    // looked up by this context's first nbx_run_noalloc call
    void* noalloc_scratch = nullptr;

    ~nbx_ctx() {
        for (auto* t : tables) delete t;
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (staged_ev) cudaEventDestroy(staged_ev);
        if (copy_stream) cudaStreamDestroy(copy_stream);
        if (stream) cudaStreamDestroy(stream);
    }
};

namespace {

// Calls without a context (file loaders, octree build) keep their message
// per host thread; nbx_last_error(NULL) returns it.
thread_local std::string g_thread_err;

int fail(nbx_ctx* ctx, int code, const std::string& msg) {
    (ctx ? ctx->err : g_thread_err) = msg;
    return code;
}

template <typename F>
int guarded(nbx_ctx* ctx, F&& f) {
    try {
        if (!ctx) g_thread_err.clear();
        if (ctx) {
            ctx->err.clear();
            if (cudaSetDevice(ctx->cfg.device) != cudaSuccess) return fail(ctx, NBX_ERR_CUDA, "cudaSetDevice failed");
        }
        return f();
    } catch (const ApiError& e) {
        return fail(ctx, e.code, e.what());
    } catch (const CudaError& e) {
        return fail(ctx, NBX_ERR_CUDA, e.what());
    } catch (const std::bad_alloc&) {
        return fail(ctx, NBX_ERR_OOM, "host allocation failed");
    } catch (const std::exception& e) {
        return fail(ctx, NBX_ERR_FORMAT, e.what());
    }
}

// All device traffic of a context goes through its own stream, which is
// created non-blocking and so does not wait for the legacy default stream: a
// plain cudaMemcpy from pageable host memory, a cudaMemset or a
// device-to-device cudaMemcpy can return before the bytes land, and a kernel
// queued on the context's stream would not wait for them.  These helpers
// queue the copy on the context's stream and wait for it.
static void to_device(nbx_ctx* ctx, void* dst, const void* src, size_t bytes, const char* what) {
    if (!bytes) return;
    ck(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->stream), what);
    ck(cudaStreamSynchronize(ctx->stream), what);
}

static void to_host(nbx_ctx* ctx, void* dst, const void* src, size_t bytes, const char* what) {
    if (!bytes) return;
    ck(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->stream), what);
    ck(cudaStreamSynchronize(ctx->stream), what);
}

static void zero(nbx_ctx* ctx, void* dst, size_t bytes, const char* what) {
    if (!bytes) return;
    ck(cudaMemsetAsync(dst, 0, bytes, ctx->stream), what);
    ck(cudaStreamSynchronize(ctx->stream), what);
}

nbx::dev::Table1D upload1d(nbx_ctx* ctx, const nbx_table1d& t) {
    if (t.n < 2 || !t.data) throw ApiError(NBX_ERR_ARG, "1D table needs at least 2 points");
    auto* b = new DevBuf<float>();
    ctx->tables.push_back(b);
    b->alloc(size_t(t.n));
    to_device(ctx, b->p, t.data, sizeof(float) * t.n, "table upload");
    return nbx::dev::Table1D{b->p, t.n, t.x_min, t.x_step};
}

nbx::dev::Table2D upload2d(nbx_ctx* ctx, const nbx_table2d& t) {
    if (t.width < 2 || t.height < 2 || !t.data) throw ApiError(NBX_ERR_ARG, "2D table needs at least 2x2 points");
    auto* b = new DevBuf<float>();
    ctx->tables.push_back(b);
    const size_t n = size_t(t.width) * size_t(t.height);
    b->alloc(n);
    to_device(ctx, b->p, t.data, sizeof(float) * n, "table upload");
    return nbx::dev::Table2D{b->p, t.width, t.height, t.x_min, t.x_step, t.y_min, t.y_step};
}

nbx::dev::Table3D upload3d(nbx_ctx* ctx, const nbx_table3d& t) {
    if (t.width < 2 || t.height < 2 || t.depth < 2 || !t.data)
        throw ApiError(NBX_ERR_ARG, "3D table needs at least 2x2x2 points");
    auto* b = new DevBuf<float>();
    ctx->tables.push_back(b);
    const size_t n = size_t(t.width) * size_t(t.height) * size_t(t.depth);
    b->alloc(n);
    to_device(ctx, b->p, t.data, sizeof(float) * n, "table upload");
    return nbx::dev::Table3D{b->p, t.width, t.height, t.depth, t.x_min, t.x_step, t.y_min, t.y_step, t.z_min, t.z_step};
}

// The inelastic and elastic log-IMFP tables interleaved per interval,
// (in[i], in[i+1], el[i], el[i+1]), when they share one axis (the same
// point count and the same scale, bit for bit); null otherwise.
const float4* upload_imfp_pair(nbx_ctx* ctx, const nbx_table1d& in, const nbx_table1d& el) {
    if (in.n != el.n || in.n < 2 || std::memcmp(&in.x_min, &el.x_min, 4) != 0 ||
        std::memcmp(&in.x_step, &el.x_step, 4) != 0)
        return nullptr;
    std::vector<float> v(4 * size_t(in.n - 1));
    for (int i = 0; i + 1 < in.n; ++i) {
        v[4 * size_t(i)] = in.data[i];
        v[4 * size_t(i) + 1] = in.data[i + 1];
        v[4 * size_t(i) + 2] = el.data[i];
        v[4 * size_t(i) + 3] = el.data[i + 1];
    }
    auto* b = new DevBuf<float>();
    ctx->tables.push_back(b);
    b->alloc(v.size());
    to_device(ctx, b->p, v.data(), sizeof(float) * v.size(), "table upload");
    return reinterpret_cast<const float4*>(b->p);
}

void ensure_tags(nbx_ctx* ctx, uint64_t n_tags) {
    if (n_tags <= ctx->n_tags) return;
    DevBuf<uint32_t> s, b;
    s.alloc(n_tags);
    b.alloc(n_tags);
    ck(cudaMemsetAsync(s.p, 0, n_tags * 4, ctx->stream), "memset");
    ck(cudaMemsetAsync(b.p, 0, n_tags * 4, ctx->stream), "memset");
    if (ctx->n_tags) {
        ck(cudaMemcpyAsync(s.p, ctx->se_count.p, ctx->n_tags * 4, cudaMemcpyDeviceToDevice, ctx->stream), "copy");
        ck(cudaMemcpyAsync(b.p, ctx->bse_count.p, ctx->n_tags * 4, cudaMemcpyDeviceToDevice, ctx->stream), "copy");
    }
    ck(cudaStreamSynchronize(ctx->stream), "sync");
    std::swap(ctx->se_count.p, s.p);
    std::swap(ctx->se_count.n, s.n);
    std::swap(ctx->bse_count.p, b.p);
    std::swap(ctx->bse_count.n, b.n);
    {
        DevBuf<float> sw, bw;
        sw.alloc(n_tags);
        bw.alloc(n_tags);
        ck(cudaMemsetAsync(sw.p, 0, n_tags * 4, ctx->stream), "memset");
        ck(cudaMemsetAsync(bw.p, 0, n_tags * 4, ctx->stream), "memset");
        if (ctx->n_tags) {
            ck(cudaMemcpyAsync(sw.p, ctx->se_w.p, ctx->n_tags * 4, cudaMemcpyDeviceToDevice, ctx->stream), "copy");
            ck(cudaMemcpyAsync(bw.p, ctx->bse_w.p, ctx->n_tags * 4, cudaMemcpyDeviceToDevice, ctx->stream), "copy");
        }
        ck(cudaStreamSynchronize(ctx->stream), "sync");
        std::swap(ctx->se_w.p, sw.p);
        std::swap(ctx->se_w.n, sw.n);
        std::swap(ctx->bse_w.p, bw.p);
        std::swap(ctx->bse_w.n, bw.n);
    }
    ctx->n_tags = n_tags;
}

void fill_material(const nbx::MaterialTables& m, nbx_material* out) {
    std::memset(out, 0, sizeof(*out));
    auto dup = [](const std::vector<float>& v) {
        float* p = static_cast<float*>(std::malloc(sizeof(float) * (v.size() + 1)));
        if (!p) throw std::bad_alloc();
        std::memcpy(p, v.data(), sizeof(float) * v.size());
        return p;
    };
    out->barrier = m.barrier;
    out->elastic_imfp = {m.el_imfp.n, m.el_imfp.x_min, m.el_imfp.x_step, dup(m.el_imfp.data)};
    out->elastic_icdf = {m.el_icdf.width, m.el_icdf.height, m.el_icdf.x_min, m.el_icdf.x_step,
                         m.el_icdf.y_min, m.el_icdf.y_step, dup(m.el_icdf.data)};
    out->phonon_loss = m.phonon_loss;
    out->recoil_const = m.recoil_const;
    out->inelastic_imfp = {m.in_imfp.n, m.in_imfp.x_min, m.in_imfp.x_step, dup(m.in_imfp.data)};
    out->inelastic_icdf = {m.in_icdf.width, m.in_icdf.height, m.in_icdf.x_min, m.in_icdf.x_step,
                           m.in_icdf.y_min, m.in_icdf.y_step, dup(m.in_icdf.data)};
    out->ionisation = {m.ionisation.width, m.ionisation.height, m.ionisation.x_min, m.ionisation.x_step,
                       m.ionisation.y_min, m.ionisation.y_step, dup(m.ionisation.data)};
    out->fermi = m.fermi;
    out->band_gap = m.band_gap;
    out->max_energy = m.max_energy(!m.has_kieft_inelastic);
    std::snprintf(out->name, sizeof(out->name), "%s", m.name.c_str());
    out->has_kieft_inelastic = m.has_kieft_inelastic ? 1 : 0;
    out->has_full_penn = m.has_penn ? 1 : 0;
    auto t3 = [&](const nbx::Table3D& t) {
        return nbx_table3d{t.width, t.height, t.depth, t.x_min, t.x_step, t.y_min, t.y_step, t.z_min, t.z_step,
                           dup(t.data)};
    };
    out->penn_imfp = {m.penn_imfp.n, m.penn_imfp.x_min, m.penn_imfp.x_step, dup(m.penn_imfp.data)};
    out->penn_omega_icdf = {m.penn_omega_icdf.width, m.penn_omega_icdf.height, m.penn_omega_icdf.x_min,
                            m.penn_omega_icdf.x_step, m.penn_omega_icdf.y_min, m.penn_omega_icdf.y_step,
                            dup(m.penn_omega_icdf.data)};
    out->penn_q_icdf = t3(m.penn_q_icdf);
    out->penn_ionisation = t3(m.penn_ionisation);
    out->penn_max_energy = m.has_penn ? m.max_energy(true) : 0.0f;
}

}  // namespace

extern "C" {

int nbx_version(int* major, int* minor, int* patch) {
    if (major) *major = NBX_VERSION_MAJOR;
    if (minor) *minor = NBX_VERSION_MINOR;
    if (patch) *patch = NBX_VERSION_PATCH;
    return NBX_OK;
}

const char* nbx_error_string(int code) {
    switch (code) {
    case NBX_OK: return "ok";
    case NBX_ERR_ARG: return "invalid argument";
    case NBX_ERR_OOM: return "out of memory";
    case NBX_ERR_CUDA: return "CUDA error";
    case NBX_ERR_TIMEOUT: return "device wait timed out";
    case NBX_ERR_FORMAT: return "malformed input";
    case NBX_ERR_STATE: return "call out of order";
    case NBX_ERR_NODEV: return "no CUDA device";
    case NBX_ERR_CAPACITY: return "device queue overflow";
    default: return "unknown error";
    }
}

void nbx_free(void* p) { std::free(p); }

int nbx_device_count(int* n) {
    if (!n) return NBX_ERR_ARG;
    int c = 0;
    if (cudaGetDeviceCount(&c) != cudaSuccess) {
        cudaGetLastError();
        *n = 0;
        return NBX_ERR_NODEV;
    }
    *n = c;
    return NBX_OK;
}

int nbx_load_tri(const char* path, nbx_triangle** out, uint64_t* n) {
    if (!path || !out || !n) return NBX_ERR_ARG;
    return guarded(nullptr, [&] {
        auto tris = nbx::load_tri_file(path);
        if (tris.empty()) return NBX_ERR_FORMAT;
        auto* p = static_cast<nbx_triangle*>(std::malloc(sizeof(nbx_triangle) * tris.size()));
        if (!p) return NBX_ERR_OOM;
        static_assert(sizeof(nbx_triangle) == sizeof(nbx::Triangle), "triangle layout");
        std::memcpy(p, tris.data(), sizeof(nbx_triangle) * tris.size());
        *out = p;
        *n = tris.size();
        return NBX_OK;
    });
}

int nbx_load_pri(const char* path, nbx_record** out, uint64_t* n) {
    if (!path || !out || !n) return NBX_ERR_ARG;
    FILE* f = std::fopen(path, "rb");
    if (!f) return NBX_ERR_FORMAT;
    std::fseek(f, 0, SEEK_END);
    const long size = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    if (size < 0 || size % 36 != 0) {
        std::fclose(f);
        return NBX_ERR_FORMAT;   // "Unexpected end of primaries file"
    }
    const uint64_t count = uint64_t(size) / 36;
    auto* p = static_cast<nbx_record*>(std::malloc(size > 0 ? size_t(size) : 1));
    if (!p) {
        std::fclose(f);
        return NBX_ERR_OOM;
    }
    const size_t got = count ? std::fread(p, 36, count, f) : 0;
    std::fclose(f);
    if (got != count) {
        std::free(p);
        return NBX_ERR_FORMAT;
    }
    *out = p;
    *n = count;
    return NBX_OK;
}

int nbx_octree_build(const nbx_triangle* tris, uint64_t n, nbx_octree** out) {
    if (!tris || n == 0 || !out) return NBX_ERR_ARG;
    return guarded(nullptr, [&] {
        std::vector<nbx::Triangle> v(n);
        std::memcpy(v.data(), tris, sizeof(nbx_triangle) * n);
        nbx::LinearOctree lin = nbx::build_octree(v);
        auto* o = static_cast<nbx_octree*>(std::calloc(1, sizeof(nbx_octree)));
        if (!o) return NBX_ERR_OOM;
        o->n_octree = lin.octree_data.size();
        o->octree_data = static_cast<int32_t*>(std::malloc(sizeof(int32_t) * (o->n_octree + 1)));
        o->n_triangles = lin.triangles.size();
        o->triangles = static_cast<nbx_triangle*>(std::malloc(sizeof(nbx_triangle) * (o->n_triangles + 1)));
        if (!o->octree_data || !o->triangles) {
            nbx_octree_free(o);
            return NBX_ERR_OOM;
        }
        std::memcpy(o->octree_data, lin.octree_data.data(), sizeof(int32_t) * o->n_octree);
        std::memcpy(o->triangles, lin.triangles.data(), sizeof(nbx_triangle) * o->n_triangles);
        o->center[0] = lin.center.x;
        o->center[1] = lin.center.y;
        o->center[2] = lin.center.z;
        o->halfsize[0] = lin.halfsize.x;
        o->halfsize[1] = lin.halfsize.y;
        o->halfsize[2] = lin.halfsize.z;
        o->duplicates_dropped = lin.duplicates_dropped;
        o->max_depth = lin.max_depth;
        *out = o;
        return NBX_OK;
    });
}

void nbx_octree_free(nbx_octree* o) {
    if (!o) return;
    std::free(o->octree_data);
    std::free(o->triangles);
    std::free(o);
}

int nbx_material_load(const char* path, nbx_material** out) {
    if (!path || !out) return NBX_ERR_ARG;
    return guarded(nullptr, [&] {
        nbx::MaterialTables m = nbx::load_material(path);
        auto* o = static_cast<nbx_material*>(std::calloc(1, sizeof(nbx_material)));
        if (!o) return NBX_ERR_OOM;
        fill_material(m, o);
        *out = o;
        return NBX_OK;
    });
}

void nbx_material_free(nbx_material* m) {
    if (!m) return;
    std::free(const_cast<float*>(m->elastic_imfp.data));
    std::free(const_cast<float*>(m->elastic_icdf.data));
    std::free(const_cast<float*>(m->inelastic_imfp.data));
    std::free(const_cast<float*>(m->inelastic_icdf.data));
    std::free(const_cast<float*>(m->ionisation.data));
    std::free(const_cast<float*>(m->penn_imfp.data));
    std::free(const_cast<float*>(m->penn_omega_icdf.data));
    std::free(const_cast<float*>(m->penn_q_icdf.data));
    std::free(const_cast<float*>(m->penn_ionisation.data));
    std::free(m);
}

void nbx_config_default(nbx_config* cfg) {
    if (!cfg) return;
    std::memset(cfg, 0, sizeof(*cfg));
    cfg->seed = 0x78c7e39b;   // gpu_main.cu:238
}

int nbx_create(nbx_ctx** out, const nbx_config* cfg) {
    if (!out) return NBX_ERR_ARG;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) {
        cudaGetLastError();
        return NBX_ERR_NODEV;
    }
    nbx_config c;
    nbx_config_default(&c);
    if (cfg) c = *cfg;
    if (c.device < 0 || c.device >= n) return NBX_ERR_ARG;
    auto* ctx = new (std::nothrow) nbx_ctx();
    if (!ctx) return NBX_ERR_OOM;
    ctx->cfg = c;
    const int rc = guarded(ctx, [&] {
        ck(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking), "stream");
        ck(cudaEventCreate(&ctx->ev0), "event");
        ck(cudaEventCreate(&ctx->ev1), "event");
        ck(cudaDeviceGetAttribute(&ctx->sms, cudaDevAttrMultiProcessorCount, c.device), "attribute");
        ctx->counters.alloc(nbx::kNumCounters);
        zero(ctx, ctx->counters.p, sizeof(unsigned long long) * nbx::kNumCounters, "memset");
        ctx->hist.alloc(kHistBins);
        zero(ctx, ctx->hist.p, sizeof(unsigned long long) * kHistBins, "memset");
        ctx->ctl.alloc(2 * kMaxGenerations + 4);   // + the overflow snapshot (8-byte aligned)
        ctx->rec_count.alloc(1);
        zero(ctx, ctx->rec_count.p, 4, "memset");
        ctx->block = c.block_size > 0 ? c.block_size : 256;
        if (ctx->block % 32 != 0 || ctx->block > 256) throw ApiError(NBX_ERR_ARG, "block_size must be a multiple of 32, <= 256");
        // Kernel variant = resident blocks per SM it was register-limited for:
        // 2, 3 or 4 blocks of 256 threads, or 7 blocks of 128 (72 registers;
        // block size capped at 128); default 4 (64 registers: the
        // autotuner's choice on most workloads).
        ctx->variant = ((c.blocks_per_sm >= 2 && c.blocks_per_sm <= 4) || c.blocks_per_sm == 7) ? c.blocks_per_sm : 4;
        if (ctx->variant == 7 && ctx->block > 128) ctx->block = 128;
        ctx->bpsm = nbx::transport_max_blocks_per_sm(ctx->block, ctx->variant);
        if (c.record_deposits) {
            ctx->dep_cap = c.deposit_capacity ? c.deposit_capacity : (1ull << 27);
            ctx->dep.alloc(ctx->dep_cap * nbx::kDepositWords);
            ctx->dep_cursor.alloc(1);
            zero(ctx, ctx->dep_cursor.p, sizeof(unsigned long long), "memset");
        }
        if (c.record_detected) {
            ctx->rec_cap = c.record_capacity ? c.record_capacity : (1ull << 24);
            ctx->rec.alloc(2 * ctx->rec_cap);
        }
        ctx->phys.seed = c.seed;
        ctx->phys.min_energy = c.energy_threshold;
        if (c.inelastic_model != NBX_INELASTIC_KIEFT && c.inelastic_model != NBX_INELASTIC_FULL_PENN)
            throw ApiError(NBX_ERR_ARG, "inelastic_model must be NBX_INELASTIC_KIEFT or NBX_INELASTIC_FULL_PENN");
        ctx->phys.penn = c.inelastic_model == NBX_INELASTIC_FULL_PENN ? 1 : 0;
        ctx->phys.max_energy = std::numeric_limits<float>::infinity();
        return NBX_OK;
    });
    if (rc != NBX_OK) {
        std::fprintf(stderr, "nbx_create: %s\n", ctx->err.c_str());
        delete ctx;
        return rc;
    }
    *out = ctx;
    return NBX_OK;
}

void nbx_destroy(nbx_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->cfg.device);
    if (ctx->copy_stream) cudaStreamSynchronize(ctx->copy_stream);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    delete ctx;
}

const char* nbx_last_error(nbx_ctx* ctx) { return ctx ? ctx->err.c_str() : g_thread_err.c_str(); }

int nbx_set_geometry(nbx_ctx* ctx, const nbx_octree* o) {
    if (!ctx || !o || !o->octree_data || o->n_octree < 8 || !o->triangles) return NBX_ERR_ARG;
    return guarded(ctx, [&] {
        ctx->octree.alloc(o->n_octree);
        to_device(ctx, ctx->octree.p, o->octree_data, sizeof(int32_t) * o->n_octree, "octree");
        std::vector<float4> t(3 * std::max<uint64_t>(o->n_triangles, 1));
        for (uint64_t i = 0; i < o->n_triangles; ++i) {
            const nbx_triangle& s = o->triangles[i];
            if (s.mat_in < -32768 || s.mat_in > 32767 || s.mat_out < -32768 || s.mat_out > 32767)
                throw ApiError(NBX_ERR_ARG, "triangle material index outside the 16-bit range");
            float a, b;
            std::memcpy(&a, &s.mat_in, 4);
            std::memcpy(&b, &s.mat_out, 4);
            t[3 * i] = make_float4(s.r0[0], s.r0[1], s.r0[2], a);
            t[3 * i + 1] = make_float4(s.e1[0], s.e1[1], s.e1[2], b);
            t[3 * i + 2] = make_float4(s.e2[0], s.e2[1], s.e2[2], 0.0f);
        }
        ctx->tris.alloc(t.size());
        to_device(ctx, ctx->tris.p, t.data(), sizeof(float4) * t.size(), "triangles");
        ctx->tri_faces.alloc(std::max<uint64_t>(o->n_triangles, 1));
        ck(nbx::launch_triangle_faces(ctx->tris.p, ctx->tri_faces.p, int(o->n_triangles), ctx->stream), "faces");
        ck(cudaStreamSynchronize(ctx->stream), "faces");
        auto& g = ctx->phys.geo;
        g.octree = ctx->octree.p;
        g.tri = ctx->tris.p;
        g.tri_face = ctx->tri_faces.p;
        g.cx = o->center[0];
        g.cy = o->center[1];
        g.cz = o->center[2];
        g.hx = o->halfsize[0];
        g.hy = o->halfsize[1];
        g.hz = o->halfsize[2];
        // octree factory: 2 * magnitude(halfsize), host sqrt (geometry/octree.inl:247-253)
        g.max_extent = 2 * std::sqrt(g.hx * g.hx + g.hy * g.hy + g.hz * g.hz);
        g.n_tri = int(o->n_triangles);
        ctx->have_geometry = true;
        return NBX_OK;
    });
}

int nbx_add_material(nbx_ctx* ctx, const nbx_material* m) {
    if (!ctx || !m) return NBX_ERR_ARG;
    if (ctx->n_mat >= NBX_MAX_MATERIALS) return fail(ctx, NBX_ERR_ARG, "too many materials");
    return guarded(ctx, [&] {
        nbx::dev::Material d{};
        d.barrier = m->barrier;
        d.phonon_loss = m->phonon_loss;
        d.recoil_const = m->recoil_const;
        d.fermi = m->fermi;
        d.band_gap = m->band_gap;
        d.el_imfp = upload1d(ctx, m->elastic_imfp);
        d.el_icdf = upload2d(ctx, m->elastic_icdf);
        float max_energy = m->max_energy;
        if (ctx->phys.penn) {
            // full_penn (physics/full_penn.h): log-IMFP and log-omega ICDF in
            // the inelastic slots, plus the two 3-D tables
            if (!m->has_full_penn)
                throw ApiError(NBX_ERR_FORMAT, std::string("material has no full Penn tables: ") + m->name);
            d.in_imfp = upload1d(ctx, m->penn_imfp);
            d.in_icdf = upload2d(ctx, m->penn_omega_icdf);
            d.q = upload3d(ctx, m->penn_q_icdf);
            d.ion3 = upload3d(ctx, m->penn_ionisation);
            max_energy = m->penn_max_energy;
        } else {
            if (!m->has_kieft_inelastic && m->inelastic_imfp.n < 2)
                throw ApiError(NBX_ERR_FORMAT, std::string("material has no Kieft inelastic tables: ") + m->name);
            d.in_imfp = upload1d(ctx, m->inelastic_imfp);
            d.in_icdf = upload2d(ctx, m->inelastic_icdf);
            d.ion = upload2d(ctx, m->ionisation);
        }
        d.imfp_pair = upload_imfp_pair(ctx, ctx->phys.penn ? m->penn_imfp : m->inelastic_imfp, m->elastic_imfp);
        ctx->phys.mat[ctx->n_mat++] = d;
        ctx->phys.n_mat = ctx->n_mat;
        // cpu_material_manager::get_max_energy (core/cpu_material_manager.inl:43-55)
        if (max_energy < ctx->max_energy) ctx->max_energy = max_energy;
        ctx->phys.max_energy = ctx->max_energy;
        return NBX_OK;
    });
}

int nbx_set_tag_range(nbx_ctx* ctx, uint64_t n_tags) {
    if (!ctx) return NBX_ERR_ARG;
    return guarded(ctx, [&] {
        ensure_tags(ctx, n_tags);
        return NBX_OK;
    });
}

namespace {
// Room for n more primaries in the primary queue (grown, keeping the queued ones).
void ensure_primary_room(nbx_ctx* ctx, uint64_t n) {
    if (ctx->prim.cap >= ctx->n_queued + n) return;
    QueueBuf nq;
    nq.ensure(std::max<uint64_t>(ctx->n_queued + n, 2 * ctx->prim.cap));
    if (ctx->n_queued) {
        ck(cudaMemcpyAsync(nq.a.p, ctx->prim.a.p, 16 * ctx->n_queued, cudaMemcpyDeviceToDevice, ctx->stream), "copy");
        ck(cudaMemcpyAsync(nq.b.p, ctx->prim.b.p, 16 * ctx->n_queued, cudaMemcpyDeviceToDevice, ctx->stream), "copy");
        ck(cudaMemcpyAsync(nq.c.p, ctx->prim.c.p, 16 * ctx->n_queued, cudaMemcpyDeviceToDevice, ctx->stream), "copy");
        ck(cudaStreamSynchronize(ctx->stream), "sync");
    }
    std::swap(ctx->prim.a.p, nq.a.p);
    std::swap(ctx->prim.a.n, nq.a.n);
    std::swap(ctx->prim.b.p, nq.b.p);
    std::swap(ctx->prim.b.n, nq.b.n);
    std::swap(ctx->prim.c.p, nq.c.p);
    std::swap(ctx->prim.c.n, nq.c.n);
    std::swap(ctx->prim.cap, nq.cap);
}
}  // namespace

int nbx_push(nbx_ctx* ctx, const nbx_particle* particles, const uint32_t* tags, uint64_t n, uint64_t* accepted) {
    if (!ctx || (n && (!particles || !tags))) return NBX_ERR_ARG;
    return guarded(ctx, [&] {
        if (accepted) *accepted = 0;
        if (n == 0) return NBX_OK;
        if (ctx->n_queued + n > 0xFFFFFFF0ull) throw ApiError(NBX_ERR_CAPACITY, "primary queue limited to 2^32 entries");
        uint32_t max_tag = 0;
        for (uint64_t i = 0; i < n; ++i) max_tag = std::max(max_tag, tags[i]);
        ensure_tags(ctx, uint64_t(max_tag) + 1);
        ensure_primary_room(ctx, n);
        ctx->stage_p.ensure(7 * n);
        ctx->stage_t.ensure(n);
        ck(cudaMemcpyAsync(ctx->stage_p.p, particles, sizeof(float) * 7 * n, cudaMemcpyHostToDevice, ctx->stream), "H2D");
        ck(cudaMemcpyAsync(ctx->stage_t.p, tags, sizeof(uint32_t) * n, cudaMemcpyHostToDevice, ctx->stream), "H2D");
        ck(nbx::launch_fill_queue(ctx->prim.q(), ctx->stage_p.p, ctx->stage_t.p, ctx->uid_next, n, ctx->n_queued,
                                  ctx->stream), "fill");
        ck(cudaStreamSynchronize(ctx->stream), "sync");
        ctx->uid_next += n;
        ctx->n_queued += n;
        ctx->pushed += n;
        if (accepted) *accepted = n;
        return NBX_OK;
    });
}

namespace {
void mlp_upload(nbx_ctx* ctx, const float* features, const float* labels, uint64_t n);

// Evaluates the network at the centres of the importance table's grid (one
// row of features per cell, on the tensor cores) into ctx->imp_table.
void build_importance_table(nbx_ctx* ctx) {
    const int nm = std::max(1, ctx->n_mat), ne = ctx->imp_ne, nd = ctx->imp_nd, nc = ctx->imp_nc;
    const uint64_t cells = uint64_t(nm) * ne * nd * nc;
    std::vector<float> f(cells * nbx::mlp::kFeatures, 0.0f);
    uint64_t r = 0;
    for (int m = 0; m < nm; ++m)
        for (int ie = 0; ie < ne; ++ie)
            for (int id = 0; id < nd; ++id)
                for (int ic = 0; ic < nc; ++ic, ++r) {
                    float* x = f.data() + r * nbx::mlp::kFeatures;
                    x[0] = (ie + 0.5f) / float(ne);
                    x[1] = (id + 0.5f) / float(nd);
                    x[2] = -1.0f + 2.0f * (ic + 0.5f) / float(nc);
                    if (m < 3) x[3 + m] = 1.0f;
                }
    mlp_upload(ctx, f.data(), nullptr, cells);
    ctx->imp_table.ensure(cells);
    ck(nbx::mlp::launch_predict(ctx->mlp_params.p, ctx->mlp_feat.p, cells, ctx->imp_table.p, ctx->stream),
       "predict kernel");
    ck(cudaStreamSynchronize(ctx->stream), "sync");
    ctx->imp_materials = nm;
    ctx->imp_version = ctx->mlp_version;
}
}  // namespace

int nbx_set_importance_table(nbx_ctx* ctx, int32_t n_energy, int32_t n_distance, int32_t n_cosine) {
    if (!ctx || n_energy < 0 || n_distance < 0 || n_cosine < 0 || n_energy > 1024 || n_distance > 1024 ||
        n_cosine > 1024)
        return NBX_ERR_ARG;
    if (n_energy == 0 || n_distance == 0 || n_cosine == 0) {
        ctx->imp_ne = ctx->imp_nd = ctx->imp_nc = 0;
        return NBX_OK;
    }
    if (!ctx->mlp_ready) return fail(ctx, NBX_ERR_STATE, "importance table without network parameters");
    return guarded(ctx, [&] {
        ctx->imp_ne = n_energy;
        ctx->imp_nd = n_distance;
        ctx->imp_nc = n_cosine;
        build_importance_table(ctx);
        return NBX_OK;
    });
}

int nbx_stage(nbx_ctx* ctx, const nbx_particle* particles, const uint32_t* tags, uint64_t n) {
    if (!ctx || (n && (!particles || !tags))) return NBX_ERR_ARG;
    if (ctx->staged_pending) return fail(ctx, NBX_ERR_STATE, "nbx_stage: a staged batch waits for nbx_push_staged");
    return guarded(ctx, [&] {
        if (!ctx->copy_stream) {
            ck(cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking), "stream");
            ck(cudaEventCreateWithFlags(&ctx->staged_ev, cudaEventDisableTiming), "event");
        }
        ctx->staged_p.ensure(std::max<uint64_t>(7 * n, 1));
        ctx->staged_t.ensure(std::max<uint64_t>(n, 1));
        if (n) {
            ck(cudaMemcpyAsync(ctx->staged_p.p, particles, sizeof(float) * 7 * n, cudaMemcpyHostToDevice,
                               ctx->copy_stream), "H2D");
            ck(cudaMemcpyAsync(ctx->staged_t.p, tags, sizeof(uint32_t) * n, cudaMemcpyHostToDevice, ctx->copy_stream),
               "H2D");
        }
        ck(cudaEventRecord(ctx->staged_ev, ctx->copy_stream), "event");
        ctx->staged_n = n;
        ctx->staged_pending = true;
        return NBX_OK;
    });
}

int nbx_host_alloc(uint64_t bytes, void** out) {
    if (!out) return NBX_ERR_ARG;
    *out = nullptr;
    if (bytes == 0) return NBX_ERR_ARG;
    if (cudaHostAlloc(out, bytes, cudaHostAllocPortable) != cudaSuccess) {
        cudaGetLastError();
        *out = nullptr;
        return NBX_ERR_OOM;
    }
    return NBX_OK;
}

void nbx_host_free(void* p) {
    if (p) cudaFreeHost(p);
}

int nbx_push_staged(nbx_ctx* ctx, uint64_t* accepted) {
    if (!ctx) return NBX_ERR_ARG;
    if (accepted) *accepted = 0;
    if (!ctx->staged_pending) return NBX_OK;
    return guarded(ctx, [&] {
        const uint64_t n = ctx->staged_n;
        ck(cudaStreamWaitEvent(ctx->stream, ctx->staged_ev, 0), "wait");
        ctx->staged_pending = false;
        if (n == 0) return NBX_OK;
        if (ctx->n_queued + n > 0xFFFFFFF0ull) throw ApiError(NBX_ERR_CAPACITY, "primary queue limited to 2^32 entries");
        ctx->staged_max.ensure(1);
        ck(cudaMemsetAsync(ctx->staged_max.p, 0, 4, ctx->stream), "memset");
        ck(nbx::launch_max_tag(ctx->staged_t.p, n, ctx->staged_max.p, ctx->stream), "max tag");
        uint32_t max_tag = 0;
        to_host(ctx, &max_tag, ctx->staged_max.p, 4, "D2H");
        ensure_tags(ctx, uint64_t(max_tag) + 1);
        ensure_primary_room(ctx, n);
        ck(nbx::launch_fill_queue(ctx->prim.q(), ctx->staged_p.p, ctx->staged_t.p, ctx->uid_next, n, ctx->n_queued,
                                  ctx->stream), "fill");
        ck(cudaStreamSynchronize(ctx->stream), "sync");
        ctx->uid_next += n;
        ctx->n_queued += n;
        ctx->pushed += n;
        if (accepted) *accepted = n;
        return NBX_OK;
    });
}

int nbx_run(nbx_ctx* ctx) {
    if (!ctx) return NBX_ERR_ARG;
    if (!ctx->have_geometry) return fail(ctx, NBX_ERR_STATE, "nbx_run before nbx_set_geometry");
    return guarded(ctx, [&] {
        ctx->generations = 0;
        ctx->last_run_ms = ctx->last_kernel_ms = 0;
        if (ctx->n_queued == 0) return NBX_OK;
        // Overflow-queue capacity (secondaries of cascades deeper than the
        // per-thread stack): explicit, else one per queued primary (at least
        // 1M), bounded by a quarter of the free device memory.
        uint64_t want = ctx->cfg.capacity ? ctx->cfg.capacity : std::max<uint64_t>(1ull << 20, ctx->n_queued);
        want = std::min<uint64_t>(want, 0xFFFFFFF0ull);
        if (ctx->qa.cap < want) {
            // the memory budget only matters when the queues would grow
            size_t free_b = 0, total_b = 0;
            ck(cudaMemGetInfo(&free_b, &total_b), "meminfo");
            const uint64_t budget = (free_b / 4) / (2 * 48);
            want = std::min<uint64_t>(want, std::max<uint64_t>(budget, 1ull << 16));
        }
        if (ctx->qa.cap < want) {
            ctx->qa.a.release(); ctx->qa.b.release(); ctx->qa.c.release(); ctx->qa.cap = 0;
            ctx->qb.a.release(); ctx->qb.b.release(); ctx->qb.c.release(); ctx->qb.cap = 0;
            ctx->qa.ensure(want);
            ctx->qb.ensure(want);
        }
        const uint32_t cap = uint32_t(std::min(ctx->qa.cap, ctx->qb.cap));
        ctx->queue_capacity = cap;
        uint32_t* ctl = ctx->ctl.p;
        ck(cudaMemsetAsync(ctl, 0, sizeof(uint32_t) * (2 * kMaxGenerations + 2), ctx->stream), "memset");
        static_assert((2 * kMaxGenerations + 2) % 2 == 0, "overflow snapshot alignment");
        // Nothing before the first launch waits on the host or on a copy
        // engine: the queue length is set by a one-thread kernel (a small
        // host-to-device copy could queue behind a staged batch's copy), and
        // the overflow counter is snapshotted on the device.
        ck(nbx::launch_set_word(ctl + 2 * kMaxGenerations, uint32_t(ctx->n_queued), ctx->stream), "set");
        unsigned long long* const ovf_snapshot = reinterpret_cast<unsigned long long*>(ctl + 2 * kMaxGenerations + 2);
        ck(cudaMemcpyAsync(ovf_snapshot, ctx->counters.p + nbx::kCntOverflow, 8, cudaMemcpyDeviceToDevice,
                           ctx->stream), "D2D");

        nbx::TransportArgs a{};
        a.se_count = ctx->se_count.p;
        a.bse_count = ctx->bse_count.p;
        a.n_tags = ctx->n_tags;
        a.counters = ctx->counters.p;
        a.rec = ctx->rec.p;
        a.rec_count = ctx->rec_count.p;
        a.rec_capacity = uint32_t(std::min<uint64_t>(ctx->rec_cap, 0xFFFFFFF0ull));
        a.hist = ctx->hist.p;
        if (ctx->spec_pixels) {
            a.pix_spec = ctx->pix_spec.p;
            a.pixel_of_tag = ctx->yield_map.p;
            a.n_map = ctx->pixel_map_len;
            a.n_pixels = ctx->spec_pixels;
            a.pix_bins = ctx->spec_bins;
            a.pix_inv_width = 1.0f / ctx->spec_width;
        }
        a.n_bins = kHistBins;
        a.inv_bin_width = 1.0f / kHistWidth;
        a.smap = ctx->smap;
        if (ctx->mode == nbx::kModeSample) {
            if (!ctx->sample_cap) throw ApiError(NBX_ERR_STATE, "sample mode without nbx_set_sample_capacity");
            a.sample_feat = ctx->sample_feat.p;
            a.sample_label = ctx->sample_label.p;
            a.sample_cost = ctx->sample_cost.p;
            a.sample_count = ctx->sample_count.p;
            a.sample_capacity = uint32_t(std::min<uint64_t>(ctx->sample_cap, 0xFFFFFFF0ull));
        }
        if (ctx->mode == nbx::kModeLearned) {
            if (!ctx->mlp_ready) throw ApiError(NBX_ERR_STATE, "learned mode without network parameters");
            a.mlp_params = ctx->mlp_params.p;
            a.se_w = ctx->se_w.p;
            a.bse_w = ctx->bse_w.p;
            a.rr_threshold = ctx->rr_threshold;
            a.split_threshold = ctx->split_threshold;
            a.max_roulette_exp = ctx->max_roulette_exp;
            if (ctx->cost_bins > 0) {
                a.cost_table = ctx->cost_table.p;
                a.cost_bins = ctx->cost_bins;
                a.cost_materials = ctx->cost_materials;
                a.cost_log_e_min = ctx->cost_log_e_min;
                a.cost_inv_width = ctx->cost_inv_width;
                a.value_per_cost = ctx->value_per_cost;
            }
            a.birth_min_distance = ctx->birth_min_distance;
            a.birth_max_energy = ctx->birth_max_energy;
            a.birth_survival = ctx->birth_survival;
        }
        int mode = ctx->mode;
        if (mode == nbx::kModeLearned &&
            (ctx->imp_ne > 0 || (ctx->birth_survival > 0.0f && ctx->birth_survival < 1.0f))) {
            // birth decisions from the importance table or the fixed rule: the
            // weighted transport without a warp-synchronous network call
            mode = nbx::kModeWeighted;
            if (ctx->imp_ne > 0) {
                if (ctx->imp_version != ctx->mlp_version) build_importance_table(ctx);
                a.imp_table = ctx->imp_table.p;
                a.imp_ne = ctx->imp_ne;
                a.imp_nd = ctx->imp_nd;
                a.imp_nc = ctx->imp_nc;
                a.imp_materials = ctx->imp_materials;
            }
        }
        if (ctx->cfg.record_deposits) {
            // energy-deposit records (cpu_energydep.cpp's driver) ride on plain transport
            if (mode != nbx::kModePlain) throw ApiError(NBX_ERR_STATE, "energy deposits need the plain mode");
            mode = nbx::kModeDeposit;
            a.dep = ctx->dep.p;
            a.dep_cursor = ctx->dep_cursor.p;
            a.dep_capacity = ctx->dep_cap;
        }
        const int bpsm = nbx::transport_max_blocks_per_sm(ctx->block, ctx->variant, mode);
        const int grid = ctx->sms * bpsm;
        // parked-ancestor stacks of the launched threads (grow-only)
        ctx->stack_mem.ensure(uint64_t(grid) * uint64_t(ctx->block) * 3 * uint64_t(ctx->stack_depth));
        a.stack_mem = ctx->stack_mem.p;
        a.stack_depth = ctx->stack_depth;
        // The primaries are popped from per-SM ranges (neighbouring queue
        // entries stay on one SM); the secondary generations, written in
        // arbitrary order, from one shared cursor.
        if (!ctx->cfg.shared_pop) {
            ctx->range_cursor.ensure(uint64_t(ctx->sms));
            ck(cudaMemsetAsync(ctx->range_cursor.p, 0, sizeof(uint32_t) * ctx->sms, ctx->stream), "memset");
            a.n_ranges = uint32_t(ctx->sms);
        }

        ck(cudaEventRecord(ctx->ev0, ctx->stream), "event");
        int g = 0;
        bool done = false;
        while (!done) {
            for (int k = 0; k < ctx->chunk && g < kMaxGenerations; ++k, ++g) {
                const QueueBuf* in = g == 0 ? &ctx->prim : (g % 2 == 1 ? &ctx->qa : &ctx->qb);
                const QueueBuf* out = (g % 2 == 0) ? &ctx->qa : &ctx->qb;
                a.in = in->q();
                a.out = out->q();
                a.n_in = g == 0 ? ctl + 2 * kMaxGenerations : ctl + kMaxGenerations + (g - 1);
                a.head = ctl + g;
                a.range_cursor = (g == 0 && !ctx->cfg.shared_pop) ? ctx->range_cursor.p : nullptr;
                a.out_tail = ctl + kMaxGenerations + g;
                a.out_capacity = cap;
                a.in_capacity = uint32_t(std::min<uint64_t>(in->cap, 0xFFFFFFF0ull));
                ck(nbx::launch_transport(ctx->phys, a, grid, ctx->block, ctx->variant, ctx->stream, mode),
                   "transport launch");
            }
            uint32_t last = 0;
            ck(cudaMemcpyAsync(&last, ctl + kMaxGenerations + (g - 1), 4, cudaMemcpyDeviceToHost, ctx->stream), "D2H");
            ck(cudaStreamSynchronize(ctx->stream), "transport");
            if (last == 0) done = true;
            if (!done && g >= kMaxGenerations) throw ApiError(NBX_ERR_CAPACITY, "secondary generations exceed limit");
        }
        ck(cudaEventRecord(ctx->ev1, ctx->stream), "event");
        ck(cudaEventSynchronize(ctx->ev1), "event");
        float ms = 0;
        ck(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1), "elapsed");
        ctx->last_run_ms = ms;
        ctx->last_kernel_ms = ms;
        ctx->generations = uint64_t(g);
        ctx->n_queued = 0;
        // electrons lost to a full overflow queue in this run (the counter is
        // cumulative until nbx_reset_tallies)
        unsigned long long ovf = 0, ovf_before = 0;
        to_host(ctx, &ovf_before, ovf_snapshot, 8, "D2H");
        to_host(ctx, &ovf, ctx->counters.p + nbx::kCntOverflow, 8, "D2H");
        if (ovf > ovf_before) throw ApiError(NBX_ERR_CAPACITY, "secondary queue overflow: electrons lost");
        return NBX_OK;
    });
}

int nbx_get_running_count(nbx_ctx* ctx, uint64_t* n) {
    if (!ctx || !n) return NBX_ERR_ARG;
    *n = ctx->n_queued;
    return NBX_OK;
}

int nbx_get_stats(nbx_ctx* ctx, nbx_stats* out) {
    if (!ctx || !out) return NBX_ERR_ARG;
    return guarded(ctx, [&] {
        unsigned long long c[nbx::kNumCounters];
        to_host(ctx, c, ctx->counters.p, sizeof(c), "D2H");
        std::memset(out, 0, sizeof(*out));
        out->primaries_pushed = ctx->pushed;
        out->primaries_done = ctx->pushed - ctx->n_queued;
        out->steps = c[nbx::kCntSteps];
        out->events_elastic = c[nbx::kCntElastic];
        out->events_inelastic = c[nbx::kCntInelastic];
        out->events_boundary = c[nbx::kCntBoundary];
        out->secondaries = c[nbx::kCntSecondaries];
        out->detected = c[nbx::kCntDetected];
        out->detected_se = c[nbx::kCntDetectedSE];
        out->detected_bse = c[nbx::kCntDetectedBSE];
        out->terminated = c[nbx::kCntTerminated];
        out->records_dropped = c[nbx::kCntRecordsDropped];
        out->queue_overflow = c[nbx::kCntOverflow];
        out->inferences = c[nbx::kCntInferences];
        out->roulette_killed = c[nbx::kCntRouletteKilled];
        out->splits = c[nbx::kCntSplit];
        out->samples = c[nbx::kCntSamples];
        out->deposits = c[nbx::kCntDeposits];
        out->deposits_dropped = c[nbx::kCntDepositsDropped];
        out->generations = ctx->generations;
        out->last_run_ms = ctx->last_run_ms;
        out->last_kernel_ms = ctx->last_kernel_ms;
        return NBX_OK;
    });
}

int nbx_flush_detected(nbx_ctx* ctx, nbx_detected* out, uint64_t cap, uint64_t* n) {
    if (!ctx || !n || (cap && !out)) return NBX_ERR_ARG;
    return guarded(ctx, [&] {
        *n = 0;
        if (!ctx->rec.p) return NBX_OK;
        uint32_t cnt = 0;
        to_host(ctx, &cnt, ctx->rec_count.p, 4, "D2H");
        const uint64_t have = std::min<uint64_t>(cnt, ctx->rec_cap);
        const uint64_t take = std::min<uint64_t>(have - std::min(ctx->rec_read, have), cap);
        // the device already holds the records in the caller's layout: one copy
        static_assert(sizeof(nbx_detected) == 2 * sizeof(float4), "record layout");
        to_host(ctx, out, ctx->rec.p + 2 * ctx->rec_read, sizeof(nbx_detected) * take, "D2H");
        ctx->rec_read += take;
        if (ctx->rec_read >= have) {
            // everything read: the next records start at the front again
            zero(ctx, ctx->rec_count.p, 4, "memset");
            ctx->rec_read = 0;
        }
        *n = take;
        return NBX_OK;
    });
}

int nbx_get_tag_counts(nbx_ctx* ctx, uint64_t first, uint64_t n, uint32_t* se, uint32_t* bse) {
    if (!ctx) return NBX_ERR_ARG;
    if (first + n > ctx->n_tags) return fail(ctx, NBX_ERR_ARG, "tag range beyond nbx_set_tag_range");
    return guarded(ctx, [&] {
        if (n == 0) return NBX_OK;
        if (se) to_host(ctx, se, ctx->se_count.p + first, 4 * n, "D2H");
        if (bse) to_host(ctx, bse, ctx->bse_count.p + first, 4 * n, "D2H");
        return NBX_OK;
    });
}

int nbx_enable_pixel_spectra(nbx_ctx* ctx, uint64_t n_pixels, int32_t n_bins, float bin_width) {
    if (!ctx || n_bins < 0 || (n_pixels && (n_bins == 0 || !(bin_width > 0)))) return NBX_ERR_ARG;
    return guarded(ctx, [&] {
        ctx->pix_spec.release();
        ctx->spec_pixels = 0;
        if (n_pixels == 0) return NBX_OK;
        ctx->pix_spec.alloc(n_pixels * uint64_t(n_bins));
        zero(ctx, ctx->pix_spec.p, sizeof(float) * n_pixels * uint64_t(n_bins), "memset");
        ctx->spec_pixels = n_pixels;
        ctx->spec_bins = n_bins;
        ctx->spec_width = bin_width;
        return NBX_OK;
    });
}

int nbx_get_pixel_spectra(nbx_ctx* ctx, float* out) {
    if (!ctx || !out) return NBX_ERR_ARG;
    if (!ctx->spec_pixels) return fail(ctx, NBX_ERR_STATE, "per-pixel spectra not enabled");
    return guarded(ctx, [&] {
        ck(cudaMemcpyAsync(out, ctx->pix_spec.p, sizeof(float) * ctx->spec_pixels * uint64_t(ctx->spec_bins),
                           cudaMemcpyDeviceToHost, ctx->stream), "D2H");
        ck(cudaStreamSynchronize(ctx->stream), "sync");
        return NBX_OK;
    });
}

int nbx_set_pixel_map(nbx_ctx* ctx, const uint32_t* pixel_of_tag, uint64_t n_tags) {
    if (!ctx || (n_tags && !pixel_of_tag)) return NBX_ERR_ARG;
    return guarded(ctx, [&] {
        ctx->yield_map.ensure(std::max<uint64_t>(n_tags, 1));
        ck(cudaMemcpyAsync(ctx->yield_map.p, pixel_of_tag, 4 * n_tags, cudaMemcpyHostToDevice, ctx->stream), "H2D");
        ck(cudaStreamSynchronize(ctx->stream), "sync");
        ctx->pixel_map_len = n_tags;
        return NBX_OK;
    });
}

int nbx_pixel_yields(nbx_ctx* ctx, const uint32_t* pixel_of_tag, uint64_t n_tags, uint64_t n_pixels, double* out) {
    if (!ctx || !out) return NBX_ERR_ARG;
    if (n_tags > ctx->n_tags) return fail(ctx, NBX_ERR_ARG, "n_tags beyond the tallied range");
    if (!pixel_of_tag && n_tags > ctx->pixel_map_len)
        return fail(ctx, NBX_ERR_STATE, "no stored pixel map covering n_tags (nbx_set_pixel_map)");
    return guarded(ctx, [&] {
        if (pixel_of_tag) {
            ctx->yield_map.ensure(std::max<uint64_t>(n_tags, 1));
            ctx->pixel_map_len = 0;   // the stored map is overwritten
        }
        ctx->yield_out.ensure(std::max<uint64_t>(5 * n_pixels, 1));
        uint32_t* map = ctx->yield_map.p;
        double* res = ctx->yield_out.p;
        if (pixel_of_tag)
            ck(cudaMemcpyAsync(map, pixel_of_tag, 4 * n_tags, cudaMemcpyHostToDevice, ctx->stream), "H2D");
        ck(cudaMemsetAsync(res, 0, 8 * 5 * n_pixels, ctx->stream), "memset");
        const bool weighted = ctx->mode == nbx::kModeLearned;
        ck(nbx::launch_pixel_yields(ctx->se_count.p, ctx->bse_count.p, weighted ? ctx->se_w.p : nullptr,
                                    weighted ? ctx->bse_w.p : nullptr, map, n_tags, n_pixels, res, ctx->stream),
           "pixel yields");
        ck(cudaMemcpyAsync(out, res, 8 * 5 * n_pixels, cudaMemcpyDeviceToHost, ctx->stream), "D2H");
        ck(cudaStreamSynchronize(ctx->stream), "sync");
        return NBX_OK;
    });
}

int nbx_get_spectrum(nbx_ctx* ctx, uint64_t* counts, uint32_t n_bins, float* bin_width) {
    if (!ctx) return NBX_ERR_ARG;
    if (bin_width) *bin_width = kHistWidth;
    if (!counts) return NBX_OK;
    return guarded(ctx, [&] {
        const uint32_t n = std::min<uint32_t>(n_bins, kHistBins);
        to_host(ctx, counts, ctx->hist.p, 8ull * n, "D2H");
        return NBX_OK;
    });
}

int nbx_reset_tallies(nbx_ctx* ctx) {
    if (!ctx) return NBX_ERR_ARG;
    return guarded(ctx, [&] {
        ck(cudaMemsetAsync(ctx->counters.p, 0, 8 * nbx::kNumCounters, ctx->stream), "memset");
        ck(cudaMemsetAsync(ctx->hist.p, 0, 8ull * kHistBins, ctx->stream), "memset");
        ck(cudaMemsetAsync(ctx->rec_count.p, 0, 4, ctx->stream), "memset");
        ctx->rec_read = 0;
        if (ctx->spec_pixels)
            ck(cudaMemsetAsync(ctx->pix_spec.p, 0, sizeof(float) * ctx->spec_pixels * uint64_t(ctx->spec_bins),
                               ctx->stream), "memset");
        if (ctx->n_tags) {
            ck(cudaMemsetAsync(ctx->se_count.p, 0, 4 * ctx->n_tags, ctx->stream), "memset");
            ck(cudaMemsetAsync(ctx->bse_count.p, 0, 4 * ctx->n_tags, ctx->stream), "memset");
            ck(cudaMemsetAsync(ctx->se_w.p, 0, 4 * ctx->n_tags, ctx->stream), "memset");
            ck(cudaMemsetAsync(ctx->bse_w.p, 0, 4 * ctx->n_tags, ctx->stream), "memset");
        }
        ck(cudaStreamSynchronize(ctx->stream), "sync");
        ctx->pushed = ctx->n_queued;
        return NBX_OK;
    });
}

int nbx_ray_query(nbx_ctx* ctx, const float* pos, const float* dir, const float* dist, const int32_t* ignore_tri,
                  const int32_t* ignore_mat, uint64_t n, float* out_dist, int32_t* out_tri) {
    if (!ctx || (n && (!pos || !dir || !dist || !ignore_tri || !ignore_mat || !out_dist || !out_tri))) return NBX_ERR_ARG;
    if (!ctx->have_geometry) return fail(ctx, NBX_ERR_STATE, "no geometry");
    return guarded(ctx, [&] {
        if (n == 0) return NBX_OK;
        DevBuf<float> p, d, l, od;
        DevBuf<int32_t> it, im, ot;
        p.alloc(3 * n); d.alloc(3 * n); l.alloc(n); od.alloc(n);
        it.alloc(n); im.alloc(n); ot.alloc(n);
        auto s = ctx->stream;
        ck(cudaMemcpyAsync(p.p, pos, 12 * n, cudaMemcpyHostToDevice, s), "H2D");
        ck(cudaMemcpyAsync(d.p, dir, 12 * n, cudaMemcpyHostToDevice, s), "H2D");
        ck(cudaMemcpyAsync(l.p, dist, 4 * n, cudaMemcpyHostToDevice, s), "H2D");
        ck(cudaMemcpyAsync(it.p, ignore_tri, 4 * n, cudaMemcpyHostToDevice, s), "H2D");
        ck(cudaMemcpyAsync(im.p, ignore_mat, 4 * n, cudaMemcpyHostToDevice, s), "H2D");
        ck(nbx::launch_ray_query(ctx->phys.geo, p.p, d.p, l.p, it.p, im.p, n, od.p, ot.p, s), "ray query");
        ck(cudaMemcpyAsync(out_dist, od.p, 4 * n, cudaMemcpyDeviceToHost, s), "D2H");
        ck(cudaMemcpyAsync(out_tri, ot.p, 4 * n, cudaMemcpyDeviceToHost, s), "D2H");
        ck(cudaStreamSynchronize(s), "sync");
        return NBX_OK;
    });
}

int nbx_table_query(nbx_ctx* ctx, int32_t material, int32_t table, const float* x, const float* y, uint64_t n,
                    float* out) {
    if (!ctx || (n && (!x || !out))) return NBX_ERR_ARG;
    if (material < 0 || material >= ctx->n_mat || table < 0 || table > 4) return fail(ctx, NBX_ERR_ARG, "bad material/table");
    if (table == 4 && ctx->phys.penn) return fail(ctx, NBX_ERR_ARG, "no Kieft ionisation table under full Penn");
    return guarded(ctx, [&] {
        if (n == 0) return NBX_OK;
        DevBuf<float> dx, dy, dout;
        dx.alloc(n); dy.alloc(n); dout.alloc(n);
        auto s = ctx->stream;
        ck(cudaMemcpyAsync(dx.p, x, 4 * n, cudaMemcpyHostToDevice, s), "H2D");
        if (y) ck(cudaMemcpyAsync(dy.p, y, 4 * n, cudaMemcpyHostToDevice, s), "H2D");
        else ck(cudaMemsetAsync(dy.p, 0, 4 * n, s), "memset");
        ck(nbx::launch_table_query(ctx->phys.mat[material], table, dx.p, dy.p, n, dout.p, s), "table query");
        ck(cudaMemcpyAsync(out, dout.p, 4 * n, cudaMemcpyDeviceToHost, s), "D2H");
        ck(cudaStreamSynchronize(s), "sync");
        return NBX_OK;
    });
}

int nbx_table3_query(nbx_ctx* ctx, int32_t material, int32_t table, const float* x, const float* y, const float* z,
                     uint64_t n, float* out) {
    if (!ctx || (n && (!x || !y || !z || !out))) return NBX_ERR_ARG;
    if (material < 0 || material >= ctx->n_mat || table < 0 || table > 1) return fail(ctx, NBX_ERR_ARG, "bad material/table");
    if (!ctx->phys.penn) return fail(ctx, NBX_ERR_STATE, "3-D tables are loaded only for the full Penn model");
    return guarded(ctx, [&] {
        if (n == 0) return NBX_OK;
        DevBuf<float> dx, dy, dz, dout;
        dx.alloc(n); dy.alloc(n); dz.alloc(n); dout.alloc(n);
        auto s = ctx->stream;
        ck(cudaMemcpyAsync(dx.p, x, 4 * n, cudaMemcpyHostToDevice, s), "H2D");
        ck(cudaMemcpyAsync(dy.p, y, 4 * n, cudaMemcpyHostToDevice, s), "H2D");
        ck(cudaMemcpyAsync(dz.p, z, 4 * n, cudaMemcpyHostToDevice, s), "H2D");
        ck(nbx::launch_table3_query(ctx->phys.mat[material], table, dx.p, dy.p, dz.p, n, dout.p, s), "table query");
        ck(cudaMemcpyAsync(out, dout.p, 4 * n, cudaMemcpyDeviceToHost, s), "D2H");
        ck(cudaStreamSynchronize(s), "sync");
        return NBX_OK;
    });
}

int nbx_flush_deposits(nbx_ctx* ctx, nbx_deposit* out, uint64_t capacity, uint64_t* n_out) {
    if (!ctx || !n_out || (capacity && !out)) return NBX_ERR_ARG;
    if (!ctx->cfg.record_deposits) return fail(ctx, NBX_ERR_STATE, "context created without record_deposits");
    return guarded(ctx, [&] {
        *n_out = 0;
        unsigned long long cursor = 0;
        ck(cudaMemcpyAsync(&cursor, ctx->dep_cursor.p, sizeof cursor, cudaMemcpyDeviceToHost, ctx->stream), "D2H");
        ck(cudaStreamSynchronize(ctx->stream), "sync");
        const uint64_t end = std::min<uint64_t>(cursor, ctx->dep_cap);
        // copy slot ranges from where the last call stopped, dropping the
        // unused tails of the threads' chunks, until `capacity` records
        std::vector<float> stage;
        const uint64_t kStage = 1ull << 20;
        while (ctx->dep_flushed < end && *n_out < capacity) {
            const uint64_t take = std::min<uint64_t>(kStage, end - ctx->dep_flushed);
            stage.resize(take * nbx::kDepositWords);
            ck(cudaMemcpyAsync(stage.data(), ctx->dep.p + ctx->dep_flushed * nbx::kDepositWords,
                               sizeof(float) * stage.size(), cudaMemcpyDeviceToHost, ctx->stream), "D2H");
            ck(cudaStreamSynchronize(ctx->stream), "sync");
            uint64_t used = 0;
            for (; used < take && *n_out < capacity; ++used) {
                const float* r = stage.data() + used * nbx::kDepositWords;
                uint32_t tag;
                std::memcpy(&tag, r + 5, 4);
                if (tag == nbx::kDepositEmpty) continue;
                nbx_deposit& d = out[(*n_out)++];
                d.pos[0] = r[0];
                d.pos[1] = r[1];
                d.pos[2] = r[2];
                d.E = r[3];
                d.dE = r[4];
                d.tag = tag;
            }
            ctx->dep_flushed += used;
        }
        if (ctx->dep_flushed >= end) {
            // everything handed out: start the buffer over
            ck(cudaMemsetAsync(ctx->dep_cursor.p, 0, sizeof(unsigned long long), ctx->stream), "memset");
            ck(cudaStreamSynchronize(ctx->stream), "sync");
            ctx->dep_flushed = 0;
        }
        return NBX_OK;
    });
}

int nbx_philox(nbx_ctx* ctx, const uint32_t* ctr, const uint32_t* key, uint64_t n, uint32_t* out) {
    if (!ctx || (n && (!ctr || !key || !out))) return NBX_ERR_ARG;
    return guarded(ctx, [&] {
        if (n == 0) return NBX_OK;
        DevBuf<uint32_t> c, k, o;
        c.alloc(4 * n); k.alloc(2 * n); o.alloc(4 * n);
        auto s = ctx->stream;
        ck(cudaMemcpyAsync(c.p, ctr, 16 * n, cudaMemcpyHostToDevice, s), "H2D");
        ck(cudaMemcpyAsync(k.p, key, 8 * n, cudaMemcpyHostToDevice, s), "H2D");
        ck(nbx::launch_philox(c.p, k.p, n, o.p, s), "philox");
        ck(cudaMemcpyAsync(out, o.p, 16 * n, cudaMemcpyDeviceToHost, s), "D2H");
        ck(cudaStreamSynchronize(s), "sync");
        return NBX_OK;
    });
}

int nbx_step_query(nbx_ctx* ctx, nbx_electron* electrons, uint64_t n, int32_t* status, int32_t* event,
                   nbx_electron* secondaries, int32_t* has_se) {
    if (!ctx || (n && (!electrons || !status || !event || !secondaries || !has_se))) return NBX_ERR_ARG;
    if (!ctx->have_geometry) return fail(ctx, NBX_ERR_STATE, "no geometry");
    static_assert(sizeof(nbx_electron) == 56, "nbx_electron layout");
    return guarded(ctx, [&] {
        if (n == 0) return NBX_OK;
        for (uint64_t i = 0; i < n; ++i) {
            const int m = electrons[i].mat;
            if (m >= ctx->n_mat) throw ApiError(NBX_ERR_ARG, "electron material index out of range");
            const int t = electrons[i].last_tri;
            if (t >= ctx->phys.geo.n_tri) throw ApiError(NBX_ERR_ARG, "electron triangle index out of range");
        }
        DevBuf<uint8_t> e, se;
        DevBuf<int32_t> st, ev, hs;
        e.alloc(56 * n); se.alloc(56 * n); st.alloc(n); ev.alloc(n); hs.alloc(n);
        auto s = ctx->stream;
        ck(cudaMemcpyAsync(e.p, electrons, 56 * n, cudaMemcpyHostToDevice, s), "H2D");
        ck(cudaMemsetAsync(se.p, 0, 56 * n, s), "memset");
        ck(nbx::launch_step_query(ctx->phys, e.p, n, st.p, ev.p, se.p, hs.p, s), "step query");
        ck(cudaMemcpyAsync(electrons, e.p, 56 * n, cudaMemcpyDeviceToHost, s), "D2H");
        ck(cudaMemcpyAsync(secondaries, se.p, 56 * n, cudaMemcpyDeviceToHost, s), "D2H");
        ck(cudaMemcpyAsync(status, st.p, 4 * n, cudaMemcpyDeviceToHost, s), "D2H");
        ck(cudaMemcpyAsync(event, ev.p, 4 * n, cudaMemcpyDeviceToHost, s), "D2H");
        ck(cudaMemcpyAsync(has_se, hs.p, 4 * n, cudaMemcpyDeviceToHost, s), "D2H");
        ck(cudaStreamSynchronize(s), "sync");
        return NBX_OK;
    });
}

int nbx_set_tuning(nbx_ctx* ctx, const nbx_tuning* t) {
    if (!ctx || !t) return NBX_ERR_ARG;
    const int v = t->blocks_per_sm, b = t->block_size;
    if (!((v >= 2 && v <= 4) || v == 7) || b <= 0 || b % 32 != 0 || b > (v == 7 ? 128 : 256) ||
        t->stack_depth < 1 || t->stack_depth > nbx::kMaxStack || t->chunk < 1 || t->chunk > 64)
        return fail(ctx, NBX_ERR_ARG, "nbx_set_tuning: variant 2/3/4 with blocks of 32..256 threads or 7 with "
                                      "32..128, stack depth 1..64, chunk 1..64");
    return guarded(ctx, [&] {
        ctx->variant = v;
        ctx->block = b;
        ctx->bpsm = nbx::transport_max_blocks_per_sm(b, v);
        ctx->stack_depth = t->stack_depth;
        ctx->chunk = t->chunk;
        return NBX_OK;
    });
}

int nbx_get_tuning(nbx_ctx* ctx, nbx_tuning* t) {
    if (!ctx || !t) return NBX_ERR_ARG;
    t->blocks_per_sm = ctx->variant;
    t->block_size = ctx->block;
    t->stack_depth = ctx->stack_depth;
    t->chunk = ctx->chunk;
    t->queue_capacity = ctx->queue_capacity;
    t->sample_ms = 0;
    return NBX_OK;
}

int nbx_autotune(nbx_ctx* ctx, const nbx_particle* particles, const uint32_t* tags, uint64_t n, nbx_tuning* out) {
    if (!ctx || !particles || !tags || n == 0) return NBX_ERR_ARG;
    if (!ctx->have_geometry) return fail(ctx, NBX_ERR_STATE, "nbx_autotune before nbx_set_geometry");
    if (ctx->n_queued) return fail(ctx, NBX_ERR_STATE, "nbx_autotune with primaries queued");
    const uint64_t uid_save = ctx->uid_next;
    // Time the sample with the context's current settings (its mode
    // included): twice on the same random streams, the first pass also
    // paying one-time costs (module load, buffer growth); the second is kept.
    // A setting whose run loses electrons to a full overflow queue (a stack
    // too shallow for the sample's cascades) is not a candidate.
    auto time_it = [&](double* ms) {
        for (int rep = 0; rep < 2; ++rep) {
            ctx->uid_next = uid_save;
            int rc = nbx_push(ctx, particles, tags, n, nullptr);
            if (rc == NBX_OK) rc = nbx_run(ctx);
            if (rc == NBX_ERR_CAPACITY) {
                *ms = 1e300;
                ctx->err.clear();
                return NBX_OK;
            }
            if (rc != NBX_OK) return rc;
        }
        *ms = ctx->last_run_ms;
        return NBX_OK;
    };
    double best = 1e300;
    // 1. launch shape: transport variant x block size
    int best_v = ctx->variant, best_b = ctx->block;
    const int variants[4] = {2, 3, 4, 7};
    const int blocks[2] = {256, 128};
    for (int v : variants) {
        for (int b : blocks) {
            if (v == 7 && b > 128) continue;   // 128-thread variant
            ctx->variant = v;
            ctx->block = b;
            ctx->bpsm = nbx::transport_max_blocks_per_sm(b, v);
            double ms = 0;
            const int rc = time_it(&ms);
            if (rc != NBX_OK) return rc;
            if (ms < best) {
                best = ms;
                best_v = v;
                best_b = b;
            }
        }
    }
    ctx->variant = best_v;
    ctx->block = best_b;
    ctx->bpsm = nbx::transport_max_blocks_per_sm(best_b, best_v);
    // 2. parked-stack depth: a shallower stack sends deep cascades' secondaries
    // through the next generation's queue sooner; a deeper one holds more
    // global memory per thread
    int best_depth = ctx->stack_depth;
    for (int d : {8, 32}) {
        ctx->stack_depth = d;
        double ms = 0;
        const int rc = time_it(&ms);
        if (rc != NBX_OK) return rc;
        if (ms < best) {
            best = ms;
            best_depth = d;
        }
    }
    ctx->stack_depth = best_depth;
    // 3. generation launches queued between two host reads of the last
    // generation's size
    int best_chunk = ctx->chunk;
    for (int c : {2, 16}) {
        ctx->chunk = c;
        double ms = 0;
        const int rc = time_it(&ms);
        if (rc != NBX_OK) return rc;
        if (ms < best) {
            best = ms;
            best_chunk = c;
        }
    }
    ctx->chunk = best_chunk;
    ctx->uid_next = uid_save;
    if (out) {
        nbx_get_tuning(ctx, out);
        out->sample_ms = best;
    }
    return nbx_reset_tallies(ctx);
}

int nbx_set_uid_base(nbx_ctx* ctx, uint64_t base) {
    if (!ctx) return NBX_ERR_ARG;
    if (base >= (1ull << 63)) return fail(ctx, NBX_ERR_ARG, "uid base must be below 2^63");
    ctx->uid_next = base;
    return NBX_OK;
}

int nbx_set_mode(nbx_ctx* ctx, int32_t mode, float rr_threshold, float split_threshold, int32_t max_roulette_exp) {
    if (!ctx || mode < 0 || mode > 2 || !(rr_threshold >= 0) || !(split_threshold > 0) || max_roulette_exp < 1 ||
        max_roulette_exp > 12)
        return NBX_ERR_ARG;
    ctx->mode = mode;
    ctx->rr_threshold = rr_threshold;
    ctx->split_threshold = split_threshold;
    ctx->max_roulette_exp = max_roulette_exp;
    return NBX_OK;
}

int nbx_set_birth_roulette(nbx_ctx* ctx, float min_distance, float max_energy, float survival) {
    if (!ctx || !(min_distance >= 0) || !(max_energy >= 0) || !(survival >= 0) || survival > 1) return NBX_ERR_ARG;
    ctx->birth_min_distance = min_distance;
    ctx->birth_max_energy = max_energy;
    ctx->birth_survival = survival;
    return NBX_OK;
}

int nbx_set_learned_cost(nbx_ctx* ctx, const float* mean_cost, int32_t n_materials, int32_t n_bins,
                         float log_e_min, float log_e_max, float value_per_cost) {
    if (!ctx || n_bins < 0) return NBX_ERR_ARG;
    if (n_bins == 0) {
        ctx->cost_bins = 0;
        return NBX_OK;
    }
    if (!mean_cost || n_materials < 1 || n_materials > NBX_MAX_MATERIALS || n_bins > 4096 ||
        !(log_e_max > log_e_min) || !(value_per_cost > 0))
        return fail(ctx, NBX_ERR_ARG, "nbx_set_learned_cost: bad table shape, energy range or value per cost");
    for (int64_t i = 0; i < int64_t(n_materials) * n_bins; ++i)
        if (!(mean_cost[i] > 0) || !std::isfinite(mean_cost[i]))
            return fail(ctx, NBX_ERR_ARG, "nbx_set_learned_cost: costs must be positive and finite");
    return guarded(ctx, [&] {
        ctx->cost_table.alloc(uint64_t(n_materials) * n_bins);
        to_device(ctx, ctx->cost_table.p, mean_cost, sizeof(float) * size_t(n_materials) * n_bins, "H2D");
        ctx->cost_bins = n_bins;
        ctx->cost_materials = n_materials;
        ctx->cost_log_e_min = log_e_min;
        ctx->cost_inv_width = float(n_bins) / (log_e_max - log_e_min);
        ctx->value_per_cost = value_per_cost;
        return NBX_OK;
    });
}

int nbx_build_surface_map(nbx_ctx* ctx, const float lo[3], const float hi[3], float cell, float d_max) {
    if (!ctx || !lo || !hi || !(cell > 0) || !(d_max > 0)) return NBX_ERR_ARG;
    if (!ctx->have_geometry) return fail(ctx, NBX_ERR_STATE, "surface map before nbx_set_geometry");
    return guarded(ctx, [&] {
        int n[3];
        for (int k = 0; k < 3; ++k) {
            if (!(hi[k] > lo[k])) throw ApiError(NBX_ERR_ARG, "empty surface-map box");
            n[k] = int(std::ceil((hi[k] - lo[k]) / cell));
        }
        const uint64_t cells = uint64_t(n[0]) * n[1] * n[2];
        if (cells > (1ull << 31)) throw ApiError(NBX_ERR_ARG, "surface map larger than 2^31 cells");
        // Candidates, binned into bricks of kBrick^3 cells: a brick lists, in
        // triangle order, every material triangle whose bounding box comes
        // within d_max of the brick.  A triangle within d_max of a cell
        // centre has its box within d_max of that centre, so each cell's
        // brick list holds every triangle the nearest search could pick,
        // and the search (strictly smaller distance wins, in list order)
        // picks what a search over all triangles would.
        constexpr int kBrick = 8;
        int nb[3];
        for (int k = 0; k < 3; ++k) nb[k] = (n[k] + kBrick - 1) / kBrick;
        const uint64_t bricks = uint64_t(nb[0]) * nb[1] * nb[2];
        const double bs = double(kBrick) * cell;
        std::vector<float4> t(3 * size_t(ctx->phys.geo.n_tri));
        to_host(ctx, t.data(), ctx->tris.p, sizeof(float4) * t.size(), "D2H");
        struct Range { int b0[3], b1[3]; };
        std::vector<std::pair<int, Range>> cand;
        for (int i = 0; i < ctx->phys.geo.n_tri; ++i) {
            const float4 r0 = t[3 * i], e1 = t[3 * i + 1], e2 = t[3 * i + 2];
            int mi;
            std::memcpy(&mi, &r0.w, 4);
            if (mi < 0) continue;   // detector / special sheets are not material surfaces
            const float xs[3] = {r0.x, r0.x + e1.x, r0.x + e2.x}, ys[3] = {r0.y, r0.y + e1.y, r0.y + e2.y},
                        zs[3] = {r0.z, r0.z + e1.z, r0.z + e2.z};
            const double mn[3] = {std::min({xs[0], xs[1], xs[2]}), std::min({ys[0], ys[1], ys[2]}), std::min({zs[0], zs[1], zs[2]})};
            const double mx[3] = {std::max({xs[0], xs[1], xs[2]}), std::max({ys[0], ys[1], ys[2]}), std::max({zs[0], zs[1], zs[2]})};
            Range r;
            bool inside = true;
            // reach: d_max plus 1e-3 nm for the float rounding of the cell
            // centres the kernel measures from
            const double reach = double(d_max) + 1e-3;
            for (int k = 0; k < 3; ++k) {
                const double a = std::floor((mn[k] - reach - lo[k]) / bs), b = std::floor((mx[k] + reach - lo[k]) / bs);
                if (b < 0 || a > nb[k] - 1) inside = false;
                r.b0[k] = int(std::max(a, 0.0));
                r.b1[k] = int(std::min(b, double(nb[k] - 1)));
            }
            if (inside) cand.push_back({i, r});
        }
        std::vector<uint64_t> start(bricks + 1, 0);
        for (const auto& c : cand)
            for (int z = c.second.b0[2]; z <= c.second.b1[2]; ++z)
                for (int y = c.second.b0[1]; y <= c.second.b1[1]; ++y)
                    for (int x = c.second.b0[0]; x <= c.second.b1[0]; ++x)
                        ++start[(uint64_t(z) * nb[1] + y) * nb[0] + x + 1];
        for (uint64_t b = 0; b < bricks; ++b) start[b + 1] += start[b];
        if (start[bricks] > 0xFFFFFFFFull) throw ApiError(NBX_ERR_ARG, "surface map: too many brick entries");
        std::vector<int32_t> list(std::max<uint64_t>(start[bricks], 1));
        {
            std::vector<uint64_t> fill(start.begin(), start.end() - 1);
            for (const auto& c : cand)
                for (int z = c.second.b0[2]; z <= c.second.b1[2]; ++z)
                    for (int y = c.second.b0[1]; y <= c.second.b1[1]; ++y)
                        for (int x = c.second.b0[0]; x <= c.second.b1[0]; ++x)
                            list[fill[(uint64_t(z) * nb[1] + y) * nb[0] + x]++] = c.first;
        }
        std::vector<uint32_t> start32(start.begin(), start.end());
        ctx->smap_cells.alloc(std::max<uint64_t>(cells, 1));
        DevBuf<uint32_t> dstart;
        DevBuf<int32_t> dlist;
        dstart.alloc(start32.size());
        dlist.alloc(list.size());
        to_device(ctx, dstart.p, start32.data(), 4 * start32.size(), "H2D");
        to_device(ctx, dlist.p, list.data(), 4 * list.size(), "H2D");
        ck(nbx::launch_build_surface_map(ctx->tris.p, dstart.p, dlist.p, nb[0], nb[1], kBrick, ctx->smap_cells.p, lo[0],
                                         lo[1], lo[2], cell, n[0], n[1], n[2], d_max, ctx->stream), "surface map");
        ck(cudaStreamSynchronize(ctx->stream), "surface map");
        ctx->smap.cell = ctx->smap_cells.p;
        ctx->smap.lox = lo[0];
        ctx->smap.loy = lo[1];
        ctx->smap.loz = lo[2];
        ctx->smap.cell_size = cell;
        ctx->smap.inv_cell = 1.0f / cell;
        ctx->smap.nx = n[0];
        ctx->smap.ny = n[1];
        ctx->smap.nz = n[2];
        ctx->smap.d_max = d_max;
        return NBX_OK;
    });
}

int nbx_set_sample_capacity(nbx_ctx* ctx, uint64_t capacity) {
    if (!ctx || capacity == 0) return NBX_ERR_ARG;
    return guarded(ctx, [&] {
        ctx->sample_feat.alloc(6 * capacity);
        ctx->sample_label.alloc(capacity);
        ctx->sample_cost.alloc(capacity);
        ctx->sample_count.alloc(1);
        zero(ctx, ctx->sample_count.p, 4, "memset");
        zero(ctx, ctx->sample_label.p, 4 * capacity, "memset");
        zero(ctx, ctx->sample_cost.p, 4 * capacity, "memset");
        ctx->sample_cap = capacity;
        return NBX_OK;
    });
}

int nbx_get_samples(nbx_ctx* ctx, float* features, float* labels, float* costs, uint64_t cap, uint64_t* n) {
    if (!ctx || !n || (cap && (!features || !labels))) return NBX_ERR_ARG;
    return guarded(ctx, [&] {
        *n = 0;
        if (!ctx->sample_cap) return NBX_OK;
        uint32_t cnt = 0;
        to_host(ctx, &cnt, ctx->sample_count.p, 4, "D2H");
        const uint64_t have = std::min<uint64_t>(cnt, ctx->sample_cap);
        const uint64_t take = std::min<uint64_t>(have, cap);
        if (take) {
            to_host(ctx, features, ctx->sample_feat.p, 24 * take, "D2H");
            to_host(ctx, labels, ctx->sample_label.p, 4 * take, "D2H");
            if (costs) to_host(ctx, costs, ctx->sample_cost.p, 4 * take, "D2H");
        }
        zero(ctx, ctx->sample_count.p, 4, "memset");
        zero(ctx, ctx->sample_label.p, 4 * ctx->sample_cap, "memset");
        zero(ctx, ctx->sample_cost.p, 4 * ctx->sample_cap, "memset");
        *n = take;
        return NBX_OK;
    });
}

int nbx_get_tag_weights(nbx_ctx* ctx, uint64_t first, uint64_t n, float* se_w, float* bse_w) {
    if (!ctx) return NBX_ERR_ARG;
    if (first + n > ctx->n_tags) return fail(ctx, NBX_ERR_ARG, "tag range beyond nbx_set_tag_range");
    return guarded(ctx, [&] {
        if (n == 0) return NBX_OK;
        if (se_w) to_host(ctx, se_w, ctx->se_w.p + first, 4 * n, "D2H");
        if (bse_w) to_host(ctx, bse_w, ctx->bse_w.p + first, 4 * n, "D2H");
        return NBX_OK;
    });
}

int nbx_features_query(nbx_ctx* ctx, const nbx_electron* electrons, uint64_t n, float* out) {
    if (!ctx || (n && (!electrons || !out))) return NBX_ERR_ARG;
    if (!ctx->have_geometry) return fail(ctx, NBX_ERR_STATE, "no geometry");
    return guarded(ctx, [&] {
        if (n == 0) return NBX_OK;
        DevBuf<uint8_t> e;
        DevBuf<float> f;
        e.alloc(56 * n);
        f.alloc(6 * n);
        ck(cudaMemcpyAsync(e.p, electrons, 56 * n, cudaMemcpyHostToDevice, ctx->stream), "H2D");
        ck(nbx::launch_features(ctx->smap, e.p, n, f.p, ctx->stream), "features");
        ck(cudaMemcpyAsync(out, f.p, 24 * n, cudaMemcpyDeviceToHost, ctx->stream), "D2H");
        ck(cudaStreamSynchronize(ctx->stream), "sync");
        return NBX_OK;
    });
}

// ---- escape-probability network ----------------------------------------
namespace {
void mlp_alloc(nbx_ctx* ctx) {
    if (ctx->mlp_params.p) return;
    ctx->mlp_params.alloc(nbx::mlp::kParams);
    ctx->mlp_m.alloc(nbx::mlp::kParams);
    ctx->mlp_v.alloc(nbx::mlp::kParams);
    ctx->mlp_grad.alloc(nbx::mlp::kParams);
    ctx->mlp_loss.alloc(1);
    zero(ctx, ctx->mlp_params.p, 4 * nbx::mlp::kParams, "memset");
    zero(ctx, ctx->mlp_m.p, 4 * nbx::mlp::kParams, "memset");
    zero(ctx, ctx->mlp_v.p, 4 * nbx::mlp::kParams, "memset");
}
void mlp_upload(nbx_ctx* ctx, const float* features, const float* labels, uint64_t n) {
    ctx->mlp_feat.ensure(std::max<uint64_t>(n, 1) * nbx::mlp::kFeatures);
    ck(cudaMemcpyAsync(ctx->mlp_feat.p, features, 4 * n * nbx::mlp::kFeatures, cudaMemcpyHostToDevice, ctx->stream), "H2D");
    if (labels) {
        ctx->mlp_lab.ensure(std::max<uint64_t>(n, 1));
        ck(cudaMemcpyAsync(ctx->mlp_lab.p, labels, 4 * n, cudaMemcpyHostToDevice, ctx->stream), "H2D");
    }
}
}  // namespace

int nbx_mlp_set_params(nbx_ctx* ctx, const float* params) {
    if (!ctx || !params) return NBX_ERR_ARG;
    return guarded(ctx, [&] {
        mlp_alloc(ctx);
        std::vector<float> p(params, params + nbx::mlp::kParams);
        // padding entries must stay zero (inputs 6..15, outputs 1..7)
        for (int o = 0; o < nbx::mlp::kHidden; ++o)
            for (int i = nbx::mlp::kFeatures; i < nbx::mlp::kIn; ++i) p[nbx::mlp::kOffW1 + o * nbx::mlp::kIn + i] = 0;
        for (int o = 1; o < nbx::mlp::kOut; ++o) {
            for (int i = 0; i < nbx::mlp::kHidden; ++i) p[nbx::mlp::kOffW3 + o * nbx::mlp::kHidden + i] = 0;
            p[nbx::mlp::kOffB3 + o] = 0;
        }
        to_device(ctx, ctx->mlp_params.p, p.data(), 4 * nbx::mlp::kParams, "H2D");
        zero(ctx, ctx->mlp_m.p, 4 * nbx::mlp::kParams, "memset");
        zero(ctx, ctx->mlp_v.p, 4 * nbx::mlp::kParams, "memset");
        ctx->mlp_step = 0;
        ctx->mlp_ready = true;
        ++ctx->mlp_version;
        return NBX_OK;
    });
}

int nbx_mlp_get_params(nbx_ctx* ctx, float* out) {
    if (!ctx || !out) return NBX_ERR_ARG;
    if (!ctx->mlp_ready) return fail(ctx, NBX_ERR_STATE, "network parameters not set");
    return guarded(ctx, [&] {
        to_host(ctx, out, ctx->mlp_params.p, 4 * nbx::mlp::kParams, "D2H");
        return NBX_OK;
    });
}

int nbx_mlp_grad(nbx_ctx* ctx, const float* features, const float* labels, uint64_t n, float* grad, float* loss) {
    if (!ctx || !features || !labels || n == 0 || !grad) return NBX_ERR_ARG;
    if (!ctx->mlp_ready) return fail(ctx, NBX_ERR_STATE, "network parameters not set");
    return guarded(ctx, [&] {
        mlp_upload(ctx, features, labels, n);
        ck(cudaMemsetAsync(ctx->mlp_grad.p, 0, 4 * nbx::mlp::kParams, ctx->stream), "memset");
        ck(cudaMemsetAsync(ctx->mlp_loss.p, 0, 4, ctx->stream), "memset");
        ck(nbx::mlp::launch_train(ctx->mlp_params.p, ctx->mlp_feat.p, ctx->mlp_lab.p, nullptr, 0, n, 1.0f / float(n),
                                  ctx->mlp_grad.p, ctx->mlp_loss.p, ctx->stream), "train kernel");
        ck(cudaMemcpyAsync(grad, ctx->mlp_grad.p, 4 * nbx::mlp::kParams, cudaMemcpyDeviceToHost, ctx->stream), "D2H");
        float l = 0;
        ck(cudaMemcpyAsync(&l, ctx->mlp_loss.p, 4, cudaMemcpyDeviceToHost, ctx->stream), "D2H");
        ck(cudaStreamSynchronize(ctx->stream), "sync");
        if (loss) *loss = l;
        return NBX_OK;
    });
}

int nbx_mlp_train(nbx_ctx* ctx, const float* features, const float* labels, uint64_t n, int32_t epochs,
                  int32_t batch, float lr, uint32_t seed, float* loss_per_epoch) {
    if (!ctx || !features || !labels || n == 0 || epochs <= 0 || batch <= 0 || !(lr > 0)) return NBX_ERR_ARG;
    if (!ctx->mlp_ready) return fail(ctx, NBX_ERR_STATE, "network parameters not set");
    return guarded(ctx, [&] {
        mlp_upload(ctx, features, labels, n);
        ctx->mlp_index.ensure(n);
        std::vector<uint32_t> perm(n);
        uint64_t state = 0x9E3779B97F4A7C15ull ^ seed;
        auto next = [&]() {   // splitmix64
            uint64_t z = (state += 0x9E3779B97F4A7C15ull);
            z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
            z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
            return z ^ (z >> 31);
        };
        for (int ep = 0; ep < epochs; ++ep) {
            for (uint64_t i = 0; i < n; ++i) perm[i] = uint32_t(i);
            for (uint64_t i = n - 1; i > 0; --i) std::swap(perm[i], perm[next() % (i + 1)]);
            ck(cudaMemcpyAsync(ctx->mlp_index.p, perm.data(), 4 * n, cudaMemcpyHostToDevice, ctx->stream), "H2D");
            ck(cudaMemsetAsync(ctx->mlp_loss.p, 0, 4, ctx->stream), "memset");
            uint64_t n_batches = 0;
            for (uint64_t first = 0; first + uint64_t(batch) <= n || (first == 0 && n < uint64_t(batch));
                 first += uint64_t(batch)) {
                const uint64_t count = std::min<uint64_t>(uint64_t(batch), n - first);
                ck(cudaMemsetAsync(ctx->mlp_grad.p, 0, 4 * nbx::mlp::kParams, ctx->stream), "memset");
                ck(nbx::mlp::launch_train(ctx->mlp_params.p, ctx->mlp_feat.p, ctx->mlp_lab.p, ctx->mlp_index.p, first,
                                          count, 1.0f / float(count), ctx->mlp_grad.p, ctx->mlp_loss.p, ctx->stream),
                   "train kernel");
                ck(nbx::mlp::launch_adam(ctx->mlp_params.p, ctx->mlp_grad.p, ctx->mlp_m.p, ctx->mlp_v.p, lr, 0.9f,
                                         0.999f, 1e-8f, ++ctx->mlp_step, ctx->stream), "adam kernel");
                ++n_batches;
            }
            float l = 0;
            ck(cudaMemcpyAsync(&l, ctx->mlp_loss.p, 4, cudaMemcpyDeviceToHost, ctx->stream), "D2H");
            ck(cudaStreamSynchronize(ctx->stream), "sync");
            if (loss_per_epoch) loss_per_epoch[ep] = l / float(std::max<uint64_t>(n_batches, 1));
        }
        ++ctx->mlp_version;
        return NBX_OK;
    });
}

int nbx_mlp_predict(nbx_ctx* ctx, const float* features, uint64_t n, float* out) {
    if (!ctx || !features || !out) return NBX_ERR_ARG;
    if (!ctx->mlp_ready) return fail(ctx, NBX_ERR_STATE, "network parameters not set");
    return guarded(ctx, [&] {
        if (n == 0) return NBX_OK;
        mlp_upload(ctx, features, nullptr, n);
        ctx->mlp_out.ensure(n);
        ck(nbx::mlp::launch_predict(ctx->mlp_params.p, ctx->mlp_feat.p, n, ctx->mlp_out.p, ctx->stream), "predict");
        ck(cudaMemcpyAsync(out, ctx->mlp_out.p, 4 * n, cudaMemcpyDeviceToHost, ctx->stream), "D2H");
        ck(cudaStreamSynchronize(ctx->stream), "sync");
        return NBX_OK;
    });
}

// Allocation-free transport (see include/nbx.h): device buffers in, device
// tallies out, scratch from the library's file-scope array.  Nothing here or
// in run_transport_noalloc allocates memory.  The array's device address is
// looked up on the context's first call, with the context's device current;
// a context never outlives the device's primary context (cudaDeviceReset
// invalidates its streams and buffers too), so the address cannot go stale.
int nbx_run_noalloc(nbx_ctx* ctx, const float* d_particles, const uint32_t* d_tags, uint32_t n, uint64_t uid_base,
                    uint32_t* d_se_count, uint32_t* d_bse_count, uint64_t n_tags, uint64_t counts[4]) {
    if (!ctx || (n && (!d_particles || !d_tags)) || (n_tags && (!d_se_count || !d_bse_count))) return NBX_ERR_ARG;
    if (!ctx->have_geometry) return fail(ctx, NBX_ERR_STATE, "nbx_run_noalloc before nbx_set_geometry");
    if (n > NBX_NOALLOC_MAX_PRIMARIES)
        return fail(ctx, NBX_ERR_ARG, "nbx_run_noalloc takes at most NBX_NOALLOC_MAX_PRIMARIES (65536) primaries per call");
    if (uid_base >= (1ull << 63) || uint64_t(n) > (1ull << 63) - uid_base)
        return fail(ctx, NBX_ERR_ARG, "nbx_run_noalloc: uid_base + n must not exceed 2^63");
    if (ctx->mode != nbx::kModePlain || ctx->cfg.record_deposits)
        return fail(ctx, NBX_ERR_STATE,
                    "nbx_run_noalloc runs plain transport only: the context is in sample or learned mode, or "
                    "records energy deposits");
    ctx->err.clear();
    if (cudaSetDevice(ctx->cfg.device) != cudaSuccess) return fail(ctx, NBX_ERR_CUDA, "cudaSetDevice failed");
    if (!ctx->noalloc_scratch) {
        void* p = nullptr;
        if (nbx::noalloc_scratch_address(&p) != cudaSuccess || !p) {
            cudaGetLastError();
            return fail(ctx, NBX_ERR_CUDA, "cudaGetSymbolAddress of the transport scratch failed");
        }
        ctx->noalloc_scratch = p;
    }
    const char* err = "";
    const int rc = nbx::run_transport_noalloc(ctx->phys, ctx->sms * ctx->bpsm, ctx->block, ctx->variant, ctx->stream,
                                              ctx->noalloc_scratch, d_particles, d_tags, n, uid_base, d_se_count,
                                              d_bse_count, n_tags, counts, &err);
    if (rc != 0) return fail(ctx, rc, err);
    return NBX_OK;
}

}  // extern "C"
