// Streaming C++ caller of the nbx C ABI (include/nbx.h): the primaries of a
// .pri file go to the device in batches, and each batch's host-to-device
// copy overlaps the run of the one before it.  Page-locked host buffers
// (nbx_host_alloc) make nbx_stage's copy asynchronous; nbx_push_staged
// queues the staged batch once the run is done.  The i-th primary of the
// file takes random-stream index i (nbx_set_uid_base), so the totals do not
// depend on the batch size.  Build from the repository root:
//   g++ -std=c++17 -Iinclude examples/nbx_stream.cpp -Lnebula_b200 -lnbx -Wl,-rpath,nebula_b200 -o nbx_stream
// Usage: nbx_stream <geometry.tri> <primaries.pri> <material.mat> [per_batch]
// It prints the SE (< 50 eV) and BSE detections per batch and in total; it
// exits with status 1, without crashing, when an input is missing or no GPU
// is present.
#include <algorithm>
#include <cstdio>
#include <cstdlib>

#include "nbx.h"

namespace {

// Batch [first, first + n) of the file's records as particles; tags are
// batch-relative.
void fill(const nbx_record* pri, uint64_t first, uint64_t n, nbx_particle* p, uint32_t* tags) {
    for (uint64_t i = 0; i < n; ++i) {
        const nbx_record& r = pri[first + i];
        p[i] = nbx_particle{{r.pos[0], r.pos[1], r.pos[2]}, {r.dir[0], r.dir[1], r.dir[2]}, r.E};
        tags[i] = uint32_t(i);
    }
}

int fail(nbx_ctx* ctx, const char* what) {
    std::fprintf(stderr, "%s: %s\n", what, nbx_last_error(ctx));
    return 1;
}

}  // namespace

int main(int argc, char** argv) {
    if (argc < 4) {
        std::fprintf(stderr, "usage: %s <geometry.tri> <primaries.pri> <material.mat> [per_batch]\n", argv[0]);
        return 1;
    }
    const uint64_t per_batch = argc > 4 ? std::strtoull(argv[4], nullptr, 10) : 100000;
    if (per_batch == 0) return 1;
    nbx_triangle* tris;
    uint64_t nt;
    nbx_octree* oct;
    nbx_record* pri;
    uint64_t n_pri;
    nbx_material* mat;
    if (nbx_load_tri(argv[1], &tris, &nt) || nbx_octree_build(tris, nt, &oct)) return fail(nullptr, "geometry");
    if (nbx_load_pri(argv[2], &pri, &n_pri) || n_pri == 0) return fail(nullptr, "primaries");
    if (nbx_material_load(argv[3], &mat)) return fail(nullptr, "material");
    nbx_config cfg;
    nbx_config_default(&cfg);
    cfg.record_detected = 1;
    nbx_ctx* ctx;
    if (nbx_create(&ctx, &cfg)) return fail(nullptr, "no CUDA device");
    if (nbx_set_geometry(ctx, oct) || nbx_add_material(ctx, mat)) return fail(ctx, "setup");

    // two page-locked batch buffers (one running, one in flight) and one for
    // the detected records
    const uint64_t cap = std::min(per_batch, n_pri);
    void* mem[5] = {};
    for (int k = 0; k < 4; ++k)
        if (nbx_host_alloc(cap * (k % 2 ? sizeof(uint32_t) : sizeof(nbx_particle)), &mem[k]))
            return fail(nullptr, "page-locked buffers");
    if (nbx_host_alloc(cap * sizeof(nbx_detected), &mem[4])) return fail(nullptr, "page-locked buffers");
    nbx_particle* part[2] = {static_cast<nbx_particle*>(mem[0]), static_cast<nbx_particle*>(mem[2])};
    uint32_t* tags[2] = {static_cast<uint32_t*>(mem[1]), static_cast<uint32_t*>(mem[3])};
    nbx_detected* det = static_cast<nbx_detected*>(mem[4]);

    uint64_t accepted = 0, se = 0, bse = 0, batch = 0;
    uint64_t n0 = std::min(cap, n_pri);
    fill(pri, 0, n0, part[0], tags[0]);
    if (nbx_set_uid_base(ctx, 0) || nbx_stage(ctx, part[0], tags[0], n0) || nbx_push_staged(ctx, &accepted))
        return fail(ctx, "first batch");
    for (uint64_t first = 0; first < n_pri; first += cap, ++batch) {
        const uint64_t next_first = first + cap;
        const uint64_t next_n = next_first < n_pri ? std::min(cap, n_pri - next_first) : 0;
        const int nb = int((batch + 1) & 1);
        if (next_n) {
            // the next batch's copy starts now and overlaps this batch's run
            fill(pri, next_first, next_n, part[nb], tags[nb]);
            if (nbx_stage(ctx, part[nb], tags[nb], next_n)) return fail(ctx, "stage");
        }
        if (nbx_run(ctx)) return fail(ctx, "run");
        uint64_t got = 0, batch_se = 0, batch_bse = 0;
        while (true) {
            if (nbx_flush_detected(ctx, det, cap, &got)) return fail(ctx, "flush");
            if (got == 0) break;
            for (uint64_t i = 0; i < got; ++i) (det[i].E < 50.0f ? batch_se : batch_bse) += 1;
        }
        std::printf("batch %llu: %llu SE, %llu BSE\n", (unsigned long long)batch, (unsigned long long)batch_se,
                    (unsigned long long)batch_bse);
        se += batch_se;
        bse += batch_bse;
        if (next_n && (nbx_set_uid_base(ctx, next_first) || nbx_push_staged(ctx, &accepted)))
            return fail(ctx, "push staged");
    }
    std::printf("total: %llu primaries, %llu SE, %llu BSE\n", (unsigned long long)n_pri, (unsigned long long)se,
                (unsigned long long)bse);
    nbx_destroy(ctx);
    for (void* m : mem) nbx_host_free(m);
    nbx_material_free(mat);
    nbx_free(pri);
    nbx_octree_free(oct);
    nbx_free(tris);
    return 0;
}
