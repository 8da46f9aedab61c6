// Minimal C++ caller of the nbx C ABI (include/nbx.h): loads a .tri geometry
// and a .mat material, simulates 1000 primaries at 1 keV and prints how many
// detected electrons it flushed.  Build from the repository root:
//   g++ -std=c++17 -Iinclude examples/nbx_caller.cpp -Lnebula_b200 -lnbx -Wl,-rpath,nebula_b200 -o nbx_caller
// Run it in a directory holding g.tri and si.mat.  It exits with status 1,
// without crashing, when an input is missing or no GPU is present.
#include <cstdio>
#include <vector>

#include "nbx.h"

int main() {
    nbx_triangle* tris;
    uint64_t nt;
    nbx_octree* oct;
    nbx_material* si;
    if (nbx_load_tri("g.tri", &tris, &nt) || nbx_octree_build(tris, nt, &oct) || nbx_material_load("si.mat", &si))
        return 1;
    nbx_config cfg;
    nbx_config_default(&cfg);
    cfg.record_detected = 1;
    nbx_ctx* ctx;
    if (nbx_create(&ctx, &cfg) || nbx_set_geometry(ctx, oct) || nbx_add_material(ctx, si)) return 1;

    // 1000 primaries at 1 keV straight down onto the centre; tag = index
    std::vector<nbx_particle> p(1000, nbx_particle{{0.0f, 0.0f, 10.0f}, {0.0f, 0.0f, -1.0f}, 1000.0f});
    std::vector<uint32_t> tags(p.size());
    for (uint32_t i = 0; i < tags.size(); ++i) tags[i] = i;
    uint64_t accepted;
    if (nbx_push(ctx, p.data(), tags.data(), p.size(), &accepted) || nbx_run(ctx)) {
        std::fprintf(stderr, "%s\n", nbx_last_error(ctx));
        return 1;
    }
    std::vector<nbx_detected> out(4096);
    uint64_t got;
    while (nbx_flush_detected(ctx, out.data(), out.size(), &got) == NBX_OK && got)
        std::printf("%llu detected\n", (unsigned long long)got);
    nbx_destroy(ctx);
    nbx_material_free(si);
    nbx_octree_free(oct);
    nbx_free(tris);
    return 0;
}
