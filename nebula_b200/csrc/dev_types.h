// Plain data shared by the host runtime and the transport kernels.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace nbx {
namespace dev {

constexpr float kEps = 10.0f * 1.1920928955078125e-07f;   // config/data_types.h:55
constexpr float kPi = 3.1415926535897932f;                 // config/config.h:32
constexpr int kNop = -128, kTerminator = -127, kDetector = -126, kDetectorLT50 = -125, kDetectorGE50 = -124,
              kVacuum = -123, kMirror = -122;               // core/cpu_material_manager.h:82-91
constexpr int kMaxMaterials = 16;

enum : int { kAlive = 0, kTerminated = 1, kDetected = 2 };
enum : int { kEvNone = 0, kEvInelastic = 1, kEvElastic = 2, kEvBoundary = 3 };

struct Table1D {
    const float* data;
    int n;
    float x_min, x_step;
};
struct Table2D {
    const float* data;
    int w, h;
    float x_min, x_step, y_min, y_step;
};
struct Table3D {
    const float* data;
    int w, h, d;
    float x_min, x_step, y_min, y_step, z_min, z_step;
};
// in_imfp / in_icdf hold the chosen inelastic model's log-IMFP and
// log-energy-loss ICDF (Kieft: omega', full Penn: omega); ion is Kieft's
// rebuilt 2-D ionisation table, q and ion3 the full Penn 3-D tables.
struct Material {
    float barrier;
    float phonon_loss, recoil_const;
    float fermi, band_gap;
    Table1D el_imfp, in_imfp;
    // The two log-IMFP tables interleaved per interval, (in[i], in[i+1],
    // el[i], el[i+1]), when both share one energy axis (else null): a step's
    // two free-path lookups then take one index and one 16-byte gather.
    const float4* imfp_pair;
    Table2D el_icdf, in_icdf, ion;
    Table3D q, ion3;
};
// Triangles as three float4: (r0, mat_in bits), (e1, mat_out bits), (e2, 0).
struct Geometry {
    const int32_t* octree;
    const float4* tri;        // per triangle: (r0, mat_in), (e1, mat_out), (e2, 0)
    const float4* tri_face;   // per triangle: (e1 x e2, (mat_out << 16) | (mat_in & 0xFFFF))
    float cx, cy, cz, hx, hy, hz;
    float max_extent;
    int n_tri;
};
struct Physics {
    Geometry geo;
    Material mat[kMaxMaterials];
    int n_mat;
    uint32_t seed;
    float min_energy, max_energy;
    int penn;   // inelastic model: 0 Kieft & Bosch, 1 full Penn
};

struct Electron {
    float px, py, pz;
    float dx, dy, dz;
    float E;
    int mat;
    int last_tri;
    uint32_t tag;
    uint64_t uid;
    uint32_t step;
};

}  // namespace dev
}  // namespace nbx
