// Launch interface between the host runtime (nbx_api.cpp) and the CUDA
// kernels (transport.cu).  Host-compilable; no device code here.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "dev_types.h"
#include "features.cuh"

namespace nbx {

// Structure-of-arrays electron queue: a = (pos, E), b = (dir, material bits),
// c = (tag, uid low, uid high, last triangle).  New electrons start at step 0.
struct Queue {
    float4* a;
    float4* b;
    uint4* c;
};

enum Counter : int {
    kCntSteps = 0,
    kCntElastic,
    kCntInelastic,
    kCntBoundary,
    kCntSecondaries,
    kCntDetected,
    kCntDetectedSE,
    kCntDetectedBSE,
    kCntTerminated,
    kCntRecordsDropped,
    kCntOverflow,
    kCntPopped,
    kCntInferences,
    kCntRouletteKilled,
    kCntSplit,
    kCntSamples,
    kCntDeposits,
    kCntDepositsDropped,
    kNumCounters
};

struct TransportArgs {
    Queue in;
    Queue out;
    const uint32_t* n_in;       // number of entries pushed to `in` (may exceed in_capacity)
    uint32_t in_capacity;
    uint32_t* head;             // pop cursor into `in`
    // Per-SM pop cursors (nullptr: every block pops from `head`).  The queue
    // is cut into n_ranges contiguous ranges, range r = [n_in * r / n_ranges,
    // n_in * (r + 1) / n_ranges).  The blocks on SM s pop from range
    // s % n_ranges and, once it is handed out, from ranges s + 1, s + 2, ...
    // in turn, so an SM's threads work on neighbouring entries of the queue
    // (for a raster scan, neighbouring pixels) and share its L1.
    uint32_t* range_cursor;
    uint32_t n_ranges;
    uint32_t* out_tail;         // push cursor into `out`
    uint32_t out_capacity;
    uint32_t* se_count;         // per-tag detections below 50 eV
    uint32_t* bse_count;        // per-tag detections at or above 50 eV
    uint64_t n_tags;
    unsigned long long* counters;
    float4* rec;                // detected records in nbx_detected's layout, two float4 each:
                                //   (pos, dir.x), (dir.y, dir.z, E, tag bits)
    uint32_t* rec_count;
    uint32_t rec_capacity;
    unsigned long long* hist;   // detected-energy histogram
    int n_bins;
    float inv_bin_width;
    // sample mode: one (features, label, cost) record per sampled newborn electron
    float* sample_feat;         // [capacity][6]: features at birth
    float* sample_label;        // [capacity]: sub-cascade produced a detected SE
    float* sample_cost;         // [capacity]: steps of the sub-cascade (nullptr: not kept)
    uint32_t* sample_count;
    uint32_t sample_capacity;
    // learned mode: every newborn secondary is scored by the network at birth
    // (mlp_params); importance p < rr_threshold: Russian roulette with
    // survival p / rr_threshold rounded to a power of two, at least
    // 2^-max_roulette_exp; p > split_threshold: split in two
    const float* mlp_params;
    float* se_w;                // per-tag weighted detections below / at or above 50 eV
    float* bse_w;
    float rr_threshold;
    float split_threshold;
    int max_roulette_exp;
    // learned mode, cost-aware survival (cost_bins > 0): a newborn of weight
    // 2^wexp, importance p and mean sub-cascade cost c survives with
    // q = 2^wexp sqrt(p * value_per_cost / c); c = cost_table[mat * cost_bins
    // + bin of log E over [cost_log_e_min, cost_log_e_min + cost_bins /
    // cost_inv_width)]
    // learned mode, importance table (imp_table != nullptr, kModeWeighted):
    // the network's escape probability tabulated at the centres of a grid over
    // its inputs, imp_table[((mat * imp_ne + e) * imp_nd + d) * imp_nc + c]
    // for the scaled log energy f0 in [0, 1) (imp_ne bins), the scaled
    // distance f1 in [0, 1] (imp_nd bins, the last one closed) and the cosine
    // f2 in [-1, 1] (imp_nc bins); features outside are clamped
    const float* imp_table;
    int imp_ne, imp_nd, imp_nc, imp_materials;
    const float* cost_table;
    int cost_bins;
    int cost_materials;
    float cost_log_e_min;
    float cost_inv_width;
    float value_per_cost;
    // learned mode, fixed rule at birth instead of the network: a secondary
    // born with energy below birth_max_energy and at least birth_min_distance
    // from the nearest surface (the surface map's distance; outside the map
    // counts as far) survives with probability birth_survival rounded to a
    // power of two and then carries its parent's weight / survival.
    // birth_survival outside (0, 1): off.
    float birth_min_distance;
    float birth_max_energy;
    float birth_survival;
    dev::SurfaceMap smap;
    // deposit mode: one record per scattering event that changed the energy
    // (drivers/cpu/energydeposit_cpu_driver.h:74-96), kDepositWords floats
    // each: position after the event, energy before, energy lost, tag bits
    float* dep;
    unsigned long long* dep_cursor;   // records handed out (chunks of kDepositChunk)
    unsigned long long dep_capacity;  // records the buffer holds
    // parked-ancestor stacks, 3 * stack_depth float4 per launched thread
    // (nullptr: a local-memory array of kLocalStack entries)
    float4* stack_mem;
    int stack_depth;            // 1 .. kMaxStack: parked ancestors per thread in stack_mem
    // per-pixel exit spectra (nullptr: off): pix_spec[pixel * pix_bins + bin]
    // counts (weights in learned mode) of detections, pixel = pixel_of_tag[tag]
    float* pix_spec;
    const uint32_t* pixel_of_tag;   // n_map entries
    uint64_t n_map;
    uint64_t n_pixels;
    int pix_bins;
    float pix_inv_width;
};

// Deposit records: x, y, z, E_before, E_before - E_after, tag; unused slots of
// a thread's last chunk carry tag kDepositEmpty.
constexpr int kDepositWords = 6;
constexpr uint32_t kDepositChunk = 32;
constexpr uint32_t kDepositEmpty = 0xFFFFFFFFu;

// kModeLearned: weighted transport, the network evaluated on the tensor
// cores for every newborn (warp-synchronous); kModeWeighted: weighted
// transport whose birth decisions come from the network's importance table
// or the fixed rule (no warp-synchronous step).
enum : int { kModePlain = 0, kModeSample = 1, kModeLearned = 2, kModeDeposit = 3, kModeWeighted = 4 };

// Per-thread stack of parked ancestors (depth-first cascades): the depth of
// the local-memory array used without a stack buffer, and the largest depth
// a stack buffer may be given.
constexpr int kLocalStack = 16;
constexpr int kMaxStack = 64;

// variant: resident blocks per SM the kernel was compiled for (2, 3 or 4);
// mode: kModePlain, kModeSample or kModeLearned.
cudaError_t launch_transport(const dev::Physics& P, const TransportArgs& a, int grid, int block, int variant,
                             cudaStream_t s, int mode = kModePlain);
int transport_max_blocks_per_sm(int block, int variant, int mode = kModePlain);
// Per-triangle face records (normal e1 x e2 and packed materials) for
// Geometry::tri_face; materials must fit in 16 bits.
cudaError_t launch_triangle_faces(const float4* tri, float4* face, int n, cudaStream_t s);
// Surface map over [lo, lo + n * cell): each cell searches the candidate
// list of its brick of `brick`^3 cells (brick_tris[brick_start[b] ..
// brick_start[b + 1]), bricks x-fastest over nbx x nby x ...) for the nearest
// triangle and stores (unit vector from its nearest point to the cell
// centre, distance); cells farther than d_max from all candidates get
// distance -1.
cudaError_t launch_build_surface_map(const float4* tri, const uint32_t* brick_start, const int32_t* brick_tris,
                                     int nbx, int nby, int brick, float4* map, float lox, float loy, float loz,
                                     float cell, int nx, int ny, int nz, float d_max, cudaStream_t s);
// Features of n electrons (56-byte nbx_electron records) for testing.
cudaError_t launch_features(const dev::SurfaceMap& S, const void* electrons, uint64_t n, float* out, cudaStream_t s);

cudaError_t launch_ray_query(const dev::Geometry& g, const float* pos, const float* dir, const float* dist,
                             const int32_t* ignore_tri, const int32_t* ignore_mat, uint64_t n, float* out_dist,
                             int32_t* out_tri, cudaStream_t s);
cudaError_t launch_table_query(const dev::Material& m, int table, const float* x, const float* y, uint64_t n,
                               float* out, cudaStream_t s);
// table 0: full Penn q ICDF (table_3D::get), 1: full Penn ionisation (get_rounddown)
cudaError_t launch_table3_query(const dev::Material& m, int table, const float* x, const float* y, const float* z,
                                uint64_t n, float* out, cudaStream_t s);
cudaError_t launch_philox(const uint32_t* ctr, const uint32_t* key, uint64_t n, uint32_t* out, cudaStream_t s);
// electrons: 56-byte nbx_electron records
cudaError_t launch_step_query(const dev::Physics& P, void* electrons, uint64_t n, int32_t* status, int32_t* event,
                              void* secondaries, int32_t* has_se, cudaStream_t s);
// se_w / bse_w: per-tag weights (learned mode) or nullptr for the counts.
cudaError_t launch_pixel_yields(const uint32_t* se, const uint32_t* bse, const float* se_w, const float* bse_w,
                                const uint32_t* pixel_of_tag, uint64_t n_tags, uint64_t n_pixels, double* out,
                                cudaStream_t s);
// Allocation-free transport on the file-scope scratch of transport.cu
// (see nbx_run_noalloc).  noalloc_scratch_address gives the scratch array's
// device address on the current device; run_transport_noalloc takes it as
// `scratch` and returns 0 or an NBX_ERR_* code with *err set.
constexpr uint32_t kNoAllocMaxPrimaries = 65536;
cudaError_t noalloc_scratch_address(void** out);
int run_transport_noalloc(const dev::Physics& P, int grid, int block, int variant, cudaStream_t s, void* scratch,
                          const float* d_particles,
                          const uint32_t* d_tags, uint32_t n, uint64_t uid_base, uint32_t* d_se, uint32_t* d_bse,
                          uint64_t n_tags, uint64_t counts[4], const char** err);
cudaError_t launch_fill_queue(Queue q, const float* particles, const uint32_t* tags, uint64_t uid_base,
                              uint64_t n, uint64_t offset, cudaStream_t s);
// *p = v on the device, in stream order.
cudaError_t launch_set_word(uint32_t* p, uint32_t v, cudaStream_t s);
// The largest of n tags into *out (which the caller zeroes first).
cudaError_t launch_max_tag(const uint32_t* tags, uint64_t n, uint32_t* out, cudaStream_t s);

}  // namespace nbx
