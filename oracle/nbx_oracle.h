/* CPU restatement of Nebula's electron-transport hot path, in plain C.
 *
 * TEST INFRASTRUCTURE ONLY: this is the checker the CUDA kernels are compared
 * against (by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg).  The product never links, loads or calls it.
 *
 * Every function follows a reference file:line (paths relative to the Nebula
 * source tree).  Float operations are written in the reference's order and
 * grouping; compiled without FMA contraction they reproduce the reference's
 * single-precision arithmetic.  Parity is pinned by tests against the
 * reference's own code compiled from its sources (oracle/_ref/libnbref.so):
 * ray queries and table lookups bit-exact, whole runs statistically.
 *
 * Random numbers: Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random
 * numbers: as easy as 1, 2, 3", SC'11), keyed by the run seed, with counter
 * (step, block, uid_lo, uid_hi) so every electron has its own reproducible
 * stream independent of scheduling (the reference draws from one mt19937 per
 * thread instead, source/common/util/random.inl:12-24).
 */
#ifndef NBX_ORACLE_H
#define NBX_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    const int32_t* octree_data;
    const float* tri;        /* n_tri x 9: r0, e1, e2 */
    const int32_t* tri_mat;  /* n_tri x 2: material_in, material_out */
    float center[3];
    float half[3];
    float max_extent;
} nbo_geometry;

typedef struct {
    int n;
    float x_min, x_step;
    const float* data;
} nbo_table1d;

typedef struct {
    int w, h;
    float x_min, x_step, y_min, y_step;
    const float* data; /* data[x * h + y] */
} nbo_table2d;

typedef struct {
    int w, h, d;
    float x_min, x_step, y_min, y_step, z_min, z_step;
    const float* data; /* data[(x * h + y) * d + z] */
} nbo_table3d;

/* in_imfp / in_icdf: the inelastic model's log-IMFP and log-energy-loss ICDF
 * (Kieft omega', full Penn omega); ion: Kieft's 2-D ionisation table;
 * q / ion3: full Penn's 3-D tables. */
typedef struct {
    float barrier;
    nbo_table1d el_imfp;
    nbo_table2d el_icdf;
    float phonon_loss, recoil_const;
    nbo_table1d in_imfp;
    nbo_table2d in_icdf;
    nbo_table2d ion;
    float fermi, band_gap;
    nbo_table3d q, ion3;
} nbo_material;

typedef struct {
    float pos[3], dir[3], E;
    int32_t mat, last_tri;
    uint32_t tag;
    uint64_t uid;
    uint32_t step;
} nbo_electron;

enum { NBO_ALIVE = 0, NBO_TERMINATED = 1, NBO_DETECTED = 2 };
enum { NBO_EV_NONE = 0, NBO_EV_INELASTIC = 1, NBO_EV_ELASTIC = 2, NBO_EV_BOUNDARY = 3 };

/* Random numbers */
void nbo_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
float nbo_u01(uint32_t x);
uint64_t nbo_secondary_uid(uint64_t parent_uid, uint32_t parent_step);

/* Geometry */
float nbo_triangle_intersect(const float tri[9], const float pos[3], const float dir[3]);
int nbo_in_domain(const nbo_geometry* g, const float pos[3]);
void nbo_propagate(const nbo_geometry* g, const float pos[3], const float dir[3], float distance,
                   int32_t ignore_tri, int32_t ignore_mat, float* out_dist, int32_t* out_tri);
void nbo_propagate_batch(const nbo_geometry* g, const float* pos, const float* dir, const float* dist,
                         const int32_t* ignore_tri, const int32_t* ignore_mat, int64_t n, float* out_dist,
                         int32_t* out_tri);

/* Octree words / triangle records read by propagate since the last reset. */
void nbo_geom_counters(uint64_t out[2]);
void nbo_geom_counters_reset(void);

/* Tables */
float nbo_table1d_get(const nbo_table1d* t, float x);
float nbo_table2d_get(const nbo_table2d* t, float x, float y);
float nbo_table2d_get_rounddown(const nbo_table2d* t, float x, float y);
float nbo_table3d_get(const nbo_table3d* t, float x, float y, float z);
float nbo_table3d_get_rounddown(const nbo_table3d* t, float x, float y, float z);

/* Events, with their uniforms given explicitly. */
void nbo_elastic(const nbo_material* m, nbo_electron* e, float u_cos, float u_phi);
/* Returns 1 and fills *se if a secondary was created. */
int nbo_inelastic(const nbo_material* m, nbo_electron* e, const float u[6], nbo_electron* se);
/* Returns NBO_ALIVE / NBO_TERMINATED / NBO_DETECTED. */
int nbo_boundary(const nbo_geometry* g, const nbo_material* mats, nbo_electron* e, float u);

typedef struct {
    uint32_t seed;
    float min_energy, max_energy;
    int penn; /* inelastic model: 0 Kieft & Bosch, 1 full Penn */
} nbo_params;

/* full_penn::execute (physics/full_penn.h:63-289) after the log-omega ICDF
 * lookup; r1 = Philox block 1 of this step, further uniforms from blocks 3
 * and 4, 5, ... of the electron's stream (same slots as the GPU). */
int nbo_penn_inelastic(const nbo_material* m, const nbo_params* p, nbo_electron* e, float log_omega, float u_phi,
                       const uint32_t r1[4], nbo_electron* se);

/* One pass of init -> intersect -> scatter for one electron
 * (source/drivers/cpu/cpu_driver.inl:73-161).  Returns the status; *event
 * receives the event type executed; *has_se is set when *se was created. */
int nbo_step(const nbo_geometry* g, const nbo_material* mats, const nbo_params* p, nbo_electron* e, int* event,
             nbo_electron* se, int* has_se);

typedef struct {
    uint64_t n_primaries, n_detected, n_dropped_records;
    uint64_t n_elastic, n_inelastic, n_boundary, n_secondaries, n_steps;
} nbo_counts;

/* Simulate primaries (7 floats each: pos, dir, E) with their tags/uids to the
 * end, cascade by cascade.  Detected electrons are written as 36-byte
 * records {pos, dir, E, tag, 0} to `records` (capacity in records).
 * se_count/bse_count[i] (may be null) count detections of primary i below /
 * at or above 50 eV. */
int nbo_run(const nbo_geometry* g, const nbo_material* mats, const nbo_params* p, const float* primaries,
            const uint32_t* tags, uint64_t uid_base, uint64_t n, void* records, uint64_t capacity,
            uint32_t* se_count, uint32_t* bse_count, nbo_counts* counts);

#ifdef __cplusplus
}
#endif

#endif
