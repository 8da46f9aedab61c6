/* nbx: B200-native electron transport for Nebula-format SEM simulations.
 *
 * C ABI of the drop-in hot path.  Plain pointers and sizes only; no C++ types
 * or exceptions cross it.  Every call returns NBX_OK (0) or a negative
 * NBX_ERR_* code; nbx_last_error() gives a message for the last failing call
 * on a context, and nbx_last_error(NULL) the message of the calling thread's
 * last failing call that takes no context (material loading, octree build).  One context per GPU, driven by one host thread (the
 * reference's worker_thread model, source/gpu_main.cu:77-218); a context is
 * not re-entrant.
 *
 * Reference interfaces each group of entry points replaces (paths relative
 * to the Nebula source tree):
 *   nbx_load_tri          nbl::load_tri_file            io/load_tri_file.cpp:8-60
 *   nbx_load_pri          nbl::load_pri_file            io/load_pri_file.cpp:134-246
 *   nbx_octree_build      octree_builder::linearized_octree(octree_root(tris))
 *                                                       geometry/octree/octree_builder.cpp:171-352
 *   nbx_material_load     material<...>::create(hdf5_file) with kieft_elastic /
 *                         kieft_inelastic / full_penn loaders
 *                                                       core/material.inl:25-34,
 *                                                       physics/kieft/elastic.h:120-166,
 *                                                       physics/kieft/inelastic.h:212-327,
 *                                                       physics/full_penn.h:296-392
 *   nbx_create            gpu_driver constructor       drivers/gpu/gpu_driver.inl:51-89
 *   nbx_set_geometry      octree<true>::create         geometry/octree.inl:280-313
 *   nbx_add_material      gpu_material_manager::create core/gpu_material_manager.inl:5-26
 *   nbx_push              gpu_driver::push             drivers/gpu/gpu_driver.h:58-80
 *   nbx_run               the frame loop of do_iteration() calls
 *                                                       gpu_main.cu:183-213, gpu_driver.inl:312-317
 *   nbx_get_running_count gpu_driver::get_running_count drivers/gpu/gpu_driver.h:100-110
 *   nbx_flush_detected    gpu_driver::flush_detected / flush_buffered
 *                                                       drivers/gpu/gpu_driver.inl:259-306
 *   nbx_flush_deposits    energydeposit_cpu_driver's deposit callback
 *                                                       drivers/cpu/energydeposit_cpu_driver.h:74-96
 *   nbx_ray_query         octree::propagate            geometry/octree.inl:33-192
 *   nbx_table_query       table_1D::get, table_2D::get / get_rounddown
 *                                                       common/util/table_1D.inl:66-80,
 *                                                       common/util/table_2D.inl:74-104
 *   nbx_table3_query      table_3D::get / get_rounddown common/util/table_3D.inl:79-122
 */
#ifndef NBX_H
#define NBX_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NBX_VERSION_MAJOR 1
#define NBX_VERSION_MINOR 0
#define NBX_VERSION_PATCH 2

#define NBX_OK 0
#define NBX_ERR_ARG (-1)      /* invalid argument */
#define NBX_ERR_OOM (-2)      /* device or host allocation failed / over the HBM budget */
#define NBX_ERR_CUDA (-3)     /* CUDA runtime error */
#define NBX_ERR_TIMEOUT (-4)  /* a bounded device wait gave up */
#define NBX_ERR_FORMAT (-5)   /* malformed .tri / .pri / .mat input */
#define NBX_ERR_STATE (-6)    /* call out of order (e.g. run before set_geometry) */
#define NBX_ERR_NODEV (-7)    /* no CUDA device / extension unavailable */
#define NBX_ERR_CAPACITY (-8) /* a device queue overflowed */

/* Special material indices (core/cpu_material_manager.h:82-91). */
#define NBX_NOP (-128)
#define NBX_TERMINATOR (-127)
#define NBX_DETECTOR (-126)
#define NBX_DETECTOR_LT50 (-125)
#define NBX_DETECTOR_GE50 (-124)
#define NBX_VACUUM (-123)
#define NBX_MIRROR (-122)

#define NBX_MAX_MATERIALS 16

typedef struct nbx_ctx nbx_ctx;

/* core/particle.h:5-10: position (nm), unnormalised direction, kinetic energy (eV). */
typedef struct {
    float pos[3];
    float dir[3];
    float E;
} nbx_particle;

/* The 36-byte .pri / detected-electron record (io/load_pri_file.cpp:134-246,
 * cpu_mt_main.cpp:183-190). */
typedef struct {
    float pos[3];
    float dir[3];
    float E;
    int32_t px, py;
} nbx_record;

/* core/triangle.h: r0, e1 = r1 - r0, e2 = r2 - r0, material_in, material_out. */
typedef struct {
    float r0[3];
    float e1[3];
    float e2[3];
    int32_t mat_in, mat_out;
} nbx_triangle;

/* A detected electron and the tag of the primary that started its cascade. */
typedef struct {
    float pos[3];
    float dir[3];
    float E;
    uint32_t tag;
} nbx_detected;

/* Linearized octree (geometry/octree/octree_builder.h:209-248). */
typedef struct {
    int32_t* octree_data;
    uint64_t n_octree;
    nbx_triangle* triangles;
    uint64_t n_triangles;
    float center[3];
    float halfsize[3];
    uint64_t duplicates_dropped;
    int32_t max_depth;
} nbx_octree;

/* util::table_1D / table_2D: x_index = (x - x_min) * x_step; 2D data is
 * row-major data[x * height + y]. */
typedef struct {
    int32_t n;
    float x_min, x_step;
    const float* data;
} nbx_table1d;

typedef struct {
    int32_t width, height;
    float x_min, x_step, y_min, y_step;
    const float* data;
} nbx_table2d;

/* util::table_3D (common/util/table_3D.inl:66-122): data[(x * height + y) *
 * depth + z]. */
typedef struct {
    int32_t width, height, depth;
    float x_min, x_step, y_min, y_step, z_min, z_step;
    const float* data;
} nbx_table3d;

/* Material tables already transformed as the reference loaders do: Kieft
 * elastic (log IMFP, clamped cos-theta ICDF) and the Kieft inelastic model
 * (log IMFP, log omega' ICDF, rebuilt ionisation table;
 * physics/kieft/inelastic.h:212-327) and/or the full Penn model (log IMFP,
 * log omega ICDF, q ICDF in eV^1/2, 3-D ionisation table with -1 for "no
 * inner shell"; physics/full_penn.h:296-392). */
typedef struct {
    float barrier;
    nbx_table1d elastic_imfp;
    nbx_table2d elastic_icdf;
    float phonon_loss;
    float recoil_const;
    nbx_table1d inelastic_imfp;
    nbx_table2d inelastic_icdf;
    nbx_table2d ionisation;
    float fermi;
    float band_gap;
    float max_energy; /* min over mechanisms of exp(IMFP axis maximum), Kieft model (Penn if no Kieft tables) */
    char name[64];
    int32_t has_kieft_inelastic;
    int32_t has_full_penn;
    nbx_table1d penn_imfp;
    nbx_table2d penn_omega_icdf;
    nbx_table3d penn_q_icdf;
    nbx_table3d penn_ionisation;
    float penn_max_energy; /* as max_energy, full Penn model */
} nbx_material;

/* Inelastic model of a context (physics_config.h:21-33 selects it at compile
 * time in the reference; the stock build uses full Penn). */
#define NBX_INELASTIC_KIEFT 0
#define NBX_INELASTIC_FULL_PENN 1

typedef struct {
    int32_t device;            /* CUDA device ordinal */
    uint32_t seed;             /* random seed (gpu_main.cu --seed) */
    float energy_threshold;    /* lowest energy w.r.t. vacuum (--energy-threshold) */
    uint64_t capacity;         /* electrons per device queue; 0 = sized from free HBM */
    int32_t record_detected;   /* keep per-electron detected records */
    uint64_t record_capacity;  /* detected records held on the device; 0 = auto */
    int32_t block_size;        /* threads per block of the transport kernel; 0 = 256 */
    int32_t blocks_per_sm;     /* transport variant: 2, 3 or 4 resident 256-thread blocks per SM, or 7
                                  128-thread blocks (block_size capped at 128); 0 = 4 (64 registers) */
    int32_t inelastic_model;   /* NBX_INELASTIC_KIEFT (0, default) or NBX_INELASTIC_FULL_PENN */
    int32_t record_deposits;   /* keep energy-deposit records (plain mode; cpu_energydep.cpp) */
    uint64_t deposit_capacity; /* deposit records held on the device; 0 = 2^27 (3.2 GB) */
    int32_t shared_pop;        /* 0: the transport blocks on each SM pop the primaries of that SM's
                                  contiguous range of the queue first (neighbouring primaries share
                                  the SM's caches; push them in scan order); 1: one shared cursor */
} nbx_config;

/* One energy deposit (drivers/cpu/energydeposit_cpu_driver.h:74-96,
 * cpu_energydep.cpp:189-207): a scattering event (not a boundary crossing)
 * that changed the electron's energy; position after the event, energy
 * before it, energy lost, and the primary's tag. */
typedef struct {
    float pos[3];
    float E;
    float dE;
    uint32_t tag;
} nbx_deposit;

typedef struct {
    uint64_t primaries_pushed;
    uint64_t primaries_done;
    uint64_t steps;           /* init passes, including those that terminate */
    uint64_t events_elastic;
    uint64_t events_inelastic;
    uint64_t events_boundary;
    uint64_t secondaries;
    uint64_t detected;
    uint64_t detected_se;     /* E < 50 eV */
    uint64_t detected_bse;    /* E >= 50 eV */
    uint64_t terminated;
    uint64_t records_dropped;
    uint64_t generations;     /* kernel launches of the last nbx_run */
    uint64_t queue_overflow;
    uint64_t inferences;      /* warp-level network evaluations at birth (learned mode) */
    uint64_t roulette_killed; /* newborn secondaries dropped by Russian roulette (learned mode) */
    uint64_t splits;          /* newborn secondaries split in two (learned mode) */
    uint64_t samples;         /* training samples recorded (sample mode) */
    double last_run_ms;       /* device time of the last nbx_run (CUDA events) */
    double last_kernel_ms;    /* device time of its transport launches only */
    uint64_t deposits;        /* energy-deposit records written (record_deposits) */
    uint64_t deposits_dropped; /* deposits lost to a full deposit buffer */
} nbx_stats;

/* ---- host-side helpers (no GPU needed) ---------------------------------- */
int nbx_version(int* major, int* minor, int* patch);
const char* nbx_error_string(int code);
void nbx_free(void* p);
int nbx_load_tri(const char* path, nbx_triangle** out, uint64_t* n);
int nbx_load_pri(const char* path, nbx_record** out, uint64_t* n);
int nbx_octree_build(const nbx_triangle* tris, uint64_t n, nbx_octree** out);
void nbx_octree_free(nbx_octree* oct);
int nbx_material_load(const char* path, nbx_material** out);
void nbx_material_free(nbx_material* mat);
int nbx_device_count(int* n);

/* ---- device context ------------------------------------------------------ */
void nbx_config_default(nbx_config* cfg);
int nbx_create(nbx_ctx** ctx, const nbx_config* cfg);
void nbx_destroy(nbx_ctx* ctx);
const char* nbx_last_error(nbx_ctx* ctx);
int nbx_set_geometry(nbx_ctx* ctx, const nbx_octree* oct);
int nbx_add_material(nbx_ctx* ctx, const nbx_material* mat);
/* Per-primary tallies are kept for tags [0, n_tags). */
int nbx_set_tag_range(nbx_ctx* ctx, uint64_t n_tags);
/* Queue primaries (host buffers).  *accepted <= n is how many fit. */
int nbx_push(nbx_ctx* ctx, const nbx_particle* particles, const uint32_t* tags, uint64_t n, uint64_t* accepted);
/* Staged push (no counterpart in the reference, whose frame loop copies the
 * next frame's primaries from pinned buffers while a frame runs,
 * gpu_driver.inl:167-306): nbx_stage starts copying a batch (host arrays as
 * for nbx_push) to the device on the context's copy stream and returns at
 * once, so the copy can overlap a following nbx_run; nbx_push_staged then
 * queues it on the device (tags checked there) exactly as nbx_push would
 * have, with the random-stream index running on from the primaries pushed
 * before it.  The host arrays must stay unchanged until nbx_push_staged
 * returns; the copy overlaps only from page-locked host memory.  One batch
 * at a time: nbx_stage with a batch still staged returns NBX_ERR_STATE;
 * nbx_push_staged with nothing staged queues nothing (*accepted = 0). */
int nbx_stage(nbx_ctx* ctx, const nbx_particle* particles, const uint32_t* tags, uint64_t n);
int nbx_push_staged(nbx_ctx* ctx, uint64_t* accepted);
/* Page-locked host memory for nbx_stage's arrays (no counterpart in the
 * reference, which pins its frame buffers inside the driver): usable by
 * every context of the process.  NBX_ERR_OOM (and *out = NULL) when the
 * allocation fails; nbx_host_free(NULL) does nothing. */
int nbx_host_alloc(uint64_t bytes, void** out);
void nbx_host_free(void* p);
/* Random-stream index of the next pushed primary (default: running count of
 * pushed primaries).  Replicas on several GPUs set it to the global index of
 * their first primary so the combined result does not depend on sharding. */
int nbx_set_uid_base(nbx_ctx* ctx, uint64_t base);
/* Simulate every queued electron and all its secondaries to the end. */
int nbx_run(nbx_ctx* ctx);
int nbx_get_running_count(nbx_ctx* ctx, uint64_t* n);
int nbx_get_stats(nbx_ctx* ctx, nbx_stats* out);
/* Energy-deposit records of the runs since the last full flush, compacted,
 * in no particular order (replaces the deposit callback of
 * energydeposit_cpu_driver::simulate_to_end, drivers/cpu/
 * energydeposit_cpu_driver.h:74-96).  Copies up to `capacity` records into
 * `out`; call again until *n comes back 0.  A run while records are still
 * pending appends to them.  The context must be created with
 * record_deposits; runs whose records overflow deposit_capacity count the
 * lost ones in nbx_stats.deposits_dropped. */
int nbx_flush_deposits(nbx_ctx* ctx, nbx_deposit* out, uint64_t capacity, uint64_t* n);
/* Copy out (and remove) up to cap detected electrons, oldest first; call
 * again until *n comes back 0.  The device keeps them in this struct's
 * layout, so a call is one device-to-host copy straight into `out` (a DMA
 * when `out` is page-locked, nbx_host_alloc).  A run while records are
 * still pending appends to them. */
int nbx_flush_detected(nbx_ctx* ctx, nbx_detected* out, uint64_t cap, uint64_t* n);
/* Detections per primary tag below / at-or-above 50 eV. */
int nbx_get_tag_counts(nbx_ctx* ctx, uint64_t first_tag, uint64_t n, uint32_t* se, uint32_t* bse);
/* Per-pixel FP64 yields: pixel_of_tag maps tags to [0, n_pixels); out has
 * n_pixels x 5 doubles {primaries, sum_se, sum_se^2, sum_bse, sum_bse^2},
 * over per-primary counts (weighted counts when the context is in learned
 * mode, so sum_se^2 is the sum of squared weights per primary).
 * pixel_of_tag = NULL uses the map last given to nbx_set_pixel_map (n_tags
 * must not exceed its length). */
int nbx_pixel_yields(nbx_ctx* ctx, const uint32_t* pixel_of_tag, uint64_t n_tags, uint64_t n_pixels, double* out);
/* Keep a tag -> pixel map on the device for later nbx_pixel_yields calls
 * (a scan that repeats does not re-send it every time) and for the per-pixel
 * spectra. */
int nbx_set_pixel_map(nbx_ctx* ctx, const uint32_t* pixel_of_tag, uint64_t n_tags);
/* Per-pixel exit spectra, tallied on the device during runs (no reference
 * counterpart; the reference writes every detected electron and bins on the
 * host): n_bins bins of bin_width eV from 0 for each of n_pixels pixels,
 * through the map of nbx_set_pixel_map (detections of tags outside it, and
 * energies past the last bin, are not binned).  Counts in plain mode, weights
 * in learned mode.  n_pixels = 0 turns them off.  nbx_reset_tallies clears
 * them. */
int nbx_enable_pixel_spectra(nbx_ctx* ctx, uint64_t n_pixels, int32_t n_bins, float bin_width);
/* Copy out n_pixels x n_bins floats, pixel-major. */
int nbx_get_pixel_spectra(nbx_ctx* ctx, float* out);
/* Detected-energy histogram: n_bins bins of bin_width eV from 0. */
int nbx_get_spectrum(nbx_ctx* ctx, uint64_t* counts, uint32_t n_bins, float* bin_width);
int nbx_reset_tallies(nbx_ctx* ctx);

/* Launch and queue settings of the transport (no counterpart in the
 * reference, whose launch shape is fixed at 32-thread blocks over the whole
 * slot capacity, drivers/gpu/gpu_driver.inl:64, and whose frame and batch
 * sizes come from a prescan, gpu_main.cu:139-157). */
typedef struct {
    int32_t blocks_per_sm;   /* transport variant: 2, 3 or 4 resident 256-thread blocks per SM, or 7
                                resident 128-thread blocks */
    int32_t block_size;      /* threads per block (multiple of 32; at most 128 for variant 7) */
    int32_t stack_depth;     /* parked ancestors per thread (1..64, default 16): a secondary born deeper
                                in its cascade goes to the next generation's queue */
    int32_t chunk;           /* generation launches queued between two host reads (1..64, default 8) */
    uint64_t queue_capacity; /* out: entries of each overflow queue in the last run */
    double sample_ms;        /* out (nbx_autotune): the sample's device time with these settings */
} nbx_tuning;
int nbx_set_tuning(nbx_ctx* ctx, const nbx_tuning* tuning);
int nbx_get_tuning(nbx_ctx* ctx, nbx_tuning* tuning);
/* Autotuner: runs the given sample in the context's current mode -- twice
 * per setting on the same random streams, timing the second pass -- first
 * over every transport variant x block size (256, 128), then over the stack
 * depths 8 and 32 against the default 16, then over the chunk sizes 2 and 16
 * against 8, keeping the fastest at each stage; applies the result, reports
 * it in *out (may be NULL) and resets the tallies.  Random streams of later
 * pushes are unaffected.  There is no refill threshold to tune: a thread
 * takes its next electron from the queue the moment its current one ends. */
int nbx_autotune(nbx_ctx* ctx, const nbx_particle* particles, const uint32_t* tags, uint64_t n, nbx_tuning* out);

/* ---- escape-probability network (no counterpart in the reference) ------- */
/* MLP 6 -> 64 -> 64 -> 1 (SiLU, sigmoid), BF16 tensor-core kernels with FP32
 * accumulation, used only as the importance function of the weighted
 * roulette / splitting.  Parameters: NBX_MLP_PARAMS floats, row-major
 * [out][in] with inputs padded to 16 and the output to 8:
 * W1[64][16] b1[64] W2[64][64] b2[64] W3[8][64] b3[8] (padding forced to 0).
 * Features (6 per sample): log(E/eV) scaled, distance to the nearest surface
 * scaled, direction cosine toward that surface, material one-hot (3). */
#define NBX_MLP_PARAMS 5768

/* Transport modes.  PLAIN: analogue transport (the reference's method).
 * SAMPLE: plain transport that also records about one in sixteen newborn
 * electrons (secondaries at their birth, in a material): the network
 * features there, the label "this electron's sub-cascade produced a detected
 * electron below 50 eV" and the number of steps that sub-cascade took
 * (nbx_set_sample_capacity, nbx_get_samples).
 * LEARNED: plain transport of weighted electrons.  Every newborn secondary
 * is scored at its birth by the network (the warp's newborns together, on
 * the tensor cores): importance p = predicted escape probability.  With
 * p < rr_threshold it plays Russian roulette: it survives with probability
 * q = p / rr_threshold rounded to a power of two (q >= 2^-max_roulette_exp)
 * and then carries its parent's weight / q; a lost secondary's cascade is not
 * simulated.  With p > split_threshold it is split into two electrons of
 * half the weight that run on different random streams.  Weights are powers
 * of two, at most 2^12 and at least 2^-4.  The expected weighted tally
 * equals the analogue one (the method stays unbiased).  Weighted detections
 * go to nbx_get_tag_weights and nbx_pixel_yields; the per-tag counts and
 * detected records stay unweighted. */
#define NBX_MODE_PLAIN 0
#define NBX_MODE_SAMPLE 1
#define NBX_MODE_LEARNED 2
int nbx_set_mode(nbx_ctx* ctx, int32_t mode, float rr_threshold, float split_threshold, int32_t max_roulette_exp);
/* Learned mode, a fixed rule at birth instead of the network (off until
 * set): a secondary born with energy below max_energy (eV) at least
 * min_distance (nm) from the nearest surface of the surface map (outside the
 * map counts as far) is given the target weight 1 / survival, rounded to a
 * power of two 2^k with 1 <= k <= max_roulette_exp; lighter than that, it
 * plays Russian roulette up to it (survives with probability weight / 2^k,
 * then carries 2^k), so a lineage is rouletted once, not again at every
 * generation.  A dropped secondary's cascade is not simulated (counted in
 * nbx_stats.roulette_killed).  survival 0 or 1 turns it off. */
int nbx_set_birth_roulette(nbx_ctx* ctx, float min_distance, float max_energy, float survival);
/* Learned mode, cost-aware survival (off until set; n_bins = 0 turns it off
 * again): minimising the variance x cost of the tally, a newborn of weight
 * w, importance p and mean sub-cascade cost c survives with
 * q = w * sqrt(p * value_per_cost / c), rounded to a power of two (roulette
 * below 1 with q >= 2^-max_roulette_exp, a split in two from sqrt(2) up when
 * p > split_threshold; split_threshold >= 1 turns splitting off); this
 * replaces the rr_threshold window.  c is looked up in
 * mean_cost[material * n_bins + bin], bins uniform in log(E / eV) over
 * [log_e_min, log_e_max) (clamped at the ends); costs are in transport steps
 * (e.g. the mean of nbx_get_samples' costs per bin).  value_per_cost is the
 * steps per primary divided by the per-primary variance of the detected SE
 * count of an analogue run. */
int nbx_set_learned_cost(nbx_ctx* ctx, const float* mean_cost, int32_t n_materials, int32_t n_bins,
                         float log_e_min, float log_e_max, float value_per_cost);
/* Learned mode, importance table (off until set; any count 0 turns it off
 * again): instead of running the network for every newborn, the network is
 * evaluated once, on the tensor cores, at the centres of a grid over its
 * inputs -- n_energy bins of the scaled log energy, n_distance of the scaled
 * distance to the nearest surface, n_cosine of the cosine toward its normal,
 * for every material -- and a newborn's importance is its grid cell's value.
 * The birth decisions are then those of the network at the cell centre, and
 * the transport needs no warp-synchronous step.  The table is rebuilt
 * automatically when the parameters change (nbx_mlp_set_params,
 * nbx_mlp_train). */
int nbx_set_importance_table(nbx_ctx* ctx, int32_t n_energy, int32_t n_distance, int32_t n_cosine);
/* Surface map over the box [lo, hi) with the given cell size (nm): per cell
 * the distance from its centre to the nearest material surface and the unit
 * vector from that surface point to the centre; a point of the cell takes
 * the first-order distance from them.  Surfaces farther than d_max (nm) count
 * as "far".  Needed for the distance and cosine features. */
int nbx_build_surface_map(nbx_ctx* ctx, const float lo[3], const float hi[3], float cell, float d_max);
int nbx_set_sample_capacity(nbx_ctx* ctx, uint64_t capacity);
/* Copy out (and clear) the recorded samples: features n x 6, labels n and,
 * when costs is not NULL, the sub-cascade step counts n. */
int nbx_get_samples(nbx_ctx* ctx, float* features, float* labels, float* costs, uint64_t cap, uint64_t* n);
int nbx_get_tag_weights(nbx_ctx* ctx, uint64_t first_tag, uint64_t n, float* se_w, float* bse_w);
int nbx_mlp_set_params(nbx_ctx* ctx, const float* params);
int nbx_mlp_get_params(nbx_ctx* ctx, float* params);
/* Gradient of the mean binary cross-entropy over n samples at the current
 * parameters (no update). */
int nbx_mlp_grad(nbx_ctx* ctx, const float* features, const float* labels, uint64_t n, float* grad, float* loss);
/* Adam (beta 0.9/0.999, eps 1e-8) over shuffled mini-batches. */
int nbx_mlp_train(nbx_ctx* ctx, const float* features, const float* labels, uint64_t n, int32_t epochs,
                  int32_t batch, float lr, uint32_t seed, float* loss_per_epoch);
int nbx_mlp_predict(nbx_ctx* ctx, const float* features, uint64_t n, float* out);

/* ---- kernel-level queries (host buffers in/out) ------------------------- */
/* Batched octree propagate; ignore_tri / out_tri index the linearized
 * triangle array (-1: none). */
int nbx_ray_query(nbx_ctx* ctx, const float* pos, const float* dir, const float* dist, const int32_t* ignore_tri,
                  const int32_t* ignore_mat, uint64_t n, float* out_dist, int32_t* out_tri);
/* table: 0 elastic log-IMFP, 1 elastic cos-theta ICDF, 2 inelastic log-IMFP,
 *        3 inelastic log-omega' ICDF (log-omega under full Penn),
 *        4 Kieft ionisation (rounddown; not under full Penn). */
int nbx_table_query(nbx_ctx* ctx, int32_t material, int32_t table, const float* x, const float* y, uint64_t n,
                    float* out);
/* Full Penn 3-D tables of a context created with NBX_INELASTIC_FULL_PENN
 * (table_3D::get / get_rounddown, common/util/table_3D.inl:79-122):
 * table 0 q ICDF at (log E, omega / E, P), 1 ionisation at
 * (log E, log(omega / E), P). */
int nbx_table3_query(nbx_ctx* ctx, int32_t material, int32_t table, const float* x, const float* y, const float* z,
                     uint64_t n, float* out);
/* Philox4x32-10 blocks: ctr n x 4, key n x 2, out n x 4. */
int nbx_philox(nbx_ctx* ctx, const uint32_t* ctr, const uint32_t* key, uint64_t n, uint32_t* out);

/* One transport step (init -> intersect -> scatter) for each electron, with
 * the per-electron random streams of nbx_run.  Electrons are 56-byte
 * nbx_electron records updated in place; status[i] receives 0 alive,
 * 1 terminated, 2 detected; event[i] 0 none, 1 inelastic, 2 elastic,
 * 3 boundary; secondaries[i] receives the created secondary when
 * has_se[i] is 1. */
typedef struct {
    float pos[3];
    float dir[3];
    float E;
    int32_t mat;
    int32_t last_tri;
    uint32_t tag;
    uint64_t uid;
    uint32_t step;
    uint32_t pad;
} nbx_electron;
int nbx_step_query(nbx_ctx* ctx, nbx_electron* electrons, uint64_t n, int32_t* status, int32_t* event,
                   nbx_electron* secondaries, int32_t* has_se);
/* The network's 6 input features for each electron (n x 6 floats). */
int nbx_features_query(nbx_ctx* ctx, const nbx_electron* electrons, uint64_t n, float* out);

/* ---- allocation-free transport ------------------------------------------- */
/* No counterpart in the reference.  For callers that cannot allocate device
 * memory (a host application whose own caching allocator owns the GPU's
 * memory, or a pipeline that must not let an allocation's implicit device
 * synchronisation stall its streams): simulates n <= NBX_NOALLOC_MAX_PRIMARIES
 * primaries and their cascades from DEVICE buffers without allocating
 * anything.  d_particles holds n x 7 floats (pos, dir, E), d_tags n tags;
 * uid_base numbers the primaries' random streams exactly as the n primaries
 * of an nbx_push starting at that running index, so both entry points give
 * identical per-tag counts; uid_base + n must not exceed 2^63.
 *
 * Plain transport only: a context in sample or learned mode, or created with
 * record_deposits, gets NBX_ERR_STATE.  Only the per-tag counts and `counts`
 * are produced: no detected records, histogram, per-pixel spectra or
 * nbx_get_stats figures.  Detections are ADDED to d_se_count / d_bse_count
 * (n_tags each, caller-zeroed).  counts (host, may be null) receives
 * {elastic, inelastic, boundary, detected} of this call.
 *
 * Ordering: the call reads its inputs on the context's own stream, so the
 * caller must make d_particles, d_tags and the zeroed tallies complete first
 * (e.g. synchronise the stream that produced them).  The call returns only
 * after the GPU has finished.
 *
 * Scratch lives in a fixed array of about 9.5 MB that every GPU loading the
 * library keeps until exit.  The first call on a context looks up the array's
 * device address and should come before any stream capture.  Calls that
 * overlap on the GPU race on the array.
 *
 * Errors: sizes beyond the maximum, or uid_base + n above 2^63, return
 * NBX_ERR_ARG.  NBX_ERR_CAPACITY means a cascade outgrew the fixed scratch
 * (more than 65,536 secondaries waiting in one generation, or more than 256
 * generations): electrons were lost, and the detections made before that
 * have ALREADY been added to d_se_count / d_bse_count, so the caller should
 * discard those tallies. */
#define NBX_NOALLOC_MAX_PRIMARIES 65536
int nbx_run_noalloc(nbx_ctx* ctx, const float* d_particles, const uint32_t* d_tags, uint32_t n, uint64_t uid_base,
                    uint32_t* d_se_count, uint32_t* d_bse_count, uint64_t n_tags, uint64_t counts[4]);

#ifdef __cplusplus
}
#endif

#endif /* NBX_H */
