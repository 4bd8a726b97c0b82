/*
 * chatcarlo_b200 -- C ABI of the B200 photon-transport engine.
 *
 * The entry points replace the NumPy hot path of ChatCarlo:
 *   cc_transport_photons  <- chatcarlo/transport.py:98-233  transport_photons(pos, dirv,
 *                            energy, geometry, rng, grid, recorder, tally_rng,
 *                            fluorescence_enabled) -> BatchResult
 *   cc_run                <- chatcarlo/transport.py:257-312,358-474  _run_batches /
 *                            run_transport(scene, n_histories, seed, batch_size, dose_grid, ...)
 *   cc_grid_*             <- chatcarlo/tally.py:27-132  VoxelGrid (+ end_batch 59-94)
 *   cc_scene_create       <- chatcarlo/geometry.py:121-231  Geometry
 *   cc_tables_create      <- chatcarlo/materials.py:202-496 (element tables, mu_en, S, F, K data)
 *                            and chatcarlo/dose_coefficients.py:32-42 (h*(10)/fluence)
 *   cc_source_create      <- chatcarlo/source.py:67-210 and chatcarlo/spectrum.py:73-82
 *
 * Conventions: every call returns 0 on success or a negative CC_E_* code;
 * cc_last_error() gives the message of the calling thread's last failure.
 * All sizes are explicit; the library copies what it needs to the device
 * and never keeps a caller pointer after a call returns.  Calls on one
 * context are synchronous at return.  Lengths in cm, energies in keV.
 */
#ifndef CHATCARLO_B200_H
#define CHATCARLO_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CC_ABI_VERSION 1

/* error codes (mirroring the ValueError cases of the NumPy path) */
#define CC_OK                   0
#define CC_E_INVALID          (-1)  /* bad argument */
#define CC_E_ENERGY_RANGE     (-2)  /* energy outside the cross-section tables: materials.py:234-237 */
#define CC_E_RAYLEIGH_Q_RANGE (-3)  /* q(E) beyond the form-factor table: physics.py:333-337 */
#define CC_E_UNKNOWN_MATERIAL (-4)  /* material index outside the table set: materials.py:66-69 */
#define CC_E_BAD_SHAPE        (-5)  /* unknown primitive type: geometry.py:158 */
#define CC_E_DEVICE           (-6)  /* CUDA runtime failure */
#define CC_E_TIMEOUT          (-7)  /* a photon exceeded the step limit */
#define CC_E_BOUNDS           (-8)  /* an index check failed inside a kernel */
#define CC_E_NOMEM            (-9)

/* primitive types (scene.py:14 VALID_SHAPES) */
#define CC_SHAPE_BOX      0
#define CC_SHAPE_SPHERE   1
#define CC_SHAPE_CYLINDER 2
#define CC_SHAPE_ELLIPSOID 3  /* axis-aligned ellipsoid: an extension with no reference
                                 counterpart (the reference has box/sphere/cylinder only) */

/* grid flags */
#define CC_GRID_STATS 1   /* batch statistics (kerma_sum2, h10_sum2, n_batches_hit) */

/* source field shapes (source.py:151-194) */
#define CC_FIELD_RECT     0
#define CC_FIELD_CONE     1
#define CC_FIELD_PARALLEL 2

typedef struct cc_ctx cc_ctx;
typedef struct cc_tables cc_tables;
typedef struct cc_scene cc_scene;
typedef struct cc_grid cc_grid;
typedef struct cc_source cc_source;
typedef struct cc_batch cc_batch;

/* One analytic primitive; list order is kept (a later one overrides an
 * earlier one where they overlap: geometry.py:205-212). */
typedef struct {
    int32_t type;          /* CC_SHAPE_* */
    int32_t material;      /* index into the material set of cc_tables */
    int32_t axis;          /* cylinder axis 0=x 1=y 2=z */
    int32_t pad;
    double center[3];
    double size[3];        /* box full edge lengths; ellipsoid full axis lengths (2 x semi-axes) */
    double radius;         /* sphere, cylinder */
    double height;         /* cylinder full length */
} cc_primitive;

/* Per-material tables.  Energies share one union grid per material. */
typedef struct {
    double density;               /* g/cm^3 */
    int32_t n_nodes;              /* union energy grid */
    int32_t n_elements;
    const double* log_e;          /* [n_nodes] ln(E/keV), strictly increasing */
    const double* log_parts;      /* [n_nodes][4] ln(photo), ln(compt), ln(rayl), ln(sum) of the
                                     mass-fraction mix, cm^2/g */
    const double* log_elem;       /* [n_elements][3][n_nodes] ln(w_i * sigma_i) for photo, compt, rayl */
    const int32_t* element_slot;  /* [n_elements] index into the element table array */
    const double* log_tally;      /* [n_nodes][2] ln(mu_en/rho) (log-log PCHIP through the NIST rows,
                                     materials.py:310-335) and ln(h*(10)/Phi) (dose_coefficients.py:
                                     32-42) at the nodes; the grid contains every mu_en and h*(10) row
                                     in range, so interpolating linearly in ln E reproduces h*(10)
                                     exactly and the PCHIP to ~1e-6 */
} cc_material_desc;

/* Per-element angular and fluorescence tables. */
typedef struct {
    int32_t z;
    int32_t n_lines;              /* <= 8 */
    const double* s_over_z;       /* [2000] S(Z,q)/Z on q = {0} U linspace(1e-3, 20, 1999) */
    const double* ray_x;          /* [2000] x = q^2, q = linspace(0, 20, 2000) */
    const double* ray_a;          /* [2000] A(x) = int_0^x F^2 dx' */
    double k_edge_kev;
    double k_shell_prob;          /* CS_Photo_Partial(K)/CS_Photo above the K edge */
    double omega_k;
    double line_e[8];             /* keV */
    double line_p[8];             /* probabilities, summing to 1 */
    int32_t emits;                /* 1 when some line reaches the 5 keV cut-off */
    int32_t pad;
} cc_element_desc;

typedef struct {
    int32_t n_materials;
    int32_t n_elements;
    const cc_material_desc* materials;
    const cc_element_desc* elements;
} cc_table_desc;

/* Heel effect of a rect or cone field (source.py:130-149,195-207): photons
 * are kept with the relative fluence at their coordinate s along the
 * anode-cathode axis on the SID plane (np.interp over the bin centres) and
 * take their energy from the spectrum of s's bin.  The reference computes
 * the bins with SpekPy (spectrum.py:88-129); the caller supplies them. */
#define CC_HEEL_MAX_BINS 64
typedef struct {
    double h_u, h_v;              /* unit anode direction projected on the beam basis (source.py:42-57) */
    double span_cm;               /* half-width of the field along the axis at the SID (source.py:60-65) */
    int32_t n_bins;               /* 1..CC_HEEL_MAX_BINS, of width 2 span / n_bins */
    int32_t pad;
    const double* centers;        /* [n_bins] bin centres on the axis (cm), increasing */
    const double* rel_fluence;    /* [n_bins] relative fluence in [0, 1], not all zero */
    const int32_t* bin_sizes;     /* [n_bins] energies of each bin's spectrum */
    const double* energies_kev;   /* the bins' spectra, concatenated */
    const double* weights;        /* their weights, concatenated (normalised per bin by the engine) */
} cc_heel_desc;

/* Point source into a field, with optional CT rotation (source.py:67-210). */
typedef struct {
    int32_t field;                /* CC_FIELD_* */
    int32_t rotation;             /* 0 = none, 1 = rotation about rot_axis */
    int32_t rot_axis;             /* 0/1/2 */
    int32_t n_angles;             /* 0 = continuous */
    double position[3];
    double direction[3];          /* unit */
    double u[3], v[3];            /* beam basis (source.py:28-35) */
    double sid_cm;
    double size_u, size_v;        /* rect/parallel field edge lengths */
    double cos_half_angle;        /* cone */
    double isocenter[3];
    double scan_length_cm;
    int32_t n_energies;           /* discrete spectrum */
    int32_t pad;
    const double* energies_kev;   /* [n_energies] */
    const double* weights;        /* [n_energies], not necessarily normalised */
    const cc_heel_desc* heel;     /* NULL: no heel effect; else rect/cone fields only, and the bins'
                                     spectra replace the spectrum above */
} cc_source_desc;

typedef struct {
    int64_t n_histories;
    int64_t n_absorbed;
    int64_t n_escaped;
    int64_t scatter_sum;
    int64_t n_fluorescence;
    int64_t n_batches;
    int64_t gpu_launches;         /* kernels launched (transport + batch folds) */
    double elapsed_ms;            /* device time of the run (CUDA events) */
    int64_t n_steps;              /* transport steps (track segments) of all histories */
    int64_t n_voxel_visits;       /* voxels crossed by the track-length tally walk (a voxel cut
                                     between two pieces of a split segment counts once) */
    double transport_ms;          /* device time of the transport kernel launches alone */
    int64_t transport_launches;
} cc_run_out;

/* -- context and error handling ------------------------------------------ */
int cc_version(void);
const char* cc_last_error(void);
int cc_ctx_create(int device, cc_ctx** out);
int cc_ctx_destroy(cc_ctx* ctx);
/* Launch shape of the transport kernels: blocks_per_sm = 0 (default) runs
 * as many blocks of 256 per SM as fit (four), or one on a grid whose batch
 * slot exceeds 32 MB, where fewer histories in flight keep fewer slots in
 * L2.  No reference counterpart (launch tuning). */
int cc_ctx_set_launch(cc_ctx* ctx, int block_size, int blocks_per_sm);
/* Transport steps a photon may take before the call fails with
 * CC_E_TIMEOUT (a guard against runaway histories; default 100000);
 * accepted range [1, 2^30]. */
int cc_ctx_set_step_limit(cc_ctx* ctx, int64_t max_steps_per_photon);

/* Tally scratch cells (no reference counterpart; the reference sums in
 * NumPy FP64).  Every batch scores into its own scratch slot, folded into
 * the FP64 totals after its launch.  By default (on = 0) the cells are FP64:
 * a seed reproduces its tallies up to the order of FP64 additions.  on = 1
 * makes a slot that sums at most 1e6 histories hold FP32 cells, so one
 * vector reduction scores kerma and H*(10) of a voxel visit: faster, with
 * sums that depend on the order of the FP32 additions (up to ~1e-3 relative
 * in the busiest voxels of a monoenergetic pencil beam). */
int cc_ctx_set_tally_fp32(cc_ctx* ctx, int32_t on);

/* Deferred tally (no reference counterpart): with on = 1 the transport
 * kernel queues its in-grid track segments in device memory and a second
 * kernel scores them; the scores are the same as the default in-kernel
 * tally's up to the order of the additions.  Off by default: slower on B200,
 * whose tally is bound by its atomics.  capacity > 0 fixes the queue's size in
 * records (segments beyond it are scored in the transport kernel); 0 sizes it
 * from the launch. */
int cc_ctx_set_tally_queue(cc_ctx* ctx, int32_t on, int64_t capacity);

/* -- tables, scene, source, grid -------------------------------------------- */
int cc_tables_create(cc_ctx* ctx, const cc_table_desc* desc, cc_tables** out);
int cc_tables_destroy(cc_tables* t);
int cc_scene_create(cc_ctx* ctx, const cc_primitive* prims, int32_t n_prims,
                    int32_t background_material, const double world_lo[3],
                    const double world_hi[3], cc_scene** out);
int cc_scene_destroy(cc_scene* s);
int cc_source_create(cc_ctx* ctx, const cc_source_desc* desc, cc_source** out);
int cc_source_destroy(cc_source* s);
int cc_grid_create(cc_ctx* ctx, const double origin[3], int32_t nx, int32_t ny, int32_t nz,
                   double voxel_cm, int32_t flags, cc_grid** out);
int cc_grid_destroy(cc_grid* g);
int cc_grid_reset(cc_grid* g);
/* Any output pointer may be NULL.  Arrays are C-ordered (nx, ny, nz).  An
 * output in page-locked host memory is written by the device directly;
 * other outputs go through a pinned staging buffer kept with the grid. */
int cc_grid_download(cc_grid* g, double* kerma_keV, double* h10_track_pSv_cm3,
                     double* kerma_sum2, double* h10_sum2, int32_t* n_batches_hit,
                     int64_t* n_batches, int64_t* n_histories);
/* Loads a grid's state (totals; for a CC_GRID_STATS grid also the sums of
 * squares, hit counts, batch and history counts) from host arrays, C-ordered
 * (nx, ny, nz), and clears any pending batch: no reference counterpart as
 * one call (the reference assigns VoxelGrid arrays or merges worker grids,
 * transport.py:416-417); for resuming a run or post-processing saved
 * tallies on the device. */
int cc_grid_upload(cc_grid* g, const double* kerma_keV, const double* h10_track_pSv_cm3,
                   const double* kerma_sum2, const double* h10_sum2, const int32_t* n_batches_hit,
                   int64_t n_batches, int64_t n_histories);
/* Output maps of a grid computed on the device, with the grid's totals as
 * cc_grid_download gives them:
 *   dose_Gy   <- chatcarlo/diagnostics.py:16-26 dose_map_Gy: kerma to dose
 *                with the density of the material at each voxel centre
 *                (tally.py:109-116 centres, geometry.py:102-118 closed point
 *                tests, the last primitive holding a centre wins, else
 *                background_density; tally.py:124-128)
 *   h10_pSv   <- tally.py:130-132 h10_map_pSv
 *   kerma_rel, h10_rel <- tally.py:96-100,135-175 relative errors (NaN where
 *                the reference gives NaN; need a CC_GRID_STATS grid)
 * prims / prim_density: the scene's primitives (as for cc_scene_create) and
 * the density of each one's material; voxel_volume_cm3: the caller's
 * voxel_cm ** 3; every map is divided by divisor last (1 for totals, the
 * history count for the per-history maps of chatcarlo/__main__.py:208-209).
 * FP64, evaluated in NumPy's order without contraction: the maps equal the
 * reference's host computation bit for bit.  on_device = 1: the outputs are
 * device pointers and nothing is copied to the host.  Any output may be
 * NULL. */
int cc_grid_maps(cc_grid* g, const cc_primitive* prims, int32_t n_prims, const double* prim_density,
                 double background_density, double voxel_volume_cm3, double divisor, int32_t on_device,
                 double* dose_Gy, double* h10_pSv, double* kerma_rel, double* h10_rel);
/* VoxelGrid.end_batch (tally.py:59-94) for photons scored outside cc_run:
 * folds the batch accumulated since the previous fold. */
int cc_grid_end_batch(cc_grid* g, int64_t n_histories_in_batch);

/* The grid's device-resident state, for summing grids of several ranks in
 * place with a collective (the reference sums its process workers' grids
 * on the host, transport.py:416-437; T, Q and the hit counts are additive).
 * totals: [nvox][2] FP64 (kerma, H*(10) interleaved per voxel); sum2s: the
 * same layout for the batch sums of squares (NULL without CC_GRID_STATS);
 * n_batches_hit: [nvox] int32 (NULL without CC_GRID_STATS).  Waits for the
 * grid's context stream first.  A batch still pending (photons scored by
 * cc_transport_photons* on a statistics grid since the last
 * cc_grid_end_batch) is not part of these arrays.  The pointers stay valid
 * until cc_grid_destroy.  Any output may be NULL. */
int cc_grid_device_buffers(cc_grid* g, double** totals, double** sum2s, int32_t** n_batches_hit,
                           int64_t* n_voxels, int64_t* n_batches, int64_t* n_histories);
/* Sets the batch and history counts (after the arrays were summed over
 * ranks, the counts are the ranks' sums). */
int cc_grid_set_counts(cc_grid* g, int64_t n_batches, int64_t n_histories);

/* -- transport ----------------------------------------------------------------
 * cc_transport_photons: transport_photons() on caller-provided photons.
 * pos/dir ([n][3]) and energy ([n]) are host arrays, updated in place with the
 * final state like the NumPy path does.  grid may be NULL.  Per-photon
 * outputs may be NULL.  edep_by_material has n_materials entries (keV),
 * accumulated into (not overwritten).  The photons' random streams are
 * Philox4x32-10 keyed by seed, counter (history index + stream_offset).
 * n_scatter is int64 like the reference's BatchResult.n_scatter. */
int cc_transport_photons(cc_ctx* ctx, const cc_scene* scene, const cc_tables* tables,
                         cc_grid* grid, int64_t n, double* pos, double* dir, double* energy,
                         uint64_t seed, uint64_t stream_offset, int32_t fluorescence,
                         int64_t* n_scatter, uint8_t* absorbed, uint8_t* escaped,
                         double* edep_by_material, int64_t* n_fluorescence);

/* Same on device-resident arrays (pointers into this device's memory). */
int cc_transport_photons_device(cc_ctx* ctx, const cc_scene* scene, const cc_tables* tables,
                                cc_grid* grid, int64_t n, double* d_pos, double* d_dir,
                                double* d_energy, uint64_t seed, uint64_t stream_offset,
                                int32_t fluorescence, int32_t* d_n_scatter, uint8_t* d_absorbed,
                                uint8_t* d_escaped, double* edep_by_material,
                                int64_t* n_fluorescence);

/* cc_run: _run_batches() with the source sampled on the device.  Histories
 * [first_history, first_history + n_histories) of the run keyed by seed are
 * simulated in batches of batch_size (the last batch may be smaller); with a
 * CC_GRID_STATS grid each batch is folded into the batch statistics. */
int cc_run(cc_ctx* ctx, const cc_scene* scene, const cc_tables* tables, const cc_source* src,
           cc_grid* grid, int64_t n_histories, int64_t batch_size, uint64_t seed,
           int64_t first_history, int32_t fluorescence, double* edep_by_material,
           double* edep_sum2_by_material, cc_run_out* out);

/* Allocation-free variant of cc_transport_photons_device.  It has no
 * counterpart in the reference.  It is for callers that cannot let the
 * library allocate device memory: an application that owns every device
 * allocation (a fixed memory pool per library), or a pipeline that forbids
 * cudaMalloc/cudaFree once it runs because they synchronise the device.
 * The scene, tables and all photon arrays are the caller's; the per-call
 * scratch (counters, work counter, status, deposited energy of up to 16
 * materials) lives in one static 512-byte __device__ array that each GPU
 * loading the library keeps until exit.  No tally grid.  The first call on
 * a device resolves that array's address (cudaGetSymbolAddress); make that
 * first call before any stream capture.  Every call clears and reuses the
 * same array, so calls that overlap on the GPU (other streams, other host
 * threads) race: serialise them.  stream is a cudaStream_t (NULL = the
 * legacy default stream); the call returns after the stream has finished
 * its work. */
int cc_transport_photons_device_noalloc(const cc_scene* scene, const cc_tables* tables, int64_t n,
                                        double* d_pos, double* d_dir, double* d_energy,
                                        uint64_t seed, uint64_t stream_offset, int32_t fluorescence,
                                        int32_t* d_n_scatter, uint8_t* d_absorbed, uint8_t* d_escaped,
                                        double* edep_by_material, int64_t* n_fluorescence, void* stream);

/* Batched multi-scene runs (no counterpart in the reference, which runs one
 * scene per run_transport call).  n_scenes scenes, each with its own source,
 * grid (grids may be NULL: no tallies) and history count, share one table
 * set and run in one persistent launch: warps take chunks of `chunk`
 * histories that never span two scenes; history i of scene s draws the
 * Philox stream of history (s << 40) + i.  With slots > 1 (grids created
 * with CC_GRID_STATS) each scene's histories form `slots` batches for the
 * batch statistics.  cc_batch_create captures the whole sequence (counter
 * reset, transport, batch folds) in a CUDA graph; cc_batch_run replays it.
 * The launch shape is the context's (cc_ctx_set_launch).  scene_counts gets
 * [n_scenes][4] absorbed, escaped, interactions, fluorescence emissions. */
int cc_batch_create(cc_ctx* ctx, const cc_tables* tables, int32_t n_scenes, const cc_scene* const* scenes,
                    const cc_source* const* sources, cc_grid* const* grids, const int64_t* n_histories,
                    int32_t slots, int32_t chunk, cc_batch** out);
int cc_batch_run(cc_batch* batch, uint64_t seed, int32_t fluorescence, int64_t* scene_counts,
                 cc_run_out* out);
int cc_batch_destroy(cc_batch* batch);

/* Sample source photons only (tests of source.py parity). */
int cc_sample_source(cc_ctx* ctx, const cc_source* src, int64_t n, uint64_t seed,
                     int64_t first_history, double* pos, double* dir, double* energy);

/* Single interactions, for sampler-by-sampler tests of the device physics
 * against the reference's samplers (physics.py:78-92,95-135,138-212,
 * 223-351; the reference calls them on whole photon arrays inside
 * transport_photons, transport.py:160-198).  Photon i of energy[i] keV in
 * material[i] (an index into the table set) takes one interaction of
 * `kind` through the transport kernel's own device code: the element draw
 * of that kind (w_i sigma_i(E) weights), then
 *   CC_INTERACT_PHOTO:    out_a = energy of the emitted K line, 0 when none
 *                         (fluorescence = 0 switches emission off)
 *   CC_INTERACT_COMPTON:  out_a = eps = E'/E, out_b = cos(theta)
 *   CC_INTERACT_RAYLEIGH: out_a = cos(theta)
 * out_z[i] = atomic number of the element drawn.  Photon i draws the
 * Philox stream of history i under seed.  Host arrays of n entries;
 * CC_E_ENERGY_RANGE / CC_E_RAYLEIGH_Q_RANGE as in transport. */
#define CC_INTERACT_PHOTO    0
#define CC_INTERACT_COMPTON  1
#define CC_INTERACT_RAYLEIGH 2
int cc_sample_interactions(cc_ctx* ctx, const cc_tables* tables, int32_t kind, int64_t n,
                           const int32_t* material, const double* energy, uint64_t seed,
                           int32_t fluorescence, double* out_a, double* out_b, int32_t* out_z);

/* Raw blocks of the device's Philox4x32-10 generator (known-answer tests;
 * the reference draws from NumPy's PCG64 instead, transport.py:120-121):
 * out[i][0..3] = Philox4x32-10(counter ctr[i][0..3], key key[i][0..1]).
 * Host arrays. */
int cc_philox4x32_10(cc_ctx* ctx, int64_t n, const uint32_t* ctr, const uint32_t* key, uint32_t* out);

/* Measured ceiling of the tally's FP64 reductions (no reference
 * counterpart; the reference tallies with np.add.at on the host,
 * tally.py:286-293).  Launches blocks x threads threads on device d_cells'
 * device, each scoring `per` voxel visits of two red.global.add.f64 into
 * one 16-byte cell of d_cells ([n_cells][2] doubles, zeroed by the caller):
 * mode 0 spreads the cells uniformly over the region, mode 1 over its
 * first `hot` cells, mode 2 walks `run` cells `stride` apart from a random
 * start.  visits_per_s = visits of `repeats` launches / their device time
 * (CUDA events, after one warm-up launch). */
int cc_measure_fp64_reductions(int device, double* d_cells, int64_t n_cells, int32_t mode, int32_t blocks,
                               int32_t threads, int32_t per, int32_t hot, int32_t run, int64_t stride,
                               int32_t repeats, double* visits_per_s);

#ifdef __cplusplus
}
#endif
#endif
