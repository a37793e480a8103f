/*
 * glide_b200 — C ABI of the B200 particle-step engine for GLIDE (mrghg/glide).
 *
 * Plain C: device pointers, sizes and a cudaStream_t passed as void*. No torch
 * types. Every entry point returns a glide_status (0 = ok); the text of the
 * last error on the calling thread is available from glide_last_error().
 * Launches are asynchronous on the given stream and perform no host
 * synchronisation, so they can be captured in a CUDA graph.
 *
 * Each entry point below names the reference interface it replaces
 * (file:line within the reference project).
 */
#ifndef GLIDE_B200_H
#define GLIDE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t glide_status;
enum {
    GLIDE_OK = 0,
    GLIDE_ERR_INVALID_ARG = 1,
    GLIDE_ERR_CUDA = 2,
    GLIDE_ERR_UNSUPPORTED = 3,
};

/* fixed-point scales of glide_step_args.diag_pos_fixed (2^20 per degree, 2^10 per metre) */
#define GLIDE_DIAG_DEG_SCALE 1048576
#define GLIDE_DIAG_M_SCALE 1024

/* storage type of the packed met bricks */
enum { GLIDE_MET_F32 = 0, GLIDE_MET_BF16 = 1, GLIDE_MET_F16 = 2 };

/* bits of the device status word (glide_step_args.status) */
enum {
    GLIDE_STATUS_NONFINITE_STATE = 1u << 0, /* a particle's state became NaN/inf */
    GLIDE_STATUS_BAD_ORDER = 1u << 1,       /* glide_step_args.order held an index outside [0, n) */
    GLIDE_STATUS_BAD_ROW = 1u << 2,         /* glide_compact_args.row_index held a row outside [0, n_rows) */
    GLIDE_STATUS_COMPACT_OVERFLOW = 1u << 3, /* glide_footprint_compact: more entries than capacity */
};

/* work classes written to glide_step_args.work_key: GLIDE_WORK_DONE, GLIDE_WORK_PENDING, or
 * for a particle stepped in the launch's last step 1 + (min(k, 3) - 1) + 3 (band + 5 regime),
 * k its substeps, band the height band of z_eval / boundary-layer height (0: below 0.25,
 * 1: below 0.5, 2: below 0.8, 3: at most 1, 4: above the boundary layer), regime the
 * stability regime (0 stable h/L > 1, 1 neutral, 2 unstable h/L < -1): classes 1 .. 45 */
enum { GLIDE_WORK_DONE = 0, GLIDE_WORK_PENDING = 63, GLIDE_WORK_CLASSES = 64 };

/* Met grid geometry: GridInterpolationBounds (src/lpdm/gpu_engine.py:100-121). */
typedef struct glide_grid {
    int32_t nz, ny, nx;
    int32_t ascending;           /* 1 if level[0] < level[nz-1] in the grid's own order */
    double lon_first, lon_last;  /* cell-centre coordinates of x = 0 and x = nx-1 */
    double lat_first, lat_last;  /* cell-centre coordinates of y = 0 and y = ny-1 */
    const float* level_sorted;   /* device [nz], AGL heights sorted ascending */
    /* optional lookup table accelerating the level search: level_lut[b] =
     * searchsorted(level_sorted, b / lut_inv_dz) for b in [0, lut_n); NULL = binary search.
     * Results are identical either way. */
    const int32_t* level_lut;
    int32_t lut_n;
    float lut_inv_dz;
} glide_grid;

/*
 * One met window [time_start, time_end]: raw fields of the two snapshots
 * (index 0 = start, 1 = end) as device float32 arrays. 3-D fields are
 * [nz][ny][nx] C-contiguous in the grid's level order; 2-D fields [ny][nx].
 */
typedef struct glide_window_desc {
    glide_grid grid;
    const float* u[2];
    const float* v[2];
    const float* w[2];
    const float* t[2];           /* 3-D temperature */
    const float* t_lowest[2];    /* [ny][nx] temperature at the lowest level */
    const float* blh[2];
    const float* sp[2];
    const float* ustar[2];
    const float* shf[2];
    const float* height3d;       /* [nz][ny][nx] AGL heights, or NULL ... */
    const float* height_level;   /* ... then [nz] per-level heights broadcast over columns */
    const float* pressure_hpa;   /* device [nz] bbox-mean pressure per level */
    float meander_coefficient;
    int32_t meander_radius;
    int32_t build_meander;
    int32_t met_dtype;           /* GLIDE_MET_* of the packed outputs */
    /* outputs (caller-allocated, sizes from glide_window_packed_bytes) */
    void* wind_packed;           /* [nz][ny][nx][8]: u0 v0 w0 u1 v1 w1 - - */
    void* surf_packed;           /* [ny][nx][16]: blh sp ustar shf t - - - (start), same (end) */
    void* support_packed;        /* [nz][ny][nx][8]: ft_sigma_w ft_T_Lw rho drho/dz meander_su meander_sv - - */
    /* optional output, device [6] float64 (added to; NULL = not computed): the sums over all
     * nz * ny * nx cells of u, v, w of the start snapshot, then of the end snapshot. Divided by
     * the cell count they are the grid means behind the runtime's per-step wind diagnostic
     * (_advection_alpha_wind_mean, src/lpdm/main.py:892-938). */
    double* wind_sum;
} glide_window_desc;

/* Per-outer-step schedule entry, computed on the host exactly as the
 * reference runtime does (src/lpdm/main.py:1386-1420, 892-919). */
typedef struct glide_step_sched {
    float cursor_off;  /* float32(cursor time - batch start), seconds */
    float delta;       /* outer step length, seconds */
    float alpha;       /* RK2 midpoint time weight in [0, 1] */
    int32_t step_index;/* global step number (Philox counter / noise row) */
} glide_step_sched;

/* Output grid of FootprintGridder (src/lpdm/footprint_gridder.py:50-115). */
typedef struct glide_footprint_grid {
    double lon_min, lon_max, lat_min, lat_max;
    int32_t n_releases, n_time_bins, n_z, n_y, n_x;
    const float* z_edges;        /* device [n_z + 1], ascending */
    /* 0: dense [n_releases][n_time_bins][n_z][n_y][n_x]. k > 0: ring of k live
     * time-ago slices per release, [n_releases][k][n_z][n_y][n_x], bin t stored in
     * slot t % k; the caller flushes a slot once its bin can no longer be reached. */
    int32_t ring;
    /* 0: float32 footprint values; 1: float64 values, each contribution weight * dt
     * formed and summed in FP64 (FootprintGridder(dtype=torch.float64),
     * src/lpdm/footprint_gridder.py:50-115) */
    int32_t value_f64;
} glide_footprint_grid;

typedef struct glide_step_args {
    int64_t n;                    /* particles */
    /* particle state (device, float32). Position fields share pos_stride:
     * 1 for structure-of-arrays, 4 for the reference's (N, 4) [lon, lat, z, weight]. */
    float* lon; float* lat; float* z; float* weight; int64_t pos_stride;
    float* u_prime; float* v_prime; float* w_prime;
    float* u_meander; float* v_meander;      /* NULL when meander is off */
    const float* rel_off;                    /* release time offsets (s after batch start) */
    const float* win_end_off;                /* release window end offsets */
    const int32_t* release_idx;              /* batch-local release index */
    uint8_t* alive;                          /* liveness (updated by the escape kill) */
    const uint8_t* active_mask;              /* if non-NULL, overrides the computed active mask */
    float sim_length_s;
    /* packed window (glide_window_pack) */
    const void* wind_packed; const void* surf_packed; const void* support_packed;
    int32_t met_dtype;
    glide_grid grid;
    /* HannaScheme parameters (src/lpdm/turbulence/hanna.py:440-520) */
    float substep_c; int32_t max_substeps; float z_ubl_m;
    int32_t flexpart_tl_floors; int32_t surface_layer_override;
    int32_t meander_enabled; float meander_timescale_s;
    /* steps of this launch: sched[0 .. n_steps) (device), or sched0 when sched == NULL and n_steps == 1.
     * Physics runs for steps j >= phys_begin, the footprint+escape post-step for j >= post_begin. */
    const glide_step_sched* sched; glide_step_sched sched0;
    int32_t n_steps; int32_t phys_begin; int32_t post_begin;
    /* noise: injected standard normals noise_substep[j][max_substeps][3][n] and
     * noise_meander[j][2][n] (j = step within this launch), or, when NULL,
     * Philox-4x32-10 draws keyed by seed and counted by (particle, step_index). */
    const float* noise_substep; const float* noise_meander; uint64_t seed;
    /* post-step (footprint + escape kill) */
    void* footprint;                         /* [R][T][Zb][Y][X] float32 (float64 when fp.value_f64),
                                              * may be NULL (no accumulation) */
    glide_footprint_grid fp;
    double dom_lon_min, dom_lon_max, dom_lat_min, dom_lat_max, dom_alt_max;
    int32_t* escaped_per_step;               /* [n_steps] counters (added to), may be NULL */
    int32_t* active_per_step;                /* [n_steps] counters (added to), may be NULL */
    uint32_t* status;                        /* device status word (GLIDE_STATUS_*), may be NULL */
    /* launch variant of the step kernel, 0 .. glide_step_launch_variants()-1: block size and
     * resident blocks per SM (0 = 128 threads x 6 blocks). The last variant is the general
     * kernel at shape 0, which every launch that sets surface_layer_override, injected noise
     * or uniforms, or active_mask runs whatever this field says. Results do not depend on it. */
    int32_t launch_variant;
    /* optional thread -> particle permutation, device [n] (NULL = identity): thread t steps
     * particle order[t]. Results do not depend on it (state and noise are keyed by particle
     * index); glide_reorder_by_key builds one that puts particles of equal work in the same
     * warps. It must be a permutation of 0..n-1: an entry outside [0, n) is skipped and sets
     * GLIDE_STATUS_BAD_ORDER; a repeated entry is not detected. */
    const int32_t* order;
    /* optional output, device [n] indexed by particle: the work class of the launch's last
     * step (GLIDE_WORK_*): done (escaped or past the simulation length), pending (alive but
     * not yet released), or the class of the branches and substep count it took. */
    uint8_t* work_key;
    /* optional convection fused into the launch: at step conv_step of the launch, after its
     * physics and before its post-step, the particles active at that step are redistributed
     * against the column in conv_column (the scratch of glide_convect with n = 0: conv_nz
     * levels) exactly as glide_convect_redistribute does. NULL = no convection. */
    const void* conv_column; int32_t conv_step; int32_t conv_nz;
    const float* conv_uniforms;   /* injected uniforms [2][n], or NULL: Philox keyed by seed */
    int32_t* conv_moved;          /* device counter of moved particles (added to), may be NULL */
    /* optional per-step diagnostic, device [n_steps][3] int64 (added to; NULL = none): the
     * sums over all n particles (active or not), after each step's post-step, of lon and
     * lat quantised to 1 / GLIDE_DIAG_DEG_SCALE degree and z to 1 / GLIDE_DIAG_M_SCALE m
     * (each value times the scale, rounded to the nearest integer). Divided by the scale
     * and n they are the runtime's mean-position diagnostic (particles[:, :3].mean(0),
     * src/lpdm/main.py:1565-1566). Integer sums: the result does not depend on the
     * launch shape or the particle order. Only steps j >= post_begin are summed; n_steps
     * is then at most 1535. Positions must stay below 2048 degrees and 2097 km. */
    int64_t* diag_pos_fixed;
} glide_step_args;

/* Emanuel convection for one window (src/lpdm/convection/emanuel.py:570-805). */
typedef struct glide_convect_args {
    int64_t n;
    float* z; int64_t z_stride;              /* particle heights (updated) */
    const float* rel_off; const uint8_t* alive; const uint8_t* active_mask;
    float sim_length_s;
    glide_step_sched sched;                  /* the first step of the window */
    int32_t nz, ny, nx;
    const float* t[2]; const float* q[2];    /* [nz][ny][nx] snapshots */
    const float* height3d; const float* height_level;
    const float* pressure_hpa;               /* [nz] */
    float alpha;
    float closure_c, trigger_dtv_k, min_cape_j_kg, min_cloud_depth_m;
    const float* uniforms;                   /* injected [2][n] uniforms, or NULL → Philox(seed) */
    uint64_t seed;
    void* scratch;                           /* glide_convect_scratch_bytes(nz) bytes, device */
    int32_t* n_moved;                        /* device counter (added to), may be NULL */
} glide_convect_args;

/* Exact-OU velocity update of the engine primitives (GPUEngine.update_langevin_velocity,
 * src/lpdm/gpu_engine.py:345-398 with _ou_step_kernel :26-42). Each per-particle input
 * is a device array [n] or, when NULL, the scalar beside it. */
typedef struct glide_ou_args {
    int64_t n;
    float* w;                                   /* velocity [n], updated in place */
    const float* t_l; float t_l_scalar;         /* Lagrangian timescale, s (> 0) */
    const float* sigma2; float sigma2_scalar;   /* velocity variance, m^2/s^2 (>= 0) */
    const float* dt; float dt_scalar;           /* step, s (> 0) */
    const float* drift; float drift_scalar;     /* deterministic acceleration, m/s^2 (drift * dt added) */
    const float* noise;                         /* standard normals [n], or NULL: drawn from (seed, counter) */
    uint64_t seed; uint32_t counter;
} glide_ou_args;

/* Pressure-level -> terrain-following (AGL) regrid of one met hour
 * (MetReader._resample_hour_to_agl, src/lpdm/met_reader.py:641-693, with
 * lpdm/vertical_grid.py:166-318). Device arrays unless noted. */
#define GLIDE_REGRID_MAX_LEVELS 256
typedef struct glide_regrid_args {
    int32_t n_channels, zp, za, ny, nx;
    const float* height_agl_p;     /* [zp][ny][nx] AGL height of each stored level (may be negative) */
    const double* agl_levels;      /* HOST [za], strictly ascending target heights */
    const float* fields_p;         /* [n_channels][zp][ny][nx] */
    float* fields_agl;             /* [n_channels][za][ny][nx] output */
    const double* pressure_p_hpa;  /* [zp][ny][nx], or NULL */
    double* pressure_level_hpa;    /* [za] output: bbox mean of the regridded pressure */
    int32_t u_channel, v_channel, w_channel; /* w_channel < 0: no slope correction of w */
    const double* dhdx; const double* dhdy;  /* [ny][nx] terrain slopes, m/m (terrain_gradient) */
    int32_t slope_f32;             /* bit 0 / 1: dhdx / dhdy hold float32 values, multiplied in float32
                                    * as numpy multiplies two float32 arrays (the reference's dhdy is
                                    * float32 when the terrain is) */
    double z_top_m;                /* top of the taper of the slope correction */
    void* scratch; size_t scratch_bytes;     /* glide_agl_regrid_scratch_bytes(za, ny, nx) */
} glide_regrid_args;

/* Sparse form of completed footprint slices (glide_footprint_compact). A slice is one
 * (release, time_ago) block [n_z][n_y][n_x] of the footprint, stored as one row of
 * `cells` float32 (float64 when value_f64). Device memory throughout. */
typedef struct glide_compact_args {
    void* rows;                    /* [n_rows][cells] slices; cleared entries are set to 0 */
    int64_t n_rows;
    int64_t cells;                 /* values per slice, 1 .. INT32_MAX */
    const int64_t* row_index;      /* [k] rows to compact, in output order */
    int32_t k;
    int32_t clear;                 /* != 0: set every compacted row to 0 (the rows must be distinct) */
    int64_t* slice_offset;         /* [k + 1] out: slice s holds entries [slice_offset[s], slice_offset[s+1]) */
    int32_t* out_cell;             /* [capacity] out: cell index within the slice, ascending per slice */
    void* out_value;               /* [capacity] out: the value, bit-unchanged (float32 or float64) */
    int64_t capacity;
    uint32_t* status;              /* device status word (GLIDE_STATUS_*), may be NULL */
    void* scratch; size_t scratch_bytes;  /* glide_footprint_compact_scratch_bytes(k, cells) */
    int32_t value_f64;             /* 1: rows and out_value hold float64 values (8-byte words) */
} glide_compact_args;

/* --- library ------------------------------------------------------------------ */

/* Version of this ABI (major * 10000 + minor * 100 + patch). */
int32_t glide_version(void);

/* Copies the last error message of the calling thread into buf (NUL-terminated). */
glide_status glide_last_error(char* buf, size_t len);

/* sizeof of the ABI structs, in declaration order: glide_grid, glide_window_desc,
 * glide_step_sched, glide_footprint_grid, glide_step_args, glide_convect_args,
 * glide_ou_args, glide_regrid_args, glide_compact_args. Lets a binding verify its
 * struct layouts. Writes min(n, 9) values. */
glide_status glide_abi_struct_sizes(size_t* out, int32_t n);

/* --- per-window met packing ------------------------------------------------------
 * Replaces the per-window device staging and support-field builds of
 * HannaScheme: _cached_raw_device_met (src/lpdm/turbulence/hanna.py:747-796),
 * _free_trop_fields (:1694-1745), _density_fields (:1747-1784) and
 * _meander_sigma_fields (:1786-1830). */
glide_status glide_window_packed_bytes(int32_t nz, int32_t ny, int32_t nx, int32_t met_dtype,
                                       size_t* wind_bytes, size_t* surf_bytes, size_t* support_bytes);
glide_status glide_window_pack(const glide_window_desc* desc, void* stream);

/* --- the fused particle step ---------------------------------------------------
 * One launch runs n_steps outer steps of the static step body for every
 * particle: HannaScheme._step_core (src/lpdm/turbulence/hanna.py:898-1068,
 * with _advect_rk2 :855-896 and _integrate_vertical_substeps_static
 * :1224-1368), and after each step the runtime's footprint scatter-add
 * (FootprintGridder.accumulate, src/lpdm/footprint_gridder.py:117-197) and
 * escape kill (src/lpdm/main.py:1459-1477, 690-711). */
glide_status glide_step(const glide_step_args* args, void* stream);

/* Several independent glide_step launches as one grouped launch: each of the `count`
 * argument sets is a batch with its own particles, schedule, met window, footprint and
 * counters, computed exactly as glide_step would; blocks of 128 threads are handed out to
 * the batches by particle count, so batches of very different sizes fill one launch. All
 * batches use the same met_dtype; the general kernel runs for all when any batch needs it;
 * launch_variant is ignored. At most GLIDE_STEP_BATCH_MAX batches (no counterpart in the
 * reference: its serving unit is one batch per process). */
#define GLIDE_STEP_BATCH_MAX 32
glide_status glide_step_batched(const glide_step_args* args, int32_t count, void* stream);

/* Number of launch variants of the step kernel and, for variant v, its block size
 * and the resident blocks per SM it is compiled for (autotuning; the last variant is
 * the general kernel, see glide_step_args.launch_variant). */
glide_status glide_step_launch_variants(int32_t* count);
glide_status glide_step_launch_variant_info(int32_t v, int32_t* threads, int32_t* min_blocks_per_sm);

/* --- particle ordering ---------------------------------------------------------
 * No counterpart in the reference (its static path runs every particle through the
 * same tensor ops). Builds order[0 .. n) for glide_step_args.order from a work_key
 * written by the previous launch: descending work class (GLIDE_WORK_PENDING first,
 * GLIDE_WORK_DONE last), stable within a class, so that the lanes of a warp take the
 * same closure branches and the same number of substeps, and finished particles fill
 * whole warps. Keys above GLIDE_WORK_PENDING count as it. Three launches on `stream`,
 * no synchronisation; scratch
 * is device memory of glide_reorder_scratch_bytes(n) bytes. n <= INT32_MAX. */
glide_status glide_reorder_scratch_bytes(int64_t n, size_t* bytes);
glide_status glide_reorder_by_key(int64_t n, const uint8_t* work_key, int32_t* order, void* scratch,
                                  size_t scratch_bytes, void* stream);

/* --- engine primitives -----------------------------------------------------------
 * The per-substep updates of glide_step as separate launches on float32 device arrays,
 * for engine-level callers and tests: GPUEngine.update_langevin_velocity,
 * apply_vertical_turbulence, apply_horizontal_turbulence, reflect_surface and the stages
 * of rk2_advect_backward (src/lpdm/gpu_engine.py:308-507). They run the same device
 * functions as the fused kernel's substep loop. Positions use a stride (4 for the
 * reference's (N, 4) particle tensor); dt is a device array [n] or, when NULL, dt_scalar;
 * backward != 0 displaces by -velocity. */
glide_status glide_ou_update(const glide_ou_args* args, void* stream);
glide_status glide_displace_vertical(int64_t n, float* z, int64_t z_stride, const float* w, const float* dt,
                                     float dt_scalar, int32_t backward, void* stream);
glide_status glide_displace_horizontal(int64_t n, float* lon, float* lat, int64_t stride, const float* u,
                                       const float* v, const float* dt, float dt_scalar, int32_t backward,
                                       void* stream);
/* (z, w) -> (2 z_surface - z, -w) where z < z_surface */
glide_status glide_reflect_surface(int64_t n, float* z, int64_t z_stride, float* w, float z_surface, void* stream);
/* out[i][0..3) = x[i][0..3) - h * v[i][0..3) (strides >= 3, in floats) */
glide_status glide_rk2_stage(int64_t n, const float* x, int64_t x_stride, const float* v, int64_t v_stride, float h,
                             float* out, int64_t out_stride, void* stream);

/* --- met regrid ------------------------------------------------------------------
 * compute_agl_regrid_weights + apply_agl_regrid + slope_correct_w + the per-level
 * bbox-mean pressure of MetReader._resample_hour_to_agl (src/lpdm/met_reader.py:
 * 641-693; src/lpdm/vertical_grid.py:166-258, 296-318) for one hour: weights in
 * FP64, channels interpolated as torch.lerp does, the slope correction in FP64. */
glide_status glide_agl_regrid_scratch_bytes(int32_t za, int32_t ny, int32_t nx, size_t* bytes);
glide_status glide_agl_regrid(const glide_regrid_args* args, void* stream);

/* --- footprint accumulation alone -----------------------------------------------
 * FootprintGridder.accumulate (src/lpdm/footprint_gridder.py:117-197) for the
 * per-step plug-in path. t_idx and release_idx are int32 [n]; positions follow
 * pos_stride as in glide_step_args. The footprint holds float32 values, or float64
 * when grid->value_f64 (weight * dt formed and added in FP64). */
glide_status glide_footprint_accumulate(int64_t n, const float* lon, const float* lat, const float* z,
                                        int64_t pos_stride, const uint8_t* active, const float* weights,
                                        int64_t weight_stride, const int32_t* t_idx,
                                        const int32_t* release_idx, float dt_seconds,
                                        const glide_footprint_grid* grid, void* footprint, void* stream);

/* --- sparse footprint slices -----------------------------------------------------
 * The device half of streaming completed footprint slices to the output writer
 * (OutputWriter.write_footprint_region, src/lpdm/output_writer.py:215-243, which takes
 * dense (release, T, Z, Y, X) blocks): most cells of a slice are zero, so the slices
 * leave the device as (cell, value) lists. Entry e of the output is a cell whose float32
 * (float64 when value_f64) bit pattern is not zero (so -0.0 and NaN are kept and a dense slice is rebuilt
 * bit-exactly by writing the values into zeros); slices in row_index order, cells
 * ascending within a slice. A row outside [0, n_rows) sets GLIDE_STATUS_BAD_ROW and
 * yields an empty slice. slice_offset is always written; when its last entry (the total)
 * exceeds capacity, GLIDE_STATUS_COMPACT_OVERFLOW is set and nothing else is written or
 * cleared. Three launches on `stream`, no synchronisation. No counterpart in the
 * reference, which copies the dense footprint to the host. */
glide_status glide_footprint_compact_scratch_bytes(int32_t k, int64_t cells, size_t* bytes);
glide_status glide_footprint_compact(const glide_compact_args* args, void* stream);

/* --- Emanuel convection ------------------------------------------------------------
 * EmanuelReducedConvection.maybe_convect (src/lpdm/convection/emanuel.py:570-716)
 * and _redistribute_particles (:720-805): bbox-mean column, FP64 column build
 * (LCL/LNB/CAPE, non-divergent mass-flux matrix, backward transition CDF), then
 * per-particle transposed-column sampling. */
glide_status glide_convect_scratch_bytes(int32_t nz, size_t* bytes);
glide_status glide_convect(const glide_convect_args* args, void* stream);

/* The per-particle half of glide_convect (_redistribute_particles,
 * src/lpdm/convection/emanuel.py:720-805) against a column already built in
 * args->scratch by an earlier glide_convect on the same scratch (with n = 0 that
 * call builds the column only). Lets a runtime build the next window's column
 * ahead of time on another stream. */
glide_status glide_convect_redistribute(const glide_convect_args* args, void* stream);

/* Maximum number of met levels that glide_convect_noalloc accepts. */
#define GLIDE_CONVECT_NOALLOC_MAX_NZ 128

/* glide_convect for callers that cannot allocate device memory. No counterpart
 * in the reference: it exists for callers that must not call cudaMalloc, such as
 * a serving loop that has already committed its whole HBM budget to particle
 * state and footprints, a process whose framework allocator holds nearly all
 * device memory (a raw cudaMalloc there fails or fragments the pool), or a
 * foreign-language caller with no access to any device allocator. The caller
 * still passes every input and output; args->scratch is ignored. The scratch
 * lives in one static device array of the library, sized for at most
 * GLIDE_CONVECT_NOALLOC_MAX_NZ levels (135 KB, held by every GPU that loads the
 * library until exit); larger grids are rejected with GLIDE_ERR_INVALID_ARG.
 * Every call made outside stream capture looks up that array's device address
 * on the current device (so a device reset, which reloads the library's module
 * and may move the array, is followed by the next such call); a call on a
 * capturing stream reuses the address the last uncaptured call on that device
 * found, so make the first call on each device before any stream capture. All calls
 * share the array: two calls that may run at the same time on the GPU (streams
 * not ordered with each other) race on it. Each call writes every part of the
 * array it reads before reading it, so nothing needs clearing between calls.
 * Allocates nothing. */
glide_status glide_convect_noalloc(const glide_convect_args* args, void* stream);

/* Reads the column result left in the scratch buffer by the last glide_convect
 * on it (synchronises the stream): fires, i_lcl, i_lnb, cape, dtv, m_b. */
glide_status glide_convect_column_info(const void* scratch, int32_t nz, void* stream, int32_t* fires,
                                       int32_t* i_lcl, int32_t* i_lnb, double* cape, double* dtv, double* m_b);

#ifdef __cplusplus
}
#endif

#endif /* GLIDE_B200_H */
