/*
 * swe_b200.h -- C ABI of the B200 shallow-water step library (libswe_b200.so).
 *
 * Drop-in boundary for the hot path of Syntaxswine/water-simulator: the
 * well-balanced finite-volume step of `ShallowWater` (src/swe.mjs) and its
 * spherical metric (src/geometry.mjs).  Host code (a Node N-API addon, the
 * Python mirror in water-simulator_b200/, or plain C) keeps the reference's
 * object model and calls these entry points; the library owns the device
 * buffers, the caller owns every host array and the library copies in and out.
 *
 * Conventions
 *   - Arrays are FP64, row-major over the padded grid W = nx + 4 by H = ny + 4
 *     (two ghost rings), index k = j*W + i, exactly as the reference's
 *     Float64Array fields (src/swe.mjs:196-220, 268).
 *   - Every function returns SWE_OK (0) or a negative status; the message of
 *     the last failure on the calling thread is swe_last_error().  Nothing
 *     aborts or traps.  Errors the reference throws (unknown limiter, bad
 *     latitudes, odd nx at a pole, bad Manning n) come back as SWE_EINVAL
 *     with the reference's message.
 *   - Each handle owns one CUDA stream; calls on one handle are synchronous
 *     with respect to the host data they return and must come from one
 *     thread at a time (the reference is single-threaded, src/swe.mjs:968).
 *   - There is no CPU fallback: if no CUDA device is usable, swe_create fails
 *     with SWE_ECUDA.
 */
#ifndef SWE_B200_H
#define SWE_B200_H

#ifdef __cplusplus
extern "C" {
#endif

#define SWE_OK          0
#define SWE_EINVAL     -1   /* bad argument; the reference would throw */
#define SWE_ECUDA      -2   /* CUDA runtime failure or no device */
#define SWE_ENONFINITE -3   /* a field went non-finite */
#define SWE_ETIMEOUT   -4   /* a bounded device wait gave up */

#define SWE_LIMITER_MC      0   /* src/swe.mjs:133 (default) */
#define SWE_LIMITER_MINMOD  1   /* src/swe.mjs:88 */
#define SWE_LIMITER_CENTRAL 2   /* src/swe.mjs:141 */

#define SWE_SIDE_WEST  0        /* side numbering of src/swe.mjs:1023 */
#define SWE_SIDE_EAST  1
#define SWE_SIDE_SOUTH 2
#define SWE_SIDE_NORTH 3

#define SWE_BC_REFLECT  0       /* reflect,  src/swe.mjs:1026 */
#define SWE_BC_OUTFLOW  1       /* outflow,  src/swe.mjs:1042 */
#define SWE_BC_PERIODIC 2       /* periodic, src/swe.mjs:1119 */
#define SWE_BC_FLATHER  3       /* flather,  src/swe.mjs:1085 */

/* field ids for swe_get_field / swe_set_field (src/swe.mjs:200-220) */
#define SWE_FIELD_B       0
#define SWE_FIELD_H       1
#define SWE_FIELD_HU      2
#define SWE_FIELD_HV      3
#define SWE_FIELD_H0      4     /* readable after a step with keep_h0 on */
#define SWE_FIELD_HU0     5
#define SWE_FIELD_HV0     6
#define SWE_FIELD_RH      7     /* readable after swe_residual */
#define SWE_FIELD_RHU     8
#define SWE_FIELD_RHV     9
#define SWE_FIELD_THETA  10
#define SWE_FIELD_MANNING 11

/* metric row ids for swe_get_geom / swe_set_geom (src/geometry.mjs:301-309) */
#define SWE_GEOM_DXROW    0
#define SWE_GEOM_DYROWN   1
#define SWE_GEOM_DYROWS   2
#define SWE_GEOM_DYCFL    3
#define SWE_GEOM_AREA     4
#define SWE_GEOM_LX       5
#define SWE_GEOM_LYN      6
#define SWE_GEOM_LYS      7
#define SWE_GEOM_BEDPHI   8
#define SWE_GEOM_PHIC     9
#define SWE_GEOM_TANPHI  10
#define SWE_GEOM_FROW    11
#define SWE_GEOM_GEOCOEF 12
#define SWE_GEOM_NROWS   13

/* scalar ids for swe_get_scalar / swe_set_scalar */
#define SWE_SCALAR_DX          0   /* NaN on a sphere (src/swe.mjs:185) */
#define SWE_SCALAR_DY          1
#define SWE_SCALAR_R           2   /* Infinity in Cartesian */
#define SWE_SCALAR_DLAM        3
#define SWE_SCALAR_DPHI        4
#define SWE_SCALAR_TOTAL_AREA  5
#define SWE_SCALAR_T           6   /* settable */
#define SWE_SCALAR_STEPS       7   /* settable */
#define SWE_SCALAR_MASS_FLOORED 8
#define SWE_SCALAR_EPS4        9

/* Constructor options, src/swe.mjs:170-174 (+ the `sphere` object,
 * src/geometry.mjs:190-192).  swe_options_init fills the reference defaults. */
typedef struct swe_options {
  int    nx, ny;
  double dx, dy;
  double manning;      /* 0.025 */
  double min_depth;    /* 1e-3 */
  double cfl;          /* 0.45 */
  double coriolis;     /* 0 */
  int    order;        /* 2 */
  int    limiter;      /* SWE_LIMITER_MC */
  int    sphere;       /* 0 Cartesian, 1 latitude-longitude */
  double R, lat0, lat1, omega;   /* sphere: 6371e3, -90, 90, 0 */
} swe_options;

typedef struct swe_sim swe_sim;

/* Select the CUDA device for handles created afterwards on this thread
 * (one process per GPU: rank r calls swe_set_device(r)). */
int swe_set_device(int ordinal);

/* Defaults of src/swe.mjs:170-174. */
int swe_options_init(swe_options* o);

/* new ShallowWater(opts), src/swe.mjs:170-244.  b and h are the sampled
 * bed and depth over the padded grid (the caller samples bed()/eta0() per
 * cell including ghosts, src/swe.mjs:222-232); hu = hv = 0.  Boundaries
 * default as the reference's (src/swe.mjs:239-241). */
int swe_create(const swe_options* o, const double* b, const double* h, swe_sim** out);
int swe_destroy(swe_sim* s);
const char* swe_last_error(void);
/* W, H, nx, ny */
int swe_get_dims(swe_sim* s, int* dims4);

/* sim.b / sim.h / ... reads and writes (src/swe.mjs:200-220). */
int swe_get_field(swe_sim* s, int field, double* out);
int swe_set_field(swe_sim* s, int field, const double* in);
/* Rows [row0, row0 + nrows) of the padded grid (row-major, W doubles per
 * row) of b, h, hu or hv: the halo exchange of a grid cut into row slabs
 * (water-simulator_b200/slabs.py).  No counterpart in the reference, which
 * runs one grid on one thread (src/swe.mjs:968-973).  Writing h, hu or hv
 * clears the dry-tile records, as swe_set_field does. */
int swe_get_rows(swe_sim* s, int field, int row0, int nrows, double* out);
int swe_set_rows(swe_sim* s, int field, int row0, int nrows, const double* in);
/* The same row copies without a host synchronisation, for a halo exchange
 * that stays on the device: dst / src may be device memory (another
 * buffer, a peer GPU's, a collective's) or pinned host memory.  They are
 * ordered on the handle's stream (swe_get_stream); the caller keeps src
 * valid until the stream has reached the copy. */
int swe_get_rows_async(swe_sim* s, int field, int row0, int nrows, double* dst);
int swe_set_rows_async(swe_sim* s, int field, int row0, int nrows, const double* src);
/* maxDt() written to the device double *dst on the handle's stream (no host
 * round trip), and step(dt) with dt read from the device double *dt when
 * the step runs: a grid cut into slabs over GPUs all-reduces the slabs'
 * maxDt on the device and steps each slab with the result.  A dt that is
 * not > 0 or not finite makes the step change nothing, as in swe_run.  No
 * counterpart in the reference (one grid, one thread, src/swe.mjs:968). */
int swe_max_dt_to(swe_sim* s, double* dst);
int swe_step_dt_from(swe_sim* s, const double* dt);
/* sim.geom.* rows (src/geometry.mjs:301-309); writes take effect from the
 * next device call, as a JS write to geom rows does (tools/verify-sphere.mjs:569). */
int swe_get_geom(swe_sim* s, int row, double* out);
int swe_set_geom(swe_sim* s, int row, const double* in);
int swe_get_scalar(swe_sim* s, int which, double* out);
int swe_set_scalar(swe_sim* s, int which, double v);

/* sim.boundaries.<side> = reflect | outflow | periodic | flather(...),
 * src/swe.mjs:1026-1126. */
int swe_set_boundary(swe_sim* s, int side, int kind);
/* flather(etaExt, uExt): the two values etaExt(sim.t), uExt(sim.t) for the
 * next step (they depend on t only, src/swe.mjs:1093). */
int swe_set_flather_values(swe_sim* s, int side, double eta_ext, double u_ext);
/* flather driven by a harmonic table evaluated on the device each step:
 * eta(t) = msl + sum amp[q] cos(omega[q] t - phase_deg[q] pi/180)
 * (Tide.eta, src/tide.mjs:103-107), u(t) = u_coef * eta(t). n <= 16. */
int swe_set_flather_tide(swe_sim* s, int side, double msl, int n, const double* amp,
                         const double* omega, const double* phase_deg, double u_coef);
/* setManningField, src/swe.mjs:714-731 (array form; NULL clears). */
int swe_set_manning_field(swe_sim* s, const double* n);
/* sim.forcing = makeSponge(sim, {side, width, strength, etaRef}),
 * src/swe.mjs:1174-1198, run on the device after friction. */
int swe_set_sponge(swe_sim* s, int side, int width, double strength, double eta_ref);
int swe_clear_sponge(swe_sim* s);
/* Keep a copy of the step's starting state readable as SWE_FIELD_H0.. */
int swe_set_keep_h0(swe_sim* s, int on);

/* applyBC(), src/swe.mjs:289-303 */
int swe_apply_bc(swe_sim* s);
/* residual(dt), src/swe.mjs:308-629: fills RH, RHU, RHV, THETA. */
int swe_residual(swe_sim* s, double dt);
/* maxDt(), src/swe.mjs:632-647 (Infinity when no cell is wet). */
int swe_max_dt(swe_sim* s, double* out);
/* applyFriction(dt), src/swe.mjs:659-704 */
int swe_apply_friction(swe_sim* s, double dt);
/* dryClean(), src/swe.mjs:734-745 */
int swe_dry_clean(swe_sim* s, double* added);
/* step(dt), src/swe.mjs:754-814: *taken = dt, or 0 when dt is not > 0 or not finite. */
int swe_step(swe_sim* s, double dt, double* taken);
/* step() with no argument: dt = maxDt(). */
int swe_step_auto(swe_sim* s, double* taken);
/* The drivers' loop `while (...) sim.step(...)` kept on the device: n steps
 * of dt = dt_fixed (if > 0) or maxDt(), each clamped to t_end - t
 * (t_end = +Infinity for none); stops early, like the loop, at the first
 * refused step.  *done = steps taken.  Launched as CUDA graphs. */
int swe_run(swe_sim* s, int n, double dt_fixed, double t_end, int* done);

/* Diagnostics, src/swe.mjs:819-917 (same summation order as the reference). */
int swe_volume(swe_sim* s, double* out);
int swe_energy(swe_sim* s, double* out);
int swe_max_surface_deviation(swe_sim* s, double ref, double* out);
/* The order of the Cartesian volume() sum.  SWE_DIAG_REFERENCE (the
 * default): one running sum over every interior cell in row-major order,
 * then one multiply by dx and dy -- the reference's own order
 * (src/swe.mjs:818-827) and its bits, but a chain of nx*ny dependent
 * additions.  SWE_DIAG_ROWS: each row summed left to right, then the rows
 * in order (the order the sphere's volume uses), then dx and dy: the same
 * result to round-off, deterministic, and parallel over rows.  Every other
 * diagnostic is in the reference's order and parallel already. */
#define SWE_DIAG_REFERENCE 0
#define SWE_DIAG_ROWS      1
int swe_set_diag_order(swe_sim* s, int order);
/* The area-weighted projection measureModePeriod() samples after every
 * step (src/globe.mjs:1414-1421): sum over interior rows j, in order, of
 * coef[j] * (sum over the row, left to right, of b + h), with coef[j] =
 * (wRow[j] / nx) * pRow[j] formed by the caller (ny doubles).  The same
 * bits as the reference's loop, and 8 bytes to the host per call. */
int swe_eta_projection(swe_sim* s, const double* coef, double* out);
int swe_max_speed(swe_sim* s, double* out);
int swe_finite(swe_sim* s, int* out);
/* Waits for the handle's stream.  SWE_ETIMEOUT when a tile copy of the
 * stepping kernels did not complete within its time bound since the last
 * call (that tile was left unwritten, so those steps are incomplete). */
int swe_synchronize(swe_sim* s);
/* The handle's CUDA stream (a cudaStream_t), so a caller can record CUDA
 * events on the stream the kernels run on. */
int swe_get_stream(swe_sim* s, void** stream);
/* step(dt) with CUDA events between its five launches (prepare, ghost fill,
 * stage 1, ghost fill, stage 2); ms[5] receives each launch's duration. */
int swe_step_timed(swe_sim* s, double dt, double* ms);
/* Launch shape of the stage kernel: grid x, grid y, threads, output
 * columns per CTA, output rows per CTA. */
int swe_get_launch_config(swe_sim* s, int* cfg5);

/* cartesianGeometry / sphericalGeometry (src/geometry.mjs:163-299) as a
 * host-side set-up call, no device needed: fills rows[13*H] (row id major)
 * and scalars[6] (SWE_SCALAR_DX .. SWE_SCALAR_TOTAL_AREA). */
int swe_compute_geometry(const swe_options* o, double* rows, double* scalars);

/* The exported hllc (src/swe.mjs:975) over a batch, on the device:
 * in = n x (hL, huL, hvL, hR, huR, hvR, dry), out = n x 3. */
int swe_hllc_batch(int n, const double* in, double* out);
/* sim.vel(hq, h) (src/swe.mjs:282) over a batch, on the device. */
int swe_vel_batch(swe_sim* s, int n, const double* hq, const double* h, double* out);

/* ---- Batched ensemble ----------------------------------------------------
 * Many independent basins of uneven sizes (each a full ShallowWater with its
 * own options, bed, boundaries, Manning n and Flather tide, and its own dt =
 * maxDt() every step) advanced together: one launch per kernel per ensemble
 * step over a tile list of all basins, captured as CUDA graphs.  The
 * schedule (the stage kernels and their tile: rows per tile 0 for the tiled
 * pair's 32 x 8 tiles, or 4..64 rows of the fused row-marching tile; CTAs --
 * 0 for one CTA per tile, else a persistent grid -- and tile order:
 * 0 basin-major, 1 largest basin first, 2 round robin) is set explicitly or
 * chosen by swe_batch_autotune, which times every candidate on the ensemble
 * itself and restores the state afterwards.  Each
 * basin's result is bit-identical to advancing it alone with swe_run.  The
 * reference drives one basin per ShallowWater (src/swe.mjs:145); this is the
 * many-basin form of that loop. */
typedef struct swe_batch swe_batch;
int swe_batch_create(int n, const swe_options* opts, const double* const* b, const double* const* h,
                     swe_batch** out);
int swe_batch_destroy(swe_batch* s);
int swe_batch_set_boundary(swe_batch* s, int basin, int side, int kind);
int swe_batch_set_flather_tide(swe_batch* s, int basin, int side, double msl, int n, const double* amp,
                               const double* omega, const double* phase_deg, double u_coef);
int swe_batch_set_schedule(swe_batch* s, int rows_per_tile, int ctas, int order);
/* rows per tile, ctas, order, number of tiles */
int swe_batch_get_schedule(swe_batch* s, int* out4);
int swe_batch_autotune(swe_batch* s, int trial_steps, int* best4, double* best_ms_per_step);
/* `steps` ensemble steps: every basin takes `steps` steps of its own maxDt(). */
int swe_batch_run(swe_batch* s, int steps);
/* Waits for the ensemble's stream; SWE_ETIMEOUT (once, then cleared) when a
 * work-queue wait of the steps run since the last call ran past its limit. */
int swe_batch_synchronize(swe_batch* s);
/* The launch form of an ensemble step with the tiled pair (rows 0).
 * 0: a launch per phase (prepare, ghost fill, faces, cells, ghost fill,
 * faces, cells).  1: ONE persistent launch per step over a device work
 * queue of every (basin, phase, tile) item in phase order; a CTA takes the
 * next item and waits, with a time limit, until the previous phase of that
 * item's basin is complete.  A wait past its limit drops the rest of the
 * step and swe_batch_synchronize returns SWE_ETIMEOUT.  Results are the same
 * bits either way.  The autotuner tries both. */
int swe_batch_set_launch(swe_batch* s, int queue);
int swe_batch_get_launch(swe_batch* s, int* queue);
/* The time limit of one work-queue wait (default 2 s). */
int swe_batch_set_wait_limit(swe_batch* s, double seconds);
/* Test hook: the prepare of `basin` is never marked complete (-1: none), so
 * that basin's next phase waits until its limit -- a wait that nothing
 * ends, for checking that it does end, with SWE_ETIMEOUT. */
int swe_batch_debug_hold(swe_batch* s, int basin);
int swe_batch_get_stream(swe_batch* s, void** stream);
int swe_batch_get_field(swe_batch* s, int basin, int field, double* out);   /* B, H, HU, HV */
int swe_batch_get_scalar(swe_batch* s, int basin, int which, double* out);  /* T, STEPS, MASS_FLOORED */

/* ---- Discrete adjoint ------------------------------------------------------
 * Gradient of a gauge misfit J = sum_steps sum_gauges (eta - obs)^2 with
 * respect to the bed b and the per-cell Manning n (both over the padded
 * grid; ghosts get 0), for `steps` self-timed steps from still water eta0
 * (h = max(0, eta0 - b), src/swe.mjs:229-231).  Cartesian; walls on every
 * side unless swe_adjoint_set_boundary says otherwise.  The forward pass
 * records dt and checkpoints the state every
 * `checkpoint_every` steps; swe_adjoint_backward recomputes each segment
 * and runs the hand-written reverse of every step, branches fixed as taken.
 * gauge_cells are padded indices k = j*W + i.  manning_field may be NULL
 * (scalar o->manning, no n gradient). */
typedef struct swe_adjoint swe_adjoint;
int swe_adjoint_create(const swe_options* o, const double* b, const double* eta0, const double* manning_field,
                       int n_gauges, const int* gauge_cells, int steps, int checkpoint_every, swe_adjoint** out);
int swe_adjoint_destroy(swe_adjoint* s);
int swe_adjoint_set_observations(swe_adjoint* s, const double* obs);      /* steps x n_gauges */
/* J, and (optional) eta at the gauges after every step (steps x n_gauges). */
int swe_adjoint_forward(swe_adjoint* s, double* J, double* gauge_eta);
int swe_adjoint_backward(swe_adjoint* s, double* grad_b, double* grad_n);
/* The dt of every step (steps doubles): read the sequence of the last
 * forward pass into dts_out, and/or hold the forward to dts_in from now on
 * (a finite-difference check needs the same frozen dts). */
int swe_adjoint_dt_sequence(swe_adjoint* s, double* dts_out, const double* dts_in);
int swe_adjoint_get_stream(swe_adjoint* s, void** stream);
/* The boundary of one side (SWE_SIDE_*) for the forward and its reverse:
 * SWE_BC_REFLECT (the default), _OUTFLOW, _PERIODIC, or _FLATHER with the
 * exterior state of swe_adjoint_set_flather_values (initially eta = u = 0),
 * as swe_set_boundary does for a simulation (src/swe.mjs:1026-1126).  A set
 * boundary asks for a new forward pass before the next backward. */
int swe_adjoint_set_boundary(swe_adjoint* s, int side, int kind);
/* Flather on `side` with the constant exterior surface eta_ext and normal
 * velocity u_ext (src/swe.mjs:1085-1115). */
int swe_adjoint_set_flather_values(swe_adjoint* s, int side, double eta_ext, double u_ext);
/* Flather on `side` with the exterior state of a tide, as
 * swe_set_flather_tide (src/tide.mjs:103-107): each step's values at its t
 * are recorded by the forward and used by the reverse. */
int swe_adjoint_set_flather_tide(swe_adjoint* s, int side, double msl, int n, const double* amp, const double* omega,
                                 const double* phase_deg, double u_coef);

/* ---- stage kernels -----------------------------------------------------------
 * Two implementations of each SSP-RK2 stage, bit-identical in their results:
 * SWE_STAGE_FUSED, one row-marching kernel per stage that keeps the stencil
 * on chip; SWE_STAGE_SPLIT, two tiled kernels (faces, then cells) that run
 * at higher occupancy through 12 extra fields in device memory (the
 * default).  The environment variable SWE_B200_STAGE=fused|split overrides
 * the default at creation. */
#define SWE_STAGE_FUSED 0
#define SWE_STAGE_SPLIT 1
int swe_set_stage_kernels(swe_sim* s, int impl);
int swe_get_stage_kernels(swe_sim* s, int* impl);

/* ---- gridlands terrain import (src/gridlands.mjs) -------------------------
 * A gridlands-terrain v1 export carries width x height float32 layers
 * (bedM, surfaceM, optional manningN), little-endian, base64-encoded, row 0 =
 * north.  The JSON document is parsed by the caller (gridlandsTerrain() checks
 * format, version, grid and rowOrder); the layers go to the device as text and
 * are decoded there.  Sampling follows gridlandsTerrain(): bed bilinear in
 * the export's cells, clamped at the edges (so the two ghost rings get
 * constant extrapolation), surface and Manning nearest-cell, with the row flip
 * that makes the sim's +y north (src/gridlands.mjs:262-291); the per-cell
 * Manning sampler is the one tools/verify-gridlands.mjs:330-331 hands to
 * setManningField(). */
typedef struct swe_gridlands {
  int width, height;           /* grid.width, grid.height: the export's cells */
  double cell_m;               /* grid.cellMeters */
  int flip_rows;               /* 1 (the default): export row 0 is the sim's top (north) row */
  const char* bed_b64;      size_t bed_len;       /* layers.bedM.data */
  const char* surface_b64;  size_t surface_len;   /* layers.surfaceM.data */
  const char* manning_b64;  size_t manning_len;   /* layers.manningN.data, or NULL */
  /* Host float32 layers used instead of the text when non-NULL (e.g. after
   * settleLakes() has lowered perched lakes on the host). */
  const float* bed_f32; const float* surface_f32; const float* manning_f32;
  int manning_field;           /* 1: also set the per-cell Manning field */
} swe_gridlands;

/* decodeF32 (src/gridlands.mjs:82-98) on the device: `len` characters of
 * base64 (standard or URL-safe alphabet, '=' padding optional) must decode to
 * exactly 4*n bytes, else SWE_EINVAL with the reference's message; writes n
 * floats to the host array `out`. */
int swe_gridlands_decode(const char* b64, size_t len, int n, float* out);

/* new ShallowWater({nx, ny, dx, dy, bed: t.bed, eta0: t.eta0, ...}) over an
 * imported terrain: o gives the grid (normally nx = width, ny = height,
 * dx = dy = cell_m; a finer or coarser grid samples the same functions) and
 * the solver options.  Cartesian only (SWE_EINVAL for a sphere).  With
 * manning_field set, a negative or non-finite n is refused as
 * setManningField() refuses it. */
int swe_gridlands_create(const swe_options* o, const swe_gridlands* g, swe_sim** out);

/* The connected waterbodies of waterbodies() (src/gridlands.mjs:107-139) as
 * a device pass: label[k] (W*H ints, host) is, for a wet cell
 * (surface - bed > 0), the lowest cell index of its 4-connected wet body --
 * the cell the reference's row-major flood fill starts that body from --
 * and -1 for a dry cell.  bed and surface are the export's float32 layers
 * (host, row 0 first).  SWE_ETIMEOUT if a union failed to settle within its
 * bounded retries (nothing is left waiting on the device). */
int swe_gridlands_bodies(int W, int H, const float* bed, const float* surface, int* label);

/* ---- headless frames (src/render.mjs, src/globe.mjs) ------------------------
 * RGBA bytes written into a device buffer (rgba_device, when non-NULL) and/or
 * copied to the host (rgba_host), stored as the reference's ImageData stores
 * a double (clamped to [0, 255], round half to even, NaN as 0).  No graphics
 * API is involved. */

/* The map panel of WaterView.draw() (src/render.mjs:220-247): nx * ny pixels,
 * row 0 = the sim's top row (+y up); water by the diverging ramp about `msl`
 * at full colour `scale` metres, darkened by the still depth when show_bed;
 * dry cells by the land ramp. */
int swe_render_map(swe_sim* s, double msl, double scale, int show_bed, unsigned char* rgba_host, void* rgba_device);

/* The colour tables, for checking: RAMP of src/render.mjs:118-131 (3 * 1025
 * doubles, unclamped sRGB) and CBYTES of src/globe.mjs:644-652 (3 * 1025
 * bytes).  Either pointer may be NULL. */
int swe_render_tables(double* ramp, unsigned char* cbytes);

/* buildGlobeLut(cam, gridOf(sim), style) (src/globe.mjs:554-629): the
 * pixel -> cell table of a size x size orthographic view at `tilt_deg`
 * with the disc inscribed at `margin`, baked once on the host and kept on
 * the device.  sun, bg, halo: 3 values each or NULL for the reference's
 * defaults ([-0.42, 0.48, 0.77], [8, 11, 16], [36, 58, 84]).  Spherical
 * sims only (SWE_EINVAL otherwise, as gridOf() throws). */
typedef struct swe_globe_lut swe_globe_lut;
int swe_globe_lut_create(swe_sim* s, int size, double tilt_deg, double margin, const double* sun,
                         const double* bg, const double* halo, swe_globe_lut** out);
int swe_globe_lut_destroy(swe_globe_lut* lut);
/* counts[4] = count (modelled pixels), inside (pixels on the disc), capped
 * (disc pixels outside the modelled band), size; then the table itself
 * (count entries each: byte offset, longitude at rotation 0 [deg], padded
 * index of the row's first interior cell, float32 light) and the baked
 * background (4 * size * size bytes).  Any pointer may be NULL. */
int swe_globe_lut_get(swe_globe_lut* lut, int* counts, int* px, double* lon_base, int* row_base, float* lit,
                      unsigned char* bg);
/* renderGlobe(out, sim, {lut, rotDeg, scale, msl, landLight})
 * (src/globe.mjs:770-812).  stats[8] = wet, dry, capped, inside, etaMin,
 * etaMax, sat, satFrac (may be NULL).  SWE_EINVAL when the grid is not the
 * one the table was baked for. */
int swe_render_globe(swe_sim* s, swe_globe_lut* lut, double rot_deg, double scale, double msl, int land_light,
                     unsigned char* rgba_host, void* rgba_device, double* stats);

/* maxDt() for callers that cannot allocate device memory.  It has no
 * counterpart in the reference; it serves callers that own all device memory
 * themselves (a fixed arena, a hard memory cap, a region where allocation is
 * forbidden) and so cannot create a handle.  Inputs are the caller's device
 * arrays over the padded grid (h, hu, hv: (nx+4)*(ny+4) doubles; dx_row,
 * dy_cfl: ny+4 doubles, the metric rows of src/geometry.mjs); the result,
 * cfl / max rate or Infinity, is written to the device double *dt_out, in
 * `stream` (a cudaStream_t, NULL for the default stream).  It allocates
 * nothing: its reduction scratch is a fixed array inside the library, so
 * ny is limited to SWE_NOALLOC_MAX_ROWS (larger grids get SWE_EINVAL), calls
 * that overlap on the GPU race, and the first call on each device looks the
 * array up and should come before any stream capture.  The looked-up
 * address belongs to the device's context: after cudaDeviceReset() the
 * entry point must not be called again in the same process. */
#define SWE_NOALLOC_MAX_ROWS 16384
int swe_max_dt_noalloc(int nx, int ny, const double* h, const double* hu, const double* hv,
                       const double* dx_row, const double* dy_cfl, double min_depth, double cfl,
                       double* dt_out, void* stream);

#ifdef __cplusplus
}
#endif
#endif
