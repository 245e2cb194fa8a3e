/*
 * fvm_b200.h -- C ABI of the B200 (sm_100a) compressible-flow hot path.
 *
 * This library replaces the device side of the reference solver class
 * `CFDSolver` (reference: src/include/solver.cuh:22-257, implemented in
 * src/solver.cu:2873-3845).  Every entry point returns an int status
 * (FVM_OK == 0) instead of calling exit() the way the reference's CUDA_CHECK
 * macro does (src/include/solver.cuh:8-19).  Signatures use plain pointers and
 * sizes only.  A handle owns one CUDA stream and every device buffer of one
 * solve; calls on one handle must be serialised by the caller, exactly like
 * the reference protocol (one solver thread, src/main.cpp:225-380).
 *
 * Field layout seen through this ABI (readback/writeback) is the reference's:
 * row-major, idx = j*nx + i, SoA float arrays of length nx*ny.
 */
#ifndef FVM_B200_H
#define FVM_B200_H

#include <stddef.h>
#include <stdint.h>
#include <stdbool.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
enum fvm_status {
    FVM_OK = 0,
    FVM_ERR_INVALID = 1,      /* bad argument (null pointer, nx<=0, unknown enum, ...) */
    FVM_ERR_CUDA = 2,         /* a CUDA runtime/driver call failed */
    FVM_ERR_ALLOC = 3,        /* device or pinned allocation failed */
    FVM_ERR_STATE = 4,        /* call out of order (e.g. step before initialize) */
    FVM_ERR_TIMEOUT = 5,      /* a bounded device wait gave up (kernel error word set) */
    FVM_ERR_NONFINITE = 6,    /* device non-finite counter tripped */
    FVM_ERR_BUDGET = 7,       /* batch/serve admission refused: over HBM budget */
    FVM_ERR_UNSUPPORTED = 8   /* feature not available on this device */
};

/* Text of the last error recorded on the calling thread (never NULL). */
const char *fvm_last_error(void);

/* ------------------------------------------------------------ parameters */
/* Obstacle shapes.  0..5 are the reference enum `ObstacleShape`
 * (src/include/common.h:39-47); 6 is a blunted cone (sphere-cone) with no
 * reference counterpart. */
enum fvm_shape {
    FVM_SHAPE_CIRCLE = 0,
    FVM_SHAPE_STAR = 1,
    FVM_SHAPE_DIAMOND = 2,
    FVM_SHAPE_CAPSULE = 3,
    FVM_SHAPE_TRIANGLE = 4,
    FVM_SHAPE_STARSHIP = 5,
    FVM_SHAPE_CONE_CAPSULE = 6
};

/* Cell classes, values of the reference enum `CellType` (src/include/common.h:105-111). */
enum fvm_cell_type {
    FVM_CELL_FLUID = 0,
    FVM_CELL_SOLID = 1,
    FVM_CELL_GHOST = 2,
    FVM_CELL_INFLOW = 3,
    FVM_CELL_OUTFLOW = 4
};

/* Byte-for-byte the reference `struct SimParams` (src/include/common.h:50-102):
 * 112 bytes, 4-byte aligned, same field order.  The C++ shim static_asserts the
 * equivalence so `SimParams*` can be passed straight through. */
typedef struct fvm_sim_params {
    int nx, ny;
    float dx, dy;
    float domain_width, domain_height;
    float mach, T_inf, p_inf, rho_inf, u_inf, v_inf, c_inf;
    float obstacle_x, obstacle_y, obstacle_r, obstacle_rotation;
    int obstacle_shape;
    float wing_rotation;
    float cfl, dt, t_current;
    int step;
    bool enable_viscosity;
    float cfl_visc;
    bool adiabatic_wall;
    float T_wall;
    bool paused;
} fvm_sim_params;

/* Host-side `SimParams::computeDerived` (src/include/common.h:93-101):
 * rho_inf, c_inf, u_inf, dx, dy and obstacle_y = domain_height/2. */
void fvm_params_compute_derived(fvm_sim_params *p);
/* The reference's default member initialisers (src/include/common.h:53-90). */
void fvm_params_default(fvm_sim_params *p);

enum fvm_flux_scheme { FVM_FLUX_HLLC = 0, FVM_FLUX_AUSM_PLUS = 1 };
enum fvm_limiter { FVM_LIMITER_MINMOD = 0, FVM_LIMITER_VAN_LEER = 1 };
enum fvm_dt_policy {
    FVM_DT_FIXED = 0,     /* use SimParams.dt as given (reference KernelBenchmark) */
    FVM_DT_RECOMPUTE = 1  /* dt of step n+1 from the CFL reduction fused into step n */
};

/* Knobs the reference hard-codes.  fvm_ext_default() reproduces the reference:
 * HLLC (src/solver.cu:1572,1658), minmod (src/solver.cu:110-150), Pr 0.71
 * (src/include/common.h:19), fixed dt. */
typedef struct fvm_ext {
    int flux_scheme;        /* enum fvm_flux_scheme */
    int limiter;            /* enum fvm_limiter */
    float prandtl;          /* 0.71 in the reference */
    int dt_policy;          /* enum fvm_dt_policy */
    float cone_half_angle;  /* FVM_SHAPE_CONE_CAPSULE: frustum half angle [rad] */
    float cone_length;      /* FVM_SHAPE_CONE_CAPSULE: frustum length along the axis [m] */
    float ref_length;       /* reference length for force coefficients [m] (0: 2*obstacle_r) */
    int reserved[8];
} fvm_ext;

void fvm_ext_default(fvm_ext *e);

/* ------------------------------------------------------------- lifecycle */
typedef struct fvm_handle fvm_handle;

int fvm_create(fvm_handle **out);
int fvm_destroy(fvm_handle *h);

/* Launch this handle's work on `stream` (a cudaStream_t); NULL restores the
 * handle's own stream.  The caller keeps ownership of the stream. */
int fvm_set_stream(fvm_handle *h, void *stream);

/* CFDSolver::initialize (src/solver.cu:3102-3111): allocate for nx*ny, then reset. */
int fvm_initialize(fvm_handle *h, const fvm_sim_params *p, const fvm_ext *ext);
/* CFDSolver::resize (src/solver.cu:3119-3129). */
int fvm_resize(fvm_handle *h, int nx, int ny);
/* CFDSolver::reset (src/solver.cu:3136-3162): freestream, SDF + cell marking,
 * boundary conditions, primitives, viscosity field. */
int fvm_reset(fvm_handle *h, const fvm_sim_params *p);
/* CFDSolver::updateObstacleGeometry (src/solver.cu:3171-3196). */
int fvm_update_obstacle(fvm_handle *h, const fvm_sim_params *p);
/* Replace the extension knobs without touching the flow state. */
int fvm_set_ext(fvm_handle *h, const fvm_ext *ext);

/* -------------------------------------------------------------- stepping */
/* CFDSolver::step (src/solver.cu:3289-3412): one SSP-RK2 step (Strang split
 * when p->enable_viscosity); advances p->t_current and p->step.  Under
 * FVM_DT_RECOMPUTE, p->dt receives the dt that was used, and the call waits
 * for the step and reports a device error word (FVM_ERR_TIMEOUT after an
 * expired bounded wait) itself.  Under FVM_DT_FIXED the call returns once the
 * work is queued; a device error of those steps is reported by the next
 * fvm_synchronize (or the next call that reads device scalars). */
int fvm_step(fvm_handle *h, fvm_sim_params *p);
/* n steps back to back.  On a non-default stream the steps replay captured
 * CUDA graphs (two steps per graph, one-step graphs for an odd remainder and
 * for fvm_step); the first call that needs a graph kind captures it for both
 * ping-pong buffer parities, and a change of launch shape, dt policy, CFL
 * numbers, viscosity switches or stream captures them again. */
int fvm_steps(fvm_handle *h, fvm_sim_params *p, int n);
/* CFDSolver::computeStableTimeStep (src/solver.cu:3273-3278). */
int fvm_compute_dt(fvm_handle *h, const fvm_sim_params *p, float *dt_out);
/* CFDSolver::queueTimeStepComputation / readTimeStepResult (src/solver.cu:3206-3265).
 * fvm_queue_dt queues the reduction and its copy to host memory and returns;
 * fvm_read_dt reads that copy without waiting, so, as with the reference,
 * the stream must have been synchronized in between (fvm_synchronize). */
int fvm_queue_dt(fvm_handle *h, const fvm_sim_params *p);
int fvm_read_dt(fvm_handle *h, const fvm_sim_params *p, float *dt_out);
/* Block until this handle's stream is idle; reports a device error word. */
int fvm_synchronize(fvm_handle *h);

/* -------------------------------------------------------------- readback */
/* CFDSolver::getCellTypes (src/solver.cu:3432-3435). */
int fvm_get_cell_types(fvm_handle *h, uint8_t *host_types);
/* The signed-distance field, nx*ny floats (no reference accessor). */
int fvm_get_sdf(fvm_handle *h, float *host_sdf);
/* Conserved fields to/from host SoA buffers (the reference has no accessor;
 * its private d_rho_ ... d_rho_e_, src/include/solver.cuh:92-96).  Any pointer
 * may be NULL to skip that field.  fvm_write_fields recomputes primitives. */
int fvm_read_fields(fvm_handle *h, float *rho, float *rho_u, float *rho_v, float *E, float *rho_e);
/* The [i0, i0+w) x [j0, j0+hgt) window of the conserved fields into host
 * arrays of w*hgt floats (row-major; NULL skips a field), for probes and
 * windows of grids too large to copy whole.  No reference counterpart. */
int fvm_read_region(fvm_handle *h, int i0, int j0, int w, int hgt, float *rho, float *rho_u, float *rho_v, float *E,
                    float *rho_e);
/* The same window of the signed distance field (w*hgt floats) and of the
 * cell classes (w*hgt bytes, getCellTypes encoding); either may be NULL. */
int fvm_read_region_geometry(fvm_handle *h, int i0, int j0, int w, int hgt, float *sdf, uint8_t *cell_types);
int fvm_write_fields(fvm_handle *h, const float *rho, const float *rho_u, const float *rho_v,
                     const float *E, const float *rho_e);
/* Primitive fields u, v, p, T as left by the last step/reset (host). */
int fvm_read_primitives(fvm_handle *h, float *u, float *v, float *p, float *T);

/* Derived field into a device pointer (CFDSolver::compute*ToDevice,
 * src/solver.cu:3632-3671); kinds follow the reference's field selector. */
enum fvm_field_kind {
    FVM_FIELD_TEMPERATURE = 0,
    FVM_FIELD_PRESSURE = 1,
    FVM_FIELD_DENSITY = 2,
    FVM_FIELD_VELOCITY_MAG = 3,
    FVM_FIELD_MACH = 4
};
int fvm_field_to_device(fvm_handle *h, int kind, float *dev_dst);
/* Registers a display field (no reference counterpart; an extension for the
 * application's per-frame compute*ToDevice call): from the next step on, the
 * last passes of every step also write field `kind` of the new state into
 * dev_dst (nx*ny floats, the layout of fvm_field_to_device), the same values
 * a derived-field pass after the step writes.  fvm_field_to_device(kind,
 * dev_dst) then returns without a launch while the state is the one a step
 * left (writing fields, reset, obstacle updates, checkpoint loads and the
 * autotuner make it launch again).  dev_dst must stay valid while it is
 * registered; dev_dst == NULL unregisters, and so do fvm_initialize and
 * fvm_resize.  Changing the registration re-captures the step graphs. */
int fvm_set_display_field(fvm_handle *h, int kind, float *dev_dst);
/* CFDSolver::convertCellTypesToDevice (src/solver.cu:3452-3459). */
int fvm_cell_types_to_device(fvm_handle *h, float *dev_dst);
/* CFDSolver::generateVectorArrows (src/solver.cu:3809-3845); *n_vertices_out
 * receives the vertex count (the reference's return value). */
int fvm_vector_arrows(fvm_handle *h, float *dev_vertex_data, int max_vertices, int step,
                      float u_inf, float max_arrow_length, float arrow_head_angle,
                      float arrow_head_length, int *n_vertices_out);

/* ----------------------------------------------------------------- stats */
/* CFDSolver::getMaxTemperature / getMaxMach (src/solver.cu:3417-3426). */
int fvm_max_temperature(fvm_handle *h, float *out);
int fvm_max_mach(fvm_handle *h, float *out);
/* Number of (cell, step) pairs whose state came out of a step with a NaN or
 * infinite field, counted on the device inside the steps' CFL reductions
 * since the solve was (re)initialised or the counter was last reset
 * (reset != 0 clears it after reading).  The reference has no such check: its
 * update rolls non-finite results back to the old value, which repairs most
 * of them but not all (a non-finite input field, viscous terms).  No
 * reference counterpart. */
int fvm_nonfinite_count(fvm_handle *h, unsigned long long *count, int reset);
/* CFDSolver::getSimulationMemoryUsage (src/solver.cu:3474-3514): bytes this handle holds. */
int fvm_memory_usage(fvm_handle *h, size_t *bytes);
/* CFDSolver::getGPUMemoryInfo (src/solver.cu:3468-3471): (free, total), the
 * implementation's positional order. */
int fvm_gpu_mem_info(size_t *free_bytes, size_t *total_bytes);

/* FP64 diagnostics reduced on the device (no reference counterpart).
 * Forces act on the obstacle per unit span; coefficients use
 * q_inf = 0.5*rho_inf*u_inf^2 and ref_length. */
typedef struct fvm_diag {
    double force_x, force_y;      /* pressure + viscous wall force [N/m] */
    double cd, cl;                /* force coefficients */
    double mass, mom_x, mom_y, energy;   /* totals over non-solid cells [per m span] */
    double wall_heat;             /* integrated wall heat flux into the wall [W/m] */
    double wall_heat_max;         /* peak wall heat flux [W/m^2] */
    double reserved[6];
} fvm_diag;
int fvm_diagnostics(fvm_handle *h, fvm_diag *out);

/* Shock standoff along row j = ny/2: distance between the shock (pressure
 * crossing halfway from p_inf to the normal-shock pressure) and the obstacle
 * surface (sdf zero crossing), both upstream of the obstacle [m]. */
int fvm_shock_standoff(fvm_handle *h, double *standoff_out);

/* Kernel time accounting for measurement: when enabled, each launch on the
 * handle's stream is bracketed by CUDA events.  fvm_kernel_times fills up to
 * `cap` entries {name, launches, total_ms} for kernels launched since the
 * last reset of the counters. */
typedef struct fvm_kernel_time {
    char name[48];
    long long launches;
    double total_ms;
} fvm_kernel_time;
int fvm_set_kernel_timing(fvm_handle *h, int enable);
int fvm_kernel_times(fvm_handle *h, fvm_kernel_time *out, int cap, int *count_out);

/* Autotuner: times every candidate launch tuning of the marching step
 * kernels (threads per CTA 128/256, TMA ring depth 4/6 rows, rows per CTA
 * 4..256) over `steps` steps of this solve, restoring the state after each,
 * keeps the fastest for this handle and caches it for the grid class (grid
 * size, viscous flag, flux scheme, limiter) for later handles in the process.
 * *best_ms_out receives the winner's time per step. */
int fvm_autotune(fvm_handle *h, const fvm_sim_params *p, int steps, float *best_ms_out);
/* The launch tuning in use. */
int fvm_get_tune(fvm_handle *h, int *nt, int *ring, int *rows);
/* Pin a launch tuning (e.g. one an earlier fvm_autotune chose): threads per
 * CTA 128 or 256, ring depth 4 or 6 rows, an even number of rows per CTA in
 * 4..65536.  Results are bitwise the same under every allowed tuning; only the
 * speed differs.  (Tiles start on even rows, so a row always takes the same
 * place in the row pair the kernels evaluate together; the two places are
 * separately compiled code and may round differently in the last bit.) */
int fvm_set_tune(fvm_handle *h, int nt, int ring, int rows);

/* ------------------------------------------------------------ batches
 * Many independent solves (different grids, Mach numbers, obstacles, Euler
 * or Navier-Stokes) advanced together: each batched step is one persistent
 * launch per stage over a tile list spanning every instance, replayed as one
 * CUDA graph.  Every instance keeps its own time step (the ext's dt policy;
 * FVM_DT_RECOMPUTE gives each its own CFL dt).  No reference counterpart. */
typedef struct fvm_batch fvm_batch;
int fvm_batch_create(fvm_batch **out, const fvm_ext *ext);
int fvm_batch_destroy(fvm_batch *b);
int fvm_batch_set_stream(fvm_batch *b, void *stream);
/* Allocate and reset one instance (as fvm_initialize); *id_out is its id. */
int fvm_batch_add(fvm_batch *b, const fvm_sim_params *p, int *id_out);
int fvm_batch_remove(fvm_batch *b, int id);
int fvm_batch_count(fvm_batch *b, int *n);
/* n batched steps (every instance advances n steps). */
int fvm_batch_step(fvm_batch *b, int n);
int fvm_batch_synchronize(fvm_batch *b);
/* Instance parameters with its t_current, step and last dt. */
int fvm_batch_instance(fvm_batch *b, int id, fvm_sim_params *p_out);
int fvm_batch_read_fields(fvm_batch *b, int id, float *rho, float *rho_u, float *rho_v, float *E, float *rho_e);
int fvm_batch_diagnostics(fvm_batch *b, int id, fvm_diag *out);
/* The instance's non-finite (cell, step) count (fvm_nonfinite_count) since it
 * was added or reset for its current solve.  No reference counterpart. */
int fvm_batch_nonfinite_count(fvm_batch *b, int id, unsigned long long *count);
int fvm_batch_memory_usage(fvm_batch *b, size_t *bytes);
int fvm_batch_launch_count(fvm_batch *b, long long *count_out);
/* Device bytes one instance of nx*ny holds (admission estimate). */
size_t fvm_batch_instance_bytes(int nx, int ny);
/* Take an instance out of the batch but keep its device memory: a later
 * fvm_batch_add of the same grid size resets it in place instead of
 * allocating.  fvm_batch_remove frees the memory instead. */
int fvm_batch_retire(fvm_batch *b, int id);
/* Free retired instances (oldest first) until at most keep_bytes remain
 * parked; *parked_bytes_out (may be NULL) receives what stays parked. */
int fvm_batch_trim(fvm_batch *b, size_t keep_bytes, size_t *parked_bytes_out);

/* ------------------------------------------------------------ serving
 * A request loop over one batch (continuous batching).  Solve requests are
 * submitted from any host thread and queue in arrival order; a worker thread
 * admits them into the batch as instance slots and the device-memory budget
 * allow (first come first served; a request larger than the whole budget is
 * rejected with FVM_ERR_BUDGET), advances all admitted solves together in
 * chunks of batched steps, and retires each one after its requested steps:
 * its final state goes to the caller's host arrays (if given), its
 * diagnostics into the result.  Each request's result equals the same solve
 * run alone.  No reference counterpart. */
typedef struct fvm_server fvm_server;
typedef struct {
    long long ticket;
    int status;        /* FVM_OK, FVM_ERR_BUDGET, FVM_ERR_NONFINITE (a step produced a NaN or
                          infinite cell, or the final diagnostics are not finite) or the
                          error that ended it */
    int steps;         /* steps taken */
    int nx, ny;
    float t_final;     /* simulated time after the last step */
    float dt_last;     /* time step of the last step */
    double submit_s, admit_s, done_s; /* host clock, seconds since the server was created */
    fvm_diag diag;     /* diagnostics of the final state */
} fvm_result;
typedef struct {
    long long submitted, completed, rejected, batched_steps;
    int active, pending;
    size_t budget_bytes, active_bytes, parked_bytes;
    double cell_updates;  /* cells x steps advanced */
    double busy_s;        /* device time of the batched steps */
    double step_ms_p50, step_ms_p99, step_ms_mean; /* device time per batched step */
    double reserved[4];
} fvm_server_stats;
/* hbm_budget_bytes: device memory the admitted solves may hold (estimated by
 * fvm_batch_instance_bytes); max_active: instance slots (0 = no limit);
 * max_chunk_steps: most batched steps between admission checks (0 = 64).
 * The worker uses the device current at creation. */
int fvm_server_create(fvm_server **out, const fvm_ext *ext, size_t hbm_budget_bytes, int max_active,
                      int max_chunk_steps);
/* Queue a solve of `steps` steps from the freestream start of *p.  The five
 * host arrays (nx*ny floats each, any may be NULL) receive the final state;
 * they must stay valid until the result is collected. */
int fvm_server_submit(fvm_server *s, const fvm_sim_params *p, int steps, float *rho, float *rho_u, float *rho_v,
                      float *E, float *rho_e, long long *ticket_out);
/* Collect up to cap finished results (completion order); *n_out receives how many. */
int fvm_server_poll(fvm_server *s, fvm_result *out, int cap, int *n_out);
/* Wait for one request's result (timeout_s < 0: no limit); FVM_ERR_TIMEOUT if it did not finish in time. */
int fvm_server_wait(fvm_server *s, long long ticket, double timeout_s, fvm_result *out);
/* Wait until every submitted request has finished (timeout_s < 0: no limit). */
int fvm_server_drain(fvm_server *s, double timeout_s);
int fvm_server_get_stats(fvm_server *s, fvm_server_stats *out);
/* Stop the worker (requests not yet finished end with FVM_ERR_STATE) and free everything. */
int fvm_server_destroy(fvm_server *s);

/* ------------------------------------------------------------ no allocation
 * Maximum temperature (what = 0) or local Mach number (what = 1) of a state
 * held in the caller's device memory: five float planes (rho, rho*u, rho*v,
 * E, rho*e) of ny rows by nx cells, `pitch` floats between rows and `plane`
 * floats between planes.  *out (host memory) receives the maximum; the call
 * returns when it is there.  No counterpart in the reference, which only
 * reduces its own solver state (getMaxTemperature, src/solver.cu:2835-2867).
 *
 * Allocates nothing, for callers that may not allocate device memory at the
 * point of the call (memory committed up front to solve instances, no handle
 * to create): the reduction scratch is a fixed array inside the library,
 * enough for ny <= 16384 rows; a larger ny is rejected with FVM_ERR_INVALID
 * before anything runs.  The array's device address is looked up
 * (cudaGetSymbolAddress) on the first call in each CUDA context and again
 * whenever the current context changes (after cudaDeviceReset, say).  Every
 * call clears the array's arrival counter, launches one kernel, copies the
 * result to *out and synchronizes `stream`, so it cannot run on a stream that
 * is being captured: it then returns FVM_ERR_STATE and does nothing.  All
 * calls on one device share the array and it keeps the last call's
 * contents, so calls must not overlap on the GPU: do not call it from two
 * host threads at once for the same device. */
int fvm_state_max_noalloc(const float *state, int nx, int ny, size_t pitch, size_t plane, int what, float *out,
                          void *stream);

/* ------------------------------------------------------------ colour images
 * Headless form of the renderer's field pass (src/renderer.cpp:47-77 and the
 * colour tables of src/renderer.cpp:672-799, enum ColormapType of
 * src/include/renderer.h:14-21): one RGBA pixel per cell, row j of the image
 * = grid row j (bottom row first, as the reference uploads its texture).
 * SOLID and GHOST cells are dark grey (0.3); other cells show the derived
 * field `field_kind` (enum fvm_field_kind) normalised by
 * (v - min_val) / (max_val - min_val + 1e-4), clamped to [0, 1], looked up in
 * the table as a linearly filtered, edge-clamped 1-D texture would.  No
 * graphics API is involved. */
enum fvm_colormap { FVM_CMAP_JET = 0, FVM_CMAP_HOT = 1, FVM_CMAP_PLASMA = 2, FVM_CMAP_INFERNO = 3, FVM_CMAP_VIRIDIS = 4 };
enum fvm_pixel_format {
    FVM_RGBA_F32 = 0,  /* 4 floats per pixel in [0, 1] */
    FVM_RGBA_U8 = 1    /* 4 bytes per pixel, round(clamp(c) * 255) */
};
/* Image into a device buffer of nx*ny pixels (enqueued on the handle's stream). */
int fvm_colormap_to_device(fvm_handle *h, int field_kind, int colormap, float min_val, float max_val,
                           void *dev_rgba, int format);
/* The 256-entry RGB table of a colormap (768 floats, host). */
int fvm_colormap_table(int colormap, float *rgb_out);

/* ------------------------------------------------------------ checkpoints
 * Save / restore a solve to a file: a 256-byte header (magic "FVMB200C",
 * version 1, grid, the solve's parameters and extension knobs, the next
 * step's dt, the device simulated time and the last step's CFL maxima) and
 * the five conserved fields as nx*ny float32 planes (fvm_read_fields layout),
 * with a CRC-32 of the fields in the header.  Loading re-initialises the
 * handle from the saved parameters and continues bit for bit where the saved
 * solve would have.  No reference counterpart (the reference has no
 * checkpoints). */
int fvm_save_checkpoint(fvm_handle *h, const fvm_sim_params *p, const char *path);
/* *p_out (may be NULL) receives the saved parameters (t_current, step, dt). */
int fvm_load_checkpoint(fvm_handle *h, const char *path, fvm_sim_params *p_out);
/* Validate a checkpoint file (header and checksum) without a handle or a
 * device; *p_out / *ext_out (may be NULL) receive its parameters. */
int fvm_checkpoint_info(const char *path, fvm_sim_params *p_out, fvm_ext *ext_out);

/* ------------------------------------------------------------ analysis
 * Vortex-shedding statistics of a force-coefficient history (samples at
 * strictly increasing times t; cd, cl from fvm_diagnostics), for the
 * Strouhal number of a cylinder wake.  Whole cycles between the first and
 * last upward zero crossing of cl - mean(cl) give the period, St =
 * ref_length / (period * u_inf), and the cycle-averaged drag and lift.
 * Host code, no device work.  No reference counterpart. */
typedef struct {
    double strouhal, period, cd_mean, cl_mean, cl_rms;
    int cycles;    /* whole shedding cycles used */
    int reserved;
} fvm_shedding;
int fvm_shedding_stats(const double *t, const double *cd, const double *cl, int n, double ref_length, double u_inf,
                       fvm_shedding *out);

/* Count of kernels this library launched on the handle since creation. */
int fvm_launch_count(fvm_handle *h, long long *count_out);

/* Test hook: run stage 1 of the next step (inviscid stage kernel, and the
 * ghost-cell pass when with_ghost != 0) from the current state with dt and
 * copy U* to the five host arrays (nx*ny each).  The state is not advanced. */
int fvm_debug_stage1(fvm_handle *h, float dt, int with_ghost, float *rho, float *rho_u, float *rho_v, float *E,
                     float *rho_e);

/* Test hook: copy the ghost-cell table (7 ints per ghost cell: pitched index
 * j*pitch+i (grids below 2^31 cells), i, j, normal x and y as float bits,
 * packed candidate codes, count) to
 * `out` (cap entries); *count_out receives the number of ghost cells. */
int fvm_debug_ghost_table(fvm_handle *h, int *out, int cap, int *count_out);

/* Test hook for the failure path of the kernels' bounded waits: launches one
 * warp that waits on a barrier nothing completes, so its wait gives up after
 * limit_cycles SM cycles (1..4e9; two million is about a millisecond) and sets
 * the timeout bit of this solve's device error word.  Returns the status a
 * step would then report (FVM_ERR_TIMEOUT), clears the error word and leaves
 * the solve's state untouched and usable.  No reference counterpart. */
int fvm_debug_wait_timeout(fvm_handle *h, long long limit_cycles);

/* Library build description (arch, flags). */
const char *fvm_build_info(void);

#ifdef __cplusplus
}
#endif

#endif /* FVM_B200_H */
