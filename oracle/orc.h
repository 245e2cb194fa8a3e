/*
 * orc.h -- CPU oracle for the compressible-flow hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * solver's per-step kernel chain (reference: src/solver.cu) used as the
 * checker for the CUDA library.  Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg may load it; the product never does.
 *
 * One source, two builds: ORC_REAL=double (liborc64.so, the FP64 oracle) and
 * ORC_REAL=float (liborc32.so, IEEE float without contraction).
 *
 * Semantics that the reference leaves undefined are fixed here and in the
 * CUDA library identically:
 *   - boundary conditions run in two phases.  Phase 1 applies the pointwise
 *     conditions (inflow, outflow NRBC, bottom/top NRBC, solid).  Phase 2
 *     fills ghost cells reading a snapshot taken after phase 1, in which ghost
 *     cells still hold their values from before the call.  The reference
 *     kernel (src/solver.cu:1891-2226) does both in one pass in place, so a
 *     ghost cell whose best neighbour is another ghost cell reads either value
 *     depending on scheduling.
 */
#ifndef ORC_H
#define ORC_H
#include <stdint.h>
#include "../include/fvm_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_solver orc_solver;

orc_solver *orc_create(int nx, int ny);
void orc_destroy(orc_solver *s);
int orc_real_size(void); /* sizeof(ORC_REAL) of this build */
int orc_set_threads(int n);

/* The reference's SimParams defaults and computeDerived
 * (src/include/common.h:53-101) and the extension defaults, in float. */
void orc_params_default(fvm_sim_params *p);
void orc_params_compute_derived(fvm_sim_params *p);
void orc_ext_default(fvm_ext *e);

/* Copy the parameter block (float SimParams layout + extension knobs). */
void orc_set_params(orc_solver *s, const fvm_sim_params *p, const fvm_ext *e);
/* initializeKernel + computeSDFKernel + BC + primitives + viscosity field. */
void orc_reset(orc_solver *s);
/* Replace the geometry (sdf + cell types) by externally supplied arrays (used
 * to share a device-computed SDF); the flow state is not touched. */
void orc_set_geometry(orc_solver *s, const float *sdf, const uint8_t *ct);
/* Freestream + BC + primitives + viscosity field on the current geometry. */
void orc_reinit(orc_solver *s);
/* SDF + cell marking only, into caller buffers (float sdf, uint8 types). */
void orc_compute_sdf(orc_solver *s, float *sdf_out, uint8_t *ct_out);
/* updateSDFWithFixupKernel + BC + primitives. */
void orc_update_obstacle(orc_solver *s);

/* One SSP-RK2 step with time step dt. */
void orc_step(orc_solver *s, double dt);
/* CFL time step from the current state (computeStableTimeStep). */
double orc_compute_dt(orc_solver *s);
/* Max wave speed and max kinematic viscosity (the two CFL reductions). */
void orc_cfl_maxima(orc_solver *s, double *max_speed, double *max_nu);

/* Field access as double arrays (nx*ny each; NULL skips). */
void orc_get_fields(orc_solver *s, double *rho, double *ru, double *rv, double *E, double *re);
void orc_set_fields(orc_solver *s, const double *rho, const double *ru, const double *rv,
                    const double *E, const double *re);
void orc_get_primitives(orc_solver *s, double *u, double *v, double *p, double *T);
void orc_get_mu(orc_solver *s, double *mu);
void orc_get_geometry(orc_solver *s, double *sdf, uint8_t *ct);

/* Stage-level entry points (for localising differences). */
void orc_stage1(orc_solver *s, double dt, int with_ghost, double *out5[5]);

/* Diagnostics with the same definitions as the device reductions. */
void orc_diagnostics(orc_solver *s, fvm_diag *out);
double orc_shock_standoff(orc_solver *s);

/* Colour images (test infrastructure for fvm_colormap_to_device): the
 * renderer's 256-entry colour tables (src/renderer.cpp:672-799) and the field
 * fragment shader (src/renderer.cpp:47-77) restated on the CPU in float.
 * field: n derived values; ct: n cell classes; fmt 0 -> n*4 floats,
 * fmt 1 -> n*4 bytes. */
void orc_colormap_table(int cmap, float rgb[768]);
void orc_colormap(const float *field, const uint8_t *ct, long n, int cmap, float lo, float hi, int fmt, void *out);

#ifdef __cplusplus
}
#endif
#endif
