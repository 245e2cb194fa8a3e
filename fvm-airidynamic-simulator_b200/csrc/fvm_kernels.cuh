// fvm_kernels.cuh -- host-side launch interface of the library's kernels.
#pragma once
#include "fvm_internal.cuh"

namespace fvm {

struct ShapeParamsHost {
    float ox, oy, r, rot, wing, cone_ang, cone_len;
    int shape;
};

// Launch configuration of the marching stage kernels (chosen per grid class
// by the tuner): threads per CTA (= columns of primitives staged per row),
// TMA ring depth and rows marched per CTA.
struct StageTune {
    int nt;          // 128 or 256
    int ring;        // TMA ring slots (prefetch distance = ring - 3)
    int rows;        // rows per CTA
};

// geometry (fvm_geometry.cu)
void launch_sdf(const GridDesc &g, const ShapeParamsHost &s, float *sdf, uint8_t *ct, float *fix_state,
                cudaStream_t st);
void launch_mask(const GridDesc &g, const uint8_t *ct, uint8_t *mask, cudaStream_t st);
void launch_ghost_table(const GridDesc &g, const float *sdf, const uint8_t *ct, GhostInfo *list, int cap, int *count,
                        cudaStream_t st);
void launch_init(const GridDesc &g, float *U, const Freestream &fs, cudaStream_t st);

// step kernels (fvm_step.cu)
// Inviscid RK stage: stage 1 writes U* from U; stage 2 writes
// 0.5*B + 0.5*(U** from U*).  Optional phase-1 BC and CFL reduction.
cudaError_t launch_stage(int stage, int scheme, int limiter, const StageTune &tn, const CUtensorMap &tm_in,
                         const CUtensorMap &tm_blend, const StepArgs &a, cudaStream_t st);
// Viscous half step out of place: out = U + dt*D(prims(U)) on interior fluid
// cells, copy elsewhere; optional phase-1 BC and CFL reduction.
cudaError_t launch_viscous(const StageTune &tn, const CUtensorMap &tm_in, const StepArgs &a, cudaStream_t st);
// Batched launches over a multi-instance tile list (persistent grids).
// early: let the next kernel launch before this grid drains (a ghost pass
// follows); pdl: launch with programmatic stream serialization
cudaError_t launch_stage_batch(int stage, int scheme, int limiter, const StageTune &tn, const BatchInst *insts,
                               const TileDesc *tiles, int ntiles, int early, bool pdl, cudaStream_t st);
cudaError_t launch_viscous_batch(const StageTune &tn, const BatchInst *insts, const TileDesc *tiles, int ntiles,
                                 int post, cudaStream_t st);
cudaError_t launch_ghost_batch(const BatchInst *insts, const GhostChunk *chunks, int nchunks, int mode,
                               cudaStream_t st);
// Ghost-cell pass over the ghost table.
cudaError_t launch_set_display(DisplayDesc *d, float *ptr, int kind, cudaStream_t st);
cudaError_t launch_ghost(const GhostArgs &a, cudaStream_t st);
// Bounded wait on an mbarrier nothing arrives on (expires after limit_cycles).
cudaError_t launch_wait_probe(DevScalars *sc, long long limit_cycles, cudaStream_t st);
// Phase-1 boundary conditions in place on a whole state (set-up path).
cudaError_t launch_bc_phase1(const GridDesc &g, float *U, const uint8_t *mask, const Freestream &fs, cudaStream_t st);
// CFL maxima of a state (speed over all cells; nu = mu(T)/rho, mu = 0 in solids),
// accumulated into sc->red, then published to sc->cfl by a one-block finalize.
cudaError_t launch_cfl_state(const GridDesc &g, const float *U, const uint8_t *mask, DevScalars *sc, cudaStream_t st);
// Set the dynamic shared-memory attribute of every step kernel of a tuning.
cudaError_t prepare_step_kernels(const StageTune &tn);
// Shared-memory bytes a stage / viscous kernel needs for a tuning.
size_t stage_smem_bytes(int stage, const StageTune &tn);
size_t viscous_smem_bytes(const StageTune &tn);
int stage_cols_per_cta(const StageTune &tn);   // output columns per CTA
int stage_box_in(const StageTune &tn);         // TMA box width of the halo'd input
int stage_box_blend(const StageTune &tn);      // TMA box width of the blend partner

// auxiliary kernels (fvm_aux.cu)
cudaError_t launch_primitives(const GridDesc &g, const float *U, float *u, float *v, float *p, float *T,
                              cudaStream_t st);  // dense nx*ny outputs
cudaError_t launch_derived(int kind, const GridDesc &g, const float *U, float *dst, cudaStream_t st);
// 256-entry RGB colour table, passed to the kernel by value.
struct ColormapLUT {
    float rgb[256 * 3];
};
cudaError_t launch_colormap(int kind, const GridDesc &g, const float *U, const uint8_t *ct, const ColormapLUT &lut,
                            float lo, float hi, void *out, int fmt, cudaStream_t st);
cudaError_t launch_ct_to_float(const GridDesc &g, const uint8_t *ct, float *dst, cudaStream_t st);
cudaError_t launch_max_reduce(int what, const GridDesc &g, const float *U, float *out_dev, cudaStream_t st);
cudaError_t launch_arrows_cap(const GridDesc &g, const float *U, float *vertex, int cap, int *counter, int step,
                              float u_inf, float max_len, float head_angle, float head_len, cudaStream_t st);
cudaError_t launch_diagnostics(const GridDesc &g, const float *U, const uint8_t *ct, const uint8_t *mask,
                               int viscous, float prandtl, int ref_prandtl, double *partials, int nparts,
                               double *out8, cudaStream_t st);
int diagnostics_parts(const GridDesc &g);
cudaError_t launch_standoff(const GridDesc &g, const float *U, const float *sdf, double p_mid, double *out,
                            cudaStream_t st);

}  // namespace fvm
