// ref_harness.cu -- C entry points around the UNMODIFIED reference solver
// (reference: src/solver.cu, src/include/solver.cuh) for parity checks.
// TEST INFRASTRUCTURE ONLY: built by oracle/build_ref.sh into oracle/_ref/,
// loaded by tests/ on a GPU box as the reference FP32 CUDA oracle.
//
// The reference keeps its device fields private and has no readback API, so
// this translation unit opens the class with `#define private public` around
// the header include and copies d_rho_ ... d_rho_e_, d_sdf_, d_cell_type_ and
// the primitives out.  No reference file is edited.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <iostream>
#include <iomanip>
#include <vector>
#include <cuda_runtime.h>

#define private public
#include "solver.cuh"
#undef private

extern "C" {

int ref_sizeof_params(void) { return (int)sizeof(SimParams); }

// CFDSolver::initialize + reset (initialize already resets)
void *ref_create(const SimParams *p) {
    CFDSolver *s = new CFDSolver();
    s->initialize(*p);
    cudaDeviceSynchronize();
    return s;
}

void ref_destroy(void *h) { delete static_cast<CFDSolver *>(h); }

// n calls of CFDSolver::step with the dt in *p (fixed-dt policy, like
// KernelBenchmark).  With recompute != 0, dt is recomputed from the state
// before every step (computeStableTimeStep), like the app's per-frame loop
// with one step per frame.
int ref_steps(void *h, SimParams *p, int n, int recompute) {
    CFDSolver *s = static_cast<CFDSolver *>(h);
    for (int k = 0; k < n; k++) {
        if (recompute) p->dt = s->computeStableTimeStep(*p);
        s->step(*p);
    }
    return (int)cudaDeviceSynchronize();
}

float ref_compute_dt(void *h, const SimParams *p) {
    return static_cast<CFDSolver *>(h)->computeStableTimeStep(*p);
}

static void d2h(float *dst, const float *src, size_t n) {
    if (dst) cudaMemcpy(dst, src, n * sizeof(float), cudaMemcpyDeviceToHost);
}

void ref_read_fields(void *h, float *rho, float *ru, float *rv, float *E, float *re) {
    CFDSolver *s = static_cast<CFDSolver *>(h);
    size_t n = (size_t)s->_nx * s->_ny;
    d2h(rho, s->d_rho_, n);
    d2h(ru, s->d_rho_u_, n);
    d2h(rv, s->d_rho_v_, n);
    d2h(E, s->d_E_, n);
    d2h(re, s->d_rho_e_, n);
}

void ref_write_fields(void *h, const float *rho, const float *ru, const float *rv, const float *E, const float *re) {
    CFDSolver *s = static_cast<CFDSolver *>(h);
    size_t n = (size_t)s->_nx * s->_ny * sizeof(float);
    cudaMemcpy(s->d_rho_, rho, n, cudaMemcpyHostToDevice);
    cudaMemcpy(s->d_rho_u_, ru, n, cudaMemcpyHostToDevice);
    cudaMemcpy(s->d_rho_v_, rv, n, cudaMemcpyHostToDevice);
    cudaMemcpy(s->d_E_, E, n, cudaMemcpyHostToDevice);
    cudaMemcpy(s->d_rho_e_, re, n, cudaMemcpyHostToDevice);
    // step() expects the primitives (and mu) of the current state, as left
    // by reset or by the previous step (src/solver.cu:3291-3293, :3148-3158)
    s->launchComputePrimitivesKernel(s->d_rho_, s->d_rho_u_, s->d_rho_v_, s->d_E_, s->d_rho_e_, s->d_u_, s->d_v_,
                                     s->d_p_, s->d_T_, s->_nx, s->_ny);
    s->launchFusedViscousDiffusionKernel(s->d_u_, s->d_v_, s->d_T_, s->d_mu_, s->d_rho_u_, s->d_rho_v_, s->d_E_,
                                         s->d_rho_e_, s->d_cell_type_, 0.0f, 1.0f, 1.0f, s->_nx, s->_ny);
    cudaDeviceSynchronize();
}

void ref_read_primitives(void *h, float *u, float *v, float *p, float *T) {
    CFDSolver *s = static_cast<CFDSolver *>(h);
    size_t n = (size_t)s->_nx * s->_ny;
    d2h(u, s->d_u_, n);
    d2h(v, s->d_v_, n);
    d2h(p, s->d_p_, n);
    d2h(T, s->d_T_, n);
}

void ref_read_geometry(void *h, float *sdf, uint8_t *ct) {
    CFDSolver *s = static_cast<CFDSolver *>(h);
    size_t n = (size_t)s->_nx * s->_ny;
    d2h(sdf, s->d_sdf_, n);
    if (ct) cudaMemcpy(ct, s->d_cell_type_, n, cudaMemcpyDeviceToHost);
}

float ref_max_temperature(void *h) { return static_cast<CFDSolver *>(h)->getMaxTemperature(); }
float ref_max_mach(void *h) { return static_cast<CFDSolver *>(h)->getMaxMach(); }

void ref_update_obstacle(void *h, const SimParams *p) {
    static_cast<CFDSolver *>(h)->updateObstacleGeometry(*p);
    cudaDeviceSynchronize();
}

// Mean device time of one CFDSolver::step over `steps` steps after `warmup`,
// timed with CUDA events on the default stream the reference launches on.
float ref_time_steps(void *h, SimParams *p, int warmup, int steps) {
    CFDSolver *s = static_cast<CFDSolver *>(h);
    for (int k = 0; k < warmup; k++) s->step(*p);
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, 0);
    for (int k = 0; k < steps; k++) s->step(*p);
    cudaEventRecord(b, 0);
    cudaEventSynchronize(b);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return steps > 0 ? ms / steps : 0.0f;
}

}  // extern "C"
