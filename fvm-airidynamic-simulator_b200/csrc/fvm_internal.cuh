// fvm_internal.cuh -- device data layout and kernel launch interface shared
// by the library's translation units.  Not part of the public C ABI.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda.h>
#include <cuda_runtime.h>

#include "fvm_math.cuh"

namespace fvm {

// A solve's grid.  Fields are SoA float planes of ny rows x `pitch` floats
// (pitch = nx rounded up to 32, so every row starts 128-byte aligned); the 5
// conserved planes of one state (rho, rho_u, rho_v, E, rho_e) are contiguous,
// plane k at base + k*plane.
struct GridDesc {
    int nx, ny;
    int pitch;
    long long plane;
    float dx, dy;
};

// Static per-ghost-cell data, built once per geometry: pitched cell index,
// unit SDF normal, and the candidate fluid neighbours in the order the
// reference's best-neighbour search would prefer them (descending dot with
// the normal, ties to the earlier neighbour; src/solver.cu:2068-2098).
// Candidate nibble k: bits 0-2 neighbour code in the reference order
// {(-1,0),(1,0),(0,-1),(0,1),(-1,-1),(1,-1),(-1,1),(1,1)}, bit 3 set when the
// neighbour is itself a ghost cell.
struct GhostInfo {  // the pitched index is j * pitch + i, formed in 64 bits where used
    int i, j;
    float gx, gy;
    uint32_t cand;
    int count;
};

// Device-resident scalars of one solve.
struct DevScalars {
    float red[2];     // running maxima of the fused CFL reduction (speed, nu)
    float cfl[2];     // maxima of the last completed step
    float dt;         // dt the next step uses (read by the step kernels)
    float t;          // simulated time (advanced on the device under recompute)
    unsigned counter; // last-block counter of the ghost pass
    unsigned err;        // error word (kErrTimeout, kErrSmemAlign)
    unsigned nonfinite;  // (cell, step) pairs with a non-finite new state
    float dt_last;    // dt of the last completed step (recompute policy)
    unsigned parity;  // batched solves: which ping-pong buffer holds U^n
    unsigned pad;
    double diag[16];  // FP64 diagnostic accumulators
};

// compute{Temperature,Pressure,VelocityMag,Mach}DirectKernel and the density
// copy (src/solver.cu:3527-3671): the derived value of one cell (kind =
// FVM_FIELD_*).  Used by the derived-field pass and, for a registered display
// field, by the last passes of a step.
__device__ __forceinline__ float derived_value(int kind, float rho, float rho_u, float rho_v, float rho_e) {
    // the quotients by rho + 1e-10 share one approximate reciprocal (the one
    // the fast-math division multiplies by)
    const float irv = rcp_approx(rho + 1e-10f);
    switch (kind) {
    case 0: return (GAMMA - 1.0f) * (rho_e * irv) * (1.0f / R_GAS);
    case 1: return (GAMMA - 1.0f) * rho_e;
    case 2: return rho;
    case 3: {
        const float u = rho_u * irv, v = rho_v * irv;
        return sqrtf(u * u + v * v);
    }
    default: {
        const float u = rho_u * irv, v = rho_v * irv;
        const float speed = sqrtf(u * u + v * v);
        const float T = (GAMMA - 1.0f) * (rho_e * irv) * (1.0f / R_GAS);
        const float cs = sqrtf(GAMMA * R_GAS * T);
        return speed * rcp_approx(cs + 1e-10f);
    }
    }
}

// A registered display field of one solve: the destination of the derived
// field the last passes of every step write (null: none), read by the
// kernels at run time so that captured step graphs stay valid when the
// application registers another buffer.
struct DisplayDesc {
    float *ptr;
    int kind;
    int pad;
};

// Step-kernel arguments common to all stage kernels.
struct StepArgs {
    GridDesc g;
    float *out;            // output state (5 planes)
    const uint8_t *mask;   // pitched mask bytes (pitch bytes per row)
    DevScalars *sc;        // dt / reductions / error word
    Freestream fs;
    WallParams wall;
    float prandtl;
    int ref_prandtl;
    int rows_per_cta;
    int apply_bc;          // phase-1 boundary conditions on the output
    int cfl;               // 0: none, 1: wave speed, 2: wave speed + kinematic viscosity
    float dt_scale;        // stage dt = sc->dt * dt_scale (0.5 for the viscous half steps)
    const DisplayDesc *disp;  // last pass of a step: display field of the output (dense nx*ny), or null
    int early_launch;         // let the next kernel (a ghost pass) launch before this grid drains
    int pdl;                  // host: launch with programmatic stream serialization
};

struct GhostArgs {
    GridDesc g;
    const GhostInfo *list;
    int n;
    float *A;              // phase-1 state: non-ghost neighbours read here, ghost cells written here
    const float *B1;       // pre-BC ghost values: B2 ? 0.5*B1 + 0.5*B2 : B1
    const float *B2;
    DevScalars *sc;
    Freestream fs;
    WallParams wall;
    int cfl;               // 0: none, 1: speed, 2: speed + nu (T from the pre-BC ghost state)
    int finalize;          // last block publishes the step's CFL maxima and next dt
    int recompute_dt;
    float cfl_num, cfl_visc, min_dx;
    int viscous;
    int flip_parity;       // batched solves: toggle sc->parity in the finalize
    const DisplayDesc *disp;  // display field of the ghost cells written (dense nx*ny), or null
};

// ---------------------------------------------------------- batched solves
// Buffer roles of a solve's state buffers.  Physical buffers 0 and 2 hold
// U^n / U^{n+1} alternately (DevScalars::parity), 1 holds U*, 3 holds
// U_d / U_b of the viscous path.
enum { ROLE_N = 0, ROLE_S = 1, ROLE_X = 2, ROLE_D = 3 };

// Per-instance descriptor of a batch (device memory; TMA maps must be 64-byte
// aligned).
struct alignas(64) BatchInst {
    CUtensorMap tm_in[4];   // halo'd row boxes, per physical buffer
    CUtensorMap tm_ctr[4];  // blend-partner boxes, per physical buffer
    float *buf[4];
    GridDesc g;
    const uint8_t *mask;
    DevScalars *sc;
    Freestream fs;
    WallParams wall;
    float prandtl;
    int ref_prandtl;
    int viscous;
    const GhostInfo *ghosts;
    int n_ghost;
    int n_gchunks;
    int recompute_dt;
    float cfl_num, cfl_visc, min_dx;
};

struct TileDesc {
    int inst, i0, j0, pad;
};

struct GhostChunk {
    int inst, first, count, pad;
};

}  // namespace fvm
