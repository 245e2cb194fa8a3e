// fvm_handle.h -- the solve handle behind the C ABI (internal).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <map>
#include <string>
#include <vector>

#include "../../include/fvm_b200.h"
#include "fvm_kernels.cuh"

using namespace fvm;

// Buffer slots of a handle (physical order at creation: U^n, U*, U^{n+1}, U_d/U_b).
enum { BUF_N = 0, BUF_S = 1, BUF_X = 2, BUF_D = 3, NBUF = 4 };

struct TimedLaunch {
    int kernel;
    cudaEvent_t a, b;
};

struct fvm_handle {
    int device = 0;
    cudaStream_t own = nullptr;
    cudaStream_t stream = nullptr;
    fvm_sim_params prm{};
    fvm_ext ext{};
    GridDesc g{};
    float *buf[NBUF] = {nullptr, nullptr, nullptr, nullptr};
    float *&Un = buf[BUF_N];
    CUtensorMap tm_in[NBUF];
    CUtensorMap tm_ctr[NBUF];
    float *sdf = nullptr;     // pitched
    uint8_t *ct = nullptr;    // dense nx*ny (reference layout)
    uint8_t *mask = nullptr;  // pitched
    GhostInfo *ghosts = nullptr;
    int n_ghost = 0, ghost_cap = 0;
    int *d_count = nullptr;
    DevScalars *sc = nullptr;
    DevScalars *h_sc = nullptr;  // pinned mirror
    float *d_tmp = nullptr;      // reduction scratch (1 float)
    int *d_counter = nullptr;    // arrows counter
    double *d_diag = nullptr;    // partials + 8 finals + standoff
    int diag_parts = 0;
    StageTune tune{128, 6, 32};
    bool dt_ready = false;       // recompute policy: sc->dt holds the next dt
    bool cfl_valid = false;      // sc->cfl holds the maxima of the current state
    // graph replay of two steps, one per buffer parity (which of the two
    // ping-pong buffers currently holds U^n)
    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    unsigned long long graph_key[2] = {0, 0};
    // graph replay of one step (single-step calls and odd remainders), per parity
    cudaGraphExec_t graph1[2] = {nullptr, nullptr};
    unsigned long long graph1_key[2] = {0, 0};
    // registered display field (fvm_set_display_field): the last passes of
    // every step write it (destination and kind in the device descriptor
    // d_disp, mirrored in disp / disp_kind); fresh while the state is the one
    // a step (or a derived-field pass into it) left
    DisplayDesc *d_disp = nullptr;
    float *disp = nullptr;
    int disp_kind = 0;
    bool disp_fresh = false;
    float fixed_dt = 0.0f;       // fixed policy: the dt sc->dt holds when dt_ready
    float *parity_base = nullptr;  // buffer holding U^n at parity 0
    // measurement
    bool timing = false;
    std::vector<TimedLaunch> pending;
    std::vector<cudaEvent_t> event_pool;
    std::map<std::string, std::pair<long long, double>> ktimes;
    std::vector<std::string> knames;
    long long launches = 0;
    long long launches_at_sc_copy = -1;  // launches when fvm_queue_dt copied the device scalars
    size_t bytes = 0;
};


// Internal entry points shared with the batch implementation (fvm_api.cu).
int fvm_internal_build_maps(fvm_handle *h);
int fvm_internal_compute_dt(fvm_handle *h, const fvm_sim_params *p, float *dt);
int fvm_internal_set_error(int code, const char *msg);
// true when the batch holds a retired instance of this grid size (reused by fvm_batch_add)
bool fvm_internal_batch_has_parked(fvm_batch *b, int nx, int ny);
