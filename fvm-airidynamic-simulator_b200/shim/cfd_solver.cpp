// cfd_solver.cpp -- CFDSolver (reference src/include/solver.cuh:22-257) over the
// C ABI of libfvm_b200.so.  The reference's exit-on-error behaviour
// (CUDA_CHECK, src/include/solver.cuh:8-19) is recreated here and only here.
#include "solver.cuh"

#include <cstddef>
#include <cstdio>
#include <cstdlib>

#include "fvm_b200.h"

static_assert(sizeof(SimParams) == sizeof(fvm_sim_params), "SimParams layout");
static_assert(offsetof(SimParams, obstacle_shape) == offsetof(fvm_sim_params, obstacle_shape), "SimParams layout");
static_assert(offsetof(SimParams, wing_rotation) == offsetof(fvm_sim_params, wing_rotation), "SimParams layout");
static_assert(offsetof(SimParams, step) == offsetof(fvm_sim_params, step), "SimParams layout");
static_assert(offsetof(SimParams, enable_viscosity) == offsetof(fvm_sim_params, enable_viscosity), "SimParams layout");
static_assert(offsetof(SimParams, cfl_visc) == offsetof(fvm_sim_params, cfl_visc), "SimParams layout");
static_assert(offsetof(SimParams, adiabatic_wall) == offsetof(fvm_sim_params, adiabatic_wall), "SimParams layout");
static_assert(offsetof(SimParams, T_wall) == offsetof(fvm_sim_params, T_wall), "SimParams layout");
static_assert(offsetof(SimParams, paused) == offsetof(fvm_sim_params, paused), "SimParams layout");

namespace {
void check(int rc, const char *what) {
    if (rc != FVM_OK) {
        std::fprintf(stderr, "CFDSolver::%s failed: %s\n", what, fvm_last_error());
        std::exit(EXIT_FAILURE);
    }
}
const fvm_sim_params *cp(const SimParams &p) { return reinterpret_cast<const fvm_sim_params *>(&p); }
fvm_sim_params *mp(SimParams &p) { return reinterpret_cast<fvm_sim_params *>(&p); }
}  // namespace

CFDSolver::CFDSolver() { check(fvm_create(&h_), "CFDSolver"); }

CFDSolver::~CFDSolver() {
    if (h_) fvm_destroy(h_);
}

void CFDSolver::initialize(const SimParams &params) {
    _nx = params.nx;
    _ny = params.ny;
    check(fvm_initialize(h_, cp(params), nullptr), "initialize");
}

void CFDSolver::resize(int nx, int ny) {
    if (nx == _nx && ny == _ny) return;
    _nx = nx;
    _ny = ny;
    check(fvm_resize(h_, nx, ny), "resize");
}

void CFDSolver::step(SimParams &params) { check(fvm_step(h_, mp(params)), "step"); }

void CFDSolver::reset(const SimParams &params) { check(fvm_reset(h_, cp(params)), "reset"); }

void CFDSolver::updateObstacleGeometry(const SimParams &params) {
    check(fvm_update_obstacle(h_, cp(params)), "updateObstacleGeometry");
}

void CFDSolver::getCellTypes(uint8_t *host_types) { check(fvm_get_cell_types(h_, host_types), "getCellTypes"); }

void CFDSolver::convertCellTypesToDevice(float *devOutput) {
    check(fvm_cell_types_to_device(h_, devOutput), "convertCellTypesToDevice");
}

void CFDSolver::computeTemperatureToDevice(float *d) {
    check(fvm_field_to_device(h_, FVM_FIELD_TEMPERATURE, d), "computeTemperatureToDevice");
}
void CFDSolver::computePressureToDevice(float *d) {
    check(fvm_field_to_device(h_, FVM_FIELD_PRESSURE, d), "computePressureToDevice");
}
void CFDSolver::computeDensityToDevice(float *d) {
    check(fvm_field_to_device(h_, FVM_FIELD_DENSITY, d), "computeDensityToDevice");
}
void CFDSolver::computeVelocityMagToDevice(float *d) {
    check(fvm_field_to_device(h_, FVM_FIELD_VELOCITY_MAG, d), "computeVelocityMagToDevice");
}
void CFDSolver::computeMachToDevice(float *d) { check(fvm_field_to_device(h_, FVM_FIELD_MACH, d), "computeMachToDevice"); }

int CFDSolver::generateVectorArrows(float *dev_vertexData, int maxVertices, int step, float u_inf,
                                    float maxArrowLength, float arrowHeadAngle, float arrowHeadLength) {
    int n = -1;
    if (fvm_vector_arrows(h_, dev_vertexData, maxVertices, step, u_inf, maxArrowLength, arrowHeadAngle,
                          arrowHeadLength, &n) != FVM_OK)
        return -1;  // the reference's documented failure value
    return n;
}

float CFDSolver::computeStableTimeStep(const SimParams &params) {
    float dt = 0.0f;
    check(fvm_compute_dt(h_, cp(params), &dt), "computeStableTimeStep");
    return dt;
}

void CFDSolver::queueTimeStepComputation(const SimParams &params) {
    check(fvm_queue_dt(h_, cp(params)), "queueTimeStepComputation");
}

float CFDSolver::readTimeStepResult(const SimParams &params) const {
    float dt = 0.0f;
    check(fvm_read_dt(h_, cp(params), &dt), "readTimeStepResult");
    return dt;
}

float CFDSolver::getMaxTemperature() {
    float v = 0.0f;
    check(fvm_max_temperature(h_, &v), "getMaxTemperature");
    return v;
}

float CFDSolver::getMaxMach() {
    float v = 0.0f;
    check(fvm_max_mach(h_, &v), "getMaxMach");
    return v;
}

void CFDSolver::getGPUMemoryInfo(size_t &freeMem, size_t &totalMem) { fvm_gpu_mem_info(&freeMem, &totalMem); }

size_t CFDSolver::getSimulationMemoryUsage() {
    size_t b = 0;
    check(fvm_memory_usage(h_, &b), "getSimulationMemoryUsage");
    return b;
}
