// solver.cuh -- drop-in replacement for the application's solver header.
//
// Same public class `CFDSolver` as the reference (src/include/solver.cuh:22-257):
// the application (main.cpp, renderer, streaming) compiles unchanged against it
// and links shim/cfd_solver.cpp + libfvm_b200.so instead of src/solver.cu.
// Every method forwards to the C ABI in fvm_b200.h; a failing call prints the
// library's error text and exits, the behaviour of the reference's CUDA_CHECK.
#pragma once

#include <cstddef>
#include <cstdint>
#include <iostream>

#include "common.h"

#ifndef CUDA_CHECK
#define CUDA_CHECK(call)                                                                               \
    do {                                                                                               \
        cudaError_t err__ = (call);                                                                    \
        if (err__ != cudaSuccess) {                                                                    \
            std::cerr << "CUDA error '" << __FILE__ << "' line " << __LINE__ << ": "                   \
                      << cudaGetErrorString(err__) << std::endl;                                       \
            exit(EXIT_FAILURE);                                                                        \
        }                                                                                              \
    } while (0)
#endif

struct fvm_handle;

class CFDSolver {
public:
    CFDSolver();
    ~CFDSolver();
    CFDSolver(const CFDSolver &) = delete;
    CFDSolver &operator=(const CFDSolver &) = delete;

    void initialize(const SimParams &params);
    void resize(int nx, int ny);
    void step(SimParams &params);
    void reset(const SimParams &params);
    void updateObstacleGeometry(const SimParams &params);

    void getCellTypes(uint8_t *host_types);
    void convertCellTypesToDevice(float *devOutput);

    void computeTemperatureToDevice(float *dev_dst);
    void computePressureToDevice(float *dev_dst);
    void computeDensityToDevice(float *dev_dst);
    void computeVelocityMagToDevice(float *dev_dst);
    void computeMachToDevice(float *dev_dst);

    int generateVectorArrows(float *dev_vertexData, int maxVertices, int step, float u_inf, float maxArrowLength,
                             float arrowHeadAngle, float arrowHeadLength);

    int getNx() const { return _nx; }
    int getNy() const { return _ny; }

    float computeStableTimeStep(const SimParams &params);
    void queueTimeStepComputation(const SimParams &params);
    float readTimeStepResult(const SimParams &params) const;

    float getMaxTemperature();
    float getMaxMach();

    // (free, total) in the order the reference implementation writes them
    static void getGPUMemoryInfo(size_t &freeMem, size_t &totalMem);
    size_t getSimulationMemoryUsage();

    // not in the reference: the underlying C-ABI handle, for extensions
    // (flux scheme, limiter, dt policy, diagnostics, field readback)
    fvm_handle *handle() const { return h_; }

private:
    fvm_handle *h_ = nullptr;
    int _nx = 1024;
    int _ny = 512;
};
