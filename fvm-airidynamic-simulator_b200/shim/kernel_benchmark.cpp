// kernel_benchmark.cpp -- the benchmark entry (counterpart of the reference's
// src/test/kernel_benchmark.cu) built on the CFDSolver shim: a viscous Mach-3
// flow past a circle (r = 0.5 m in a 10 m x 5 m domain, T = 300 K,
// p = 101325 Pa, CFL 0.5 / 0.4), grid from argv (default 1024 x 512), dt
// fixed from the start state, 10 settling steps, 3 warm-up steps, then the
// mean of 5 timed steps.  Timing is the host clock between two
// cudaDeviceSynchronize calls, as in the reference entry: the solver works on
// its own stream, which events on the legacy default stream would not see.
#include <cuda_runtime.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>

#include "solver.cuh"

int main(int argc, char **argv) {
    const int nx = argc > 1 ? std::atoi(argv[1]) : 1024;
    const int ny = argc > 2 ? std::atoi(argv[2]) : 512;
    const int steps = argc > 3 ? std::atoi(argv[3]) : 5;
    if (nx <= 0 || ny <= 0 || steps <= 0) {
        std::fprintf(stderr, "usage: %s [nx=1024] [ny=512] [timed_steps=5]\n", argv[0]);
        return 1;
    }
    cudaDeviceProp prop;
    cudaGetDeviceProperties(&prop, 0);
    std::printf("device %s, %d SMs; grid %d x %d (%d cells)\n", prop.name, prop.multiProcessorCount, nx, ny, nx * ny);

    SimParams params;
    params.nx = nx;
    params.ny = ny;
    params.mach = 3.0f;
    params.T_inf = 300.0f;
    params.p_inf = 101325.0f;
    params.enable_viscosity = true;
    params.cfl = 0.5f;
    params.cfl_visc = 0.4f;
    params.obstacle_shape = ObstacleShape::CIRCLE;
    params.obstacle_r = 0.5f;
    params.domain_width = 10.0f;
    params.domain_height = 5.0f;
    params.computeDerived();

    CFDSolver solver;
    solver.initialize(params);
    params.dt = solver.computeStableTimeStep(params);
    std::printf("dx %.4f dy %.4f dt %.3e s\n", params.dx, params.dy, params.dt);

    for (int i = 0; i < 10; i++) solver.step(params);
    for (int i = 0; i < 3; i++) solver.step(params);
    cudaDeviceSynchronize();

    const auto t0 = std::chrono::steady_clock::now();
    for (int i = 0; i < steps; i++) solver.step(params);
    cudaDeviceSynchronize();
    const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    std::printf("steps %d, t = %.4e s, max T %.1f K, max Mach %.3f\n", params.step, params.t_current,
                solver.getMaxTemperature(), solver.getMaxMach());
    std::printf("Avg per step: %.4f ms  (%.3e cell-updates/s)\n", ms / steps, (double)nx * ny * steps / (ms * 1e-3));
    return 0;
}
