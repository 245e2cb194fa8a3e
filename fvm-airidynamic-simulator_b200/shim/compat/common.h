// compat/common.h -- stand-in for the application's common.h, used to build the
// CFDSolver shim and the benchmark entry inside this repository.  The
// application keeps its own header; what must match is the SimParams layout
// (checked with static_asserts in cfd_solver.cpp against fvm_sim_params),
// the enum values and computeDerived's arithmetic (reference:
// src/include/common.h:7-19, :39-47, :50-111).
#pragma once
#include <cmath>
#include <cstdint>
#include <cuda_runtime.h>

constexpr float GAMMA = 1.4f;
constexpr float R_GAS = 287.05f;
constexpr float CV = R_GAS / (GAMMA - 1.0f);
constexpr float CP = GAMMA * CV;
constexpr float PI = 3.14159265358979323846f;
constexpr float MU_REF = 1.716e-5f;
constexpr float T_REF = 273.15f;
constexpr float S_SUTHERLAND = 110.4f;
constexpr float PRANDTL_NUMBER = 0.71f;

enum class ObstacleShape { CIRCLE = 0, STAR = 1, DIAMOND = 2, CAPSULE = 3, TRIANGLE = 4, STARSHIP = 5 };

struct SimParams {
    int nx = 512;
    int ny = 256;
    float dx = 1.0f;
    float dy = 1.0f;
    float domain_width = 10.0f;
    float domain_height = 5.0f;
    float mach = 3.0f;
    float T_inf = 300.0f;
    float p_inf = 101325.0f;
    float rho_inf = 0.0f;
    float u_inf = 0.0f;
    float v_inf = 0.0f;
    float c_inf = 0.0f;
    float obstacle_x = 2.5f;
    float obstacle_y = 2.5f;
    float obstacle_r = 0.5f;
    float obstacle_rotation = 0.0f;
    ObstacleShape obstacle_shape = ObstacleShape::CIRCLE;
    float wing_rotation = 0.0f;
    float cfl = 0.5f;
    float dt = 1e-6f;
    float t_current = 0.0f;
    int step = 0;
    bool enable_viscosity = false;
    float cfl_visc = 0.4f;
    bool adiabatic_wall = true;
    float T_wall = 300.0f;
    bool paused = true;

    // freestream density, sound speed and velocity from Mach/T/p; grid
    // spacing; obstacle centred vertically
    void computeDerived() {
        rho_inf = p_inf / (R_GAS * T_inf);
        c_inf = sqrtf(GAMMA * R_GAS * T_inf);
        u_inf = mach * c_inf;
        dx = domain_width / (float)nx;
        dy = domain_height / (float)ny;
        obstacle_y = domain_height / 2.0f;
    }
};

enum CellType : uint8_t { CELL_FLUID = 0, CELL_SOLID = 1, CELL_GHOST = 2, CELL_INFLOW = 3, CELL_OUTFLOW = 4 };
