// fvm_math.cuh -- per-cell / per-face device arithmetic of the hot path.
//
// Every function restates one piece of the reference solver (src/solver.cu)
// in the same FP32 expression order, so that compiled with the reference's
// flags (--use_fast_math) the results track the reference kernels closely.
// Functions with no reference counterpart (AUSM+, van Leer) say so.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace fvm {

// Physical constants (src/include/common.h:7-19)
constexpr float GAMMA = 1.4f;
constexpr float R_GAS = 287.05f;
constexpr float CV = R_GAS / (GAMMA - 1.0f);
constexpr float CP = GAMMA * CV;
constexpr float PI_F = 3.14159265358979323846f;
constexpr float MU_REF = 1.716e-5f;
constexpr float T_REF = 273.15f;
constexpr float S_SUTH = 110.4f;
constexpr float PRANDTL_REF = 0.71f;
// Clamps and thresholds (src/solver.cu:10-53)
constexpr float MIN_DENSITY = 1e-4f;
constexpr float MIN_PRESSURE = 1e-2f;
constexpr float MAX_TEMPERATURE = 5000.0f;
constexpr float MIN_TEMPERATURE = 50.0f;
constexpr float ETA_THRESHOLD = 0.001f;
constexpr float ENTROPY_FIX = 0.1f;
constexpr float LOW_DENSITY = 0.01f;
constexpr float MAX_VEL = 5000.0f;
constexpr float MAX_GHOST_VEL = 2500.0f;
constexpr float SLIP_VREF = 100.0f;
constexpr float SLIP_MAX = 0.8f;

// Cell classes (src/include/common.h:105-111)
enum : uint8_t { CT_FLUID = 0, CT_SOLID = 1, CT_GHOST = 2, CT_INFLOW = 3, CT_OUTFLOW = 4 };

// Per-cell mask byte precomputed from the cell classes at geometry set-up.
// It carries what the stencil kernels need about the cell and about the two
// faces it owns (x-face i+1/2 and y-face j+1/2):
enum : uint32_t {
    MB_WALL = 1u << 0,  // cell is SOLID or GHOST
    MB_XV = 1u << 1,    // x-face i+1/2: neither side is a wall (and i < nx-1)
    MB_XN = 1u << 2,    // x-face i+1/2: a wall at i-1 or i+2 (clamped) -> first order
    MB_YV = 1u << 3,    // y-face j+1/2: neither side is a wall (and j < ny-1)
    MB_YN = 1u << 4,    // y-face j+1/2: a wall at j-1 or j+2 (clamped)
    MB_TYPE_SHIFT = 5   // bits 5..7: cell class
};
__device__ __forceinline__ uint32_t mb_type(uint32_t m) { return (m >> MB_TYPE_SHIFT) & 7u; }

struct Prim {  // flux-stencil state: raw conserved density + primitive velocity/pressure
    float rho, u, v, p;
};

// Approximate reciprocal (the same hardware approximation the fast-math
// division a / b multiplies by); one reciprocal serves every quotient with
// the same divisor.
__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

// The dual-energy switch eta = rho_e / E < 1e-3 of the reference (eta = 1
// when E <= 0), evaluated as rho_e < 1e-3 * E for E > 0 (no division).
__device__ __forceinline__ bool dual_energy_low(float rho_e, float E) {
    return E > 0.0f && rho_e < ETA_THRESHOLD * E;
}

// computePrimitivesKernelInline (src/solver.cu:862-894)
__device__ __forceinline__ void prim_from_cons(float rho, float rho_u, float rho_v, float E, float rho_e,
                                               float &u, float &v, float &p, float &T) {
    float rho_val = fmaxf(rho, MIN_DENSITY);
    const float inv_rho = rcp_approx(rho_val);
    float u_val = rho_u * inv_rho;
    float v_val = rho_v * inv_rho;
    float ke = 0.5f * rho_val * (u_val * u_val + v_val * v_val);
    float e_from_E = E - ke;
    float e_internal = dual_energy_low(rho_e, E) ? rho_e : e_from_E;
    float p_val = (GAMMA - 1.0f) * e_internal;
    p_val = fmaxf(p_val, MIN_PRESSURE);
    float T_val = p_val * inv_rho * (1.0f / R_GAS);
    T_val = fminf(T_val, MAX_TEMPERATURE);
    T_val = fmaxf(T_val, MIN_TEMPERATURE);
    u = u_val;
    v = v_val;
    p = p_val;
    T = T_val;
}

// Limited slopes: minmod (src/solver.cu:110-150); van Leer harmonic mean
// (van Leer 1974, J. Comput. Phys. 14:361; no reference counterpart).
template <int LIM>
__device__ __forceinline__ float limited_slope(float qm1, float q0, float qp1) {
    float dL = q0 - qm1;
    float dR = qp1 - q0;
    if (LIM == 0) {
        return 0.5f * (copysignf(1.0f, dL) + copysignf(1.0f, dR)) * fminf(fabsf(dL), fabsf(dR));
    } else {
        float ab = dL * dR;
        return (ab > 0.0f) ? (2.0f * ab / (dL + dR)) : 0.0f;
    }
}

// Physical flux along the face normal (src/solver.cu:1005-1037): mass, normal
// momentum, tangential momentum, energy.  rho*u*v evaluates as (rho*u)*v.
template <bool XDIR>
__device__ __forceinline__ void phys_flux(float rho, float un, float ut, float p, float E, float f[4]) {
    f[0] = rho * un;
    f[1] = rho * un * un + p;
    f[2] = XDIR ? (rho * un * ut) : (rho * ut * un);
    f[3] = (E + p) * un;
}

// HLLC with Roe-averaged Davis wave speeds (x: src/solver.cu:1112-1223,
// y: :1315-1430), written in normal/tangential form.
template <bool XDIR>
__device__ __forceinline__ void hllc_flux(float rhoL, float unL, float utL, float pL, float EL, float rhoR,
                                          float unR, float utR, float pR, float ER, float f[4]) {
    float cL = sqrtf(GAMMA * pL / rhoL);
    float cR = sqrtf(GAMMA * pR / rhoR);
    float sqrtRhoL = sqrtf(rhoL);
    float sqrtRhoR = sqrtf(rhoR);
    float denom = sqrtRhoL + sqrtRhoR + 1e-10f;
    float un_roe = (sqrtRhoL * unL + sqrtRhoR * unR) / denom;
    float ut_roe = (sqrtRhoL * utL + sqrtRhoR * utR) / denom;
    float H_L = (EL + pL) / rhoL;
    float H_R = (ER + pR) / rhoR;
    float H_roe = (sqrtRhoL * H_L + sqrtRhoR * H_R) / denom;
    float c_roe_sq = XDIR ? (GAMMA - 1.0f) * (H_roe - 0.5f * (un_roe * un_roe + ut_roe * ut_roe))
                          : (GAMMA - 1.0f) * (H_roe - 0.5f * (ut_roe * ut_roe + un_roe * un_roe));
    float c_roe = (c_roe_sq > 0.0f) ? sqrtf(c_roe_sq) : 0.5f * (cL + cR);
    float SL = fminf(unL - cL, un_roe - c_roe);
    float SR = fmaxf(unR + cR, un_roe + c_roe);
    float delta = ENTROPY_FIX * fmaxf(cL, cR);
    if (fabsf(SL) < delta) SL = -delta;
    if (fabsf(SR) < delta) SR = delta;
    float denom_star = rhoL * (SL - unL) - rhoR * (SR - unR);
    float safe_denom_star = copysignf(fmaxf(fabsf(denom_star), 1e-10f), denom_star);
    float S_star = (pR - pL + rhoL * unL * (SL - unL) - rhoR * unR * (SR - unR)) / safe_denom_star;
    // Upwind side K of the wave fan: L if all waves move right (SL >= 0) or
    // the contact does (S* >= 0), R otherwise.  The reference branches four
    // ways (src/solver.cu:1160-1222); selecting K's operands and evaluating
    // the shared star-state expressions once gives the same value per face
    // without divergence.
    const bool supL = SL >= 0.0f;
    const bool supR = !supL && SR <= 0.0f;
    const bool useL = supL || (!supR && S_star >= 0.0f);
    const float rK = useL ? rhoL : rhoR;
    const float unK = useL ? unL : unR;
    const float utK = useL ? utL : utR;
    const float pK = useL ? pL : pR;
    const float EK = useL ? EL : ER;
    const float SK = useL ? SL : SR;
    float fK[4];
    phys_flux<XDIR>(rK, unK, utK, pK, EK, fK);
    float coeff_denom = SK - S_star;
    if (fabsf(coeff_denom) < 1e-10f) coeff_denom = (coeff_denom >= 0) ? 1e-10f : -1e-10f;
    float rho_star = rK * (SK - unK) / coeff_denom;
    rho_star = fmaxf(rho_star, MIN_DENSITY);
    float mn_star = rho_star * S_star;
    float mt_star = rho_star * utK;
    float p_star = pK + rK * (SK - unK) * (S_star - unK);
    p_star = fmaxf(p_star, MIN_PRESSURE);
    float E_star = (EK * (SK - unK) + p_star * S_star - pK * unK) / coeff_denom;
    const bool star = !(supL || supR);
    f[0] = star ? fK[0] + SK * (rho_star - rK) : fK[0];
    f[1] = star ? fK[1] + SK * (mn_star - rK * unK) : fK[1];
    f[2] = star ? fK[2] + SK * (mt_star - rK * utK) : fK[2];
    f[3] = star ? fK[3] + SK * (E_star - EK) : fK[3];
}

// AUSM+ (Liou 1996, J. Comput. Phys. 129:364-382); no reference counterpart.
// Interface sound speed from the critical sound speed, split Mach numbers of
// degree 4 (beta = 1/8) and split pressures of degree 5 (alpha = 3/16).
__device__ __forceinline__ float ausm_mplus(float M) {
    if (fabsf(M) >= 1.0f) return 0.5f * (M + fabsf(M));
    float a = M + 1.0f, b = M * M - 1.0f;
    return 0.25f * a * a + 0.125f * b * b;
}
__device__ __forceinline__ float ausm_mminus(float M) {
    if (fabsf(M) >= 1.0f) return 0.5f * (M - fabsf(M));
    float a = M - 1.0f, b = M * M - 1.0f;
    return -0.25f * a * a - 0.125f * b * b;
}
__device__ __forceinline__ float ausm_pplus(float M) {
    if (fabsf(M) >= 1.0f) return (M > 0.0f) ? 1.0f : 0.0f;
    float a = M + 1.0f, b = M * M - 1.0f;
    return 0.25f * a * a * (2.0f - M) + 0.1875f * M * b * b;
}
__device__ __forceinline__ float ausm_pminus(float M) {
    if (fabsf(M) >= 1.0f) return (M < 0.0f) ? 1.0f : 0.0f;
    float a = M - 1.0f, b = M * M - 1.0f;
    return 0.25f * a * a * (2.0f + M) - 0.1875f * M * b * b;
}
__device__ __forceinline__ void ausm_plus_flux(float rhoL, float unL, float utL, float pL, float EL, float rhoR,
                                               float unR, float utR, float pR, float ER, float f[4]) {
    float HL = (EL + pL) / rhoL;
    float HR = (ER + pR) / rhoR;
    const float kcrit = 2.0f * (GAMMA - 1.0f) / (GAMMA + 1.0f);
    float csL = sqrtf(kcrit * HL);
    float csR = sqrtf(kcrit * HR);
    float ctL = csL * csL / fmaxf(csL, unL);
    float ctR = csR * csR / fmaxf(csR, -unR);
    float c12 = fminf(ctL, ctR);
    float ML = unL / c12;
    float MR = unR / c12;
    float m12 = ausm_mplus(ML) + ausm_mminus(MR);
    float p12 = ausm_pplus(ML) * pL + ausm_pminus(MR) * pR;
    float mp = 0.5f * (m12 + fabsf(m12));
    float mm = 0.5f * (m12 - fabsf(m12));
    float a = c12 * mp, b = c12 * mm;
    f[0] = a * rhoL + b * rhoR;
    f[1] = a * rhoL * unL + b * rhoR * unR + p12;
    f[2] = a * rhoL * utL + b * rhoR * utR;
    f[3] = a * rhoL * HL + b * rhoR * HR;
}

// One face of computeFluxesKernel (x: src/solver.cu:1502-1598, y: :1601-1682)
// from the two cells a | b and their limited slopes sa, sb (cell_slopes):
// MUSCL reconstruction of (rho, u, v, p), clamps, Riemann flux and the
// upwinded rho_e flux.  `valid`: neither a nor b is a wall; `near_wall`:
// first order (a wall at the outer stencil cells; the density test is done
// here).  out = {mass, x-momentum, y-momentum, energy, rho_e}.
template <bool XDIR, int SCHEME>
__device__ __forceinline__ void face_flux_sl(bool valid, bool near_wall, const Prim &a, const float sa[4],
                                             const Prim &b, const float sb[4], float out[5]) {
    if (valid) {
        bool lowDensity = (a.rho < LOW_DENSITY || b.rho < LOW_DENSITY);
        float order_mask = (near_wall || lowDensity) ? 0.0f : 1.0f;
        const float aa = XDIR ? a.u : a.v, ab = XDIR ? b.u : b.v;
        const float ta = XDIR ? a.v : a.u, tb = XDIR ? b.v : b.u;
        float rhoL = a.rho + 0.5f * sa[0] * order_mask;
        float unL = aa + 0.5f * sa[1] * order_mask;
        float utL = ta + 0.5f * sa[2] * order_mask;
        float pL = a.p + 0.5f * sa[3] * order_mask;
        float rhoR = b.rho - 0.5f * sb[0] * order_mask;
        float unR = ab - 0.5f * sb[1] * order_mask;
        float utR = tb - 0.5f * sb[2] * order_mask;
        float pR = b.p - 0.5f * sb[3] * order_mask;
        rhoL = fmaxf(rhoL, MIN_DENSITY);
        pL = fmaxf(pL, MIN_PRESSURE);
        rhoR = fmaxf(rhoR, MIN_DENSITY);
        pR = fmaxf(pR, MIN_PRESSURE);
        // E = p/(gamma-1) + 0.5*rho*(u^2 + v^2), x component squared first
        float keL = XDIR ? 0.5f * rhoL * (unL * unL + utL * utL) : 0.5f * rhoL * (utL * utL + unL * unL);
        float EL = pL / (GAMMA - 1.0f) + keL;
        float keR = XDIR ? 0.5f * rhoR * (unR * unR + utR * utR) : 0.5f * rhoR * (utR * utR + unR * unR);
        float ER = pR / (GAMMA - 1.0f) + keR;
        float f[4];
        if (SCHEME == 0)
            hllc_flux<XDIR>(rhoL, unL, utL, pL, EL, rhoR, unR, utR, pR, ER, f);
        else
            ausm_plus_flux(rhoL, unL, utL, pL, EL, rhoR, unR, utR, pR, ER, f);
        out[0] = f[0];
        out[1] = XDIR ? f[1] : f[2];
        out[2] = XDIR ? f[2] : f[1];
        out[3] = f[3];
        float u_face = 0.5f * (unL + unR);
        float rho_e_L = pL / (GAMMA - 1.0f);
        float rho_e_R = pR / (GAMMA - 1.0f);
        out[4] = (u_face >= 0.0f) ? rho_e_L * unL : rho_e_R * unR;
    } else {
        // wall face: mass/energy do not cross, pressure of the left/bottom cell acts
        out[0] = 0.0f;
        out[1] = XDIR ? a.p : 0.0f;
        out[2] = XDIR ? 0.0f : a.p;
        out[3] = 0.0f;
        out[4] = 0.0f;
    }
}

// Step coefficients of the update: dt, 1/dx, 1/dy.
struct UpdateArgs {
    float dt, inv_dx, inv_dy;
};
// Bounds of the specific internal energy per unit density in the update's
// dual-energy resync: R T_min / (gamma - 1) and R T_max / (gamma - 1)
// (src/solver.cu:1857-1864).
constexpr float kEminPerRho = R_GAS * MIN_TEMPERATURE / (GAMMA - 1.0f);
constexpr float kEmaxPerRho = R_GAS * MAX_TEMPERATURE / (GAMMA - 1.0f);

// ------------------------------------------------------ boundary conditions
// Riemann invariants along a boundary normal (src/solver.cu:680-841): un is
// the normal velocity, ut the tangential one.
__device__ __forceinline__ void riemann_from_prim(float rho, float un, float ut, float p, float &R1, float &R2,
                                                  float &R3, float &R4) {
    float c = sqrtf(GAMMA * p / rho);
    float log_rho = logf(rho);
    R1 = expf(-GAMMA * log_rho) * p;
    R2 = ut;
    constexpr float two_over_gamma_minus_1 = 2.0f / (GAMMA - 1.0f);
    R3 = un + c * two_over_gamma_minus_1;
    R4 = un - c * two_over_gamma_minus_1;
}
__device__ __forceinline__ void prim_from_riemann(float R1, float R2, float R3, float R4, float &rho, float &un,
                                                  float &ut, float &p) {
    ut = R2;
    un = (R3 + R4) * 0.5f;
    constexpr float gamma_minus_1_over_4 = (GAMMA - 1.0f) * 0.25f;
    constexpr float inv_gamma_minus_1 = 1.0f / (GAMMA - 1.0f);
    constexpr float inv_gamma = 1.0f / GAMMA;
    float c = (R3 - R4) * gamma_minus_1_over_4;
    float c_sq = c * c;
    float log_arg = c_sq * inv_gamma / R1;
    rho = expf(inv_gamma_minus_1 * logf(log_arg));
    p = rho * c_sq * inv_gamma;
}

struct Freestream {
    float rho, u, v, p;
};

// Neighbour k of the ghost-cell search in the reference's order
// {(-1,0),(1,0),(0,-1),(0,1),(-1,-1),(1,-1),(-1,1),(1,1)} (src/solver.cu:2072),
// computed arithmetically (no constant-memory table).
__host__ __device__ __forceinline__ void ghost_neighbour(int k, int &di, int &dj) {
    if (k < 2) {
        di = (k == 0) ? -1 : 1;
        dj = 0;
    } else if (k < 4) {
        di = 0;
        dj = (k == 2) ? -1 : 1;
    } else {
        di = (k & 1) ? 1 : -1;
        dj = (k < 6) ? -1 : 1;
    }
}

// Phase 1 of applyBoundaryConditionsKernel (src/solver.cu:1905-2042) for a
// non-ghost cell: inflow, right-outflow NRBC, bottom/top NRBC, solid.
// U is updated in place.  Ghost cells are left for the ghost pass.
__device__ __forceinline__ void bc_pointwise(float U[5], uint32_t ctype, int i, int j, int nx, int ny,
                                             const Freestream &fs) {
    float ke_inf = 0.5f * fs.rho * (fs.u * fs.u + fs.v * fs.v);
    float e_inf = fs.p / (GAMMA - 1.0f);
    float E_inf = e_inf + ke_inf;
    if (ctype == CT_INFLOW || i == 0) {
        U[0] = fs.rho;
        U[1] = fs.rho * fs.u;
        U[2] = fs.rho * fs.v;
        U[3] = E_inf;
        U[4] = e_inf;
        return;
    }
    if (ctype == CT_OUTFLOW || i == nx - 1) {
        float rho_loc = fmaxf(U[0], MIN_DENSITY);
        float u_loc, v_loc, p_loc, t_loc;
        prim_from_cons(U[0], U[1], U[2], U[3], U[4], u_loc, v_loc, p_loc, t_loc);
        float c_loc = sqrtf(GAMMA * p_loc / rho_loc);
        bool o1 = u_loc > 0.0f, o3 = u_loc + c_loc > 0.0f, o4 = u_loc - c_loc > 0.0f;
        float R1, R2, R3, R4, F1, F2, F3, F4;
        riemann_from_prim(U[0], u_loc, v_loc, p_loc, R1, R2, R3, R4);
        riemann_from_prim(fs.rho, fs.u, fs.v, fs.p, F1, F2, F3, F4);
        R1 = o1 ? R1 : F1;
        R2 = o1 ? R2 : F2;
        R3 = o3 ? R3 : F3;
        R4 = o4 ? R4 : F4;
        float rho_n;
        prim_from_riemann(R1, R2, R3, R4, rho_n, u_loc, v_loc, p_loc);
        U[0] = rho_n;
        U[1] = rho_n * u_loc;
        U[2] = rho_n * v_loc;
        U[4] = p_loc / (GAMMA - 1.0f);
        U[3] = U[4] + 0.5f * rho_n * (u_loc * u_loc + v_loc * v_loc);
        return;
    }
    if (ctype == CT_GHOST) return;
#pragma unroll
    for (int side = 0; side < 2; side++) {
        if (side == 0 ? (j != 0) : (j != ny - 1)) continue;
        float rho_loc = fmaxf(U[0], MIN_DENSITY);
        float u_loc, v_loc, p_loc, t_loc;
        prim_from_cons(rho_loc, U[1], U[2], U[3], U[4], u_loc, v_loc, p_loc, t_loc);
        float c_loc = sqrtf(GAMMA * p_loc / rho_loc);
        bool o1, o3, o4;
        if (side == 0) {
            o1 = v_loc < 0.0f;
            o3 = v_loc + c_loc < 0.0f;
            o4 = v_loc - c_loc < 0.0f;
        } else {
            o1 = v_loc > 0.0f;
            o3 = v_loc + c_loc > 0.0f;
            o4 = v_loc - c_loc > 0.0f;
        }
        float R1, R2, R3, R4, F1, F2, F3, F4;
        riemann_from_prim(rho_loc, v_loc, u_loc, p_loc, R1, R2, R3, R4);
        riemann_from_prim(fs.rho, fs.v, fs.u, fs.p, F1, F2, F3, F4);
        R1 = o1 ? R1 : F1;
        R2 = o1 ? R2 : F2;
        R3 = o3 ? R3 : F3;
        R4 = o4 ? R4 : F4;
        prim_from_riemann(R1, R2, R3, R4, rho_loc, v_loc, u_loc, p_loc);
        U[0] = rho_loc;
        U[1] = rho_loc * u_loc;
        U[2] = rho_loc * v_loc;
        U[4] = p_loc / (GAMMA - 1.0f);
        U[3] = U[4] + 0.5f * rho_loc * (u_loc * u_loc + v_loc * v_loc);
    }
    if (ctype == CT_SOLID) {
        U[0] = fs.rho;
        U[1] = 0.0f;
        U[2] = 0.0f;
        U[3] = e_inf;
        U[4] = e_inf;
    }
}

struct WallParams {
    bool viscous, adiabatic;
    float T_wall;
};

// Ghost-cell state from the chosen fluid neighbour (src/solver.cu:2111-2224).
// (gx, gy): unit SDF normal; fluid state given as conserved rho, rho_u, rho_v, E.
__device__ __forceinline__ void ghost_state(float rho_f, float rho_u_f, float rho_v_f, float E_f, float gx,
                                            float gy, const WallParams &w, float out[5]) {
    float u_f = rho_u_f / rho_f;
    float v_f = rho_v_f / rho_f;
    float ke_f = 0.5f * rho_f * (u_f * u_f + v_f * v_f);
    float p_f = (GAMMA - 1.0f) * (E_f - ke_f);
    rho_f = fmaxf(rho_f, MIN_DENSITY);
    p_f = fmaxf(p_f, MIN_PRESSURE);
    float vn = u_f * gx + v_f * gy;
    float vt = -v_f * gx + u_f * gy;
    float T_f = p_f / (rho_f * R_GAS);
    T_f = fminf(T_f, MAX_TEMPERATURE);
    T_f = fmaxf(T_f, MIN_TEMPERATURE);
    p_f = rho_f * R_GAS * T_f;
    float u_g, v_g;
    if (w.viscous) {
        u_g = -u_f;
        v_g = -v_f;
    } else {
        float slip_factor = 0.0f;
        if (vn > 0.0f) slip_factor = fminf(SLIP_MAX, vn / (vn + SLIP_VREF));
        float u_noslip = -u_f, v_noslip = -v_f;
        float u_slip = -vn * gx + vt * gy;
        float v_slip = -vn * gy - vt * gx;
        u_g = (1.0f - slip_factor) * u_noslip + slip_factor * u_slip;
        v_g = (1.0f - slip_factor) * v_noslip + slip_factor * v_slip;
    }
    float vel_g_mag = sqrtf(u_g * u_g + v_g * v_g);
    if (vel_g_mag > MAX_GHOST_VEL) {
        float scale = MAX_GHOST_VEL / vel_g_mag;
        u_g *= scale;
        v_g *= scale;
    }
    float p_g = p_f;
    float T_g;
    if (w.adiabatic) {
        T_g = T_f;
    } else {
        T_g = 2.0f * w.T_wall - T_f;
        T_g = fmaxf(T_g, MIN_TEMPERATURE);
        T_g = fminf(T_g, MAX_TEMPERATURE);
    }
    float rho_g = p_g / (R_GAS * T_g);
    rho_g = fmaxf(rho_g, MIN_DENSITY);
    float e_g = p_g / (GAMMA - 1.0f);
    float ke_g = 0.5f * rho_g * (u_g * u_g + v_g * v_g);
    out[0] = rho_g;
    out[1] = rho_g * u_g;
    out[2] = rho_g * v_g;
    out[3] = e_g + ke_g;
    out[4] = e_g;
}

// ------------------------------------------------------------ viscous terms
// Sutherland viscosity (src/solver.cu:2319, :2351)
__device__ __forceinline__ float sutherland_mu(float T_val) {
    float T_ratio = T_val * (1.0f / T_REF);
    return MU_REF * (T_ratio * sqrtf(T_ratio)) * (T_REF + S_SUTH) * rcp_approx(T_val + S_SUTH);
}

// Stress and heat flux at one cell (src/solver.cu:2336-2415) from its 4
// neighbours; edge flags select one-sided differences at the domain edges.
// out = {tau_xx, tau_yy, tau_xy, q_x, q_y}.  `pr` < 0 selects the reference
// Prandtl constant.
struct ViscArgs {
    float inv_2dx, inv_2dy, inv_dx, inv_dy, prandtl;
    bool ref_prandtl;
    float cp_over_pr;  // c_p / Pr (the reference Prandtl number or `prandtl`), set by viscous_args
};
// The divisions of a viscous pass computed once: 1/(2dx), 1/dx, ..., c_p / Pr.
__host__ __device__ __forceinline__ ViscArgs viscous_args(float dx, float dy, float prandtl, bool ref_prandtl) {
    ViscArgs va;
    va.inv_2dx = 0.5f / dx;
    va.inv_2dy = 0.5f / dy;
    va.inv_dx = 1.0f / dx;
    va.inv_dy = 1.0f / dy;
    va.prandtl = prandtl;
    va.ref_prandtl = ref_prandtl;
    va.cp_over_pr = ref_prandtl ? CP / PRANDTL_REF : CP / prandtl;
    return va;
}
// `mu_val` is sutherland_mu(TC), computed by the caller.
__device__ __forceinline__ void stress_heat_mu(float mu_val, float uC, float vC, float TC, float uE, float uW,
                                               float uN, float uS, float vE, float vW, float vN, float vS, float TE,
                                               float TW, float TN, float TS, bool i_lo, bool i_hi, bool j_lo,
                                               bool j_hi, const ViscArgs &va, float out[5]) {
    float k_val = mu_val * va.cp_over_pr;
    float du_dx = (uE - uW) * va.inv_2dx;
    float du_dy = (uN - uS) * va.inv_2dy;
    float dv_dx = (vE - vW) * va.inv_2dx;
    float dv_dy = (vN - vS) * va.inv_2dy;
    if (i_lo) {
        du_dx = (uE - uC) * va.inv_dx;
        dv_dx = (vE - vC) * va.inv_dx;
    } else if (i_hi) {
        du_dx = (uC - uW) * va.inv_dx;
        dv_dx = (vC - vW) * va.inv_dx;
    }
    if (j_lo) {
        du_dy = (uN - uC) * va.inv_dy;
        dv_dy = (vN - vC) * va.inv_dy;
    } else if (j_hi) {
        du_dy = (uC - uS) * va.inv_dy;
        dv_dy = (vC - vS) * va.inv_dy;
    }
    float div_v = du_dx + dv_dy;
    out[0] = mu_val * (2.0f * du_dx - (2.0f / 3.0f) * div_v);
    out[1] = mu_val * (2.0f * dv_dy - (2.0f / 3.0f) * div_v);
    out[2] = mu_val * (du_dy + dv_dx);
    float dT_dx = (TE - TW) * va.inv_2dx;
    float dT_dy = (TN - TS) * va.inv_2dy;
    if (i_lo)
        dT_dx = (TE - TC) * va.inv_dx;
    else if (i_hi)
        dT_dx = (TC - TW) * va.inv_dx;
    if (j_lo)
        dT_dy = (TN - TC) * va.inv_dy;
    else if (j_hi)
        dT_dy = (TC - TS) * va.inv_dy;
    out[3] = -k_val * dT_dx;
    out[4] = -k_val * dT_dy;
}
// The same stress and heat flux with the edge choice made by the caller: at a
// left (bottom) domain edge the west (south) neighbour passed is the cell
// itself and fx (fy) = 1/dx (1/dy); at a right (top) edge the east (north)
// one, likewise; in the interior the neighbours and 1/(2dx), 1/(2dy).  Every
// difference is then the one stress_heat_mu takes, with identical operations.
__device__ __forceinline__ void stress_heat_sel(float mu_val, float uE, float uW, float uN, float uS, float vE,
                                                float vW, float vN, float vS, float TE, float TW, float TN, float TS,
                                                float fx, float fy, const ViscArgs &va, float out[5]) {
    float k_val = mu_val * va.cp_over_pr;
    float du_dx = (uE - uW) * fx;
    float du_dy = (uN - uS) * fy;
    float dv_dx = (vE - vW) * fx;
    float dv_dy = (vN - vS) * fy;
    float div_v = du_dx + dv_dy;
    out[0] = mu_val * (2.0f * du_dx - (2.0f / 3.0f) * div_v);
    out[1] = mu_val * (2.0f * dv_dy - (2.0f / 3.0f) * div_v);
    out[2] = mu_val * (du_dy + dv_dx);
    out[3] = -k_val * ((TE - TW) * fx);
    out[4] = -k_val * ((TN - TS) * fy);
}
// stress_heat_sel plus what the divergence of the viscous update needs from
// this cell: the work terms u tau_xx + v tau_xy and u tau_xy + v tau_yy, and
// the dissipation Phi = tau_xx du/dx + tau_yy dv/dy + tau_xy (du/dy + dv/dx)
// (src/solver.cu:2437-2510).  out = {txx, tyy, txy, qx, qy, wx, wy, phi}.
// In the interior (the only cells the update changes) the velocity
// gradients are the central differences the reference's update uses.
__device__ __forceinline__ void stress_heat_work_sel(float mu_val, float uC, float vC, float uE, float uW, float uN,
                                                     float uS, float vE, float vW, float vN, float vS, float TE,
                                                     float TW, float TN, float TS, float fx, float fy,
                                                     const ViscArgs &va, float out[8]) {
    float k_val = mu_val * va.cp_over_pr;
    float du_dx = (uE - uW) * fx;
    float du_dy = (uN - uS) * fy;
    float dv_dx = (vE - vW) * fx;
    float dv_dy = (vN - vS) * fy;
    float div_v = du_dx + dv_dy;
    out[0] = mu_val * (2.0f * du_dx - (2.0f / 3.0f) * div_v);
    out[1] = mu_val * (2.0f * dv_dy - (2.0f / 3.0f) * div_v);
    out[2] = mu_val * (du_dy + dv_dx);
    out[3] = -k_val * ((TE - TW) * fx);
    out[4] = -k_val * ((TN - TS) * fy);
    out[5] = uC * out[0] + vC * out[2];
    out[6] = uC * out[2] + vC * out[1];
    out[7] = out[0] * du_dx + out[1] * dv_dy + out[2] * (du_dy + dv_dx);
}
__device__ __forceinline__ void stress_heat(float uC, float vC, float TC, float uE, float uW, float uN, float uS,
                                            float vE, float vW, float vN, float vS, float TE, float TW, float TN,
                                            float TS, bool i_lo, bool i_hi, bool j_lo, bool j_hi,
                                            const ViscArgs &va, float out[5]) {
    stress_heat_mu(sutherland_mu(TC), uC, vC, TC, uE, uW, uN, uS, vE, vW, vN, vS, TE, TW, TN, TS, i_lo, i_hi, j_lo,
                   j_hi, va, out);
}

// CFL quantities (src/solver.cu:2729-2739, :2679-2687)
__device__ __forceinline__ float wave_speed(float u, float v, float p, float rho_raw) {
    float c = sqrtf(GAMMA * p * rcp_approx(rho_raw + 1e-10f));
    return sqrtf(u * u + v * v) + c;
}

}  // namespace fvm
