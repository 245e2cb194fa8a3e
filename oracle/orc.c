/*
 * orc.c -- CPU oracle: a plain-C restatement of the reference solver's
 * per-step kernel chain.  TEST INFRASTRUCTURE ONLY (see orc.h).
 *
 * Every function below names the reference lines it restates (paths inside the
 * reference project).  Operation order follows the reference expressions so
 * the FP32 build (ORC_REAL=float, no FMA contraction, correctly rounded libm)
 * tracks the device result closely and the FP64 build gives the exact-method
 * answer.  Two points are defined here where the reference is not:
 *   - ghost-cell boundary conditions read a phase-1 snapshot (see orc.h);
 *   - AUSM+, van Leer and the blunted-cone SDF have no reference counterpart:
 *     they follow the published methods named at each function.
 */
#include "orc.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <float.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#ifndef ORC_REAL
#define ORC_REAL double
#endif
typedef ORC_REAL R;

#define IS_F32 (sizeof(R) == 4)
/* libm in the precision of R */
#define SQRT(x) ((R)(IS_F32 ? (R)sqrtf((float)(x)) : (R)sqrt((double)(x))))
#define EXP(x) ((R)(IS_F32 ? (R)expf((float)(x)) : (R)exp((double)(x))))
#define LOG(x) ((R)(IS_F32 ? (R)logf((float)(x)) : (R)log((double)(x))))
#define COS(x) ((R)(IS_F32 ? (R)cosf((float)(x)) : (R)cos((double)(x))))
#define SIN(x) ((R)(IS_F32 ? (R)sinf((float)(x)) : (R)sin((double)(x))))
#define ATAN2(y, x) ((R)(IS_F32 ? (R)atan2f((float)(y), (float)(x)) : (R)atan2((double)(y), (double)(x))))
#define FABS(x) ((R)(IS_F32 ? (R)fabsf((float)(x)) : (R)fabs((double)(x))))
#define COPYSIGN(a, b) ((R)(IS_F32 ? (R)copysignf((float)(a), (float)(b)) : (R)copysign((double)(a), (double)(b))))
#define ISFINITE(x) (isfinite(x))

static inline R fmaxR(R a, R b) { return a > b ? a : (b > a ? b : (a != a ? b : a)); }
static inline R fminR(R a, R b) { return a < b ? a : (b < a ? b : (a != a ? b : a)); }

/* Physical constants (src/include/common.h:7-19) */
#define GAMMA ((R)1.4)
#define GM1 (GAMMA - (R)1.0)
#define R_GAS ((R)287.05)
#define CV (R_GAS / GM1)
#define CP (GAMMA * CV)
#define PI_ ((R)3.14159265358979323846)
#define MU_REF ((R)1.716e-5)
#define T_REF ((R)273.15)
#define S_SUTH ((R)110.4)
/* Clamps and thresholds (src/solver.cu:10-53) */
#define MIN_DENSITY ((R)1e-4)
#define MIN_PRESSURE ((R)1e-2)
#define MAX_TEMPERATURE ((R)5000.0)
#define MIN_TEMPERATURE ((R)50.0)
#define ETA_THRESHOLD ((R)0.001)
#define ENTROPY_FIX ((R)0.1)
#define LOW_DENSITY ((R)0.01)
#define MAX_VEL ((R)5000.0)
#define MAX_GHOST_VEL ((R)2500.0)
#define BAND_FACTOR ((R)1.5)
#define STAR_RATIO ((R)0.38)
#define DIAMOND_K ((R)0.7071)
#define CAPSULE_HALF_LEN ((R)1.5)
#define CAPSULE_CAP ((R)0.5)
#define TRI_K ((R)0.866025404)
#define SLIP_VREF ((R)100.0)
#define SLIP_MAX ((R)0.8)

enum { CT_FLUID = 0, CT_SOLID = 1, CT_GHOST = 2, CT_INFLOW = 3, CT_OUTFLOW = 4 };

struct orc_solver {
    int nx, ny;
    size_t n;
    R *U[5];    /* rho, rho_u, rho_v, E, rho_e (current state U^n) */
    R *Us[5];   /* stage-1 result U* */
    R *Uk[5];   /* stage-2 result U** */
    R *snap[5]; /* BC phase-1 snapshot */
    R *u, *v, *p, *T, *mu;
    R *sdf;
    uint8_t *ct;
    R *fx[5], *fy[5];
    R *tau[5]; /* tau_xx, tau_yy, tau_xy, q_x, q_y */
    fvm_sim_params prm;
    fvm_ext ext;
    /* parameters in R precision */
    R dx, dy, rho_inf, u_inf, v_inf, p_inf, T_wall, cfl, cfl_visc, prandtl;
    R obs_x, obs_y, obs_r, obs_rot, wing_rot, cone_angle, cone_len;
    int shape, viscous, adiabatic, flux_scheme, limiter;
};

static R *alloc_r(size_t n) { return (R *)calloc(n ? n : 1, sizeof(R)); }

orc_solver *orc_create(int nx, int ny) {
    if (nx <= 0 || ny <= 0) return NULL;
    orc_solver *s = (orc_solver *)calloc(1, sizeof(orc_solver));
    s->nx = nx;
    s->ny = ny;
    s->n = (size_t)nx * ny;
    for (int k = 0; k < 5; k++) {
        s->U[k] = alloc_r(s->n);
        s->Us[k] = alloc_r(s->n);
        s->Uk[k] = alloc_r(s->n);
        s->snap[k] = alloc_r(s->n);
        s->fx[k] = alloc_r(s->n);
        s->fy[k] = alloc_r(s->n);
        s->tau[k] = alloc_r(s->n);
    }
    s->u = alloc_r(s->n);
    s->v = alloc_r(s->n);
    s->p = alloc_r(s->n);
    s->T = alloc_r(s->n);
    s->mu = alloc_r(s->n);
    s->sdf = alloc_r(s->n);
    s->ct = (uint8_t *)calloc(s->n, 1);
    orc_ext_default(&s->ext);
    orc_params_default(&s->prm);
    return s;
}

void orc_destroy(orc_solver *s) {
    if (!s) return;
    for (int k = 0; k < 5; k++) {
        free(s->U[k]); free(s->Us[k]); free(s->Uk[k]); free(s->snap[k]);
        free(s->fx[k]); free(s->fy[k]); free(s->tau[k]);
    }
    free(s->u); free(s->v); free(s->p); free(s->T); free(s->mu);
    free(s->sdf); free(s->ct);
    free(s);
}

int orc_real_size(void) { return (int)sizeof(R); }

int orc_set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
    return omp_get_max_threads();
#else
    (void)n;
    return 1;
#endif
}

/* SimParams defaults (src/include/common.h:53-90) and computeDerived
 * (src/include/common.h:93-101), both in float like the reference host code. */
void orc_params_default(fvm_sim_params *p) {
    memset(p, 0, sizeof(*p));
    p->nx = 512; p->ny = 256; p->dx = 1.0f; p->dy = 1.0f;
    p->domain_width = 10.0f; p->domain_height = 5.0f;
    p->mach = 3.0f; p->T_inf = 300.0f; p->p_inf = 101325.0f;
    p->obstacle_x = 2.5f; p->obstacle_y = 2.5f; p->obstacle_r = 0.5f;
    p->obstacle_shape = 0;
    p->cfl = 0.5f; p->dt = 1e-6f;
    p->enable_viscosity = false; p->cfl_visc = 0.4f;
    p->adiabatic_wall = true; p->T_wall = 300.0f; p->paused = true;
}

void orc_params_compute_derived(fvm_sim_params *p) {
    const float g = 1.4f, rg = 287.05f;
    p->rho_inf = p->p_inf / (rg * p->T_inf);
    p->c_inf = sqrtf(g * rg * p->T_inf);
    p->u_inf = p->mach * p->c_inf;
    p->dx = p->domain_width / (float)p->nx;
    p->dy = p->domain_height / (float)p->ny;
    p->obstacle_y = p->domain_height / 2.0f;
}

void orc_ext_default(fvm_ext *e) {
    memset(e, 0, sizeof(*e));
    e->flux_scheme = 0;
    e->limiter = 0;
    e->prandtl = 0.71f;
    e->dt_policy = 0;
    e->cone_half_angle = 0.2617993877991494f; /* 15 degrees */
    e->cone_length = 0.3f;
    e->ref_length = 0.0f;
}

void orc_set_params(orc_solver *s, const fvm_sim_params *p, const fvm_ext *e) {
    s->prm = *p;
    if (e) s->ext = *e;
    else orc_ext_default(&s->ext);
    s->dx = (R)p->dx; s->dy = (R)p->dy;
    s->rho_inf = (R)p->rho_inf; s->u_inf = (R)p->u_inf; s->v_inf = (R)p->v_inf; s->p_inf = (R)p->p_inf;
    s->T_wall = (R)p->T_wall; s->cfl = (R)p->cfl; s->cfl_visc = (R)p->cfl_visc;
    s->prandtl = (R)s->ext.prandtl;
    s->obs_x = (R)p->obstacle_x; s->obs_y = (R)p->obstacle_y; s->obs_r = (R)p->obstacle_r;
    s->obs_rot = (R)p->obstacle_rotation; s->wing_rot = (R)p->wing_rotation;
    s->cone_angle = (R)s->ext.cone_half_angle; s->cone_len = (R)s->ext.cone_length;
    s->shape = p->obstacle_shape;
    s->viscous = p->enable_viscosity ? 1 : 0;
    s->adiabatic = p->adiabatic_wall ? 1 : 0;
    s->flux_scheme = s->ext.flux_scheme;
    s->limiter = s->ext.limiter;
}

/* ====================================================== SDF geometry
 * src/solver.cu:67-102 (segment distance, cross product), :163-521 (shapes). */
static R seg_dist(R px, R py, R ax, R ay, R bx, R by) {
    R abx = bx - ax, aby = by - ay;
    R apx = px - ax, apy = py - ay;
    R t = (apx * abx + apy * aby) / (abx * abx + aby * aby + (R)1e-10);
    t = fmaxR((R)0, fminR((R)1, t));
    R cx = ax + t * abx, cy = ay + t * aby;
    R ddx = px - cx, ddy = py - cy;
    return SQRT(ddx * ddx + ddy * ddy);
}
static R cross2(R ax, R ay, R bx, R by) { return ax * by - ay * bx; }

static R sdf_circle(R px, R py, R cx, R cy, R r) {
    return SQRT((px - cx) * (px - cx) + (py - cy) * (py - cy)) - r;
}

static void rotate_in(R px, R py, R cx, R cy, R rot, R *qx, R *qy) {
    R lx = px - cx, ly = py - cy;
    R c = COS(-rot), s = SIN(-rot);
    *qx = lx * c - ly * s;
    *qy = lx * s + ly * c;
}

/* star: 10-vertex polygon, distance to edges, winding-number sign (src/solver.cu:179-240) */
static R sdf_star(R px, R py, R cx, R cy, R r, R rot) {
    const int N = 5;
    R qx, qy;
    rotate_in(px, py, cx, cy, rot, &qx, &qy);
    R vx[10], vy[10];
    R inner = r * STAR_RATIO;
    for (int i = 0; i < N; i++) {
        R a_out = (R)2.0 * PI_ * (R)i / (R)N - PI_ / (R)2.0;
        R a_in = a_out + PI_ / (R)N;
        vx[2 * i] = r * COS(a_out);
        vy[2 * i] = r * SIN(a_out);
        vx[2 * i + 1] = inner * COS(a_in);
        vy[2 * i + 1] = inner * SIN(a_in);
    }
    R best = (R)1e10, wind = 0;
    for (int i = 0; i < 2 * N; i++) {
        int k = (i + 1) % (2 * N);
        R d = seg_dist(qx, qy, vx[i], vy[i], vx[k], vy[k]);
        best = fminR(best, d);
        R ax = vx[i] - qx, ay = vy[i] - qy, bx = vx[k] - qx, by = vy[k] - qy;
        wind += ATAN2(cross2(ax, ay, bx, by), ax * bx + ay * by);
    }
    R sign = (FABS(wind) > PI_) ? (R)-1 : (R)1;
    return sign * best;
}

/* diamond: scaled L1 norm (src/solver.cu:252-272) */
static R sdf_diamond(R px, R py, R cx, R cy, R r, R rot) {
    R qx, qy;
    rotate_in(px, py, cx, cy, rot, &qx, &qy);
    R ax = FABS(qx) / r, ay = FABS(qy) / r;
    return (ax + ay - (R)1) * r * DIAMOND_K;
}

/* stadium: segment of half-length 1.5r-0.5r swept by radius 0.5r (src/solver.cu:284-311) */
static R sdf_capsule(R px, R py, R cx, R cy, R r, R rot) {
    R qx, qy;
    rotate_in(px, py, cx, cy, rot, &qx, &qy);
    R half = r * CAPSULE_HALF_LEN, cap = r * CAPSULE_CAP;
    R cxx = fmaxR(-half + cap, fminR(half - cap, qx));
    R ddx = qx - cxx, ddy = qy;
    return SQRT(ddx * ddx + ddy * ddy) - cap;
}

static int inside3(R c0, R c1, R c2) {
    return (c0 >= 0 && c1 >= 0 && c2 >= 0) || (c0 <= 0 && c1 <= 0 && c2 <= 0);
}

/* equilateral triangle, tip on +x (src/solver.cu:323-362) */
static R sdf_triangle(R px, R py, R cx, R cy, R r, R rot) {
    R qx, qy;
    rotate_in(px, py, cx, cy, rot, &qx, &qy);
    R v0x = r, v0y = 0, v1x = -r * (R)0.5, v1y = r * TRI_K, v2x = -r * (R)0.5, v2y = -r * TRI_K;
    R d0 = seg_dist(qx, qy, v0x, v0y, v1x, v1y);
    R d1 = seg_dist(qx, qy, v1x, v1y, v2x, v2y);
    R d2 = seg_dist(qx, qy, v2x, v2y, v0x, v0y);
    R md = fminR(d0, fminR(d1, d2));
    R c0 = cross2(v1x - v0x, v1y - v0y, qx - v0x, qy - v0y);
    R c1 = cross2(v2x - v1x, v2y - v1y, qx - v1x, qy - v1y);
    R c2 = cross2(v0x - v2x, v0y - v2y, qx - v2x, qy - v2y);
    return inside3(c0, c1, c2) ? -md : md;
}

/* convex quadrilateral (src/solver.cu:374-399) */
static R sdf_quad(R px, R py, R v0x, R v0y, R v1x, R v1y, R v2x, R v2y, R v3x, R v3y) {
    R d0 = seg_dist(px, py, v0x, v0y, v1x, v1y);
    R d1 = seg_dist(px, py, v1x, v1y, v2x, v2y);
    R d2 = seg_dist(px, py, v2x, v2y, v3x, v3y);
    R d3 = seg_dist(px, py, v3x, v3y, v0x, v0y);
    R md = fminR(fminR(d0, d1), fminR(d2, d3));
    R c0 = cross2(v1x - v0x, v1y - v0y, px - v0x, py - v0y);
    R c1 = cross2(v2x - v1x, v2y - v1y, px - v1x, py - v1y);
    R c2 = cross2(v3x - v2x, v3y - v2y, px - v2x, py - v2y);
    R c3 = cross2(v0x - v3x, v0y - v3y, px - v3x, py - v3y);
    int in = (c0 >= 0 && c1 >= 0 && c2 >= 0 && c3 >= 0) || (c0 <= 0 && c1 <= 0 && c2 <= 0 && c3 <= 0);
    return in ? -md : md;
}

/* starship: body circle + mirrored fixed root quad + rotating flap quad
 * (src/solver.cu:414-486; vertex table src/include/common.h:28-36) */
static R sdf_starship(R px, R py, R cx, R cy, R r, R rot, R wing) {
    R qx, qy;
    rotate_in(px, py, cx, cy, rot, &qx, &qy);
    R body = SQRT(qx * qx + qy * qy) - r;
    R scale = r / (R)90.0;
    R rx = qx / scale, ry = FABS(qy) / scale;
    R root = sdf_quad(rx, ry, (R)-45.0, (R)77.9422, (R)10.9682, (R)89.329, (R)6.0, (R)112.0, (R)-6.0, (R)112.0) * scale;
    R pvx = (R)-6.0, pvy = (R)112.0;
    R cw = COS(-wing), sw = SIN(-wing);
    R d1x = (R)6.0 - pvx, d1y = (R)112.0 - pvy;
    R d2x = (R)3.0 - pvx, d2y = (R)186.0 - pvy;
    R d3x = (R)-3.0 - pvx, d3y = (R)186.0 - pvy;
    R w1x = pvx + d1x * cw - d1y * sw, w1y = pvy + d1x * sw + d1y * cw;
    R w2x = pvx + d2x * cw - d2y * sw, w2y = pvy + d2x * sw + d2y * cw;
    R w3x = pvx + d3x * cw - d3y * sw, w3y = pvy + d3x * sw + d3y * cw;
    R flap = sdf_quad(rx, ry, pvx, pvy, w1x, w1y, w2x, w2y, w3x, w3y) * scale;
    return fminR(body, fminR(root, flap));
}

/* Blunted cone (no reference counterpart): nose circle of radius r centred at
 * (cx,cy) facing -x, joined tangentially to a frustum of half angle `ang`
 * extending `len` along +x from the tangent points.  SDF = min(circle, quad). */
static R sdf_cone_capsule(R px, R py, R cx, R cy, R r, R rot, R ang, R len) {
    R qx, qy;
    rotate_in(px, py, cx, cy, rot, &qx, &qy);
    R circ = SQRT(qx * qx + qy * qy) - r;
    R sa = SIN(ang), ca = COS(ang);
    R tx = -r * sa, ty = r * ca;
    R bx = tx + len, by = ty + len * (sa / ca);
    R quad = sdf_quad(qx, qy, tx, -ty, bx, -by, bx, by, tx, ty);
    return fminR(circ, quad);
}

static R shape_sdf(const orc_solver *s, R px, R py) {
    switch (s->shape) {
    case 0: return sdf_circle(px, py, s->obs_x, s->obs_y, s->obs_r);
    case 1: return sdf_star(px, py, s->obs_x, s->obs_y, s->obs_r, s->obs_rot);
    case 2: return sdf_diamond(px, py, s->obs_x, s->obs_y, s->obs_r, s->obs_rot);
    case 3: return sdf_capsule(px, py, s->obs_x, s->obs_y, s->obs_r, s->obs_rot);
    case 4: return sdf_triangle(px, py, s->obs_x, s->obs_y, s->obs_r, s->obs_rot);
    case 5: return sdf_starship(px, py, s->obs_x, s->obs_y, s->obs_r, s->obs_rot, s->wing_rot);
    case 6: return sdf_cone_capsule(px, py, s->obs_x, s->obs_y, s->obs_r, s->obs_rot, s->cone_angle, s->cone_len);
    default: return sdf_circle(px, py, s->obs_x, s->obs_y, s->obs_r);
    }
}

/* cell class from distance (src/solver.cu:560-588) */
static uint8_t classify(R dist, R band, int i, int nx) {
    uint8_t t;
    if (dist < -band) t = CT_SOLID;
    else if (dist < band && dist >= -band) t = CT_GHOST;
    else t = CT_FLUID;
    if (i == 0) t = CT_INFLOW;
    else if (i == nx - 1) t = CT_OUTFLOW;
    return t;
}

/* computeSDFKernel (src/solver.cu:536-589) */
static void compute_sdf(orc_solver *s) {
    const int nx = s->nx, ny = s->ny;
    R band = BAND_FACTOR * fmaxR(s->dx, s->dy);
#pragma omp parallel for schedule(static)
    for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
            size_t c = (size_t)j * nx + i;
            R x = ((R)i + (R)0.5) * s->dx;
            R y = ((R)j + (R)0.5) * s->dy;
            R d = shape_sdf(s, x, y);
            s->sdf[c] = d;
            s->ct[c] = classify(d, band, i, nx);
        }
}

/* =========================================================== primitives
 * computePrimitivesKernelInline (src/solver.cu:862-894) */
static inline void prim_from_cons(R rho, R ru, R rv, R E, R re, R *u, R *v, R *p, R *T) {
    R r = fmaxR(rho, MIN_DENSITY);
    R uu = ru / r, vv = rv / r;
    R ke = (R)0.5 * r * (uu * uu + vv * vv);
    R eE = E - ke;
    R eta = (E > 0) ? (re / E) : (R)1;
    R e = (eta < ETA_THRESHOLD) ? re : eE;
    R pp = GM1 * e;
    pp = fmaxR(pp, MIN_PRESSURE);
    R TT = pp / (r * R_GAS);
    TT = fminR(TT, MAX_TEMPERATURE);
    TT = fmaxR(TT, MIN_TEMPERATURE);
    *u = uu; *v = vv; *p = pp; *T = TT;
}

static void primitives(orc_solver *s, R *const U[5]) {
#pragma omp parallel for schedule(static)
    for (size_t c = 0; c < s->n; c++)
        prim_from_cons(U[0][c], U[1][c], U[2][c], U[3][c], U[4][c], &s->u[c], &s->v[c], &s->p[c], &s->T[c]);
}

/* initializeKernel (src/solver.cu:911-940) */
static void initialize(orc_solver *s) {
    R ke = (R)0.5 * s->rho_inf * (s->u_inf * s->u_inf + s->v_inf * s->v_inf);
    R e = s->p_inf / GM1;
    for (size_t c = 0; c < s->n; c++) {
        s->U[0][c] = s->rho_inf;
        s->U[1][c] = s->rho_inf * s->u_inf;
        s->U[2][c] = s->rho_inf * s->v_inf;
        s->U[3][c] = e + ke;
        s->U[4][c] = e;
    }
}

/* =============================================================== fluxes */
/* minmod slope (src/solver.cu:110-150) */
static inline R slope_minmod(R qm, R q0, R qp) {
    R a = q0 - qm, b = qp - q0;
    return (R)0.5 * (COPYSIGN((R)1, a) + COPYSIGN((R)1, b)) * fminR(FABS(a), FABS(b));
}
/* van Leer limited slope (van Leer 1974, J. Comput. Phys. 14:361): harmonic
 * mean of the one-sided differences when they share a sign, else zero. */
static inline R slope_vanleer(R qm, R q0, R qp) {
    R a = q0 - qm, b = qp - q0;
    R ab = a * b;
    return (ab > 0) ? ((R)2 * ab / (a + b)) : (R)0;
}
static inline R slope(const orc_solver *s, R qm, R q0, R qp) {
    return s->limiter == 1 ? slope_vanleer(qm, q0, qp) : slope_minmod(qm, q0, qp);
}

/* Physical flux along the face normal (src/solver.cu:1005-1037); `un` is the
 * normal velocity, `ut` the tangential one.  Output order: mass, normal
 * momentum, tangential momentum, energy. */
static inline void phys_flux(int xdir, R rho, R un, R ut, R p, R E, R f[4]) {
    f[0] = rho * un;
    f[1] = rho * un * un + p;
    /* rho*u*v is evaluated left to right in both directions: (rho*u)*v */
    f[2] = xdir ? (rho * un) * ut : (rho * ut) * un;
    f[3] = (E + p) * un;
}

/* HLLC with Roe-averaged Davis speeds (src/solver.cu:1112-1223 for x,
 * :1315-1430 for y; both directions share this normal/tangential form). */
static void hllc(int xd, R rL, R unL, R utL, R pL, R EL, R rR, R unR, R utR, R pR, R ER, R f[4]) {
    R cL = SQRT(GAMMA * pL / rL);
    R cR = SQRT(GAMMA * pR / rR);
    R sL = SQRT(rL), sR = SQRT(rR);
    R den = sL + sR + (R)1e-10;
    R un_roe = (sL * unL + sR * unR) / den;
    R ut_roe = (sL * utL + sR * utR) / den;
    R HL = (EL + pL) / rL, HR = (ER + pR) / rR;
    R H_roe = (sL * HL + sR * HR) / den;
    /* the reference forms u_roe^2 + v_roe^2 with the x component first */
    R c2 = GM1 * (H_roe - (R)0.5 * (un_roe * un_roe + ut_roe * ut_roe));
    R c_roe = (c2 > 0) ? SQRT(c2) : (R)0.5 * (cL + cR);
    R SL = fminR(unL - cL, un_roe - c_roe);
    R SR = fmaxR(unR + cR, un_roe + c_roe);
    R delta = ENTROPY_FIX * fmaxR(cL, cR);
    if (FABS(SL) < delta) SL = -delta;
    if (FABS(SR) < delta) SR = delta;
    R dstar = rL * (SL - unL) - rR * (SR - unR);
    R dsafe = COPYSIGN(fmaxR(FABS(dstar), (R)1e-10), dstar);
    R Sst = (pR - pL + rL * unL * (SL - unL) - rR * unR * (SR - unR)) / dsafe;
    if (SL >= 0) {
        phys_flux(xd, rL, unL, utL, pL, EL, f);
    } else if (SR <= 0) {
        phys_flux(xd, rR, unR, utR, pR, ER, f);
    } else if (Sst >= 0) {
        R cd = SL - Sst;
        if (FABS(cd) < (R)1e-10) cd = (cd >= 0) ? (R)1e-10 : (R)-1e-10;
        R rs = rL * (SL - unL) / cd;
        rs = fmaxR(rs, MIN_DENSITY);
        R mn = rs * Sst, mt = rs * utL;
        R ps = pL + rL * (SL - unL) * (Sst - unL);
        ps = fmaxR(ps, MIN_PRESSURE);
        R Es = (EL * (SL - unL) + ps * Sst - pL * unL) / cd;
        R fl[4];
        phys_flux(xd, rL, unL, utL, pL, EL, fl);
        f[0] = fl[0] + SL * (rs - rL);
        f[1] = fl[1] + SL * (mn - rL * unL);
        f[2] = fl[2] + SL * (mt - rL * utL);
        f[3] = fl[3] + SL * (Es - EL);
    } else {
        R cd = SR - Sst;
        if (FABS(cd) < (R)1e-10) cd = (cd >= 0) ? (R)1e-10 : (R)-1e-10;
        R rs = rR * (SR - unR) / cd;
        rs = fmaxR(rs, MIN_DENSITY);
        R mn = rs * Sst, mt = rs * utR;
        R ps = pR + rR * (SR - unR) * (Sst - unR);
        ps = fmaxR(ps, MIN_PRESSURE);
        R Es = (ER * (SR - unR) + ps * Sst - pR * unR) / cd;
        R fr[4];
        phys_flux(xd, rR, unR, utR, pR, ER, fr);
        f[0] = fr[0] + SR * (rs - rR);
        f[1] = fr[1] + SR * (mn - rR * unR);
        f[2] = fr[2] + SR * (mt - rR * utR);
        f[3] = fr[3] + SR * (Es - ER);
    }
}

/* AUSM+ (Liou 1996, J. Comput. Phys. 129:364-382), no reference counterpart.
 * Interface speed of sound from the critical speed of sound (eq. 30-31),
 * fourth-degree split Mach numbers with beta = 1/8 and fifth-degree split
 * pressures with alpha = 3/16 (eq. 19-21), mass flux upwinded on the sign of
 * the interface Mach number (eq. 10). */
static inline R ausm_mplus(R M) {
    if (FABS(M) >= 1) return (R)0.5 * (M + FABS(M));
    R a = M + (R)1, b = M * M - (R)1;
    return (R)0.25 * a * a + (R)0.125 * b * b;
}
static inline R ausm_mminus(R M) {
    if (FABS(M) >= 1) return (R)0.5 * (M - FABS(M));
    R a = M - (R)1, b = M * M - (R)1;
    return (R)-0.25 * a * a - (R)0.125 * b * b;
}
static inline R ausm_pplus(R M) {
    if (FABS(M) >= 1) return (M > 0) ? (R)1 : (R)0;
    R a = M + (R)1, b = M * M - (R)1;
    return (R)0.25 * a * a * ((R)2 - M) + (R)0.1875 * M * b * b;
}
static inline R ausm_pminus(R M) {
    if (FABS(M) >= 1) return (M < 0) ? (R)1 : (R)0;
    R a = M - (R)1, b = M * M - (R)1;
    return (R)0.25 * a * a * ((R)2 + M) - (R)0.1875 * M * b * b;
}
static void ausm_plus(R rL, R unL, R utL, R pL, R EL, R rR, R unR, R utR, R pR, R ER, R f[4]) {
    R HL = (EL + pL) / rL, HR = (ER + pR) / rR;
    R kcrit = (R)2 * GM1 / (GAMMA + (R)1);
    R csL = SQRT(kcrit * HL), csR = SQRT(kcrit * HR);
    R ctL = csL * csL / fmaxR(csL, unL);
    R ctR = csR * csR / fmaxR(csR, -unR);
    R c12 = fminR(ctL, ctR);
    R ML = unL / c12, MR = unR / c12;
    R m12 = ausm_mplus(ML) + ausm_mminus(MR);
    R p12 = ausm_pplus(ML) * pL + ausm_pminus(MR) * pR;
    R mp = (R)0.5 * (m12 + FABS(m12)), mm = (R)0.5 * (m12 - FABS(m12));
    R a = c12 * mp, b = c12 * mm;
    f[0] = a * rL + b * rR;
    f[1] = a * rL * unL + b * rR * unR + p12;
    f[2] = a * rL * utL + b * rR * utR;
    f[3] = a * rL * HL + b * rR * HR;
}

static inline int is_wall(uint8_t t) { return t == CT_SOLID || t == CT_GHOST; }

/* One face: reconstruct (rho,un,ut,p) from cells m1,a | b,p2 along the face
 * normal, then Riemann flux.  Follows computeFluxesKernel
 * (src/solver.cu:1502-1598 for x, :1601-1682 for y).  out[5] = mass, normal
 * momentum, tangential momentum, energy, rho_e. */
static void face_flux(const orc_solver *s, int xd, const R *rho, const R *un, const R *ut, const R *p,
                      size_t m1, size_t a, size_t b, size_t p2, R out[5]) {
    const uint8_t *ct = s->ct;
    if (!is_wall(ct[a]) && !is_wall(ct[b])) {
        int near = is_wall(ct[m1]) || is_wall(ct[p2]);
        int low = rho[a] < LOW_DENSITY || rho[b] < LOW_DENSITY;
        R mask = (near || low) ? (R)0 : (R)1;
        R srL = slope(s, rho[m1], rho[a], rho[b]);
        R snL = slope(s, un[m1], un[a], un[b]);
        R stL = slope(s, ut[m1], ut[a], ut[b]);
        R spL = slope(s, p[m1], p[a], p[b]);
        R rL = rho[a] + (R)0.5 * srL * mask;
        R nL = un[a] + (R)0.5 * snL * mask;
        R tL = ut[a] + (R)0.5 * stL * mask;
        R pL = p[a] + (R)0.5 * spL * mask;
        R srR = slope(s, rho[a], rho[b], rho[p2]);
        R snR = slope(s, un[a], un[b], un[p2]);
        R stR = slope(s, ut[a], ut[b], ut[p2]);
        R spR = slope(s, p[a], p[b], p[p2]);
        R rR = rho[b] - (R)0.5 * srR * mask;
        R nR = un[b] - (R)0.5 * snR * mask;
        R tR = ut[b] - (R)0.5 * stR * mask;
        R pR = p[b] - (R)0.5 * spR * mask;
        rL = fmaxR(rL, MIN_DENSITY);
        pL = fmaxR(pL, MIN_PRESSURE);
        rR = fmaxR(rR, MIN_DENSITY);
        pR = fmaxR(pR, MIN_PRESSURE);
        R EL = pL / GM1 + (R)0.5 * rL * (nL * nL + tL * tL);
        R ER = pR / GM1 + (R)0.5 * rR * (nR * nR + tR * tR);
        R f[4];
        if (s->flux_scheme == 1)
            ausm_plus(rL, nL, tL, pL, EL, rR, nR, tR, pR, ER, f);
        else
            hllc(xd, rL, nL, tL, pL, EL, rR, nR, tR, pR, ER, f);
        out[0] = f[0];
        out[1] = f[1];
        out[2] = f[2];
        out[3] = f[3];
        R uf = (R)0.5 * (nL + nR);
        R eL = pL / GM1, eR = pR / GM1;
        out[4] = (uf >= 0) ? eL * nL : eR * nR;
    } else {
        out[0] = 0;
        out[1] = p[a];
        out[2] = 0;
        out[3] = 0;
        out[4] = 0;
    }
}

/* computeFluxesKernel (src/solver.cu:1450-1684).  Stencil indices are clamped
 * to the domain like the reference's shared-memory tile load (:1484-1488).
 * x-face i+1/2 is stored at i (not written for i = nx-1); likewise y. */
static void fluxes(orc_solver *s, R *const U[5]) {
    const int nx = s->nx, ny = s->ny;
    const R *rho = U[0];
#pragma omp parallel for schedule(static)
    for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
            size_t c = (size_t)j * nx + i;
            R o[5];
            if (i < nx - 1) {
                int im1 = i > 0 ? i - 1 : 0;
                int ip2 = i + 2 < nx ? i + 2 : nx - 1;
                face_flux(s, 1, rho, s->u, s->v, s->p, (size_t)j * nx + im1, c, c + 1, (size_t)j * nx + ip2, o);
                s->fx[0][c] = o[0];
                s->fx[1][c] = o[1];
                s->fx[2][c] = o[2];
                s->fx[3][c] = o[3];
                s->fx[4][c] = o[4];
            }
            if (j < ny - 1) {
                int jm1 = j > 0 ? j - 1 : 0;
                int jp2 = j + 2 < ny ? j + 2 : ny - 1;
                face_flux(s, 0, rho, s->v, s->u, s->p, (size_t)jm1 * nx + i, c, c + (size_t)nx, (size_t)jp2 * nx + i, o);
                s->fy[0][c] = o[0];
                s->fy[1][c] = o[2]; /* x-momentum = tangential for y-faces */
                s->fy[2][c] = o[1]; /* y-momentum = normal */
                s->fy[3][c] = o[3];
                s->fy[4][c] = o[4];
            }
        }
}

/* updateKernel (src/solver.cu:1704-1876): flux divergence, rho_e source from
 * Riemann face velocities, forward Euler, non-finite rollback, velocity cap,
 * dual-energy resync.  Reads U and the primitive p; writes Uo. */
static void update(orc_solver *s, R *const U[5], R *const Uo[5], R dt) {
    const int nx = s->nx, ny = s->ny;
    const R inv_dx = (R)1 / s->dx, inv_dy = (R)1 / s->dy;
#pragma omp parallel for schedule(static)
    for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
            size_t c = (size_t)j * nx + i;
            if (is_wall(s->ct[c])) {
                for (int k = 0; k < 5; k++) Uo[k][c] = U[k][c];
                continue;
            }
            size_t cim = i > 0 ? c - 1 : c;
            size_t cjm = j > 0 ? c - nx : c;
            R dFx[5], dFy[5];
            for (int k = 0; k < 5; k++) {
                dFx[k] = (s->fx[k][c] - s->fx[k][cim]) * inv_dx;
                dFy[k] = (s->fy[k][c] - s->fy[k][cjm]) * inv_dy;
            }
            if (i == 0 || i == nx - 1)
                for (int k = 0; k < 5; k++) dFx[k] = 0;
            if (j == 0 || j == ny - 1)
                for (int k = 0; k < 5; k++) dFy[k] = 0;
            R src = 0;
            if (i > 0 && i < nx - 1 && j > 0 && j < ny - 1) {
                R rc = fmaxR(U[0][c], MIN_DENSITY);
                R rxR = fmaxR(U[0][c + 1], MIN_DENSITY);
                R rxL = fmaxR(U[0][c - 1], MIN_DENSITY);
                R ufR = s->fx[0][c] / ((R)0.5 * (rc + rxR));
                R ufL = s->fx[0][c - 1] / ((R)0.5 * (rxL + rc));
                R ryT = fmaxR(U[0][c + nx], MIN_DENSITY);
                R ryB = fmaxR(U[0][c - nx], MIN_DENSITY);
                R vfT = s->fy[0][c] / ((R)0.5 * (rc + ryT));
                R vfB = s->fy[0][c - nx] / ((R)0.5 * (ryB + rc));
                R div = (ufR - ufL) * inv_dx + (vfT - vfB) * inv_dy;
                src = -s->p[c] * div;
            }
            R nr = U[0][c] - dt * (dFx[0] + dFy[0]);
            R nru = U[1][c] - dt * (dFx[1] + dFy[1]);
            R nrv = U[2][c] - dt * (dFx[2] + dFy[2]);
            R nE = U[3][c] - dt * (dFx[3] + dFy[3]);
            R nre = U[4][c] - dt * (dFx[4] + dFy[4]) + dt * src;
            if (!ISFINITE(nr) || nr < MIN_DENSITY) nr = fmaxR(U[0][c], MIN_DENSITY);
            if (!ISFINITE(nru)) nru = U[1][c];
            if (!ISFINITE(nrv)) nrv = U[2][c];
            if (!ISFINITE(nE)) nE = U[3][c];
            if (!ISFINITE(nre) || nre < MIN_PRESSURE / GM1) nre = U[4][c];
            nr = fmaxR(nr, MIN_DENSITY);
            R uu = nru / nr, vv = nrv / nr;
            R vm = SQRT(uu * uu + vv * vv);
            if (vm > MAX_VEL) {
                R sc = MAX_VEL / vm;
                uu *= sc;
                vv *= sc;
                nru = nr * uu;
                nrv = nr * vv;
            }
            R ke = (R)0.5 * nr * (uu * uu + vv * vv);
            R eta = (nE > 0) ? (nre / nE) : (R)1;
            R e = (eta < ETA_THRESHOLD) ? nre : (nE - ke);
            R emin = nr * R_GAS * MIN_TEMPERATURE / GM1;
            R emax = nr * R_GAS * MAX_TEMPERATURE / GM1;
            e = fmaxR(e, emin);
            e = fminR(e, emax);
            Uo[0][c] = nr;
            Uo[1][c] = nru;
            Uo[2][c] = nrv;
            Uo[3][c] = e + ke;
            Uo[4][c] = e;
        }
}

/* ===================================================== boundary conditions
 * applyBoundaryConditionsKernel (src/solver.cu:1891-2226) with the Riemann
 * invariant helpers (src/solver.cu:680-841). */
static void inv_from_prim(R rho, R un, R ut, R p, R *R1, R *R2, R *R3, R *R4) {
    R c = SQRT(GAMMA * p / rho);
    R lr = LOG(rho);
    *R1 = EXP(-GAMMA * lr) * p;
    *R2 = ut;
    const R k = (R)2.0 / GM1;
    *R3 = un + c * k;
    *R4 = un - c * k;
}
static void prim_from_inv(R R1, R R2, R R3, R R4, R *rho, R *un, R *ut, R *p) {
    *ut = R2;
    *un = (R3 + R4) * (R)0.5;
    const R gm1_4 = GM1 * (R)0.25;
    const R inv_gm1 = (R)1.0 / GM1;
    const R inv_g = (R)1.0 / GAMMA;
    R c = (R3 - R4) * gm1_4;
    R c2 = c * c;
    R arg = c2 * inv_g / R1;
    *rho = EXP(inv_gm1 * LOG(arg));
    *p = *rho * c2 * inv_g;
}

/* phase 1: pointwise conditions for one cell; returns 1 if the cell is a ghost
 * cell left for phase 2. */
static int bc_pointwise(const orc_solver *s, R *const U[5], int i, int j) {
    const int nx = s->nx, ny = s->ny;
    size_t c = (size_t)j * nx + i;
    uint8_t t = s->ct[c];
    R ke_inf = (R)0.5 * s->rho_inf * (s->u_inf * s->u_inf + s->v_inf * s->v_inf);
    R e_inf = s->p_inf / GM1;
    R E_inf = e_inf + ke_inf;
    if (t == CT_INFLOW || i == 0) {
        U[0][c] = s->rho_inf;
        U[1][c] = s->rho_inf * s->u_inf;
        U[2][c] = s->rho_inf * s->v_inf;
        U[3][c] = E_inf;
        U[4][c] = e_inf;
        return 0;
    }
    if (t == CT_OUTFLOW || i == nx - 1) {
        R rho = U[0][c];
        R rl = fmaxR(rho, MIN_DENSITY);
        R u, v, p, T;
        prim_from_cons(rho, U[1][c], U[2][c], U[3][c], U[4][c], &u, &v, &p, &T);
        R cl = SQRT(GAMMA * p / rl);
        int o1 = u > 0, o3 = u + cl > 0, o4 = u - cl > 0;
        R a1, a2, a3, a4, f1, f2, f3, f4;
        inv_from_prim(rho, u, v, p, &a1, &a2, &a3, &a4);
        inv_from_prim(s->rho_inf, s->u_inf, s->v_inf, s->p_inf, &f1, &f2, &f3, &f4);
        a1 = o1 ? a1 : f1;
        a2 = o1 ? a2 : f2;
        a3 = o3 ? a3 : f3;
        a4 = o4 ? a4 : f4;
        R nr, nu, nv, np;
        prim_from_inv(a1, a2, a3, a4, &nr, &nu, &nv, &np);
        U[0][c] = nr;
        U[1][c] = nr * nu;
        U[2][c] = nr * nv;
        U[4][c] = np / GM1;
        U[3][c] = U[4][c] + (R)0.5 * nr * (nu * nu + nv * nv);
        return 0;
    }
    if (t == CT_GHOST) return 1; /* left untouched for phase 2 */
    for (int side = 0; side < 2; side++) {
        int active = side == 0 ? (j == 0) : (j == ny - 1);
        if (!active) continue;
        R rl = fmaxR(U[0][c], MIN_DENSITY);
        R u, v, p, T;
        prim_from_cons(rl, U[1][c], U[2][c], U[3][c], U[4][c], &u, &v, &p, &T);
        R cl = SQRT(GAMMA * p / rl);
        int o1, o3, o4;
        if (side == 0) { o1 = v < 0; o3 = v + cl < 0; o4 = v - cl < 0; }
        else { o1 = v > 0; o3 = v + cl > 0; o4 = v - cl > 0; }
        R a1, a2, a3, a4, f1, f2, f3, f4;
        inv_from_prim(rl, v, u, p, &a1, &a2, &a3, &a4);
        inv_from_prim(s->rho_inf, s->v_inf, s->u_inf, s->p_inf, &f1, &f2, &f3, &f4);
        a1 = o1 ? a1 : f1;
        a2 = o1 ? a2 : f2;
        a3 = o3 ? a3 : f3;
        a4 = o4 ? a4 : f4;
        R nr, nv, nu, np;
        prim_from_inv(a1, a2, a3, a4, &nr, &nv, &nu, &np);
        U[0][c] = nr;
        U[1][c] = nr * nu;
        U[2][c] = nr * nv;
        U[4][c] = np / GM1;
        U[3][c] = U[4][c] + (R)0.5 * nr * (nu * nu + nv * nv);
    }
    if (t == CT_SOLID) {
        U[0][c] = s->rho_inf;
        U[1][c] = 0;
        U[2][c] = 0;
        U[3][c] = e_inf;
        U[4][c] = e_inf;
        return 0;
    }
    return 0;
}

/* phase 2: immersed-boundary ghost cell from the best fluid neighbour of the
 * snapshot S (src/solver.cu:2045-2225). */
static void bc_ghost(const orc_solver *s, R *const S[5], R *const U[5], int i, int j) {
    const int nx = s->nx, ny = s->ny;
    size_t c = (size_t)j * nx + i;
    const R *sdf = s->sdf;
    R sxp = (i < nx - 1) ? sdf[c + 1] : sdf[c];
    R sxm = (i > 0) ? sdf[c - 1] : sdf[c];
    R syp = (j < ny - 1) ? sdf[c + nx] : sdf[c];
    R sym = (j > 0) ? sdf[c - nx] : sdf[c];
    R gx = (sxp - sxm) / ((R)2.0 * s->dx);
    R gy = (syp - sym) / ((R)2.0 * s->dy);
    R len = SQRT(gx * gx + gy * gy) + (R)1e-10;
    gx /= len;
    gy /= len;
    static const int nb[8][2] = {{-1, 0}, {1, 0}, {0, -1}, {0, 1}, {-1, -1}, {1, -1}, {-1, 1}, {1, 1}};
    long best = -1;
    R best_dot = (R)-1;
    for (int k = 0; k < 8; k++) {
        int ni = i + nb[k][0], nj = j + nb[k][1];
        if (ni < 0 || ni >= nx || nj < 0 || nj >= ny) continue;
        size_t q = (size_t)nj * nx + ni;
        if (sdf[q] > 0 && S[0][q] >= MIN_DENSITY) {
            R dxn = (R)nb[k][0], dyn = (R)nb[k][1];
            R l = SQRT(dxn * dxn + dyn * dyn);
            R dot = (dxn * gx + dyn * gy) / l;
            if (dot > best_dot) {
                best_dot = dot;
                best = (long)q;
            }
        }
    }
    R e_inf = s->p_inf / GM1;
    if (best < 0) {
        U[0][c] = s->rho_inf;
        U[1][c] = 0;
        U[2][c] = 0;
        U[3][c] = e_inf;
        U[4][c] = e_inf;
        return;
    }
    R rf = S[0][best];
    R uf = S[1][best] / rf;
    R vf = S[2][best] / rf;
    R Ef = S[3][best];
    R kef = (R)0.5 * rf * (uf * uf + vf * vf);
    R pf = GM1 * (Ef - kef);
    rf = fmaxR(rf, MIN_DENSITY);
    pf = fmaxR(pf, MIN_PRESSURE);
    R vn = uf * gx + vf * gy;
    R vt = -vf * gx + uf * gy;
    R Tf = pf / (rf * R_GAS);
    Tf = fminR(Tf, MAX_TEMPERATURE);
    Tf = fmaxR(Tf, MIN_TEMPERATURE);
    pf = rf * R_GAS * Tf;
    R ug, vg;
    if (s->viscous) {
        ug = -uf;
        vg = -vf;
    } else {
        R slip = 0;
        if (vn > 0) slip = fminR(SLIP_MAX, vn / (vn + SLIP_VREF));
        R uns = -uf, vns = -vf;
        R us = -vn * gx + vt * gy;
        R vs = -vn * gy - vt * gx;
        ug = ((R)1 - slip) * uns + slip * us;
        vg = ((R)1 - slip) * vns + slip * vs;
    }
    R vmag = SQRT(ug * ug + vg * vg);
    if (vmag > MAX_GHOST_VEL) {
        R sc = MAX_GHOST_VEL / vmag;
        ug *= sc;
        vg *= sc;
    }
    R Tg;
    if (s->adiabatic) {
        Tg = Tf;
    } else {
        Tg = (R)2.0 * s->T_wall - Tf;
        Tg = fmaxR(Tg, MIN_TEMPERATURE);
        Tg = fminR(Tg, MAX_TEMPERATURE);
    }
    R pg = pf;
    R rg = pg / (R_GAS * Tg);
    rg = fmaxR(rg, MIN_DENSITY);
    R eg = pg / GM1;
    R keg = (R)0.5 * rg * (ug * ug + vg * vg);
    U[0][c] = rg;
    U[1][c] = rg * ug;
    U[2][c] = rg * vg;
    U[3][c] = eg + keg;
    U[4][c] = eg;
}

static void apply_bc(orc_solver *s, R *const U[5]) {
    const int nx = s->nx, ny = s->ny;
#pragma omp parallel for schedule(static)
    for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) bc_pointwise(s, U, i, j);
    for (int k = 0; k < 5; k++) memcpy(s->snap[k], U[k], s->n * sizeof(R));
#pragma omp parallel for schedule(static)
    for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++)
            if (s->ct[(size_t)j * nx + i] == CT_GHOST && i != 0 && i != nx - 1) bc_ghost(s, s->snap, U, i, j);
}

/* sspRK2BlendKernel (src/solver.cu:949-967) */
static void blend(orc_solver *s, R *const A[5], R *const B[5]) {
#pragma omp parallel for schedule(static)
    for (size_t c = 0; c < s->n; c++)
        for (int k = 0; k < 5; k++) A[k][c] = (R)0.5 * A[k][c] + (R)0.5 * B[k][c];
}

/* ====================================================== viscous terms
 * fusedViscousDiffusionKernel (src/solver.cu:2251-2511): Sutherland mu,
 * Newtonian stress (Stokes hypothesis), Fourier heat flux, viscous work and
 * dissipation, forward Euler on rho_u, rho_v, E, rho_e of interior fluid cells;
 * writes mu for every cell (solid: 0). */
static inline R sutherland(R T) {
    R tr = T / T_REF;
    return MU_REF * (tr * SQRT(tr)) * (T_REF + S_SUTH) / (T + S_SUTH);
}

static void viscous_stress(const orc_solver *s, int i, int j, R t5[5]) {
    const int nx = s->nx, ny = s->ny;
    size_t c = (size_t)j * nx + i;
    const R inv_2dx = (R)0.5 / s->dx, inv_2dy = (R)0.5 / s->dy;
    const R inv_dx = (R)1 / s->dx, inv_dy = (R)1 / s->dy;
    if (s->ct[c] == CT_SOLID) {
        for (int k = 0; k < 5; k++) t5[k] = 0;
        return;
    }
    const R *u = s->u, *v = s->v, *T = s->T;
    R mu = sutherland(T[c]);
    R kk = mu * CP / s->prandtl;
    size_t xp = i < nx - 1 ? c + 1 : c, xm = i > 0 ? c - 1 : c;
    size_t yp = j < ny - 1 ? c + nx : c, ym = j > 0 ? c - nx : c;
    R dudx = (u[xp] - u[xm]) * inv_2dx, dudy = (u[yp] - u[ym]) * inv_2dy;
    R dvdx = (v[xp] - v[xm]) * inv_2dx, dvdy = (v[yp] - v[ym]) * inv_2dy;
    if (i == 0) { dudx = (u[xp] - u[c]) * inv_dx; dvdx = (v[xp] - v[c]) * inv_dx; }
    else if (i == nx - 1) { dudx = (u[c] - u[xm]) * inv_dx; dvdx = (v[c] - v[xm]) * inv_dx; }
    if (j == 0) { dudy = (u[yp] - u[c]) * inv_dy; dvdy = (v[yp] - v[c]) * inv_dy; }
    else if (j == ny - 1) { dudy = (u[c] - u[ym]) * inv_dy; dvdy = (v[c] - v[ym]) * inv_dy; }
    R div = dudx + dvdy;
    const R two3 = (R)2.0 / (R)3.0;
    t5[0] = mu * ((R)2.0 * dudx - two3 * div);
    t5[1] = mu * ((R)2.0 * dvdy - two3 * div);
    t5[2] = mu * (dudy + dvdx);
    R dTdx = (T[xp] - T[xm]) * inv_2dx, dTdy = (T[yp] - T[ym]) * inv_2dy;
    if (i == 0) dTdx = (T[xp] - T[c]) * inv_dx;
    else if (i == nx - 1) dTdx = (T[c] - T[xm]) * inv_dx;
    if (j == 0) dTdy = (T[yp] - T[c]) * inv_dy;
    else if (j == ny - 1) dTdy = (T[c] - T[ym]) * inv_dy;
    t5[3] = -kk * dTdx;
    t5[4] = -kk * dTdy;
}

/* U <- U + dt * D(prims of U); the caller must have made s->u,v,T = prims(U). */
static void viscous(orc_solver *s, R *const U[5], R dt) {
    const int nx = s->nx, ny = s->ny;
#pragma omp parallel for schedule(static)
    for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
            size_t c = (size_t)j * nx + i;
            R t5[5];
            viscous_stress(s, i, j, t5);
            for (int k = 0; k < 5; k++) s->tau[k][c] = t5[k];
            s->mu[c] = (s->ct[c] == CT_SOLID) ? (R)0 : sutherland(s->T[c]);
        }
    const R inv_2dx = (R)0.5 / s->dx, inv_2dy = (R)0.5 / s->dy;
#pragma omp parallel for schedule(static)
    for (int j = 1; j < ny - 1; j++)
        for (int i = 1; i < nx - 1; i++) {
            size_t c = (size_t)j * nx + i;
            if (is_wall(s->ct[c])) continue;
            R *txx = s->tau[0], *tyy = s->tau[1], *txy = s->tau[2], *qx = s->tau[3], *qy = s->tau[4];
            const R *u = s->u, *v = s->v;
            R dtxx = (txx[c + 1] - txx[c - 1]) * inv_2dx;
            R dtxy_y = (txy[c + nx] - txy[c - nx]) * inv_2dy;
            R dtxy_x = (txy[c + 1] - txy[c - 1]) * inv_2dx;
            R dtyy = (tyy[c + nx] - tyy[c - nx]) * inv_2dy;
            R dqx = (qx[c + 1] - qx[c - 1]) * inv_2dx;
            R dqy = (qy[c + nx] - qy[c - nx]) * inv_2dy;
            R dudx = (u[c + 1] - u[c - 1]) * inv_2dx;
            R dudy = (u[c + nx] - u[c - nx]) * inv_2dy;
            R dvdx = (v[c + 1] - v[c - 1]) * inv_2dx;
            R dvdy = (v[c + nx] - v[c - nx]) * inv_2dy;
            R phi = txx[c] * dudx + tyy[c] * dvdy + txy[c] * (dudy + dvdx);
            R rhs_ru = dtxx + dtxy_y;
            R rhs_rv = dtxy_x + dtyy;
            R wxp = u[c + 1] * txx[c + 1] + v[c + 1] * txy[c + 1];
            R wxm = u[c - 1] * txx[c - 1] + v[c - 1] * txy[c - 1];
            R wyp = u[c + nx] * txy[c + nx] + v[c + nx] * tyy[c + nx];
            R wym = u[c - nx] * txy[c - nx] + v[c - nx] * tyy[c - nx];
            R dwx = (wxp - wxm) * inv_2dx;
            R dwy = (wyp - wym) * inv_2dy;
            R rhs_E = -dqx - dqy + dwx + dwy;
            R rhs_re = -dqx - dqy + phi;
            U[1][c] += dt * rhs_ru;
            U[2][c] += dt * rhs_rv;
            U[3][c] += dt * rhs_E;
            U[4][c] += dt * rhs_re;
        }
}

/* ============================================================ step chain */
static void fill_mu(orc_solver *s) {
    for (size_t c = 0; c < s->n; c++) s->mu[c] = (s->ct[c] == CT_SOLID) ? (R)0 : sutherland(s->T[c]);
}

void orc_reset(orc_solver *s) {
    initialize(s);
    compute_sdf(s);
    apply_bc(s, s->U);
    primitives(s, s->U);
    fill_mu(s); /* the reference runs the viscous kernel with dt = 0 for mu */
}

void orc_set_geometry(orc_solver *s, const float *sdf, const uint8_t *ct) {
    for (size_t c = 0; c < s->n; c++) {
        s->sdf[c] = (R)sdf[c];
        s->ct[c] = ct[c];
    }
}

void orc_reinit(orc_solver *s) {
    initialize(s);
    apply_bc(s, s->U);
    primitives(s, s->U);
    fill_mu(s);
}

void orc_compute_sdf(orc_solver *s, float *sdf_out, uint8_t *ct_out) {
    compute_sdf(s);
    for (size_t c = 0; c < s->n; c++) {
        if (sdf_out) sdf_out[c] = (float)s->sdf[c];
        if (ct_out) ct_out[c] = s->ct[c];
    }
}

/* updateSDFWithFixupKernel (src/solver.cu:607-664): newly exposed fluid cells
 * get a zero state (the reference's behaviour), then BC and primitives. */
void orc_update_obstacle(orc_solver *s) {
    uint8_t *old = (uint8_t *)malloc(s->n);
    memcpy(old, s->ct, s->n);
    compute_sdf(s);
    for (size_t c = 0; c < s->n; c++) {
        int was = old[c] == CT_SOLID || old[c] == CT_GHOST;
        if (was && s->ct[c] == CT_FLUID)
            for (int k = 0; k < 5; k++) s->U[k][c] = 0;
    }
    free(old);
    apply_bc(s, s->U);
    primitives(s, s->U);
}

/* CFDSolver::step (src/solver.cu:3289-3412) */
void orc_step(orc_solver *s, double dt_in) {
    R dt = (R)dt_in;
    if (s->viscous) {
        R half = dt * (R)0.5;
        viscous(s, s->U, half);
        primitives(s, s->U);
    }
    fluxes(s, s->U);
    update(s, s->U, s->Us, dt);
    apply_bc(s, s->Us);
    primitives(s, s->Us);
    fluxes(s, s->Us);
    update(s, s->Us, s->Uk, dt);
    blend(s, s->U, s->Uk);
    if (s->viscous) {
        primitives(s, s->U);
        viscous(s, s->U, dt * (R)0.5);
    }
    apply_bc(s, s->U);
    primitives(s, s->U);
}

void orc_stage1(orc_solver *s, double dt, int with_ghost, double *out5[5]) {
    fluxes(s, s->U);
    update(s, s->U, s->Us, (R)dt);
    if (with_ghost) {
        apply_bc(s, s->Us);
    } else {
        const int nx = s->nx, ny = s->ny;
        for (int j = 0; j < ny; j++)
            for (int i = 0; i < nx; i++) bc_pointwise(s, s->Us, i, j);
    }
    for (int k = 0; k < 5; k++)
        if (out5[k])
            for (size_t c = 0; c < s->n; c++) out5[k][c] = (double)s->Us[k][c];
}

/* computeWaveSpeedKernel / computeViscousNumberKernel (src/solver.cu:2679-2739) */
void orc_cfl_maxima(orc_solver *s, double *max_speed, double *max_nu) {
    R ms = -INFINITY, mn = -INFINITY;
    for (size_t c = 0; c < s->n; c++) {
        R cc = SQRT(GAMMA * s->p[c] / (s->U[0][c] + (R)1e-10));
        R sp = SQRT(s->u[c] * s->u[c] + s->v[c] * s->v[c]) + cc;
        if (sp > ms) ms = sp;
        R nu = s->mu[c] / (s->U[0][c] + (R)1e-10);
        if (nu > mn) mn = nu;
    }
    if (max_speed) *max_speed = (double)ms;
    if (max_nu) *max_nu = (double)mn;
}

/* readTimeStepResult (src/solver.cu:3250-3265) */
double orc_compute_dt(orc_solver *s) {
    double ms, mn;
    orc_cfl_maxima(s, &ms, &mn);
    R min_dx = fminR(s->dx, s->dy);
    R dt = s->cfl * min_dx / ((R)ms + (R)1e-10);
    if (s->viscous) {
        R dv = s->cfl_visc * min_dx * min_dx / ((R)mn + (R)1e-10);
        dt = fminR(dt, dv);
    }
    return (double)dt;
}

/* ============================================================ accessors */
void orc_get_fields(orc_solver *s, double *rho, double *ru, double *rv, double *E, double *re) {
    double *o[5] = {rho, ru, rv, E, re};
    for (int k = 0; k < 5; k++)
        if (o[k])
            for (size_t c = 0; c < s->n; c++) o[k][c] = (double)s->U[k][c];
}
void orc_set_fields(orc_solver *s, const double *rho, const double *ru, const double *rv, const double *E,
                    const double *re) {
    const double *in[5] = {rho, ru, rv, E, re};
    for (int k = 0; k < 5; k++)
        if (in[k])
            for (size_t c = 0; c < s->n; c++) s->U[k][c] = (R)in[k][c];
    primitives(s, s->U);
    fill_mu(s);
}
void orc_get_primitives(orc_solver *s, double *u, double *v, double *p, double *T) {
    for (size_t c = 0; c < s->n; c++) {
        if (u) u[c] = (double)s->u[c];
        if (v) v[c] = (double)s->v[c];
        if (p) p[c] = (double)s->p[c];
        if (T) T[c] = (double)s->T[c];
    }
}
void orc_get_mu(orc_solver *s, double *mu) {
    for (size_t c = 0; c < s->n; c++) mu[c] = (double)s->mu[c];
}
void orc_get_geometry(orc_solver *s, double *sdf, uint8_t *ct) {
    for (size_t c = 0; c < s->n; c++) {
        if (sdf) sdf[c] = (double)s->sdf[c];
        if (ct) ct[c] = s->ct[c];
    }
}

/* ========================================================== diagnostics
 * No reference counterpart.  Wall faces are faces between a wall cell
 * (solid/ghost) and a non-wall cell.  On each, the force on the obstacle is
 * (-p_face n + tau.n) dA with n the unit normal from the wall cell to the
 * fluid cell, p_face the reference's wall-face pressure (the left/bottom
 * cell's p, src/solver.cu:1594,1679) and tau the fluid cell's viscous stress
 * (viscous runs only).  Wall heat = -(q.n) dA into the wall, q = -k grad T at
 * the fluid cell (viscous runs only). */
void orc_diagnostics(orc_solver *s, fvm_diag *out) {
    const int nx = s->nx, ny = s->ny;
    double fx = 0, fy = 0, mass = 0, mx = 0, my = 0, en = 0, heat = 0, hmax = 0;
    double dxd = (double)s->dx, dyd = (double)s->dy, area = dxd * dyd;
    for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
            size_t c = (size_t)j * nx + i;
            if (!is_wall(s->ct[c])) {
                mass += (double)s->U[0][c] * area;
                mx += (double)s->U[1][c] * area;
                my += (double)s->U[2][c] * area;
                en += (double)s->U[3][c] * area;
            }
            for (int dir = 0; dir < 2; dir++) {
                if (dir == 0 && i >= nx - 1) continue;
                if (dir == 1 && j >= ny - 1) continue;
                size_t b = dir == 0 ? c + 1 : c + (size_t)nx;
                int wa = is_wall(s->ct[c]), wb = is_wall(s->ct[b]);
                if (wa == wb) continue;
                /* n: from wall cell to fluid cell along the axis */
                double sgn = wa ? 1.0 : -1.0; /* a wall, b fluid: +axis */
                size_t f = wa ? b : c;
                int fi = wa ? (dir == 0 ? i + 1 : i) : i;
                int fj = wa ? (dir == 0 ? j : j + 1) : j;
                double dA = dir == 0 ? dyd : dxd;
                double nxn = dir == 0 ? sgn : 0.0, nyn = dir == 1 ? sgn : 0.0;
                double pf = (double)s->p[c];
                double fxx = -pf * nxn * dA, fyy = -pf * nyn * dA;
                if (s->viscous) {
                    R t5[5];
                    viscous_stress(s, fi, fj, t5);
                    fxx += ((double)t5[0] * nxn + (double)t5[2] * nyn) * dA;
                    fyy += ((double)t5[2] * nxn + (double)t5[1] * nyn) * dA;
                    double qn = (double)t5[3] * nxn + (double)t5[4] * nyn;
                    double qw = -qn;
                    heat += qw * dA;
                    if (qw > hmax) hmax = qw;
                }
                (void)f;
                fx += fxx;
                fy += fyy;
            }
        }
    memset(out, 0, sizeof(*out));
    out->force_x = fx;
    out->force_y = fy;
    double q_inf = 0.5 * (double)s->rho_inf * (double)s->u_inf * (double)s->u_inf;
    double L = s->ext.ref_length > 0 ? (double)s->ext.ref_length : 2.0 * (double)s->obs_r;
    out->cd = (q_inf > 0 && L > 0) ? fx / (q_inf * L) : 0.0;
    out->cl = (q_inf > 0 && L > 0) ? fy / (q_inf * L) : 0.0;
    out->mass = mass;
    out->mom_x = mx;
    out->mom_y = my;
    out->energy = en;
    out->wall_heat = heat;
    out->wall_heat_max = hmax;
}

/* Shock standoff on row j = ny/2 (no reference counterpart): obstacle surface
 * = first sign change of the sdf scanning from the inflow, shock = first
 * crossing of p_mid = p_inf + 0.5*(p2 - p_inf), p2 the normal-shock pressure
 * (Rankine-Hugoniot) at the freestream Mach number; both linearly
 * interpolated between cell centres.  Returns NaN when either is missing. */
double orc_shock_standoff(orc_solver *s) {
    const int nx = s->nx, j = s->ny / 2;
    double dxd = (double)s->dx;
    double xb = NAN;
    int ib = -1;
    for (int i = 0; i + 1 < nx; i++) {
        double a = (double)s->sdf[(size_t)j * nx + i], b = (double)s->sdf[(size_t)j * nx + i + 1];
        if (a > 0 && b <= 0) {
            xb = ((double)i + 0.5) * dxd + dxd * a / (a - b);
            ib = i;
            break;
        }
    }
    if (ib < 0) return NAN;
    double g = 1.4, pinf = (double)s->p_inf;
    double cinf = sqrt(g * pinf / (double)s->rho_inf);
    double M = (double)s->u_inf / cinf;
    if (M <= 1.0) return NAN;
    double p2 = pinf * (1.0 + 2.0 * g / (g + 1.0) * (M * M - 1.0));
    double pm = pinf + 0.5 * (p2 - pinf);
    for (int i = 1; i <= ib; i++) {
        double a = (double)s->p[(size_t)j * nx + i - 1], b = (double)s->p[(size_t)j * nx + i];
        if (a < pm && b >= pm) {
            double xs = ((double)(i - 1) + 0.5) * dxd + dxd * (pm - a) / (b - a);
            return xb - xs;
        }
    }
    return NAN;
}


/* ------------------------------------------------------------ colour images
 * Renderer::generate{Jet,Hot,Plasma,Inferno,Viridis}Colormap
 * (src/renderer.cpp:672-716, 719-734, 737-754, 757-779, 782-799), t = i/255. */
static float clampf01(float x, float lo, float hi) { return x < lo ? lo : (x > hi ? hi : x); }

void orc_colormap_table(int cmap, float rgb[768]) {
    for (int i = 0; i < 256; i++) {
        const float t = (float)i / 255.0f;
        float c[3];
        if (cmap == 0) { /* jet: five linear pieces */
            if (t < 0.125f) { c[0] = 0.0f; c[1] = 0.0f; c[2] = 0.5f + 4.0f * t; }
            else if (t < 0.375f) { c[0] = 0.0f; c[1] = 4.0f * (t - 0.125f); c[2] = 1.0f; }
            else if (t < 0.625f) { c[0] = 4.0f * (t - 0.375f); c[1] = 1.0f; c[2] = 1.0f - 4.0f * (t - 0.375f); }
            else if (t < 0.875f) { c[0] = 1.0f; c[1] = 1.0f - 4.0f * (t - 0.625f); c[2] = 0.0f; }
            else { c[0] = 1.0f - 4.0f * (t - 0.875f); c[1] = 0.0f; c[2] = 0.0f; }
        } else if (cmap == 1) { /* hot */
            c[0] = t * 2.5f < 1.0f ? t * 2.5f : 1.0f;
            c[1] = clampf01((t - 0.4f) * 2.5f, 0.0f, 1.0f);
            c[2] = (t - 0.8f) * 5.0f > 0.0f ? (t - 0.8f) * 5.0f : 0.0f;
        } else if (cmap == 2) { /* plasma: cubic / quartic fits */
            c[0] = 0.050383f + t * (2.028462f + t * (-1.312035f + t * 0.233106f));
            c[1] = 0.029803f + t * (0.192182f + t * (1.429032f + t * (-1.651143f + t * 0.500000f)));
            c[2] = 0.527975f + t * (1.573141f + t * (-2.481592f + t * 0.880392f));
            for (int k = 0; k < 3; k++) c[k] = clampf01(c[k], 0.0f, 1.0f);
        } else if (cmap == 3) { /* inferno: the generator's final (linear) form */
            c[0] = clampf01(1.5f * t, 0.0f, 1.0f);
            c[1] = clampf01(2.0f * (t - 0.25f), 0.0f, 1.0f);
            c[2] = clampf01(0.6f - 1.2f * t, 0.0f, 0.6f);
        } else { /* viridis: cubic fits */
            c[0] = 0.267004f + t * (0.003991f + t * (0.494266f + t * 0.234652f));
            c[1] = 0.004874f + t * (1.014627f + t * (-0.531556f + t * 0.512042f));
            c[2] = 0.329415f + t * (1.423671f + t * (-2.252694f + t * 0.499477f));
            for (int k = 0; k < 3; k++) c[k] = clampf01(c[k], 0.0f, 1.0f);
        }
        for (int k = 0; k < 3; k++) rgb[3 * i + k] = c[k];
    }
}

/* FIELD_FRAGMENT_SHADER (src/renderer.cpp:47-77) per cell: classes 1 and 2
 * (cellType in (0.5, 2.5)) grey 0.3; otherwise clamp((v-lo)/(hi-lo+1e-4)),
 * then the OpenGL LINEAR / CLAMP_TO_EDGE lookup of a 256-texel 1-D texture:
 * u = s*256 - 1/2, texels floor(u) and floor(u)+1 clamped to [0,255],
 * weights 1-frac(u), frac(u).  RGBA8 = round-to-nearest(c*255). */
void orc_colormap(const float *field, const uint8_t *ct, long n, int cmap, float lo, float hi, int fmt, void *out) {
    float tab[768];
    orc_colormap_table(cmap, tab);
    for (long e = 0; e < n; e++) {
        float c[3];
        if (ct[e] == 1 || ct[e] == 2) {
            c[0] = c[1] = c[2] = 0.3f;
        } else {
            float sn = clampf01((field[e] - lo) / (hi - lo + 0.0001f), 0.0f, 1.0f);
            float u = sn * 256.0f - 0.5f;
            float fl = floorf(u);
            float w = u - fl;
            int a = (int)fl, b = (int)fl + 1;
            a = a < 0 ? 0 : (a > 255 ? 255 : a);
            b = b < 0 ? 0 : (b > 255 ? 255 : b);
            for (int k = 0; k < 3; k++) c[k] = (1.0f - w) * tab[3 * a + k] + w * tab[3 * b + k];
        }
        if (fmt == 0) {
            float *o = (float *)out + 4 * e;
            o[0] = c[0]; o[1] = c[1]; o[2] = c[2]; o[3] = 1.0f;
        } else {
            uint8_t *o = (uint8_t *)out + 4 * e;
            for (int k = 0; k < 3; k++) o[k] = (uint8_t)nearbyintf(clampf01(c[k], 0.0f, 1.0f) * 255.0f);
            o[3] = 255;
        }
    }
}
