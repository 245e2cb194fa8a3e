// fvm_geometry.cu -- obstacle signed distance, cell marking, the per-cell
// mask byte, the static ghost-cell table, freestream initialisation and the
// geometry-change fix-up.  Set-up path (runs on reset / obstacle updates).
//
// The SDF expressions restate the reference (src/solver.cu:67-589) in the
// same FP32 order; compiled with the reference's --use_fast_math the cell
// classes come out bit-identical.
#include "fvm_internal.cuh"
#include "fvm_kernels.cuh"

namespace fvm {

constexpr float SDF_BAND = 1.5f;
constexpr float STAR_RATIO = 0.38f;
constexpr float DIAMOND_K = 0.7071f;
constexpr float CAPSULE_HALF_LEN = 1.5f;
constexpr float CAPSULE_CAP = 0.5f;
constexpr float TRI_K = 0.866025404f;

__device__ __forceinline__ float seg_dist(float px, float py, float ax, float ay, float bx, float by) {
    float abx = bx - ax, aby = by - ay;
    float apx = px - ax, apy = py - ay;
    float t = (apx * abx + apy * aby) / (abx * abx + aby * aby + 1e-10f);
    t = fmaxf(0.0f, fminf(1.0f, t));
    float closestX = ax + t * abx;
    float closestY = ay + t * aby;
    float ddx = px - closestX;
    float ddy = py - closestY;
    return sqrtf(ddx * ddx + ddy * ddy);
}

__device__ __forceinline__ float cross2(float ax, float ay, float bx, float by) { return ax * by - ay * bx; }

// rotation into the shape frame: (lx, ly) by -rot
__device__ __forceinline__ void to_local(float px, float py, float cx, float cy, float rot, float &qx, float &qy) {
    float lx = px - cx;
    float ly = py - cy;
    float cosR = cosf(-rot);
    float sinR = sinf(-rot);
    qx = lx * cosR - ly * sinR;
    qy = lx * sinR + ly * cosR;
}

__device__ __forceinline__ float sdf_circle(float px, float py, float cx, float cy, float r) {
    return sqrtf((px - cx) * (px - cx) + (py - cy) * (py - cy)) - r;
}

// 5-point star: 10-vertex polygon, winding-number inside test (src/solver.cu:179-240)
__device__ __forceinline__ float sdf_star(float px, float py, float cx, float cy, float r, float rot) {
    const int N = 5;
    const float outerR = r;
    const float innerR = r * STAR_RATIO;
    float qx, qy;
    to_local(px, py, cx, cy, rot, qx, qy);
    float verts[20];
    for (int i = 0; i < N; i++) {
        float outerAngle = 2.0f * PI_F * i / N - PI_F / 2.0f;
        float innerAngle = outerAngle + PI_F / N;
        verts[i * 4 + 0] = outerR * cosf(outerAngle);
        verts[i * 4 + 1] = outerR * sinf(outerAngle);
        verts[i * 4 + 2] = innerR * cosf(innerAngle);
        verts[i * 4 + 3] = innerR * sinf(innerAngle);
    }
    float minDist = 1e10f;
    float windingSum = 0.0f;
    for (int i = 0; i < 2 * N; i++) {
        int j = (i + 1) % (2 * N);
        float ax = verts[i * 2], ay = verts[i * 2 + 1];
        float bx = verts[j * 2], by = verts[j * 2 + 1];
        float d = seg_dist(qx, qy, ax, ay, bx, by);
        minDist = fminf(minDist, d);
        float eax = ax - qx, eay = ay - qy;
        float ebx = bx - qx, eby = by - qy;
        windingSum += atan2f(cross2(eax, eay, ebx, eby), eax * ebx + eay * eby);
    }
    float sign = (fabsf(windingSum) > PI_F) ? -1.0f : 1.0f;
    return sign * minDist;
}

// diamond (src/solver.cu:252-272)
__device__ __forceinline__ float sdf_diamond(float px, float py, float cx, float cy, float r, float rot) {
    float rx, ry;
    to_local(px, py, cx, cy, rot, rx, ry);
    float ndx = fabsf(rx) / r;
    float ndy = fabsf(ry) / r;
    return (ndx + ndy - 1.0f) * r * DIAMOND_K;
}

// stadium capsule (src/solver.cu:284-311)
__device__ __forceinline__ float sdf_capsule(float px, float py, float cx, float cy, float r, float rot) {
    float rx, ry;
    to_local(px, py, cx, cy, rot, rx, ry);
    float halfWidth = r * CAPSULE_HALF_LEN;
    float capRadius = r * CAPSULE_CAP;
    float clampedX = fmaxf(-halfWidth + capRadius, fminf(halfWidth - capRadius, rx));
    float ddx = rx - clampedX;
    float ddy = ry;
    return sqrtf(ddx * ddx + ddy * ddy) - capRadius;
}

// equilateral triangle, tip on +x (src/solver.cu:323-362)
__device__ __forceinline__ float sdf_triangle(float px, float py, float cx, float cy, float r, float rot) {
    float qx, qy;
    to_local(px, py, cx, cy, rot, qx, qy);
    const float sqrt3_2 = TRI_K;
    float v0x = r, v0y = 0.0f;
    float v1x = -r * 0.5f, v1y = r * sqrt3_2;
    float v2x = -r * 0.5f, v2y = -r * sqrt3_2;
    float d0 = seg_dist(qx, qy, v0x, v0y, v1x, v1y);
    float d1 = seg_dist(qx, qy, v1x, v1y, v2x, v2y);
    float d2 = seg_dist(qx, qy, v2x, v2y, v0x, v0y);
    float minDist = fminf(d0, fminf(d1, d2));
    float c0 = cross2(v1x - v0x, v1y - v0y, qx - v0x, qy - v0y);
    float c1 = cross2(v2x - v1x, v2y - v1y, qx - v1x, qy - v1y);
    float c2 = cross2(v0x - v2x, v0y - v2y, qx - v2x, qy - v2y);
    bool inside = (c0 >= 0 && c1 >= 0 && c2 >= 0) || (c0 <= 0 && c1 <= 0 && c2 <= 0);
    return inside ? -minDist : minDist;
}

// convex quadrilateral, counter-clockwise vertices (src/solver.cu:374-399)
__device__ __forceinline__ float sdf_quad(float px, float py, float v0x, float v0y, float v1x, float v1y, float v2x,
                                          float v2y, float v3x, float v3y) {
    float d0 = seg_dist(px, py, v0x, v0y, v1x, v1y);
    float d1 = seg_dist(px, py, v1x, v1y, v2x, v2y);
    float d2 = seg_dist(px, py, v2x, v2y, v3x, v3y);
    float d3 = seg_dist(px, py, v3x, v3y, v0x, v0y);
    float minDist = fminf(fminf(d0, d1), fminf(d2, d3));
    float c0 = cross2(v1x - v0x, v1y - v0y, px - v0x, py - v0y);
    float c1 = cross2(v2x - v1x, v2y - v1y, px - v1x, py - v1y);
    float c2 = cross2(v3x - v2x, v3y - v2y, px - v2x, py - v2y);
    float c3 = cross2(v0x - v3x, v0y - v3y, px - v3x, py - v3y);
    bool inside = (c0 >= 0 && c1 >= 0 && c2 >= 0 && c3 >= 0) || (c0 <= 0 && c1 <= 0 && c2 <= 0 && c3 <= 0);
    return inside ? -minDist : minDist;
}

// starship: body circle, mirrored fixed root quad, rotating flap quad
// (src/solver.cu:414-486; vertex table src/include/common.h:28-36)
__device__ __forceinline__ float sdf_starship(float px, float py, float cx, float cy, float r, float rot, float wing) {
    const float rootRadius = 90.0f;
    float qx, qy;
    to_local(px, py, cx, cy, rot, qx, qy);
    float distToCircle = sqrtf(qx * qx + qy * qy) - r;
    float scale = r / rootRadius;
    float refX = qx / scale;
    float refY = fabsf(qy) / scale;
    float distToRoot =
        sdf_quad(refX, refY, -45.0f, 77.9422f, 10.9682f, 89.329f, 6.0f, 112.0f, -6.0f, 112.0f) * scale;
    const float pivotX = -6.0f, pivotY = 112.0f;
    float cosW = cosf(-wing);
    float sinW = sinf(-wing);
    float wv0x = pivotX, wv0y = pivotY;
    float dx1 = 6.0f - pivotX, dy1 = 112.0f - pivotY;
    float wv1x = pivotX + dx1 * cosW - dy1 * sinW;
    float wv1y = pivotY + dx1 * sinW + dy1 * cosW;
    float dx2 = 3.0f - pivotX, dy2 = 186.0f - pivotY;
    float wv2x = pivotX + dx2 * cosW - dy2 * sinW;
    float wv2y = pivotY + dx2 * sinW + dy2 * cosW;
    float dx3 = -3.0f - pivotX, dy3 = 186.0f - pivotY;
    float wv3x = pivotX + dx3 * cosW - dy3 * sinW;
    float wv3y = pivotY + dx3 * sinW + dy3 * cosW;
    float distToWing = sdf_quad(refX, refY, wv0x, wv0y, wv1x, wv1y, wv2x, wv2y, wv3x, wv3y) * scale;
    return fminf(distToCircle, fminf(distToRoot, distToWing));
}

// Blunted cone (no reference counterpart): nose circle radius r centred at
// (cx, cy) facing -x, tangent frustum of half angle `ang` extending `len`
// along +x from the tangent points; union = min(circle, convex quad).
__device__ __forceinline__ float sdf_cone_capsule(float px, float py, float cx, float cy, float r, float rot,
                                                  float ang, float len) {
    float qx, qy;
    to_local(px, py, cx, cy, rot, qx, qy);
    float circ = sqrtf(qx * qx + qy * qy) - r;
    float sa = sinf(ang), ca = cosf(ang);
    float tx = -r * sa, ty = r * ca;
    float bx = tx + len, by = ty + len * (sa / ca);
    float quad = sdf_quad(qx, qy, tx, -ty, bx, -by, bx, by, tx, ty);
    return fminf(circ, quad);
}

struct ShapeArgs {
    float ox, oy, r, rot, wing, cone_ang, cone_len;
    int shape;
};

__device__ __forceinline__ float shape_sdf(float px, float py, const ShapeArgs &s) {
    switch (s.shape) {
    case 0: return sdf_circle(px, py, s.ox, s.oy, s.r);
    case 1: return sdf_star(px, py, s.ox, s.oy, s.r, s.rot);
    case 2: return sdf_diamond(px, py, s.ox, s.oy, s.r, s.rot);
    case 3: return sdf_capsule(px, py, s.ox, s.oy, s.r, s.rot);
    case 4: return sdf_triangle(px, py, s.ox, s.oy, s.r, s.rot);
    case 5: return sdf_starship(px, py, s.ox, s.oy, s.r, s.rot, s.wing);
    case 6: return sdf_cone_capsule(px, py, s.ox, s.oy, s.r, s.rot, s.cone_ang, s.cone_len);
    default: return sdf_circle(px, py, s.ox, s.oy, s.r);
    }
}

__device__ __forceinline__ uint8_t classify(float dist, float band, int i, int nx) {
    uint8_t t;
    if (dist < -band)
        t = CT_SOLID;
    else if (dist < band && dist >= -band)
        t = CT_GHOST;
    else
        t = CT_FLUID;
    if (i == 0)
        t = CT_INFLOW;
    else if (i == nx - 1)
        t = CT_OUTFLOW;
    return t;
}

// computeSDFKernel (src/solver.cu:536-589) and, with `fix` non-null, the
// fix-up of updateSDFWithFixupKernel (src/solver.cu:607-664): cells that turn
// from solid/ghost to fluid get a zero state, as in the reference.
__global__ void k_sdf(GridDesc g, ShapeArgs s, float *sdf, uint8_t *ct, float *fix_state) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= g.nx || j >= g.ny) return;
    size_t dense = (size_t)j * g.nx + i;
    size_t pidx = (size_t)j * g.pitch + i;
    float x = (i + 0.5f) * g.dx;
    float y = (j + 0.5f) * g.dy;
    float dist = shape_sdf(x, y, s);
    sdf[pidx] = dist;
    float band = SDF_BAND * fmaxf(g.dx, g.dy);
    uint8_t t = classify(dist, band, i, g.nx);
    if (fix_state) {
        uint8_t old = ct[dense];
        bool was = (old == CT_SOLID || old == CT_GHOST);
        if (was && t == CT_FLUID)
            for (int k = 0; k < 5; k++) fix_state[k * g.plane + pidx] = 0.0f;
    }
    ct[dense] = t;
}

__device__ __forceinline__ bool is_wall_ct(uint8_t t) { return t == CT_SOLID || t == CT_GHOST; }

// Mask byte of each cell (see fvm_math.cuh), from the dense cell classes.
__global__ void k_mask(GridDesc g, const uint8_t *ct, uint8_t *mask) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= g.nx || j >= g.ny) return;
    const int nx = g.nx, ny = g.ny;
    auto at = [&](int ii, int jj) {
        ii = max(0, min(ii, nx - 1));
        jj = max(0, min(jj, ny - 1));
        return ct[(size_t)jj * nx + ii];
    };
    uint8_t t = at(i, j);
    uint32_t m = (uint32_t)t << MB_TYPE_SHIFT;
    if (is_wall_ct(t)) m |= MB_WALL;
    if (i < nx - 1) {
        if (!is_wall_ct(t) && !is_wall_ct(at(i + 1, j))) m |= MB_XV;
        if (is_wall_ct(at(i - 1, j)) || is_wall_ct(at(i + 2, j))) m |= MB_XN;
    }
    if (j < ny - 1) {
        if (!is_wall_ct(t) && !is_wall_ct(at(i, j + 1))) m |= MB_YV;
        if (is_wall_ct(at(i, j - 1)) || is_wall_ct(at(i, j + 2))) m |= MB_YN;
    }
    mask[(size_t)j * g.pitch + i] = (uint8_t)m;
}

// Ghost-cell table: count pass (list == nullptr) or fill pass.
// Normal and neighbour dot products use the reference's expressions
// (src/solver.cu:2054-2098); a candidate must have sdf > 0 and dot > -1 (the
// reference's initial best_dot), its density is checked at run time.
__global__ void k_ghost_table(GridDesc g, const float *sdf, const uint8_t *ct, GhostInfo *list, int cap,
                              int *count) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= g.nx || j >= g.ny) return;
    const int nx = g.nx, ny = g.ny;
    if (ct[(size_t)j * nx + i] != CT_GHOST) return;
    int slot = atomicAdd(count, 1);
    if (!list || slot >= cap) return;
    size_t c = (size_t)j * g.pitch + i;
    float sdf_xp = (i < nx - 1) ? sdf[c + 1] : sdf[c];
    float sdf_xm = (i > 0) ? sdf[c - 1] : sdf[c];
    float sdf_yp = (j < ny - 1) ? sdf[c + g.pitch] : sdf[c];
    float sdf_ym = (j > 0) ? sdf[c - g.pitch] : sdf[c];
    float gx = (sdf_xp - sdf_xm) / (2.0f * g.dx);
    float gy = (sdf_yp - sdf_ym) / (2.0f * g.dy);
    float norm_len = sqrtf(gx * gx + gy * gy) + 1e-10f;
    gx /= norm_len;
    gy /= norm_len;
    float dots[8];
    int codes[8];
    int n = 0;
    for (int k = 0; k < 8; k++) {
        int di, dj;
        ghost_neighbour(k, di, dj);
        int ni = i + di, nj = j + dj;
        if (ni < 0 || ni >= nx || nj < 0 || nj >= ny) continue;
        size_t q = (size_t)nj * g.pitch + ni;
        if (!(sdf[q] > 0.0f)) continue;
        float dir_x = (float)di;
        float dir_y = (float)dj;
        float len = sqrtf(dir_x * dir_x + dir_y * dir_y);
        float dot = (dir_x * gx + dir_y * gy) / len;
        if (!(dot > -1.0f)) continue;
        int code = k | ((ct[(size_t)nj * nx + ni] == CT_GHOST) ? 8 : 0);
        // stable insertion by descending dot (earlier neighbour wins ties)
        int p = n;
        while (p > 0 && dots[p - 1] < dot) {
            dots[p] = dots[p - 1];
            codes[p] = codes[p - 1];
            --p;
        }
        dots[p] = dot;
        codes[p] = code;
        ++n;
    }
    uint32_t cand = 0;
    for (int k = 0; k < n; k++) cand |= (uint32_t)codes[k] << (4 * k);
    GhostInfo gi;
    gi.i = i;
    gi.j = j;
    gi.gx = gx;
    gi.gy = gy;
    gi.cand = cand;
    gi.count = n;
    list[slot] = gi;
}

// initializeKernel (src/solver.cu:911-940)
__global__ void k_init(GridDesc g, float *U, Freestream fs) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= g.nx || j >= g.ny) return;
    size_t c = (size_t)j * g.pitch + i;
    U[c] = fs.rho;
    U[g.plane + c] = fs.rho * fs.u;
    U[2 * g.plane + c] = fs.rho * fs.v;
    float ke = 0.5f * fs.rho * (fs.u * fs.u + fs.v * fs.v);
    float e_internal = fs.p / (GAMMA - 1.0f);
    U[3 * g.plane + c] = e_internal + ke;
    U[4 * g.plane + c] = e_internal;
}

// ------------------------------------------------------------ host launchers
static dim3 grid2d(const GridDesc &g, dim3 b) { return dim3((g.nx + b.x - 1) / b.x, (g.ny + b.y - 1) / b.y); }

void launch_sdf(const GridDesc &g, const ShapeParamsHost &s, float *sdf, uint8_t *ct, float *fix_state,
                cudaStream_t st) {
    ShapeArgs a{s.ox, s.oy, s.r, s.rot, s.wing, s.cone_ang, s.cone_len, s.shape};
    dim3 b(32, 8);
    k_sdf<<<grid2d(g, b), b, 0, st>>>(g, a, sdf, ct, fix_state);
}

void launch_mask(const GridDesc &g, const uint8_t *ct, uint8_t *mask, cudaStream_t st) {
    dim3 b(32, 8);
    k_mask<<<grid2d(g, b), b, 0, st>>>(g, ct, mask);
}

void launch_ghost_table(const GridDesc &g, const float *sdf, const uint8_t *ct, GhostInfo *list, int cap, int *count,
                        cudaStream_t st) {
    dim3 b(32, 8);
    k_ghost_table<<<grid2d(g, b), b, 0, st>>>(g, sdf, ct, list, cap, count);
}

void launch_init(const GridDesc &g, float *U, const Freestream &fs, cudaStream_t st) {
    dim3 b(32, 8);
    k_init<<<grid2d(g, b), b, 0, st>>>(g, U, fs);
}

}  // namespace fvm
