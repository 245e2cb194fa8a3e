// fvm_aux.cu -- off-step kernels behind the reference's readback / statistics
// API: derived fields into device buffers, max-temperature / max-Mach
// reductions, velocity arrows, FP64 diagnostics and the shock standoff scan.
#include "fvm_kernels.cuh"
#include "fvm_tma.cuh"

namespace fvm {

__global__ void k_primitives(GridDesc g, const float *U, float *u, float *v, float *p, float *T) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= g.nx || j >= g.ny) return;
    size_t c = (size_t)j * g.pitch + i, d = (size_t)j * g.nx + i;
    float uu, vv, pp, TT;
    prim_from_cons(U[c], U[g.plane + c], U[2 * g.plane + c], U[3 * g.plane + c], U[4 * g.plane + c], uu, vv, pp, TT);
    if (u) u[d] = uu;
    if (v) v[d] = vv;
    if (p) p[d] = pp;
    if (T) T[d] = TT;
}

// Derived field into a dense nx*ny destination.
__global__ void k_derived(int kind, GridDesc g, const float *U, float *dst) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= g.nx || j >= g.ny) return;
    size_t c = (size_t)j * g.pitch + i, d = (size_t)j * g.nx + i;
    dst[d] = derived_value(kind, U[c], U[g.plane + c], U[2 * g.plane + c], U[4 * g.plane + c]);
}

// The renderer's field pass (FIELD_FRAGMENT_SHADER, src/renderer.cpp:47-77)
// with one pixel per cell: SOLID and GHOST cells dark grey, others the
// derived value normalised by (v - lo) / (hi - lo + 1e-4), clamped to [0, 1],
// then looked up in the 256-entry colour table the way a linearly filtered,
// edge-clamped 1-D texture samples it.  fmt 0: RGBA float, fmt 1: RGBA8.
__global__ void k_colormap(int kind, GridDesc g, const float *U, const uint8_t *ct,
                           const __grid_constant__ ColormapLUT lut, float lo, float hi, void *out, int fmt) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= g.nx || j >= g.ny) return;
    const size_t c = (size_t)j * g.pitch + i, d = (size_t)j * g.nx + i;
    const uint8_t t = ct[d];
    float r, gr, b;
    if (t == CT_SOLID || t == CT_GHOST) {
        r = gr = b = 0.3f;
    } else {
        const float v = derived_value(kind, U[c], U[g.plane + c], U[2 * g.plane + c], U[4 * g.plane + c]);
        const float s = fminf(fmaxf((v - lo) / (hi - lo + 0.0001f), 0.0f), 1.0f);
        const float u = s * 256.0f - 0.5f;
        const float fl = floorf(u);
        const float a = u - fl;
        const int i0 = min(max((int)fl, 0), 255), i1 = min(max((int)fl + 1, 0), 255);
        r = (1.0f - a) * lut.rgb[3 * i0] + a * lut.rgb[3 * i1];
        gr = (1.0f - a) * lut.rgb[3 * i0 + 1] + a * lut.rgb[3 * i1 + 1];
        b = (1.0f - a) * lut.rgb[3 * i0 + 2] + a * lut.rgb[3 * i1 + 2];
    }
    if (fmt == 0) {
        reinterpret_cast<float4 *>(out)[d] = make_float4(r, gr, b, 1.0f);
    } else {
        auto q = [](float x) { return (unsigned)__float2int_rn(fminf(fmaxf(x, 0.0f), 1.0f) * 255.0f); };
        reinterpret_cast<uchar4 *>(out)[d] = make_uchar4(q(r), q(gr), q(b), 255);
    }
}

// cellTypeToFloatKernel (src/solver.cu:3444-3450)
__global__ void k_ct_to_float(long long n, const uint8_t *ct, float *dst) {
    long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (e < n) dst[e] = static_cast<float>(ct[e]);
}

// what = 0: max temperature of the primitives (getMaxTemperature,
// src/solver.cu:2835-2867); what = 1: max local Mach (computeMachNumberKernel,
// src/solver.cu:2782-2794).  out_dev must be zeroed by the caller.
__global__ void __launch_bounds__(256) k_max_reduce(int what, GridDesc g, const float *U, float *out_dev) {
    float m = 0.0f;
    const long long n = (long long)g.nx * g.ny;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(e / g.nx), i = (int)(e % g.nx);
        const size_t c = (size_t)j * g.pitch + i;
        float u, v, p, T;
        const float rho = U[c];
        prim_from_cons(rho, U[g.plane + c], U[2 * g.plane + c], U[3 * g.plane + c], U[4 * g.plane + c], u, v, p, T);
        if (what == 0) {
            m = fmaxf(m, T);
        } else {
            float rho_val = rho + 1e-10f;
            float speed = sqrtf(u * u + v * v);
            float cs = sqrtf(GAMMA * p / rho_val);
            m = fmaxf(m, speed / (cs + 1e-10f));
        }
    }
    __shared__ float ws[8];
    m = warp_max(m);
    if ((threadIdx.x & 31) == 0) ws[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        float mm = 0.0f;
        for (int k = 0; k < 8; k++) mm = fmaxf(mm, ws[k]);
        atomic_max_nonneg(out_dev, mm);
    }
}

// generateVectorArrowsKernel (src/solver.cu:3689-3796).  Slots come from an
// atomic counter like the reference; writes past `cap_vertices` are skipped
// (the reference does not check), the counter still reports the total.
__global__ void k_arrows(GridDesc g, const float *U, float *vertexData, int *counter, int cap_vertices, int step,
                         float u_inf, float maxArrowLength, float arrowHeadAngle, float arrowHeadLength) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int j = blockIdx.y * blockDim.y + threadIdx.y;
    i = i * step + step / 2;
    j = j * step + step / 2;
    if (i >= g.nx || j >= g.ny) return;
    size_t c = (size_t)j * g.pitch + i;
    float u_val, v_val, pp, TT;
    prim_from_cons(U[c], U[g.plane + c], U[2 * g.plane + c], U[3 * g.plane + c], U[4 * g.plane + c], u_val, v_val,
                   pp, TT);
    float speed = sqrtf(u_val * u_val + v_val * v_val);
    if (speed < 1e-6f * u_inf) return;
    float normalizedSpeed = fminf(speed / (u_inf * 1.5f), 1.0f);
    float startX = (float)i / g.nx * 2.0f - 1.0f;
    float startY = (float)j / g.ny * 2.0f - 1.0f;
    float dirX = u_val / speed;
    float dirY = v_val / speed;
    float arrowLength = maxArrowLength * normalizedSpeed;
    float endX = startX + dirX * arrowLength;
    float endY = startY + dirY * arrowLength;
    float headLen = arrowLength * arrowHeadLength;
    float cosA = cosf(arrowHeadAngle);
    float sinA = sinf(arrowHeadAngle);
    float head1X = endX - headLen * (dirX * cosA - dirY * sinA);
    float head1Y = endY - headLen * (dirX * sinA + dirY * cosA);
    float head2X = endX - headLen * (dirX * cosA + dirY * sinA);
    float head2Y = endY - headLen * (-dirX * sinA + dirY * cosA);
    int vertexOffset = atomicAdd(counter, 8);
    if (vertexOffset + 8 > cap_vertices) return;
    float *o = vertexData + (size_t)vertexOffset * 5;
    const float xs[6] = {startX, endX, endX, head1X, endX, head2X};
    const float ys[6] = {startY, endY, endY, head1Y, endY, head2Y};
    for (int k = 0; k < 6; k++) {
        o[k * 5 + 0] = xs[k];
        o[k * 5 + 1] = ys[k];
        o[k * 5 + 2] = 0.0f;
        o[k * 5 + 3] = 0.0f;
        o[k * 5 + 4] = 0.0f;
    }
}

// ---------------------------------------------------------------- diagnostics
// FP64 wall forces, heat flux and conserved totals (no reference counterpart).
// Wall faces lie between a wall cell (solid/ghost) and a non-wall cell; the
// force on the obstacle is (-p_face n + tau.n) dA, n the unit normal from the
// wall cell to the fluid cell, p_face the pressure of the left/bottom cell
// (the reference's wall-face flux, src/solver.cu:1594,1679), tau and q at the
// fluid cell.  Per-CTA partials then one ordered final sum: deterministic.
constexpr int kDiag = 8;  // fx, fy, mass, mx, my, E, heat, heat_max

struct DiagCtx {
    GridDesc g;
    const float *U;
    const uint8_t *mask;
    ViscArgs va;
};

__device__ __forceinline__ void prim_at(const DiagCtx &d, int i, int j, float &u, float &v, float &p, float &T) {
    size_t c = (size_t)j * d.g.pitch + i;
    const long long pl = d.g.plane;
    prim_from_cons(d.U[c], d.U[pl + c], d.U[2 * pl + c], d.U[3 * pl + c], d.U[4 * pl + c], u, v, p, T);
}

__device__ void stress_at(const DiagCtx &d, int i, int j, float out[5]) {
    const int nx = d.g.nx, ny = d.g.ny;
    float uC, vC, pC, TC, uE, vE, pE, TE, uW, vW, pW, TW, uN, vN, pN, TN, uS, vS, pS, TS;
    prim_at(d, i, j, uC, vC, pC, TC);
    prim_at(d, min(i + 1, nx - 1), j, uE, vE, pE, TE);
    prim_at(d, max(i - 1, 0), j, uW, vW, pW, TW);
    prim_at(d, i, min(j + 1, ny - 1), uN, vN, pN, TN);
    prim_at(d, i, max(j - 1, 0), uS, vS, pS, TS);
    stress_heat(uC, vC, TC, uE, uW, uN, uS, vE, vW, vN, vS, TE, TW, TN, TS, i == 0, i == nx - 1, j == 0, j == ny - 1,
                d.va, out);
}

__global__ void __launch_bounds__(256) k_diag_partial(DiagCtx d, int viscous, double *partials) {
    double acc[kDiag];
    for (int k = 0; k < kDiag; k++) acc[k] = 0.0;
    const GridDesc g = d.g;
    const long long n = (long long)g.nx * g.ny;
    const double dxd = g.dx, dyd = g.dy, area = dxd * dyd;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(e / g.nx), i = (int)(e % g.nx);
        const size_t c = (size_t)j * g.pitch + i;
        const bool wa = (d.mask[c] & MB_WALL) != 0;
        if (!wa) {
            acc[2] += (double)d.U[c] * area;
            acc[3] += (double)d.U[g.plane + c] * area;
            acc[4] += (double)d.U[2 * g.plane + c] * area;
            acc[5] += (double)d.U[3 * g.plane + c] * area;
        }
        for (int dir = 0; dir < 2; dir++) {
            if (dir == 0 && i >= g.nx - 1) continue;
            if (dir == 1 && j >= g.ny - 1) continue;
            const size_t b = dir == 0 ? c + 1 : c + g.pitch;
            const bool wb = (d.mask[b] & MB_WALL) != 0;
            if (wa == wb) continue;
            const double sgn = wa ? 1.0 : -1.0;
            const int fi = wa ? (dir == 0 ? i + 1 : i) : i;
            const int fj = wa ? (dir == 0 ? j : j + 1) : j;
            const double dA = dir == 0 ? dyd : dxd;
            const double nxn = dir == 0 ? sgn : 0.0, nyn = dir == 1 ? sgn : 0.0;
            float u, v, p, T;
            prim_at(d, i, j, u, v, p, T);
            double fx = -(double)p * nxn * dA, fy = -(double)p * nyn * dA;
            if (viscous) {
                float t5[5];
                stress_at(d, fi, fj, t5);
                fx += ((double)t5[0] * nxn + (double)t5[2] * nyn) * dA;
                fy += ((double)t5[2] * nxn + (double)t5[1] * nyn) * dA;
                const double qw = -((double)t5[3] * nxn + (double)t5[4] * nyn);
                acc[6] += qw * dA;
                acc[7] = fmax(acc[7], qw);
            }
            acc[0] += fx;
            acc[1] += fy;
        }
    }
    __shared__ double s[kDiag][256];
    for (int k = 0; k < kDiag; k++) s[k][threadIdx.x] = acc[k];
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w)
            for (int k = 0; k < kDiag; k++)
                s[k][threadIdx.x] = (k == 7) ? fmax(s[k][threadIdx.x], s[k][threadIdx.x + w])
                                             : s[k][threadIdx.x] + s[k][threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0)
        for (int k = 0; k < kDiag; k++) partials[(size_t)blockIdx.x * kDiag + k] = s[k][0];
}

__global__ void k_diag_final(const double *partials, int nparts, double *out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    double acc[kDiag];
    for (int k = 0; k < kDiag; k++) acc[k] = 0.0;
    for (int b = 0; b < nparts; b++)
        for (int k = 0; k < kDiag; k++)
            acc[k] = (k == 7) ? fmax(acc[k], partials[(size_t)b * kDiag + k]) : acc[k] + partials[(size_t)b * kDiag + k];
    for (int k = 0; k < kDiag; k++) out[k] = acc[k];
}

// Shock standoff along row ny/2 (see fvm_b200.h); one thread scans the row.
__global__ void k_standoff(GridDesc g, const float *U, const float *sdf, double p_mid, double *out) {
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    const int j = g.ny / 2;
    const double dxd = g.dx;
    int ib = -1;
    double xb = 0.0;
    for (int i = 0; i + 1 < g.nx; i++) {
        double a = sdf[(size_t)j * g.pitch + i], b = sdf[(size_t)j * g.pitch + i + 1];
        if (a > 0 && b <= 0) {
            xb = (i + 0.5) * dxd + dxd * a / (a - b);
            ib = i;
            break;
        }
    }
    *out = __longlong_as_double(0x7ff8000000000000ULL);
    if (ib < 0) return;
    float pprev = 0.0f;
    for (int i = 0; i <= ib; i++) {
        size_t c = (size_t)j * g.pitch + i;
        float u, v, p, T;
        prim_from_cons(U[c], U[g.plane + c], U[2 * g.plane + c], U[3 * g.plane + c], U[4 * g.plane + c], u, v, p, T);
        if (i > 0 && (double)pprev < p_mid && (double)p >= p_mid) {
            double xs = (i - 1 + 0.5) * dxd + dxd * (p_mid - (double)pprev) / ((double)p - (double)pprev);
            *out = xb - xs;
            return;
        }
        pprev = p;
    }
}

// ------------------------------------------------------------- launchers
static dim3 grid2d(const GridDesc &g, dim3 b) { return dim3((g.nx + b.x - 1) / b.x, (g.ny + b.y - 1) / b.y); }

cudaError_t launch_primitives(const GridDesc &g, const float *U, float *u, float *v, float *p, float *T,
                              cudaStream_t st) {
    dim3 b(32, 8);
    k_primitives<<<grid2d(g, b), b, 0, st>>>(g, U, u, v, p, T);
    return cudaGetLastError();
}

cudaError_t launch_colormap(int kind, const GridDesc &g, const float *U, const uint8_t *ct, const ColormapLUT &lut,
                            float lo, float hi, void *out, int fmt, cudaStream_t st) {
    dim3 b(32, 8);
    k_colormap<<<grid2d(g, b), b, 0, st>>>(kind, g, U, ct, lut, lo, hi, out, fmt);
    return cudaGetLastError();
}

cudaError_t launch_derived(int kind, const GridDesc &g, const float *U, float *dst, cudaStream_t st) {
    dim3 b(32, 8);
    k_derived<<<grid2d(g, b), b, 0, st>>>(kind, g, U, dst);
    return cudaGetLastError();
}

cudaError_t launch_ct_to_float(const GridDesc &g, const uint8_t *ct, float *dst, cudaStream_t st) {
    long long n = (long long)g.nx * g.ny;
    k_ct_to_float<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, ct, dst);
    return cudaGetLastError();
}

cudaError_t launch_max_reduce(int what, const GridDesc &g, const float *U, float *out_dev, cudaStream_t st) {
    long long n = (long long)g.nx * g.ny;
    int blocks = (int)((n + 255) / 256);
    if (blocks > 148 * 8) blocks = 148 * 8;
    k_max_reduce<<<blocks, 256, 0, st>>>(what, g, U, out_dev);
    return cudaGetLastError();
}

cudaError_t launch_arrows_cap(const GridDesc &g, const float *U, float *vertex, int cap, int *counter, int step,
                              float u_inf, float max_len, float head_angle, float head_len, cudaStream_t st) {
    int ax = (g.nx + step - 1) / step, ay = (g.ny + step - 1) / step;
    dim3 b(16, 16), gr((ax + 15) / 16, (ay + 15) / 16);
    k_arrows<<<gr, b, 0, st>>>(g, U, vertex, counter, cap, step, u_inf, max_len, head_angle, head_len);
    return cudaGetLastError();
}

int diagnostics_parts(const GridDesc &g) {
    long long n = (long long)g.nx * g.ny;
    long long b = (n + 255) / 256;
    return (int)(b < 592 ? b : 592);
}

cudaError_t launch_diagnostics(const GridDesc &g, const float *U, const uint8_t *ct, const uint8_t *mask, int viscous,
                               float prandtl, int ref_prandtl, double *partials, int nparts, double *out8,
                               cudaStream_t st) {
    (void)ct;
    DiagCtx d;
    d.g = g;
    d.U = U;
    d.mask = mask;
    d.va = viscous_args(g.dx, g.dy, prandtl, ref_prandtl != 0);
    k_diag_partial<<<nparts, 256, 0, st>>>(d, viscous, partials);
    k_diag_final<<<1, 32, 0, st>>>(partials, nparts, out8);
    return cudaGetLastError();
}

cudaError_t launch_standoff(const GridDesc &g, const float *U, const float *sdf, double p_mid, double *out,
                            cudaStream_t st) {
    k_standoff<<<1, 32, 0, st>>>(g, U, sdf, p_mid, out);
    return cudaGetLastError();
}

}  // namespace fvm
