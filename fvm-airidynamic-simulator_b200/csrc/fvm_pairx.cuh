// fvm_pairx.cuh -- what a stage-kernel thread evaluates per step, in packed
// FP32x2 arithmetic: the two x-faces (same column, rows r and r+1), the two
// y-faces (r-2 | r-1) and (r-1 | r), and the update of rows r-2 and r-1.
//
// sm_100 issues two FP32 adds, multiplies or FMAs per instruction
// (__fadd2_rn / __fmul2_rn / __ffma2_rn) at the same FMA throughput as the
// scalar forms, so packing saves issue slots, which is what the stage kernels
// are bound by.  The primitive ring stores each row pair interleaved, {rho_r,
// rho_r+1, u_r, u_r+1} and {v_r, v_r+1, p_r, p_r+1}, so one shared-memory
// vector load yields both rows' operands as aligned register pairs and no
// register moves are needed; lane .x is row r, lane .y row r+1.  The y-faces'
// upper cells straddle two row pairs and are paired from those loads.
// Square roots, reciprocals, min/max and the wave-fan selections stay per
// lane.
//
// The face arithmetic is face_flux_sl + hllc_flux (fvm_math.cuh; reference
// computeFluxesKernel, src/solver.cu:1502-1598 / :1601-1682, and its HLLC,
// :1112-1223 / :1315-1430), the update that of updateKernel (:1736-1875),
// with explicit fused multiply-adds and one approximate reciprocal per
// shared divisor, so results can differ from the reference's in the last
// bits.  The x-face ring stores each row pair interleaved as well, so the
// update's flux differences come out of vector loads as register pairs.
#pragma once
#include "fvm_math.cuh"

namespace fvm {

using f2 = float2;

__device__ __forceinline__ f2 mk2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ f2 splat(float a) { return make_float2(a, a); }
__device__ __forceinline__ f2 p_add(f2 a, f2 b) { return __fadd2_rn(a, b); }
// a - b as a + b*(-1): one rounding, the value of a subtraction
__device__ __forceinline__ f2 p_sub(f2 a, f2 b) { return __ffma2_rn(b, splat(-1.0f), a); }
__device__ __forceinline__ f2 p_mul(f2 a, f2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ f2 p_fma(f2 a, f2 b, f2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ f2 p_min(f2 a, f2 b) { return mk2(fminf(a.x, b.x), fminf(a.y, b.y)); }
__device__ __forceinline__ f2 p_max(f2 a, f2 b) { return mk2(fmaxf(a.x, b.x), fmaxf(a.y, b.y)); }
__device__ __forceinline__ f2 p_max(f2 a, float b) { return mk2(fmaxf(a.x, b), fmaxf(a.y, b)); }
__device__ __forceinline__ f2 p_sqrt(f2 a) { return mk2(sqrtf(a.x), sqrtf(a.y)); }
// per-lane approximate reciprocal, shared by quotients with one divisor
__device__ __forceinline__ f2 p_rcp(f2 a) { return mk2(rcp_approx(a.x), rcp_approx(a.y)); }
// division a / b in the fast approximate form the scalar path uses
// (__fdividef: a times the approximate reciprocal of b, flushed to zero for
// |b| > 2^126), with the two products packed into one instruction
__device__ __forceinline__ f2 p_div(f2 a, f2 b) { return p_mul(a, p_rcp(b)); }
// per-lane approximate reciprocal square root
__device__ __forceinline__ f2 p_rsqrt(f2 a) { return mk2(rsqrtf(a.x), rsqrtf(a.y)); }
__device__ __forceinline__ f2 p_sel(bool cx, bool cy, f2 a, f2 b) { return mk2(cx ? a.x : b.x, cy ? a.y : b.y); }

// Limited slope per lane (as limited_slope).
template <int LIM>
__device__ __forceinline__ f2 p_slope(f2 qm1, f2 q0, f2 qp1) {
    const f2 dL = p_sub(q0, qm1), dR = p_sub(qp1, q0);
    if (LIM == 0) {
        const f2 s = p_mul(splat(0.5f), p_add(mk2(copysignf(1.0f, dL.x), copysignf(1.0f, dL.y)),
                                               mk2(copysignf(1.0f, dR.x), copysignf(1.0f, dR.y))));
        return p_mul(s, mk2(fminf(fabsf(dL.x), fabsf(dR.x)), fminf(fabsf(dL.y), fabsf(dR.y))));
    } else {
        const f2 ab = p_mul(dL, dR);
        const f2 q = p_div(p_mul(splat(2.0f), ab), p_add(dL, dR));
        return mk2(ab.x > 0.0f ? q.x : 0.0f, ab.y > 0.0f ? q.y : 0.0f);
    }
}

// Primitive states of one column for a row pair: lane .x row r, lane .y row r+1.
struct PairPrim {
    f2 rho, u, v, p;
};
__device__ __forceinline__ PairPrim pair_prim(const float4 &A, const float4 &B) {
    return PairPrim{mk2(A.x, A.y), mk2(A.z, A.w), mk2(B.x, B.y), mk2(B.z, B.w)};
}

// Limited slopes of a cell pair in the face frame: normal and tangential
// velocity components (x-faces: u, v; y-faces: v, u).
struct PairSl {
    f2 rho, n, t, p;
};

// Two faces between cells a | b (lane .x: face 0, lane .y: face 1) from the
// cells' primitives and limited slopes sa, sb (face frame); F = {mass,
// x-momentum, y-momentum, energy, rho_e}, each a lane pair.  valid*: neither
// side a wall; near*: first order (wall at the outer stencil cells).
template <bool XDIR>
__device__ __forceinline__ void face_pair_core(bool valid0, bool near0, bool valid1, bool near1, const PairPrim &a,
                                               const PairSl &sa, const PairPrim &b, const PairSl &sb, f2 F[5]) {
    const bool fo0 = near0 || a.rho.x < LOW_DENSITY || b.rho.x < LOW_DENSITY;
    const bool fo1 = near1 || a.rho.y < LOW_DENSITY || b.rho.y < LOW_DENSITY;
    const f2 hp = splat(0.5f);
    const f2 omh = mk2(fo0 ? 0.0f : 0.5f, fo1 ? 0.0f : 0.5f);  // half order mask
    const f2 an = XDIR ? a.u : a.v, at = XDIR ? a.v : a.u;
    const f2 bn = XDIR ? b.u : b.v, bt = XDIR ? b.v : b.u;
    // MUSCL: left = a + slope_a/2, right = b - slope_b/2
    f2 rL = p_fma(sa.rho, omh, a.rho);
    const f2 nL = p_fma(sa.n, omh, an);
    const f2 tL = p_fma(sa.t, omh, at);
    f2 pL = p_fma(sa.p, omh, a.p);
    const f2 omm = mk2(-omh.x, -omh.y);
    f2 rR = p_fma(sb.rho, omm, b.rho);
    const f2 nR = p_fma(sb.n, omm, bn);
    const f2 tR = p_fma(sb.t, omm, bt);
    f2 pR = p_fma(sb.p, omm, b.p);
    rL = p_max(rL, MIN_DENSITY);
    pL = p_max(pL, MIN_PRESSURE);
    rR = p_max(rR, MIN_DENSITY);
    pR = p_max(pR, MIN_PRESSURE);
    // E = p/(gamma-1) + rho*(u^2 + v^2)/2, the x component squared first
    const f2 igm1 = splat(1.0f / (GAMMA - 1.0f));
    const f2 eL = p_mul(pL, igm1), eR = p_mul(pR, igm1);
    const f2 qL = XDIR ? p_fma(nL, nL, p_mul(tL, tL)) : p_fma(tL, tL, p_mul(nL, nL));
    const f2 qR = XDIR ? p_fma(nR, nR, p_mul(tR, tR)) : p_fma(tR, tR, p_mul(nR, nR));
    const f2 EL = p_fma(p_mul(hp, rL), qL, eL);
    const f2 ER = p_fma(p_mul(hp, rR), qR, eR);

    // ---- HLLC with Roe-averaged Davis wave speeds; quotients that share a
    // divisor (1/rho of each side, the Roe weight sum, the star-state
    // denominator) multiply by one reciprocal
    // one reciprocal square root per side gives sqrt(rho) = rho / sqrt(rho)
    // and 1/rho = (1/sqrt(rho))^2
    const f2 rqL = p_rsqrt(rL), rqR = p_rsqrt(rR);
    const f2 sqL = p_mul(rL, rqL), sqR = p_mul(rR, rqR);
    const f2 irL = p_mul(rqL, rqL), irR = p_mul(rqR, rqR);
    const f2 cL = p_sqrt(p_mul(p_mul(splat(GAMMA), pL), irL));
    const f2 cR = p_sqrt(p_mul(p_mul(splat(GAMMA), pR), irR));
    const f2 iden = p_rcp(p_add(p_add(sqL, sqR), splat(1e-10f)));
    const f2 un_roe = p_mul(p_fma(sqL, nL, p_mul(sqR, nR)), iden);
    const f2 ut_roe = p_mul(p_fma(sqL, tL, p_mul(sqR, tR)), iden);
    const f2 HL = p_mul(p_add(EL, pL), irL), HR = p_mul(p_add(ER, pR), irR);
    const f2 H_roe = p_mul(p_fma(sqL, HL, p_mul(sqR, HR)), iden);
    const f2 q_roe = XDIR ? p_fma(un_roe, un_roe, p_mul(ut_roe, ut_roe)) : p_fma(ut_roe, ut_roe, p_mul(un_roe, un_roe));
    const f2 c2 = p_mul(splat(GAMMA - 1.0f), p_fma(splat(-0.5f), q_roe, H_roe));
    const f2 c_avg = p_mul(hp, p_add(cL, cR));
    const f2 c_roe = mk2(c2.x > 0.0f ? sqrtf(c2.x) : c_avg.x, c2.y > 0.0f ? sqrtf(c2.y) : c_avg.y);
    f2 SL = p_min(p_sub(nL, cL), p_sub(un_roe, c_roe));
    f2 SR = p_max(p_add(nR, cR), p_add(un_roe, c_roe));
    const f2 delta = p_mul(splat(ENTROPY_FIX), p_max(cL, cR));
    SL = mk2(fabsf(SL.x) < delta.x ? -delta.x : SL.x, fabsf(SL.y) < delta.y ? -delta.y : SL.y);
    SR = mk2(fabsf(SR.x) < delta.x ? delta.x : SR.x, fabsf(SR.y) < delta.y ? delta.y : SR.y);
    const f2 aL = p_sub(SL, nL), aR = p_sub(SR, nR);
    const f2 mL = p_mul(rL, aL), mR = p_mul(rR, aR);
    const f2 ds = p_sub(mL, mR);
    const f2 sds = mk2(copysignf(fmaxf(fabsf(ds.x), 1e-10f), ds.x), copysignf(fmaxf(fabsf(ds.y), 1e-10f), ds.y));
    const f2 Ss = p_div(p_sub(p_fma(mL, nL, p_sub(pR, pL)), p_mul(mR, nR)), sds);
    // upwind side K of the wave fan (see hllc_flux)
    const bool supL0 = SL.x >= 0.0f, supL1 = SL.y >= 0.0f;
    const bool supR0 = !supL0 && SR.x <= 0.0f, supR1 = !supL1 && SR.y <= 0.0f;
    const bool useL0 = supL0 || (!supR0 && Ss.x >= 0.0f), useL1 = supL1 || (!supR1 && Ss.y >= 0.0f);
    const f2 rK = p_sel(useL0, useL1, rL, rR), nK = p_sel(useL0, useL1, nL, nR), tK = p_sel(useL0, useL1, tL, tR);
    const f2 pK = p_sel(useL0, useL1, pL, pR), EK = p_sel(useL0, useL1, EL, ER), SK = p_sel(useL0, useL1, SL, SR);
    const f2 d = p_sub(SK, nK);   // SK - unK
    const f2 rkd = p_mul(rK, d);  // rK (SK - unK): the same product as mL / mR
    const f2 fK0 = p_mul(rK, nK);
    const f2 fK1 = p_fma(fK0, nK, pK);
    const f2 fK2 = XDIR ? p_mul(fK0, tK) : p_mul(p_mul(rK, tK), nK);  // (rho u) v either way
    const f2 fK3 = p_mul(p_add(EK, pK), nK);
    // |S_K - S*| floored at 1e-10 with its sign (the reference's
    // `cd >= 0 ? 1e-10 : -1e-10`; S_K is never zero after the entropy fix,
    // so the difference is never -0)
    f2 cd = p_sub(SK, Ss);
    cd = mk2(copysignf(fmaxf(fabsf(cd.x), 1e-10f), cd.x), copysignf(fmaxf(fabsf(cd.y), 1e-10f), cd.y));
    const f2 icd = p_rcp(cd);
    const f2 rs = p_max(p_mul(rkd, icd), MIN_DENSITY);
    const f2 ps = p_max(p_fma(rkd, p_sub(Ss, nK), pK), MIN_PRESSURE);
    const f2 Es = p_mul(p_sub(p_fma(EK, d, p_mul(ps, Ss)), p_mul(pK, nK)), icd);
    // star region: F = F_K + S_K (U*_K - U_K); supersonic: F = F_K, written
    // as F_K + 0 * (U*_K - U_K) (there the wave fan keeps |ds| >= rho c, so
    // the star quantities are finite and the product is exactly zero)
    const bool st0 = !(supL0 || supR0), st1 = !(supL1 || supR1);
    const f2 SKs = p_sel(st0, st1, SK, splat(0.0f));
    const f2 F0 = p_fma(SKs, p_sub(rs, rK), fK0);
    const f2 Fn = p_fma(SKs, p_sub(p_mul(rs, Ss), fK0), fK1);
    const f2 Ft = p_fma(SKs, p_mul(p_sub(rs, rK), tK), fK2);
    const f2 F3 = p_fma(SKs, p_sub(Es, EK), fK3);
    // upwinded internal-energy flux
    const f2 uf = p_add(nL, nR);  // sign of 0.5 (unL + unR)
    const f2 F4 = p_sel(uf.x >= 0.0f, uf.y >= 0.0f, p_mul(eL, nL), p_mul(eR, nR));
    const f2 Fx = XDIR ? Fn : Ft, Fy = XDIR ? Ft : Fn;
    // wall faces: no mass/energy flux, normal momentum flux = pressure of the left/bottom cell
    const f2 zero = splat(0.0f);
    F[0] = p_sel(valid0, valid1, F0, zero);
    F[1] = p_sel(valid0, valid1, Fx, XDIR ? a.p : zero);
    F[2] = p_sel(valid0, valid1, Fy, XDIR ? zero : a.p);
    F[3] = p_sel(valid0, valid1, F3, zero);
    F[4] = p_sel(valid0, valid1, F4, zero);
}

// The scalar per-lane fluxes of the AUSM+ path as lane pairs.
__device__ __forceinline__ void pair_from_lanes(const float f0[5], const float f1[5], f2 F[5]) {
#pragma unroll
    for (int k = 0; k < 5; k++) F[k] = mk2(f0[k], f1[k]);
}

// Limited x-slopes of a row pair from the slope ring's interleaved entries
// {rho_r, rho_r+1, u_r, u_r+1}, {v_r, v_r+1, p_r, p_r+1} (x-face frame).
__device__ __forceinline__ PairSl pair_sl(const float4 &A, const float4 &B) {
    return PairSl{mk2(A.x, A.y), mk2(A.z, A.w), mk2(B.x, B.y), mk2(B.z, B.w)};
}

// x-faces of rows r (lane .x) and r+1 (lane .y) between cells a | b from
// their primitives and limited x-slopes sa, sb.
template <int SCHEME>
__device__ __forceinline__ void face_pair_x_sl(bool valid0, bool near0, bool valid1, bool near1, const PairPrim &a,
                                               const PairSl &sa, const PairPrim &b, const PairSl &sb, f2 F[5]) {
    if (SCHEME != 0) {  // AUSM+: per lane through the scalar path
        float f0[5], f1[5];
        const float sa0[4] = {sa.rho.x, sa.n.x, sa.t.x, sa.p.x}, sb0[4] = {sb.rho.x, sb.n.x, sb.t.x, sb.p.x};
        const float sa1[4] = {sa.rho.y, sa.n.y, sa.t.y, sa.p.y}, sb1[4] = {sb.rho.y, sb.n.y, sb.t.y, sb.p.y};
        face_flux_sl<true, SCHEME>(valid0, near0, Prim{a.rho.x, a.u.x, a.v.x, a.p.x}, sa0,
                                   Prim{b.rho.x, b.u.x, b.v.x, b.p.x}, sb0, f0);
        face_flux_sl<true, SCHEME>(valid1, near1, Prim{a.rho.y, a.u.y, a.v.y, a.p.y}, sa1,
                                   Prim{b.rho.y, b.u.y, b.v.y, b.p.y}, sb1, f1);
        pair_from_lanes(f0, f1, F);
        return;
    }
    face_pair_core<true>(valid0, near0, valid1, near1, a, sa, b, sb, F);
}

// The two y-faces a stage-kernel thread evaluates per step, (r-2 | r-1) in
// lane .x and (r-1 | r) in lane .y, from the primitives of rows
// (r-2, r-1) = lo, (r-1, r) = mid and (r, r+1) = hi of one column and the
// y-slopes of row r-2 (carried from the previous step; `sy_lo` in, the slopes
// of row r out for the next step).
template <int SCHEME, int LIM>
__device__ __forceinline__ void face_pair_y(bool valid0, bool near0, bool valid1, bool near1, const PairPrim &lo,
                                            const PairPrim &mid, const PairPrim &hi, float sy_lo[4], f2 F[5]) {
    // slopes of rows (r-1, r): limited(row-1, row, row+1), face frame (v normal, u tangential)
    const PairSl sm{p_slope<LIM>(lo.rho, mid.rho, hi.rho), p_slope<LIM>(lo.v, mid.v, hi.v),
                    p_slope<LIM>(lo.u, mid.u, hi.u), p_slope<LIM>(lo.p, mid.p, hi.p)};
    // slopes of rows (r-2, r-1)
    const PairSl sl{mk2(sy_lo[0], sm.rho.x), mk2(sy_lo[1], sm.n.x), mk2(sy_lo[2], sm.t.x), mk2(sy_lo[3], sm.p.x)};
    if (SCHEME != 0) {  // AUSM+: per lane through the scalar path
        float f0[5], f1[5];
        const float sa0[4] = {sl.rho.x, sl.n.x, sl.t.x, sl.p.x}, sb0[4] = {sm.rho.x, sm.n.x, sm.t.x, sm.p.x};
        const float sb1[4] = {sm.rho.y, sm.n.y, sm.t.y, sm.p.y};
        face_flux_sl<false, SCHEME>(valid0, near0, Prim{lo.rho.x, lo.u.x, lo.v.x, lo.p.x}, sa0,
                                    Prim{mid.rho.x, mid.u.x, mid.v.x, mid.p.x}, sb0, f0);
        face_flux_sl<false, SCHEME>(valid1, near1, Prim{lo.rho.y, lo.u.y, lo.v.y, lo.p.y}, sb0,
                                    Prim{mid.rho.y, mid.u.y, mid.v.y, mid.p.y}, sb1, f1);
        pair_from_lanes(f0, f1, F);
    } else {
        face_pair_core<false>(valid0, near0, valid1, near1, lo, sl, mid, sm, F);
    }
    sy_lo[0] = sm.rho.y;
    sy_lo[1] = sm.n.y;
    sy_lo[2] = sm.t.y;
    sy_lo[3] = sm.p.y;
}

// Face velocities of the rho_e source for two faces (lanes): mass flux over
// the mean of the two cells' clamped densities (src/solver.cu:1772-1794).
__device__ __forceinline__ f2 p_face_velocity(f2 mass, f2 rho_a, f2 rho_b) {
    const f2 mean = p_mul(splat(0.5f), p_add(p_max(rho_a, MIN_DENSITY), p_max(rho_b, MIN_DENSITY)));
    return p_mul(mass, p_rcp(mean));
}

// Rollback of one updated cell (src/solver.cu:1812-1824): a non-finite or
// too small density takes the old one (clamped), a non-finite momentum or
// energy the old value, a non-finite or too small rho_e the old rho_e.  The
// density is >= MIN_DENSITY afterwards, so the reference's second clamp to
// MIN_DENSITY changes nothing and is left out.
__device__ __forceinline__ void rollback_lane(float &rho, float &ru, float &rv, float &E, float &re, float U0, float U1,
                                              float U2, float U3, float U4) {
    if (!isfinite(rho) || rho < MIN_DENSITY) rho = fmaxf(U0, MIN_DENSITY);
    if (!isfinite(ru)) ru = U1;
    if (!isfinite(rv)) rv = U2;
    if (!isfinite(E)) E = U3;
    if (!isfinite(re) || re < MIN_PRESSURE / (GAMMA - 1.0f)) re = U4;
}

// |u| > MAX_VEL (compared in squares): velocity rescaled to MAX_VEL, momenta
// and |u|^2 recomputed (src/solver.cu:1827-1839).
__device__ __forceinline__ void velocity_cap_lane(float rho, float &u, float &v, float &ru, float &rv, float &q) {
    if (q > MAX_VEL * MAX_VEL) {
        const float scale = MAX_VEL / sqrtf(q);
        u *= scale;
        v *= scale;
        ru = rho * u;
        rv = rho * v;
        q = u * u + v * v;
    }
}

// updateKernel body (src/solver.cu:1736-1875) for the two cells of one
// column in rows j (lane .x) and j+1 (lane .y), not walls: U - (dt/dx) dX -
// (dt/dy) dY with dX = F(i+1/2) - F(i-1/2), dY = F(j+1/2) - F(j-1/2) per
// field; the reference zeroes a flux difference across a domain edge
// (i = 0 or nx-1 for x, j = 0 or ny-1 for y), done here by zeroing its
// coefficient.  The rho_e source -p div(v) (interior cells) takes du =
// u(i+1/2) - u(i-1/2) and dv = v(j+1/2) - v(j-1/2) of the face velocities
// and p_c, the cells' primitive pressures.  Then the rollback, the velocity
// cap and the dual-energy resync with e in [rho R T_min, rho R T_max]/(gamma-1).
__device__ __forceinline__ void update_pair(const f2 U[5], const f2 dX[5], const f2 dY[5], f2 du, f2 dv, f2 p_c,
                                            bool edge_x, bool edge_y0, bool edge_y1, const UpdateArgs &a,
                                            f2 out[5]) {
    const f2 ncx = splat(edge_x ? -0.0f : -(a.dt * a.inv_dx));
    const f2 ncy = mk2(edge_y0 ? -0.0f : -(a.dt * a.inv_dy), edge_y1 ? -0.0f : -(a.dt * a.inv_dy));
    f2 n[5];
#pragma unroll
    for (int k = 0; k < 5; k++) n[k] = p_fma(ncy, dY[k], p_fma(ncx, dX[k], U[k]));
    const f2 div_v = p_fma(du, splat(a.inv_dx), p_mul(dv, splat(a.inv_dy)));
    const f2 n4s = p_fma(p_mul(p_c, div_v), splat(-a.dt), n[4]);
    n[4] = p_sel(!edge_x && !edge_y0, !edge_x && !edge_y1, n4s, n[4]);
    rollback_lane(n[0].x, n[1].x, n[2].x, n[3].x, n[4].x, U[0].x, U[1].x, U[2].x, U[3].x, U[4].x);
    rollback_lane(n[0].y, n[1].y, n[2].y, n[3].y, n[4].y, U[0].y, U[1].y, U[2].y, U[3].y, U[4].y);
    const f2 rho = n[0];
    f2 ru = n[1], rv = n[2];
    const f2 E = n[3], re = n[4];
    const f2 inv_rho = p_rcp(rho);
    f2 u = p_mul(ru, inv_rho), v = p_mul(rv, inv_rho);
    f2 q = p_fma(u, u, p_mul(v, v));
    velocity_cap_lane(rho.x, u.x, v.x, ru.x, rv.x, q.x);
    velocity_cap_lane(rho.y, u.y, v.y, ru.y, rv.y, q.y);
    const f2 ke = p_mul(p_mul(splat(0.5f), rho), q);
    const f2 e_from_E = p_sub(E, ke);
    const f2 thr = p_mul(splat(ETA_THRESHOLD), E);  // dual-energy switch rho_e < 1e-3 E, E > 0
    f2 e = p_sel(E.x > 0.0f && re.x < thr.x, E.y > 0.0f && re.y < thr.y, re, e_from_E);
    e = p_min(p_max(e, p_mul(rho, splat(kEminPerRho))), p_mul(rho, splat(kEmaxPerRho)));
    out[0] = rho;
    out[1] = ru;
    out[2] = rv;
    out[3] = p_add(e, ke);
    out[4] = e;
}

// Divergence terms of the viscous half step for one interior fluid cell
// (src/solver.cu:2437-2510): rhs = {d(tau_xx)/dx + d(tau_xy)/dy,
// d(tau_xy)/dx + d(tau_yy)/dy, -div q + div(tau . v), -div q + Phi}, central
// differences of the per-cell quantities stress_heat_work_sel produced, with
// the x and y parts of each derivative pair in one FP32x2 lane pair:
// (dtau_xx/dx, dtau_xy/dx), (dtau_xy/dy, dtau_yy/dy), (dqx/dx, dqy/dy),
// (dwork_x/dx, dwork_y/dy).  {txx, txy, qx, wx} of the east / west
// neighbours, {tyy, txy, qy, wy} of the north / south ones, Phi of the cell.
struct ViscX {
    float txx, txy, qx, wx;
};
struct ViscY {
    float tyy, txy, qy, wy;
};
__device__ __forceinline__ void viscous_rhs_w(const ViscX &E, const ViscX &W, const ViscY &N, const ViscY &S, float phi,
                                              const ViscArgs &va, float rhs[4]) {
    const f2 i2x = splat(va.inv_2dx), i2y = splat(va.inv_2dy), i2xy = mk2(va.inv_2dx, va.inv_2dy);
    const f2 dtx = p_mul(p_sub(mk2(E.txx, E.txy), mk2(W.txx, W.txy)), i2x);  // (dtau_xx_dx, dtau_xy_dx)
    const f2 dty = p_mul(p_sub(mk2(N.txy, N.tyy), mk2(S.txy, S.tyy)), i2y);  // (dtau_xy_dy, dtau_yy_dy)
    const f2 dq = p_mul(p_sub(mk2(E.qx, N.qy), mk2(W.qx, S.qy)), i2xy);      // (dqx_dx, dqy_dy)
    const f2 dw = p_mul(p_sub(mk2(E.wx, N.wy), mk2(W.wx, S.wy)), i2xy);      // (dwork_dx, dwork_dy)
    const f2 r01 = p_add(dtx, dty);
    rhs[0] = r01.x;
    rhs[1] = r01.y;
    rhs[2] = -dq.x - dq.y + dw.x + dw.y;
    rhs[3] = -dq.x - dq.y + phi;
}

}  // namespace fvm
