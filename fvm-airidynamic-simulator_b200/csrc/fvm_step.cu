// fvm_step.cu -- the per-step hot path: fused marching RK-stage kernels, the
// viscous half step, the ghost-cell pass and the CFL reduction.
//
// Structure of a marching kernel.  A CTA of NT threads owns a strip of
// W = NT-4 output columns and `rows` output rows.  It walks the strip from
// bottom to top.  Each incoming row (the 5 conserved planes of the input
// state, columns [i0-4, i0+W+4)) is staged into a shared-memory ring by a 3-D
// TMA load (x, y, field) signalled on an mbarrier, issued ahead of use.  Both
// kernel families advance two rows per step (stage: primitives of the
// incoming rows, their x-faces and two y-faces, update of the two rows two
// behind; viscous: primitives, stress of the two rows one behind, update of
// the two rows two behind), so every face flux is computed exactly once per
// strip and each input cell crosses HBM once (halo re-reads hit L2).
// Domain-edge halos use the reference's clamp-to-edge semantics
// (src/solver.cu:1484-1488): rows by clamping the TMA row coordinate, columns
// by clamping the shared-memory column.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <utility>

#include "fvm_kernels.cuh"
#include "fvm_pairx.cuh"
#include "fvm_tma.cuh"

namespace fvm {

__device__ __forceinline__ int clampi(int v, int lo, int hi) { return max(lo, min(v, hi)); }

__device__ __forceinline__ void record_error(DevScalars *sc, unsigned bit) { atomicOr(&sc->err, bit); }

// Block-wide max of two non-negative values, one atomic per CTA.
template <int NT>
__device__ __forceinline__ void block_max2_publish(float a, float b, float *dst) {
    __shared__ float ws[2][NT / 32];
    a = warp_max(a);
    b = warp_max(b);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) {
        ws[0][w] = a;
        ws[1][w] = b;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        float ma = 0.0f, mb = 0.0f;
        for (int k = 0; k < NT / 32; k++) {
            ma = fmaxf(ma, ws[0][k]);
            mb = fmaxf(mb, ws[1][k]);
        }
        atomic_max_nonneg(&dst[0], ma);
        atomic_max_nonneg(&dst[1], mb);
    }
}

// CFL maxima of the block plus the number of non-finite cells its threads
// saw (one atomic per warp that saw any); every thread of the block calls it.
template <int NT>
__device__ __forceinline__ void block_publish(float a, float b, unsigned bad, DevScalars *sc) {
    block_max2_publish<NT>(a, b, sc->red);
    bad = __reduce_add_sync(0xffffffffu, bad);
    if ((threadIdx.x & 31) == 0 && bad) atomicAdd(&sc->nonfinite, bad);
}

// A conserved state with a NaN or infinite field (their sum is then not
// finite; finite states are far below the float range).
__device__ __forceinline__ unsigned nonfinite5(const float U[5]) {
    return isfinite(U[0] + U[1] + U[2] + U[3] + U[4]) ? 0u : 1u;
}

// Width of one TMA box of the halo'd input (a TMA box spans at most 256
// elements per dimension; 132 floats = 528 B keeps every box start 16-byte
// aligned).  A staged row is NB boxes, each stored as [field][kBox].
constexpr int kBox = 132;
// TMA tensor-copy destinations must be 128-byte aligned: each staged box
// ([5][kBox] floats = 2640 B) occupies a 2688-byte (672-float) stride.
constexpr int kBoxStride = 672;
constexpr size_t align128(size_t b) { return (b + 127) & ~(size_t)127; }

// Address of (field f, staged column x) in a ring slot of NB boxes.
template <int NB>
__device__ __forceinline__ float ring_at(const float *slot_base, int f, int x) {
    if (NB == 1) return slot_base[f * kBox + x];
    const int b = x / kBox;
    return slot_base[b * kBoxStride + f * kBox + (x - b * kBox)];
}

// Dynamic shared memory rounded up to a 128-byte boundary (the launch asks
// for 128 extra bytes).  The dynamic array follows the kernels' static shared
// memory, so its start is only 16-byte aligned and the offset is computed at
// run time.  The result is `p` plus that offset, never a pointer rebuilt from
// an integer, so the compiler still knows it addresses shared memory and
// emits shared loads/stores with 32-bit addressing instead of generic
// accesses with 64-bit address arithmetic.
__device__ __forceinline__ unsigned char *aligned_smem(unsigned char *p) {
    const uint32_t a = smem_addr_opaque(p);
    return p + (((a + 127u) & ~127u) - a);
}

// True (and the error recorded) when the staging area is not 128-byte
// aligned; TMA destinations inside it would be misaligned.  Uniform over the
// CTA, so every thread returns together.
__device__ __forceinline__ bool smem_misaligned(const unsigned char *smem, DevScalars *sc) {
    if ((smem_addr_opaque(smem) & 127u) == 0u) return false;
    if (threadIdx.x == 0) atomicOr(&sc->err, kErrSmemAlign);
    return true;
}

template <int NT, int K, int STAGE>
struct StageLayout {
    static constexpr int W = NT - 4;   // output columns
    static constexpr int NB = (NT + 4 + kBox - 1) / kBox;  // TMA boxes per row
    static constexpr int BW = NB * kBox;  // staged columns [i0-4, i0-4+BW)
    static constexpr int KP = K / 2;   // input ring: K rows staged as K/2 row pairs
    static constexpr int PP = 2;       // primitive / mask ring (row pairs)
    static constexpr int XP = 1;       // x-face ring (row pairs)
    static constexpr int SLOT = NB * kBoxStride;                       // floats per staged input row
    static constexpr int BSLOT = (int)(align128((size_t)5 * W * 4) / 4);  // floats per staged blend row
    static constexpr size_t raw_off = 0;
    static constexpr size_t raw_bytes = (size_t)K * SLOT * 4;
    static constexpr size_t bl_off = raw_off + raw_bytes;
    // stage 2: the blend partner's rows of the row pair updated next, one pair
    static constexpr size_t bl_bytes = STAGE == 2 ? (size_t)2 * BSLOT * 4 : 0;
    static constexpr size_t p_off = bl_off + bl_bytes;
    static constexpr size_t p_bytes = (size_t)PP * 2 * NT * 16;
    // x-slopes of the row pair whose x-faces are evaluated next, one pair
    static constexpr size_t s_off = p_off + p_bytes;
    static constexpr size_t s_bytes = (size_t)2 * NT * 16;
    static constexpr size_t x_off = s_off + s_bytes;
    // x-faces of a row pair, interleaved like the primitives: per column
    // {mass_r, mass_r+1, x-mom_r, x-mom_r+1}, {y-mom, energy}, {rho_e flux,
    // face velocity}, three float4 planes
    static constexpr size_t x_bytes = (size_t)XP * 3 * NT * 16;
    static constexpr size_t m_off = x_off + x_bytes;
    static constexpr size_t m_bytes = (size_t)PP * 2 * NT;
    static constexpr size_t bar_off = (m_off + m_bytes + 15) & ~(size_t)15;
    static constexpr int NBAR = KP + (STAGE == 2 ? 1 : 0);  // input pairs + the blend pair
    static constexpr size_t total = bar_off + NBAR * 8 + 128;  // + alignment slack
    static constexpr uint32_t tx_bytes = 2 * 5 * BW * 4;       // one input row pair
    static constexpr uint32_t btx_bytes = 2 * 5 * W * 4;       // one blend row pair
};

// Slot bookkeeping of a row ring of N slots: rotating the indices of the
// last few rows avoids integer division in the row loop.
template <int N>
__device__ __forceinline__ int ring_next(int s) {
    return (s + 1 == N) ? 0 : s + 1;
}

// TMA ring position carried across the tiles a CTA processes: `base` counts
// input row pairs staged so far (slot = base % KP, mbarrier phase parity
// (base / KP) & 1 for the pair staged at `base`); `bbase` counts the blend
// row pairs staged so far (one slot; phase parity bbase & 1).
struct RingPos {
    int base;
    int bbase;
};

// Inviscid SSP-RK2 stage on one tile (strip [i0, i0+W) x rows [j0, j1))
// (computeFluxesKernel + updateKernel + [blend] + phase-1 BC,
// src/solver.cu:1450-1876, :949-967, :1891-2042), marching two rows per step.
// Per step q (incoming rows r = j0-2+2q and r+1):
//   phase 1  primitives + masks of rows r, r+1 (one column per thread)
//   -- barrier --
//   phase 2  y-faces (r-2|r-1), (r-1|r) of column i0+t and the update of
//            rows r-2, r-1 at column i0+t (x-faces of those rows from step
//            q-1); then the limited x-slopes of rows r, r+1 at column i0-1+t
//   -- barrier --
//   phase 3  x-faces of rows r, r+1 (thread t: the face left of column i0+t)
//            from the primitives and x-slopes of the two cells beside it
// The thread that computes a column's y-faces also updates that column, so
// y-fluxes stay in registers (the face below row r-2 is carried from the
// previous step).  Every cell's x-slopes are computed once and read by both
// of its x-faces.  After the second barrier nothing reads the previous row
// pair's input slot or primitives again, which keeps the rings at K/2 input
// pairs, 2 primitive pairs, 1 slope pair and 1 x-face pair.  Stage 2 stages
// the blend partner's rows of pair q into one blend slot after the second
// barrier of step q (the update of pair q-1 has read the slot by then); the
// update of pair q in step q+1 waits for them with the input.  Returns
// false when a bounded wait expired (error recorded; caller must stop).
template <int NT, int K, int STAGE, int SCHEME, int LIM, bool DISP = false>
__device__ __forceinline__ bool stage_tile(const CUtensorMap *tm_in, const CUtensorMap *tm_blend, const StepArgs &a,
                                           int i0, int j0, unsigned char *smem, RingPos &rp, float &lmax_speed,
                                           unsigned &nbad) {
    using L = StageLayout<NT, K, STAGE>;
    constexpr int W = L::W, KP = L::KP;
    static_assert(L::PP == 2 && L::XP == 1 && KP >= 2, "ring sizes");
    float *raw = reinterpret_cast<float *>(smem + L::raw_off);
    float *bl = reinterpret_cast<float *>(smem + L::bl_off);
    // primitives of a row pair, interleaved: PA = {rho_r, rho_r+1, u_r, u_r+1},
    // PB = {v_r, v_r+1, p_r, p_r+1}, one float4 each per column and pair slot
    float4 *PA = reinterpret_cast<float4 *>(smem + L::p_off);
    float4 *PB = PA + L::PP * NT;
    // x-slopes of a row pair, interleaved like the primitives (face frame:
    // normal u, tangential v): SA = {rho_r, rho_r+1, u_r, u_r+1}, SB = {v, p}
    float4 *SA = reinterpret_cast<float4 *>(smem + L::s_off);
    float4 *SB = SA + NT;
    float4 *XA = reinterpret_cast<float4 *>(smem + L::x_off);  // [column]: mass, x-momentum
    float4 *XB = XA + NT;                                         // y-momentum, energy
    float4 *XC = XB + NT;                                         // rho_e flux, face velocity
    uint8_t *M = smem + L::m_off;
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + L::bar_off);
    uint64_t *bbar = bars + KP;  // blend pair (stage 2)

    const GridDesc g = a.g;
    const int nx = g.nx, ny = g.ny;
    const int t = threadIdx.x;
    const int j1 = min(j0 + a.rows_per_cta, ny);
    const int rs = j0 - 2;
    const int npairs = (j1 - j0 + 5) / 2;  // incoming rows rs .. j1+1 (one spare row when odd)
    // steps 1 .. qx_end hold rows of the tile (rows r, r+1 meet [j0, j1))
    const int qx_end = (j1 - j0 + 1) / 2;
    const float dt = a.sc->dt * a.dt_scale;
    const UpdateArgs ua{dt, 1.0f / g.dx, 1.0f / g.dy};

    // slots of the previous tile are free once every thread is past its last read
    fence_proxy_async_smem();
    __syncthreads();
    const int base = rp.base;  // row pairs this CTA staged before this tile
    const int bbase = rp.bbase;
    // stage input row pair q of this tile into its slot (base + q) % KP
    auto issue = [&](int q) {
        const int slot = (base + q) % KP;
        mbar_arrive_expect_tx(&bars[slot], L::tx_bytes);
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int row = clampi(rs + 2 * q + h, 0, ny - 1);
            float *dst = raw + (size_t)(slot * 2 + h) * L::SLOT;
#pragma unroll
            for (int b = 0; b < L::NB; b++)
                tma_load_3d(dst + b * kBoxStride, tm_in, &bars[slot], i0 - 4 + b * kBox, row, 0);
        }
    };
    // blend partner rows of pair p (updated in step p+1; pair 0 and the last
    // pair are never updated)
    const int nblend = STAGE == 2 ? max(0, npairs - 2) : 0;
    int bissued = 0;  // blend pairs staged in this tile (the same count in every thread)
    auto issue_blend = [&](int p) {
        mbar_arrive_expect_tx(bbar, L::btx_bytes);
#pragma unroll
        for (int h = 0; h < 2; h++)
            tma_load_3d(bl + (size_t)h * L::BSLOT, tm_blend, bbar, i0, clampi(rs + 2 * p + h, 0, ny - 1), 0);
    };
    int issued = min(KP, npairs);
    if (t == 0)
        for (int q = 0; q < issued; q++) issue(q);

    const int ic_t = clampi(i0 - 2 + t, 0, nx - 1);
    const int rc_t = ic_t - i0 + 4;
    const uint8_t *mcol = a.mask + ic_t;
    uint32_t mA = __ldg(mcol + (size_t)clampi(rs, 0, ny - 1) * g.pitch);
    uint32_t mB = __ldg(mcol + (size_t)clampi(rs + 1, 0, ny - 1) * g.pitch);
    const int iu = i0 + t;
    const bool col_ok = (t < W) && (iu < nx);
    const bool edge_x = (iu == 0 || iu == nx - 1);
    const int tx = min(t, W);
    const int cy = min(t, W - 1) + 2;
    float *outp = a.out + iu;

    int kr = base % KP, par = (base / KP) & 1, ku = (base + KP - 1) % KP;
    int pc0 = 0, pc1 = 2;  // P/M rows of row pairs q, q-1
    float fyB[5] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f};  // y-face below row r-2
    float vfB = 0.0f;                                // and its face velocity
    float sy2[4] = {0.0f, 0.0f, 0.0f, 0.0f};         // y-slopes of row r-2
    bool ok_all = true;

    for (int q = 0; q < npairs; q++) {
        const int r = rs + 2 * q;
        const uint32_t nA = __ldg(mcol + (size_t)clampi(r + 2, 0, ny - 1) * g.pitch);
        const uint32_t nB = __ldg(mcol + (size_t)clampi(r + 3, 0, ny - 1) * g.pitch);
        // ---- phase 1: primitives + masks of rows r, r+1
        const int s0 = pc0 >> 1, s1 = pc1 >> 1;  // pair slots of q, q-1
        bool ok = mbar_wait_bounded(&bars[kr], (uint32_t)par);
        if (STAGE == 2 && q >= 2) ok = ok && mbar_wait_bounded(bbar, (uint32_t)((bbase + q - 2) & 1));
        if (ok) {
            float rho[2], u[2], v[2], p[2];
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const float *src = raw + (size_t)(kr * 2 + h) * L::SLOT;
                float T;
                rho[h] = ring_at<L::NB>(src, 0, rc_t);
                prim_from_cons(rho[h], ring_at<L::NB>(src, 1, rc_t), ring_at<L::NB>(src, 2, rc_t),
                               ring_at<L::NB>(src, 3, rc_t), ring_at<L::NB>(src, 4, rc_t), u[h], v[h], p[h], T);
                M[(pc0 + h) * NT + t] = (uint8_t)(h ? mB : mA);
            }
            PA[s0 * NT + t] = make_float4(rho[0], rho[1], u[0], u[1]);
            PB[s0 * NT + t] = make_float4(v[0], v[1], p[0], p[1]);
        }
        mA = nA;
        mB = nB;
        if (__syncthreads_or(!ok)) {
            ok_all = false;
            break;
        }
        // step 0 stages only: its y-faces lie below the tile's first update,
        // its rows take no x-faces, it issues no load, and nothing it would
        // write is read before the next step's first barrier (the y-slopes of
        // row r-2 it leaves at zero feed only the unused face (j0-2 | j0-1)).
        // Stage 1 only: in stage 2 the extra path cost more than it saved.
        if (STAGE == 1 && q == 0) {
            pc1 = pc0;
            pc0 = 2 - pc0;
            kr = ring_next<KP>(kr);
            par ^= (kr == 0) ? 1 : 0;
            ku = ring_next<KP>(ku);
            continue;
        }
        // ---- phase 2: y-faces of column cy, then the update of rows r-2, r-1
        // column cy, rows r-3 .. r: pairs q-2 (rows r-4, r-3), q-1 (r-2, r-1), q (r, r+1)
        const float4 A1 = PA[s1 * NT + cy], B1 = PB[s1 * NT + cy];
        const float4 A0 = PA[s0 * NT + cy], B0 = PB[s0 * NT + cy];
        // y-faces (r-2 | r-1), (r-1 | r) as one lane pair; the y-slopes of row
        // r-2 are those of row r in step q-1
        const uint32_t my0 = M[pc1 * NT + cy], my1 = M[(pc1 + 1) * NT + cy];
        const PairPrim lo = pair_prim(A1, B1), hi = pair_prim(A0, B0);
        const PairPrim mid{mk2(A1.y, A0.x), mk2(A1.w, A0.z), mk2(B1.y, B0.x), mk2(B1.w, B0.z)};
        f2 Fy[5];
        face_pair_y<SCHEME, LIM>((my0 & MB_YV) != 0, (my0 & MB_YN) != 0, (my1 & MB_YV) != 0, (my1 & MB_YN) != 0, lo,
                                 mid, hi, sy2, Fy);
        // their face velocities (the face below row r-2 is carried)
        const f2 vfy = p_face_velocity(Fy[0], lo.rho, mid.rho);
        {
            const int u0 = r - 2;  // rows u0 (lane .x) and u0+1 (lane .y)
            const bool st0 = col_ok && u0 >= j0 && u0 < j1, st1 = col_ok && u0 + 1 >= j0 && u0 + 1 < j1;
            if (st0 || st1) {
                const float *src = raw + (size_t)(ku * 2) * L::SLOT;
                f2 Uc[5], Un[5];
#pragma unroll
                for (int k = 0; k < 5; k++)
                    Uc[k] = mk2(ring_at<L::NB>(src, k, t + 4), ring_at<L::NB>(src + L::SLOT, k, t + 4));
                // flux differences: x from the x-face ring (step q-1), y
                // from this step's faces and the carried one below
                const float4 LA = XA[t], RA = XA[t + 1], LB = XB[t], RB = XB[t + 1], LC = XC[t], RC = XC[t + 1];
                const f2 dX[5] = {p_sub(mk2(RA.x, RA.y), mk2(LA.x, LA.y)), p_sub(mk2(RA.z, RA.w), mk2(LA.z, LA.w)),
                                  p_sub(mk2(RB.x, RB.y), mk2(LB.x, LB.y)), p_sub(mk2(RB.z, RB.w), mk2(LB.z, LB.w)),
                                  p_sub(mk2(RC.x, RC.y), mk2(LC.x, LC.y))};
                const f2 du = p_sub(mk2(RC.z, RC.w), mk2(LC.z, LC.w));
                f2 dY[5];
#pragma unroll
                for (int k = 0; k < 5; k++) dY[k] = mk2(Fy[k].x - fyB[k], Fy[k].y - Fy[k].x);
                const f2 dv = mk2(vfy.x - vfB, vfy.y - vfy.x);
                const bool ey0 = (u0 == 0 || u0 == ny - 1), ey1 = (u0 + 1 == 0 || u0 + 1 == ny - 1);
                update_pair(Uc, dX, dY, du, dv, mk2(B1.z, B1.w), edge_x, ey0, ey1, ua, Un);
                // wall cells keep their state
                const bool w0 = (my0 & MB_WALL) != 0, w1 = (my1 & MB_WALL) != 0;
                if (w0 || w1) {
#pragma unroll
                    for (int k = 0; k < 5; k++) Un[k] = p_sel(w0, w1, Uc[k], Un[k]);
                }
                if (STAGE == 2) {
                    const float *b = bl + t;
#pragma unroll
                    for (int k = 0; k < 5; k++)
                        Un[k] = p_fma(splat(0.5f), Un[k], p_mul(splat(0.5f), mk2(b[k * W], b[L::BSLOT + k * W])));
                }
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    if (!(h ? st1 : st0)) continue;
                    const int urow = u0 + h;
                    float Ur[5];
#pragma unroll
                    for (int k = 0; k < 5; k++) Ur[k] = h ? Un[k].y : Un[k].x;
                    const uint32_t ctype = mb_type(h ? my1 : my0);
                    // phase-1 conditions act only on non-fluid cells and the domain's edge cells
                    if (a.apply_bc && (ctype != CT_FLUID || edge_x || (h ? ey1 : ey0)))
                        bc_pointwise(Ur, ctype, iu, urow, nx, ny, a.fs);
                    if (a.cfl && ctype != CT_GHOST) {
                        float uu, vv, pp, TT;
                        prim_from_cons(Ur[0], Ur[1], Ur[2], Ur[3], Ur[4], uu, vv, pp, TT);
                        lmax_speed = fmaxf(lmax_speed, wave_speed(uu, vv, pp, Ur[0]));
                        nbad += nonfinite5(Ur);
                    }
                    float *dst = outp + (size_t)urow * g.pitch;
#pragma unroll
                    for (int k = 0; k < 5; k++) dst[k * g.plane] = Ur[k];
                    // a registered display field of the step's result (the descriptor
                    // is read here, not held in registers across the loop)
                    if (DISP && STAGE == 2) {
                        float *const dptr = a.disp->ptr;
                        if (dptr)
                            dptr[(size_t)urow * nx + iu] = derived_value(a.disp->kind, Ur[0], Ur[1], Ur[2], Ur[4]);
                    }
                }
            }
        }
#pragma unroll
        for (int k = 0; k < 5; k++) fyB[k] = Fy[k].y;
        vfB = vfy.y;
        // the x-faces of rows r, r+1 feed only the update of those rows: none
        // for the halo pairs above and below the tile (step 0 and, for an even
        // tile height, the last step; uniform over the CTA).  The x-slopes
        // below stay unconditional: skipping them too made stage 2 spill.
        const bool xrows = (unsigned)(q - 1) < (unsigned)qx_end;
        // x-slopes of rows r, r+1 at staged column t+1 (columns 1 .. NT-2 are
        // the cells beside the x-faces of phase 3)
        if (t < NT - 2) {
            const float4 *A = PA + s0 * NT + t, *B = PB + s0 * NT + t;
            const PairPrim m = pair_prim(A[0], B[0]), c = pair_prim(A[1], B[1]), p = pair_prim(A[2], B[2]);
            const f2 sr = p_slope<LIM>(m.rho, c.rho, p.rho), su = p_slope<LIM>(m.u, c.u, p.u);
            const f2 sv = p_slope<LIM>(m.v, c.v, p.v), sp = p_slope<LIM>(m.p, c.p, p.p);
            SA[t + 1] = make_float4(sr.x, sr.y, su.x, su.y);
            SB[t + 1] = make_float4(sv.x, sv.y, sp.x, sp.y);
        }
        fence_proxy_async_smem();
        __syncthreads();
        // the input slot of pair q-1 is free now: stage pair q-1+KP into it;
        // the blend slot too: stage the blend rows of pair q.  Lane 0 of warp
        // q mod (NT/32) issues, so no warp carries the issue work every step
        // (the barriers wait for the slowest warp)
        {
            const int who = (q % (NT / 32)) * 32;
            if (issued < npairs && issued <= q + KP - 1) {
                if (t == who) issue(issued);
                ++issued;
            }
            if (STAGE == 2 && q >= 1 && q <= nblend) {
                if (t == who) issue_blend(q);
                ++bissued;
            }
        }
        // ---- phase 3: x-faces of rows r, r+1 (read by the update in step q+1)
        if (xrows) {
            f2 Fx[5];
            const float4 *A = PA + s0 * NT, *B = PB + s0 * NT;
            const uint32_t mb0 = M[pc0 * NT + tx + 1], mb1 = M[(pc0 + 1) * NT + tx + 1];
            const PairPrim ca = pair_prim(A[tx + 1], B[tx + 1]), cb = pair_prim(A[tx + 2], B[tx + 2]);
            face_pair_x_sl<SCHEME>((mb0 & MB_XV) != 0, (mb0 & MB_XN) != 0, (mb1 & MB_XV) != 0, (mb1 & MB_XN) != 0, ca,
                                   pair_sl(SA[tx + 1], SB[tx + 1]), cb, pair_sl(SA[tx + 2], SB[tx + 2]), Fx);
            if (t <= W) {
                XA[t] = make_float4(Fx[0].x, Fx[0].y, Fx[1].x, Fx[1].y);
                XB[t] = make_float4(Fx[2].x, Fx[2].y, Fx[3].x, Fx[3].y);
                // with the face velocities for the rho_e source of both adjacent cells
                const f2 vel = p_face_velocity(Fx[0], ca.rho, cb.rho);
                XC[t] = make_float4(Fx[4].x, Fx[4].y, vel.x, vel.y);
            }
        }
        pc1 = pc0;
        pc0 = 2 - pc0;
        kr = ring_next<KP>(kr);
        par ^= (kr == 0) ? 1 : 0;
        ku = ring_next<KP>(ku);
    }
    if (!ok_all) {
        if (t == 0) {
            record_error(a.sc, kErrTimeout);
            // drain loads still in flight before the shared memory is released
            for (int q = 0; q < issued; q++)
                mbar_wait_bounded(&bars[(base + q) % KP], (uint32_t)(((base + q) / KP) & 1), 20000000LL);
            // each blend pair is consumed one step after it is staged, so at
            // most the last one staged can still be in flight
            if (bissued > 0) mbar_wait_bounded(bbar, (uint32_t)((bbase + bissued - 1) & 1), 20000000LL);
        }
        return false;
    }
    rp.base = base + npairs;
    rp.bbase = bbase + nblend;
    return true;
}

// Occupancy target: 6 CTAs of 128 threads per SM (80 registers, no spills;
// ~30 KB of shared memory per CTA for stage 1, ~35 KB for stage 2 with its
// blend pair).
template <int NT, int K, int STAGE, int SCHEME, int LIM, bool DISP>
__global__ void __launch_bounds__(NT, 768 / NT)
    k_stage(const __grid_constant__ CUtensorMap tm_in, const __grid_constant__ CUtensorMap tm_blend,
            const StepArgs a) {
    using L = StageLayout<NT, K, STAGE>;
    static_assert(L::total <= 227 * 1024, "shared memory");
    extern __shared__ __align__(16) unsigned char smem_raw[];
    unsigned char *smem = aligned_smem(smem_raw);
    const bool misaligned = (smem_addr_opaque(smem) & 127u) != 0u;
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + L::bar_off);
    if (threadIdx.x == 0 && !misaligned) {
        prefetch_tensormap(&tm_in);
        if (STAGE == 2) prefetch_tensormap(&tm_blend);
        for (int k = 0; k < L::NBAR; k++) mbar_init(&bars[k], 1);
        fence_barrier_init();
    }
    // the prologue above overlaps the previous step kernel's tail
    pdl_wait();
    if (smem_misaligned(smem, a.sc)) return;
    RingPos rp{0, 0};
    float lmax = 0.0f;
    unsigned nbad = 0;
    const bool ok = stage_tile<NT, K, STAGE, SCHEME, LIM, DISP>(&tm_in, &tm_blend, a, blockIdx.x * L::W,
                                                                blockIdx.y * a.rows_per_cta, smem, rp, lmax, nbad);
    if (a.early_launch) pdl_trigger();
    if (!ok) return;
    if (a.cfl) block_publish<NT>(lmax, 0.0f, nbad, a.sc);
}

template <int NT, int K>
struct ViscLayout {
    static constexpr int W = NT - 4;
    static constexpr int NB = (NT + 4 + kBox - 1) / kBox;
    static constexpr int BW = NB * kBox;
    static constexpr int KP = K / 2;   // input ring: K rows staged as K/2 row pairs
    static constexpr int PP = 2;       // primitive / mask ring (row pairs)
    static constexpr int TP = 2;       // stress / heat-flux ring (row pairs)
    static constexpr int TQ = 4;       // per cell: txx, txy, qx, work_x (what east / west neighbours read)
    static constexpr int SLOT = NB * kBoxStride;
    static constexpr size_t raw_off = 0;
    static constexpr size_t raw_bytes = (size_t)K * SLOT * 4;
    static constexpr size_t p_off = raw_off + raw_bytes;
    static constexpr size_t p_bytes = (size_t)PP * 2 * NT * 16;
    // the x-derivative operands of the divergence (tau_xx, tau_xy, q_x,
    // work_x), one float plane each; the y-derivative operands and Phi stay in
    // the registers of the thread that owns the column
    static constexpr size_t t_off = p_off + p_bytes;
    static constexpr size_t t_bytes = (size_t)TP * 2 * TQ * NT * 4;
    static constexpr size_t bar_off = (t_off + t_bytes + 15) & ~(size_t)15;
    static constexpr size_t total = bar_off + KP * 8 + 128;  // + alignment slack
    static constexpr uint32_t tx_bytes = 2 * 5 * BW * 4;  // one row pair
};

// Viscous half step on one tile (fusedViscousDiffusionKernel,
// src/solver.cu:2251-2511), out of place, marching two rows per step.
// Thread t owns column i0-2+t in every phase.  Per step q (incoming rows
// r = j0-2+2q and r+1):
//   phase 1  primitives (u, v, T) and Sutherland viscosity of rows r, r+1 on
//            NT columns into the primitive ring; the thread keeps them, the
//            cells' mask bytes and the conserved state of its own column in
//            registers (the stress and the update of that column one and two
//            steps later read them from there), so the input slot is free
//            after the first barrier and is refilled there
//   -- barrier --
//   phase 2  stress, heat flux, work terms (u tau_xx + v tau_xy, u tau_xy +
//            v tau_yy) and dissipation of rows r-1, r on NT-2 columns: the
//            column's own rows from registers, the east / west neighbours
//            from the primitive ring
//   -- barrier --
//   phase 3  viscous update of rows r-2, r-1 on the W = NT-4 middle columns:
//            east / west operands from the stress ring, the column's own
//            north / south operands and Phi from registers (the primitive
//            ring's pair q-1 may be refilled by a faster thread's next
//            phase 1 meanwhile)
// Both rows of a phase are evaluated in straight-line code (validity applied
// by selects and predicated stores), so their dependency chains interleave.
template <int NT, int K, bool DISP = false>
__device__ __forceinline__ bool viscous_tile(const CUtensorMap *tm_in, const StepArgs &a, int i0, int j0,
                                             unsigned char *smem, RingPos &rp, float &lmax_speed, float &lmax_nu,
                                             unsigned &nbad) {
    using L = ViscLayout<NT, K>;
    constexpr int KP = L::KP;
    static_assert(L::PP == 2 && L::TP == 2 && KP >= 2, "ring sizes");
    constexpr int TQ = L::TQ;
    float *raw = reinterpret_cast<float *>(smem + L::raw_off);
    float4 *P = reinterpret_cast<float4 *>(smem + L::p_off);  // {u, v, T, mu}
    float *Tq = reinterpret_cast<float *>(smem + L::t_off);   // TQ planes per row
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + L::bar_off);

    const GridDesc g = a.g;
    const int nx = g.nx, ny = g.ny;
    const int t = threadIdx.x;
    const int j1 = min(j0 + a.rows_per_cta, ny);
    const int rs = j0 - 2;
    const int npairs = (j1 - j0 + 5) / 2;  // incoming rows rs .. j1+1 (one spare row when odd)
    const float dt = a.sc->dt * a.dt_scale;
    const ViscArgs va = viscous_args(g.dx, g.dy, a.prandtl, a.ref_prandtl != 0);

    fence_proxy_async_smem();
    __syncthreads();
    const int base = rp.base;  // row pairs this CTA staged before this tile
    int islot = base % KP;
    auto issue = [&](int q) {
        mbar_arrive_expect_tx(&bars[islot], L::tx_bytes);
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const int row = clampi(rs + 2 * q + h, 0, ny - 1);
            float *dst = raw + (size_t)(islot * 2 + h) * L::SLOT;
#pragma unroll
            for (int b = 0; b < L::NB; b++)
                tma_load_3d(dst + b * kBoxStride, tm_in, &bars[islot], i0 - 4 + b * kBox, row, 0);
        }
        islot = ring_next<KP>(islot);
    };
    int issued = min(KP, npairs);
    if (t == 0)
        for (int q = 0; q < issued; q++) issue(q);

    const int ic = i0 - 2 + t;                  // this thread's column
    const int ic_t = clampi(ic, 0, nx - 1);     // column whose state it loads
    const int rc_t = ic_t - i0 + 4;             // its staged position
    const uint8_t *mcol = a.mask + ic_t;
    uint32_t mA = __ldg(mcol + (size_t)clampi(rs, 0, ny - 1) * g.pitch);
    uint32_t mB = __ldg(mcol + (size_t)clampi(rs + 1, 0, ny - 1) * g.pitch);
    const bool stress_thread = t >= 1 && t < NT - 1;
    const bool stress_col_in = ic >= 0 && ic < nx;
    const bool i_lo = ic == 0, i_hi = ic == nx - 1;
    // x-differences of the stress: one-sided at the domain edges (the cell
    // itself stands in for the missing neighbour), central elsewhere
    const int tW = i_lo ? t : t - 1, tE = (i_hi && !i_lo) ? t : t + 1;
    const float fx = (i_lo || i_hi) ? va.inv_dx : va.inv_2dx;
    const bool col_ok = t >= 2 && t < NT - 2 && ic < nx;
    const bool interior_x = ic > 0 && ic < nx - 1;
    const int tp = min(max(t, 1), NT - 2);  // stencil centre kept inside the rings

    int kr = base % KP, par = (base / KP) & 1;
    int pc0 = 0, pc1 = 2;  // primitive-ring rows of row pairs q, q-1
    int tc0 = 0, tc1 = 2;  // stress rows of row pairs q (rows r-1, r) and q-1
    float Uprev[2][5];     // conserved state of rows r-2, r-1 at column ic
    float4 Pprev[2];       // {u, v, T, mu} of rows r-2, r-1 at this thread's column
    uint32_t mprev[2];     // and their mask bytes
    ViscY yprev[2];        // {tyy, -, qy, work_y} of rows r-3, r-2 at this column (txy is in the ring)
    float phi_prev = 0.0f; // Phi of row r-2 at this column
#pragma unroll
    for (int h = 0; h < 2; h++) {
#pragma unroll
        for (int k = 0; k < 5; k++) Uprev[h][k] = 0.0f;
        Pprev[h] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        mprev[h] = 0u;
        yprev[h] = ViscY{0.0f, 0.0f, 0.0f, 0.0f};
    }
    bool ok_all = true;

    for (int q = 0; q < npairs; q++) {
        const int r = rs + 2 * q;
        const uint32_t nA = __ldg(mcol + (size_t)clampi(r + 2, 0, ny - 1) * g.pitch);
        const uint32_t nB = __ldg(mcol + (size_t)clampi(r + 3, 0, ny - 1) * g.pitch);
        // ---- phase 1: primitives, viscosity and masks of rows r, r+1
        float Unext[2][5];
        float4 Pcur[2] = {make_float4(0.0f, 0.0f, 0.0f, 0.0f), make_float4(0.0f, 0.0f, 0.0f, 0.0f)};
        const uint32_t mcur[2] = {mA, mB};
        bool ok = mbar_wait_bounded(&bars[kr], (uint32_t)par);
        if (ok) {
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const float *src = raw + (size_t)(kr * 2 + h) * L::SLOT;
#pragma unroll
                for (int k = 0; k < 5; k++) Unext[h][k] = ring_at<L::NB>(src, k, rc_t);
                float u, v, p, T;
                prim_from_cons(Unext[h][0], Unext[h][1], Unext[h][2], Unext[h][3], Unext[h][4], u, v, p, T);
                Pcur[h] = make_float4(u, v, T, sutherland_mu(T));
                P[(pc0 + h) * NT + t] = Pcur[h];
            }
        } else {
#pragma unroll
            for (int h = 0; h < 2; h++)
#pragma unroll
                for (int k = 0; k < 5; k++) Unext[h][k] = 0.0f;
        }
        mA = nA;
        mB = nB;
        fence_proxy_async_smem();
        if (__syncthreads_or(!ok)) {
            ok_all = false;
            break;
        }
        // the input slot of pair q is free now: stage pair q+KP into it
        // (thread 0 issues; rotating the issuing warp as the stage kernels do
        // made this pass 1 % slower)
        if (t == 0 && issued < npairs && issued <= q + KP) {
            issue(issued);
            ++issued;
        }
        // ---- phase 2: stress, heat flux, work terms and dissipation of rows
        // r-1, r at column ic (step 0 holds rows j0-3, j0-2, which no update
        // of this tile reads)
        ViscY ycur[2] = {ViscY{0.0f, 0.0f, 0.0f, 0.0f}, ViscY{0.0f, 0.0f, 0.0f, 0.0f}};
        float phi_cur[2] = {0.0f, 0.0f};
        if (stress_thread && q > 0) {
            float out[2][8];
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int trow = r - 1 + h;
                // rows trow-1, trow, trow+1 of the primitive ring; at the
                // bottom (top) domain edge the row itself replaces the south
                // (north) one and the y-difference is one-sided
                const bool j_lo = trow == 0, j_hi = trow == ny - 1 && !j_lo;
                const int rowC = h ? pc0 : pc1 + 1;
                const float fy = (j_lo || j_hi) ? va.inv_dy : va.inv_2dy;
                // the column's own rows trow-1, trow, trow+1 from registers
                const float4 C = h ? Pcur[0] : Pprev[1];
                const float4 N = j_hi ? C : (h ? Pcur[1] : Pcur[0]);
                const float4 S = j_lo ? C : (h ? Pprev[1] : Pprev[0]);
                const float4 E = P[rowC * NT + tE], Wc = P[rowC * NT + tW];
                stress_heat_work_sel(C.w, C.x, C.y, E.x, Wc.x, N.x, S.x, E.y, Wc.y, N.y, S.y, E.z, Wc.z, N.z, S.z,
                                     fx, fy, va, out[h]);
                const bool live = stress_col_in && trow >= 0 && trow < ny &&
                                  mb_type(h ? mcur[0] : mprev[1]) != CT_SOLID;
#pragma unroll
                for (int k = 0; k < 8; k++) out[h][k] = live ? out[h][k] : 0.0f;
            }
            // out = {txx, tyy, txy, qx, qy, wx, wy, phi}
#pragma unroll
            for (int h = 0; h < 2; h++) {
                float *Ts = Tq + (tc0 + h) * TQ * NT + t;
                Ts[0] = out[h][0];
                Ts[NT] = out[h][2];
                Ts[2 * NT] = out[h][3];
                Ts[3 * NT] = out[h][5];
                ycur[h] = ViscY{out[h][1], out[h][2], out[h][4], out[h][6]};
                phi_cur[h] = out[h][7];
            }
        }
        // classes and viscosity of rows r-2, r-1 for phase 3 (the threads that
        // store updates have tp == t, so their own column's registers)
        uint32_t ctype[2];
        float mu_c[2];
#pragma unroll
        for (int h = 0; h < 2; h++) {
            ctype[h] = mb_type(mprev[h]);
            mu_c[h] = Pprev[h].w;
        }
        __syncthreads();
        // ---- phase 3: viscous update of rows r-2, r-1 at column ic (rows
        // of this tile from step 2 on)
        if (q >= 2) {
            float U[2][5];
            bool store[2];
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int urow = r - 2 + h;
                store[h] = col_ok && urow >= j0 && urow < j1;
                // east / west operands of row urow from the ring; north /
                // south (rows urow+1, urow-1) and Phi from this column's registers
                const int tC0 = h ? tc0 : tc1 + 1;
                const float *T0 = Tq + tC0 * TQ * NT + tp;
                const ViscX Ex{T0[1], T0[NT + 1], T0[2 * NT + 1], T0[3 * NT + 1]};
                const ViscX Wx{T0[-1], T0[NT - 1], T0[2 * NT - 1], T0[3 * NT - 1]};
                const ViscY &Ny = h ? ycur[1] : ycur[0];
                // the south row's txy from the ring (row r-3 or r-2, pair slot tc1)
                const ViscY Sy{h ? yprev[1].tyy : yprev[0].tyy, Tq[(tc1 + h) * TQ * NT + NT + tp],
                               h ? yprev[1].qy : yprev[0].qy, h ? yprev[1].wy : yprev[0].wy};
                float rhs[4];
                viscous_rhs_w(Ex, Wx, Ny, Sy, h ? phi_cur[0] : phi_prev, va, rhs);
                const bool upd = ctype[h] == CT_FLUID && interior_x && urow > 0 && urow < ny - 1;
                U[h][0] = Uprev[h][0];
#pragma unroll
                for (int k = 1; k < 5; k++) U[h][k] = upd ? Uprev[h][k] + dt * rhs[k - 1] : Uprev[h][k];
            }
            if (a.apply_bc) {
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const int row = r - 2 + h;
                    if (ctype[h] != CT_FLUID || !interior_x || row == 0 || row == ny - 1)
                        bc_pointwise(U[h], ctype[h], ic, row, nx, ny, a.fs);
                }
            }
            if (a.cfl) {
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    float uu, vv, pp, TT;
                    prim_from_cons(U[h][0], U[h][1], U[h][2], U[h][3], U[h][4], uu, vv, pp, TT);
                    const bool counted = store[h] && ctype[h] != CT_GHOST;
                    const float ws = wave_speed(uu, vv, pp, U[h][0]);
                    lmax_speed = counted ? fmaxf(lmax_speed, ws) : lmax_speed;
                    nbad += counted ? nonfinite5(U[h]) : 0u;
                    if (a.cfl == 2) {
                        const float mu = (ctype[h] == CT_SOLID) ? 0.0f : mu_c[h];
                        const float nu = mu * rcp_approx(U[h][0] + 1e-10f);
                        lmax_nu = counted ? fmaxf(lmax_nu, nu) : lmax_nu;
                    }
                }
            }
#pragma unroll
            for (int h = 0; h < 2; h++) {
                if (store[h]) {
                    float *dst = a.out + (size_t)(r - 2 + h) * g.pitch + ic;
#pragma unroll
                    for (int k = 0; k < 5; k++) dst[k * g.plane] = U[h][k];
                    // a registered display field of the step's result (post pass)
                    if (DISP) {
                        float *const dptr = a.disp->ptr;
                        if (dptr)
                            dptr[(size_t)(r - 2 + h) * nx + ic] =
                                derived_value(a.disp->kind, U[h][0], U[h][1], U[h][2], U[h][4]);
                    }
                }
            }
        }
#pragma unroll
        for (int h = 0; h < 2; h++) {
#pragma unroll
            for (int k = 0; k < 5; k++) Uprev[h][k] = Unext[h][k];
            Pprev[h] = Pcur[h];
            mprev[h] = mcur[h];
            yprev[h] = ViscY{ycur[h].tyy, 0.0f, ycur[h].qy, ycur[h].wy};
        }
        phi_prev = phi_cur[1];
        kr = ring_next<KP>(kr);
        par ^= (kr == 0) ? 1 : 0;
        pc1 = pc0;
        pc0 = 2 - pc0;
        tc1 = tc0;
        tc0 = 2 - tc0;
    }
    if (!ok_all) {
        if (t == 0) {
            record_error(a.sc, kErrTimeout);
            for (int q = 0; q < issued; q++)
                mbar_wait_bounded(&bars[(base + q) % KP], (uint32_t)(((base + q) / KP) & 1), 20000000LL);
        }
        return false;
    }
    rp.base = base + npairs;
    return true;
}

// 5 CTAs of 128 threads per SM (96 registers, no spills; ~28 KB of shared
// memory each): the column's own primitives and stress operands live in
// registers across steps, which at 80 registers (6 CTAs) spilled and ran
// 15-20 % slower.
template <int NT, int K, bool DISP>
__global__ void __launch_bounds__(NT, 640 / NT) k_viscous(const __grid_constant__ CUtensorMap tm_in, const StepArgs a) {
    using L = ViscLayout<NT, K>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    unsigned char *smem = aligned_smem(smem_raw);
    const bool misaligned = (smem_addr_opaque(smem) & 127u) != 0u;
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + L::bar_off);
    if (threadIdx.x == 0 && !misaligned) {
        prefetch_tensormap(&tm_in);
        for (int k = 0; k < L::KP; k++) mbar_init(&bars[k], 1);
        fence_barrier_init();
    }
    // the prologue above overlaps the previous step kernel's tail
    pdl_wait();
    if (smem_misaligned(smem, a.sc)) return;
    RingPos rp{0, 0};
    float ls = 0.0f, ln = 0.0f;
    unsigned nbad = 0;
    const bool ok =
        viscous_tile<NT, K, DISP>(&tm_in, a, blockIdx.x * L::W, blockIdx.y * a.rows_per_cta, smem, rp, ls, ln, nbad);
    if (a.early_launch) pdl_trigger();
    if (!ok) return;
    if (a.cfl) block_publish<NT>(ls, ln, nbad, a.sc);
}

// --------------------------------------------------------- batched launches
// One persistent launch advances one stage of every instance of a batch:
// CTAs walk a static tile list (instance, strip, row band); per-instance
// descriptors give buffers, tensor maps, parameters and device scalars.  The
// buffer that holds U^n alternates per step; each instance keeps its own
// parity in its device scalars (flipped by its ghost-pass finalize).
__device__ __forceinline__ int role_buf(const BatchInst &I, int role) {
    const int parity = (int)I.sc->parity;
    if (role == ROLE_N) return parity ? 2 : 0;
    if (role == ROLE_X) return parity ? 0 : 2;
    return role == ROLE_S ? 1 : 3;
}

__device__ __forceinline__ StepArgs batch_args(const BatchInst &I, int out_role, int apply_bc, int cfl, float dts,
                                               int rows) {
    StepArgs a;
    a.g = I.g;
    a.out = I.buf[role_buf(I, out_role)];
    a.mask = I.mask;
    a.sc = I.sc;
    a.fs = I.fs;
    a.wall = I.wall;
    a.prandtl = I.prandtl;
    a.ref_prandtl = I.ref_prandtl;
    a.rows_per_cta = rows;
    a.apply_bc = apply_bc;
    a.cfl = cfl;
    a.dt_scale = dts;
    a.disp = nullptr;
    a.early_launch = 0;
    a.pdl = 0;
    return a;
}

template <int NT, int K, int STAGE, int SCHEME, int LIM>
__global__ void __launch_bounds__(NT, 640 / NT) k_stage_batch(const BatchInst *__restrict__ insts,
                                                    const TileDesc *__restrict__ tiles, int ntiles, int rows,
                                                    int early_launch) {
    using L = StageLayout<NT, K, STAGE>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ StepArgs s_args;
    unsigned char *smem = aligned_smem(smem_raw);
    if (smem_misaligned(smem, insts[0].sc)) return;
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + L::bar_off);
    if (threadIdx.x == 0) {
        for (int k = 0; k < L::NBAR; k++) mbar_init(&bars[k], 1);
        fence_barrier_init();
    }
    // the prologue above overlaps the previous kernel's tail; the buffer
    // roles (device parity) and the states are read after the wait
    pdl_wait();
    RingPos rp{0, 0};
    for (int ti = blockIdx.x; ti < ntiles; ti += gridDim.x) {
        const TileDesc td = tiles[ti];
        const BatchInst &I = insts[td.inst];
        const bool visc = I.viscous != 0;
        int in_role, blend_role, out_role, bc, cfl;
        if (STAGE == 1) {
            in_role = visc ? ROLE_D : ROLE_N;
            blend_role = in_role;
            out_role = ROLE_S;
            bc = 1;
            cfl = 0;
        } else {
            in_role = ROLE_S;
            blend_role = visc ? ROLE_D : ROLE_N;
            out_role = visc ? ROLE_D : ROLE_X;
            bc = visc ? 0 : 1;
            cfl = visc ? 0 : 1;
        }
        // the tile's arguments live in shared memory, not in registers
        __syncthreads();  // every thread is done with the previous tile's arguments
        if (threadIdx.x == 0) s_args = batch_args(I, out_role, bc, cfl, 1.0f, rows);
        __syncthreads();
        float lmax = 0.0f;
        unsigned nbad = 0;
        if (!stage_tile<NT, K, STAGE, SCHEME, LIM>(&I.tm_in[role_buf(I, in_role)], &I.tm_ctr[role_buf(I, blend_role)],
                                                   s_args, td.i0, td.j0, smem, rp, lmax, nbad))
            return;
        if (cfl) block_publish<NT>(lmax, 0.0f, nbad, I.sc);
    }
    if (early_launch) pdl_trigger();
}

template <int NT, int K>
__global__ void __launch_bounds__(NT, 640 / NT) k_viscous_batch(const BatchInst *__restrict__ insts,
                                                      const TileDesc *__restrict__ tiles, int ntiles, int rows,
                                                      int post) {
    using L = ViscLayout<NT, K>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    __shared__ StepArgs s_args;
    unsigned char *smem = aligned_smem(smem_raw);
    if (smem_misaligned(smem, insts[0].sc)) return;
    uint64_t *bars = reinterpret_cast<uint64_t *>(smem + L::bar_off);
    if (threadIdx.x == 0) {
        for (int k = 0; k < L::KP; k++) mbar_init(&bars[k], 1);
        fence_barrier_init();
    }
    pdl_wait();
    RingPos rp{0, 0};
    for (int ti = blockIdx.x; ti < ntiles; ti += gridDim.x) {
        const TileDesc td = tiles[ti];
        const BatchInst &I = insts[td.inst];
        // pre: U^n -> U_d (no BC); post: U_b -> U^{n+1} with BC and CFL
        const int in_role = post ? ROLE_D : ROLE_N;
        __syncthreads();  // every thread is done with the previous tile's arguments
        if (threadIdx.x == 0) s_args = batch_args(I, post ? ROLE_X : ROLE_D, post, post ? 2 : 0, 0.5f, rows);
        __syncthreads();
        float ls = 0.0f, ln = 0.0f;
        unsigned nbad = 0;
        if (!viscous_tile<NT, K>(&I.tm_in[role_buf(I, in_role)], s_args, td.i0, td.j0, smem, rp, ls, ln, nbad))
            return;
        if (post) block_publish<NT>(ls, ln, nbad, I.sc);
    }
    if (post) pdl_trigger();  // a ghost pass follows the post half step
}

// ------------------------------------------------------------- ghost pass
__device__ __forceinline__ float pre_bc(const GhostArgs &a, long long q, int k) {
    const long long o = (long long)k * a.g.plane + q;
    return a.B2 ? (0.5f * a.B1[o] + 0.5f * a.B2[o]) : a.B1[o];
}

// Publishes the completed step's CFL maxima and, under the recompute policy,
// the next step's dt (readTimeStepResult, src/solver.cu:3250-3265, in IEEE
// float like the reference's host code) and the advanced simulated time.
__device__ void finalize_cfl(const GhostArgs &a) {
    DevScalars *sc = a.sc;
    volatile float *red = sc->red;
    float ms = red[0], mn = red[1];
    sc->cfl[0] = ms;
    sc->cfl[1] = mn;
    if (a.recompute_dt) {
        float used = sc->dt;
        sc->dt_last = used;
        sc->t = __fadd_rn(sc->t, used);
        float d = __fdiv_rn(__fmul_rn(a.cfl_num, a.min_dx), __fadd_rn(ms, 1e-10f));
        if (a.viscous) {
            float dv = __fdiv_rn(__fmul_rn(__fmul_rn(a.cfl_visc, a.min_dx), a.min_dx), __fadd_rn(mn, 1e-10f));
            d = fminf(d, dv);
        }
        sc->dt = d;
    }
    red[0] = 0.0f;
    red[1] = 0.0f;
    if (a.flip_parity) sc->parity ^= 1u;
    __threadfence();
    sc->counter = 0;
}

// Ghost cells (src/solver.cu:2045-2225) with phase-2 semantics: neighbours
// are read from the phase-1 state A, except neighbours that are themselves
// ghost cells, whose pre-call value comes from B1/B2.  Handles table entries
// [first, first + count) with this block's threads; returns the thread's CFL
// contributions.
__device__ __forceinline__ void ghost_chunk(const GhostArgs &a, int first, int count, float &ls, float &ln,
                                            unsigned &nbad) {
    const int k = first + (int)threadIdx.x;
    if ((int)threadIdx.x >= count || k >= a.n) return;
    const GhostInfo gi = a.list[k];
    const long long plane = a.g.plane;
    const long long pidx = (long long)gi.j * a.g.pitch + gi.i;
    long long best = -1;
    bool best_gh = false;
    for (int m = 0; m < gi.count; m++) {
        const int code = (gi.cand >> (4 * m)) & 0xF;
        const int d = code & 7;
        const bool gh = (code & 8) != 0;
        int di, dj;
        ghost_neighbour(d, di, dj);
        const long long q = pidx + di + (long long)dj * a.g.pitch;
        const float rq = gh ? pre_bc(a, q, 0) : a.A[q];
        if (rq >= MIN_DENSITY) {
            best = q;
            best_gh = gh;
            break;
        }
    }
    float out[5];
    if (best < 0) {
        const float e_inf = a.fs.p / (GAMMA - 1.0f);
        out[0] = a.fs.rho;
        out[1] = 0.0f;
        out[2] = 0.0f;
        out[3] = e_inf;
        out[4] = e_inf;
    } else {
        float s[4];
#pragma unroll
        for (int f = 0; f < 4; f++) s[f] = best_gh ? pre_bc(a, best, f) : a.A[f * plane + best];
        ghost_state(s[0], s[1], s[2], s[3], gi.gx, gi.gy, a.wall, out);
    }
#pragma unroll
    for (int f = 0; f < 5; f++) a.A[f * plane + pidx] = out[f];
    if (a.disp) {
        float *const dptr = a.disp->ptr;
        if (dptr) dptr[(size_t)gi.j * a.g.nx + gi.i] = derived_value(a.disp->kind, out[0], out[1], out[2], out[4]);
    }
    if (a.cfl) {
        float uu, vv, pp, TT;
        prim_from_cons(out[0], out[1], out[2], out[3], out[4], uu, vv, pp, TT);
        ls = wave_speed(uu, vv, pp, out[0]);
        nbad = nonfinite5(out);
        if (a.cfl == 2) {
            float pu, pv, ppp, pT;
            prim_from_cons(pre_bc(a, pidx, 0), pre_bc(a, pidx, 1), pre_bc(a, pidx, 2), pre_bc(a, pidx, 3),
                           pre_bc(a, pidx, 4), pu, pv, ppp, pT);
            ln = sutherland_mu(pT) / (out[0] + 1e-10f);
        }
    }
}

// Reduce the block's CFL contributions and, for the last of `nblocks`
// blocks of this solve, publish the step's maxima / next dt.
__device__ __forceinline__ void ghost_publish(const GhostArgs &a, float ls, float ln, unsigned nbad,
                                              unsigned nblocks) {
    if (a.cfl) block_publish<128>(ls, ln, nbad, a.sc);
    if (a.finalize) {
        __shared__ bool last;
        __threadfence();
        __syncthreads();
        if (threadIdx.x == 0) last = (atomicAdd(&a.sc->counter, 1u) == nblocks - 1);
        __syncthreads();
        if (last && threadIdx.x == 0) {
            __threadfence();
            finalize_cfl(a);
        }
    }
}

__global__ void __launch_bounds__(128) k_ghost(const GhostArgs a) {
    float ls = 0.0f, ln = 0.0f;
    unsigned nbad = 0;
    pdl_wait();
    // the few CTAs of this pass are all resident: the next step kernel may
    // launch now (it waits for this grid's completion before reading)
    pdl_trigger();
    ghost_chunk(a, blockIdx.x * 128, 128, ls, ln, nbad);
    ghost_publish(a, ls, ln, nbad, gridDim.x);
}

// Batched ghost pass: one block per (instance, chunk of <=128 ghost cells).
// mode 1 = after stage 1, mode 2 = end of step (CFL, finalize, parity flip).
__global__ void __launch_bounds__(128) k_ghost_batch(const BatchInst *__restrict__ insts,
                                                    const GhostChunk *__restrict__ chunks, int mode) {
    pdl_wait();
    pdl_trigger();
    const GhostChunk ch = chunks[blockIdx.x];
    const BatchInst &I = insts[ch.inst];
    const bool visc = I.viscous != 0;
    GhostArgs a{};
    a.g = I.g;
    a.list = I.ghosts;
    a.n = I.n_ghost;
    a.sc = I.sc;
    a.fs = I.fs;
    a.wall = I.wall;
    a.recompute_dt = I.recompute_dt;
    a.cfl_num = I.cfl_num;
    a.cfl_visc = I.cfl_visc;
    a.min_dx = I.min_dx;
    a.viscous = I.viscous;
    if (mode == 1) {
        a.A = I.buf[role_buf(I, ROLE_S)];
        a.B1 = I.buf[role_buf(I, visc ? ROLE_D : ROLE_N)];
        a.B2 = nullptr;
        a.cfl = 0;
        a.finalize = 0;
    } else {
        a.A = I.buf[role_buf(I, ROLE_X)];
        a.B1 = I.buf[role_buf(I, visc ? ROLE_D : ROLE_N)];
        a.B2 = visc ? nullptr : I.buf[role_buf(I, ROLE_S)];
        a.cfl = visc ? 2 : 1;
        a.finalize = 1;
        a.flip_parity = 1;
    }
    float ls = 0.0f, ln = 0.0f;
    unsigned nbad = 0;
    ghost_chunk(a, ch.first, ch.count, ls, ln, nbad);
    ghost_publish(a, ls, ln, nbad, (unsigned)I.n_gchunks);
}

// Phase-1 boundary conditions in place (set-up path).
__global__ void k_bc_phase1(GridDesc g, float *U, const uint8_t *mask, Freestream fs) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int j = blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= g.nx || j >= g.ny) return;
    size_t c = (size_t)j * g.pitch + i;
    float s[5];
    for (int k = 0; k < 5; k++) s[k] = U[k * g.plane + c];
    bc_pointwise(s, mb_type(mask[c]), i, j, g.nx, g.ny, fs);
    for (int k = 0; k < 5; k++) U[k * g.plane + c] = s[k];
}

// CFL maxima of a whole state (computeWaveSpeedKernel / computeViscousNumberKernel).
__global__ void __launch_bounds__(256) k_cfl_state(GridDesc g, const float *U, const uint8_t *mask, DevScalars *sc) {
    float ls = 0.0f, ln = 0.0f;
    const long long n = (long long)g.nx * g.ny;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        const int j = (int)(e / g.nx), i = (int)(e % g.nx);
        const size_t c = (size_t)j * g.pitch + i;
        float u, v, p, T;
        const float rho = U[c];
        prim_from_cons(rho, U[g.plane + c], U[2 * g.plane + c], U[3 * g.plane + c], U[4 * g.plane + c], u, v, p, T);
        ls = fmaxf(ls, wave_speed(u, v, p, rho));
        const float mu = (mb_type(mask[c]) == CT_SOLID) ? 0.0f : sutherland_mu(T);
        ln = fmaxf(ln, mu / (rho + 1e-10f));
    }
    block_max2_publish<256>(ls, ln, sc->red);
}

__global__ void k_cfl_publish(DevScalars *sc) {
    sc->cfl[0] = sc->red[0];
    sc->cfl[1] = sc->red[1];
    sc->red[0] = 0.0f;
    sc->red[1] = 0.0f;
}

// ------------------------------------------------------------ launchers
size_t stage_smem_bytes(int stage, const StageTune &tn) {
#define FVM_SZ(NT, K)                                                                              \
    if (tn.nt == NT && tn.ring == K)                                                               \
        return stage == 1 ? StageLayout<NT, K, 1>::total : StageLayout<NT, K, 2>::total;
    FVM_SZ(128, 4) FVM_SZ(128, 6) FVM_SZ(256, 4) FVM_SZ(256, 6)
#undef FVM_SZ
    return 0;
}
size_t viscous_smem_bytes(const StageTune &tn) {
    if (tn.nt == 128 && tn.ring == 6) return ViscLayout<128, 6>::total;
    if (tn.nt == 128 && tn.ring == 4) return ViscLayout<128, 4>::total;
    if (tn.nt == 256 && tn.ring == 6) return ViscLayout<256, 6>::total;
    if (tn.nt == 256 && tn.ring == 4) return ViscLayout<256, 4>::total;
    return 0;
}
int stage_cols_per_cta(const StageTune &tn) { return tn.nt - 4; }
int stage_box_in(const StageTune &) { return kBox; }
int stage_box_blend(const StageTune &tn) { return tn.nt - 4; }

template <int NT, int K, int STAGE, int SCHEME, int LIM>
static cudaError_t stage_attr_t() {
    using L = StageLayout<NT, K, STAGE>;
    cudaError_t e = cudaFuncSetAttribute(k_stage<NT, K, STAGE, SCHEME, LIM, false>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L::total);
    if (STAGE == 2 && e == cudaSuccess)
        e = cudaFuncSetAttribute(k_stage<NT, K, STAGE, SCHEME, LIM, STAGE == 2>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L::total);
    return e;
}

template <int NT, int K>
static cudaError_t visc_attr_t() {
    cudaError_t e = cudaFuncSetAttribute(k_viscous<NT, K, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)ViscLayout<NT, K>::total);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k_viscous<NT, K, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)ViscLayout<NT, K>::total);
    return e;
}

template <int NT, int K, int STAGE, int SCHEME, int LIM>
static cudaError_t stage_batch_attr_t() {
    using L = StageLayout<NT, K, STAGE>;
    return cudaFuncSetAttribute(k_stage_batch<NT, K, STAGE, SCHEME, LIM>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)L::total);
}

template <int NT, int K>
static cudaError_t prepare_t() {
    cudaError_t e = cudaSuccess, r;
#define FVM_A(S, A, B)                                                          \
    if ((r = stage_attr_t<NT, K, S, A, B>()) != cudaSuccess) e = r;             \
    if ((r = stage_batch_attr_t<NT, K, S, A, B>()) != cudaSuccess) e = r;
    FVM_A(1, 0, 0) FVM_A(1, 0, 1) FVM_A(1, 1, 0) FVM_A(1, 1, 1)
    FVM_A(2, 0, 0) FVM_A(2, 0, 1) FVM_A(2, 1, 0) FVM_A(2, 1, 1)
#undef FVM_A
    if ((r = visc_attr_t<NT, K>()) != cudaSuccess) e = r;
    if ((r = cudaFuncSetAttribute(k_viscous_batch<NT, K>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)ViscLayout<NT, K>::total)) != cudaSuccess)
        e = r;
    return e;
}

// Opt the step kernels of a tuning into their dynamic shared memory (done
// once at set-up, outside any stream capture).
cudaError_t prepare_step_kernels(const StageTune &tn) {
    if (tn.nt == 128 && tn.ring == 6) return prepare_t<128, 6>();
    if (tn.nt == 128 && tn.ring == 4) return prepare_t<128, 4>();
    if (tn.nt == 256 && tn.ring == 6) return prepare_t<256, 6>();
    if (tn.nt == 256 && tn.ring == 4) return prepare_t<256, 4>();
    return cudaErrorInvalidValue;
}

// Step kernels launch with programmatic stream serialization: each may start
// while its predecessor in the stream drains (see pdl_wait / pdl_trigger);
// FVM_NO_PDL set in the environment launches them plainly.
static bool pdl_enabled() {
    static const bool on = getenv("FVM_NO_PDL") == nullptr;
    return on;
}

template <typename... KArgs, typename... Args>
static cudaError_t launch_step_kernel(bool pdl, void (*kern)(KArgs...), dim3 grid, dim3 block, size_t smem,
                                      cudaStream_t st, Args &&...args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = (pdl && pdl_enabled()) ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kern, std::forward<Args>(args)...);
}

template <int NT, int K, int STAGE, int SCHEME, int LIM>
static cudaError_t launch_stage_t(const StageTune &tn, const CUtensorMap &tm_in, const CUtensorMap &tm_blend,
                                  const StepArgs &a, cudaStream_t st) {
    using L = StageLayout<NT, K, STAGE>;
    // the display-field variant only for a stage 2 that writes one
    auto kern = (STAGE == 2 && a.disp) ? k_stage<NT, K, STAGE, SCHEME, LIM, STAGE == 2>
                                       : k_stage<NT, K, STAGE, SCHEME, LIM, false>;
    dim3 grid((a.g.nx + L::W - 1) / L::W, (a.g.ny + a.rows_per_cta - 1) / a.rows_per_cta);
    return launch_step_kernel(a.pdl != 0, kern, grid, dim3(NT), L::total, st, tm_in, tm_blend, a);
}

template <int NT, int K, int STAGE>
static cudaError_t launch_stage_s(int scheme, int lim, const StageTune &tn, const CUtensorMap &tm_in,
                                  const CUtensorMap &tm_blend, const StepArgs &a, cudaStream_t st) {
    if (scheme == 0 && lim == 0) return launch_stage_t<NT, K, STAGE, 0, 0>(tn, tm_in, tm_blend, a, st);
    if (scheme == 0 && lim == 1) return launch_stage_t<NT, K, STAGE, 0, 1>(tn, tm_in, tm_blend, a, st);
    if (scheme == 1 && lim == 0) return launch_stage_t<NT, K, STAGE, 1, 0>(tn, tm_in, tm_blend, a, st);
    return launch_stage_t<NT, K, STAGE, 1, 1>(tn, tm_in, tm_blend, a, st);
}

cudaError_t launch_stage(int stage, int scheme, int limiter, const StageTune &tn, const CUtensorMap &tm_in,
                         const CUtensorMap &tm_blend, const StepArgs &a, cudaStream_t st) {
#define FVM_ST(NT, K)                                                                                      \
    if (tn.nt == NT && tn.ring == K)                                                                       \
        return stage == 1 ? launch_stage_s<NT, K, 1>(scheme, limiter, tn, tm_in, tm_blend, a, st)          \
                          : launch_stage_s<NT, K, 2>(scheme, limiter, tn, tm_in, tm_blend, a, st);
    FVM_ST(128, 4) FVM_ST(128, 6) FVM_ST(256, 4) FVM_ST(256, 6)
#undef FVM_ST
    return cudaErrorInvalidValue;
}

template <int NT, int K>
static cudaError_t launch_viscous_t(const CUtensorMap &tm_in, const StepArgs &a, cudaStream_t st) {
    using L = ViscLayout<NT, K>;
    auto kern = a.disp ? k_viscous<NT, K, true> : k_viscous<NT, K, false>;
    dim3 grid((a.g.nx + L::W - 1) / L::W, (a.g.ny + a.rows_per_cta - 1) / a.rows_per_cta);
    return launch_step_kernel(a.pdl != 0, kern, grid, dim3(NT), L::total, st, tm_in, a);
}

cudaError_t launch_viscous(const StageTune &tn, const CUtensorMap &tm_in, const StepArgs &a, cudaStream_t st) {
    if (tn.nt == 128 && tn.ring == 6) return launch_viscous_t<128, 6>(tm_in, a, st);
    if (tn.nt == 128 && tn.ring == 4) return launch_viscous_t<128, 4>(tm_in, a, st);
    if (tn.nt == 256 && tn.ring == 6) return launch_viscous_t<256, 6>(tm_in, a, st);
    if (tn.nt == 256 && tn.ring == 4) return launch_viscous_t<256, 4>(tm_in, a, st);
    return cudaErrorInvalidValue;
}

// ---- batched launches: persistent grids sized by occupancy
template <class KERN>
static int persistent_grid(KERN kern, int threads, size_t smem, int ntiles) {
    int per_sm = 0, sms = 0, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, threads, smem);
    int g = std::max(1, per_sm) * std::max(1, sms);
    return std::max(1, std::min(g, ntiles));
}

template <int NT, int K, int STAGE, int SCHEME, int LIM>
static cudaError_t launch_stage_batch_t(const BatchInst *insts, const TileDesc *tiles, int ntiles, int rows,
                                        int early, bool pdl, cudaStream_t st) {
    using L = StageLayout<NT, K, STAGE>;
    auto kern = k_stage_batch<NT, K, STAGE, SCHEME, LIM>;
    const int grid = persistent_grid(kern, NT, L::total, ntiles);
    return launch_step_kernel(pdl, kern, dim3(grid), dim3(NT), L::total, st, insts, tiles, ntiles, rows, early);
}

template <int NT, int K, int STAGE>
static cudaError_t launch_stage_batch_s(int scheme, int lim, const BatchInst *insts, const TileDesc *tiles,
                                        int ntiles, int rows, int early, bool pdl, cudaStream_t st) {
#define FVM_SBT(A, B) launch_stage_batch_t<NT, K, STAGE, A, B>(insts, tiles, ntiles, rows, early, pdl, st)
    if (scheme == 0 && lim == 0) return FVM_SBT(0, 0);
    if (scheme == 0 && lim == 1) return FVM_SBT(0, 1);
    if (scheme == 1 && lim == 0) return FVM_SBT(1, 0);
    return FVM_SBT(1, 1);
#undef FVM_SBT
}

cudaError_t launch_stage_batch(int stage, int scheme, int limiter, const StageTune &tn, const BatchInst *insts,
                               const TileDesc *tiles, int ntiles, int early, bool pdl, cudaStream_t st) {
    if (ntiles <= 0) return cudaSuccess;
#define FVM_SB(NT, K)                                                                                             \
    if (tn.nt == NT && tn.ring == K)                                                                              \
        return stage == 1                                                                                         \
                   ? launch_stage_batch_s<NT, K, 1>(scheme, limiter, insts, tiles, ntiles, tn.rows, early, pdl, st) \
                   : launch_stage_batch_s<NT, K, 2>(scheme, limiter, insts, tiles, ntiles, tn.rows, early, pdl, st);
    FVM_SB(128, 4) FVM_SB(128, 6) FVM_SB(256, 4) FVM_SB(256, 6)
#undef FVM_SB
    return cudaErrorInvalidValue;
}

template <int NT, int K>
static cudaError_t launch_viscous_batch_t(const BatchInst *insts, const TileDesc *tiles, int ntiles, int rows,
                                          int post, cudaStream_t st) {
    auto kern = k_viscous_batch<NT, K>;
    const int grid = persistent_grid(kern, NT, ViscLayout<NT, K>::total, ntiles);
    return launch_step_kernel(true, kern, dim3(grid), dim3(NT), ViscLayout<NT, K>::total, st, insts, tiles, ntiles,
                              rows, post);
}

cudaError_t launch_viscous_batch(const StageTune &tn, const BatchInst *insts, const TileDesc *tiles, int ntiles,
                                 int post, cudaStream_t st) {
    if (ntiles <= 0) return cudaSuccess;
    if (tn.nt == 128 && tn.ring == 6) return launch_viscous_batch_t<128, 6>(insts, tiles, ntiles, tn.rows, post, st);
    if (tn.nt == 128 && tn.ring == 4) return launch_viscous_batch_t<128, 4>(insts, tiles, ntiles, tn.rows, post, st);
    if (tn.nt == 256 && tn.ring == 6) return launch_viscous_batch_t<256, 6>(insts, tiles, ntiles, tn.rows, post, st);
    if (tn.nt == 256 && tn.ring == 4) return launch_viscous_batch_t<256, 4>(insts, tiles, ntiles, tn.rows, post, st);
    return cudaErrorInvalidValue;
}

cudaError_t launch_ghost_batch(const BatchInst *insts, const GhostChunk *chunks, int nchunks, int mode,
                               cudaStream_t st) {
    if (nchunks <= 0) return cudaSuccess;
    return launch_step_kernel(true, k_ghost_batch, dim3(nchunks), dim3(128), 0, st, insts, chunks, mode);
}

// Failure-path probe: one warp waits, through the kernels' own bounded wait,
// on an mbarrier nothing arrives on, so the wait must give up after `limit`
// SM cycles and record the timeout in the error word, as a stuck staging
// load would.
__global__ void k_wait_probe(DevScalars *sc, long long limit) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        fence_barrier_init();
    }
    __syncthreads();
    const bool ok = mbar_wait_bounded(&bar, 0u, limit);
    if (!ok && threadIdx.x == 0) record_error(sc, kErrTimeout);
}

cudaError_t launch_wait_probe(DevScalars *sc, long long limit_cycles, cudaStream_t st) {
    k_wait_probe<<<1, 32, 0, st>>>(sc, limit_cycles);
    return cudaGetLastError();
}

__global__ void k_set_display(DisplayDesc *d, float *ptr, int kind) {
    d->ptr = ptr;
    d->kind = kind;
}

cudaError_t launch_set_display(DisplayDesc *d, float *ptr, int kind, cudaStream_t st) {
    k_set_display<<<1, 1, 0, st>>>(d, ptr, kind);
    return cudaGetLastError();
}

cudaError_t launch_ghost(const GhostArgs &a, cudaStream_t st) {
    int blocks = (a.n + 127) / 128;
    if (blocks < 1) blocks = 1;
    return launch_step_kernel(true, k_ghost, dim3(blocks), dim3(128), 0, st, a);
}

cudaError_t launch_bc_phase1(const GridDesc &g, float *U, const uint8_t *mask, const Freestream &fs, cudaStream_t st) {
    dim3 b(32, 8), gr((g.nx + 31) / 32, (g.ny + 7) / 8);
    k_bc_phase1<<<gr, b, 0, st>>>(g, U, mask, fs);
    return cudaGetLastError();
}

cudaError_t launch_cfl_state(const GridDesc &g, const float *U, const uint8_t *mask, DevScalars *sc, cudaStream_t st) {
    long long n = (long long)g.nx * g.ny;
    int blocks = (int)((n + 255) / 256);
    if (blocks > 148 * 8) blocks = 148 * 8;
    k_cfl_state<<<blocks, 256, 0, st>>>(g, U, mask, sc);
    k_cfl_publish<<<1, 1, 0, st>>>(sc);
    return cudaGetLastError();
}

}  // namespace fvm
