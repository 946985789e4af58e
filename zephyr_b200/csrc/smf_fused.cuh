// smf_fused.cuh -- the whole second-order step of a structured rectangle in
// ONE kernel per stage: limited gradients, predictor, face-once corrector,
// update and the next step's CFL minimum, for a tile of cells held in shared
// memory.  Nothing but the state (and the isolation counters) crosses HBM:
// the gradients and the half-step state of the two-pass form (smf_tiled.cuh
// k_grad_predict -> k_faces) never leave the SM.
//
// Scheme: math/solver/sm_fluid.cpp:81-102 (compute_grad 116-125, fluxes_stage1
// 176-253, fluxes_stage2 255-366) in the precisions of the two-pass tiled
// kernels (FAST: FP64; MIXED: FP32 primitive states, gradients and fluxes
// with FP64 conserved sums, update, pressure recovery and dt).  The rectangle
// is uniform, so the least-squares geometry of gradient.h:226-282 reduces to
// per-axis constants: with cell size h along an axis and the differences
// dL = z_low - z, dR = z_high - z to the two neighbours (a boundary slot takes
// the reflected own value, sm_fluid.cpp:69-79), the unlimited slope is
// (dR - dL) / 2h, and the limited refit of gradient.h:412-474 becomes
//     g = (phi(-dL, dR) dR - phi(-dR, dL) dL) / 2h,
// because 2 g0 (dr . n) - dF equals -dR on the low face and -dL on the high
// one.  For van Albada 1 (limiter.cxx:69-82) both limiter values vanish
// unless dL dR < 0, and then g = -dL dR (dR - dL) / ((dL^2 + dR^2) h): one
// division per component instead of two.  Face centres sit at +-h/2 along
// the face normal.  These are the reference's formulas up to the rounding of
// the mesh coordinates, far inside the FAST form's 1e-12 per-step bound.
//
// Tile geometry (block = 32 x (TH + 2) threads, thread (l, r)):
//   interior cells  rows i0 .. i0 + TH - 1, columns j0 .. j0 + 29   (30 x TH)
//   G region        rows i0 - 1 .. i0 + TH, columns j0 - 1 .. j0 + 30: one
//                   cell per thread; gradients (and the half step) of every
//                   cell whose face touches an interior cell
//   Z region        rows i0 - 2 .. i0 + TH + 1, columns j0 - 2 .. j0 + 31:
//                   the state the G region's gradients read
// Phases, separated by block barriers:
//   0  stage Z from HBM (wrapped on periodic axes)
//   1  per G cell: limited gradient, for the predictor-corrector also the
//      half step (physical flux of the cell's own face values)
//   2  per thread: the +x face (G rows r | r + 1) and the +y face (G columns
//      l | l + 1) that bound an interior cell, each computed once
//   3  per interior cell: flux sum in the reference's slot order, update,
//      pressure recovery, isolation counters, CFL term, block minimum
#pragma once

#include <type_traits>

#include "smf_tiled.cuh"

namespace zg {
namespace tiled {

// Stage of the fused kernel.
enum : int { FUSED_PC = 1, FUSED_HEUN_A = 2, FUSED_HEUN_B = 3 };

// ---------------------------------------------------------------------------
// Reciprocals.  FP64: Newton-Raphson iteration for 1/x (y <- y + y (1 - x y),
// each step doubling the correct bits; e.g. P. Markstein, IBM J. Res. Dev.
// 34(1), 1990) from the hardware's approximate reciprocal (PTX
// rcp.approx.ftz.f64), two steps; within 2 ulp of 1/x for normal finite x.
// FP32 (MIXED, compiled with approximate division): 1 / x.
__device__ __forceinline__ double rcp_nr(double x) {
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    double e = fma(-x, y, 1.0);
    y = fma(y, e, y);
    e = fma(-x, y, 1.0);
    return fma(y, e, y);
}
__device__ __forceinline__ float rcp_r(float x) { return 1.0f / x; }
__device__ __forceinline__ double rcp_r(double x) { return rcp_nr(x); }

// A face state with its reciprocal density.
template <typename R>
struct FS {
    R r, u, v, p, e, ri;
};

template <typename R>
__device__ __forceinline__ R energy_ri(const EosR<R> &eos, R P, R ri, R igm1) {
    return eos.kind == EOS_IDEAL ? P * ri * igm1 : eos.e0 + (P + eos.gamma * eos.P0) * ri * igm1;
}

// models.cpp:58-63 (is_bad) without integer classification: every compare
// with a NaN is false, and the infinities fail the range tests.
template <typename R>
__device__ __forceinline__ bool bad_fs(const FS<R> &z, R pmin) {
    const R inf = R(INFINITY);
    const bool ok = z.r > R(0) && z.r < inf && z.p >= pmin && z.p < inf && z.e > -inf && z.e < inf;
    return !ok;
}

// phys flux along x of z (models.cpp:131-137 with the normal (1, 0))
template <typename R>
__device__ __forceinline__ C4<R> flux_x(const FS<R> &z) {
    const R ru = z.r * z.u;
    return C4<R>{ru, ru * z.u + z.p, ru * z.v, (z.r * (z.e + R(0.5) * (z.u * z.u + z.v * z.v)) + z.p) * z.u};
}

// HLLC (hllc.cpp:23-83) in the face frame.  hllc.cpp writes the flux in its
// symmetric form 1/2 (F_L + F_R + S_L (Q*_L - Q_L) + |S_C| (Q*_L - Q*_R) +
// S_R (Q*_R - Q_R)); through the Rankine-Hugoniot relations that define the
// star states this is the star flux on the side of the contact the face
// lies on: F_L + S_L (Q*_L - Q_L) for S_C >= 0, F_R + S_R (Q*_R - Q_R)
// otherwise.  The kernel evaluates that one side (the two forms agree to
// rounding), with the side's state chosen before the arithmetic so that a
// warp runs one path.
template <typename R>
__device__ __forceinline__ C4<R> hllc_fs(const FS<R> &L, const FS<R> &Rs, const EosR<R> &eos) {
    const R cL = sqrt(eos.gamma * (L.p + eos.P0) * L.ri), cR = sqrt(eos.gamma * (Rs.p + eos.P0) * Rs.ri);
    // (the states are finite here: a NaN ordering of std::min does not arise)
    const R SL = fmin(L.u - cL, Rs.u - cR);
    const R SR = fmax(L.u + cL, Rs.u + cR);
    if (SL >= R(0)) return flux_x(L);
    if (SR <= R(0)) return flux_x(Rs);
    const R aL = L.r * (SL - L.u), aR = Rs.r * (SR - Rs.u);
    const R SC = (L.p - Rs.p + aR * Rs.u - aL * L.u) * rcp_r(aR - aL);
    const bool left = SC >= R(0);
    FS<R> X;
    X.r = left ? L.r : Rs.r;
    X.u = left ? L.u : Rs.u;
    X.v = left ? L.v : Rs.v;
    X.p = left ? L.p : Rs.p;
    X.e = left ? L.e : Rs.e;
    const R SX = left ? SL : SR, aX = left ? aL : aR;
    const R rs = aX * rcp_r(SX - SC);
    const R EX = X.e + R(0.5) * (X.u * X.u + X.v * X.v);
    const R Es = EX + (SC - X.u) * (SC + X.p * rcp_r(aX));
    const R ru = X.r * X.u;
    const R rE = X.r * EX;
    C4<R> f;
    f.r = ru + SX * (rs - X.r);
    f.mu = ru * X.u + X.p + SX * (rs * SC - ru);
    f.mv = ru * X.v + SX * (rs * X.v - X.r * X.v);
    f.E = (rE + X.p) * X.u + SX * (rs * Es - rE);
    return f;
}

// HLL (hll.cpp:23-57) in the face frame (isolated cells, and the HLL method)
template <typename R>
__device__ __forceinline__ C4<R> hll_fs(const FS<R> &L, const FS<R> &Rs, const EosR<R> &eos) {
    const R cL = sqrt(eos.gamma * (L.p + eos.P0) * L.ri), cR = sqrt(eos.gamma * (Rs.p + eos.P0) * Rs.ri);
    const R SL = fmin(L.u - cL, fmin(Rs.u - cR, R(0)));
    const R SR = fmax(L.u + cL, fmax(Rs.u + cR, R(0)));
    const C4<R> FL = flux_x(L), FR = flux_x(Rs);
    const R EL = L.e + R(0.5) * (L.u * L.u + L.v * L.v);
    const R ER = Rs.e + R(0.5) * (Rs.u * Rs.u + Rs.v * Rs.v);
    const R QL[4] = {L.r, L.r * L.u, L.r * L.v, L.r * EL};
    const R QR[4] = {Rs.r, Rs.r * Rs.u, Rs.r * Rs.v, Rs.r * ER};
    const R fl[4] = {FL.r, FL.mu, FL.mv, FL.E}, fr[4] = {FR.r, FR.mu, FR.mv, FR.E};
    const R inv = rcp_r(SR - SL), SLR = SL * SR;
    R o[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) o[k] = (SR * fl[k] - SL * fr[k] + SLR * (QR[k] - QL[k])) * inv;
    return C4<R>{o[0], o[1], o[2], o[3]};
}

// Limited slope of one component along one axis (see the header comment);
// inv2h = 1 / 2h, invh = 1 / h.
template <int LIM, typename R>
__device__ __forceinline__ R slope(int kind, R dL, R dR, R inv2h, R invh) {
    if (LIM == LIM_VANALBADA1) {
        const R p = dL * dR;
        if (p >= R(0)) return R(0);
        return -p * (dR - dL) * rcp_r(dL * dL + dR * dR) * invh;
    }
    return (limit<LIM, R>(kind, -dL, dR) * dR - limit<LIM, R>(kind, -dR, dL) * dL) * inv2h;
}

// FP64 primitive state from conserved variables (models.cpp:27-32) with the
// reciprocal density kept for the sound speed.
__device__ __forceinline__ P5<double> prim_ri(const C4<double> &q, const EosD &eos, double &ri) {
    P5<double> z;
    z.r = q.r;
    ri = rcp_nr(q.r);
    z.u = q.mu * ri;
    z.v = q.mv * ri;
    z.e = q.E * ri - 0.5 * (z.u * z.u + z.v * z.v);
    z.p = eos.kind == EOS_IDEAL ? eos.gm1 * z.r * z.e : eos.gm1 * z.r * (z.e - eos.e0) - eos.gamma * eos.P0;
    return z;
}

// Flux across a boundary face (WALL / ZOE, sm_fluid.cpp:69-79) from the
// reconstructed state zm of its only cell, whose slot s_own it is: the ghost
// state reflects the normal velocity at a wall; the flux is returned in the
// +x / +y direction (negated when the cell lies on the face's high side).
// Out of line: boundary faces are few, and one copy of the Riemann solver
// serves all of them.
template <typename R>
__device__ __noinline__ C4<R> boundary_flux(FS<R> zm, int s_own, int bc, bool use_hll, EosR<R> eos, bool own_a) {
    FS<R> zp = zm;
    if (bc == BC_WALL) {
        if (s_own < 2) zp.u = -zp.u;
        else zp.v = -zp.v;
    }
    to_local(s_own, zm.u, zm.v);
    to_local(s_own, zp.u, zp.v);
    C4<R> lf = use_hll ? hll_fs(zm, zp, eos) : hllc_fs(zm, zp, eos);
    to_global(s_own, lf.mu, lf.mv);
    if (!own_a) {
        lf.r = -lf.r;
        lf.mu = -lf.mu;
        lf.mv = -lf.mv;
        lf.E = -lf.E;
    }
    return lf;
}

template <typename R, int TH, int MODE>
struct FusedLayout {
    static constexpr int ZR = TH + 4, ZC = 34;  // Z region
    static constexpr int GR = TH + 2, GC = 32;  // G region (= the block)
    static constexpr int NT = 32 * GR;
    static constexpr bool PC = MODE == FUSED_PC;
    static constexpr size_t al(size_t x) { return (x + 15) / 16 * 16; }
    static constexpr size_t z_bytes = al(sizeof(R) * 5 * ZR * ZC);
    // face fluxes (widened to FP64 once, where they are computed): +x faces
    // of G rows 0..TH, +y faces of G rows 1..TH
    static constexpr size_t fx_bytes = al(sizeof(double) * 4 * (TH + 1) * GC);
    static constexpr size_t fy_bytes = al(sizeof(double) * 4 * TH * GC);
    // The predictor-corrector reads only the G region after phase 1, so the
    // fluxes may overwrite Z; the Heun stages reconstruct from Z itself.
    static constexpr size_t off_z = 0;
    static constexpr size_t off_fx = PC ? 0 : z_bytes;
    static constexpr size_t off_fy = off_fx + fx_bytes;
    static constexpr size_t zf_end = PC ? (z_bytes > fx_bytes + fy_bytes ? z_bytes : fx_bytes + fy_bytes)
                                        : z_bytes + fx_bytes + fy_bytes;
    static constexpr size_t off_g = zf_end;
    static constexpr size_t g_bytes = al(sizeof(R) * 8 * GR * GC);
    static constexpr size_t off_h = off_g + g_bytes;
    static constexpr size_t h_bytes = PC ? al(sizeof(R) * 5 * GR * GC) : 0;
    // conserved state at t^n of the G cells (predictor-corrector)
    static constexpr size_t off_q = off_h + h_bytes;
    static constexpr size_t q_bytes = PC ? al(sizeof(double) * 4 * GR * GC) : 0;
    static constexpr size_t off_zin = off_q + q_bytes;
    static constexpr size_t zin_bytes = al(ZR * ZC);
    static constexpr size_t off_wt = off_zin + zin_bytes;
    static constexpr size_t wt_bytes = al(GR * GC);
    static constexpr size_t off_red = off_wt + wt_bytes;
    static constexpr size_t bytes = off_red + al(8 * GR);
};

// x wrapped into [0, n) for any x (the Z region reaches two cells beyond the
// mesh, more than one period when n == 1).
__device__ __forceinline__ int wrap_any(int x, int n) {
    x = wrap_idx(x, n);
    return x < 0 ? (x % n + n) % n : x;
}

// Global cell of Z entry (zr, zc) (entry (2, 2) is cell (i0, j0)); false
// outside a non-periodic side.
__device__ __forceinline__ bool z_cell(const StructMesh &m, int i0, int j0, int zr, int zc, int &gi, int &gj) {
    gi = i0 + zr - 2;
    gj = j0 + zc - 2;
    if (gi < 0 || gi >= m.nx) {
        if (!m.xper) return false;
        gi = wrap_any(gi, m.nx);
    }
    if (gj < 0 || gj >= m.ny) {
        if (!m.yper) return false;
        gj = wrap_any(gj, m.ny);
    }
    return true;
}

template <typename R, bool MIXED, int MODE, int LIM, int TH, int MINB>
__global__ void __launch_bounds__(32 * (TH + 2), MINB) k_step(SmfArgs a, Fields<R> f) {
    using L = FusedLayout<R, TH, MODE>;
    constexpr int ZR = L::ZR, ZC = L::ZC, GR = L::GR, GC = L::GC, NT = L::NT;
    constexpr bool PC = MODE == FUSED_PC;
    extern __shared__ __align__(16) unsigned char smem[];
    R(*Z)[ZR][ZC] = reinterpret_cast<R(*)[ZR][ZC]>(smem + L::off_z);
    double(*FX)[TH + 1][GC] = reinterpret_cast<double(*)[TH + 1][GC]>(smem + L::off_fx);
    double(*FY)[TH][GC] = reinterpret_cast<double(*)[TH][GC]>(smem + L::off_fy);
    R(*G)[GR][GC] = reinterpret_cast<R(*)[GR][GC]>(smem + L::off_g);
    R(*H)[GR][GC] = reinterpret_cast<R(*)[GR][GC]>(smem + L::off_h);
    double(*Q)[GR][GC] = reinterpret_cast<double(*)[GR][GC]>(smem + L::off_q);
    unsigned char(*zin)[ZC] = reinterpret_cast<unsigned char(*)[ZC]>(smem + L::off_zin);
    unsigned char(*wt)[GC] = reinterpret_cast<unsigned char(*)[GC]>(smem + L::off_wt);
    unsigned long long *red = reinterpret_cast<unsigned long long *>(smem + L::off_red);

    const StructMesh &m = a.mesh;
    const int l = threadIdx.x, r = threadIdx.y, tid = r * 32 + l;
    const int i0 = blockIdx.y * TH, j0 = blockIdx.x * 30;
    const EosR<R> eos = eos_as<R>(a.eos);
    const R igm1 = R(1.0 / a.eos.gm1);
    // per-axis geometry of the uniform rectangle
    const R halfx = R(0.5 * m.hx), halfy = R(0.5 * m.hy);
    const R inv2hx = R(0.5 / m.hx), inv2hy = R(0.5 / m.hy), invhx = R(1.0 / m.hx), invhy = R(1.0 / m.hy);
    // source of the stage: the state at t^n, or the Heun stage value z*
    const R *const *src = MODE == FUSED_HEUN_B ? const_cast<const R *const *>(f.h) : f.w;

    if (MODE != FUSED_HEUN_B && blockIdx.x == 0 && blockIdx.y == 0 && tid == 0) {
        *f.dt_out = step_dt(a, f.slot_cur);
        *f.slot_clr = 0x7FEFFFFFFFFFFFFFull;
    }
    const double dt = step_dt(a, f.slot_cur);

    // ---- phase 0: stage Z ----------------------------------------------------
    for (int k = tid; k < ZR * ZC; k += NT) {
        const int zr = k / ZC, zc = k - zr * ZC;
        int gi, gj;
        const bool in = z_cell(m, i0, j0, zr, zc, gi, gj);
        zin[zr][zc] = in;
        if (in) {
            const int g = gi * m.ny + gj;
#pragma unroll
            for (int q = 0; q < 5; ++q) Z[q][zr][zc] = src[q][g];
        }
    }
    __syncthreads();

    // ---- phase 1: gradients (and the half step) of the G cell (r, l) ---------
    if (zin[r + 1][l + 1]) {
        int gi = i0 - 1 + r, gj = j0 - 1 + l;  // wrapped global coordinates
        if (m.xper) gi = wrap_idx(gi, m.nx);
        if (m.yper) gj = wrap_idx(gj, m.ny);
        const int zr = r + 1, zc = l + 1;
        // conserved state of the cell at t^n (predictor-corrector): FAST from
        // the staged primitive state, MIXED from the FP64 fields (loaded here,
        // ahead of the gradient arithmetic)
        C4<double> q0{0.0, 0.0, 0.0, 0.0};
        if (PC) {
            if (MIXED) {
                const int g = gi * m.ny + gj;
                q0 = C4<double>{f.q[0][g], f.q[1][g], f.q[2][g], f.q[3][g]};
            } else {
                const double rr = Z[0][zr][zc], u = Z[1][zr][zc], v = Z[2][zr][zc], e = Z[4][zr][zc];
                q0 = C4<double>{rr, rr * u, rr * v, rr * (e + 0.5 * (u * u + v * v))};
            }
        }
        // boundary flags of the four slots (the normals are the axes)
        const int fL = gi > 0 ? BC_INNER : m.bc[0];
        const int fR = gi < m.nx - 1 ? BC_INNER : m.bc[1];
        const int fB = gj > 0 ? BC_INNER : m.bc[2];
        const int fT = gj < m.ny - 1 ? BC_INNER : m.bc[3];
        const bool bL = is_boundary(fL), bR = is_boundary(fR), bB = is_boundary(fB), bT = is_boundary(fT);
        R gx[4], gy[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            // a boundary slot takes the reflected own value (only the normal
            // velocity changes sign at a wall)
            const R c = Z[q][zr][zc];
            const R nL = bL ? ((q == 1 && fL == BC_WALL) ? -c : c) : Z[q][zr - 1][zc];
            const R nR = bR ? ((q == 1 && fR == BC_WALL) ? -c : c) : Z[q][zr + 1][zc];
            const R nB = bB ? ((q == 2 && fB == BC_WALL) ? -c : c) : Z[q][zr][zc - 1];
            const R nT = bT ? ((q == 2 && fT == BC_WALL) ? -c : c) : Z[q][zr][zc + 1];
            gx[q] = slope<LIM, R>(a.limiter, nL - c, nR - c, inv2hx, invhx);
            gy[q] = slope<LIM, R>(a.limiter, nB - c, nT - c, inv2hy, invhy);
            G[q][r][l] = gx[q];
            G[4 + q][r][l] = gy[q];
        }
        if (PC) {
            const int g = gi * m.ny + gj;
            const bool waiting = f.wait_in[g] > 0;
            wt[r][l] = waiting;
            const FS<R> zc5{Z[0][zr][zc], Z[1][zr][zc], Z[2][zr][zc], Z[3][zr][zc], Z[4][zr][zc], R(0)};
            P5<R> hz{zc5.r, zc5.u, zc5.v, zc5.p, zc5.e};
            if (!waiting) {
                // predictor (sm_fluid.cpp:176-253): half step with the physical
                // flux of the cell's own face values; the flux of the low face
                // (normal -x or -y) is minus the flux along the axis
                double F[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
                for (int s = 0; s < 4; ++s) {
                    const bool ax = s < 2;
                    const R off = s == 0 ? -halfx : (s == 1 ? halfx : (s == 2 ? -halfy : halfy));
                    const R *gg = ax ? gx : gy;
                    FS<R> zm{zc5.r + gg[0] * off, zc5.u + gg[1] * off, zc5.v + gg[2] * off, zc5.p + gg[3] * off,
                             R(0), R(0)};
                    zm.ri = rcp_r(zm.r);
                    zm.e = energy_ri(eos, zm.p, zm.ri, igm1);
                    if (bad_fs(zm, eos.pmin)) zm = zc5;
                    C4<R> lf;
                    if (ax) {
                        lf = flux_x(zm);
                    } else {  // flux along y: swap the velocity components
                        const FS<R> zt{zm.r, zm.v, zm.u, zm.p, zm.e, zm.ri};
                        const C4<R> t = flux_x(zt);
                        lf = C4<R>{t.r, t.mv, t.mu, t.E};
                    }
                    const double w = (s == 0 || s == 2) ? -(ax ? m.hy : m.hx) : (ax ? m.hy : m.hx);
                    F[0] += (double)lf.r * w;
                    F[1] += (double)lf.mu * w;
                    F[2] += (double)lf.mv * w;
                    F[3] += (double)lf.E * w;
                }
                const double coef = 0.5 * dt / m.vol;
                C4<double> q = q0;
                q.r -= coef * F[0];
                q.mu -= coef * F[1];
                q.mv -= coef * F[2];
                q.E -= coef * F[3];
                double ri;
                const P5<double> hd = prim_ri(q, a.eos, ri);
                if (!bad64(hd, a.eos)) hz = down<R>(hd);
            }
            H[0][r][l] = hz.r;
            H[1][r][l] = hz.u;
            H[2][r][l] = hz.v;
            H[3][r][l] = hz.p;
            H[4][r][l] = hz.e;
            Q[0][r][l] = q0.r;
            Q[1][r][l] = q0.mu;
            Q[2][r][l] = q0.mv;
            Q[3][r][l] = q0.E;
        }
    }
    __syncthreads();

    // ---- phase 2: the faces bounding interior cells, each once ---------------
    // face-state source of G cell (gr, gc): the half step, or the Z state
    // (its reciprocal density is formed only where the state itself is used)
    auto sc = [&](int gr, int gc) {
        if (PC) return FS<R>{H[0][gr][gc], H[1][gr][gc], H[2][gr][gc], H[3][gr][gc], H[4][gr][gc], R(0)};
        return FS<R>{Z[0][gr + 1][gc + 1], Z[1][gr + 1][gc + 1], Z[2][gr + 1][gc + 1], Z[3][gr + 1][gc + 1],
                     Z[4][gr + 1][gc + 1], R(0)};
    };
    auto sc_ri = [&](int gr, int gc) {
        FS<R> z = sc(gr, gc);
        z.ri = rcp_r(z.r);
        return z;
    };
    // reconstruction of G cell (gr, gc) at its face on axis `ax` (0: x, 1: y),
    // side `hi` (the +x / +y face, else the low one), FaceExtra::Direct
    // (face_extra.h:121-184); a bad value falls back to the cell state
    auto recon = [&](int gr, int gc, int ax, bool hi) {
        const FS<R> z = sc(gr, gc);
        const R off = ax == 0 ? (hi ? halfx : -halfx) : (hi ? halfy : -halfy);
        const int b = 4 * ax;
        FS<R> o{z.r + G[b][gr][gc] * off, z.u + G[b + 1][gr][gc] * off, z.v + G[b + 2][gr][gc] * off,
                z.p + G[b + 3][gr][gc] * off, R(0), R(0)};
        o.ri = rcp_r(o.r);
        o.e = energy_ri(eos, o.p, o.ri, igm1);
        if (bad_fs(o, eos.pmin)) {
            o = z;
            o.ri = rcp_r(z.r);
        }
        return o;
    };
    // interior face: the frame of the +x (DIR 0) or +y (DIR 1) normal, where
    // the rotation of rotate.cpp is the identity or (u, v) -> (v, -u)
    auto face_interior = [&](auto dirc) {
        constexpr int DIR = decltype(dirc)::value;
        const int rB = r + (DIR == 0), lB = l + (DIR == 1);
        const bool robust = PC && (wt[r][l] || wt[rB][lB]);
        FS<R> zm, zp;
        if (robust) {
            zm = sc_ri(r, l);
            zp = sc_ri(rB, lB);
        } else {
            zm = recon(r, l, DIR, true);
            zp = recon(rB, lB, DIR, false);
        }
        if (DIR == 1) {
            R t = zm.u;
            zm.u = zm.v;
            zm.v = -t;
            t = zp.u;
            zp.u = zp.v;
            zp.v = -t;
        }
        C4<R> lf = (robust || a.flux == FLUX_HLL) ? hll_fs(zm, zp, eos) : hllc_fs(zm, zp, eos);
        if (DIR == 1) {
            const R t = lf.mu;
            lf.mu = -lf.mv;
            lf.mv = t;
        }
        return lf;
    };
    // boundary face (WALL / ZOE) seen from its only cell (out of line)
    auto face_boundary = [&](int dir, bool own_a) {
        const int gr = own_a ? r : r + (dir == 0), gc = own_a ? l : l + (dir == 1);
        const int s_own = own_a ? (dir == 0 ? 1 : 3) : (dir == 0 ? 0 : 2);
        const bool robust = PC && wt[gr][gc];
        const FS<R> zm = robust ? sc_ri(gr, gc) : recon(gr, gc, dir, own_a);
        return boundary_flux<R>(zm, s_own, m.bc[s_own], robust || a.flux == FLUX_HLL, eos, own_a);
    };
    // (predictor-corrector: the fluxes overwrite Z, which no thread reads
    // after phase 1)
    if (r <= TH && l >= 1 && l <= 30) {  // +x face between G cells (r, l) and (r + 1, l)
        const bool inA = zin[r + 1][l + 1], inB = zin[r + 2][l + 1];
        C4<R> lf{R(0), R(0), R(0), R(0)};
        if (inA && inB) lf = face_interior(std::integral_constant<int, 0>{});
        else if (inA || inB) lf = face_boundary(0, inA);
        FX[0][r][l] = lf.r;
        FX[1][r][l] = lf.mu;
        FX[2][r][l] = lf.mv;
        FX[3][r][l] = lf.E;
    }
    if (r >= 1 && r <= TH && l <= 30) {  // +y face between G cells (r, l) and (r, l + 1)
        const bool inA = zin[r + 1][l + 1], inB = zin[r + 1][l + 2];
        C4<R> lf{R(0), R(0), R(0), R(0)};
        if (inA && inB) lf = face_interior(std::integral_constant<int, 1>{});
        else if (inA || inB) lf = face_boundary(1, inA);
        FY[0][r - 1][l] = lf.r;
        FY[1][r - 1][l] = lf.mu;
        FY[2][r - 1][l] = lf.mv;
        FY[3][r - 1][l] = lf.E;
    }
    __syncthreads();

    // ---- phase 3: update of the interior cells --------------------------------
    unsigned long long best = 0x7FEFFFFFFFFFFFFFull;
    const int i = i0 - 1 + r, j = j0 - 1 + l;
    if (r >= 1 && r <= TH && l >= 1 && l <= 30 && i < m.nx && j < m.ny) {
        const int ic = i * m.ny + j;
        const double hy = m.hy, hx = m.hx;
        double F[4];
#pragma unroll
        for (int k = 0; k < 4; ++k)
            F[k] = ((-FX[k][r - 1][l] * hy + FX[k][r][l] * hy) - FY[k][r - 1][l - 1] * hx) + FY[k][r - 1][l] * hx;
        const double coef = dt / m.vol;
        C4<double> q;
        if (PC) {
            q = C4<double>{Q[0][r][l], Q[1][r][l], Q[2][r][l], Q[3][r][l]};
        } else if (MODE == FUSED_HEUN_B) {
            // Q(z*) of the stage value
            const double rr = Z[0][r + 1][l + 1], u = Z[1][r + 1][l + 1], v = Z[2][r + 1][l + 1],
                         e = Z[4][r + 1][l + 1];
            q = C4<double>{rr, rr * u, rr * v, rr * (e + 0.5 * (u * u + v * v))};
        } else {
            q = q_of<R, MIXED>(f, ic);
        }
        q.r -= coef * F[0];
        q.mu -= coef * F[1];
        q.mv -= coef * F[2];
        q.E -= coef * F[3];
        if (MODE == FUSED_HEUN_B) {
            const C4<double> q0 = q_of<R, MIXED>(f, ic);
            q.r = 0.5 * (q0.r + q.r);
            q.mu = 0.5 * (q0.mu + q.mu);
            q.mv = 0.5 * (q0.mv + q.mv);
            q.E = 0.5 * (q0.E + q.E);
        }
        double ri;
        P5<double> zn = prim_ri(q, a.eos, ri);
        if (MODE == FUSED_HEUN_A) {
            st5(f.h, ic, down<R>(zn));  // Heun stage value
        } else {
            if (PC) {
                int wn = f.wait_in[ic];
                if (bad64(zn, a.eos)) {
                    // isolation (sm_fluid.cpp:354-358): keep the old state
                    zn = P5<double>{(double)f.w[0][ic], (double)f.w[1][ic], (double)f.w[2][ic],
                                    (double)f.w[3][ic], (double)f.w[4][ic]};
                    q = q_of<R, MIXED>(f, ic);
                    ri = rcp_nr(zn.r);
                    wn = 3;
                } else if (wn > 0) {
                    --wn;
                }
                f.wait_out[ic] = wn;
            }
            if (MIXED) {
                f.qn[0][ic] = q.r;
                f.qn[1][ic] = q.mu;
                f.qn[2][ic] = q.mv;
                f.qn[3][ic] = q.E;
            }
            st5(f.wn, ic, down<R>(zn));
            // CFL term of the new state for the next step (sm_fluid.cpp:104-111),
            // with the arithmetic of k_cfl, which takes the minimum after an
            // upload or a halo exchange: the same state gives the same dt
            const double c = sqrt(a.eos.gamma * (zn.p + a.eos.P0) / zn.r);
            const double dinc = sqrt(smin(m.inc2x[i], m.inc2y[j]));
            const double lam = dinc / (sqrt(zn.u * zn.u + zn.v * zn.v) + c);
            if (lam >= 0.0) best = dbits(lam);
        }
    }
    if (MODE != FUSED_HEUN_A) {
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long t2 = __shfl_xor_sync(0xffffffffu, best, o);
            best = t2 < best ? t2 : best;
        }
        if (l == 0) red[r] = best;
        __syncthreads();
        if (r == 0) {
            best = l < GR ? red[l] : 0x7FEFFFFFFFFFFFFFull;
            for (int o = 16; o > 0; o >>= 1) {
                const unsigned long long t2 = __shfl_xor_sync(0xffffffffu, best, o);
                best = t2 < best ? t2 : best;
            }
            if (l == 0) atomicMin(f.slot_nxt, best);
        }
    }
}

// Launch one stage of the fused step on `stream` (dynamic shared memory of
// FusedLayout::bytes, above the 48 KB default).
template <typename R, bool MIXED, int MODE, int LIM, int TH, int MINB>
inline void launch_fused_stage(const SmfArgs &a, const Fields<R> &f, cudaStream_t s) {
    using L = FusedLayout<R, TH, MODE>;
    static unsigned long long attr_set = 0;  // devices on which the attribute is set
    auto kern = k_step<R, MIXED, MODE, LIM, TH, MINB>;
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 64 || !(attr_set >> dev & 1ull)) {
        cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L::bytes);
        if (dev < 64) attr_set |= 1ull << dev;
    }
    dim3 block(32, TH + 2);
    dim3 grid((a.mesh.ny + 29) / 30, (a.mesh.nx + TH - 1) / TH);
    kern<<<grid, block, L::bytes, s>>>(a, f);
}

// One stage (FUSED_PC, FUSED_HEUN_A or FUSED_HEUN_B) with the limiter
// compiled in for the common ones.  HLLC and HLL only: the fused kernels
// carry neither Godunov's exact solver nor Rusanov.
template <typename R, bool MIXED, int TH, int MINB, int MODE>
inline void fused_stage(const SmfArgs &a, const Fields<R> &f, cudaStream_t s) {
    switch (a.limiter) {
        case LIM_VANALBADA1: launch_fused_stage<R, MIXED, MODE, LIM_VANALBADA1, TH, MINB>(a, f, s); break;
        case LIM_MC: launch_fused_stage<R, MIXED, MODE, LIM_MC, TH, MINB>(a, f, s); break;
        case LIM_MINMOD: launch_fused_stage<R, MIXED, MODE, LIM_MINMOD, TH, MINB>(a, f, s); break;
        default: launch_fused_stage<R, MIXED, MODE, -1, TH, MINB>(a, f, s); break;
    }
}

template <typename R, bool MIXED, int TH, int MINB>
inline void fused_dispatch(const SmfArgs &a, const Fields<R> &f, int mode, cudaStream_t s) {
    if (mode == FUSED_PC) fused_stage<R, MIXED, TH, MINB, FUSED_PC>(a, f, s);
    else if (mode == FUSED_HEUN_A) fused_stage<R, MIXED, TH, MINB, FUSED_HEUN_A>(a, f, s);
    else fused_stage<R, MIXED, TH, MINB, FUSED_HEUN_B>(a, f, s);
}

}  // namespace tiled
}  // namespace zg
