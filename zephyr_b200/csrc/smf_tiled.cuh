// smf_tiled.cuh -- throughput kernels of the single-material step on a
// structured rectangle, in two arithmetic flavours:
//   FAST   (Real = double): FP64 everywhere; the compiler may fuse multiply-adds.
//   MIXED  (Real = float):  primitive states, gradients, reconstruction and
//          Riemann fluxes in FP32; conserved variables, their accumulation and
//          update, pressure recovery from total energy, and the dt reduction
//          in FP64.
//
// Same scheme as math/solver/sm_fluid.cpp (and the parity kernels), with three
// changes of work layout that leave the mathematics unchanged:
//  * predictor fused with the gradient computation (one pass, no re-read);
//  * the corrector computes every face flux once, for a tile of cells staged
//    in shared memory, instead of once from each side (F_BA = -F_AB);
//  * the CFL minimum of the new state is reduced inside the corrector
//    (three rotating accumulator slots; no separate dt pass).
#pragma once

#include <cuda_runtime.h>

#include "smf_math.cuh"
#include "smf_types.h"

namespace zg {
namespace tiled {

// ---------------------------------------------------------------------------
// Pointwise numerics in precision R (see smf_math.cuh for the reference lines).
template <typename R>
struct P5 {
    R r, u, v, p, e;
};
template <typename R>
struct C4 {
    R r, mu, mv, E;
};

template <typename R>
struct EosR {
    int kind;
    R gamma, gm1, P0, e0, pmin;
    __device__ inline R energy_rP(R rho, R P) const {
        return kind == EOS_IDEAL ? P / (gm1 * rho) : e0 + (P + gamma * P0) / (gm1 * rho);
    }
    __device__ inline R sound(R rho, R P) const { return sqrt(gamma * (P + P0) / rho); }
};

template <typename R>
__device__ inline EosR<R> eos_as(const EosD &e) {
    EosR<R> o;
    o.kind = e.kind;
    o.gamma = (R)e.gamma;
    o.gm1 = (R)e.gm1;
    o.P0 = (R)e.P0;
    o.e0 = (R)e.e0;
    o.pmin = (R)e.pmin;
    return o;
}

template <typename R>
__device__ inline bool bad(const P5<R> &z, const EosR<R> &eos) {
    if (!isfinite(z.r) || !isfinite(z.p) || !isfinite(z.e)) return true;
    return z.r <= R(0) || z.p < eos.pmin;
}

template <typename R>
__device__ inline C4<R> phys_flux(const P5<R> &z) {
    R ru = z.r * z.u;
    C4<R> f;
    f.r = ru;
    f.mu = ru * z.u + z.p;
    f.mv = ru * z.v;
    f.E = (z.r * (z.e + R(0.5) * (z.u * z.u + z.v * z.v)) + z.p) * z.u;
    return f;
}

template <typename R>
__device__ inline C4<R> hllc(const P5<R> &L, const P5<R> &Rs, const EosR<R> &eos) {
    R cL = eos.sound(L.r, L.p), cR = eos.sound(Rs.r, Rs.p);
    R SL = smin_t(L.u - cL, Rs.u - cR);
    R SR = smax_t(L.u + cL, Rs.u + cR);
    if (SL >= R(0)) return phys_flux(L);
    if (SR <= R(0)) return phys_flux(Rs);
    R aL = L.r * (SL - L.u), aR = Rs.r * (SR - Rs.u);
    R SC = (L.p - Rs.p + aR * Rs.u - aL * L.u) / (aR - aL);
    R rsL = aL / (SL - SC), rsR = aR / (SR - SC);
    R EL = L.e + R(0.5) * (L.u * L.u + L.v * L.v);
    R ER = Rs.e + R(0.5) * (Rs.u * Rs.u + Rs.v * Rs.v);
    R EsL = EL + (SC - L.u) * (SC + L.p / aL);
    R EsR = ER + (SC - Rs.u) * (SC + Rs.p / aR);
    C4<R> FL = phys_flux(L), FR = phys_flux(Rs);
    R QL[4] = {L.r, L.r * L.u, L.r * L.v, L.r * EL};
    R QR[4] = {Rs.r, Rs.r * Rs.u, Rs.r * Rs.v, Rs.r * ER};
    R QsL[4] = {rsL, rsL * SC, rsL * L.v, rsL * EsL};
    R QsR[4] = {rsR, rsR * SC, rsR * Rs.v, rsR * EsR};
    R fl[4] = {FL.r, FL.mu, FL.mv, FL.E}, fr[4] = {FR.r, FR.mu, FR.mv, FR.E};
    R aSC = fabs(SC);
    R o[4];
#pragma unroll
    for (int k = 0; k < 4; ++k)
        o[k] = R(0.5) * (fl[k] + fr[k] + SL * (QsL[k] - QL[k]) + aSC * (QsL[k] - QsR[k]) + SR * (QsR[k] - QR[k]));
    return C4<R>{o[0], o[1], o[2], o[3]};
}

template <typename R>
__device__ inline C4<R> hll(const P5<R> &L, const P5<R> &Rs, const EosR<R> &eos) {
    R cL = eos.sound(L.r, L.p), cR = eos.sound(Rs.r, Rs.p);
    R SL = smin_t(L.u - cL, smin_t(Rs.u - cR, R(0)));
    R SR = smax_t(L.u + cL, smax_t(Rs.u + cR, R(0)));
    C4<R> FL = phys_flux(L), FR = phys_flux(Rs);
    R EL = L.e + R(0.5) * (L.u * L.u + L.v * L.v);
    R ER = Rs.e + R(0.5) * (Rs.u * Rs.u + Rs.v * Rs.v);
    R QL[4] = {L.r, L.r * L.u, L.r * L.v, L.r * EL};
    R QR[4] = {Rs.r, Rs.r * Rs.u, Rs.r * Rs.v, Rs.r * ER};
    R fl[4] = {FL.r, FL.mu, FL.mv, FL.E}, fr[4] = {FR.r, FR.mu, FR.mv, FR.E};
    R inv = R(1) / (SR - SL), SLR = SL * SR;
    R o[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) o[k] = (SR * fl[k] - SL * fr[k] + SLR * (QR[k] - QL[k])) * inv;
    return C4<R>{o[0], o[1], o[2], o[3]};
}

// rusanov.cpp:15-43 in precision R
template <typename R>
__device__ inline C4<R> rusanov(const P5<R> &L, const P5<R> &Rs, const EosR<R> &eos) {
    R cL = eos.sound(L.r, L.p), cR = eos.sound(Rs.r, Rs.p);
    R SL = L.u - cL, SR = L.u + cL;
    if (Rs.u - cR < SL) SL = Rs.u - cR;
    if (R(0) < SL) SL = R(0);
    if (SR < Rs.u + cR) SR = Rs.u + cR;
    if (SR < R(0)) SR = R(0);
    const R hS = R(0.5) * smax_t(fabs(SL), SR);
    R EL = L.e + R(0.5) * (L.u * L.u + L.v * L.v);
    R ER = Rs.e + R(0.5) * (Rs.u * Rs.u + Rs.v * Rs.v);
    C4<R> FL = phys_flux(L), FR = phys_flux(Rs);
    R QL[4] = {L.r, L.r * L.u, L.r * L.v, L.r * EL};
    R QR[4] = {Rs.r, Rs.r * Rs.u, Rs.r * Rs.v, Rs.r * ER};
    R fl[4] = {FL.r, FL.mu, FL.mv, FL.E}, fr[4] = {FR.r, FR.mu, FR.mv, FR.E};
    R o[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) o[k] = R(0.5) * (fl[k] + fr[k]) + hS * (QL[k] - QR[k]);
    return C4<R>{o[0], o[1], o[2], o[3]};
}

// The selected numerical flux in the face frame (HLL on isolated cells).
// Godunov's exact Riemann solver runs in FP64 whatever R is.  GEN = false:
// the kernel was launched for HLLC or HLL only, and carries neither the
// exact solver's call nor Rusanov.
template <typename R, bool GEN = true>
__device__ inline C4<R> face_flux(int kind, bool robust, const P5<R> &L, const P5<R> &Rs, const EosR<R> &eos,
                                  const EosD &eosd) {
    if (robust || kind == FLUX_HLL) return hll(L, Rs, eos);
    if (!GEN) return hllc(L, Rs, eos);
    if (kind == FLUX_GODUNOV) {
        const Prim a{(double)L.r, (double)L.u, (double)L.v, (double)L.p, (double)L.e};
        const Prim b{(double)Rs.r, (double)Rs.u, (double)Rs.v, (double)Rs.p, (double)Rs.e};
        const Cons f = godunov_ool(a, b, eosd);
        return C4<R>{(R)f.r, (R)f.mu, (R)f.mv, (R)f.E};
    }
    if (kind == FLUX_RUSANOV) return rusanov(L, Rs, eos);
    return hllc(L, Rs, eos);
}

template <typename R>
__device__ inline R lim2(int kind, R a, R b) {
    switch (kind) {
        case LIM_NONE: return R(0);
        case LIM_UNIT: return R(1);
        case LIM_MINMOD:
            if (a * b <= R(0)) return R(0);
            return smin_t(a / b, R(1));
        case LIM_MC: {
            R r = a / b;
            if (isnan(r)) return R(0);
            return smax_t(R(0), smin_t(R(2) * r, smin_t(R(0.5) * (R(1) + r), R(2))));
        }
        case LIM_VANLEER:
            if (a * b < R(0) || a == R(0)) return R(0);
            return R(2) * fabs(a) / (fabs(a) + fabs(b));
        case LIM_VANALBADA1:
            if (a * b <= R(0)) return R(0);
            if (b == R(0)) return R(1);
            return a * (a + b) / (a * a + b * b);
        case LIM_VANALBADA2: {
            if (a * b <= R(0)) return R(0);
            const R eps = R(10e-6);
            return (R(2) * a * b + eps) / (a * a + b * b + eps);
        }
        case LIM_CHARM: {
            if (a * b <= R(0)) return R(0);
            R s = a + b;
            return a * (R(3) * a + b) / (s * s);
        }
        case LIM_HCUS:
            if (a * b <= R(0)) return R(0);
            return (R(3) * a) / (a + R(2) * b);
        case LIM_HQUICK:
            if (a * b <= R(0)) return R(0);
            return (R(4) * a) / (a + R(3) * b);
        case LIM_KOREN: {
            R r = a / b;
            if (isnan(r)) return R(0);
            return smax_t(R(0), smin_t(R(2) * r, smin_t(R(2), (R(1) + R(2) * r) / R(3))));
        }
        case LIM_SMART: {
            R r = a / b;
            if (isnan(r)) return R(0);
            return smax_t(R(0), smin_t(R(2) * r, smin_t(R(0.25) + R(0.75) * r, R(4))));
        }
        case LIM_SUPERBEE: {
            R r = a / b;
            if (isnan(r)) return R(0);
            return smax_t(R(0), smin_t(smin_t(R(2) * r, R(1)), smin_t(r, R(2))));
        }
        default: return R(0);
    }
}

// ---------------------------------------------------------------------------
// Neighbour and boundary flag of slot s (0 L, 1 R, 2 B, 3 T) of cell (i, j);
// the normals are the axes, so the rotation into the face frame is an exact
// permutation.
__device__ inline int slot_nb(const StructMesh &m, int i, int j, int ic, int s, int &flag) {
    if (s == 0) {
        flag = i > 0 ? BC_INNER : m.bc[0];
        return i > 0 ? ic - m.ny : (m.xper ? ic + (m.nx - 1) * m.ny : ic);
    } else if (s == 1) {
        flag = i < m.nx - 1 ? BC_INNER : m.bc[1];
        return i < m.nx - 1 ? ic + m.ny : (m.xper ? ic - (m.nx - 1) * m.ny : ic);
    } else if (s == 2) {
        flag = j > 0 ? BC_INNER : m.bc[2];
        return j > 0 ? ic - 1 : (m.yper ? ic + (m.ny - 1) : ic);
    }
    flag = j < m.ny - 1 ? BC_INNER : m.bc[3];
    return j < m.ny - 1 ? ic + 1 : (m.yper ? ic - (m.ny - 1) : ic);
}

// Rotation of (u, v) into the frame of the axis normal of slot s and back.
template <typename R>
__device__ inline void to_local(int s, R &u, R &v) {
    R a = u, b = v;
    if (s == 0) { u = -a; v = -b; }
    else if (s == 1) { u = a; v = b; }
    else if (s == 2) { u = -b; v = a; }
    else { u = b; v = -a; }
}
template <typename R>
__device__ inline void to_global(int s, R &mu, R &mv) {
    R a = mu, b = mv;
    if (s == 0) { mu = -a; mv = -b; }
    else if (s == 1) { mu = a; mv = b; }
    else if (s == 2) { mu = b; mv = -a; }
    else { mu = -b; mv = a; }
}

// Wall reflection (sm_fluid.cpp:69-79) for an axis normal: the normal
// velocity changes sign.
template <typename R>
__device__ inline P5<R> wall_value(const P5<R> &z, int s, int flag) {
    if (flag != BC_WALL) return z;
    P5<R> o = z;
    if (s < 2) o.u = -z.u;
    else o.v = -z.v;
    return o;
}

// ---------------------------------------------------------------------------
// Storage of the step's fields.  FAST keeps the reference's primitive state
// (FP64); MIXED keeps FP64 conserved variables plus an FP32 primitive mirror.
// Per-axis geometry of the uniform mesh in precision R, filled on the host
// with the reference's least-squares formulas (gradient.h:251-258): for the
// low (L / B) and high (R / T) face of every column / row, the weight times
// the normal distance w * (dr . n), the normal distance dr . n itself, the
// inverse diagonal 1 / A of the least-squares matrix, and the offsets of the
// face centres from the cell centre (face_extra.h:140-147).
template <typename R>
struct AxisGeo {
    const R *wl, *wh;  // w * (dr . n), low / high face
    const R *rl, *rh;  // dr . n, low / high face
    const R *binv;     // 1 / A (A = sum of w (dr . n)^2 over the two faces)
    const R *ol, *oh;  // face centre - cell centre along the axis, low / high face
    const R *om;       // mid-edge - cell centre along the axis (faces of the other axis)
};

template <typename R>
struct Fields {
    AxisGeo<R> gxa, gya;  // geometry of columns (x) and rows (y)
    // state at t^n
    const double *q[4];   // MIXED: conserved FP64 (rho, rho u, rho v, rho E); FAST: unused
    const R *w[5];        // primitive (rho, u, v, p, e) in R
    // stage value (half step or Heun z*)
    R *h[5];
    // limited gradients of rho, u, v, p
    R *gx[4], *gy[4];
    // outputs of the corrector
    double *qn[4];  // MIXED
    R *wn[5];
    const int *wait_in;
    int *wait_out;
    unsigned long long *slot_cur, *slot_nxt, *slot_clr;
    double *dt_out;
};

template <typename R>
__device__ inline P5<R> ld5(R *const *p, int ic) {
    return P5<R>{p[0][ic], p[1][ic], p[2][ic], p[3][ic], p[4][ic]};
}
template <typename R>
__device__ inline P5<R> ld5(const R *const *p, int ic) {
    return P5<R>{p[0][ic], p[1][ic], p[2][ic], p[3][ic], p[4][ic]};
}
template <typename R>
__device__ inline void st5(R *const *p, int ic, const P5<R> &z) {
    p[0][ic] = z.r;
    p[1][ic] = z.u;
    p[2][ic] = z.v;
    p[3][ic] = z.p;
    p[4][ic] = z.e;
}

// Conservative vector of cell ic at t^n in FP64.
template <typename R, bool MIXED>
__device__ inline C4<double> q_of(const Fields<R> &f, int ic) {
    if (MIXED) return C4<double>{f.q[0][ic], f.q[1][ic], f.q[2][ic], f.q[3][ic]};
    double r = (double)f.w[0][ic], u = (double)f.w[1][ic], v = (double)f.w[2][ic], e = (double)f.w[4][ic];
    return C4<double>{r, r * u, r * v, r * (e + 0.5 * (u * u + v * v))};
}

// models.cpp:27-32 in FP64 (the pressure recovery stays FP64 in both flavours).
__device__ inline P5<double> prim_of(const C4<double> &q, const EosD &eos) {
    P5<double> z;
    z.r = q.r;
    double inv = 1.0 / q.r;
    z.u = q.mu * inv;
    z.v = q.mv * inv;
    z.e = q.E * inv - 0.5 * (z.u * z.u + z.v * z.v);
    z.p = eos.kind == EOS_IDEAL ? eos.gm1 * z.r * z.e : eos.gm1 * z.r * (z.e - eos.e0) - eos.gamma * eos.P0;
    return z;
}
__device__ inline bool bad64(const P5<double> &z, const EosD &eos) {
    if (!isfinite(z.r) || !isfinite(z.p) || !isfinite(z.e)) return true;
    return z.r <= 0.0 || z.p < eos.pmin;
}

template <typename R>
__device__ inline P5<R> down(const P5<double> &z) {
    return P5<R>{(R)z.r, (R)z.u, (R)z.v, (R)z.p, (R)z.e};
}

__device__ inline double step_dt(const SmfArgs &a, const unsigned long long *slot) {
    double dmin = __longlong_as_double((long long)*slot);
    return smin(a.CFL * dmin, a.max_dt);
}

// face centre - cell centre for slot s of cell (i, j)
template <typename R>
__device__ inline void face_offset(const Fields<R> &f, int i, int j, int s, R &dx, R &dy) {
    if (s == 0) { dx = f.gxa.ol[i]; dy = f.gya.om[j]; }
    else if (s == 1) { dx = f.gxa.oh[i]; dy = f.gya.om[j]; }
    else if (s == 2) { dx = f.gxa.om[i]; dy = f.gya.ol[j]; }
    else { dx = f.gxa.om[i]; dy = f.gya.oh[j]; }
}

// Slope limiter phi(a, b): LIM >= 0 fixes the limiter at compile time, -1
// selects it at run time.
template <int LIM, typename R>
__device__ inline R limit(int kind, R a, R b) {
    return lim2<R>(LIM >= 0 ? LIM : kind, a, b);
}

template <typename R>
__device__ inline P5<R> extrap(const P5<R> &z, const R gx[4], const R gy[4], R dx, R dy) {
    P5<R> o;
    o.r = z.r + (gx[0] * dx + gy[0] * dy);
    o.u = z.u + (gx[1] * dx + gy[1] * dy);
    o.v = z.v + (gx[2] * dx + gy[2] * dy);
    o.p = z.p + (gx[3] * dx + gy[3] * dy);
    o.e = R(0);
    return o;
}

// ---------------------------------------------------------------------------
// Tile of cell data in shared memory: rows i0 + a - H, columns j0 + b - H of
// the mesh (wrapped on periodic axes); `in` marks cells inside the domain.
template <typename R, int NF, int ROWS, int COLS>
struct CellTile {
    R f[NF][ROWS][COLS];
    unsigned char in[ROWS][COLS];
};

// x wrapped into [0, n) for x >= -n: a compare and an add in the common case
// instead of an integer division.
__device__ __forceinline__ int wrap_idx(int x, int n) {
    if (x < 0) x += n;
    if (x >= n) {
        x -= n;
        if (x >= n) x %= n;
    }
    return x;
}

// Global cell of tile entry (a, b) for a tile whose entry (H, H) is (i0, j0):
// returns false outside a non-periodic side.
__device__ inline bool tile_cell(const StructMesh &m, int i0, int j0, int a, int b, int H, int &gi, int &gj) {
    gi = i0 + a - H;
    gj = j0 + b - H;
    if (gi < 0 || gi >= m.nx) {
        if (!m.xper) return false;
        gi = wrap_idx(gi, m.nx);
    }
    if (gj < 0 || gj >= m.ny) {
        if (!m.yper) return false;
        gj = wrap_idx(gj, m.ny);
    }
    return true;
}

// ---------------------------------------------------------------------------
// Pass A: limited gradients of w (stored) and, for the predictor-corrector,
// the half step (sm_fluid.cpp:176-253) of every cell.  Block TX x TY cells
// (x = j, contiguous in memory), stencil staged with a one-cell halo.
template <typename R, bool MIXED, bool PREDICT, int LIM, int TX, int TY, int MINB = (sizeof(R) == 8 ? 4 : 6)>
__global__ void __launch_bounds__(TX *TY, MINB) k_grad_predict(SmfArgs a, Fields<R> f) {
    constexpr int ROWS = TY + 2, COLS = TX + 2;
    __shared__ CellTile<R, 5, ROWS, COLS> t;
    const StructMesh &m = a.mesh;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
    const int i0 = blockIdx.y * TY, j0 = blockIdx.x * TX;
    if (blockIdx.x == 0 && blockIdx.y == 0 && tid == 0) {
        *f.dt_out = step_dt(a, f.slot_cur);
        *f.slot_clr = 0x7FEFFFFFFFFFFFFFull;
    }
    for (int k = tid; k < ROWS * COLS; k += TX * TY) {
        int ra = k / COLS, cb = k - ra * COLS, gi, gj;
        bool in = tile_cell(m, i0, j0, ra, cb, 1, gi, gj);
        t.in[ra][cb] = in;
        if (in) {
            int g = gi * m.ny + gj;
#pragma unroll
            for (int q = 0; q < 5; ++q) t.f[q][ra][cb] = f.w[q][g];
        }
    }
    __syncthreads();
    const int i = i0 + ty, j = j0 + tx;
    if (i >= m.nx || j >= m.ny) return;
    const int ic = i * m.ny + j;
    auto cell = [&](int ra, int cb) {
        return P5<R>{t.f[0][ra][cb], t.f[1][ra][cb], t.f[2][ra][cb], t.f[3][ra][cb], t.f[4][ra][cb]};
    };
    const P5<R> zc = cell(ty + 1, tx + 1);

    // ---- limited least-squares gradient (gradient.h:226-282, 412-474) ----
    // Faces are axis-aligned, so dr . n lies on the face's axis and the
    // least-squares matrix is diagonal.
    const R gw[4] = {f.gxa.wl[i], f.gxa.wh[i], f.gya.wl[j], f.gya.wh[j]};
    const R gr[4] = {f.gxa.rl[i], f.gxa.rh[i], f.gya.rl[j], f.gya.rh[j]};
    const R B00 = f.gxa.binv[i], B11 = f.gya.binv[j];
    R dn[4][4];
    R Fx[4] = {R(0), R(0), R(0), R(0)}, Fy[4] = {R(0), R(0), R(0), R(0)};
    const R zcv[4] = {zc.r, zc.u, zc.v, zc.p};
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        int flag;
        slot_nb(m, i, j, ic, s, flag);
        const int ra = ty + 1 + (s == 0 ? -1 : (s == 1 ? 1 : 0));
        const int cb = tx + 1 + (s == 2 ? -1 : (s == 3 ? 1 : 0));
        P5<R> zn = is_boundary(flag) ? wall_value(zc, s, flag) : cell(ra, cb);
        const R znv[4] = {zn.r, zn.u, zn.v, zn.p};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            R dF = znv[k] - zcv[k];
            dn[s][k] = dF;
            if (s < 2) Fx[k] += gw[s] * dF;
            else Fy[k] += gw[s] * dF;
        }
    }
    R gx[4], gy[4];
    {
        R g0x[4], g0y[4], Lx[4] = {R(0), R(0), R(0), R(0)}, Ly[4] = {R(0), R(0), R(0), R(0)};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            g0x[k] = B00 * Fx[k];
            g0y[k] = B11 * Fy[k];
        }
#pragma unroll
        for (int s = 0; s < 4; ++s) {
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                R dFp = dn[s][k];
                R dun = (s < 2 ? g0x[k] : g0y[k]) * gr[s];
                R dFm = R(2) * dun - dFp;
                R dl = limit<LIM, R>(a.limiter, dFm, dFp) * dFp;
                if (s < 2) Lx[k] += gw[s] * dl;
                else Ly[k] += gw[s] * dl;
            }
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            gx[k] = B00 * Lx[k];
            gy[k] = B11 * Ly[k];
            f.gx[k][ic] = gx[k];
            f.gy[k][ic] = gy[k];
        }
    }
    if (!PREDICT) return;
    if (f.wait_in[ic] > 0) {
        st5(f.h, ic, zc);
        return;
    }
    // ---- predictor: half step with the physical flux of the face values ----
    const EosR<R> eos = eos_as<R>(a.eos);
    double F[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        R dx, dy;
        face_offset(f, i, j, s, dx, dy);
        P5<R> zm = extrap(zc, gx, gy, dx, dy);
        zm.e = eos.energy_rP(zm.r, zm.p);
        if (bad(zm, eos)) zm = zc;
        to_local(s, zm.u, zm.v);
        C4<R> lf = phys_flux(zm);
        to_global(s, lf.mu, lf.mv);
        const double area = s < 2 ? m.hy : m.hx;
        F[0] += (double)lf.r * area;
        F[1] += (double)lf.mu * area;
        F[2] += (double)lf.mv * area;
        F[3] += (double)lf.E * area;
    }
    const double coef = 0.5 * step_dt(a, f.slot_cur) / m.vol;
    C4<double> q = q_of<R, MIXED>(f, ic);
    q.r -= coef * F[0];
    q.mu -= coef * F[1];
    q.mv -= coef * F[2];
    q.E -= coef * F[3];
    P5<double> hz = prim_of(q, a.eos);
    st5(f.h, ic, bad64(hz, a.eos) ? zc : down<R>(hz));
}

// ---------------------------------------------------------------------------
// Pass B: face-once corrector on tiles.  Thread (tx, ty) of a TX x TY block
// owns cell (i0 - 1 + ty, j0 - 1 + tx) and computes its right (+x) and top
// (+y) face; cells with tx, ty >= 1 are the tile's interior and are updated
// from their four faces.  Face fluxes are stored as the flux across the face
// in the +x / +y direction (F_AB), so the cell on the far side adds -F_AB.
//
// MODE 0: first order (faces from the cell states, sm_fluid.cpp:127-174)
// MODE 1: corrector of the predictor-corrector scheme (sm_fluid.cpp:255-366)
// MODE 2: Heun stage A: z* = P(Q(z^n) - dt/V sum F(z^n))
// MODE 3: Heun stage B: P(0.5 (Q(z^n) + Q(z*) - dt/V sum F(z*)))
template <typename R, int TX, int TY>
struct FaceSmem {
    R h[5][TY + 1][TX + 1];   // face-state source (stage value or state)
    R g[8][TY + 1][TX + 1];   // gradients (x: 0-3, y: 4-7)
    int w[TY + 1][TX + 1];    // isolation counters
    unsigned char in[TY + 1][TX + 1];
    R fx[TY][TX][4];  // face fluxes as computed (in R; widened exactly for the FP64 sums)
    R fy[TY][TX][4];
    unsigned long long red[TX * TY / 32];
};

template <typename R, bool MIXED, int MODE, int TX, int TY, int MINB = 1, bool GEN = true>
__global__ void __launch_bounds__(TX *TY, MINB) k_faces(SmfArgs a, Fields<R> f) {
    __shared__ FaceSmem<R, TX, TY> sm;
    const StructMesh &m = a.mesh;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
    // interior cells of the block: rows i0 .. i0 + TY - 2, columns j0 .. j0 + TX - 2
    const int i0 = blockIdx.y * (TY - 1), j0 = blockIdx.x * (TX - 1);
    const EosR<R> eos = eos_as<R>(a.eos);
    // Face-state source: first order and Heun A read the state at t^n (w);
    // the corrector and Heun B read the stage value (h).
    R *const *src = (MODE == 1 || MODE == 3) ? f.h : const_cast<R *const *>(f.w);
    constexpr bool use_grad = MODE != 0;
    constexpr bool robust_on = MODE == 1;

    if (MODE == 0 && blockIdx.x == 0 && blockIdx.y == 0 && tid == 0) {
        *f.dt_out = step_dt(a, f.slot_cur);
        *f.slot_clr = 0x7FEFFFFFFFFFFFFFull;
    }

    // ---- stage the (TY + 1) x (TX + 1) cells: owners and their +1 neighbours ----
    for (int k = tid; k < (TY + 1) * (TX + 1); k += TX * TY) {
        int ra = k / (TX + 1), cb = k - ra * (TX + 1), gi, gj;
        bool in = tile_cell(m, i0, j0, ra, cb, 1, gi, gj);
        sm.in[ra][cb] = in;
        if (in) {
            int g = gi * m.ny + gj;
#pragma unroll
            for (int q = 0; q < 5; ++q) sm.h[q][ra][cb] = src[q][g];
            if (use_grad) {
#pragma unroll
                for (int q = 0; q < 4; ++q) {
                    sm.g[q][ra][cb] = f.gx[q][g];
                    sm.g[4 + q][ra][cb] = f.gy[q][g];
                }
            }
            if (robust_on) sm.w[ra][cb] = f.wait_in[g];
        }
    }
    __syncthreads();

    auto cell = [&](int ra, int cb) {
        return P5<R>{sm.h[0][ra][cb], sm.h[1][ra][cb], sm.h[2][ra][cb], sm.h[3][ra][cb], sm.h[4][ra][cb]};
    };
    auto recon = [&](int ra, int cb, int gi, int gj, int s, const P5<R> &z) {
        R gx[4], gy[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            gx[q] = sm.g[q][ra][cb];
            gy[q] = sm.g[4 + q][ra][cb];
        }
        R dx, dy;
        face_offset(f, gi, gj, s, dx, dy);
        P5<R> o = extrap(z, gx, gy, dx, dy);
        o.e = eos.energy_rP(o.r, o.p);
        return bad(o, eos) ? z : o;
    };

    // ---- the right (+x) and top (+y) face of the owner cell (ty, tx) ----
#pragma unroll
    for (int dir = 0; dir < 2; ++dir) {
        R out[4] = {R(0), R(0), R(0), R(0)};
        const bool needed = dir == 0 ? tx >= 1 : ty >= 1;
        const int raB = dir == 0 ? ty + 1 : ty, cbB = dir == 0 ? tx : tx + 1;
        const bool inA = sm.in[ty][tx], inB = sm.in[raB][cbB];
        if (needed && (inA || inB)) {
            // global (wrapped) coordinates of both sides
            int giA = i0 + ty - 1, gjA = j0 + tx - 1;
            int giB = giA + (dir == 0), gjB = gjA + (dir == 1);
            if (m.xper) {
                giA = wrap_idx(giA, m.nx);
                giB = wrap_idx(giB, m.nx);
            }
            if (m.yper) {
                gjA = wrap_idx(gjA, m.ny);
                gjB = wrap_idx(gjB, m.ny);
            }
            const int sA = dir == 0 ? 1 : 3, sB = dir == 0 ? 0 : 2;
            P5<R> zm, zp;
            bool robust;
            int s_own;
            R sgn = R(1);
            if (inA && inB) {
                s_own = sA;
                P5<R> zA = cell(ty, tx), zB = cell(raB, cbB);
                robust = robust_on && (sm.w[ty][tx] > 0 || sm.w[raB][cbB] > 0);
                if (robust || !use_grad) {
                    zm = zA;
                    zp = zB;
                } else {
                    zm = recon(ty, tx, giA, gjA, sA, zA);
                    zp = recon(raB, cbB, giB, gjB, sB, zB);
                }
            } else {
                // boundary face (WALL / ZOE) seen from its only cell
                const bool own_a = inA;
                const int ra = own_a ? ty : raB, cb = own_a ? tx : cbB;
                s_own = own_a ? sA : sB;
                sgn = own_a ? R(1) : R(-1);
                const int flag = m.bc[s_own];
                P5<R> zo = cell(ra, cb);
                robust = robust_on && sm.w[ra][cb] > 0;
                zm = (robust || !use_grad) ? zo : recon(ra, cb, own_a ? giA : giB, own_a ? gjA : gjB, s_own, zo);
                zp = wall_value(zm, s_own, flag);
            }
            to_local(s_own, zm.u, zm.v);
            to_local(s_own, zp.u, zp.v);
            C4<R> lf = face_flux<R, GEN>(a.flux, robust, zm, zp, eos, a.eos);
            to_global(s_own, lf.mu, lf.mv);
            out[0] = sgn * lf.r;
            out[1] = sgn * lf.mu;
            out[2] = sgn * lf.mv;
            out[3] = sgn * lf.E;
        }
        R(*dst)[TX][4] = dir == 0 ? sm.fx : sm.fy;
#pragma unroll
        for (int k = 0; k < 4; ++k) dst[ty][tx][k] = out[k];
    }
    __syncthreads();

    // ---- update of the interior cells ----------------------------------------
    unsigned long long best = 0x7FEFFFFFFFFFFFFFull;
    const int i = i0 + ty - 1, j = j0 + tx - 1;
    if (tx >= 1 && ty >= 1 && i < m.nx && j < m.ny) {
        const int ic = i * m.ny + j;
        const double dt = step_dt(a, f.slot_cur);
        const double hy = m.hy, hx = m.hx;
        double F[4];
#pragma unroll
        for (int k = 0; k < 4; ++k)
            F[k] = ((-(double)sm.fx[ty - 1][tx][k] * hy + (double)sm.fx[ty][tx][k] * hy) -
                    (double)sm.fy[ty][tx - 1][k] * hx) +
                   (double)sm.fy[ty][tx][k] * hx;
        const double coef = dt / m.vol;
        C4<double> q;
        if (MODE == 3) {
            P5<R> zs = cell(ty, tx);  // Q(z*) of the stage value
            double r = zs.r, u = zs.u, v = zs.v, e = zs.e;
            q = C4<double>{r, r * u, r * v, r * (e + 0.5 * (u * u + v * v))};
        } else {
            q = q_of<R, MIXED>(f, ic);
        }
        q.r -= coef * F[0];
        q.mu -= coef * F[1];
        q.mv -= coef * F[2];
        q.E -= coef * F[3];
        if (MODE == 3) {
            C4<double> q0 = q_of<R, MIXED>(f, ic);
            q.r = 0.5 * (q0.r + q.r);
            q.mu = 0.5 * (q0.mu + q.mu);
            q.mv = 0.5 * (q0.mv + q.mv);
            q.E = 0.5 * (q0.E + q.E);
        }
        P5<double> zn = prim_of(q, a.eos);
        if (MODE == 2) {
            st5(f.h, ic, down<R>(zn));  // Heun stage value
        } else {
            int wn = MODE == 1 ? sm.w[ty][tx] : 0;
            if (MODE == 1 && bad64(zn, a.eos)) {
                // isolation (sm_fluid.cpp:354-358): keep the old state
                zn = P5<double>{(double)f.w[0][ic], (double)f.w[1][ic], (double)f.w[2][ic], (double)f.w[3][ic],
                                (double)f.w[4][ic]};
                q = q_of<R, MIXED>(f, ic);
                wn = 3;
            } else if (wn > 0) {
                --wn;
            }
            if (MODE == 1) f.wait_out[ic] = wn;
            if (MIXED) {
                f.qn[0][ic] = q.r;
                f.qn[1][ic] = q.mu;
                f.qn[2][ic] = q.mv;
                f.qn[3][ic] = q.E;
            }
            st5(f.wn, ic, down<R>(zn));
            // CFL term of the new state for the next step (sm_fluid.cpp:104-111)
            double c = sqrt(a.eos.gamma * (zn.p + a.eos.P0) / zn.r);
            double dinc = sqrt(smin(m.inc2x[i], m.inc2y[j]));
            double lam = dinc / (sqrt(zn.u * zn.u + zn.v * zn.v) + c);
            if (lam >= 0.0) best = dbits(lam);
        }
    }
    if (MODE != 2) {
        const int lane = tid & 31, warp = tid >> 5;
        for (int o = 16; o > 0; o >>= 1) {
            unsigned long long t2 = __shfl_xor_sync(0xffffffffu, best, o);
            best = t2 < best ? t2 : best;
        }
        if (lane == 0) sm.red[warp] = best;
        __syncthreads();
        if (warp == 0) {
            best = lane < TX * TY / 32 ? sm.red[lane] : 0x7FEFFFFFFFFFFFFFull;
            for (int o = 16; o > 0; o >>= 1) {
                unsigned long long t2 = __shfl_xor_sync(0xffffffffu, best, o);
                best = t2 < best ? t2 : best;
            }
            if (lane == 0) atomicMin(f.slot_nxt, best);
        }
    }
}

// Stand-alone CFL minimum of state w into `slot` (first step after an upload).
template <typename R, int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_cfl(SmfArgs a, Fields<R> f) {
    const StructMesh &m = a.mesh;
    int ic = blockIdx.x * BLOCK + threadIdx.x;
    unsigned long long best = 0x7FEFFFFFFFFFFFFFull;
    if (ic < m.n) {
        int i = ic / m.ny, j = ic - i * m.ny;
        double rho, u, v, p;
        if (sizeof(R) == 4) {
            // MIXED: from the FP64 conserved state (the FP32 mirror only feeds
            // the face arithmetic)
            const P5<double> z = prim_of(C4<double>{f.q[0][ic], f.q[1][ic], f.q[2][ic], f.q[3][ic]}, a.eos);
            rho = z.r, u = z.u, v = z.v, p = z.p;
        } else {
            rho = f.w[0][ic], u = f.w[1][ic], v = f.w[2][ic], p = f.w[3][ic];
        }
        double c = sqrt(a.eos.gamma * (p + a.eos.P0) / rho);
        double dinc = sqrt(smin(m.inc2x[i], m.inc2y[j]));
        double lam = dinc / (sqrt(u * u + v * v) + c);
        if (lam >= 0.0) best = dbits(lam);
    }
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long t = __shfl_xor_sync(0xffffffffu, best, o);
        best = t < best ? t : best;
    }
    __shared__ unsigned long long red[BLOCK / 32];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = best;
    __syncthreads();
    if (threadIdx.x < 32) {
        best = threadIdx.x < BLOCK / 32 ? red[threadIdx.x] : 0x7FEFFFFFFFFFFFFFull;
        for (int o = 16; o > 0; o >>= 1) {
            unsigned long long t = __shfl_xor_sync(0xffffffffu, best, o);
            best = t < best ? t : best;
        }
        if (threadIdx.x == 0) atomicMin(f.slot_cur, best);
    }
}

// Conversions between the FP64 primitive state (the ABI's layout) and the
// MIXED layout (FP64 conserved + FP32 primitive mirror).
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_to_mixed(int n, PrimPtr z, Fields<float> f) {
    int ic = blockIdx.x * BLOCK + threadIdx.x;
    if (ic >= n) return;
    double r = z.r[ic], u = z.u[ic], v = z.v[ic], p = z.p[ic], e = z.e[ic];
    f.qn[0][ic] = r;
    f.qn[1][ic] = r * u;
    f.qn[2][ic] = r * v;
    f.qn[3][ic] = r * (e + 0.5 * (u * u + v * v));
    f.wn[0][ic] = (float)r;
    f.wn[1][ic] = (float)u;
    f.wn[2][ic] = (float)v;
    f.wn[3][ic] = (float)p;
    f.wn[4][ic] = (float)e;
}

template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_to_prim(int n, Fields<float> f, EosD eos, PrimPtr z) {
    int ic = blockIdx.x * BLOCK + threadIdx.x;
    if (ic >= n) return;
    P5<double> w = prim_of(C4<double>{f.q[0][ic], f.q[1][ic], f.q[2][ic], f.q[3][ic]}, eos);
    z.r[ic] = w.r;
    z.u[ic] = w.u;
    z.v[ic] = w.v;
    z.p[ic] = w.p;
    z.e[ic] = w.e;
}

}  // namespace tiled
}  // namespace zg
