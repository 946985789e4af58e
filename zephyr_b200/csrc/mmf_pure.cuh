// mmf_pure.cuh -- the pure-stencil face loop of the multi-material step
// (a cell and its four neighbours each hold one material), templated on the
// precision of the face arithmetic: double in mmf_parity.cu (the reference's
// arithmetic, bit-exact), float in mmf_mixed.cu (the mixed form).
#pragma once

#include <cuda_runtime.h>

#include "mmf_types.h"
#include "smf_struct.cuh"

namespace zg {
namespace mmf {

constexpr int BLOCK = 128;
constexpr int NM = NMAT;

// a face the sub-step of direction `dir` leaves out (slots 0, 1 are the x
// faces, 2, 3 the y faces of a rectangle cell)
__device__ __forceinline__ bool skip_face(int dir, int s) { return (dir == 1 && s >= 2) || (dir == 2 && s < 2); }

__device__ __forceinline__ void store(const MmField &f, int ic, const MSt<NM> &z) {
    f.rho[ic] = z.rho;
    f.vx[ic] = z.vx;
    f.vy[ic] = z.vy;
    f.P[ic] = z.P;
    f.e[ic] = z.e;
    f.T[ic] = z.T;
#pragma unroll
    for (int i = 0; i < NM; ++i) {
        f.b[i][ic] = z.b.f[i];
        f.r[i][ic] = z.r[i];
    }
}

// boundary_value (mm_fluid.cpp:88-97): the wall mirrors the normal velocity
__device__ __forceinline__ void wall_velocity(const FaceG &g, double vx, double vy, double &ox, double &oy) {
    double d = vx * g.nx + vy * g.ny + 0.0 * 0.0;
    ox = vx - 2.0 * (d * g.nx);
    oy = vy - 2.0 * (d * g.ny);
}

// --- pure stencils ---------------------------------------------------------
// A cell whose own state and whose neighbours' states each hold one material
// only: every face takes calc_flux's plain-HLLC branch (mm_fluid.cpp:358-361)
// with the materials' own sound speeds (mixture_pt.cpp:101-106), and an
// update that stays pure takes get_rPT's one-material branch
// (mixture_pt.cpp:199-208).  The same arithmetic as the general path, in a
// kernel small enough to keep many warps resident; everything else is
// handed to the work lists.
template <typename R>
struct PureSt {
    R rho, vx, vy, P, e;
    R b[NM];
    int idx;
};
template <typename R>
__device__ __forceinline__ R rmin(R a, R b) { return b < a ? b : a; }  // std::min
template <typename R>
__device__ __forceinline__ R rmax(R a, R b) { return a < b ? b : a; }  // std::max
// the material's sound speed c(rho, P) in R
template <typename R>
__device__ __forceinline__ R sound_R(const MatD &m, R rho, R P) {
    if constexpr (sizeof(R) == 8) {
        return m_sound_speed_rP(m, rho, P);
    } else {
        if (!m.stiff) return sqrtf(R(m.gamma) * P / rho);
        return sqrtf(R(m.gamma) * (P + R(m.P0)) / rho);
    }
}
template <typename R>
__device__ __forceinline__ void pure_flux_of(const PureSt<R> &z, const MixD<NM> &mx, R *F, R &c) {
    R E = z.e + R(0.5) * (z.vx * z.vx + z.vy * z.vy + R(0) * R(0));
    F[0] = z.rho * z.vx;
    F[1] = z.rho * z.vx * z.vx + z.P;
    F[2] = z.rho * z.vx * z.vy;
    F[3] = (z.rho * E + z.P) * z.vx;
#pragma unroll
    for (int i = 0; i < NM; ++i) F[4 + i] = z.rho * z.vx * z.b[i];
    MatD m = mx.mat[0];
#pragma unroll
    for (int i = 1; i < NM; ++i)
        if (i == z.idx) m = mx.mat[i];
    c = sound_R<R>(m, z.rho, z.P);
}
// hllc (hllc.cpp:344-421) for two one-material states, in precision R
template <typename R>
__device__ void hllc_pure(const MixD<NM> &mx, const PureSt<R> &zL, const PureSt<R> &zR, R *F, bool &bad) {
    R FL[4 + NM], FR[4 + NM], c_L, c_R;
    pure_flux_of(zL, mx, FL, c_L);
    pure_flux_of(zR, mx, FR, c_R);
    R S_L = rmin<R>(zL.vx - c_L, zR.vx - c_L);
    R S_R = rmax<R>(zL.vx + c_R, zR.vx + c_R);
    if (S_L >= S_R || zL.idx == zR.idx) {
        S_L = rmin<R>(zL.vx - c_L, zR.vx - c_R);
        S_R = rmax<R>(zL.vx + c_L, zR.vx + c_R);
    }
    if (S_L >= R(0)) {
#pragma unroll
        for (int k = 0; k < 4 + NM; ++k) F[k] = FL[k];
        return;
    }
    if (S_R <= R(0)) {
#pragma unroll
        for (int k = 0; k < 4 + NM; ++k) F[k] = FR[k];
        return;
    }
    R a_L = zL.rho * (S_L - zL.vx);
    R a_R = zR.rho * (S_R - zR.vx);
    R S_C = (zL.P - zR.P + a_R * zR.vx - a_L * zL.vx) / (a_R - a_L);
    if (S_C < S_L) S_C = S_L + R(1.0e-9) * rmax<R>(c_L, c_R);
    if (S_C > S_R) S_C = S_R - R(1.0e-9) * rmax<R>(c_L, c_R);
    R rho_sL = a_L / (S_L - S_C);
    R rho_sR = a_R / (S_R - S_C);
    R E_L = zL.e + R(0.5) * (zL.vx * zL.vx + zL.vy * zL.vy + R(0) * R(0));
    R E_R = zR.e + R(0.5) * (zR.vx * zR.vx + zR.vy * zR.vy + R(0) * R(0));
    R E_sL = E_L + (S_C - zL.vx) * (S_C + zL.P / a_L);
    R E_sR = E_R + (S_C - zR.vx) * (S_C + zR.P / a_R);
    R QsL[4 + NM], QsR[4 + NM], QL[4 + NM], QR[4 + NM];
    QsL[0] = rho_sL;
    QsR[0] = rho_sR;
    QsL[1] = rho_sL * S_C;
    QsL[2] = rho_sL * zL.vy;
    QsR[1] = rho_sR * S_C;
    QsR[2] = rho_sR * zR.vy;
    QsL[3] = rho_sL * E_sL;
    QsR[3] = rho_sR * E_sR;
    QL[0] = zL.rho;
    QL[1] = zL.rho * zL.vx;
    QL[2] = zL.rho * zL.vy;
    QL[3] = zL.rho * E_L;
    QR[0] = zR.rho;
    QR[1] = zR.rho * zR.vx;
    QR[2] = zR.rho * zR.vy;
    QR[3] = zR.rho * E_R;
#pragma unroll
    for (int i = 0; i < NM; ++i) {
        QsL[4 + i] = rho_sL * zL.b[i];
        QsR[4 + i] = rho_sR * zR.b[i];
        QL[4 + i] = zL.rho * zL.b[i];
        QR[4 + i] = zR.rho * zR.b[i];
    }
    R aSC = fabs(S_C);
#pragma unroll
    for (int k = 0; k < 4 + NM; ++k) {
        F[k] = R(0.5) * (FL[k] + FR[k] + S_L * (QsL[k] - QL[k]) + aSC * (QsL[k] - QsR[k]) + S_R * (QsR[k] - QR[k]));
        if (isnan(F[k])) bad = true;
    }
}
__device__ __forceinline__ int pure_index(const MmField &f, int ic) {
    Frac<NM> b;
#pragma unroll
    for (int i = 0; i < NM; ++i) b.f[i] = f.b[i][ic];
    return frac_index(b);
}
template <typename R>
__device__ __forceinline__ PureSt<R> load_pure(const MmField &f, int ic, int idx) {
    PureSt<R> z;
    z.rho = (R)f.rho[ic];
    z.vx = (R)f.vx[ic];
    z.vy = (R)f.vy[ic];
    z.P = (R)f.P[ic];
    z.e = (R)f.e[ic];
#pragma unroll
    for (int i = 0; i < NM; ++i) z.b[i] = (R)f.b[i][ic];
    z.idx = idx;
    return z;
}

// The pure-stencil face loop.  R = double: the reference's arithmetic (the
// parity form).  R = float: the mixed form -- face states, wave speeds and
// HLLC fluxes in FP32, each face flux widened to FP64 for the accumulation,
// the update and the closure (EoS pressure recovery) in FP64.
template <typename R, int MINB = 6>
__global__ void __launch_bounds__(BLOCK, MINB) k_flux_pure(MmArgs a) {
    int ic = blockIdx.x * BLOCK + threadIdx.x;
    if (ic >= a.mesh.n) return;
    StructAcc c(a.mesh, ic);
    int idx_c = pure_index(a.z, ic);
    bool pure = idx_c >= 0;
    int idx_n[4];
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        FaceG g = c.face(s);
        idx_n[s] = is_boundary(g.flag) ? idx_c : pure_index(a.z, g.nb);
        pure = pure && idx_n[s] >= 0;
    }
    if (!pure) {  // a mixed state in the stencil: the general path
        if (!a.presorted) {
            int k = atomicAdd(&a.counts[0], 1);
            a.list_crp[k] = ic;
        }
        return;
    }
    const double dt = a.dt_scale * *a.dt_out;
    const double V_c = c.vol();
    const PureSt<double> zc = load_pure<double>(a.z, ic, idx_c);
    const PureSt<R> zcR = load_pure<R>(a.z, ic, idx_c);
    double flux[4 + NM];
#pragma unroll
    for (int k = 0; k < 4 + NM; ++k) flux[k] = 0.0;
    bool bad = false;
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        if (skip_face(a.dir, s)) continue;
        FaceG g = c.face(s);
        PureSt<R> zn;
        if (!is_boundary(g.flag)) {
            zn = load_pure<R>(a.z, g.nb, idx_n[s]);
        } else {
            zn = zcR;
            if (g.flag == BC_WALL) {
                double wx, wy;
                wall_velocity(g, zc.vx, zc.vy, wx, wy);
                zn.vx = (R)wx;
                zn.vy = (R)wy;
            }
        }
        const R cs = (R)g.nx, sn = (R)g.ny;
        PureSt<R> zm = zcR, zp = zn;
        zm.vx = cs * zcR.vx + sn * zcR.vy + R(0) * R(0);
        zm.vy = -sn * zcR.vx + cs * zcR.vy + R(0) * R(0);
        zp.vx = cs * zn.vx + sn * zn.vy + R(0) * R(0);
        zp.vy = -sn * zn.vx + cs * zn.vy + R(0) * R(0);
        R lf[4 + NM];
        hllc_pure<R>(a.mix, zm, zp, lf, bad);
        R mx = cs * lf[1] + -sn * lf[2] + R(0) * R(0);
        R my = sn * lf[1] + cs * lf[2] + R(0) * R(0);
        lf[1] = mx;
        lf[2] = my;
        const double S = g.area;
#pragma unroll
        for (int k = 0; k < 4 + NM; ++k) flux[k] += (double)lf[k] * S;
    }
    // QState(z_c) (models.cpp:421-428) and the update
    double E = zc.e + 0.5 * (zc.vx * zc.vx + zc.vy * zc.vy + 0.0 * 0.0);
    QVd<NM> q;
    q.a[0] = zc.rho;
    q.a[1] = zc.rho * zc.vx;
    q.a[2] = zc.rho * zc.vy;
    q.a[3] = zc.rho * E;
#pragma unroll
    for (int i = 0; i < NM; ++i) q.a[4 + i] = zc.rho * zc.b[i];
    double coef = dt / V_c;
#pragma unroll
    for (int k = 0; k < 4 + NM; ++k) q.a[k] -= coef * flux[k];
    if (q.a[0] < 0.0) bad = true;
    // PState(QState, ...) (models.cpp:190-204): the one-material closure here,
    // mixed results go to the closure list
    MSt<NM> z;
    z.rho = q.a[0];
    z.vx = q.a[1] / z.rho;
    z.vy = q.a[2] / z.rho;
    z.e = q.a[3] / z.rho - 0.5 * (z.vx * z.vx + z.vy * z.vy + 0.0 * 0.0);
#pragma unroll
    for (int i = 0; i < NM; ++i) z.b.f[i] = q.a[4 + i] / z.rho;
    cutoff(z.b, 1.0e-12);
    normalize(z.b);
    int idx = frac_index(z.b);
    if (idx >= 0) {
        MatD m = a.mix.mat[0];
#pragma unroll
        for (int i = 1; i < NM; ++i)
            if (i == idx) m = a.mix.mat[i];
#pragma unroll
        for (int i = 0; i < NM; ++i) z.r[i] = i == idx ? z.rho : MM_NAN;
        z.P = m_pressure_re(m, z.rho, z.e);
        z.T = m_temperature_rP(m, z.rho, z.P);
        store(a.znext, ic, z);
    } else {
        int k = atomicAdd(&a.counts[1], 1);
        a.list_closure[k] = ic;
#pragma unroll
        for (int j = 0; j < 4 + NM; ++j) a.qbuf[(size_t)k * (4 + NM) + j] = q.a[j];
    }
    if (bad) atomicOr(a.err, 1);
}

}  // namespace mmf
}  // namespace zg
