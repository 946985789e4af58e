// mmf_parity.cu -- kernels of zephyr's multi-material first-order step
// MmFluid::update (math/solver/mm_fluid.cpp:112-171, DirSplit::NONE,
// accuracy 1) on a rectangle: CFL time step, PLIC interface reconstruction,
// and the face loop with mixture HLLC / composite Riemann fluxes and the
// PT-equilibrium closure of every updated cell.  One thread per cell; each
// cell evaluates its own faces in the reference's order (gather form).
// Compiled with -fmad=false: results agree bit for bit with the reference.
#include <cuda_runtime.h>

#include <algorithm>

#include "mmf_types.h"
#include "smf_struct.cuh"

namespace zg {
namespace mmf {

constexpr int BLOCK = 128;
constexpr int NM = NMAT;

__device__ __forceinline__ MSt<NM> load(const MmField &f, int ic) {
    MSt<NM> z;
    z.rho = f.rho[ic];
    z.vx = f.vx[ic];
    z.vy = f.vy[ic];
    z.P = f.P[ic];
    z.e = f.e[ic];
    z.T = f.T[ic];
#pragma unroll
    for (int i = 0; i < NM; ++i) {
        z.b.f[i] = f.b[i][ic];
        z.r[i] = f.r[i][ic];
    }
    return z;
}
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

// alpha of material i (models.cpp:234-237) for a runtime index
__device__ __forceinline__ double alpha_rt(const MSt<NM> &z, int idx) {
    double r = z.r[0], b = z.b.f[0];
#pragma unroll
    for (int i = 1; i < NM; ++i)
        if (i == idx) {
            r = z.r[i];
            b = z.b.f[i];
        }
    return isnan(r) ? 0.0 : fmax_std(0.0, fmin_std(b * z.rho / r, 1.0));
}

// ---------------------------------------------------------------------------
// CFL time step (mm_fluid.cpp:173-196): per cell min over faces of
// V / (S (|v.n| + c)), c the mixture sound speed; the last block to finish
// writes dt = min(CFL * min, max_dt) and resets the accumulator.
__global__ void __launch_bounds__(BLOCK) k_dt(MmArgs a) {
    int ic = blockIdx.x * BLOCK + threadIdx.x;
    if (ic == 0) {  // empty work lists for this step's face loop
        a.counts[0] = 0;
        a.counts[1] = 0;
    }
    unsigned long long best = 0x7FEFFFFFFFFFFFFFull;
    if (ic < a.mesh.n) {
        StructAcc c(a.mesh, ic);
        MSt<NM> z = load(a.z, ic);
        double cs = sound_speed_rP(a.mix, z.rho, z.P, z.b, z.T, z.r);
        double d = 1.7976931348623157e308;  // std::numeric_limits<double>::max()
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            FaceG g = c.face(s);
            double vn = z.vx * g.nx + z.vy * g.ny + 0.0 * 0.0;
            double lambda = fabs(vn) + cs;
            d = fmin_std(d, c.vol() / (g.area * lambda));
        }
        best = dbits(d);
    }
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long t = __shfl_xor_sync(0xffffffffu, best, o);
        best = t < best ? t : best;
    }
    __shared__ unsigned long long sm[BLOCK / 32];
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = best;
    __syncthreads();
    if (threadIdx.x < 32) {
        best = threadIdx.x < BLOCK / 32 ? sm[threadIdx.x] : 0x7FEFFFFFFFFFFFFFull;
        for (int o = 16; o > 0; o >>= 1) {
            unsigned long long t = __shfl_xor_sync(0xffffffffu, best, o);
            best = t < best ? t : best;
        }
        if (threadIdx.x == 0) {
            atomicMin(a.dmin_bits, best);
            __threadfence();
            unsigned int ticket = atomicAdd(a.dt_ticket, 1u);
            if (ticket == gridDim.x - 1) {
                unsigned long long bits = atomicMin(a.dmin_bits, 0x7FEFFFFFFFFFFFFFull);
                double dmin = __longlong_as_double((long long)bits);
                *a.dt_out = fmin_std(a.CFL * dmin, a.max_dt);
                *a.dmin_bits = 0x7FEFFFFFFFFFFFFFull;
                *a.dt_ticket = 0u;
                __threadfence();
            }
        }
    }
}

// ---------------------------------------------------------------------------
// PLIC reconstruction (interface_recovery, mm_fluid.cpp:484-519): for every
// material present in a mixed cell, the normal -sum face_fraction(a_c, a_n) S
// over the faces, normalised, and the plane offset quad_find_section.
__global__ void __launch_bounds__(BLOCK) k_recover(MmArgs a) {
    int ic = blockIdx.x * BLOCK + threadIdx.x;
    if (ic >= a.mesh.n) return;
    StructAcc c(a.mesh, ic);
    MSt<NM> z = load(a.z, ic);
    double nx[NM], ny[NM], ac[NM];
#pragma unroll
    for (int i = 0; i < NM; ++i) {
        nx[i] = 0.0;
        ny[i] = 0.0;
        ac[i] = z.b.f[i] > 0.0 ? z.b.f[i] * z.rho / z.r[i] : 0.0;  // volume_fractions()
    }
    bool pure = frac_index(z.b) >= 0;
    if (!pure) {
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            FaceG g = c.face(s);
            double Sx = g.area * g.nx, Sy = g.area * g.ny;
            MSt<NM> zn = load(a.z, g.nb);
#pragma unroll
            for (int i = 0; i < NM; ++i) {
                if (ac[i] > 0.0) {
                    double a_n = isnan(zn.r[i]) ? 0.0 : fmax_std(0.0, fmin_std(zn.b.f[i] * zn.rho / zn.r[i], 1.0));
                    double ff = face_fraction(ac[i], a_n);
                    nx[i] = nx[i] - ff * Sx;
                    ny[i] = ny[i] - ff * Sy;
                }
            }
        }
    }
    double hx = sqrt(a.mesh.inc2x[c.i]), hy = sqrt(a.mesh.inc2y[c.j]);  // AmrCells::hx / hy
#pragma unroll
    for (int i = 0; i < NM; ++i) {
        double off = 0.0;
        if (!pure && ac[i] > 0.0) {
            double sn = nx[i] * nx[i] + ny[i] * ny[i] + 0.0 * 0.0;
            if (sn > 0.0) {
                double r = sqrt(sn);
                nx[i] = nx[i] / r;
                ny[i] = ny[i] / r;
            }
            off = quad_find_section(ac[i], nx[i], ny[i], hx, hy);
        }
        a.nrm_x[i][ic] = pure ? 0.0 : nx[i];
        a.nrm_y[i][ic] = pure ? 0.0 : ny[i];
        a.off[i][ic] = off;
    }
}

// ---------------------------------------------------------------------------
// master_component (mm_fluid.cpp:201-226)
__device__ __forceinline__ int master_component(const MSt<NM> &zm, const MSt<NM> &zp) {
    double vi = 0.5 * (zm.vx + zp.vx);
    const MSt<NM> &w = vi > 0.0 ? zm : zp;
    int master = 0;
    double alpha_max = 0.0;
#pragma unroll
    for (int i = 0; i < NM; ++i) {
        if (w.b.f[i] > 0.0) {
            double al = isnan(w.r[i]) ? 0.0 : fmax_std(0.0, fmin_std(w.b.f[i] * w.rho / w.r[i], 1.0));
            if (al > alpha_max) {
                alpha_max = al;
                master = i;
            }
        }
    }
    return master;
}

__device__ __forceinline__ double normal_of(double *const arr[NM], int idx, int ic) {
    double v = arr[0][ic];
#pragma unroll
    for (int i = 1; i < NM; ++i)
        if (i == idx) v = arr[i][ic];
    return v;
}

// The face flux of calc_flux (mm_fluid.cpp:347-371) with alpha_sigma
// (229-261); states in the face frame.
__device__ QVd<NM> calc_flux(const MmArgs &a, double dt, int ic, const FaceG &g, const MSt<NM> &zm,
                             const MSt<NM> &zp, double hL, double hR, bool &bad) {
    if (a.crp == CRP_NONE) return hllc(a.mix, zm, zp, bad);
    int iL = frac_index(zm.b), iR = frac_index(zp.b);
    if (iL >= 0 && iR >= 0) return hllc(a.mix, zm, zp, bad);
    int iA = master_component(zm, zp);
    double a_L = alpha_rt(zm, iA), a_R = alpha_rt(zp, iA);
    double a_sig;
    if (a.crp == CRP_V3) {
        a_sig = face_fraction_v3(a_L, a_R);
    } else if (a.crp == CRP_V5) {
        a_sig = face_fraction_v5(a_L, a_R);
    } else if (a.crp == CRP_VS) {
        a_sig = face_fraction_s(a_L, a_R);
    } else {
        double vi = 0.5 * (zm.vx + zp.vx);
        bool upwind = vi > 0.0;
        double cfl = dt * fabs(vi) / (upwind ? hL : hR);
        int owner = upwind ? ic : g.nb;
        double nx = normal_of(a.nrm_x, iA, owner), ny = normal_of(a.nrm_y, iA, owner);
        if (!upwind) {
            nx = -nx;
            ny = -ny;
        }
        double cs = g.nx * nx + g.ny * ny + 0.0 * 0.0;
        a_sig = between(average_flux(upwind ? a_L : a_R, cs, cfl), a_L, a_R);
    }
    return crp_flux(a.mix, zm, zp, hL, hR, iA, a_sig, dt, bad);
}

// Rotate::to_local of a velocity (rotate.cpp:7-41); axis normals are unit
// vectors, so normalized() leaves them unchanged.
__device__ __forceinline__ void to_local(double cs, double sn, double vx, double vy, double &ox, double &oy) {
    ox = cs * vx + sn * vy + 0.0 * 0.0;
    oy = -sn * vx + cs * vy + 0.0 * 0.0;
}
// boundary_value (mm_fluid.cpp:88-97): the wall mirrors the normal velocity
__device__ __forceinline__ void wall_velocity(const FaceG &g, double vx, double vy, double &ox, double &oy) {
    double d = vx * g.nx + vy * g.ny + 0.0 * 0.0;
    ox = vx - 2.0 * (d * g.nx);
    oy = vy - 2.0 * (d * g.ny);
}

// One face of the first-order face loop (fluxes, mm_fluid.cpp:385-420):
// the flux through face s of cell ic, turned back to the global frame and
// multiplied by the face area.
__device__ void face_term(const MmArgs &a, int ic, int s, double dt, double *out, bool &bad) {
    StructAcc c(a.mesh, ic);
    const double V_c = c.vol();
    MSt<NM> zc = load(a.z, ic);
    FaceG g = c.face(s);
    MSt<NM> zn;
    if (!is_boundary(g.flag)) {
        zn = load(a.z, g.nb);
    } else {
        zn = zc;
        if (g.flag == BC_WALL) wall_velocity(g, zc.vx, zc.vy, zn.vx, zn.vy);
    }
    const double V_n = V_c;
    const double cs = g.nx, sn = g.ny;
    MSt<NM> zm = zc, zp = zn;
    to_local(cs, sn, zc.vx, zc.vy, zm.vx, zm.vy);
    to_local(cs, sn, zn.vx, zn.vy, zp.vx, zp.vy);
    const double S = g.area;
    QVd<NM> lf = calc_flux(a, dt, ic, g, zm, zp, V_c / S, V_n / S, bad);
    // Rotate::to_global of the momentum (rotate.cpp:43-77)
    double mx = cs * lf.a[1] + -sn * lf.a[2] + 0.0 * 0.0;
    double my = sn * lf.a[1] + cs * lf.a[2] + 0.0 * 0.0;
    lf.a[1] = mx;
    lf.a[2] = my;
#pragma unroll
    for (int k = 0; k < 4 + NM; ++k) out[k] = lf.a[k] * S;
}

// --- pure stencils ---------------------------------------------------------
// A cell whose own state and whose neighbours' states each hold one material
// only: every face takes calc_flux's plain-HLLC branch (mm_fluid.cpp:358-361)
// with the materials' own sound speeds (mixture_pt.cpp:101-106), and an
// update that stays pure takes get_rPT's one-material branch
// (mixture_pt.cpp:199-208).  The same arithmetic as the general path, in a
// kernel small enough to keep many warps resident; everything else is
// handed to the work lists.
struct PureSt {
    double rho, vx, vy, P, e;
    double b[NM];
    int idx;
};
__device__ __forceinline__ void pure_flux_of(const PureSt &z, const MixD<NM> &mx, double *F, double &c) {
    double E = z.e + 0.5 * (z.vx * z.vx + z.vy * z.vy + 0.0 * 0.0);
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
    c = m_sound_speed_rP(m, z.rho, z.P);
}
// hllc (hllc.cpp:344-421) for two one-material states
__device__ void hllc_pure(const MixD<NM> &mx, const PureSt &zL, const PureSt &zR, double *F, bool &bad) {
    double FL[4 + NM], FR[4 + NM], c_L, c_R;
    pure_flux_of(zL, mx, FL, c_L);
    pure_flux_of(zR, mx, FR, c_R);
    double S_L = fmin_std(zL.vx - c_L, zR.vx - c_L);
    double S_R = fmax_std(zL.vx + c_R, zR.vx + c_R);
    if (S_L >= S_R || zL.idx == zR.idx) {
        S_L = fmin_std(zL.vx - c_L, zR.vx - c_R);
        S_R = fmax_std(zL.vx + c_L, zR.vx + c_R);
    }
    if (S_L >= 0.0) {
#pragma unroll
        for (int k = 0; k < 4 + NM; ++k) F[k] = FL[k];
        return;
    }
    if (S_R <= 0.0) {
#pragma unroll
        for (int k = 0; k < 4 + NM; ++k) F[k] = FR[k];
        return;
    }
    double a_L = zL.rho * (S_L - zL.vx);
    double a_R = zR.rho * (S_R - zR.vx);
    double S_C = (zL.P - zR.P + a_R * zR.vx - a_L * zL.vx) / (a_R - a_L);
    if (S_C < S_L) S_C = S_L + 1.0e-9 * fmax_std(c_L, c_R);
    if (S_C > S_R) S_C = S_R - 1.0e-9 * fmax_std(c_L, c_R);
    double rho_sL = a_L / (S_L - S_C);
    double rho_sR = a_R / (S_R - S_C);
    double E_L = zL.e + 0.5 * (zL.vx * zL.vx + zL.vy * zL.vy + 0.0 * 0.0);
    double E_R = zR.e + 0.5 * (zR.vx * zR.vx + zR.vy * zR.vy + 0.0 * 0.0);
    double E_sL = E_L + (S_C - zL.vx) * (S_C + zL.P / a_L);
    double E_sR = E_R + (S_C - zR.vx) * (S_C + zR.P / a_R);
    double QsL[4 + NM], QsR[4 + NM], QL[4 + NM], QR[4 + NM];
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
    double aSC = fabs(S_C);
#pragma unroll
    for (int k = 0; k < 4 + NM; ++k) {
        F[k] = 0.5 * (FL[k] + FR[k] + S_L * (QsL[k] - QL[k]) + aSC * (QsL[k] - QsR[k]) + S_R * (QsR[k] - QR[k]));
        if (isnan(F[k])) bad = true;
    }
}
__device__ __forceinline__ int pure_index(const MmField &f, int ic) {
    Frac<NM> b;
#pragma unroll
    for (int i = 0; i < NM; ++i) b.f[i] = f.b[i][ic];
    return frac_index(b);
}
__device__ __forceinline__ PureSt load_pure(const MmField &f, int ic, int idx) {
    PureSt z;
    z.rho = f.rho[ic];
    z.vx = f.vx[ic];
    z.vy = f.vy[ic];
    z.P = f.P[ic];
    z.e = f.e[ic];
#pragma unroll
    for (int i = 0; i < NM; ++i) z.b[i] = f.b[i][ic];
    z.idx = idx;
    return z;
}

__global__ void __launch_bounds__(BLOCK, 6) k_flux_pure(MmArgs a) {
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
        int k = atomicAdd(&a.counts[0], 1);
        a.list_crp[k] = ic;
        return;
    }
    const double dt = *a.dt_out;
    const double V_c = c.vol();
    PureSt zc = load_pure(a.z, ic, idx_c);
    double flux[4 + NM];
#pragma unroll
    for (int k = 0; k < 4 + NM; ++k) flux[k] = 0.0;
    bool bad = false;
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        FaceG g = c.face(s);
        PureSt zn;
        if (!is_boundary(g.flag)) {
            zn = load_pure(a.z, g.nb, idx_n[s]);
        } else {
            zn = zc;
            if (g.flag == BC_WALL) wall_velocity(g, zc.vx, zc.vy, zn.vx, zn.vy);
        }
        const double cs = g.nx, sn = g.ny;
        PureSt zm = zc, zp = zn;
        to_local(cs, sn, zc.vx, zc.vy, zm.vx, zm.vy);
        to_local(cs, sn, zn.vx, zn.vy, zp.vx, zp.vy);
        double lf[4 + NM];
        hllc_pure(a.mix, zm, zp, lf, bad);
        double mx = cs * lf[1] + -sn * lf[2] + 0.0 * 0.0;
        double my = sn * lf[1] + cs * lf[2] + 0.0 * 0.0;
        lf[1] = mx;
        lf[2] = my;
        const double S = g.area;
#pragma unroll
        for (int k = 0; k < 4 + NM; ++k) flux[k] += lf[k] * S;
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

// --- work lists ------------------------------------------------------------
constexpr int LIST_BLOCKS = 148 * 4;

// Cells next to a mixed state: one thread per face (the faces of a cell are
// independent), then one per cell summing its four face terms in slot order
// as the reference's loop does, updating and closing the state.
__global__ void __launch_bounds__(BLOCK) k_crp_faces(MmArgs a) {
    const double dt = *a.dt_out;
    const int count = 4 * a.counts[0];
    for (int t = blockIdx.x * BLOCK + threadIdx.x; t < count; t += gridDim.x * BLOCK) {
        bool bad = false;
        double term[4 + NM];
        face_term(a, a.list_crp[t >> 2], t & 3, dt, term, bad);
#pragma unroll
        for (int k = 0; k < 4 + NM; ++k) a.fbuf[(size_t)t * (4 + NM) + k] = term[k];
        if (bad) atomicOr(a.err, 1);
    }
}
__global__ void __launch_bounds__(BLOCK) k_crp_update(MmArgs a) {
    const double dt = *a.dt_out;
    const int count = a.counts[0];
    for (int k = blockIdx.x * BLOCK + threadIdx.x; k < count; k += gridDim.x * BLOCK) {
        int ic = a.list_crp[k];
        MSt<NM> zc = load(a.z, ic);
        QVd<NM> flux = qv_zero<NM>();
#pragma unroll
        for (int s = 0; s < 4; ++s)
#pragma unroll
            for (int j = 0; j < 4 + NM; ++j) flux.a[j] += a.fbuf[(size_t)(4 * k + s) * (4 + NM) + j];
        QVd<NM> q = q_of(zc);
        double coef = dt / a.mesh.vol;
#pragma unroll
        for (int j = 0; j < 4 + NM; ++j) q.a[j] -= coef * flux.a[j];
        if (q.a[0] < 0.0) atomicOr(a.err, 1);  // the reference throws (mm_fluid.cpp:431-433)
        store(a.znext, ic, state_of_q(a.mix, q, zc.P, zc.T, zc.r));
    }
}

// get_rPT's Newton closure (mixture_pt.cpp:410-478) for updates that came out
// mixed, with the cell's previous P, T and true densities as the guesses.
__global__ void __launch_bounds__(BLOCK) k_closure(MmArgs a) {
    const int count = a.counts[1];
    for (int k = blockIdx.x * BLOCK + threadIdx.x; k < count; k += gridDim.x * BLOCK) {
        int ic = a.list_closure[k];
        QVd<NM> q;
#pragma unroll
        for (int j = 0; j < 4 + NM; ++j) q.a[j] = a.qbuf[(size_t)k * (4 + NM) + j];
        double r0[NM];
#pragma unroll
        for (int i = 0; i < NM; ++i) r0[i] = a.z.r[i][ic];
        store(a.znext, ic, state_of_q(a.mix, q, a.z.P[ic], a.z.T[ic], r0));
    }
}

// Refinement flags (MmFluid::set_flags, mm_fluid.cpp:836-885).
__global__ void __launch_bounds__(BLOCK) k_flags(MmArgs a, int *flags) {
    int ic = blockIdx.x * BLOCK + threadIdx.x;
    if (ic >= a.mesh.n) return;
    StructAcc c(a.mesh, ic);
    Frac<NM> b;
#pragma unroll
    for (int i = 0; i < NM; ++i) b.f[i] = a.z.b[i][ic];
    int idx = frac_index(b);
    if (idx < 0) {
        flags[ic] = 1;
        return;
    }
    bool need = false;
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        FaceG g = c.face(s);
        if (is_boundary(g.flag)) continue;
        Frac<NM> bn;
#pragma unroll
        for (int i = 0; i < NM; ++i) bn.f[i] = a.z.b[i][g.nb];
        if (frac_index(bn) != idx) need = true;
    }
    flags[ic] = need ? 1 : -1;
}

// Initial states from (density, velocity, pressure, mass fractions): the
// PState(density, velocity, pressure, Fractions, mixture) constructor
// (models.cpp:180-188); the fractions are normalised first, as the
// Fractions constructor does.  beta holds 4 fractions per cell.
__global__ void __launch_bounds__(BLOCK) k_make_states(MmArgs a, const double *rho, const double *vx,
                                                       const double *vy, const double *P, const double *beta) {
    int ic = blockIdx.x * BLOCK + threadIdx.x;
    if (ic >= a.mesh.n) return;
    Frac<NM> b;
#pragma unroll
    for (int i = 0; i < NM; ++i) b.f[i] = beta[4 * (size_t)ic + i];
    normalize(b);
    store(a.z, ic, state_of_rvp(a.mix, rho[ic], vx[ic], vy[ic], P[ic], b));
}

static inline unsigned blocks(const MmArgs &a) { return (unsigned)((a.mesh.n + BLOCK - 1) / BLOCK); }

void launch_dt(const MmArgs &a, void *stream) { k_dt<<<blocks(a), BLOCK, 0, (cudaStream_t)stream>>>(a); }
void launch_recover(const MmArgs &a, void *stream) { k_recover<<<blocks(a), BLOCK, 0, (cudaStream_t)stream>>>(a); }
void launch_flux_pure(const MmArgs &a, void *stream) {
    k_flux_pure<<<blocks(a), BLOCK, 0, (cudaStream_t)stream>>>(a);
}
void launch_flux_crp(const MmArgs &a, void *stream) {
    k_crp_faces<<<std::min<unsigned>(4 * blocks(a), LIST_BLOCKS), BLOCK, 0, (cudaStream_t)stream>>>(a);
    k_crp_update<<<std::min<unsigned>(blocks(a), LIST_BLOCKS), BLOCK, 0, (cudaStream_t)stream>>>(a);
}
void launch_closure(const MmArgs &a, void *stream) {
    k_closure<<<std::min<unsigned>(blocks(a), LIST_BLOCKS), BLOCK, 0, (cudaStream_t)stream>>>(a);
}
void launch_flags(const MmArgs &a, int *flags, void *stream) {
    k_flags<<<blocks(a), BLOCK, 0, (cudaStream_t)stream>>>(a, flags);
}
void launch_make_states(const MmArgs &a, const double *rho, const double *vx, const double *vy, const double *P,
                        const double *beta, void *stream) {
    k_make_states<<<blocks(a), BLOCK, 0, (cudaStream_t)stream>>>(a, rho, vx, vy, P, beta);
}

}  // namespace mmf
}  // namespace zg
