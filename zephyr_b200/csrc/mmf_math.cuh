// mmf_math.cuh -- device arithmetic of zephyr's multi-material step
// (MmFluid, math/solver/mm_fluid.cpp) for NM materials in pressure and
// temperature equilibrium:
//   * the material equations of state (phys/matter/eos/ideal_gas.cpp,
//     stiffened_gas.cpp) and the mixture closure MixturePT
//     (phys/matter/mixture_pt.cpp, its default "old" Newton solvers),
//   * mixture states mmf::PState / QState / Flux (math/cfd/models.cpp:168-541)
//     and mass-fraction vectors (phys/fractions.cpp),
//   * the mixture HLLC flux and wave configuration (math/cfd/flux/hllc.cpp),
//   * the composite Riemann problem (math/cfd/flux/crp_flux.cpp),
//   * the PLIC helpers (geom/sections.cpp, math/funcs.h).
// Every operation keeps the reference's order and association, and the file
// that includes this header is compiled with -fmad=false, so results agree
// bit for bit with the reference.  Where the reference loops over the four
// slots of a Fractions / ScalarSet, the slots past NM hold 0 (fractions) or
// NaN (true densities) and change no result, so the loops here stop at NM.
// std::min / std::max are restated with their argument-order semantics.
#pragma once

#include <cuda_runtime.h>

#include <cmath>
#include <limits>

#include "smf_math.cuh"

namespace zg {
namespace mmf {

__device__ __forceinline__ double fmin_std(double a, double b) { return b < a ? b : a; }  // std::min
__device__ __forceinline__ double fmax_std(double a, double b) { return a < b ? b : a; }  // std::max

constexpr double MM_INF = std::numeric_limits<double>::infinity();
constexpr double MM_NAN = std::numeric_limits<double>::quiet_NaN();
constexpr double FR_MIN = std::numeric_limits<double>::epsilon() / 4;  // Fractions::minimal
constexpr int MAX_COUNTER = 30;                              // mixture_pt.cpp:297
constexpr double EPS_V = 1.0e-12, EPS_E = 1.0e-12;           // mixture_pt.cpp:298-301

// A material: IdealGas (stiff = 0) or StiffenedGas (stiff = 1).
struct MatD {
    int stiff;
    double gamma, P0, e0, Cv, T0, rho_ref;
};
struct DPT {  // a value and its two partial derivatives
    double val, d1, d2;
};

__device__ __forceinline__ double m_pressure_re(const MatD &m, double rho, double e) {
    if (!m.stiff) return (m.gamma - 1.0) * rho * e;
    return (m.gamma - 1.0) * rho * (e - m.e0) - m.gamma * m.P0;
}
__device__ __forceinline__ double m_temperature_rP(const MatD &m, double rho, double P) {
    if (!m.stiff) return P / ((m.gamma - 1.0) * m.Cv * rho);
    return m.T0 + (P + m.P0) / ((m.gamma - 1.0) * m.Cv * rho);
}
__device__ __forceinline__ double m_energy_rP(const MatD &m, double rho, double P) {
    if (!m.stiff) return P / ((m.gamma - 1.0) * rho);
    return m.e0 + (P + m.gamma * m.P0) / ((m.gamma - 1.0) * rho);
}
__device__ __forceinline__ double m_energy_rT(const MatD &m, double rho, double T) {
    if (!m.stiff) return m.Cv * T;
    return m.e0 + m.Cv * (T - m.T0) + m.P0 / rho;
}
__device__ __forceinline__ double m_sound_speed_rP(const MatD &m, double rho, double P) {
    if (!m.stiff) return sqrt(m.gamma * P / rho);
    return sqrt(m.gamma * (P + m.P0) / rho);
}
__device__ __forceinline__ double m_sound_speed_re(const MatD &m, double rho, double e) {
    if (!m.stiff) return sqrt(m.gamma * (m.gamma - 1.0) * e);
    return sqrt(m.gamma * (m.gamma - 1.0) * ((e - m.e0) - m.P0 / rho));
}
// specific volume v(P, T) with dv/dP, dv/dT
__device__ __forceinline__ DPT m_volume_PT(const MatD &m, double P, double T) {
    DPT r;
    if (!m.stiff) {
        r.val = ((m.gamma - 1.0) * m.Cv * T) / P;
        r.d1 = -r.val / P;
        r.d2 = +r.val / T;
    } else {
        r.val = ((m.gamma - 1.0) * m.Cv * (T - m.T0)) / (P + m.P0);
        r.d1 = -r.val / (P + m.P0);
        r.d2 = +r.val / (T - m.T0);
    }
    return r;
}
// specific energy e(P, T) with de/dP, de/dT
__device__ __forceinline__ DPT m_energy_PT(const MatD &m, double P, double T) {
    DPT r;
    if (!m.stiff) {
        r.val = m.Cv * T;
        r.d1 = 0.0;
        r.d2 = m.Cv;
    } else {
        r.val = m.e0 + ((P + m.gamma * m.P0) / (P + m.P0)) * m.Cv * (T - m.T0);
        double s = P + m.P0;
        r.d1 = (1.0 - m.gamma) * m.P0 * m.Cv * (T - m.T0) / (s * s);
        r.d2 = ((P + m.gamma * m.P0) / (P + m.P0)) * m.Cv;
    }
    return r;
}
__device__ __forceinline__ double m_min_pressure(const MatD &m) { return m.stiff ? -m.P0 : 0.0; }

template <int NM>
struct MixD {
    MatD mat[NM];
};

// ---------------------------------------------------------------------------
// Fractions
template <int NM>
struct Frac {
    double f[NM];
};
template <int NM>
__device__ __forceinline__ int frac_index(const Frac<NM> &b) {
    int idx = -1;
#pragma unroll
    for (int i = 0; i < NM; ++i) {
        if (b.f[i] > 0.0) {
            if (idx < 0) idx = i;
            else return -1;
        }
    }
    return idx;
}
template <int NM>
__device__ __forceinline__ void cutoff(Frac<NM> &b, double eps) {
    double sum = 0.0;
#pragma unroll
    for (int i = 0; i < NM; ++i) {
        if (b.f[i] < eps) b.f[i] = 0.0;
        else if (b.f[i] > 1.0) b.f[i] = 1.0;
        sum += b.f[i];
    }
#pragma unroll
    for (int i = 0; i < NM; ++i) b.f[i] /= sum;
}
template <int NM>
__device__ __forceinline__ void normalize(Frac<NM> &b) {
    cutoff(b, FR_MIN);
}

// ---------------------------------------------------------------------------
// Mixture closure
template <int NM>
struct RhoSet {
    double r[NM];
};

template <int NM>
__device__ __forceinline__ double min_pressure(const MixD<NM> &mx, const Frac<NM> &b) {
    double P_min = -MM_INF;
#pragma unroll
    for (int i = 0; i < NM; ++i)
        if (b.f[i] > 0.0) P_min = fmax_std(P_min, m_min_pressure(mx.mat[i]));
    return P_min;
}
// init_densities: the given guesses (rhos0 != nullptr) or the materials'
// reference densities, for the materials present; NaN elsewhere.
template <int NM>
__device__ __forceinline__ RhoSet<NM> init_densities(const MixD<NM> &mx, const Frac<NM> &b, const double *rhos0) {
    RhoSet<NM> r;
#pragma unroll
    for (int i = 0; i < NM; ++i) r.r[i] = b.f[i] > 0.0 ? (rhos0 ? rhos0[i] : mx.mat[i].rho_ref) : MM_NAN;
    return r;
}

// T and true densities from (rho, P) (find_rT_rP_old); with `deriv`, dT/drho
// and dT/dP.
template <int NM>
__device__ double find_rT_rP(const MixD<NM> &mx, double rho, double P, const Frac<NM> &b, double T0,
                             const double *rhos0, RhoSet<NM> &rhos, bool deriv, double &dR, double &dP) {
    double v_mix = 1.0 / rho;
    double T = isnan(T0) ? 300.0 : T0;
    rhos = init_densities(mx, b, rhos0);
    DPT v{MM_NAN, MM_NAN, MM_NAN};
    for (int counter = 0; counter < MAX_COUNTER; ++counter) {
        double err = 0.0;
        v = {0.0, 0.0, 0.0};
#pragma unroll
        for (int i = 0; i < NM; ++i) {
            if (b.f[i] > 0.0) {
                DPT vi = m_volume_PT(mx.mat[i], P, T);
                v.val += b.f[i] * vi.val;
                v.d1 += b.f[i] * vi.d1;
                v.d2 += b.f[i] * vi.d2;
                err = fmax_std(err, fabs(1.0 - rhos.r[i] * vi.val));
                rhos.r[i] = 1.0 / vi.val;
            }
        }
        err = fmax_std(err, fabs(1.0 - rho * v.val));
        if (err < EPS_V) break;
        T += (v_mix - v.val) / v.d2;
    }
    if (deriv) {
        dR = -(v.val * v.val) / v.d2;
        dP = -v.d1 / v.d2;
    }
    return T;
}

template <int NM>
__device__ __forceinline__ DPT mix_energy_PT(const MixD<NM> &mx, double P, double T, const Frac<NM> &b) {
    DPT e{0.0, 0.0, 0.0};
#pragma unroll
    for (int i = 0; i < NM; ++i) {
        if (b.f[i] > 0.0) {
            DPT ei = m_energy_PT(mx.mat[i], P, T);
            e.val += b.f[i] * ei.val;
            e.d1 += b.f[i] * ei.d1;
            e.d2 += b.f[i] * ei.d2;
        }
    }
    return e;
}

// energy (value, d/drho, d/dP), T and true densities from (rho, P) (find_reT_rP_old)
template <int NM>
__device__ DPT find_reT_rP(const MixD<NM> &mx, double rho, double P, const Frac<NM> &b, double T0,
                           const double *rhos0, RhoSet<NM> &rhos, double &T, bool deriv) {
    double TdR = MM_NAN, TdP = MM_NAN;
    T = find_rT_rP(mx, rho, P, b, T0, rhos0, rhos, deriv, TdR, TdP);
    DPT e1 = mix_energy_PT(mx, P, T, b);
    DPT e2{e1.val, MM_NAN, MM_NAN};
    if (deriv) {
        e2.d1 = e1.d2 * TdR;
        e2.d2 = e1.d2 * TdP + e1.d1;
    }
    return e2;
}

// P (value, d/drho, d/de), T and true densities from (rho, e) (find_rPT_old):
// Newton on the 2x2 system v_mix = sum b_i v_i(P, T), e_mix = sum b_i e_i(P, T).
template <int NM>
__device__ DPT find_rPT(const MixD<NM> &mx, double rho, double e_mix, const Frac<NM> &b, double P0, double T0,
                        const double *rhos0, RhoSet<NM> &rhos, double &Tout, bool deriv) {
    double v_mix = 1.0 / rho;
    double P = isnan(P0) ? 1.0e5 : P0;
    double T = isnan(T0) ? 300.0 : T0;
    double P_min = min_pressure(mx, b);
    if (P < P_min) P = P_min + 1;
    rhos = init_densities(mx, b, rhos0);
    DPT v{MM_NAN, MM_NAN, MM_NAN}, e{MM_NAN, MM_NAN, MM_NAN};
    for (int counter = 0; counter < MAX_COUNTER; ++counter) {
        double err = 0.0;
        v = {0.0, 0.0, 0.0};
        e = {0.0, 0.0, 0.0};
#pragma unroll
        for (int i = 0; i < NM; ++i) {
            if (b.f[i] > 0.0) {
                DPT vi = m_volume_PT(mx.mat[i], P, T);
                v.val += b.f[i] * vi.val;
                v.d1 += b.f[i] * vi.d1;
                v.d2 += b.f[i] * vi.d2;
                err = fmax_std(err, fabs(1.0 - rhos.r[i] * vi.val));
                rhos.r[i] = 1.0 / vi.val;
                DPT ei = m_energy_PT(mx.mat[i], P, T);
                e.val += b.f[i] * ei.val;
                e.d1 += b.f[i] * ei.d1;
                e.d2 += b.f[i] * ei.d2;
            }
        }
        err = fmax_std(err, fabs(1.0 - rho * v.val));
        double err_e = fabs(1.0 - e.val / e_mix);
        if (err < EPS_V && err_e < EPS_E) break;
        double inv_D = 1.0 / (v.d2 * e.d1 - v.d1 * e.d2);
        double dP = inv_D * ((e_mix - e.val) * v.d2 - (v_mix - v.val) * e.d2);
        double dT = inv_D * ((v_mix - v.val) * e.d1 - (e_mix - e.val) * v.d1);
        double dP_lim = dP;
        if (P + dP < P_min) dP_lim = (1.0 - 0.1) * P_min + (0.1 - 1.0) * P;
        double dT_lim = dP != 0.0 ? (dP_lim / dP) * dT : dT;
        P += dP_lim;
        T += dT_lim;
    }
    DPT P1{P, MM_NAN, MM_NAN};
    if (deriv) {
        double inv_D = 1.0 / (v.d2 * e.d1 - v.d1 * e.d2);
        P1.d2 = inv_D * v.d2;
        P1.d1 = inv_D * e.d2 * (v.val * v.val);
    }
    Tout = T;
    return P1;
}

template <int NM>
__device__ __forceinline__ double sound_speed_rP(const MixD<NM> &mx, double rho, double P, const Frac<NM> &b,
                                                 double T0, const double *rhos0) {
    int idx = frac_index(b);
    if (idx >= 0) return m_sound_speed_rP(mx.mat[idx], rho, P);
    RhoSet<NM> rh;
    double T;
    DPT e = find_reT_rP(mx, rho, P, b, T0, rhos0, rh, T, true);
    double c2 = (P / (rho * rho) - e.d1) / e.d2;
    return sqrt(c2);
}
template <int NM>
__device__ __forceinline__ double sound_speed_re(const MixD<NM> &mx, double rho, double e, const Frac<NM> &b) {
    int idx = frac_index(b);
    if (idx >= 0) return m_sound_speed_re(mx.mat[idx], rho, e);
    RhoSet<NM> rh;
    double T;
    DPT P = find_rPT(mx, rho, e, b, MM_NAN, MM_NAN, (const double *)nullptr, rh, T, true);
    double c2 = P.d1 + P.val * P.d2 / (rho * rho);
    return sqrt(c2);
}

// ---------------------------------------------------------------------------
// Mixture states
template <int NM>
struct MSt {
    double rho, vx, vy, P, e, T;
    Frac<NM> b;
    double r[NM];  // true densities
};
template <int NM>
struct QVd {  // density, momentum x, momentum y, total energy, partial densities
    double a[4 + NM];
};
template <int NM>
__device__ __forceinline__ QVd<NM> qv_zero() {
    QVd<NM> q;
#pragma unroll
    for (int k = 0; k < 4 + NM; ++k) q.a[k] = 0.0;
    return q;
}
template <int NM>
__device__ __forceinline__ double E_of(const MSt<NM> &z) {
    return z.e + 0.5 * (z.vx * z.vx + z.vy * z.vy + 0.0 * 0.0);
}
template <int NM>
__device__ __forceinline__ double alpha(const MSt<NM> &z, int i) {
    return isnan(z.r[i]) ? 0.0 : fmax_std(0.0, fmin_std(z.b.f[i] * z.rho / z.r[i], 1.0));
}
template <int NM>
__device__ __forceinline__ QVd<NM> q_of(const MSt<NM> &z) {
    QVd<NM> q;
    q.a[0] = z.rho;
    q.a[1] = z.rho * z.vx;
    q.a[2] = z.rho * z.vy;
    q.a[3] = z.rho * E_of(z);
#pragma unroll
    for (int i = 0; i < NM; ++i) q.a[4 + i] = z.rho * z.b.f[i];
    return q;
}
template <int NM>
__device__ __forceinline__ QVd<NM> f_of(const MSt<NM> &z) {
    QVd<NM> f;
    f.a[0] = z.rho * z.vx;
    f.a[1] = z.rho * z.vx * z.vx + z.P;
    f.a[2] = z.rho * z.vx * z.vy;
    f.a[3] = (z.rho * E_of(z) + z.P) * z.vx;
#pragma unroll
    for (int i = 0; i < NM; ++i) f.a[4 + i] = z.rho * z.vx * z.b.f[i];
    return f;
}
// PState(QState, mixture, P0, T0, rhos): velocity, energy, fractions (cut off
// at 1e-12, normalised) and the closure (get_rPT).
template <int NM>
__device__ MSt<NM> state_of_q(const MixD<NM> &mx, const QVd<NM> &q, double P0, double T0, const double *rhos0) {
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
#pragma unroll
        for (int i = 0; i < NM; ++i) z.r[i] = i == idx ? z.rho : MM_NAN;
        z.P = m_pressure_re(mx.mat[idx], z.rho, z.e);
        z.T = m_temperature_rP(mx.mat[idx], z.rho, z.P);
    } else {
        RhoSet<NM> rh;
        z.P = find_rPT(mx, z.rho, z.e, z.b, P0, T0, rhos0, rh, z.T, false).val;
#pragma unroll
        for (int i = 0; i < NM; ++i) z.r[i] = rh.r[i];
    }
    return z;
}
// PState(density, velocity, pressure, mass fractions, mixture): get_reT
template <int NM>
__device__ MSt<NM> state_of_rvp(const MixD<NM> &mx, double rho, double vx, double vy, double P, const Frac<NM> &b) {
    MSt<NM> z;
    z.rho = rho;
    z.vx = vx;
    z.vy = vy;
    z.P = P;
    z.b = b;
    int idx = frac_index(b);
    if (idx >= 0) {
#pragma unroll
        for (int i = 0; i < NM; ++i) z.r[i] = i == idx ? rho : MM_NAN;
        z.e = m_energy_rP(mx.mat[idx], rho, P);
        z.T = m_temperature_rP(mx.mat[idx], rho, P);
    } else {
        RhoSet<NM> rh;
        z.e = find_reT_rP(mx, rho, P, b, MM_NAN, (const double *)nullptr, rh, z.T, false).val;
#pragma unroll
        for (int i = 0; i < NM; ++i) z.r[i] = rh.r[i];
    }
    return z;
}
template <int NM>
__device__ __forceinline__ void flux_inverse(QVd<NM> &f) {
    f.a[0] = -f.a[0];
    f.a[2] = -f.a[2];
    f.a[3] = -f.a[3];
#pragma unroll
    for (int i = 0; i < NM; ++i) f.a[4 + i] = -f.a[4 + i];
}

// Split a mixed state into pure material A and the rest (PState::split).
template <int NM>
__device__ void split(const MixD<NM> &mx, const MSt<NM> &z, int iA, MSt<NM> &zA, MSt<NM> &zB) {
    double rA = 0.0, bA = 0.0;
#pragma unroll
    for (int i = 0; i < NM; ++i)
        if (i == iA) {
            rA = z.r[i];
            bA = z.b.f[i];
        }
    MatD mA = mx.mat[0];
#pragma unroll
    for (int i = 1; i < NM; ++i)
        if (i == iA) mA = mx.mat[i];
    double energy_A = m_energy_rT(mA, rA, z.T);
    zA.rho = rA;
    zA.vx = z.vx;
    zA.vy = z.vy;
    zA.P = z.P;
    zA.e = energy_A;
    zA.T = z.T;
#pragma unroll
    for (int i = 0; i < NM; ++i) {
        zA.b.f[i] = i == iA ? 1.0 : 0.0;
        zA.r[i] = i == iA ? rA : MM_NAN;
    }
    zB.vx = z.vx;
    zB.vy = z.vy;
    zB.P = z.P;
    zB.T = z.T;
    double beta_B = 1.0 - bA;
    Frac<NM> al;
#pragma unroll
    for (int i = 0; i < NM; ++i) {
        bool h = z.b.f[i] > 0.0;
        zB.r[i] = h && i != iA ? z.r[i] : MM_NAN;
        zB.b.f[i] = h && i != iA ? z.b.f[i] / beta_B : 0.0;
        al.f[i] = h ? alpha(z, i) : 0.0;
    }
    normalize(zB.b);
    double alA = 0.0;
#pragma unroll
    for (int i = 0; i < NM; ++i)
        if (i == iA) alA = al.f[i];
    double alpha_B = 1.0 - alA;
#pragma unroll
    for (int i = 0; i < NM; ++i) {
        if (i == iA) al.f[i] = 0.0;
        else if (z.b.f[i] > 0.0) al.f[i] = al.f[i] / alpha_B;
    }
    normalize(al);
    zB.rho = 0.0;
#pragma unroll
    for (int i = 0; i < NM; ++i)
        if (z.b.f[i] > 0.0 && i != iA) zB.rho = zB.rho + z.r[i] * al.f[i];
    zB.e = 0.0;
#pragma unroll
    for (int i = 0; i < NM; ++i) {
        if (z.b.f[i] > 0.0 && i != iA) {
            zB.b.f[i] = al.f[i] * z.r[i] / zB.rho;
            zB.e += zB.b.f[i] * m_energy_rT(mx.mat[i], z.r[i], z.T);
        }
    }
}

// ---------------------------------------------------------------------------
// Mixture HLLC (hllc.cpp:344-421); `bad` is raised on a NaN flux.
template <int NM>
__device__ QVd<NM> hllc(const MixD<NM> &mx, const MSt<NM> &zL, const MSt<NM> &zR, bool &bad) {
    double c_L = sound_speed_rP(mx, zL.rho, zL.P, zL.b, zL.T, zL.r);
    double c_R = sound_speed_rP(mx, zR.rho, zR.P, zR.b, zR.T, zR.r);
    double S_L = fmin_std(zL.vx - c_L, zR.vx - c_L);
    double S_R = fmax_std(zL.vx + c_R, zR.vx + c_R);
    if (S_L >= S_R || frac_index(zL.b) == frac_index(zR.b)) {
        S_L = fmin_std(zL.vx - c_L, zR.vx - c_R);
        S_R = fmax_std(zL.vx + c_L, zR.vx + c_R);
    }
    if (S_L >= 0.0) return f_of(zL);
    if (S_R <= 0.0) return f_of(zR);
    double a_L = zL.rho * (S_L - zL.vx);
    double a_R = zR.rho * (S_R - zR.vx);
    double S_C = (zL.P - zR.P + a_R * zR.vx - a_L * zL.vx) / (a_R - a_L);
    if (S_C < S_L) S_C = S_L + 1.0e-9 * fmax_std(c_L, c_R);
    if (S_C > S_R) S_C = S_R - 1.0e-9 * fmax_std(c_L, c_R);
    double rho_sL = a_L / (S_L - S_C);
    double rho_sR = a_R / (S_R - S_C);
    double E_sL = E_of(zL) + (S_C - zL.vx) * (S_C + zL.P / a_L);
    double E_sR = E_of(zR) + (S_C - zR.vx) * (S_C + zR.P / a_R);
    QVd<NM> QsL, QsR;
    QsL.a[0] = rho_sL;
    QsR.a[0] = rho_sR;
    QsL.a[1] = rho_sL * S_C;
    QsL.a[2] = rho_sL * zL.vy;
    QsR.a[1] = rho_sR * S_C;
    QsR.a[2] = rho_sR * zR.vy;
    QsL.a[3] = rho_sL * E_sL;
    QsR.a[3] = rho_sR * E_sR;
#pragma unroll
    for (int i = 0; i < NM; ++i) {
        QsL.a[4 + i] = rho_sL * zL.b.f[i];
        QsR.a[4 + i] = rho_sR * zR.b.f[i];
    }
    QVd<NM> QL = q_of(zL), QR = q_of(zR), FL = f_of(zL), FR = f_of(zR), F;
    double aSC = fabs(S_C);
#pragma unroll
    for (int k = 0; k < 4 + NM; ++k) {
        F.a[k] = 0.5 * (FL.a[k] + FR.a[k] + S_L * (QsL.a[k] - QL.a[k]) + aSC * (QsL.a[k] - QsR.a[k]) +
                        S_R * (QsR.a[k] - QR.a[k]));
        if (isnan(F.a[k])) bad = true;
    }
    return F;
}

// HLLC wave configuration from conservative states and fluxes (hllc.cpp:262-338)
template <int NM>
struct Wave {
    double S_L, S_C, S_R;
    QVd<NM> QsL, FsL, QsR, FsR;
};
template <int NM>
__device__ void wave_config(const MixD<NM> &mx, const QVd<NM> &QL, const QVd<NM> &FL, const QVd<NM> &QR,
                            const QVd<NM> &FR, Wave<NM> &w) {
    double vLx = QL.a[1] / QL.a[0], vLy = QL.a[2] / QL.a[0];
    double vRx = QR.a[1] / QR.a[0], vRy = QR.a[2] / QR.a[0];
    double vLz = 0.0 / QL.a[0], vRz = 0.0 / QR.a[0];
    double e_L = QL.a[3] / QL.a[0] - 0.5 * (vLx * vLx + vLy * vLy + vLz * vLz);
    double e_R = QR.a[3] / QR.a[0] - 0.5 * (vRx * vRx + vRy * vRy + vRz * vRz);
    Frac<NM> bL, bR;
#pragma unroll
    for (int i = 0; i < NM; ++i) {
        bL.f[i] = QL.a[4 + i] / QL.a[0];
        bR.f[i] = QR.a[4 + i] / QR.a[0];
    }
    double c_L = sound_speed_re(mx, QL.a[0], e_L, bL);
    double c_R = sound_speed_re(mx, QR.a[0], e_R, bR);
    double S_L = fmin_std(vLx - c_L, vRx - c_L);
    double S_R = fmax_std(vLx + c_R, vRx + c_R);
    if (S_L >= S_R || frac_index(bL) == frac_index(bR)) {
        S_L = fmin_std(vLx - c_L, vRx - c_R);
        S_R = fmax_std(vLx + c_L, vRx + c_R);
    }
    QVd<NM> aL, aR;
#pragma unroll
    for (int k = 0; k < 4 + NM; ++k) {
        aL.a[k] = FL.a[k] - S_L * QL.a[k];
        aR.a[k] = FR.a[k] - S_R * QR.a[k];
    }
    double S_C = (aR.a[1] - aL.a[1]) / (aR.a[0] - aL.a[0]);
    if (S_C < S_L) S_C = S_L + 1.0e-9 * fmax_std(c_L, c_R);
    if (S_C > S_R) S_C = S_R - 1.0e-9 * fmax_std(c_L, c_R);
    double rho_sL = aL.a[0] / (S_C - S_L);
    double rho_sR = aR.a[0] / (S_C - S_R);
    double E_sL = S_C * S_C + (aL.a[3] - S_C * aL.a[1]) / aL.a[0];
    double E_sR = S_C * S_C + (aR.a[3] - S_C * aR.a[1]) / aR.a[0];
    w.S_L = S_L;
    w.S_C = S_C;
    w.S_R = S_R;
    w.QsL.a[0] = rho_sL;
    w.QsR.a[0] = rho_sR;
    w.QsL.a[1] = rho_sL * S_C;
    w.QsL.a[2] = rho_sL * vLy;
    w.QsR.a[1] = rho_sR * S_C;
    w.QsR.a[2] = rho_sR * vRy;
    w.QsL.a[3] = rho_sL * E_sL;
    w.QsR.a[3] = rho_sR * E_sR;
#pragma unroll
    for (int i = 0; i < NM; ++i) {
        w.QsL.a[4 + i] = rho_sL * bL.f[i];
        w.QsR.a[4 + i] = rho_sR * bR.f[i];
    }
#pragma unroll
    for (int k = 0; k < 4 + NM; ++k) {
        w.FsL.a[k] = aL.a[k] + S_L * w.QsL.a[k];
        w.FsR.a[k] = aR.a[k] + S_R * w.QsR.a[k];
    }
}

// ---------------------------------------------------------------------------
// Composite Riemann problem (crp_flux.cpp)
struct Pt {
    double x, t;
};
struct Chr {
    double x, t, S;
    __device__ double edge_t() const {
        double ts = (S * t - x) / S;
        return ts < t ? MM_INF : ts;
    }
    __device__ Pt cross(const Chr &c) const {
        if (S == c.S) return {0.5 * (x + c.x), MM_INF};
        Pt p;
        p.t = (c.x - x + S * t - c.S * c.t) / (S - c.S);
        if (p.t <= fmax_std(t, c.t)) return {0.5 * (x + c.x), MM_INF};
        p.x = 0.5 * (x + c.x + S * (p.t - t) + c.S * (p.t - c.t));
        return p;
    }
};
// (F (a.t - b.t) - Q (a.x - b.x)) accumulated into r (r += ...)
template <int NM>
__device__ __forceinline__ void g_edge(const QVd<NM> &F, const QVd<NM> &Q, Pt a, Pt b, QVd<NM> &g) {
    double dt_ = a.t - b.t, dx_ = a.x - b.x;
#pragma unroll
    for (int k = 0; k < 4 + NM; ++k) g.a[k] = F.a[k] * dt_ - Q.a[k] * dx_;
}

// CrpFlux::classic (the active branch, crp_flux.cpp:232-457)
template <int NM>
__device__ __noinline__ QVd<NM> crp_classic(const MixD<NM> &mx, const MSt<NM> &zLA, const MSt<NM> &zLB,
                                            const MSt<NM> &zRB, double delta, double dt, bool &bad) {
    QVd<NM> qLB = q_of(zLB), fLB = f_of(zLB);
    Wave<NM> w0;
    {
        QVd<NM> Q_R = q_of(zRB), F_R = f_of(zRB);
        wave_config(mx, qLB, fLB, Q_R, F_R, w0);
    }
    Chr C_0{-delta, 0.0, zLA.vx};
    Chr C_0L{0.0, 0.0, w0.S_L};
    Pt O1 = C_0.cross(C_0L);
    const Pt O0{0.0, 0.0}, Odt{0.0, dt};
    QVd<NM> r, g1, g2;
    if (O1.x >= 0.0) {
        double t2u = C_0.edge_t();
        if (dt <= t2u) return fLB;
        QVd<NM> qLA = q_of(zLA), fLA = f_of(zLA);
        Wave<NM> w1;
        wave_config(mx, qLA, fLA, w0.QsL, w0.FsL, w1);
        double lb = -O1.x / (dt - O1.t);
        const QVd<NM> *F = &fLA, *Q = &qLA;
        if (dt > O1.t) {
            if (lb < w1.S_L) {
                F = &fLA;
                Q = &qLA;
            } else if (lb < w1.S_C) {
                F = &w1.FsL;
                Q = &w1.QsL;
            } else if (lb < w1.S_R) {
                F = &w1.FsR;
                Q = &w1.QsR;
            } else {
                F = &w0.FsL;
                Q = &w0.QsL;
            }
        }
        g_edge(*F, *Q, O1, Odt, g1);
        g_edge(fLB, qLB, O0, O1, g2);
#pragma unroll
        for (int k = 0; k < 4 + NM; ++k) r.a[k] = (g1.a[k] + g2.a[k]) / (0.0 - dt);
        return r;
    }
    if (w0.S_C >= 0.0) {
        if (dt <= O1.t && O1.x < 0.0) return w0.FsL;
        QVd<NM> Q_L = q_of(zLA), F_L = f_of(zLA);
        Wave<NM> w1;
        wave_config(mx, Q_L, F_L, w0.QsL, w0.FsL, w1);
        Chr C_1R{O1.x, O1.t, w1.S_R};
        double t1 = C_1R.edge_t();
        if (dt <= t1 && O1.x < 0.0) return w0.FsL;
        double lb = -O1.x / (dt - O1.t);
        const QVd<NM> *F = lb < w1.S_L ? &F_L : (lb < w1.S_C ? &w1.FsL : &w1.FsR);
        const QVd<NM> *Q = lb < w1.S_L ? &Q_L : (lb < w1.S_C ? &w1.QsL : &w1.QsR);
        g_edge(*F, *Q, O1, Odt, g1);
        g_edge(w0.FsL, w0.QsL, O0, O1, g2);
#pragma unroll
        for (int k = 0; k < 4 + NM; ++k) r.a[k] = (g1.a[k] + g2.a[k]) / (0.0 - dt);
        return r;
    }
    if (O1.t >= dt) return w0.FsR;
    Wave<NM> w1;
    {
        QVd<NM> Q_L = q_of(zLA), F_L = f_of(zLA);
        wave_config(mx, Q_L, F_L, w0.QsL, w0.FsL, w1);
    }
    Chr C_0C{0.0, 0.0, w0.S_C};
    Chr C_1R{O1.x, O1.t, w1.S_R};
    Pt O2 = C_1R.cross(C_0C);
    if (O2.t > dt || O2.x > 0.0) return w0.FsR;
    Wave<NM> w2;
    wave_config(mx, w1.QsR, w1.FsR, w0.QsR, w0.FsR, w2);
    Chr C_2L{O2.x, O2.t, w2.S_L};
    Chr C_1C{O1.x, O1.t, w1.S_C};
    Pt O3 = C_1C.cross(C_2L);
    if (O3.x >= 0.0) {  // the reference throws here (crp_flux.cpp:394-396)
        bad = true;
        return w0.FsR;
    }
    Chr C_2R{O2.x, O2.t, w2.S_R};
    double t1 = C_2R.edge_t();
    Wave<NM> w3;
    wave_config(mx, w1.QsL, w1.FsL, w2.QsL, w2.FsL, w3);
    Chr C_3R{O3.x, O3.t, w3.S_R};
    double t4 = C_3R.edge_t();
    if (dt <= t4) {
        if (dt <= t1) return w0.FsR;
        double lb = -O2.x / (dt - O2.t);
        const QVd<NM> *F = lb < w2.S_C ? &w2.FsL : (lb < w2.S_R ? &w2.FsR : &w0.FsR);
        const QVd<NM> *Q = lb < w2.S_C ? &w2.QsL : (lb < w2.S_R ? &w2.QsR : &w0.QsR);
        g_edge(*F, *Q, O2, Odt, g1);
        g_edge(w0.FsR, w0.QsR, O0, O2, g2);
#pragma unroll
        for (int k = 0; k < 4 + NM; ++k) r.a[k] = (g1.a[k] + g2.a[k]) / (0.0 - dt);
        return r;
    }
    double lb = -O3.x / (dt - O3.t);
    const QVd<NM> *F = lb < w3.S_L ? &w1.FsL : (lb < w3.S_C ? &w3.FsL : &w3.FsR);
    const QVd<NM> *Q = lb < w3.S_L ? &w1.QsL : (lb < w3.S_C ? &w3.QsL : &w3.QsR);
    QVd<NM> g3;
    g_edge(*F, *Q, O3, Odt, g1);
    g_edge(w2.FsL, w2.QsL, O2, O3, g2);
    g_edge(w0.FsR, w0.QsR, O0, O2, g3);
#pragma unroll
    for (int k = 0; k < 4 + NM; ++k) r.a[k] = (g1.a[k] + g2.a[k] + g3.a[k]) / (0.0 - dt);
    return r;
}

// CrpFlux::inverse (crp_flux.cpp:460-480)
template <int NM>
__device__ __forceinline__ QVd<NM> crp_inverse(const MixD<NM> &mx, MSt<NM> zLA, MSt<NM> zRA, MSt<NM> zRB,
                                               double delta, double dt, bool &bad) {
    zLA.vx = -zLA.vx;
    zRA.vx = -zRA.vx;
    zRB.vx = -zRB.vx;
    QVd<NM> f = crp_classic(mx, zRB, zRA, zLA, delta, dt, bad);
    flux_inverse(f);
    return f;
}

template <int NM>
__device__ __forceinline__ QVd<NM> blend(double a_sig, const QVd<NM> &A, const QVd<NM> &B) {
    QVd<NM> r;
#pragma unroll
    for (int k = 0; k < 4 + NM; ++k) r.a[k] = a_sig * A.a[k] + (1.0 - a_sig) * B.a[k];
    return r;
}

// calc_crp_flux's plain-HLLC case: neither state holds a fraction of
// material iA strictly between 0 and 1 (mm_fluid.cpp:270-272)
template <int NM>
__device__ __forceinline__ bool crp_plain(const MSt<NM> &zL, const MSt<NM> &zR, int iA) {
    double aL = alpha(zL, iA), aR = alpha(zR, iA);
    return (aL == 0.0 || aL == 1.0) && (aR == 0.0 || aR == 1.0);
}

// MmFluid::calc_crp_flux (mm_fluid.cpp:266-345)
template <int NM>
__device__ __noinline__ QVd<NM> crp_flux(const MixD<NM> &mx, const MSt<NM> &zL, const MSt<NM> &zR, double hL,
                                         double hR, int iA, double a_sig, double dt, bool &bad) {
    double aL = alpha(zL, iA), aR = alpha(zR, iA);
    if ((aL == 0.0 || aL == 1.0) && (aR == 0.0 || aR == 1.0)) return hllc(mx, zL, zR, bad);
    double delta_L = (aL < a_sig ? aL / a_sig : (1.0 - aL) / (1.0 - a_sig)) * hL;
    double delta_R = (aR < a_sig ? aR / a_sig : (1.0 - aR) / (1.0 - a_sig)) * hR;
    MSt<NM> zA, zB;
    if (aL == 0.0 || aL == 1.0) {
        split(mx, zR, iA, zA, zB);  // zA = zRA, zB = zRB
        QVd<NM> fA, fB;
        if (aL == 0.0) {
            fA = hllc(mx, zL, zA, bad);
            fB = crp_inverse(mx, zL, zB, zA, delta_R, dt, bad);
        } else {
            fA = crp_inverse(mx, zL, zA, zB, delta_R, dt, bad);
            fB = hllc(mx, zL, zB, bad);
        }
        return blend(a_sig, fA, fB);
    }
    if (aR == 0.0 || aR == 1.0) {
        split(mx, zL, iA, zA, zB);  // zA = zLA, zB = zLB
        QVd<NM> fA, fB;
        if (aR == 0.0) {
            fA = hllc(mx, zA, zR, bad);
            fB = crp_classic(mx, zA, zB, zR, delta_L, dt, bad);
        } else {
            fA = crp_classic(mx, zB, zA, zR, delta_L, dt, bad);
            fB = hllc(mx, zB, zR, bad);
        }
        return blend(a_sig, fA, fB);
    }
    MSt<NM> zRA, zRB;
    split(mx, zL, iA, zA, zB);
    split(mx, zR, iA, zRA, zRB);
    QVd<NM> fA, fB;
    if (aL < aR) {
        fA = crp_classic(mx, zB, zA, zRA, delta_L, dt, bad);
        fB = crp_inverse(mx, zB, zRB, zRA, delta_R, dt, bad);
    } else {
        fA = crp_inverse(mx, zA, zRA, zRB, delta_R, dt, bad);
        fB = crp_classic(mx, zA, zB, zRB, delta_L, dt, bad);
    }
    return blend(a_sig, fA, fB);
}

// calc_crp_flux in two parts for two threads of different warps: every
// composite flux above is blend(a_sig, fA, fB) of two sub-fluxes, one of them
// a CrpFlux::classic (inverse being classic on mirrored states), the other a
// plain HLLC or a second classic.  Part 0 computes the classic one, part 1
// the other; `isA` says whether the result is fA.  The arguments are chosen
// first and each sub-flux is evaluated at one call site, so the lanes of a
// warp that need a classic run it together whatever case they are in.  Each
// sub-flux gets the same arguments as in crp_flux, so blend(a_sig, fA, fB)
// gives crp_flux's result bit for bit.  Not called when aL and aR are both
// 0 or 1 (crp_flux's plain HLLC).
template <int NM>
__device__ __forceinline__ void mirror(MSt<NM> &z) {
    z.vx = -z.vx;
}
template <int NM>
__device__ __noinline__ QVd<NM> crp_part(const MixD<NM> &mx, const MSt<NM> &zL, const MSt<NM> &zR, double hL,
                                         double hR, int iA, double a_sig, double dt, int part, bool &isA, bool &bad) {
    double aL = alpha(zL, iA), aR = alpha(zR, iA);
    double delta_L = (aL < a_sig ? aL / a_sig : (1.0 - aL) / (1.0 - a_sig)) * hL;
    double delta_R = (aR < a_sig ? aR / a_sig : (1.0 - aR) / (1.0 - a_sig)) * hR;
    // classic(p1, p2, p3, delta), inverted when inv; or hllc(p1, p2)
    MSt<NM> p1, p2, p3;
    double delta = 0.0;
    bool inv = false, plain = false;
    MSt<NM> zA, zB;
    if (aL == 0.0 || aL == 1.0) {
        split(mx, zR, iA, zA, zB);  // zA = zRA, zB = zRB
        if (aL == 0.0) {
            // fA = hllc(zL, zA); fB = inverse(zL, zB, zA) = classic(m zA, m zB, m zL), inverted
            isA = part != 0;
            if (part == 0) {
                p1 = zA; p2 = zB; p3 = zL; inv = true; delta = delta_R;
            } else {
                p1 = zL; p2 = zA; plain = true;
            }
        } else {
            // fA = inverse(zL, zA, zB) = classic(m zB, m zA, m zL), inverted; fB = hllc(zL, zB)
            isA = part == 0;
            if (part == 0) {
                p1 = zB; p2 = zA; p3 = zL; inv = true; delta = delta_R;
            } else {
                p1 = zL; p2 = zB; plain = true;
            }
        }
    } else if (aR == 0.0 || aR == 1.0) {
        split(mx, zL, iA, zA, zB);  // zA = zLA, zB = zLB
        if (aR == 0.0) {
            // fA = hllc(zA, zR); fB = classic(zA, zB, zR)
            isA = part != 0;
            if (part == 0) {
                p1 = zA; p2 = zB; p3 = zR; delta = delta_L;
            } else {
                p1 = zA; p2 = zR; plain = true;
            }
        } else {
            // fA = classic(zB, zA, zR); fB = hllc(zB, zR)
            isA = part == 0;
            if (part == 0) {
                p1 = zB; p2 = zA; p3 = zR; delta = delta_L;
            } else {
                p1 = zB; p2 = zR; plain = true;
            }
        }
    } else {
        MSt<NM> zRA, zRB;
        split(mx, zL, iA, zA, zB);
        split(mx, zR, iA, zRA, zRB);
        if (aL < aR) {
            // fA = classic(zB, zA, zRA); fB = inverse(zB, zRB, zRA) = classic(m zRA, m zRB, m zB), inverted
            isA = part == 0;
            if (part == 0) {
                p1 = zB; p2 = zA; p3 = zRA; delta = delta_L;
            } else {
                p1 = zRA; p2 = zRB; p3 = zB; inv = true; delta = delta_R;
            }
        } else {
            // fA = inverse(zA, zRA, zRB) = classic(m zRB, m zRA, m zA), inverted; fB = classic(zA, zB, zRB)
            isA = part == 0;
            if (part == 0) {
                p1 = zRB; p2 = zRA; p3 = zA; inv = true; delta = delta_R;
            } else {
                p1 = zA; p2 = zB; p3 = zRB; delta = delta_L;
            }
        }
    }
    if (plain) return hllc(mx, p1, p2, bad);
    if (inv) {
        mirror(p1);
        mirror(p2);
        mirror(p3);
    }
    QVd<NM> f = crp_classic(mx, p1, p2, p3, delta, dt, bad);
    if (inv) flux_inverse(f);
    return f;
}

// ---------------------------------------------------------------------------
// PLIC helpers
__device__ __forceinline__ double sgn(double x) { return x > 0.0 ? 1.0 : (x < 0.0 ? -1.0 : 0.0); }
__device__ __forceinline__ double heav(double x) { return x > 0.0 ? 1.0 : 0.0; }
__device__ __forceinline__ void sorted2(double a, double b, double &lo, double &hi) {
    if (a < b) {
        lo = a;
        hi = b;
    } else {
        lo = b;
        hi = a;
    }
}
__device__ __forceinline__ double between(double x, double x1, double x2) {
    double lo, hi;
    sorted2(x1, x2, lo, hi);
    return fmax_std(lo, fmin_std(x, hi));
}
__device__ __forceinline__ double quad_find_section(double alpha, double nx, double ny, double A, double B) {
    double a, b;
    sorted2(A * fabs(nx), B * fabs(ny), a, b);
    if (alpha <= 0.5 * a / b) return -0.5 * (a + b) + sqrt(2.0 * alpha * a * b);
    if (alpha < 1.0 - 0.5 * a / b) return (alpha - 0.5) * b;
    return +0.5 * (a + b) - sqrt(2.0 * (1.0 - alpha) * a * b);
}
__device__ __forceinline__ void minmax_unit(double a1, double a2, double &lo, double &hi) {
    if (a1 < a2) {
        lo = fmax_std(0.0, a1);
        hi = fmin_std(a2, 1.0);
    } else {
        lo = fmax_std(0.0, a2);
        hi = fmin_std(a1, 1.0);
    }
}
__device__ __forceinline__ double face_fraction(double a1, double a2) {
    double a_min, a_max;
    minmax_unit(a1, a2, a_min, a_max);
    double hm = a_max - 0.5, hn = a_min - 0.5;
    if (3.0 * a_min >= a_max && a_min >= 3.0 * a_max - 2.0) return 0.5 * (a_min + a_max);
    if (a_max <= 0.5 || a_min * (1.0 - a_max) >= hm * hm) return -2.0 * a_min + 2.0 * sqrt(a_min * (a_min + a_max));
    if (a_min >= 0.5 || a_min * (1.0 - a_max) >= hn * hn)
        return 3.0 - 2.0 * a_max - 2.0 * sqrt((1.0 - a_max) * (2.0 - a_min - a_max));
    if (a_min == 0.0 && a_max == 1.0) return 0.5;
    return sqrt(a_min) / (sqrt(1.0 - a_max) + sqrt(a_min));
}
__device__ __forceinline__ double face_fraction_v3(double a1, double a2) {
    double a_min, a_max;
    minmax_unit(a1, a2, a_min, a_max);
    if (a_min == 0.0) return 0.0;
    if (a_max == 1.0) return 1.0;
    if (a1 + a2 < 1.0) return a_max;
    if (a1 + a2 > 1.0) return a_min;
    return 0.5 * (a1 + a2);
}
__device__ __forceinline__ double face_fraction_v5(double a1, double a2) {
    double a_min, a_max;
    minmax_unit(a1, a2, a_min, a_max);
    if (a_min == 0.0) return 0.0;
    if (a_max == 1.0) return 1.0;
    return 0.5 * (a1 + a2);
}
__device__ __forceinline__ double face_fraction_s(double a1, double a2) {
    double a_min, a_max;
    minmax_unit(a1, a2, a_min, a_max);
    double a_sig = a_min / (1.0 - (a_max - a_min));
    if (isnan(a_sig)) a_sig = 0.5;
    return between(a_sig, a_min, a_max);
}
__device__ __forceinline__ double average_flux(double alpha, double cs, double CFL) {
    double a1, b1, a2, b2;
    double sn = sqrt(1.0 - cs * cs);
    sorted2(fabs(cs), sn, a1, b1);
    sorted2(CFL * fabs(cs), sn, a2, b2);
    double P1;
    if (fabs(2.0 * alpha - 1.0) <= 1.0 - a1 / b1) {
        P1 = (alpha - 0.5) * b1;
    } else {
        P1 = sgn(alpha - 0.5) * (0.5 * (a1 + b1) - sqrt((1.0 - fabs(2.0 * alpha - 1.0)) * a1 * b1));
    }
    double P2 = P1 + 0.5 * (CFL - 1.0) * cs;
    if (fabs(P2) <= 0.5 * (b2 - a2)) return 0.5 + P2 / b2;
    if (fabs(P2) < 0.5 * (b2 + a2)) {
        double d = fabs(P2) - 0.5 * (a2 + b2);
        return heav(P2) - 0.5 * sgn(P2) * (d * d) / (a2 * b2);
    }
    return heav(P2);
}

enum : int { CRP_NONE = 0, CRP_V3 = 1, CRP_V5 = 2, CRP_VS = 3, CRP_PLIC = 4, CRP_MUSCL = 5 };

}  // namespace mmf
}  // namespace zg
