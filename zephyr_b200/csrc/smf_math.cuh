// smf_math.cuh -- pointwise FP64 numerics of zephyr's single-material step,
// written for sm_100a.  The FP64 forms keep the reference's operation order
// term by term; translation units that include this header for the parity
// kernels are compiled with -fmad=false so that no product is fused into an
// add, which makes the results bit-identical to the reference's x86-64 build
// (apart from the signs of exact zeros).
//
// Reference lines (zephyr source tree):
//   EoS            phys/matter/eos/ideal_gas.cpp:32-106, stiffened_gas.cpp:103-175
//   PState/QState  math/cfd/models.cpp:27-32 (P from Q), 85-89 (Q from P), 131-137 (Flux)
//   is_bad         math/cfd/models.cpp:58-63
//   HLLC           math/cfd/flux/hllc.cpp:23-83
//   HLL            math/cfd/flux/hll.cpp:23-57
//   limiters       math/cfd/limiter.cxx:15-153 (binary forms)
//   rotation       math/cfd/rotate.cpp:7-77 (2-D branch)
#pragma once

#include <math_constants.h>

#include <cstdint>

namespace zg {

enum : int { EOS_IDEAL = 0, EOS_STIFFENED = 1 };
enum : int {
    FLUX_GODUNOV = 0, FLUX_RUSANOV = 1, FLUX_HLL = 2, FLUX_HLLC = 3, FLUX_HLLC_M = 4, FLUX_HLLC_LM = 5,
    FLUX_CIR1 = 6, FLUX_CIR2 = 7
};
enum : int {
    LIM_NONE = 0, LIM_UNIT, LIM_MINMOD, LIM_MC, LIM_VANLEER, LIM_VANALBADA1, LIM_VANALBADA2,
    LIM_CHARM, LIM_HCUS, LIM_HQUICK, LIM_KOREN, LIM_SMART, LIM_SUPERBEE
};
enum : int { BC_UNDEFINED = -1, BC_INNER = 0, BC_WALL = 1, BC_ZOE = 2, BC_PERIODIC = 3, BC_FUNCTION = 4 };

// amr_faces.h:157-161
__host__ __device__ inline bool is_boundary(int flag) {
    return flag != BC_INNER && flag != BC_PERIODIC && flag != BC_UNDEFINED;
}

// std::min / std::max as the reference uses them (NaN in the second slot
// loses, ties return the first argument).
__host__ __device__ inline double smin(double a, double b) { return (b < a) ? b : a; }
__host__ __device__ inline double smax(double a, double b) { return (a < b) ? b : a; }
template <typename T>
__host__ __device__ inline T smin_t(T a, T b) { return (b < a) ? b : a; }
template <typename T>
__host__ __device__ inline T smax_t(T a, T b) { return (a < b) ? b : a; }

// Correctly rounded x^3 (stands in for glibc pow(x, 3) in gradient.h:256):
// Dekker/Knuth error-free products give x^3 = q + qe + pe*x exactly, and the
// final sum rounds once.  Exact whenever x^3 is representable.
__host__ __device__ inline double cube_rn(double x) {
    double p = x * x;
    double pe = fma(x, x, -p);
    double q = p * x;
    double qe = fma(p, x, -q);
    return q + (qe + pe * x);
}

struct EosD {
    int kind;
    double gamma, gm1, P0, e0, pmin;

    __host__ __device__ inline double pressure_re(double rho, double e) const {
        if (kind == EOS_IDEAL) return gm1 * rho * e;
        return gm1 * rho * (e - e0) - gamma * P0;
    }
    __host__ __device__ inline double energy_rP(double rho, double P) const {
        if (kind == EOS_IDEAL) return P / (gm1 * rho);
        return e0 + (P + gamma * P0) / (gm1 * rho);
    }
    __host__ __device__ inline double sound_speed_rP(double rho, double P) const {
        if (kind == EOS_IDEAL) return sqrt(gamma * P / rho);
        return sqrt(gamma * (P + P0) / rho);
    }
};

// 2-D primitive state (the reference's PState with vz == 0).
struct Prim {
    double r, u, v, p, e;
};
// Conservative vector / flux (density, momentum x, momentum y, total energy).
struct Cons {
    double r, mu, mv, E;
};

__host__ __device__ inline double v2(const Prim &z) { return z.u * z.u + z.v * z.v; }

// models.cpp:85-89
__host__ __device__ inline Cons q_from_p(const Prim &z) {
    Cons q;
    q.r = z.r;
    q.mu = z.r * z.u;
    q.mv = z.r * z.v;
    q.E = z.r * (z.e + 0.5 * v2(z));
    return q;
}
// models.cpp:27-32
__host__ __device__ inline Prim p_from_q(const Cons &q, const EosD &eos) {
    Prim z;
    z.r = q.r;
    z.u = q.mu / z.r;
    z.v = q.mv / z.r;
    z.e = q.E / z.r - 0.5 * v2(z);
    z.p = eos.pressure_re(z.r, z.e);
    return z;
}
// models.cpp:131-137
__device__ inline Cons flux_from_p(const Prim &z) {
    Cons f;
    double ru = z.r * z.u;
    f.r = ru;
    f.mu = ru * z.u + z.p;
    f.mv = ru * z.v;
    f.E = (z.r * (z.e + 0.5 * v2(z)) + z.p) * z.u;
    return f;
}
// models.cpp:58-63
__host__ __device__ inline bool is_bad(const Prim &z, const EosD &eos) {
    if (!isfinite(z.r) || !isfinite(z.p) || !isfinite(z.e)) return true;
    return z.r <= 0.0 || z.p < eos.pmin;
}

// rotate.cpp:7-41: velocity into the frame of the unit normal (c, s).
__device__ inline void rot_local(double &u, double &v, double c, double s) {
    double a = c * u + s * v;
    double b = -s * u + c * v;
    u = a;
    v = b;
}
// rotate.cpp:43-77
__device__ inline void rot_global(double &u, double &v, double c, double s) {
    double a = c * u + -s * v;
    double b = s * u + c * v;
    u = a;
    v = b;
}

// hllc.cpp:23-83
__device__ inline Cons hllc(const Prim &zL, const Prim &zR, const EosD &eos) {
    double c_L = eos.sound_speed_rP(zL.r, zL.p);
    double c_R = eos.sound_speed_rP(zR.r, zR.p);
    double S_L = smin(zL.u - c_L, zR.u - c_R);
    double S_R = smax(zL.u + c_L, zR.u + c_R);
    if (S_L >= 0.0) return flux_from_p(zL);
    if (S_R <= 0.0) return flux_from_p(zR);

    double a_L = zL.r * (S_L - zL.u);
    double a_R = zR.r * (S_R - zR.u);
    double S_C = (zL.p - zR.p + a_R * zR.u - a_L * zL.u) / (a_R - a_L);
    double rho_sL = a_L / (S_L - S_C);
    double rho_sR = a_R / (S_R - S_C);
    double EL = zL.e + 0.5 * v2(zL);
    double ER = zR.e + 0.5 * v2(zR);
    double E_sL = EL + (S_C - zL.u) * (S_C + zL.p / a_L);
    double E_sR = ER + (S_C - zR.u) * (S_C + zR.p / a_R);

    Cons QsL{rho_sL, rho_sL * S_C, rho_sL * zL.v, rho_sL * E_sL};
    Cons QsR{rho_sR, rho_sR * S_C, rho_sR * zR.v, rho_sR * E_sR};
    Cons QL = q_from_p(zL), QR = q_from_p(zR);
    Cons FL = flux_from_p(zL), FR = flux_from_p(zR);
    double aSC = fabs(S_C);
    Cons F;
    F.r = 0.5 * (FL.r + FR.r + S_L * (QsL.r - QL.r) + aSC * (QsL.r - QsR.r) + S_R * (QsR.r - QR.r));
    F.mu = 0.5 * (FL.mu + FR.mu + S_L * (QsL.mu - QL.mu) + aSC * (QsL.mu - QsR.mu) + S_R * (QsR.mu - QR.mu));
    F.mv = 0.5 * (FL.mv + FR.mv + S_L * (QsL.mv - QL.mv) + aSC * (QsL.mv - QsR.mv) + S_R * (QsR.mv - QR.mv));
    F.E = 0.5 * (FL.E + FR.E + S_L * (QsL.E - QL.E) + aSC * (QsL.E - QsR.E) + S_R * (QsR.E - QR.E));
    return F;
}

// hll.cpp:23-57
__device__ inline Cons hll(const Prim &zL, const Prim &zR, const EosD &eos) {
    double c_L = eos.sound_speed_rP(zL.r, zL.p);
    double c_R = eos.sound_speed_rP(zR.r, zR.p);
    double S_L = smin(zL.u - c_L, smin(zR.u - c_R, 0.0));
    double S_R = smax(zL.u + c_L, smax(zR.u + c_R, 0.0));
    Cons QL = q_from_p(zL), QR = q_from_p(zR);
    Cons FL = flux_from_p(zL), FR = flux_from_p(zR);
    double SLR = S_L * S_R;
    double den = S_R - S_L;
    Cons F;
    F.r = (S_R * FL.r - S_L * FR.r + SLR * (QR.r - QL.r)) / den;
    F.mu = (S_R * FL.mu - S_L * FR.mu + SLR * (QR.mu - QL.mu)) / den;
    F.mv = (S_R * FL.mv - S_L * FR.mv + SLR * (QR.mv - QL.mv)) / den;
    F.E = (S_R * FL.E - S_L * FR.E + SLR * (QR.E - QL.E)) / den;
    return F;
}

// rusanov.cpp:15-43 (std::min / std::max of an initializer list keep the
// first extreme element)
__device__ inline Cons rusanov(const Prim &zL, const Prim &zR, const EosD &eos) {
    double c_L = eos.sound_speed_rP(zL.r, zL.p);
    double c_R = eos.sound_speed_rP(zR.r, zR.p);
    double S_L = zL.u - c_L, S_R = zL.u + c_L;
    if (zR.u - c_R < S_L) S_L = zR.u - c_R;
    if (0.0 < S_L) S_L = 0.0;
    if (S_R < zR.u + c_R) S_R = zR.u + c_R;
    if (S_R < 0.0) S_R = 0.0;
    const double S = smax(fabs(S_L), S_R), hS = 0.5 * S;
    Cons QL = q_from_p(zL), QR = q_from_p(zR);
    Cons FL = flux_from_p(zL), FR = flux_from_p(zR);
    Cons F;
    F.r = 0.5 * (FL.r + FR.r) + hS * (QL.r - QR.r);
    F.mu = 0.5 * (FL.mu + FR.mu) + hS * (QL.mu - QR.mu);
    F.mv = 0.5 * (FL.mv + FR.mv) + hS * (QL.mv - QR.mv);
    F.E = 0.5 * (FL.E + FR.E) + hS * (QL.E - QR.E);
    return F;
}

// ---------------------------------------------------------------------------
// Exact Riemann solver for two stiffened gases (math/solver/riemann.cpp) and
// the Godunov flux of its face state (godunov.cpp:16-32).  The powers of the
// rarefaction branches use CUDA's pow, so this flux agrees with the
// reference to a few ulps rather than bit for bit.
namespace riemann {

__device__ inline double fK(double P, double rK, double pK, double cK, double gK, double p0K, double AK, double BK,
                            double GK) {  // riemann.cpp:76-84
    if (P >= pK) return (P - pK) * sqrt(AK / (P + BK));
    return 2.0 * cK / (gK - 1.0) * (pow((P + p0K) / (pK + p0K), GK) - 1.0);
}
__device__ inline double dfK(double P, double rK, double pK, double cK, double gK, double p0K, double AK, double BK,
                             double GK) {  // riemann.cpp:86-94
    if (P >= pK) return (1.0 - (P - pK) / (2.0 * (P + BK))) * sqrt(AK / (P + BK));
    return pow((P + p0K) / (pK + p0K), GK - 1.0) / (rK * cK);
}
// the acoustic initial guess (riemann.cpp:32-61: all three cases use it)
__device__ inline double p_init(double rL, double uL, double pL, double cL, double p0L, double rR, double uR,
                                double pR, double cR, double p0R) {
    double rcL = rL * cL, rcR = rR * cR;
    double P = (pL * rcR + pR * rcL + (uL - uR) * rcL * rcR) / (rcL + rcR);
    double Pmin = -smin(p0L, p0R) + 1.0e-2 * smin(pL + p0L, pR + p0R);
    return smax(Pmin, P);
}

// contact_p (riemann.cpp:118-236): pressure and velocity of the contact.
// `failed`: the case where the reference throws (no convergence, far off).
__device__ inline void contact(double rL, double uL, double pL, double cL, double gL, double p0L, double rR,
                               double uR, double pR, double cR, double gR, double p0R, double &P_out, double &U_out,
                               bool &failed) {
    const double AL = 2.0 / ((gL + 1) * rL), AR = 2.0 / ((gR + 1) * rR);
    const double BL = (gL - 1.0) * pL / (gL + 1.0) + 2.0 * gL * p0L / (gL + 1.0);
    const double BR = (gR - 1.0) * pR / (gR + 1.0) + 2.0 * gR * p0R / (gR + 1.0);
    const double GL = (gL - 1.0) / (2.0 * gL), GR = (gR - 1.0) / (2.0 * gR);
    const double p_dno = smax(-p0L, -p0R);
    failed = false;
    const double f_dno =
        fK(p_dno, rL, pL, cL, gL, p0L, AL, BL, GL) + fK(p_dno, rR, pR, cR, gR, p0R, AR, BR, GR) + uR - uL;
    if (f_dno > 0.0) {  // vacuum
        P_out = p_dno;
        U_out = 0.0;
        return;
    }
    double P = p_init(rL, uL, pL, cL, p0L, rR, uR, pR, cR, p0R);
    const double DP1 = 1.0e-5 * fabs(pL - pR);
    const double DP2 = 1.0e-12 * fabs(smax(pL + p0L, pR + p0R));
    const double DP = smax(DP1, DP2);
    double fL = 0.0, fR = 0.0, Pn = P;
    int counter = 0;
    for (; counter < 50; ++counter) {
        fL = fK(P, rL, pL, cL, gL, p0L, AL, BL, GL);
        fR = fK(P, rR, pR, cR, gR, p0R, AR, BR, GR);
        const double dfL = dfK(P, rL, pL, cL, gL, p0L, AL, BL, GL);
        const double dfR = dfK(P, rR, pR, cR, gR, p0R, AR, BR, GR);
        Pn = P - (fL + fR + uR - uL) / (dfL + dfR);
        if (Pn < p_dno) Pn = (p_dno + P) / 2;
        if (fabs(Pn - P) < DP && counter > 3) break;
        P = Pn;
    }
    if (counter >= 50 && fabs((P - Pn) / (P + Pn)) > 0.02) failed = true;
    P_out = P;
    U_out = 0.5 * (uL + uR + fR - fL);
}

// RiemannSolver::solve (riemann.cpp:366-460): density, velocity and pressure
// on the face x / t = 0, and the contact velocity U.
__device__ inline void solve(double rL, double uL, double pL, double gL, double p0L, double rR, double uR, double pR,
                             double gR, double p0R, double &rho, double &Uf, double &Pf, double &U, bool &failed) {
    const double cL = sqrt(gL * (pL + p0L) / rL);
    const double cR = sqrt(gR * (pR + p0R) / rR);
    double P;
    contact(rL, uL, pL, cL, gL, p0L, rR, uR, pR, cR, gR, p0R, P, U, failed);
    if (U > 0.0) {
        if (pL < P) {
            const double D = uL + (P - pL) / (rL * (U - uL));
            if (D > 0.0) {
                rho = rL; Uf = uL; Pf = pL;
            } else {
                rho = rL * (P - pL) / ((P - pL) - rL * ((U - uL) * (U - uL)));
                Uf = U; Pf = P;
            }
        } else if (uL - cL > 0.0) {
            rho = rL; Uf = uL; Pf = pL;
        } else {
            const double cl = cL + 0.5 * (gL - 1.0) * (uL - U);
            if (U - cl < 0.0) {
                rho = gL * (P + p0L) / (cl * cl);
                Uf = U; Pf = P;
            } else {
                const double base = 2.0 / (gL + 1.0) + ((gL - 1.0) * (uL - 0.0)) / ((gL + 1.0) * cL);
                rho = rL * pow(base, 2.0 / (gL - 1.0));
                Uf = ((gL - 1.0) * uL + 2.0 * (cL + 0.0)) / (gL + 1.0);
                Pf = (pL + p0L) * pow(base, 2.0 * gL / (gL - 1.0)) - p0L;
            }
        }
    } else {
        if (P > pR) {
            const double D = uR + (P - pR) / (rR * (U - uR));
            if (D < 0.0) {
                rho = rR; Uf = uR; Pf = pR;
            } else {
                rho = rR * (P - pR) / ((P - pR) - rR * ((U - uR) * (U - uR)));
                Uf = U; Pf = P;
            }
        } else if (uR + cR < 0.0) {
            rho = rR; Uf = uR; Pf = pR;
        } else {
            const double cr = cR - 0.5 * (gR - 1.0) * (uR - U);
            if (U + cr > 0.0) {
                rho = gR * (P + p0R) / (cr * cr);
                Uf = U; Pf = P;
            } else {
                const double base = 2.0 / (gR + 1.0) - ((gR - 1.0) * (uR - 0.0)) / ((gR + 1.0) * cR);
                rho = rR * pow(base, 2.0 / (gR - 1.0));
                Uf = ((gR - 1.0) * uR + 2.0 * (0.0 - cR)) / (gR + 1.0);
                Pf = (pR + p0R) * pow(base, 2.0 * gR / (gR - 1.0)) - p0R;
            }
        }
    }
}

}  // namespace riemann

// Godunov::calc_flux (godunov.cpp:16-32): the gas's own stiffened-gas
// parameters (IdealGas / StiffenedGas::stiffened_gas: gamma, P0), the exact
// face state, its physical flux.
__device__ inline Cons godunov(const Prim &zL, const Prim &zR, const EosD &eos) {
    const double P0 = eos.kind == EOS_IDEAL ? 0.0 : eos.P0;
    double rho, Uf, Pf, U;
    bool failed;
    riemann::solve(zL.r, zL.u, zL.p, eos.gamma, P0, zR.r, zR.u, zR.p, eos.gamma, P0, rho, Uf, Pf, U, failed);
    Prim z;
    z.r = rho;
    z.u = Uf;
    z.v = U > 0.0 ? zL.v : zR.v;
    z.p = Pf;
    z.e = eos.energy_rP(rho, Pf);
    if (failed) z.r = CUDART_NAN;  // the reference throws here; the flux becomes NaN instead
    return flux_from_p(z);
}

// The exact solver out of line: inlined, its Newton and fan code raised the
// register demand of every face kernel and made the HLLC path spill.
static __device__ __noinline__ Cons godunov_ool(const Prim zL, const Prim zR, const EosD eos) {
    return godunov(zL, zR, eos);
}

// The symmetric HLLC sum 0.5 (F_L + F_R + a S_L (Q*L - Q_L) + |S_C| (Q*L - Q*R)
// + b S_R (Q*R - Q_R)) of hllc.cpp, component by component.
__device__ inline double hllc_sum(double fl, double fr, double aSL, double ql, double qsl, double aSC, double qsr,
                                  double bSR, double qr) {
    return 0.5 * (fl + fr + aSL * (qsl - ql) + aSC * (qsl - qsr) + bSR * (qsr - qr));
}

// hllc.cpp:427-495 (HLLC_LM): the HLLC flux with the outer-wave terms scaled
// by phi = sin(pi/2 min(Ma / 0.1, 1)), Ma the larger face Mach number.  The
// sine is CUDA's: phi, and so the flux, agrees with glibc's to rounding.
static __device__ __noinline__ Cons hllc_lm(const Prim zL, const Prim zR, const EosD eos) {
    double c_L = eos.sound_speed_rP(zL.r, zL.p);
    double c_R = eos.sound_speed_rP(zR.r, zR.p);
    double S_L = smin(zL.u - c_L, zR.u - c_R);
    double S_R = smax(zL.u + c_L, zR.u + c_R);
    if (S_L >= 0.0) return flux_from_p(zL);
    if (S_R <= 0.0) return flux_from_p(zR);
    double a_L = zL.r * (S_L - zL.u);
    double a_R = zR.r * (S_R - zR.u);
    double S_C = (zL.p - zR.p + a_R * zR.u - a_L * zL.u) / (a_R - a_L);
    double rho_sL = a_L / (S_L - S_C);
    double rho_sR = a_R / (S_R - S_C);
    double E_sL = (zL.e + 0.5 * v2(zL)) + (S_C - zL.u) * (S_C + zL.p / a_L);
    double E_sR = (zR.e + 0.5 * v2(zR)) + (S_C - zR.u) * (S_C + zR.p / a_R);
    Cons QsL{rho_sL, rho_sL * S_C, rho_sL * zL.v, rho_sL * E_sL};
    Cons QsR{rho_sR, rho_sR * S_C, rho_sR * zR.v, rho_sR * E_sR};
    Cons QL = q_from_p(zL), QR = q_from_p(zR), FL = flux_from_p(zL), FR = flux_from_p(zR);
    double Ma = smax(fabs(zL.u / c_L), fabs(zR.u / c_R));
    double xi = Ma / 0.1;
    double phi = xi > 1.0 ? 1.0 : sin(1.57079632679489661923 * xi);  // M_PI_2
    double pSL = phi * S_L, pSR = phi * S_R, aSC = fabs(S_C);
    return Cons{hllc_sum(FL.r, FR.r, pSL, QL.r, QsL.r, aSC, QsR.r, pSR, QR.r),
                hllc_sum(FL.mu, FR.mu, pSL, QL.mu, QsL.mu, aSC, QsR.mu, pSR, QR.mu),
                hllc_sum(FL.mv, FR.mv, pSL, QL.mv, QsL.mv, aSC, QsR.mv, pSR, QR.mv),
                hllc_sum(FL.E, FR.E, pSL, QL.E, QsL.E, aSC, QsR.E, pSR, QR.E)};
}

// hllc.cpp:499-570 (HLLC_M): the tangential velocity is averaged across the
// contact as well, with the matching energy correction (v_z = 0 in 2-D;
// pow(x, 2) is the correctly rounded square x * x).
static __device__ __noinline__ Cons hllc_m(const Prim zL, const Prim zR, const EosD eos) {
    double c_L = eos.sound_speed_rP(zL.r, zL.p);
    double c_R = eos.sound_speed_rP(zR.r, zR.p);
    double S_L = smin(zL.u - c_L, zR.u - c_R);
    double S_R = smax(zL.u + c_L, zR.u + c_R);
    if (S_L >= 0.0) return flux_from_p(zL);
    if (S_R <= 0.0) return flux_from_p(zR);
    double a_L = zL.r * (S_L - zL.u);
    double a_R = zR.r * (S_R - zR.u);
    double S_C = (zL.p - zR.p + a_R * zR.u - a_L * zL.u) / (a_R - a_L);
    double V_C = (a_R * zR.v - a_L * zL.v) / (a_R - a_L);
    double rho_sL = a_L / (S_L - S_C);
    double rho_sR = a_R / (S_R - S_C);
    double E_sL = (zL.e + 0.5 * v2(zL)) + (S_C - zL.u) * (S_C + zL.p / a_L);
    double E_sR = (zR.e + 0.5 * v2(zR)) + (S_C - zR.u) * (S_C + zR.p / a_R);
    double v_L2 = zL.v * zL.v + 0.0, v_R2 = zR.v * zR.v + 0.0;
    E_sL += 0.5 * ((a_R * v_R2 - a_L * v_L2) / (a_R - a_L) - v_L2);
    E_sR += 0.5 * ((a_R * v_R2 - a_L * v_L2) / (a_R - a_L) - v_R2);
    Cons QsL{rho_sL, rho_sL * S_C, rho_sL * V_C, rho_sL * E_sL};
    Cons QsR{rho_sR, rho_sR * S_C, rho_sR * V_C, rho_sR * E_sR};
    Cons QL = q_from_p(zL), QR = q_from_p(zR), FL = flux_from_p(zL), FR = flux_from_p(zR);
    double aSC = fabs(S_C);
    return Cons{hllc_sum(FL.r, FR.r, S_L, QL.r, QsL.r, aSC, QsR.r, S_R, QR.r),
                hllc_sum(FL.mu, FR.mu, S_L, QL.mu, QsL.mu, aSC, QsR.mu, S_R, QR.mu),
                hllc_sum(FL.mv, FR.mv, S_L, QL.mv, QsL.mv, aSC, QsR.mv, S_R, QR.mv),
                hllc_sum(FL.E, FR.E, S_L, QL.E, QsL.E, aSC, QsR.E, S_R, QR.E)};
}

// Courant-Isaacson-Rees fluxes (cir.cpp:20-125 CIR1, 129-234 CIR2):
// F = (F_L + F_R) / 2 + (|A| / 2) (q_L - q_R) with |A| = R |Lambda| L of the
// Jacobian at the averaged state.  Vectors carry the reference's five (six)
// components (density, momentum x, y, z, energy[, pressure]) with z = 0; the
// dense products sum k in increasing order from the k = 0 term, the order of
// the Eigen stand-in the reference is built with here.  The consistency
// check of CIR2 (cir.cpp:180-211, which throws when R Lambda L misses the
// Jacobian by more than 1e-10) is not made.
template <int NV>
__device__ inline Cons cir_flux(const Prim &zL, const Prim &zR, const EosD &eos) {
    const double rho = 0.5 * (zL.r + zR.r), u = 0.5 * (zL.u + zR.u), v = 0.5 * (zL.v + zR.v), w = 0.5 * (0.0 + 0.0);
    const double p = 0.5 * (zL.p + zR.p);
    const double eps = eos.energy_rP(rho, p);
    const double u2 = u * u, vv = v * v, w2 = w * w;
    const double q2 = u2 + vv + w2;
    const double E = rho * (eps + 0.5 * q2);
    const double c = eos.sound_speed_rP(rho, p);
    const double c2 = c * c;
    const double h = (E + p) / rho;
    double RL[5][NV], L[NV][NV];
    if (NV == 5) {
        const double dE = eos.gm1 * rho;  // pressure_re's dP/de (ideal_gas.cpp:32-39, stiffened_gas.cpp:103-110)
        const double b = dE / rho;
        const double T = b * (q2 - h) + c2;
        const double lam[5] = {fabs(u - c), fabs(u), fabs(u), fabs(u), fabs(u + c)};
        const double R[5][5] = {{1, 0, 0, 1, 1},
                                {u - c, 0, 0, u, u + c},
                                {v, 1, 0, v, v},
                                {w, 0, 1, w, w},
                                {h - u * c, v, w, h - c2 / b, h + u * c}};
        const double Lm[5][5] = {{T + u * c, -b * u - c, -b * v, -b * w, b},
                                 {-2 * v * c2, 0, 2 * c2, 0, 0},
                                 {-2 * w * c2, 0, 0, 2 * c2, 0},
                                 {2 * b * (h - q2), 2 * b * u, 2 * b * v, 2 * b * w, -2 * b},
                                 {T - u * c, -b * u + c, -b * v, -b * w, b}};
        const double den = 2.0 * c2;
        for (int i = 0; i < 5; ++i)
            for (int j = 0; j < 5; ++j) {
                RL[i][j] = R[i][j] * lam[j];
                L[i][j] = Lm[i][j] / den;
            }
    } else {
        const double lam[6] = {fabs(u - c), fabs(u), fabs(u), fabs(u), fabs(u + c), fabs(u)};
        const double R[5][6] = {{1, 0, 0, 0, 1, 1},
                                {u - c, 0, 0, 0, u + c, u},
                                {v, 1, 0, 0, v, 0},
                                {w, 0, 1, 0, w, 0},
                                {h - u * c, 0, 0, 1, h + u * c, 0}};
        const double Lm[6][6] = {{u / (2 * c), -1 / (2 * c), 0, 0, 0, 1 / (2 * c2)},
                                 {0, 0, 1, 0, 0, -v / c2},
                                 {0, 0, 0, 1, 0, -w / c2},
                                 {u2, -u, 0, 0, 1, -h / c2},
                                 {-u / (2 * c), 1 / (2 * c), 0, 0, 0, 1 / (2 * c2)},
                                 {1, 0, 0, 0, 0, -1 / c2}};
        for (int i = 0; i < 5; ++i)
            for (int j = 0; j < NV; ++j) RL[i][j] = R[i][j] * lam[j];
        for (int i = 0; i < NV; ++i)
            for (int j = 0; j < NV; ++j) L[i][j] = Lm[i][j];
    }
    // |A| / 2 times (q_L - q_R)
    const Cons qL = q_from_p(zL), qR = q_from_p(zR), fL = flux_from_p(zL), fR = flux_from_p(zR);
    const double dq[6] = {qL.r - qR.r, qL.mu - qR.mu, qL.mv - qR.mv, 0.0 - 0.0, qL.E - qR.E, zL.p - zR.p};
    double out[5];
    for (int i = 0; i < 5; ++i) {
        double acc = 0.0;
        for (int j = 0; j < NV; ++j) {
            double a = RL[i][0] * L[0][j];
            for (int k = 1; k < NV; ++k) a = a + RL[i][k] * L[k][j];
            const double term = (0.5 * a) * dq[j];
            acc = j == 0 ? term : acc + term;
        }
        out[i] = acc;
    }
    return Cons{0.5 * (fL.r + fR.r) + out[0], 0.5 * (fL.mu + fR.mu) + out[1], 0.5 * (fL.mv + fR.mv) + out[2],
                0.5 * (fL.E + fR.E) + out[4]};
}
static __device__ __noinline__ Cons cir1(const Prim zL, const Prim zR, const EosD eos) {
    return cir_flux<5>(zL, zR, eos);
}
static __device__ __noinline__ Cons cir2(const Prim zL, const Prim zR, const EosD eos) {
    return cir_flux<6>(zL, zR, eos);
}

__device__ inline Cons num_flux(int kind, const Prim &zL, const Prim &zR, const EosD &eos) {
    switch (kind) {
        case FLUX_GODUNOV: return godunov_ool(zL, zR, eos);
        case FLUX_RUSANOV: return rusanov(zL, zR, eos);
        case FLUX_HLL: return hll(zL, zR, eos);
        case FLUX_HLLC_M: return hllc_m(zL, zR, eos);
        case FLUX_HLLC_LM: return hllc_lm(zL, zR, eos);
        case FLUX_CIR1: return cir1(zL, zR, eos);
        case FLUX_CIR2: return cir2(zL, zR, eos);
        default: return hllc(zL, zR, eos);
    }
}

// The flux of a kernel instantiated for one flux family: FX = FLUX_HLLC or
// FLUX_HLL calls that flux directly (the kernel then carries none of the
// other fluxes' code or registers); FX = -1 takes the run-time switch.
template <int FX>
__device__ inline Cons flux_fx(int kind, const Prim &zL, const Prim &zR, const EosD &eos) {
    if constexpr (FX == FLUX_HLLC) return hllc(zL, zR, eos);
    else if constexpr (FX == FLUX_HLL) return hll(zL, zR, eos);
    else return num_flux(kind, zL, zR, eos);
}

// limiter.cxx binary forms phi(a, b)
__device__ inline double lim_MC1(double r) {
    if (isnan(r)) return 0.0;
    return smax(0.0, smin(2 * r, smin(0.5 * (1.0 + r), 2.0)));
}
__device__ inline double limiter2(int kind, double a, double b) {
    switch (kind) {
        case LIM_NONE: return 0.0;
        case LIM_UNIT: return 1.0;
        case LIM_MINMOD:
            if (a * b <= 0.0) return 0.0;
            return smin(a / b, 1.0);
        case LIM_MC: return lim_MC1(a / b);
        case LIM_VANLEER:
            if (a * b < 0.0) return 0.0;
            if (a == 0.0) return 0.0;
            return 2 * fabs(a) / (fabs(a) + fabs(b));
        case LIM_VANALBADA1:
            if (a * b <= 0.0) return 0.0;
            if (b == 0.0) return 1.0;
            return a * (a + b) / (a * a + b * b);
        case LIM_VANALBADA2: {
            if (a * b <= 0.0) return 0.0;
            const double eps = 10e-6;
            return (2.0 * a * b + eps) / (a * a + b * b + eps);
        }
        case LIM_CHARM: {
            if (a * b <= 0.0) return 0.0;
            double s = a + b;
            return a * (3 * a + b) / (s * s);
        }
        case LIM_HCUS:
            if (a * b <= 0.0) return 0.0;
            return (3.0 * a) / (a + 2.0 * b);
        case LIM_HQUICK:
            if (a * b <= 0.0) return 0.0;
            return (4.0 * a) / (a + 3.0 * b);
        case LIM_KOREN: {
            double r = a / b;
            if (isnan(r)) return 0.0;
            return smax(0.0, smin(2 * r, smin(2.0, (1 + 2 * r) / 3.0)));
        }
        case LIM_SMART: {
            double r = a / b;
            if (isnan(r)) return 0.0;
            return smax(0.0, smin(2.0 * r, smin(0.25 + 0.75 * r, 4.0)));
        }
        case LIM_SUPERBEE: {
            double r = a / b;
            if (isnan(r)) return 0.0;
            return smax(0.0, smin(smin(2 * r, 1.0), smin(r, 2.0)));
        }
        default: return 0.0;
    }
}

// Ordered-integer image of a non-negative double, for atomicMin reductions.
__device__ inline unsigned long long dbits(double x) { return (unsigned long long)__double_as_longlong(x); }

}  // namespace zg
