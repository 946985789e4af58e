// zoracle.cpp -- TEST INFRASTRUCTURE ONLY (the oracle).
//
// A plain C++ restatement, on the CPU, of zephyr's single-material explicit
// finite-volume step (SmFluid) and of the mesh pieces it reads.  It exists to
// check the CUDA library: tests, the smoke check and the bench's CPU-baseline
// leg call it; the product never links or calls it.
//
// Every function below names the reference file:line it restates.  Paths are
// relative to the zephyr source tree.  Floating point follows the reference's
// operation order term by term (compile with -ffp-contract=off so that no
// multiply-add is contracted, as in the reference's x86-64 -O3 build), so that
// the restatement is bit-identical to the reference wherever the reference
// itself is deterministic.
//
// Deliberate, documented deviations (none change results on the workloads):
//  * SmFluid::fluxes_stage2 (sm_fluid.cpp:293) reads the neighbour's `wait`
//    while the same parallel loop rewrites it (sm_fluid.cpp:354-364); the
//    result then depends on thread scheduling.  Here `wait` is read from a
//    snapshot taken before the stage (deterministic; identical to the
//    reference whenever no cell changes its `wait` in that stage).
//  * Velocities keep the z component (always 0 in 2-D) so that every dot
//    product and rotation has the reference's three terms.

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <limits>
#include <string>
#include <thread>
#include <vector>

namespace zo {

// ---------------------------------------------------------------------------
// 3-vector with the element order of Eigen::Matrix<double,3,1> expressions
// (zephyr/geom/vector.h:19).  Reductions run x, y, z left to right.
struct V3 {
    double x, y, z;
};
static inline V3 add(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
static inline V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
static inline V3 mul(double s, V3 a) { return {s * a.x, s * a.y, s * a.z}; }
static inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline double sqnorm(V3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
static inline double norm(V3 a) { return std::sqrt(sqnorm(a)); }
// Eigen normalized(): divide by sqrt(squaredNorm) when it is positive.
static inline V3 normalized(V3 a) {
    double sn = sqnorm(a);
    if (sn > 0.0) {
        double s = std::sqrt(sn);
        return {a.x / s, a.y / s, a.z / s};
    }
    return a;
}

// ---------------------------------------------------------------------------
// Equations of state: zephyr/phys/matter/eos/ideal_gas.cpp,
// stiffened_gas.cpp.  IdealGas is the stiffened gas with P0 = e0 = 0, but the
// formulas differ in operation order, so both are kept.
enum EosKind { EOS_IDEAL = 0, EOS_STIFFENED = 1 };

struct Eos {
    int kind;
    double gamma, P0, e0;

    // ideal_gas.cpp:32-39 / stiffened_gas.cpp:103-110
    double pressure_re(double rho, double e) const {
        if (kind == EOS_IDEAL) return (gamma - 1.0) * rho * e;
        return (gamma - 1.0) * rho * (e - e0) - gamma * P0;
    }
    // Derivatives of pressure_re (same lines, options.deriv branch).
    void pressure_re_deriv(double rho, double e, double &dR, double &dE) const {
        if (kind == EOS_IDEAL) {
            dR = (gamma - 1.0) * e;
            dE = (gamma - 1.0) * rho;
        } else {
            dR = (gamma - 1.0) * (e - e0);
            dE = (gamma - 1.0) * rho;
        }
    }
    // ideal_gas.cpp:50-57 / stiffened_gas.cpp:121-128
    double energy_rP(double rho, double P) const {
        if (kind == EOS_IDEAL) return P / ((gamma - 1.0) * rho);
        return e0 + (P + gamma * P0) / ((gamma - 1.0) * rho);
    }
    // ideal_gas.cpp:76-78 / stiffened_gas.cpp:147-149
    double sound_speed_rP(double rho, double P) const {
        if (kind == EOS_IDEAL) return std::sqrt(gamma * P / rho);
        return std::sqrt(gamma * (P + P0) / rho);
    }
    // ideal_gas.cpp:104-106 / stiffened_gas.cpp:173-175
    double min_pressure() const {
        if (kind == EOS_IDEAL) return 0.0;
        return -P0;
    }
};

// ---------------------------------------------------------------------------
// States: zephyr/math/cfd/models.h:24-150, models.cpp:12-137.
struct PState {
    double density;
    V3 velocity;
    double pressure;
    double energy;
};
struct QState {  // also used for smf::Flux (same five components)
    double density;
    V3 momentum;
    double energy;
};
static inline void q_zero(QState &q) { q = {0.0, {0.0, 0.0, 0.0}, 0.0}; }

// models.cpp:27-32  PState(QState, eos)
static inline PState p_from_q(const QState &q, const Eos &eos) {
    PState z;
    z.density = q.density;
    z.velocity = {q.momentum.x / z.density, q.momentum.y / z.density, q.momentum.z / z.density};
    z.energy = q.energy / z.density - 0.5 * sqnorm(z.velocity);
    z.pressure = eos.pressure_re(z.density, z.energy);
    return z;
}
// models.cpp:85-89  QState(PState)
static inline QState q_from_p(const PState &z) {
    QState q;
    q.density = z.density;
    q.momentum = mul(z.density, z.velocity);
    q.energy = z.density * (z.energy + 0.5 * sqnorm(z.velocity));
    return q;
}
// models.cpp:131-137  Flux(PState)
static inline QState flux_from_p(const PState &z) {
    QState f;
    f.density = z.density * z.velocity.x;
    f.momentum.x = z.density * z.velocity.x * z.velocity.x + z.pressure;
    f.momentum.y = z.density * z.velocity.x * z.velocity.y;
    f.momentum.z = z.density * z.velocity.x * z.velocity.z;
    f.energy = (z.density * (z.energy + 0.5 * sqnorm(z.velocity)) + z.pressure) * z.velocity.x;
    return f;
}
// models.h:68  E() = e + v^2/2
static inline double p_E(const PState &z) { return z.energy + 0.5 * sqnorm(z.velocity); }

// models.cpp:58-63
static inline bool is_bad(const PState &z, const Eos &eos) {
    if (!std::isfinite(z.density) || !std::isfinite(z.pressure) || !std::isfinite(z.energy)) {
        return true;
    }
    return z.density <= 0.0 || z.pressure < eos.min_pressure();
}

// Rotation to the face frame: zephyr/math/cfd/rotate.cpp:7-41 (to_local),
// 43-77 (to_global).  Only the 2-D branch (normal.z == 0) is reachable.
static inline V3 rot_local(V3 v, V3 no) {
    V3 n = normalized(no);
    double c = n.x, s = n.y;
    // R = [c s 0; -s c 0; 0 0 1];  velocity = R * velocity
    return {c * v.x + s * v.y + 0.0 * v.z,
            -s * v.x + c * v.y + 0.0 * v.z,
            0.0 * v.x + 0.0 * v.y + 1.0 * v.z};
}
static inline V3 rot_global(V3 v, V3 no) {
    V3 n = normalized(no);
    double c = n.x, s = n.y;
    // R = [c -s 0; s c 0; 0 0 1]
    return {c * v.x + -s * v.y + 0.0 * v.z,
            s * v.x + c * v.y + 0.0 * v.z,
            0.0 * v.x + 0.0 * v.y + 1.0 * v.z};
}

// ---------------------------------------------------------------------------
// Numerical fluxes; values follow zephyr's `enum class Fluxes`
// (zephyr/math/cfd/flux/num_flux.h:11-21).
enum FluxKind {
    FLUX_GODUNOV = 0, FLUX_RUSANOV = 1, FLUX_HLL = 2, FLUX_HLLC = 3, FLUX_HLLC_M = 4, FLUX_HLLC_LM = 5,
    FLUX_CIR1 = 6, FLUX_CIR2 = 7
};

// zephyr/math/cfd/flux/hllc.cpp:23-83  HLLC::calc_flux (smf)
static QState hllc(const PState &zL, const PState &zR, const Eos &eos) {
    double c_L = eos.sound_speed_rP(zL.density, zL.pressure);
    double c_R = eos.sound_speed_rP(zR.density, zR.pressure);

    double S_L = std::min(zL.velocity.x - c_L, zR.velocity.x - c_R);
    double S_R = std::max(zL.velocity.x + c_L, zR.velocity.x + c_R);

    if (S_L >= 0.0) return flux_from_p(zL);
    if (S_R <= 0.0) return flux_from_p(zR);

    double a_L = zL.density * (S_L - zL.velocity.x);
    double a_R = zR.density * (S_R - zR.velocity.x);

    double S_C = (zL.pressure - zR.pressure + a_R * zR.velocity.x - a_L * zL.velocity.x) / (a_R - a_L);

    double rho_sL = a_L / (S_L - S_C);
    double rho_sR = a_R / (S_R - S_C);

    double E_sL = p_E(zL) + (S_C - zL.velocity.x) * (S_C + zL.pressure / a_L);
    double E_sR = p_E(zR) + (S_C - zR.velocity.x) * (S_C + zR.pressure / a_R);

    QState Q_sL{rho_sL, {rho_sL * S_C, rho_sL * zL.velocity.y, rho_sL * zL.velocity.z}, rho_sL * E_sL};
    QState Q_sR{rho_sR, {rho_sR * S_C, rho_sR * zR.velocity.y, rho_sR * zR.velocity.z}, rho_sR * E_sR};
    QState Q_L = q_from_p(zL), Q_R = q_from_p(zR);
    QState F_L = flux_from_p(zL), F_R = flux_from_p(zR);

    const double *fl = &F_L.density, *fr = &F_R.density;
    const double *qsl = &Q_sL.density, *qsr = &Q_sR.density;
    const double *ql = &Q_L.density, *qr = &Q_R.density;
    QState F;
    double *f = &F.density;
    double aSC = std::abs(S_C);
    for (int i = 0; i < 5; ++i) {
        f[i] = 0.5 * (fl[i] + fr[i] + S_L * (qsl[i] - ql[i]) + aSC * (qsl[i] - qsr[i]) +
                      S_R * (qsr[i] - qr[i]));
    }
    return F;
}

// zephyr/math/cfd/flux/hll.cpp:23-57  HLL::calc_flux (smf)
static QState hll(const PState &zL, const PState &zR, const Eos &eos) {
    const double u_L = zL.velocity.x;
    const double u_R = zR.velocity.x;
    double c_L = eos.sound_speed_rP(zL.density, zL.pressure);
    double c_R = eos.sound_speed_rP(zR.density, zR.pressure);
    // hll.cpp:11-17  min/max of three
    double S_L = std::min(u_L - c_L, std::min(u_R - c_R, 0.0));
    double S_R = std::max(u_L + c_L, std::max(u_R + c_R, 0.0));
    QState Q_L = q_from_p(zL), Q_R = q_from_p(zR);
    QState F_L = flux_from_p(zL), F_R = flux_from_p(zR);
    const double *fl = &F_L.density, *fr = &F_R.density, *ql = &Q_L.density, *qr = &Q_R.density;
    QState F;
    double *f = &F.density;
    double SLR = S_L * S_R;
    double den = S_R - S_L;
    for (int i = 0; i < 5; ++i) {
        f[i] = (S_R * fl[i] - S_L * fr[i] + SLR * (qr[i] - ql[i])) / den;
    }
    return F;
}

// zephyr/math/cfd/flux/rusanov.cpp:15-43  Rusanov::calc_flux (smf)
static QState rusanov(const PState &zL, const PState &zR, const Eos &eos) {
    const double u_L = zL.velocity.x;
    const double u_R = zR.velocity.x;
    double c_L = eos.sound_speed_rP(zL.density, zL.pressure);
    double c_R = eos.sound_speed_rP(zR.density, zR.pressure);
    // std::min / std::max of an initializer list: the first extreme element
    double S_L = u_L - c_L, S_R = u_L + c_L;
    if (u_R - c_R < S_L) S_L = u_R - c_R;
    if (0.0 < S_L) S_L = 0.0;
    if (S_R < u_R + c_R) S_R = u_R + c_R;
    if (S_R < 0.0) S_R = 0.0;
    double S = std::max(std::abs(S_L), S_R);
    QState Q_L = q_from_p(zL), Q_R = q_from_p(zR);
    QState F_L = flux_from_p(zL), F_R = flux_from_p(zR);
    const double *fl = &F_L.density, *fr = &F_R.density, *ql = &Q_L.density, *qr = &Q_R.density;
    QState F;
    double *f = &F.density;
    for (int i = 0; i < 5; ++i) f[i] = 0.5 * (fl[i] + fr[i]) + 0.5 * S * (ql[i] - qr[i]);
    return F;
}

// ---------------------------------------------------------------------------
// Exact Riemann solver for two stiffened gases, zephyr/math/solver/riemann.cpp
namespace riemann {

static inline double sq(double x) { return x * x; }  // riemann.cpp:12-14

static inline double eos_sound(double rho, double p, double g, double p0) {  // :17-19
    return std::sqrt(g * (p + p0) / rho);
}
static inline double eos_density(double p, double c, double g, double p0) {  // :22-24
    return g * (p + p0) / sq(c);
}
// acoustic initial guess (:32-45); the two-shock and two-rarefaction guesses
// of :47-61 are the same formula
static inline double p_init(double rL, double uL, double pL, double cL, double p0L, double rR, double uR, double pR,
                            double cR, double p0R) {
    double rcL = rL * cL, rcR = rR * cR;
    double P = (pL * rcR + pR * rcL + (uL - uR) * rcL * rcR) / (rcL + rcR);
    double Pmin = -std::min(p0L, p0R) + 1.0e-2 * std::min(pL + p0L, pR + p0R);
    return std::max(Pmin, P);
}
static inline double fK(double P, double rK, double pK, double cK, double gK, double p0K, double AK, double BK,
                        double GK) {  // :76-84
    if (P >= pK) return (P - pK) * std::sqrt(AK / (P + BK));
    return 2.0 * cK / (gK - 1.0) * (std::pow((P + p0K) / (pK + p0K), GK) - 1.0);
}
static inline double dfK(double P, double rK, double pK, double cK, double gK, double p0K, double AK, double BK,
                         double GK) {  // :86-94
    if (P >= pK) return (1.0 - (P - pK) / (2.0 * (P + BK))) * std::sqrt(AK / (P + BK));
    return std::pow((P + p0K) / (pK + p0K), GK - 1.0) / (rK * cK);
}

struct Sol {
    double rho, Uf, Pf, U, P;
    bool conv, vacuum, failed;
};

// contact_p (:118-236): Newton for the contact pressure and velocity
static void contact(double rL, double uL, double pL, double cL, double gL, double p0L, double rR, double uR,
                    double pR, double cR, double gR, double p0R, double &P_out, double &U_out, bool &conv,
                    bool &vacuum, bool &failed) {
    double AL = 2.0 / ((gL + 1) * rL), AR = 2.0 / ((gR + 1) * rR);
    double BL = (gL - 1.0) * pL / (gL + 1.0) + 2.0 * gL * p0L / (gL + 1.0);
    double BR = (gR - 1.0) * pR / (gR + 1.0) + 2.0 * gR * p0R / (gR + 1.0);
    double GL = (gL - 1.0) / (2.0 * gL), GR = (gR - 1.0) / (2.0 * gR);
    double p_dno = std::max(-p0L, -p0R);
    double p_min = std::min(pL, pR);
    double p_max = std::max(pL, pR);
    vacuum = failed = false;
    double f_dno = fK(p_dno, rL, pL, cL, gL, p0L, AL, BL, GL) + fK(p_dno, rR, pR, cR, gR, p0R, AR, BR, GR) + uR - uL;
    if (f_dno > 0.0) {
        vacuum = true;
        P_out = p_dno;
        U_out = 0.0;
        conv = true;
        return;
    }
    double P = 0.5 * (pL + pR);
    double f_min = fK(p_min, rL, pL, cL, gL, p0L, AL, BL, GL) + fK(p_min, rR, pR, cR, gR, p0R, AR, BR, GR) + uR - uL;
    if (f_min > 0.0) {
        P = p_init(rL, uL, pL, cL, p0L, rR, uR, pR, cR, p0R);
    } else {
        double f_max = fK(p_max, rL, pL, cL, gL, p0L, AL, BL, GL) + fK(p_max, rR, pR, cR, gR, p0R, AR, BR, GR) + uR -
                       uL;
        P = p_init(rL, uL, pL, cL, p0L, rR, uR, pR, cR, p0R);
        (void)f_max;
    }
    const int max_iterations = 50;
    double DP1 = 1.0e-5 * std::abs(pL - pR);
    double DP2 = 1.0e-12 * std::abs(std::max(pL + p0L, pR + p0R));
    double DP = std::max(DP1, DP2);
    double fL = 0.0, fR = 0.0, dfL, dfR, Pn = P;
    int counter = 0;
    for (; counter < max_iterations; ++counter) {
        fL = fK(P, rL, pL, cL, gL, p0L, AL, BL, GL);
        fR = fK(P, rR, pR, cR, gR, p0R, AR, BR, GR);
        dfL = dfK(P, rL, pL, cL, gL, p0L, AL, BL, GL);
        dfR = dfK(P, rR, pR, cR, gR, p0R, AR, BR, GR);
        Pn = P - (fL + fR + uR - uL) / (dfL + dfR);
        if (Pn < p_dno) Pn = (p_dno + P) / 2;
        if (std::abs(Pn - P) < DP) {
            if (counter > 3) break;
        }
        P = Pn;
    }
    conv = counter < max_iterations;
    // the reference throws when a non-converged solve is far off (:224-230)
    if (!conv && std::abs((P - Pn) / (P + Pn)) > 0.02) failed = true;
    P_out = P;
    U_out = 0.5 * (uL + uR + fR - fL);
}

// RiemannSolver::solve (:366-460): the state on the face x / t = 0
static Sol solve(double rL, double uL, double pL, double gL, double p0L, double rR, double uR, double pR, double gR,
                 double p0R) {
    double cL = eos_sound(rL, pL, gL, p0L);
    double cR = eos_sound(rR, pR, gR, p0R);
    Sol s{};
    double P, U;
    contact(rL, uL, pL, cL, gL, p0L, rR, uR, pR, cR, gR, p0R, P, U, s.conv, s.vacuum, s.failed);
    s.U = U;
    s.P = P;
    auto set = [&s](double rho, double Uf, double Pf) {
        s.rho = rho;
        s.Uf = Uf;
        s.Pf = Pf;
    };
    if (U > 0.0) {
        if (pL < P) {
            double D = uL + (P - pL) / (rL * (U - uL));  // shock_wave_speed (:239-241)
            if (D > 0.0) set(rL, uL, pL);
            else set(rL * (P - pL) / ((P - pL) - rL * sq(U - uL)), U, P);  // shock_wave_density (:246-248)
        } else {
            double DL1 = uL - cL;
            if (DL1 > 0.0) {
                set(rL, uL, pL);
            } else {
                double cl = cL + 0.5 * (gL - 1.0) * (uL - U);  // rarefaction_sound_L (:254-256)
                double DL2 = U - cl;
                if (DL2 < 0.0) {
                    set(eos_density(P, cl, gL, p0L), U, P);
                } else {
                    // the fan on the face, xi = 0 (:280-308)
                    double base = 2.0 / (gL + 1.0) + ((gL - 1.0) * (uL - 0.0)) / ((gL + 1.0) * cL);
                    set(rL * std::pow(base, 2.0 / (gL - 1.0)), ((gL - 1.0) * uL + 2.0 * (cL + 0.0)) / (gL + 1.0),
                        (pL + p0L) * std::pow(base, 2.0 * gL / (gL - 1.0)) - p0L);
                }
            }
        }
    } else {
        if (P > pR) {
            double D = uR + (P - pR) / (rR * (U - uR));
            if (D < 0.0) set(rR, uR, pR);
            else set(rR * (P - pR) / ((P - pR) - rR * sq(U - uR)), U, P);
        } else {
            double DR2 = uR + cR;
            if (DR2 < 0.0) {
                set(rR, uR, pR);
            } else {
                double cr = cR - 0.5 * (gR - 1.0) * (uR - U);  // rarefaction_sound_R (:262-264)
                double DR1 = U + cr;
                if (DR1 > 0.0) {
                    set(eos_density(P, cr, gR, p0R), U, P);
                } else {
                    double base = 2.0 / (gR + 1.0) - ((gR - 1.0) * (uR - 0.0)) / ((gR + 1.0) * cR);
                    set(rR * std::pow(base, 2.0 / (gR - 1.0)), ((gR - 1.0) * uR + 2.0 * (0.0 - cR)) / (gR + 1.0),
                        (pR + p0R) * std::pow(base, 2.0 * gR / (gR - 1.0)) - p0R);
                }
            }
        }
    }
    return s;
}

}  // namespace riemann

// IdealGas::stiffened_gas (ideal_gas.cpp:98-100) and StiffenedGas::
// stiffened_gas (stiffened_gas.cpp:169-171): the gas's own gamma and P0.
static inline void local_stiffened(const Eos &eos, double, double, double &g, double &P0) {
    g = eos.gamma;
    P0 = eos.kind == EOS_IDEAL ? 0.0 : eos.P0;
}

// zephyr/math/cfd/flux/godunov.cpp:16-32  Godunov::calc_flux (smf)
static QState godunov(const PState &zL, const PState &zR, const Eos &eos) {
    double gL, p0L, gR, p0R;
    local_stiffened(eos, zL.density, zL.pressure, gL, p0L);
    local_stiffened(eos, zR.density, zR.pressure, gR, p0R);
    riemann::Sol s = riemann::solve(zL.density, zL.velocity.x, zL.pressure, gL, p0L, zR.density, zR.velocity.x,
                                    zR.pressure, gR, p0R);
    PState z;
    z.density = s.rho;
    z.velocity = {s.Uf, s.U > 0.0 ? zL.velocity.y : zR.velocity.y, s.U > 0.0 ? zL.velocity.z : zR.velocity.z};
    z.pressure = s.Pf;
    z.energy = eos.energy_rP(s.rho, s.Pf);
    return flux_from_p(z);
}

// zephyr/math/cfd/flux/hllc.cpp:427-495  HLLC_LM::calc_flux (smf): the
// HLLC flux whose outer-wave terms are scaled by phi = sin(pi/2 min(Ma / 0.1, 1))
static QState hllc_lm(const PState &zL, const PState &zR, const Eos &eos) {
    double c_L = eos.sound_speed_rP(zL.density, zL.pressure);
    double c_R = eos.sound_speed_rP(zR.density, zR.pressure);
    double S_L = std::min(zL.velocity.x - c_L, zR.velocity.x - c_R);
    double S_R = std::max(zL.velocity.x + c_L, zR.velocity.x + c_R);
    if (S_L >= 0.0) return flux_from_p(zL);
    if (S_R <= 0.0) return flux_from_p(zR);
    double a_L = zL.density * (S_L - zL.velocity.x);
    double a_R = zR.density * (S_R - zR.velocity.x);
    double S_C = (zL.pressure - zR.pressure + a_R * zR.velocity.x - a_L * zL.velocity.x) / (a_R - a_L);
    double rho_sL = a_L / (S_L - S_C);
    double rho_sR = a_R / (S_R - S_C);
    double E_sL = p_E(zL) + (S_C - zL.velocity.x) * (S_C + zL.pressure / a_L);
    double E_sR = p_E(zR) + (S_C - zR.velocity.x) * (S_C + zR.pressure / a_R);
    QState Q_sL{rho_sL, {rho_sL * S_C, rho_sL * zL.velocity.y, rho_sL * zL.velocity.z}, rho_sL * E_sL};
    QState Q_sR{rho_sR, {rho_sR * S_C, rho_sR * zR.velocity.y, rho_sR * zR.velocity.z}, rho_sR * E_sR};
    QState Q_L = q_from_p(zL), Q_R = q_from_p(zR);
    QState F_L = flux_from_p(zL), F_R = flux_from_p(zR);
    double Ma_local = std::max(std::abs(zL.velocity.x / c_L), std::abs(zR.velocity.x / c_R));
    double xi = Ma_local / 0.1;
    double phi = xi > 1.0 ? 1.0 : std::sin(M_PI_2 * xi);
    const double *fl = &F_L.density, *fr = &F_R.density;
    const double *qsl = &Q_sL.density, *qsr = &Q_sR.density;
    const double *ql = &Q_L.density, *qr = &Q_R.density;
    QState F;
    double *f = &F.density;
    double aSC = std::abs(S_C);
    for (int i = 0; i < 5; ++i) {
        f[i] = 0.5 * (fl[i] + fr[i] + phi * S_L * (qsl[i] - ql[i]) + aSC * (qsl[i] - qsr[i]) +
                      phi * S_R * (qsr[i] - qr[i]));
    }
    return F;
}

// zephyr/math/cfd/flux/hllc.cpp:499-570  HLLC_M::calc_flux (smf): the
// tangential velocities are averaged across the contact too
static QState hllc_m(const PState &zL, const PState &zR, const Eos &eos) {
    double c_L = eos.sound_speed_rP(zL.density, zL.pressure);
    double c_R = eos.sound_speed_rP(zR.density, zR.pressure);
    double S_L = std::min(zL.velocity.x - c_L, zR.velocity.x - c_R);
    double S_R = std::max(zL.velocity.x + c_L, zR.velocity.x + c_R);
    if (S_L >= 0.0) return flux_from_p(zL);
    if (S_R <= 0.0) return flux_from_p(zR);
    double a_L = zL.density * (S_L - zL.velocity.x);
    double a_R = zR.density * (S_R - zR.velocity.x);
    double S_C = (zL.pressure - zR.pressure + a_R * zR.velocity.x - a_L * zL.velocity.x) / (a_R - a_L);
    double V_C = (a_R * zR.velocity.y - a_L * zL.velocity.y) / (a_R - a_L);
    double W_C = (a_R * zR.velocity.z - a_L * zL.velocity.z) / (a_R - a_L);
    double rho_sL = a_L / (S_L - S_C);
    double rho_sR = a_R / (S_R - S_C);
    double E_sL = p_E(zL) + (S_C - zL.velocity.x) * (S_C + zL.pressure / a_L);
    double E_sR = p_E(zR) + (S_C - zR.velocity.x) * (S_C + zR.pressure / a_R);
    double v_L2 = std::pow(zL.velocity.y, 2) + std::pow(zL.velocity.z, 2);
    double v_R2 = std::pow(zR.velocity.y, 2) + std::pow(zR.velocity.z, 2);
    E_sL += 0.5 * ((a_R * v_R2 - a_L * v_L2) / (a_R - a_L) - v_L2);
    E_sR += 0.5 * ((a_R * v_R2 - a_L * v_L2) / (a_R - a_L) - v_R2);
    QState Q_sL{rho_sL, {rho_sL * S_C, rho_sL * V_C, rho_sL * W_C}, rho_sL * E_sL};
    QState Q_sR{rho_sR, {rho_sR * S_C, rho_sR * V_C, rho_sR * W_C}, rho_sR * E_sR};
    QState Q_L = q_from_p(zL), Q_R = q_from_p(zR);
    QState F_L = flux_from_p(zL), F_R = flux_from_p(zR);
    const double *fl = &F_L.density, *fr = &F_R.density;
    const double *qsl = &Q_sL.density, *qsr = &Q_sR.density;
    const double *ql = &Q_L.density, *qr = &Q_R.density;
    QState F;
    double *f = &F.density;
    double aSC = std::abs(S_C);
    for (int i = 0; i < 5; ++i) {
        f[i] = 0.5 * (fl[i] + fr[i] + S_L * (qsl[i] - ql[i]) + aSC * (qsl[i] - qsr[i]) +
                      S_R * (qsr[i] - qr[i]));
    }
    return F;
}

// Dense products in the evaluation order of the Eigen stand-in the reference
// is built with here: c_ij = a_i0 b_0j, then c_ij += a_ik b_kj for k = 1, 2, ...
template <int R, int K, int C>
static void matmul(const double (&a)[R][K], const double (&b)[K][C], double (&c)[R][C]) {
    for (int i = 0; i < R; ++i)
        for (int j = 0; j < C; ++j) {
            double acc = a[i][0] * b[0][j];
            for (int k = 1; k < K; ++k) acc = acc + a[i][k] * b[k][j];
            c[i][j] = acc;
        }
}

// CIR face state: zE = (zL + zR) / 2 component by component, energy from
// (density, pressure) (cir.cpp:20-30, 129-137)
static PState cir_face_state(const PState &zL, const PState &zR, const Eos &eos) {
    PState zE;
    zE.density = 0.5 * (zL.density + zR.density);
    zE.velocity = {0.5 * (zL.velocity.x + zR.velocity.x), 0.5 * (zL.velocity.y + zR.velocity.y),
                   0.5 * (zL.velocity.z + zR.velocity.z)};
    zE.pressure = 0.5 * (zL.pressure + zR.pressure);
    zE.energy = eos.energy_rP(zE.density, zE.pressure);
    return zE;
}

// zephyr/math/cfd/flux/cir.cpp:20-125  CIR1::calc_flux: Courant-Isaacson-Rees
// flux with |A| = R |Lambda| L of the Jacobian at the averaged state
static QState cir1(const PState &zL, const PState &zR, const Eos &eos) {
    const PState zE = cir_face_state(zL, zR, eos);
    double dR, dE;
    eos.pressure_re_deriv(zE.density, zE.energy, dR, dE);
    const double rho = zE.density, u = zE.velocity.x, v = zE.velocity.y, w = zE.velocity.z;
    const double p = zE.pressure, eps = zE.energy;
    const double u2 = u * u, v2 = v * v, w2 = w * w;
    const double q2 = u2 + v2 + w2;
    const double E = rho * (eps + 0.5 * q2);
    const double c = eos.sound_speed_rP(rho, p);
    const double c2 = c * c;
    const double h = (E + p) / rho;
    const double b = dE / rho;
    const double T = b * (q2 - h) + c2;
    const double lam[5] = {std::abs(u - c), std::abs(u), std::abs(u), std::abs(u), std::abs(u + c)};
    double OmR[5][5] = {{1, 0, 0, 1, 1},
                        {u - c, 0, 0, u, u + c},
                        {v, 1, 0, v, v},
                        {w, 0, 1, w, w},
                        {h - u * c, v, w, h - c2 / b, h + u * c}};
    double OmL[5][5] = {{T + u * c, -b * u - c, -b * v, -b * w, b},
                        {-2 * v * c2, 0, 2 * c2, 0, 0},
                        {-2 * w * c2, 0, 0, 2 * c2, 0},
                        {2 * b * (h - q2), 2 * b * u, 2 * b * v, 2 * b * w, -2 * b},
                        {T - u * c, -b * u + c, -b * v, -b * w, b}};
    const double den = 2.0 * c2;
    for (auto &row : OmL)
        for (double &x : row) x /= den;
    double RL[5][5], A[5][5];
    for (int i = 0; i < 5; ++i)
        for (int j = 0; j < 5; ++j) RL[i][j] = OmR[i][j] * lam[j];
    matmul(RL, OmL, A);
    const QState qL = q_from_p(zL), qR = q_from_p(zR), fL = flux_from_p(zL), fR = flux_from_p(zR);
    const double *ql = &qL.density, *qr = &qR.density, *fl = &fL.density, *fr = &fR.density;
    double dq[5][1], hA[5][5], Adq[5][1];
    for (int k = 0; k < 5; ++k) dq[k][0] = ql[k] - qr[k];
    for (int i = 0; i < 5; ++i)
        for (int j = 0; j < 5; ++j) hA[i][j] = 0.5 * A[i][j];
    matmul(hA, dq, Adq);
    QState F;
    double *f = &F.density;
    for (int k = 0; k < 5; ++k) f[k] = 0.5 * (fl[k] + fr[k]) + Adq[k][0];
    return F;
}

// zephyr/math/cfd/flux/cir.cpp:129-234  CIR2::calc_flux: the same with the
// pressure as a sixth variable (the consistency check of cir.cpp:180-211,
// which throws when the decomposition is off by more than 1e-10, is not
// restated)
static QState cir2(const PState &zL, const PState &zR, const Eos &eos) {
    const PState zE = cir_face_state(zL, zR, eos);
    const double rho = zE.density, u = zE.velocity.x, v = zE.velocity.y, w = zE.velocity.z;
    const double p = zE.pressure, eps = zE.energy;
    const double u2 = u * u, v2 = v * v, w2 = w * w;
    const double q2 = u2 + v2 + w2;
    const double E = rho * (eps + 0.5 * q2);
    const double c = eos.sound_speed_rP(rho, p);
    const double c2 = c * c;
    const double h = (E + p) / rho;
    const double lam[6] = {std::abs(u - c), std::abs(u), std::abs(u), std::abs(u), std::abs(u + c), std::abs(u)};
    double OmR[5][6] = {{1, 0, 0, 0, 1, 1},
                        {u - c, 0, 0, 0, u + c, u},
                        {v, 1, 0, 0, v, 0},
                        {w, 0, 1, 0, w, 0},
                        {h - u * c, 0, 0, 1, h + u * c, 0}};
    double OmL[6][6] = {{u / (2 * c), -1 / (2 * c), 0, 0, 0, 1 / (2 * c2)},
                        {0, 0, 1, 0, 0, -v / c2},
                        {0, 0, 0, 1, 0, -w / c2},
                        {u2, -u, 0, 0, 1, -h / c2},
                        {-u / (2 * c), 1 / (2 * c), 0, 0, 0, 1 / (2 * c2)},
                        {1, 0, 0, 0, 0, -1 / c2}};
    double RL[5][6], A[5][6];
    for (int i = 0; i < 5; ++i)
        for (int j = 0; j < 6; ++j) RL[i][j] = OmR[i][j] * lam[j];
    matmul(RL, OmL, A);
    const QState qL = q_from_p(zL), qR = q_from_p(zR), fL = flux_from_p(zL), fR = flux_from_p(zR);
    const double *ql = &qL.density, *qr = &qR.density, *fl = &fL.density, *fr = &fR.density;
    double dq[6][1], hA[5][6], Adq[5][1];
    for (int k = 0; k < 5; ++k) dq[k][0] = ql[k] - qr[k];
    dq[5][0] = zL.pressure - zR.pressure;
    for (int i = 0; i < 5; ++i)
        for (int j = 0; j < 6; ++j) hA[i][j] = 0.5 * A[i][j];
    matmul(hA, dq, Adq);
    QState F;
    double *f = &F.density;
    for (int k = 0; k < 5; ++k) f[k] = 0.5 * (fl[k] + fr[k]) + Adq[k][0];
    return F;
}

static inline QState num_flux(int kind, const PState &zL, const PState &zR, const Eos &eos) {
    switch (kind) {
        case FLUX_GODUNOV: return godunov(zL, zR, eos);
        case FLUX_RUSANOV: return rusanov(zL, zR, eos);
        case FLUX_HLL: return hll(zL, zR, eos);
        case FLUX_HLLC_M: return hllc_m(zL, zR, eos);
        case FLUX_HLLC_LM: return hllc_lm(zL, zR, eos);
        case FLUX_CIR1: return cir1(zL, zR, eos);
        case FLUX_CIR2: return cir2(zL, zR, eos);
        default: return hllc(zL, zR, eos);
    }
}

// ---------------------------------------------------------------------------
// Limiters, binary form phi(a, b): zephyr/math/cfd/limiter.cxx:15-153.
enum LimKind {
    LIM_NONE = 0, LIM_UNIT, LIM_MINMOD, LIM_MC, LIM_VANLEER, LIM_VANALBADA1,
    LIM_VANALBADA2, LIM_CHARM, LIM_HCUS, LIM_HQUICK, LIM_KOREN, LIM_SMART, LIM_SUPERBEE
};
static inline double sqr(double x) { return x * x; }
static inline double lim_MC1(double r) {  // limiter.cxx:45-48
    if (std::isnan(r)) return 0.0;
    return std::max(0.0, std::min(2 * r, std::min(0.5 * (1.0 + r), 2.0)));
}
static inline double lim_koren1(double r) {  // limiter.cxx:128-131
    if (std::isnan(r)) return 0.0;
    return std::max(0.0, std::min(2 * r, std::min(2.0, (1 + 2 * r) / 3.0)));
}
static inline double lim_smart1(double r) {  // limiter.cxx:137-140
    if (std::isnan(r)) return 0.0;
    return std::max(0.0, std::min(2.0 * r, std::min(0.25 + 0.75 * r, 4.0)));
}
static inline double lim_superbee1(double r) {  // limiter.cxx:146-149
    if (std::isnan(r)) return 0.0;
    return std::max(0.0, std::min(std::min(2 * r, 1.0), std::min(r, 2.0)));
}
static double limiter2(int kind, double a, double b) {
    switch (kind) {
        case LIM_NONE: return 0.0;                                   // 23-25
        case LIM_UNIT: return 1.0;                                   // 31-33
        case LIM_MINMOD:                                             // 40-43
            if (a * b <= 0.0) return 0.0;
            return std::min(a / b, 1.0);
        case LIM_MC: return lim_MC1(a / b);                          // 50-52
        case LIM_VANLEER:                                            // 62-67
            if (a * b < 0.0) return 0.0;
            if (a == 0.0) return 0.0;
            return 2 * std::abs(a) / (std::abs(a) + std::abs(b));
        case LIM_VANALBADA1:                                         // 77-82
            if (a * b <= 0.0) return 0.0;
            if (b == 0.0) return 1.0;
            return a * (a + b) / (sqr(a) + sqr(b));
        case LIM_VANALBADA2: {                                       // 92-96
            if (a * b <= 0.0) return 0.0;
            double eps = 10e-6;
            return (2.0 * a * b + eps) / (sqr(a) + sqr(b) + eps);
        }
        case LIM_CHARM:                                              // 103-106
            if (a * b <= 0.0) return 0.0;
            return a * (3 * a + b) / sqr(a + b);
        case LIM_HCUS:                                               // 113-116
            if (a * b <= 0.0) return 0.0;
            return (3.0 * a) / (a + 2.0 * b);
        case LIM_HQUICK:                                             // 123-126
            if (a * b <= 0.0) return 0.0;
            return (4.0 * a) / (a + 3.0 * b);
        case LIM_KOREN: return lim_koren1(a / b);                    // 133-135
        case LIM_SMART: return lim_smart1(a / b);                    // 142-144
        case LIM_SUPERBEE: return lim_superbee1(a / b);              // 151-153
        default: return 0.0;
    }
}

// ---------------------------------------------------------------------------
// Mesh: the 2-D part of AmrCells/AmrFaces (zephyr/mesh/euler/amr_cells.h:49-104,
// amr_faces.h:83-154) with 8 face slots per cell (face_begin = 8 * ic) and
// 9 mapping vertices per cell.
enum Boundary { B_UNDEFINED = -1, B_INNER = 0, B_WALL = 1, B_ZOE = 2, B_PERIODIC = 3, B_FUNCTION = 4 };

struct Mesh {
    int n_cells = 0;
    int nx = 0, ny = 0;  // a rectangle's cells per axis (0 for meshes built from arrays)
    // cells
    std::vector<V3> center;
    std::vector<double> volume;
    std::vector<V3> verts;  // 9 per cell, SqQuad order (quad.h:187-190: vs<i,j> = verts[3j+i+4])
    std::vector<int> level, flag, b_idx, z_idx;
    // faces (8 slots per cell)
    std::vector<int> boundary;
    std::vector<int> adj;  // neighbour cell index (self index on boundary slots)
    std::vector<V3> fnormal, fcenter;
    std::vector<double> farea;
    std::vector<double> incircle;  // given diameters (meshes built from arrays)
};

// zephyr/mesh/euler/amr_cells_gen.cpp:128-281  AmrCells(const Rectangle&),
// with SqQuad(v00, v01, v10, v11) from zephyr/geom/primitives/quad.cpp:429-436.
// bounds: left, right, bottom, top; PERIODIC on a side makes both sides of
// that axis periodic (rectangle.cpp:182-189).
static void make_rectangle(Mesh &m, int nx, int ny, double x_min, double x_max, double y_min,
                           double y_max, const int bounds_in[4]) {
    int bounds[4] = {bounds_in[0], bounds_in[1], bounds_in[2], bounds_in[3]};
    const bool x_period = bounds[0] == B_PERIODIC || bounds[1] == B_PERIODIC;
    const bool y_period = bounds[2] == B_PERIODIC || bounds[3] == B_PERIODIC;
    if (x_period) bounds[0] = bounds[1] = B_PERIODIC;
    if (y_period) bounds[2] = bounds[3] = B_PERIODIC;
    const double hx = (x_max - x_min) / nx;
    const double hy = (y_max - y_min) / ny;

    auto get_index = [ny](int i, int j) { return i * ny + j; };
    auto get_vertex = [&](int i, int j) -> V3 {
        return {x_min + ((x_max - x_min) * i) / nx, y_min + ((y_max - y_min) * j) / ny, 0.0};
    };
    auto neib_index = [&](int i, int j, int side) -> int {
        if (side == 0) return i == 0 && !x_period ? get_index(i, j) : get_index((i - 1 + nx) % nx, j);
        if (side == 1) return i == nx - 1 && !x_period ? get_index(i, j) : get_index((i + 1 + nx) % nx, j);
        if (side == 2) return j == 0 && !y_period ? get_index(i, j) : get_index(i, (j - 1 + ny) % ny);
        return j == ny - 1 && !y_period ? get_index(i, j) : get_index(i, (j + 1 + ny) % ny);
    };

    const int N = nx * ny;
    m.n_cells = N;
    m.nx = nx;
    m.ny = ny;
    m.center.resize(N);
    m.volume.resize(N);
    m.verts.resize(9 * (size_t)N);
    m.level.assign(N, 0);
    m.flag.assign(N, 0);
    m.b_idx.resize(N);
    m.z_idx.assign(N, 0);
    m.boundary.assign(8 * (size_t)N, B_UNDEFINED);
    m.adj.assign(8 * (size_t)N, -1);
    m.fnormal.assign(8 * (size_t)N, V3{0, 0, 0});
    m.fcenter.assign(8 * (size_t)N, V3{0, 0, 0});
    m.farea.assign(8 * (size_t)N, 0.0);

    for (int ic = 0; ic < N; ++ic) {
        int i = ic / ny, j = ic % ny;
        m.b_idx[ic] = ic;
        V3 v00 = get_vertex(i, j), v01 = get_vertex(i + 1, j);
        V3 v10 = get_vertex(i, j + 1), v11 = get_vertex(i + 1, j + 1);
        V3 *q = &m.verts[9 * (size_t)ic];
        q[0] = v00;
        q[1] = mul(0.5, add(v00, v01));
        q[2] = v01;
        q[3] = mul(0.5, add(v00, v10));
        q[4] = mul(0.25, add(add(add(v00, v01), v10), v11));
        q[5] = mul(0.5, add(v01, v11));
        q[6] = v10;
        q[7] = mul(0.5, add(v10, v11));
        q[8] = v11;

        m.center[ic] = q[4];  // vs<0,0>
        m.volume[ic] = hx * hy;

        size_t f = 8 * (size_t)ic;
        m.boundary[f + 0] = i > 0 ? B_INNER : bounds[0];
        m.boundary[f + 1] = i < nx - 1 ? B_INNER : bounds[1];
        m.boundary[f + 2] = j > 0 ? B_INNER : bounds[2];
        m.boundary[f + 3] = j < ny - 1 ? B_INNER : bounds[3];
        for (int s = 0; s < 4; ++s) m.adj[f + s] = neib_index(i, j, s);
        m.fnormal[f + 0] = {-1.0, -0.0, -0.0};  // -Vector3d::UnitX()
        m.fnormal[f + 1] = {1.0, 0.0, 0.0};
        m.fnormal[f + 2] = {-0.0, -1.0, -0.0};  // -Vector3d::UnitY()
        m.fnormal[f + 3] = {0.0, 1.0, 0.0};
        m.fcenter[f + 0] = q[3];  // vs<-1,0>
        m.fcenter[f + 1] = q[5];  // vs<+1,0>
        m.fcenter[f + 2] = q[1];  // vs<0,-1>
        m.fcenter[f + 3] = q[7];  // vs<0,+1>
        m.farea[f + 0] = hy;
        m.farea[f + 1] = hy;
        m.farea[f + 2] = hx;
        m.farea[f + 3] = hx;
    }
}

// amr_faces.h:157-161
static inline bool is_boundary(int flag) {
    return flag != B_INNER && flag != B_PERIODIC && flag != B_UNDEFINED;
}
// amr_faces.h:197-199
static inline V3 symm_point(const Mesh &m, size_t f, V3 p) {
    return add(p, mul(2.0 * dot(sub(m.fcenter[f], p), m.fnormal[f]), m.fnormal[f]));
}
// amr_cells.cpp:107-116  incircle_diameter (adaptive, 2-D)
static inline double incircle_diameter(const Mesh &m, int ic) {
    if (!m.incircle.empty()) return m.incircle[ic];
    const V3 *q = &m.verts[9 * (size_t)ic];
    return std::sqrt(std::min(sqnorm(sub(q[5], q[3])), sqnorm(sub(q[7], q[1]))));
}

// sm_fluid.cpp:69-79  boundary_value
static inline PState boundary_value(const PState &zc, V3 normal, int flag) {
    if (flag != B_WALL) return zc;
    PState zn = zc;
    V3 Vn = mul(dot(zc.velocity, normal), normal);
    zn.velocity = sub(zc.velocity, mul(2.0, Vn));
    return zn;
}

// ---------------------------------------------------------------------------
// Parallel loops: the reference's utils::threads::for_each splits the range
// into n_threads * 10 tasks (threads.h:18-21); the split does not change any
// result here (each cell writes only itself).
template <class F>
static void parallel_cells(int n, int n_threads, F &&func) {
    if (n_threads <= 1 || n < 1000) {
        func(0, n);
        return;
    }
    int n_tasks = n_threads * 10;
    std::atomic<int> next{0};
    int chunk = (n + n_tasks - 1) / n_tasks;
    std::vector<std::thread> pool;
    for (int t = 0; t < n_threads; ++t) {
        pool.emplace_back([&]() {
            for (;;) {
                int k = next.fetch_add(1);
                int b = k * chunk;
                if (b >= n) break;
                func(b, std::min(n, b + chunk));
            }
        });
    }
    for (auto &th : pool) th.join();
}

// ---------------------------------------------------------------------------
// SmFluid: zephyr/math/solver/sm_fluid.{h,cpp}.
enum Scheme { SCHEME_REF = 0, SCHEME_HEUN = 1 };

struct Solver {
    Mesh *mesh;
    Eos eos;
    int flux_kind = FLUX_HLLC;
    int limiter = LIM_MC;
    int acc = 1;
    int scheme = SCHEME_REF;
    double CFL = 0.5;
    double dt = NAN;
    double max_dt = std::numeric_limits<double>::max();
    int n_threads = 1;

    std::vector<PState> init, half, next, d_dx, d_dy, d_dz;
    std::vector<int> wait, wait_snap;
    std::vector<QState> qstar;  // Heun stage value (extension mode)

    void resize() {
        size_t n = mesh->n_cells;
        init.resize(n);
        half.resize(n);
        next.resize(n);
        d_dx.resize(n);
        d_dy.resize(n);
        d_dz.resize(n);
        wait.assign(n, 0);
        wait_snap.assign(n, 0);
    }

    // sm_fluid.cpp:104-114  compute_dt
    void compute_dt() {
        const Mesh &m = *mesh;
        // threads::min (threads.h:95-110) starts from numeric_limits::max();
        // the minimum does not depend on the order of the cells.
        double res = std::numeric_limits<double>::max();
        for (int ic = 0; ic < m.n_cells; ++ic) {
            double c = eos.sound_speed_rP(init[ic].density, init[ic].pressure);
            double v = incircle_diameter(m, ic) / (norm(init[ic].velocity) + c);
            res = std::min(res, v);
        }
        double d = std::min(CFL * res, max_dt);
        dt = d;
    }

    // gradient.h:226-282  LSM, then gradient.h:412-474  limiting; stored as in
    // sm_fluid.cpp:116-125  compute_grad.
    void grad_cell(const std::vector<PState> &z, int ic, PState &gx, PState &gy, PState &gz) const {
        const Mesh &m = *mesh;
        const double w0 = 1.0;  // cell.dim() < 3
        const PState zc = z[ic];
        const V3 cell_c = m.center[ic];
        const double *zcp = &zc.density;

        double Fx[6] = {0}, Fy[6] = {0}, Fz[6] = {0};
        double A[3][3] = {{0}};
        for (int s = 0; s < 8; ++s) {
            size_t f = 8 * (size_t)ic + s;
            int flag = m.boundary[f];
            if (flag == B_UNDEFINED) continue;
            V3 normal = m.fnormal[f];
            PState zn = !is_boundary(flag) ? z[m.adj[f]] : boundary_value(zc, normal, flag);
            V3 dr = sub(flag == B_INNER ? m.center[m.adj[f]] : symm_point(m, f, cell_c), cell_c);
            V3 drn = mul(dot(dr, normal), normal);
            double w = w0 * m.farea[f] / std::pow(norm(drn), 3);
            V3 wd = mul(w, drn);
            const double wdv[3] = {wd.x, wd.y, wd.z}, drv[3] = {dr.x, dr.y, dr.z};
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) A[a][b] += wdv[a] * drv[b];
            const double *znp = &zn.density;
            for (int k = 0; k < 6; ++k) {
                double dF = znp[k] - zcp[k];
                Fx[k] += w * dF * drn.x;
                Fy[k] += w * dF * drn.y;
                Fz[k] += w * dF * drn.z;
            }
        }
        double B[3][3];
        fix_and_invert(A, B);
        double g0x[6], g0y[6], g0z[6];
        for (int k = 0; k < 6; ++k) {
            g0x[k] = B[0][0] * Fx[k] + B[0][1] * Fy[k] + B[0][2] * Fz[k];
            g0y[k] = B[1][0] * Fx[k] + B[1][1] * Fy[k] + B[1][2] * Fz[k];
            g0z[k] = B[2][0] * Fx[k] + B[2][1] * Fy[k] + B[2][2] * Fz[k];
        }

        // limiting (gradient.h:412-474)
        double Lx[6] = {0}, Ly[6] = {0}, Lz[6] = {0};
        double A2[3][3] = {{0}};
        for (int s = 0; s < 8; ++s) {
            size_t f = 8 * (size_t)ic + s;
            int flag = m.boundary[f];
            if (flag == B_UNDEFINED) continue;
            V3 normal = m.fnormal[f];
            PState zn = !is_boundary(flag) ? z[m.adj[f]] : boundary_value(zc, normal, flag);
            V3 dr = sub(flag == B_INNER ? m.center[m.adj[f]] : symm_point(m, f, cell_c), cell_c);
            V3 drn = mul(dot(dr, normal), normal);
            double w = w0 * m.farea[f] / std::pow(norm(drn), 3);
            V3 wd = mul(w, drn);
            const double wdv[3] = {wd.x, wd.y, wd.z}, drv[3] = {dr.x, dr.y, dr.z};
            for (int a = 0; a < 3; ++a)
                for (int b = 0; b < 3; ++b) A2[a][b] += wdv[a] * drv[b];
            const double *znp = &zn.density;
            for (int k = 0; k < 6; ++k) {
                double dF_p = znp[k] - zcp[k];
                double du_n = g0x[k] * dr.x + g0y[k] * dr.y + g0z[k] * dr.z;
                double dF_m = 2.0 * du_n - dF_p;
                double dF_lim = limiter2(limiter, dF_m, dF_p) * dF_p;
                Lx[k] += w * dF_lim * drn.x;
                Ly[k] += w * dF_lim * drn.y;
                Lz[k] += w * dF_lim * drn.z;
            }
        }
        double B2[3][3];
        fix_and_invert(A2, B2);
        double *ox = &gx.density, *oy = &gy.density, *oz = &gz.density;
        for (int k = 0; k < 6; ++k) {
            ox[k] = B2[0][0] * Lx[k] + B2[0][1] * Ly[k] + B2[0][2] * Lz[k];
            oy[k] = B2[1][0] * Lx[k] + B2[1][1] * Ly[k] + B2[1][2] * Lz[k];
            oz[k] = B2[2][0] * Lx[k] + B2[2][1] * Ly[k] + B2[2][2] * Lz[k];
        }
    }

    // gradient.h:267-275: 2-D fix of A(2,2) (and the 1-D fix of A(1,1)),
    // then the 3x3 inverse.  The inverse restates Eigen's cofactor formula
    // for fixed 3x3 matrices (Eigen/src/LU/InverseImpl.h, compute_inverse
    // size 3): column-0 cofactors, det = their dot with column 0,
    // invdet = 1/det, inverse = adjugate * invdet.
    static double cof(const double m[3][3], int i, int j) {
        int i1 = (i + 1) % 3, i2 = (i + 2) % 3, j1 = (j + 1) % 3, j2 = (j + 2) % 3;
        return m[i1][j1] * m[i2][j2] - m[i1][j2] * m[i2][j1];
    }
    static void fix_and_invert(double A[3][3], double B[3][3]) {
        if (std::abs(A[2][2]) < 1e-8) {
            A[2][2] = 1.0;
            if (std::abs(A[1][1]) < 1e-8) A[1][1] = 1.0;
        }
        double c0 = cof(A, 0, 0), c1 = cof(A, 1, 0), c2 = cof(A, 2, 0);
        double det = c0 * A[0][0] + c1 * A[1][0] + c2 * A[2][0];
        double invdet = 1.0 / det;
        double c01 = cof(A, 0, 1) * invdet;
        double c11 = cof(A, 1, 1) * invdet;
        double c02 = cof(A, 0, 2) * invdet;
        B[1][2] = cof(A, 2, 1) * invdet;
        B[2][1] = cof(A, 1, 2) * invdet;
        B[2][2] = cof(A, 2, 2) * invdet;
        B[1][0] = c01;
        B[1][1] = c11;
        B[2][0] = c02;
        B[0][0] = c0 * invdet;
        B[0][1] = c1 * invdet;
        B[0][2] = c2 * invdet;
    }

    void compute_grad(const std::vector<PState> &z) {
        parallel_cells(mesh->n_cells, n_threads, [&](int b, int e) {
            for (int ic = b; ic < e; ++ic) grad_cell(z, ic, d_dx[ic], d_dy[ic], d_dz[ic]);
        });
    }

    // sm_fluid.cpp:127-174  fluxes (first order)
    void fluxes() {
        const Mesh &m = *mesh;
        parallel_cells(m.n_cells, n_threads, [&](int b, int e) {
            for (int ic = b; ic < e; ++ic) {
                PState z_c = init[ic];
                QState q_c = q_from_p(z_c);
                QState flux;
                q_zero(flux);
                for (int s = 0; s < 8; ++s) {
                    size_t f = 8 * (size_t)ic + s;
                    int flag = m.boundary[f];
                    if (flag == B_UNDEFINED) continue;
                    V3 normal = m.fnormal[f];
                    PState z_n = !is_boundary(flag) ? init[m.adj[f]] : boundary_value(z_c, normal, flag);
                    PState zm = z_c, zp = z_n;
                    zm.velocity = rot_local(zm.velocity, normal);
                    zp.velocity = rot_local(zp.velocity, normal);
                    QState lf = num_flux(flux_kind, zm, zp, eos);
                    lf.momentum = rot_global(lf.momentum, normal);
                    accumulate(flux, lf, m.farea[f]);
                }
                update(q_c, dt / m.volume[ic], flux);
                next[ic] = p_from_q(q_c, eos);
            }
        });
    }

    static inline void accumulate(QState &acc, const QState &lf, double area) {
        double *a = &acc.density;
        const double *l = &lf.density;
        for (int k = 0; k < 5; ++k) a[k] += l[k] * area;
    }
    static inline void update(QState &q, double coef, const QState &flux) {
        double *qq = &q.density;
        const double *fl = &flux.density;
        for (int k = 0; k < 5; ++k) qq[k] -= coef * fl[k];
    }

    // face_extra.h:135-177  FaceExtraDirect: du = grad . (x_face - x_centre)
    static inline PState extrap(const PState &u, const PState &gx, const PState &gy, const PState &gz,
                                V3 dr) {
        PState o;
        const double *uu = &u.density, *x = &gx.density, *y = &gy.density, *zz = &gz.density;
        double *oo = &o.density;
        for (int k = 0; k < 6; ++k) oo[k] = uu[k] + (x[k] * dr.x + y[k] * dr.y + zz[k] * dr.z);
        return o;
    }

    // sm_fluid.cpp:176-253  fluxes_stage1 (predictor, half step)
    void fluxes_stage1() {
        const Mesh &m = *mesh;
        parallel_cells(m.n_cells, n_threads, [&](int b, int e) {
            for (int ic = b; ic < e; ++ic) {
                if (wait[ic] > 0) {
                    half[ic] = init[ic];
                    continue;
                }
                V3 cell_c = m.center[ic];
                PState z_c = init[ic];
                QState q_c = q_from_p(z_c);
                QState flux;
                q_zero(flux);
                for (int s = 0; s < 8; ++s) {
                    size_t f = 8 * (size_t)ic + s;
                    int flag = m.boundary[f];
                    if (flag == B_UNDEFINED) continue;
                    V3 normal = m.fnormal[f];
                    V3 face_c = m.fcenter[f];
                    PState zm = extrap(z_c, d_dx[ic], d_dy[ic], d_dz[ic], sub(face_c, cell_c));
                    zm.energy = eos.energy_rP(zm.density, zm.pressure);
                    if (is_bad(zm, eos)) zm = z_c;
                    zm.velocity = rot_local(zm.velocity, normal);
                    QState lf = flux_from_p(zm);
                    lf.momentum = rot_global(lf.momentum, normal);
                    accumulate(flux, lf, m.farea[f]);
                }
                update(q_c, 0.5 * dt / m.volume[ic], flux);
                half[ic] = p_from_q(q_c, eos);
                if (is_bad(half[ic], eos)) half[ic] = z_c;
            }
        });
    }

    // Face flux of stage 2 (sm_fluid.cpp:271-341) for cell ic and slot f:
    // reconstruct from z (gradients of z) at states zh, Riemann-solve.
    inline QState stage2_face(int ic, size_t f, const std::vector<PState> &z,
                              const std::vector<PState> &zh, const std::vector<int> &wt) const {
        const Mesh &m = *mesh;
        int flag = m.boundary[f];
        V3 normal = m.fnormal[f];
        V3 face_c = m.fcenter[f];
        V3 cell_c = m.center[ic];
        int in = m.adj[f];  // face.neib(): the cell itself on boundary slots
        PState z_c = z[ic], z_ch = zh[ic];
        PState z_n, z_nh;
        if (!is_boundary(flag)) {
            z_n = z[in];
            z_nh = zh[in];
        } else {
            z_n = boundary_value(z_c, normal, flag);
            z_nh = boundary_value(z_ch, normal, flag);
        }
        (void)z_n;
        PState zm, zp;
        bool robust = wt[ic] > 0 || wt[in] > 0;
        if (robust) {
            zm = z_ch;
            zp = z_nh;
        } else {
            V3 neib_c = flag == B_INNER ? m.center[in] : symm_point(m, f, cell_c);
            zm = extrap(z_ch, d_dx[ic], d_dy[ic], d_dz[ic], sub(face_c, cell_c));
            zm.energy = eos.energy_rP(zm.density, zm.pressure);
            if (is_bad(zm, eos)) zm = z_ch;
            if (!is_boundary(flag)) {
                zp = extrap(z_nh, d_dx[in], d_dy[in], d_dz[in], sub(face_c, neib_c));
                zp.energy = eos.energy_rP(zp.density, zp.pressure);
                if (is_bad(zp, eos)) zp = z_nh;
            } else {
                zp = boundary_value(zm, normal, flag);
            }
        }
        zm.velocity = rot_local(zm.velocity, normal);
        zp.velocity = rot_local(zp.velocity, normal);
        QState lf = robust ? hll(zm, zp, eos) : num_flux(flux_kind, zm, zp, eos);
        lf.momentum = rot_global(lf.momentum, normal);
        return lf;
    }

    // sm_fluid.cpp:255-366  fluxes_stage2 (corrector)
    void fluxes_stage2() {
        const Mesh &m = *mesh;
        wait_snap = wait;
        parallel_cells(m.n_cells, n_threads, [&](int b, int e) {
            for (int ic = b; ic < e; ++ic) {
                PState z_c = init[ic];
                QState q_c = q_from_p(z_c);
                QState flux;
                q_zero(flux);
                for (int s = 0; s < 8; ++s) {
                    size_t f = 8 * (size_t)ic + s;
                    if (m.boundary[f] == B_UNDEFINED) continue;
                    QState lf = stage2_face(ic, f, init, half, wait_snap);
                    accumulate(flux, lf, m.farea[f]);
                }
                update(q_c, dt / m.volume[ic], flux);
                next[ic] = p_from_q(q_c, eos);
                if (is_bad(next[ic], eos)) {
                    next[ic] = z_c;
                    wait[ic] = 3;
                } else if (wait[ic] > 0) {
                    --wait[ic];
                }
            }
        });
    }

    // Extension scheme (no counterpart in the reference): Heun's two-stage
    // Runge-Kutta on the same semi-discrete operator L(z) that the corrector
    // uses, with the half-step state replaced by the state itself:
    //   q*  = q^n - dt/V * sum F(z^n)          (gradients of z^n)
    //   q** = q*  - dt/V * sum F(z*),  z* = P(q*)  (gradients of z*)
    //   q^{n+1} = 0.5 * (q^n + q**)
    // `wait` is not used (no isolation in this mode).
    void heun_stage(const std::vector<PState> &z, std::vector<PState> &out, const std::vector<PState> *zn,
                    bool final) {
        const Mesh &m = *mesh;
        std::vector<int> zero_wait(m.n_cells, 0);
        parallel_cells(m.n_cells, n_threads, [&](int b, int e) {
            for (int ic = b; ic < e; ++ic) {
                QState q = q_from_p(z[ic]);
                QState flux;
                q_zero(flux);
                for (int s = 0; s < 8; ++s) {
                    size_t f = 8 * (size_t)ic + s;
                    if (m.boundary[f] == B_UNDEFINED) continue;
                    QState lf = stage2_face(ic, f, z, z, zero_wait);
                    accumulate(flux, lf, m.farea[f]);
                }
                update(q, dt / m.volume[ic], flux);
                if (final) {
                    QState q0 = q_from_p((*zn)[ic]);
                    double *a = &q.density;
                    const double *a0 = &q0.density;
                    for (int k = 0; k < 5; ++k) a[k] = 0.5 * (a0[k] + a[k]);
                }
                out[ic] = p_from_q(q, eos);
            }
        });
    }

    // sm_fluid.cpp:81-102  update
    void step() {
        compute_dt();
        if (acc == 1) {
            fluxes();
        } else if (scheme == SCHEME_REF) {
            compute_grad(init);
            fluxes_stage1();
            fluxes_stage2();
        } else {
            compute_grad(init);
            heun_stage(init, half, nullptr, false);
            compute_grad(half);
            heun_stage(half, next, &init, true);
        }
        init.swap(next);  // sm_fluid.cpp:368-370 (Storage::swap)
    }

    // sm_fluid.cpp:517-559  set_flags (flags only; compute_grad's side
    // effect on d_dx/d_dy/d_dz is kept for the distributor).
    void set_flags(int *flags) {
        const Mesh &m = *mesh;
        compute_grad(init);
        const double xi_dens = 0.05, xi_pres = 0.05;
        for (int ic = 0; ic < m.n_cells; ++ic) {
            int fl = -1;
            double dens = init[ic].density, pres = init[ic].pressure;
            double dens_split = xi_dens * std::abs(dens);
            double pres_split = xi_pres * std::abs(pres);
            for (int s = 0; s < 8; ++s) {
                size_t f = 8 * (size_t)ic + s;
                int flag = m.boundary[f];
                if (flag == B_UNDEFINED || is_boundary(flag)) continue;
                double dens_n = init[m.adj[f]].density, pres_n = init[m.adj[f]].pressure;
                if (std::abs(dens_n - dens) > dens_split || std::abs(pres_n - pres) > pres_split) {
                    fl = 1;
                    break;
                }
                if (std::abs(dens_n - dens) > 0.4 * dens_split || std::abs(pres_n - pres) > 0.4 * pres_split) {
                    fl = 0;
                }
            }
            flags[ic] = fl;
        }
    }
};

// Multi-material step (MmFluid): namespace zo::mm.
#include "zoracle_mm.inc"

// Scalar VOF transport (Transfer): namespace zo::tr.
#include "zoracle_tr.inc"

}  // namespace zo

// ---------------------------------------------------------------------------
// C interface used by the tests (ctypes).  States cross it as five SoA
// arrays (density, vx, vy, pressure, energy); vz is 0.
extern "C" {

void *zo_mesh_rect(int nx, int ny, double x_min, double x_max, double y_min, double y_max,
                   const int *bounds) {
    auto *m = new zo::Mesh();
    zo::make_rectangle(*m, nx, ny, x_min, x_max, y_min, y_max, bounds);
    return m;
}
// A mesh given cell by cell (8 slots per cell), e.g. a refined zephyr mesh.
// The incircle diameters are given; verts then hold them on the vs<+1,0> /
// vs<-1,0> axis so that incircle_diameter() returns them unchanged.
void *zo_mesh_arrays(int n, const double *cx, const double *cy, const double *vol, const double *inc,
                     const int *boundary, const int *adj, const double *nx, const double *ny, const double *fx,
                     const double *fy, const double *area) {
    auto *m = new zo::Mesh();
    m->n_cells = n;
    m->center.resize(n);
    m->volume.assign(vol, vol + n);
    m->verts.assign(9 * (size_t)n, zo::V3{0, 0, 0});
    m->level.assign(n, 0);
    m->flag.assign(n, 0);
    m->b_idx.assign(n, 0);
    m->z_idx.assign(n, 0);
    m->boundary.assign(boundary, boundary + 8 * (size_t)n);
    m->adj.assign(adj, adj + 8 * (size_t)n);
    m->fnormal.resize(8 * (size_t)n);
    m->fcenter.resize(8 * (size_t)n);
    m->farea.assign(area, area + 8 * (size_t)n);
    m->incircle.assign(inc, inc + n);
    for (int i = 0; i < n; ++i) m->center[i] = zo::V3{cx[i], cy[i], 0.0};
    for (size_t f = 0; f < 8 * (size_t)n; ++f) {
        m->fnormal[f] = zo::V3{nx[f], ny[f], 0.0};
        m->fcenter[f] = zo::V3{fx[f], fy[f], 0.0};
    }
    return m;
}

void zo_mesh_free(void *m) { delete static_cast<zo::Mesh *>(m); }
int zo_mesh_ncells(void *m) { return static_cast<zo::Mesh *>(m)->n_cells; }

// Cell centres (x, y), volumes, and per slot: boundary, neighbour, normal
// (x, y), face centre (x, y), area.  Arrays sized n, n, 8n ...
void zo_mesh_geometry(void *mp, double *cx, double *cy, double *vol, int *boundary, int *adj, double *nx,
                      double *ny, double *fx, double *fy, double *area) {
    auto &m = *static_cast<zo::Mesh *>(mp);
    for (int i = 0; i < m.n_cells; ++i) {
        cx[i] = m.center[i].x;
        cy[i] = m.center[i].y;
        vol[i] = m.volume[i];
    }
    for (size_t f = 0; f < 8 * (size_t)m.n_cells; ++f) {
        boundary[f] = m.boundary[f];
        adj[f] = m.adj[f];
        nx[f] = m.fnormal[f].x;
        ny[f] = m.fnormal[f].y;
        fx[f] = m.fcenter[f].x;
        fy[f] = m.fcenter[f].y;
        area[f] = m.farea[f];
    }
}

void *zo_solver_create(void *mesh, int eos_kind, double gamma, double P0, double e0, int flux, int limiter,
                       int acc, int scheme, double CFL, int n_threads) {
    auto *s = new zo::Solver();
    s->mesh = static_cast<zo::Mesh *>(mesh);
    s->eos = zo::Eos{eos_kind, gamma, P0, e0};
    s->flux_kind = flux;
    s->limiter = limiter;
    s->acc = acc;
    s->scheme = scheme;
    s->CFL = std::max(0.0, std::min(CFL, 1.0));  // sm_fluid.cpp:37-39
    s->n_threads = n_threads;
    s->resize();
    return s;
}
void zo_solver_free(void *s) { delete static_cast<zo::Solver *>(s); }
void zo_solver_set_max_dt(void *s, double dt) { static_cast<zo::Solver *>(s)->max_dt = dt; }
void zo_solver_set_threads(void *s, int n) { static_cast<zo::Solver *>(s)->n_threads = n; }

void zo_solver_set_state(void *sp, const double *rho, const double *u, const double *v, const double *p,
                         const double *e) {
    auto &s = *static_cast<zo::Solver *>(sp);
    for (int i = 0; i < s.mesh->n_cells; ++i) {
        s.init[i] = zo::PState{rho[i], {u[i], v[i], 0.0}, p[i], e[i]};
    }
}
void zo_solver_get_state(void *sp, double *rho, double *u, double *v, double *p, double *e) {
    auto &s = *static_cast<zo::Solver *>(sp);
    for (int i = 0; i < s.mesh->n_cells; ++i) {
        rho[i] = s.init[i].density;
        u[i] = s.init[i].velocity.x;
        v[i] = s.init[i].velocity.y;
        p[i] = s.init[i].pressure;
        e[i] = s.init[i].energy;
    }
}
void zo_solver_get_wait(void *sp, int *w) {
    auto &s = *static_cast<zo::Solver *>(sp);
    for (int i = 0; i < s.mesh->n_cells; ++i) w[i] = s.wait[i];
}
void zo_solver_set_wait(void *sp, const int *w) {
    auto &s = *static_cast<zo::Solver *>(sp);
    for (int i = 0; i < s.mesh->n_cells; ++i) s.wait[i] = w[i];
}
// Limited gradients of the current state (x and y components, 5 fields each).
void zo_solver_grad(void *sp, double *gx, double *gy) {
    auto &s = *static_cast<zo::Solver *>(sp);
    s.compute_grad(s.init);
    int n = s.mesh->n_cells;
    for (int i = 0; i < n; ++i) {
        const zo::PState &a = s.d_dx[i], &b = s.d_dy[i];
        double ax[5] = {a.density, a.velocity.x, a.velocity.y, a.pressure, a.energy};
        double by[5] = {b.density, b.velocity.x, b.velocity.y, b.pressure, b.energy};
        for (int k = 0; k < 5; ++k) {
            gx[(size_t)k * n + i] = ax[k];
            gy[(size_t)k * n + i] = by[k];
        }
    }
}
// The CFL quantity before CFL and max_dt: min over cells of
// incircle / (|v| + c) (sm_fluid.cpp:104-111).
double zo_solver_cfl_min(void *sp) {
    auto &s = *static_cast<zo::Solver *>(sp);
    const zo::Mesh &m = *s.mesh;
    double res = std::numeric_limits<double>::max();
    for (int ic = 0; ic < m.n_cells; ++ic) {
        double c = s.eos.sound_speed_rP(s.init[ic].density, s.init[ic].pressure);
        double v = zo::incircle_diameter(m, ic) / (zo::norm(s.init[ic].velocity) + c);
        res = std::min(res, v);
    }
    return res;
}
double zo_solver_compute_dt(void *sp) {
    auto &s = *static_cast<zo::Solver *>(sp);
    s.compute_dt();
    return s.dt;
}
double zo_solver_step(void *sp) {
    auto &s = *static_cast<zo::Solver *>(sp);
    s.step();
    return s.dt;
}
double zo_solver_steps(void *sp, int n, double *dts) {
    auto &s = *static_cast<zo::Solver *>(sp);
    for (int k = 0; k < n; ++k) {
        s.step();
        if (dts) dts[k] = s.dt;
    }
    return s.dt;
}
void zo_solver_set_flags(void *sp, int *flags) { static_cast<zo::Solver *>(sp)->set_flags(flags); }

// Pointwise pieces (states as 6 doubles: rho, vx, vy, vz, p, e).
static zo::PState mk(const double *z) { return zo::PState{z[0], {z[1], z[2], z[3]}, z[4], z[5]}; }
static void put(const zo::QState &f, double *o) {
    o[0] = f.density;
    o[1] = f.momentum.x;
    o[2] = f.momentum.y;
    o[3] = f.momentum.z;
    o[4] = f.energy;
}
void zo_flux(int kind, const double *zL, const double *zR, int eos_kind, double gamma, double P0, double e0,
             double *out) {
    zo::Eos eos{eos_kind, gamma, P0, e0};
    put(zo::num_flux(kind, mk(zL), mk(zR), eos), out);
}
double zo_limiter(int kind, double a, double b) { return zo::limiter2(kind, a, b); }
void zo_eos(int eos_kind, double gamma, double P0, double e0, double rho, double x, double *out) {
    // out: pressure_re(rho, x), energy_rP(rho, x), sound_speed_rP(rho, x)
    zo::Eos eos{eos_kind, gamma, P0, e0};
    out[0] = eos.pressure_re(rho, x);
    out[1] = eos.energy_rP(rho, x);
    out[2] = eos.sound_speed_rP(rho, x);
}

// ---- multi-material step (zo::mm) ----
// Material presets: out = stiffened flag, gamma, P0, e0, Cv, T0, rho_ref.
int zo_mm_material(const char *kind, const char *name, double *out) {
    zo::mm::Mat m;
    if (!zo::mm::named_material(kind, name, m)) return -1;
    double v[7] = {double(m.stiffened), m.gamma, m.P0, m.e0, m.Cv, m.T0, m.rho_ref};
    std::memcpy(out, v, sizeof(v));
    return 0;
}
// nm materials, 7 parameters each as from zo_mm_material.
void *zo_mm_create(void *mesh, int nm, const double *mats, double CFL, int crp_mode, int threads) {
    auto *s = new zo::mm::MmSolver(*static_cast<zo::Mesh *>(mesh));
    s->mx.nm = nm;
    for (int i = 0; i < nm; ++i) {
        const double *p = mats + 7 * i;
        s->mx.mat[i] = {int(p[0]), p[1], p[2], p[3], p[4], p[5], p[6]};
    }
    s->CFL = std::max(0.0, std::min(CFL, 1.0));
    s->crp = crp_mode;
    s->threads = threads;
    return s;
}
void zo_mm_free(void *p) { delete static_cast<zo::mm::MmSolver *>(p); }
void zo_mm_set_max_dt(void *p, double dt) { static_cast<zo::mm::MmSolver *>(p)->max_dt = dt; }
void zo_mm_set_threads(void *p, int n) { static_cast<zo::mm::MmSolver *>(p)->threads = n; }
// MmFluid::set_splitting (mm_fluid.cpp:75-77): 0 NONE, 1 SIMPLE, 2 STRANG
void zo_mm_set_split(void *p, int split) { static_cast<zo::mm::MmSolver *>(p)->split = split; }
// MmFluid::set_accuracy / set_limiter (mm_fluid.cpp:46-48, 72-74)
void zo_mm_set_accuracy(void *p, int acc, int limiter) {
    auto *s = static_cast<zo::mm::MmSolver *>(p);
    s->acc = std::min(std::max(1, acc), 2);
    s->limiter = limiter;
}
// States from (density, velocity, pressure, mass fractions) through the
// mixture closure, as PState(density, velocity, pressure, Fractions(array),
// mixture); beta holds 4 fractions per cell and is normalised first.
void zo_mm_make_states(void *p, const double *rho, const double *vx, const double *vy, const double *P,
                       const double *beta) {
    auto *s = static_cast<zo::mm::MmSolver *>(p);
    for (int i = 0; i < s->m.n_cells; ++i) {
        zo::mm::Frac b;
        for (int k = 0; k < 4; ++k) b.f[k] = beta[4 * (size_t)i + k];
        zo::mm::normalize(b);
        s->z[i] = zo::mm::state_of_rvp(s->mx, rho[i], {vx[i], vy[i], 0.0}, P[i], b);
    }
}
void zo_mm_set_states(void *p, const double *st) {
    auto *s = static_cast<zo::mm::MmSolver *>(p);
    for (int i = 0; i < s->m.n_cells; ++i) s->z[i] = zo::mm::unpack(st + 14 * (size_t)i);
}
void zo_mm_get_states(void *p, double *st) {
    auto *s = static_cast<zo::mm::MmSolver *>(p);
    for (int i = 0; i < s->m.n_cells; ++i) zo::mm::pack(s->z[i], st + 14 * (size_t)i);
}
double zo_mm_step(void *p) { return static_cast<zo::mm::MmSolver *>(p)->step(); }
double zo_mm_steps(void *p, int n, double *dts) {
    auto *s = static_cast<zo::mm::MmSolver *>(p);
    for (int k = 0; k < n; ++k) {
        double d = s->step();
        if (dts) dts[k] = d;
    }
    return s->dt;
}
double zo_mm_compute_dt(void *p) { return static_cast<zo::mm::MmSolver *>(p)->compute_dt(); }
int zo_mm_bad(void *p) { return static_cast<zo::mm::MmSolver *>(p)->bad ? 1 : 0; }
void zo_mm_interface(void *p, double *nrm, double *off) {
    auto *s = static_cast<zo::mm::MmSolver *>(p);
    int nm = s->mx.nm;
    s->nrm.assign((size_t)s->m.n_cells * nm, zo::V3{0.0, 0.0, 0.0});
    s->off.assign((size_t)s->m.n_cells * nm, 0.0);
    for (int ic = 0; ic < s->m.n_cells; ++ic) s->recover(ic);
    for (size_t k = 0; k < s->nrm.size(); ++k) {
        nrm[2 * k] = s->nrm[k].x;
        nrm[2 * k + 1] = s->nrm[k].y;
        off[k] = s->off[k];
    }
}
void zo_mm_flags(void *p, int *flags) { static_cast<zo::mm::MmSolver *>(p)->set_flags(flags); }
void zo_mm_state_from_q(void *p, const double *q, const double *guess, double *out) {
    auto *s = static_cast<zo::mm::MmSolver *>(p);
    zo::mm::QV Q;
    for (int k = 0; k < zo::mm::NQ; ++k) Q.a[k] = q[k];
    zo::mm::pack(zo::mm::state_of_q(s->mx, Q, guess[0], guess[1], guess + 2), out);
}
double zo_mm_sound_speed(void *p, const double *st) {
    auto *s = static_cast<zo::mm::MmSolver *>(p);
    zo::mm::MState z = zo::mm::unpack(st);
    zo::mm::Opts o;
    o.T0 = z.T;
    o.rhos = z.rhos;
    return zo::mm::sound_speed_rP(s->mx, z.rho, z.P, z.beta, o);
}
int zo_mm_hllc(void *p, const double *sl, const double *sr, double *out) {
    auto *s = static_cast<zo::mm::MmSolver *>(p);
    bool bad = false;
    zo::mm::QV f = zo::mm::hllc(s->mx, zo::mm::unpack(sl), zo::mm::unpack(sr), bad);
    std::memcpy(out, f.a, sizeof(f.a));
    return bad ? 1 : 0;
}
int zo_mm_crp_flux(void *p, const double *sl, const double *sr, double hL, double hR, int iA, double a_sig,
                   double dt, double *out) {
    auto *s = static_cast<zo::mm::MmSolver *>(p);
    bool bad = false;
    zo::mm::QV f = zo::mm::crp_flux(s->mx, zo::mm::unpack(sl), zo::mm::unpack(sr), hL, hR, iA, a_sig, dt, bad);
    std::memcpy(out, f.a, sizeof(f.a));
    return bad ? 1 : 0;
}
double zo_mm_face_fraction(double a1, double a2) { return zo::mm::face_fraction(a1, a2); }
double zo_mm_quad_find_section(double alpha, double nx, double ny, double A, double B) {
    return zo::mm::quad_find_section(alpha, {nx, ny, 0.0}, A, B);
}
double zo_mm_quad_volume_fraction(double p, double nx, double ny, double A, double B) {
    return zo::mm::quad_volume_fraction(p, {nx, ny, 0.0}, A, B);
}
double zo_mm_average_flux(double alpha, double cos, double CFL) { return zo::mm::average_flux(alpha, cos, CFL); }

// ---- Transfer (zo::tr) ----
// method: Transfer::Method value (VOF and CRP families); vel_kind 0: vel =
// {vx, vy}; 1: vel = {cx, cy, omega}.
void *zo_tr_create(void *mesh, int method, double CFL, int vel_kind, const double *vel) {
    auto *s = new zo::tr::TrSolver(*static_cast<zo::Mesh *>(mesh));
    s->method = method;
    s->CFL = std::max(0.0, std::min(CFL, 1.0));  // Transfer::set_CFL (transfer.cpp:65-67)
    s->vel_kind = vel_kind;
    if (vel_kind == 0) {
        s->V0 = {vel[0], vel[1], 0.0};
    } else {
        s->center = {vel[0], vel[1], 0.0};
        s->omega = {0.0, 0.0, vel[2]};
    }
    return s;
}
void zo_tr_free(void *p) { delete static_cast<zo::tr::TrSolver *>(p); }
void zo_tr_set_u(void *p, const double *u1) {
    auto *s = static_cast<zo::tr::TrSolver *>(p);
    for (int i = 0; i < s->m.n_cells; ++i) {
        s->u1[i] = u1[i];
        s->u2[i] = 0.0;
    }
}
void zo_tr_update_interface(void *p, int smoothing) { static_cast<zo::tr::TrSolver *>(p)->update_interface(smoothing); }
double zo_tr_compute_dt(void *p) { return static_cast<zo::tr::TrSolver *>(p)->compute_dt(); }
void zo_tr_set_dt(void *p, double dt) { static_cast<zo::tr::TrSolver *>(p)->dt = dt; }
void zo_tr_update(void *p, int dir) { static_cast<zo::tr::TrSolver *>(p)->update(dir); }
void zo_tr_get(void *p, double *u1, double *nrm, double *pt) {
    auto *s = static_cast<zo::tr::TrSolver *>(p);
    for (int i = 0; i < s->m.n_cells; ++i) {
        u1[i] = s->u1[i];
        nrm[2 * i] = s->n[i].x;
        nrm[2 * i + 1] = s->n[i].y;
        pt[2 * i] = s->p[i].x;
        pt[2 * i + 1] = s->p[i].y;
    }
}
void zo_tr_flags(void *p, int *flags) { static_cast<zo::tr::TrSolver *>(p)->set_flags(flags); }

}  // extern "C"
