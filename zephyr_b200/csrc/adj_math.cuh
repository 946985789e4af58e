// adj_math.cuh -- the differentiable forward of the adjoint mode and its
// hand-written reverse, templated on the face arithmetic: double (the FP64
// form) or float (the mixed form).  Constants are written T(x), so that the
// double instantiation performs exactly the FP64 operations.
//
// The step differentiated is Heun's method on the finite-volume operator
//   L(U)_c = -(1/V) sum_faces S F(face states),
// on a uniform periodic rectangle, at a fixed dt:
//   U* = U + dt L(U),   U^{n+1} = 1/2 (U + U* + dt L(U*)).
// U = (rho, rho u, rho v, rho E) per cell, ideal gas with adiabatic index
// gamma.  Face states: primitive W = (rho, u, v, p) extrapolated from the
// cell centre with the limited least-squares gradient of zephyr's
// gradient::LSM + gradient::limiting (gradient.h:226-282, 412-474), which on
// a uniform axis-aligned mesh reduces per axis and per field to
//   dL = W_{i-1} - W_i,  dR = W_{i+1} - W_i,
//   g  = (phi(-dL, dR) dR - phi(-dR, dL) dL) / (2 h),
// with the smooth van Albada limiter phi(a, b) = (a (a + b) + eps) /
// (a^2 + b^2 + eps) (no clipping, so that the step is differentiable; the
// reference's vanAlbada1 clips at a b <= 0, limiter.cxx:69-82).  Fluxes: HLLC
// with Davis wave speeds (hllc.cpp:23-83); its branches (supersonic sides,
// the min / max of the speed estimates, the sign of S_C) are the ones the
// forward takes, and the adjoint differentiates that branch.
#pragma once

#include <cuda_runtime.h>

#include <cmath>

namespace zg {
namespace adj {

// ---- scalar helpers for T = double (FP64 form) and T = float (mixed form) ----
__device__ __forceinline__ double tsqrt(double x) { return ::sqrt(x); }
__device__ __forceinline__ float tsqrt(float x) { return ::sqrtf(x); }
__device__ __forceinline__ double tabs(double x) { return ::fabs(x); }
__device__ __forceinline__ float tabs(float x) { return ::fabsf(x); }
// min / max: the argument the forward picks (first unless the second is
// strictly better); the reverse differentiates that side
template <class T>
__device__ __forceinline__ T tmin(const T &a, const T &b) {
    return b < a ? b : a;
}
template <class T>
__device__ __forceinline__ T tmax(const T &a, const T &b) {
    return a < b ? b : a;
}

// ---- the step's pieces, generic in T ----------------------------------------
// primitive (rho, u, v, p) of a conservative state, ideal gas
template <class T>
__device__ __forceinline__ void prim(const T U[4], const T &gamma, T W[4]) {
    W[0] = U[0];
    W[1] = U[1] / U[0];
    W[2] = U[2] / U[0];
    W[3] = (gamma - T(1)) * (U[3] - T(0.5) * ((U[1] * U[1] + U[2] * U[2]) / U[0]));
}

// limited slope of one field along one axis from the differences
// a = w_{i-1} - w_i and b = w_{i+1} - w_i of its three values:
//   (phi(-a, b) b - phi(-b, a) a) / (2h)
// where both limiter values share the denominator a^2 + b^2 + eps, so that
//   = (a - b) (2 a b - eps) / (a^2 + b^2 + eps) / (2h).
// The differences are taken by the caller in FP64 (the values are FP64 in
// both forms): in FP32 the difference of two neighbouring values of a smooth
// field keeps only the digits their FP32 roundings share.
template <class T>
__device__ __forceinline__ T slope(T a, T b, T inv2h, T eps) {
    return inv2h * ((a - b) * (T(2) * a * b - eps)) / (a * a + b * b + eps);
}
// its partial derivatives with respect to (w_{i-1}, w_i, w_{i+1})
template <class T>
__device__ __forceinline__ void slope_partials(T a, T b, T inv2h, T eps, T d[3]) {
    T q = T(2) * a * b - eps, P = (a - b) * q;
    T iD = T(1) / (a * a + b * b + eps);
    T Pa = q + (a - b) * (T(2) * b), Pb = -q + (a - b) * (T(2) * a);
    T ga = inv2h * (Pa - P * (T(2) * a) * iD) * iD;
    T gb = inv2h * (Pb - P * (T(2) * b) * iD) * iD;
    d[0] = ga;
    d[1] = -(ga + gb);
    d[2] = gb;
}

// physical flux of a face-frame primitive state (models.cpp:131-137)
template <class T>
__device__ __forceinline__ void phys_flux(const T &r, const T &u, const T &v, const T &p, const T &rE, T F[4]) {
    F[0] = r * u;
    F[1] = r * u * u + p;
    F[2] = r * u * v;
    F[3] = (rE + p) * u;
}

// HLLC flux of two face-frame primitive states (hllc.cpp:23-83, Davis speeds)
template <class T>
__device__ void hllc(const T L[4], const T R[4], const T &gamma, T F[4]) {
    const T &rL = L[0], &uL = L[1], &vL = L[2], &pL = L[3];
    const T &rR = R[0], &uR = R[1], &vR = R[2], &pR = R[3];
    T gm1 = gamma - T(1);
    T rEL = pL / gm1 + T(0.5) * (rL * (uL * uL + vL * vL));
    T rER = pR / gm1 + T(0.5) * (rR * (uR * uR + vR * vR));
    T cL = tsqrt(gamma * pL / rL), cR = tsqrt(gamma * pR / rR);
    T SL = tmin(uL - cL, uR - cR);
    T SR = tmax(uL + cL, uR + cR);
    if (SL >= T(0)) {
        phys_flux(rL, uL, vL, pL, rEL, F);
        return;
    }
    if (SR <= T(0)) {
        phys_flux(rR, uR, vR, pR, rER, F);
        return;
    }
    T aL = rL * (SL - uL), aR = rR * (SR - uR);
    T SC = (pL - pR + aR * uR - aL * uL) / (aR - aL);
    T rsL = aL / (SL - SC), rsR = aR / (SR - SC);
    T EL = rEL / rL, ER = rER / rR;
    T EsL = EL + (SC - uL) * (SC + pL / aL);
    T EsR = ER + (SC - uR) * (SC + pR / aR);
    T FL[4], FR[4];
    phys_flux(rL, uL, vL, pL, rEL, FL);
    phys_flux(rR, uR, vR, pR, rER, FR);
    T QL[4] = {rL, rL * uL, rL * vL, rEL};
    T QR[4] = {rR, rR * uR, rR * vR, rER};
    T QsL[4] = {rsL, rsL * SC, rsL * vL, rsL * EsL};
    T QsR[4] = {rsR, rsR * SC, rsR * vR, rsR * EsR};
    T aSC = tabs(SC);
#pragma unroll
    for (int k = 0; k < 4; ++k)
        F[k] = T(0.5) * (FL[k] + FR[k] + SL * (QsL[k] - QL[k]) + aSC * (QsL[k] - QsR[k]) + SR * (QsR[k] - QR[k]));
}

// Reverse of hllc<T>: given the cotangent Fb of the flux, the
// cotangents of the two face states (Lb, Rb, overwritten) and of gamma
// (added to gb).  The forward is re-evaluated first; every min / max / abs /
// branch takes the side the forward took.
template <class T>
__device__ inline void hllc_vjp(const T L[4], const T R[4], T gamma, const T Fb[4], T Lb[4], T Rb[4], T &gb) {
    const T rL = L[0], uL = L[1], vL = L[2], pL = L[3];
    const T rR = R[0], uR = R[1], vR = R[2], pR = R[3];
    const T gm1 = gamma - T(1.0), igm1 = T(1.0) / gm1;
    const T irL = T(1.0) / rL, irR = T(1.0) / rR;
    const T kL = uL * uL + vL * vL, kR = uR * uR + vR * vR;
    const T rEL = pL * igm1 + T(0.5) * (rL * kL), rER = pR * igm1 + T(0.5) * (rR * kR);
    const T xL = gamma * pL * irL, xR = gamma * pR * irR;
    const T cL = tsqrt(xL), cR = tsqrt(xR);
    const T A = uL - cL, B = uR - cR, C = uL + cL, D = uR + cR;
    const bool selB = B < A, selD = C < D;  // tmin / tmax choices
    const T SL = selB ? B : A, SR = selD ? D : C;
    T rLb = T(0.0), uLb = T(0.0), vLb = T(0.0), pLb = T(0.0), rELb = T(0.0);
    T rRb = T(0.0), uRb = T(0.0), vRb = T(0.0), pRb = T(0.0), rERb = T(0.0);
    T SLb = T(0.0), SRb = T(0.0);
    // reverse of phys_flux(r, u, v, p, rE) scaled by w: F = w * Fb
    auto phys_rev = [](T r, T u, T v, T p, T rE, const T *Fw, T &rb, T &ub,
                       T &vb, T &pb, T &rEb) {
        rb += Fw[0] * u + Fw[1] * (u * u) + Fw[2] * (u * v);
        ub += Fw[0] * r + Fw[1] * (T(2.0) * r * u) + Fw[2] * (r * v) + Fw[3] * (rE + p);
        vb += Fw[2] * (r * u);
        pb += Fw[1] + Fw[3] * u;
        rEb += Fw[3] * u;
    };
    if (SL >= T(0.0)) {
        phys_rev(rL, uL, vL, pL, rEL, Fb, rLb, uLb, vLb, pLb, rELb);
    } else if (SR <= T(0.0)) {
        phys_rev(rR, uR, vR, pR, rER, Fb, rRb, uRb, vRb, pRb, rERb);
    } else {
        const T aL = rL * (SL - uL), aR = rR * (SR - uR);
        const T num = pL - pR + aR * uR - aL * uL, den = aR - aL, iden = T(1.0) / den;
        const T SC = num * iden;
        const T dLs = SL - SC, dRs = SR - SC, idL = T(1.0) / dLs, idR = T(1.0) / dRs;
        const T rsL = aL * idL, rsR = aR * idR;
        const T EL = rEL * irL, ER = rER * irR;
        const T iaL = T(1.0) / aL, iaR = T(1.0) / aR;
        const T tL = SC - uL, wL = SC + pL * iaL, tR = SC - uR, wR = SC + pR * iaR;
        const T EsL = EL + tL * wL, EsR = ER + tR * wR;
        const T QL[4] = {rL, rL * uL, rL * vL, rEL}, QR[4] = {rR, rR * uR, rR * vR, rER};
        const T QsL[4] = {rsL, rsL * SC, rsL * vL, rsL * EsL}, QsR[4] = {rsR, rsR * SC, rsR * vR, rsR * EsR};
        const T sgn = SC < T(0.0) ? -T(1.0) : T(1.0), aSC = sgn * SC;
        T half[4], QsLb[4], QsRb[4], QLb[4], QRb[4], aSCb = T(0.0);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            half[k] = T(0.5) * Fb[k];
            SLb += half[k] * (QsL[k] - QL[k]);
            SRb += half[k] * (QsR[k] - QR[k]);
            aSCb += half[k] * (QsL[k] - QsR[k]);
            QsLb[k] = half[k] * (SL + aSC);
            QsRb[k] = half[k] * (SR - aSC);
            QLb[k] = -half[k] * SL;
            QRb[k] = -half[k] * SR;
        }
        phys_rev(rL, uL, vL, pL, rEL, half, rLb, uLb, vLb, pLb, rELb);
        phys_rev(rR, uR, vR, pR, rER, half, rRb, uRb, vRb, pRb, rERb);
        T SCb = aSCb * sgn;
        // Qs = (rs, rs SC, rs v, rs Es)
        T rsLb = QsLb[0] + QsLb[1] * SC + QsLb[2] * vL + QsLb[3] * EsL;
        T rsRb = QsRb[0] + QsRb[1] * SC + QsRb[2] * vR + QsRb[3] * EsR;
        SCb += QsLb[1] * rsL + QsRb[1] * rsR;
        vLb += QsLb[2] * rsL;
        vRb += QsRb[2] * rsR;
        const T EsLb = QsLb[3] * rsL, EsRb = QsRb[3] * rsR;
        // Q = (r, r u, r v, rE)
        rLb += QLb[0] + QLb[1] * uL + QLb[2] * vL;
        uLb += QLb[1] * rL;
        vLb += QLb[2] * rL;
        rELb += QLb[3];
        rRb += QRb[0] + QRb[1] * uR + QRb[2] * vR;
        uRb += QRb[1] * rR;
        vRb += QRb[2] * rR;
        rERb += QRb[3];
        // Es = E + t w,  t = SC - u,  w = SC + p / a,  E = rE / r
        T aLb = T(0.0), aRb = T(0.0);
        {
            T ELb = EsLb, tLb = EsLb * wL, wLb = EsLb * tL;
            SCb += tLb + wLb;
            uLb -= tLb;
            pLb += wLb * iaL;
            aLb -= wLb * pL * (iaL * iaL);
            rELb += ELb * irL;
            rLb -= ELb * EL * irL;
            T ERb = EsRb, tRb = EsRb * wR, wRb = EsRb * tR;
            SCb += tRb + wRb;
            uRb -= tRb;
            pRb += wRb * iaR;
            aRb -= wRb * pR * (iaR * iaR);
            rERb += ERb * irR;
            rRb -= ERb * ER * irR;
        }
        // rs = a / (S - SC)
        aLb += rsLb * idL;
        T dLsb = -rsLb * rsL * idL;
        SLb += dLsb;
        SCb -= dLsb;
        aRb += rsRb * idR;
        T dRsb = -rsRb * rsR * idR;
        SRb += dRsb;
        SCb -= dRsb;
        // SC = num / den
        const T numb = SCb * iden, denb = -SCb * SC * iden;
        aRb += denb;
        aLb -= denb;
        pLb += numb;
        pRb -= numb;
        aRb += numb * uR;
        uRb += numb * aR;
        aLb -= numb * uL;
        uLb -= numb * aL;
        // a = r (S - u)
        rLb += aLb * (SL - uL);
        SLb += aLb * rL;
        uLb -= aLb * rL;
        rRb += aRb * (SR - uR);
        SRb += aRb * rR;
        uRb -= aRb * rR;
    }
    // SL = min(uL - cL, uR - cR), SR = max(uL + cL, uR + cR)
    T cLb = T(0.0), cRb = T(0.0);
    if (selB) {
        uRb += SLb;
        cRb -= SLb;
    } else {
        uLb += SLb;
        cLb -= SLb;
    }
    if (selD) {
        uRb += SRb;
        cRb += SRb;
    } else {
        uLb += SRb;
        cLb += SRb;
    }
    // c = sqrt(gamma p / r)
    const T xLb = cLb * T(0.5) / cL, xRb = cRb * T(0.5) / cR;
    gb += xLb * (pL * irL) + xRb * (pR * irR);
    pLb += xLb * gamma * irL;
    rLb -= xLb * xL * irL;
    pRb += xRb * gamma * irR;
    rRb -= xRb * xR * irR;
    // rE = p / (gamma - 1) + r k / 2,  k = u^2 + v^2
    pLb += rELb * igm1;
    pRb += rERb * igm1;
    gb -= (rELb * pL + rERb * pR) * (igm1 * igm1);
    rLb += rELb * T(0.5) * kL;
    rRb += rERb * T(0.5) * kR;
    uLb += rELb * rL * uL;
    vLb += rELb * rL * vL;
    uRb += rERb * rR * uR;
    vRb += rERb * rR * vR;
    Lb[0] = rLb;
    Lb[1] = uLb;
    Lb[2] = vLb;
    Lb[3] = pLb;
    Rb[0] = rRb;
    Rb[1] = uRb;
    Rb[2] = vRb;
    Rb[3] = pRb;
}

}  // namespace adj
}  // namespace zg
