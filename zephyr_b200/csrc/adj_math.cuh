// adj_math.cuh -- the differentiable forward of the adjoint mode, written
// once for plain doubles and for dual numbers.
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

// ---- dual numbers: value and N partial derivatives ------------------------
template <int N>
struct Dual {
    double v;
    double d[N];
};
template <int N>
__device__ __forceinline__ Dual<N> dconst(double x) {
    Dual<N> r;
    r.v = x;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = 0.0;
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> dvar(double x, int k) {
    Dual<N> r = dconst<N>(x);
    r.d[k] = 1.0;
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator+(const Dual<N> &a, const Dual<N> &b) {
    Dual<N> r;
    r.v = a.v + b.v;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = a.d[k] + b.d[k];
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(const Dual<N> &a, const Dual<N> &b) {
    Dual<N> r;
    r.v = a.v - b.v;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = a.d[k] - b.d[k];
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(const Dual<N> &a) {
    Dual<N> r;
    r.v = -a.v;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = -a.d[k];
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator*(const Dual<N> &a, const Dual<N> &b) {
    Dual<N> r;
    r.v = a.v * b.v;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator/(const Dual<N> &a, const Dual<N> &b) {
    Dual<N> r;
    double inv = 1.0 / b.v;
    r.v = a.v * inv;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = (a.d[k] - r.v * b.d[k]) * inv;
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator*(double s, const Dual<N> &a) {
    Dual<N> r;
    r.v = s * a.v;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = s * a.d[k];
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator+(const Dual<N> &a, double s) {
    Dual<N> r = a;
    r.v += s;
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> operator-(const Dual<N> &a, double s) {
    Dual<N> r = a;
    r.v -= s;
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> tsqrt(const Dual<N> &a) {
    Dual<N> r;
    r.v = ::sqrt(a.v);
    double h = 0.5 / r.v;
#pragma unroll
    for (int k = 0; k < N; ++k) r.d[k] = h * a.d[k];
    return r;
}
template <int N>
__device__ __forceinline__ Dual<N> tabs(const Dual<N> &a) {
    return a.v < 0.0 ? -a : a;
}
__device__ __forceinline__ double tsqrt(double x) { return ::sqrt(x); }
__device__ __forceinline__ double tabs(double x) { return ::fabs(x); }
__device__ __forceinline__ double val(double x) { return x; }
template <int N>
__device__ __forceinline__ double val(const Dual<N> &x) {
    return x.v;
}
// min / max: the argument the forward picks (first unless the second is
// strictly better), differentiated on that side
template <class T>
__device__ __forceinline__ T tmin(const T &a, const T &b) {
    return val(b) < val(a) ? b : a;
}
template <class T>
__device__ __forceinline__ T tmax(const T &a, const T &b) {
    return val(a) < val(b) ? b : a;
}

// ---- the step's pieces, generic in T ----------------------------------------
// primitive (rho, u, v, p) of a conservative state, ideal gas
template <class T>
__device__ __forceinline__ void prim(const T U[4], const T &gamma, T W[4]) {
    W[0] = U[0];
    W[1] = U[1] / U[0];
    W[2] = U[2] / U[0];
    W[3] = (gamma - 1.0) * (U[3] - 0.5 * ((U[1] * U[1] + U[2] * U[2]) / U[0]));
}

// limited slope of one field along one axis from its three values
template <class T>
__device__ __forceinline__ T slope(const T &wm, const T &w0, const T &wp, double inv2h, double eps) {
    T dL = wm - w0, dR = wp - w0;
    T a1 = -dL, a2 = -dR;
    T phiR = (a1 * (a1 + dR) + eps) / (a1 * a1 + dR * dR + eps);  // phi(-dL, dR)
    T phiL = (a2 * (a2 + dL) + eps) / (a2 * a2 + dL * dL + eps);  // phi(-dR, dL)
    return inv2h * (phiR * dR - phiL * dL);
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
    T gm1 = gamma - 1.0;
    T rEL = pL / gm1 + 0.5 * (rL * (uL * uL + vL * vL));
    T rER = pR / gm1 + 0.5 * (rR * (uR * uR + vR * vR));
    T cL = tsqrt(gamma * pL / rL), cR = tsqrt(gamma * pR / rR);
    T SL = tmin(uL - cL, uR - cR);
    T SR = tmax(uL + cL, uR + cR);
    if (val(SL) >= 0.0) {
        phys_flux(rL, uL, vL, pL, rEL, F);
        return;
    }
    if (val(SR) <= 0.0) {
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
        F[k] = 0.5 * (FL[k] + FR[k] + SL * (QsL[k] - QL[k]) + aSC * (QsL[k] - QsR[k]) + SR * (QsR[k] - QR[k]));
}

}  // namespace adj
}  // namespace zg
