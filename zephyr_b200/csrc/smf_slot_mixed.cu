// smf_slot_mixed.cu -- the MIXED form of the step on an adaptive rectangle:
// FP32 primitive states, limited least-squares gradients, reconstruction and
// Riemann fluxes over the face slots (geometry from SlotFastAcc, offsets
// formed in FP64 and rounded once); FP64 conserved variables, flux sums,
// update, pressure recovery and the dt reduction.  Approximate FP32 division
// and square root (the flags of the rectangle's MIXED kernels).
#include <cuda_runtime.h>

#include "smf_struct.cuh"
#include "smf_tiled.cuh"
#include "smf_tiled_launch.h"

namespace zg {
namespace slotmixed {

using tiled::C4;
using tiled::EosR;
using tiled::Fields;
using tiled::P5;
using R = float;

constexpr int BLOCK = 128;
// Minimum resident blocks per SM (register caps; -D overrides for sweeps)
#ifndef ZG_SLOTMX_GRAD_MINB
#define ZG_SLOTMX_GRAD_MINB 8
#endif
#ifndef ZG_SLOTMX_S2_MINB
#define ZG_SLOTMX_S2_MINB 6
#endif

static inline unsigned blocks(const SmfArgs &a) { return (unsigned)((a.smesh.n + BLOCK - 1) / BLOCK); }

__device__ __forceinline__ P5<R> ldw(const R *const p[5], int ic) {
    return P5<R>{p[0][ic], p[1][ic], p[2][ic], p[3][ic], p[4][ic]};
}
__device__ __forceinline__ void stw(R *const p[5], int ic, const P5<R> &z) {
    p[0][ic] = z.r;
    p[1][ic] = z.u;
    p[2][ic] = z.v;
    p[3][ic] = z.p;
    p[4][ic] = z.e;
}
// wall reflection (sm_fluid.cpp:69-79) for the unit normal (nx, ny)
__device__ __forceinline__ P5<R> wall_of(const P5<R> &z, R nx, R ny, int flag) {
    if (flag != BC_WALL) return z;
    P5<R> o = z;
    R d = z.u * nx + z.v * ny;
    o.u = z.u - R(2) * (nx * d);
    o.v = z.v - R(2) * (ny * d);
    return o;
}
// rotation into the face frame and back (rotate.cpp) for a unit normal
__device__ __forceinline__ void rot_in(R nx, R ny, R &u, R &v) {
    R a = u, b = v;
    u = nx * a + ny * b;
    v = -ny * a + nx * b;
}
__device__ __forceinline__ void rot_out(R nx, R ny, R &mu, R &mv) {
    R a = mu, b = mv;
    mu = nx * a - ny * b;
    mv = ny * a + nx * b;
}
__device__ __forceinline__ P5<R> recon(const P5<R> &z, const R gx[4], const R gy[4], R dx, R dy,
                                       const EosR<R> &eos) {
    P5<R> o;
    o.r = z.r + (gx[0] * dx + gy[0] * dy);
    o.u = z.u + (gx[1] * dx + gy[1] * dy);
    o.v = z.v + (gx[2] * dx + gy[2] * dy);
    o.p = z.p + (gx[3] * dx + gy[3] * dy);
    o.e = eos.energy_rP(o.r, o.p);
    return tiled::bad(o, eos) ? z : o;
}
__device__ __forceinline__ void ldg(const Fields<R> &f, int ic, R gx[4], R gy[4]) {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        gx[k] = f.gx[k][ic];
        gy[k] = f.gy[k][ic];
    }
}
__device__ __forceinline__ C4<double> ldq(const Fields<R> &f, int ic) {
    return C4<double>{f.q[0][ic], f.q[1][ic], f.q[2][ic], f.q[3][ic]};
}

// CFL time step from the FP64 conserved state (sm_fluid.cpp:104-114): the
// last block turns the minimum into dt and resets the accumulator.
__global__ void __launch_bounds__(BLOCK) k_dt(SmfArgs a, Fields<R> f) {
    int ic = blockIdx.x * BLOCK + threadIdx.x;
    unsigned long long best = 0x7FEFFFFFFFFFFFFFull;
    if (ic < a.smesh.n) {
        SlotFastAcc c(a, ic);
        P5<double> z = tiled::prim_of(ldq(f, ic), a.eos);
        double cs = a.eos.sound_speed_rP(z.r, z.p);
        double lam = c.dinc() / (sqrt(z.u * z.u + z.v * z.v) + cs);
        if (lam >= 0.0) best = dbits(lam);
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
                *a.dt_out = smin(a.CFL * dmin, a.max_dt);
                *a.dmin_bits = 0x7FEFFFFFFFFFFFFFull;
                *a.dt_ticket = 0u;
                __threadfence();
            }
        }
    }
}

// Predictor (sm_fluid.cpp:176-253): half step with the physical flux of the
// reconstructed face states from the cell's gradients gx, gy; FP64 sums,
// update and pressure recovery.
__device__ __forceinline__ void predictor(const SmfArgs &a, const Fields<R> &f, const SlotFastAcc &c, int ic,
                                          const P5<R> &zc, const R gx[4], const R gy[4]) {
    if (f.wait_in[ic] > 0) {
        stw(f.h, ic, zc);
        return;
    }
    const EosR<R> eos = tiled::eos_as<R>(a.eos);
    double F[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll 1
    for (int s = 0; s < 8; ++s) {
        FaceG g = c.face(s);
        if (g.flag == BC_UNDEFINED) continue;
        const R nx = (R)g.nx, ny = (R)g.ny;
        P5<R> zm = recon(zc, gx, gy, (R)(g.fcx - c.cx()), (R)(g.fcy - c.cy()), eos);
        rot_in(nx, ny, zm.u, zm.v);
        C4<R> lf = tiled::phys_flux(zm);
        rot_out(nx, ny, lf.mu, lf.mv);
        F[0] += (double)lf.r * g.area;
        F[1] += (double)lf.mu * g.area;
        F[2] += (double)lf.mv * g.area;
        F[3] += (double)lf.E * g.area;
    }
    const double coef = 0.5 * (*a.dt_out) / c.vol();
    C4<double> q = ldq(f, ic);
    q.r -= coef * F[0];
    q.mu -= coef * F[1];
    q.mv -= coef * F[2];
    q.E -= coef * F[3];
    P5<double> hz = tiled::prim_of(q, a.eos);
    stw(f.h, ic, tiled::bad64(hz, a.eos) ? zc : tiled::down<R>(hz));
}


// Limited least-squares gradients of the FP32 state (two passes over the
// slots; gradient.h:226-282 and 412-474) over the slot geometry built once
// per mesh change for the FAST step (slotfast::launch_grad_geometry: sg =
// (rx, ry, w nx^, w ny^) per slot, bm = the inverse least-squares matrix per
// cell) in FP64, rounded to FP32 here.  PRED: the predictor follows in the
// same thread from the gradients just computed.
template <int LIM, bool PRED>
__global__ void __launch_bounds__(BLOCK, ZG_SLOTMX_GRAD_MINB) k_grad_pre(SmfArgs a, Fields<R> f, const double4 *sg,
                                                                         const double4 *bm) {
    int ic = blockIdx.x * BLOCK + threadIdx.x;
    if (ic >= a.smesh.n) return;
    const P5<R> zc = ldw(f.w, ic);
    const R zcv[4] = {zc.r, zc.u, zc.v, zc.p};
    // the neighbour's (or the wall's) FP32 values across slot s
    auto values = [&](int s, int flag, R zn[4]) {
        P5<R> z;
        if (!is_boundary(flag)) {
            z = ldw(f.w, a.smesh.fn[8 * ic + s]);
        } else {
            const int side = s & 3;  // the axis normal of the side (SlotFastAcc::face)
            const R nx = side == 0 ? R(-1) : (side == 1 ? R(1) : R(0));
            const R ny = side == 2 ? R(-1) : (side == 3 ? R(1) : R(0));
            z = wall_of(zc, nx, ny, flag);
        }
        zn[0] = z.r;
        zn[1] = z.u;
        zn[2] = z.v;
        zn[3] = z.p;
    };
    R Fx[4] = {0, 0, 0, 0}, Fy[4] = {0, 0, 0, 0};
#pragma unroll 1
    for (int s = 0; s < 8; ++s) {
        const int flag = a.smesh.fb[8 * ic + s];
        if (flag == BC_UNDEFINED) continue;
        R zn[4];
        values(s, flag, zn);
        const double4 G = sg[8 * ic + s];
        const R wdx = (R)G.z, wdy = (R)G.w;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const R dF = zn[k] - zcv[k];
            Fx[k] += wdx * dF;
            Fy[k] += wdy * dF;
        }
    }
    const double4 Bd = bm[ic];
    const R B00 = (R)Bd.x, B01 = (R)Bd.y, B10 = (R)Bd.z, B11 = (R)Bd.w;
    R g0x[4], g0y[4], Lx[4] = {0, 0, 0, 0}, Ly[4] = {0, 0, 0, 0};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        g0x[k] = B00 * Fx[k] + B01 * Fy[k];
        g0y[k] = B10 * Fx[k] + B11 * Fy[k];
    }
#pragma unroll 1
    for (int s = 0; s < 8; ++s) {
        const int flag = a.smesh.fb[8 * ic + s];
        if (flag == BC_UNDEFINED) continue;
        R zn[4];
        values(s, flag, zn);
        const double4 G = sg[8 * ic + s];
        const R rx = (R)G.x, ry = (R)G.y, wdx = (R)G.z, wdy = (R)G.w;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const R dF_p = zn[k] - zcv[k];
            const R dF_m = R(2) * (g0x[k] * rx + g0y[k] * ry) - dF_p;
            const R dl = tiled::limit<LIM, R>(a.limiter, dF_m, dF_p) * dF_p;
            Lx[k] += wdx * dl;
            Ly[k] += wdy * dl;
        }
    }
    R gx[4], gy[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        gx[k] = B00 * Lx[k] + B01 * Ly[k];
        gy[k] = B10 * Lx[k] + B11 * Ly[k];
        f.gx[k][ic] = gx[k];
        f.gy[k][ic] = gy[k];
    }
    if constexpr (PRED) {
        SlotFastAcc c(a, ic);
        predictor(a, f, c, ic, zc, gx, gy);
    }
}

// Face-once form over the FAST step's face list (slotfast::FaceFlux): one
// thread per face, the face flux of k_faces times the face's area into the
// face's FP64 record; then per cell the records in slot order and the update
// of k_faces, with the CFL minimum of the new state for the next step's dt
// (ff.dt_next).
template <int MODE>
__global__ void __launch_bounds__(BLOCK, ZG_SLOTMX_S2_MINB) k_faces_once(SmfArgs a, Fields<R> f,
                                                                          slotfast::FaceFlux ff) {
    int t = blockIdx.x * BLOCK + threadIdx.x;
    if (t >= ff.nfaces) return;
    const int fi = ff.list[t], ic = fi >> 3, s = fi & 7;
    SlotFastAcc c(a, ic);
    const FaceG g = c.face(s);
    const EosR<R> eos = tiled::eos_as<R>(a.eos);
    const R *const *src = MODE == 1 ? const_cast<const R *const *>(f.h) : f.w;
    const P5<R> zch = ldw(src, ic);
    const int wc = MODE == 1 ? f.wait_in[ic] : 0;
    const bool bnd = is_boundary(g.flag);
    const R nx = (R)g.nx, ny = (R)g.ny;
    const P5<R> z_nh = bnd ? wall_of(zch, nx, ny, g.flag) : ldw(src, g.nb);
    const bool robust = MODE == 1 && (wc > 0 || f.wait_in[g.nb] > 0);
    P5<R> zm = zch, zp = z_nh;
    if (MODE == 1 && !robust) {
        R gx[4], gy[4];
        ldg(f, ic, gx, gy);
        double ncx, ncy;
        neib_center(c, g, s, c.cx(), c.cy(), ncx, ncy);
        zm = recon(zch, gx, gy, (R)(g.fcx - c.cx()), (R)(g.fcy - c.cy()), eos);
        if (!bnd) {
            R hx[4], hy[4];
            ldg(f, g.nb, hx, hy);
            zp = recon(z_nh, hx, hy, (R)(g.fcx - ncx), (R)(g.fcy - ncy), eos);
        } else {
            zp = wall_of(zm, nx, ny, g.flag);
        }
    }
    rot_in(nx, ny, zm.u, zm.v);
    rot_in(nx, ny, zp.u, zp.v);
    C4<R> lf = tiled::face_flux(a.flux, robust, zm, zp, eos, a.eos);
    rot_out(nx, ny, lf.mu, lf.mv);
    ff.f[t] = make_double4((double)lf.r * g.area, (double)lf.mu * g.area, (double)lf.mv * g.area,
                           (double)lf.E * g.area);
}

template <int MODE>
__global__ void __launch_bounds__(BLOCK) k_sum(SmfArgs a, Fields<R> f, slotfast::FaceFlux ff) {
    int ic = blockIdx.x * BLOCK + threadIdx.x;
    unsigned long long best = 0x7FEFFFFFFFFFFFFFull;  // bits of DBL_MAX
    if (ic < a.smesh.n) {
        const Cons F = sum_faces(ic, ff);
        const double coef = (*a.dt_out) / a.smesh.vol[ic];
        const C4<double> q0 = ldq(f, ic);
        C4<double> q = q0;
        q.r -= coef * F.r;
        q.mu -= coef * F.mu;
        q.mv -= coef * F.mv;
        q.E -= coef * F.E;
        P5<double> zn = tiled::prim_of(q, a.eos);
        if (MODE == 1) {
            const int wc = f.wait_in[ic];
            int wn = wc;
            if (tiled::bad64(zn, a.eos)) {  // isolation: keep the old state
                q = q0;
                zn = tiled::prim_of(q0, a.eos);
                wn = 3;
            } else if (wn > 0) {
                --wn;
            }
            f.wait_out[ic] = wn;
        }
        f.qn[0][ic] = q.r;
        f.qn[1][ic] = q.mu;
        f.qn[2][ic] = q.mv;
        f.qn[3][ic] = q.E;
        stw(f.wn, ic, tiled::down<R>(zn));
        if (ff.dt_next) best = cfl_bits(a, a.smesh.inc[ic], zn.r, zn.u, zn.v, zn.p);
    }
    if (ff.dt_next) commit_cfl_min<BLOCK>(a, best, ff.dt_next);  // every thread, one call site
}

void launch_faces_once(const SmfArgs &a, const Fields<R> &f, int mode, const slotfast::FaceFlux &ff, void *stream) {
    if (ff.nfaces <= 0) return;
    const unsigned nb = (unsigned)((ff.nfaces + BLOCK - 1) / BLOCK);
    if (mode == 0) k_faces_once<0><<<nb, BLOCK, 0, (cudaStream_t)stream>>>(a, f, ff);
    else k_faces_once<1><<<nb, BLOCK, 0, (cudaStream_t)stream>>>(a, f, ff);
}
void launch_sum(const SmfArgs &a, const Fields<R> &f, int mode, const slotfast::FaceFlux &ff, void *stream) {
    if (mode == 0) k_sum<0><<<blocks(a), BLOCK, 0, (cudaStream_t)stream>>>(a, f, ff);
    else k_sum<1><<<blocks(a), BLOCK, 0, (cudaStream_t)stream>>>(a, f, ff);
}

void launch_dt(const SmfArgs &a, const Fields<R> &f, void *stream) {
    k_dt<<<blocks(a), BLOCK, 0, (cudaStream_t)stream>>>(a, f);
}
template <bool PRED>
static void grad_pred(const SmfArgs &a, const Fields<R> &f, const double4 *sg, const double4 *bm, cudaStream_t s) {
    switch (a.limiter) {  // the common limiters compiled in, the others at run time
        case LIM_VANALBADA1: k_grad_pre<LIM_VANALBADA1, PRED><<<blocks(a), BLOCK, 0, s>>>(a, f, sg, bm); break;
        case LIM_MC: k_grad_pre<LIM_MC, PRED><<<blocks(a), BLOCK, 0, s>>>(a, f, sg, bm); break;
        case LIM_MINMOD: k_grad_pre<LIM_MINMOD, PRED><<<blocks(a), BLOCK, 0, s>>>(a, f, sg, bm); break;
        default: k_grad_pre<-1, PRED><<<blocks(a), BLOCK, 0, s>>>(a, f, sg, bm); break;
    }
}
void launch_grad(const SmfArgs &a, const Fields<R> &f, const double4 *sg, const double4 *bm, bool predictor,
                 void *stream) {
    if (predictor) grad_pred<true>(a, f, sg, bm, (cudaStream_t)stream);
    else grad_pred<false>(a, f, sg, bm, (cudaStream_t)stream);
}

}  // namespace slotmixed
}  // namespace zg
