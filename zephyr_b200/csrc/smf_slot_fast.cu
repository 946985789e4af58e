// smf_slot_fast.cu -- the FAST form of the step on an adaptive rectangle: the
// kernels of smf_struct.cuh over SlotFastAcc (face geometry from the cell's
// centre and level instead of five stored arrays per slot), compiled with
// fused multiply-adds and register caps, with the corrector and the Heun
// stages face-once.  Results match the parity form to rounding (not bit for
// bit).
#include <cuda_runtime.h>

#include "smf_struct.cuh"

namespace zg {
namespace slotfast {

constexpr int BLOCK = 128;
// Minimum resident blocks per SM: register caps chosen by timing the AMR
// blast (512^2, 3 levels) over a sweep on a B200 (-D overrides)
#ifndef ZG_SLOT_GRAD_MINB
#define ZG_SLOT_GRAD_MINB 6
#endif
#ifndef ZG_SLOT_S2_MINB
#define ZG_SLOT_S2_MINB 5
#endif
constexpr int GM = ZG_SLOT_GRAD_MINB, S2M = ZG_SLOT_S2_MINB;

static inline unsigned blocks(const SmfArgs &a) { return (unsigned)((a.smesh.n + BLOCK - 1) / BLOCK); }

void launch_dt(const SmfArgs &a, PrimPtr z, void *stream) {
    SmfArgs b = a;
    b.z = z;
    k_dt<SlotFastAcc, BLOCK><<<blocks(a), BLOCK, 0, (cudaStream_t)stream>>>(b);
}
// the face-flux kernels per flux family (HLLC, HLL, the general switch)
#define ZG_FLUX_FAMILY(FN, ...)                                        \
    do {                                                               \
        if (a.flux == FLUX_HLLC) FN<FLUX_HLLC>(__VA_ARGS__);           \
        else if (a.flux == FLUX_HLL) FN<FLUX_HLL>(__VA_ARGS__);        \
        else FN<-1>(__VA_ARGS__);                                      \
    } while (0)
template <int FX>
static void flux1_fx(const SmfArgs &a, void *stream) {
    k_flux1<SlotFastAcc, BLOCK, S2M, FX><<<blocks(a), BLOCK, 0, (cudaStream_t)stream>>>(a);
}

void launch_flux1(const SmfArgs &a, void *stream) { ZG_FLUX_FAMILY(flux1_fx, a, stream); }
void launch_grad(const SmfArgs &a, PrimPtr z, void *stream) {
    k_grad<SlotFastAcc, BLOCK, GM><<<blocks(a), BLOCK, 0, (cudaStream_t)stream>>>(a, z);
}

// --- least-squares gradients over precomputed geometry ------------------------
// lsm_limited_2pass (smf_struct.cuh, gradient.h:226-282 with the limiting of
// sm_fluid.cpp:143-174) with the slot geometry, its weights and the inverse
// matrix computed once per mesh change instead of in both passes of every
// gradient evaluation.
__global__ void __launch_bounds__(BLOCK) k_grad_geometry(SmfArgs a, double4 *sg, double4 *bm) {
    int ic = blockIdx.x * BLOCK + threadIdx.x;
    if (ic >= a.smesh.n) return;
    SlotFastAcc c(a, ic);
    const double pcx = c.cx(), pcy = c.cy();
    double A00 = 0.0, A01 = 0.0, A10 = 0.0, A11 = 0.0;
#pragma unroll 1
    for (int s = 0; s < 8; ++s) {
        const FaceG g = c.face(s);
        if (g.flag == BC_UNDEFINED) {
            sg[8 * ic + s] = make_double4(0.0, 0.0, 0.0, 0.0);
            continue;
        }
        double ncx, ncy;
        neib_center(c, g, s, pcx, pcy, ncx, ncy);
        const double rx = ncx - pcx, ry = ncy - pcy;
        const double d = rx * g.nx + ry * g.ny, nxx = d * g.nx, nyy = d * g.ny;
        const double w = g.area / cube_rn(sqrt(nxx * nxx + nyy * nyy));
        const double wdx = w * nxx, wdy = w * nyy;
        A00 += wdx * rx;
        A01 += wdx * ry;
        A10 += wdy * rx;
        A11 += wdy * ry;
        sg[8 * ic + s] = make_double4(rx, ry, wdx, wdy);
    }
    if (fabs(A11) < 1e-8) A11 = 1.0;  // 1-D case (gradient.h:270-272)
    const double det = A11 * A00 + (-A01) * A10, inv = 1.0 / det;
    bm[ic] = make_double4(A11 * inv, (-A01) * inv, (-A10) * inv, A00 * inv);
}

// 1/x: Newton-Raphson (y <- y + y (1 - x y), two steps; P. Markstein, IBM
// J. Res. Dev. 34(1), 1990) from the hardware's approximate reciprocal
// (PTX rcp.approx.ftz.f64); within 2 ulp of 1/x for normal finite x
__device__ __forceinline__ double rcp2(double x) {
    double y;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    double e = fma(-x, y, 1.0);
    y = fma(y, e, y);
    e = fma(-x, y, 1.0);
    return fma(y, e, y);
}
// limiter2 (limiter.cxx binary forms) with its divisions as reciprocals for
// the common limiters, the others as limiter2
__device__ __forceinline__ double limiter_rcp(int kind, double a, double b) {
    switch (kind) {
        case LIM_VANALBADA1:
            if (a * b <= 0.0) return 0.0;
            if (b == 0.0) return 1.0;
            return a * (a + b) * rcp2(a * a + b * b);
        case LIM_MC:
            return b == 0.0 ? limiter2(kind, a, b) : lim_MC1(a * rcp2(b));
        case LIM_MINMOD:
            if (a * b <= 0.0) return 0.0;
            return smin(a * rcp2(b), 1.0);
        default: return limiter2(kind, a, b);
    }
}

// the neighbour's (or the boundary's) primitive values across slot s
__device__ __forceinline__ void slot_values(const SmfArgs &a, const PrimPtr &z, const Prim &zc, int ic, int s,
                                            int flag, double zn[4]) {
    Prim p;
    if (!is_boundary(flag)) {
        const int nb = a.smesh.fn[8 * ic + s];
        zn[0] = z.r[nb];
        zn[1] = z.u[nb];
        zn[2] = z.v[nb];
        zn[3] = z.p[nb];
        return;
    }
    const int side = s & 3;  // the axis normal of the side (SlotFastAcc::face)
    const double nx = side == 0 ? -1.0 : (side == 1 ? 1.0 : (side == 2 ? -0.0 : 0.0));
    const double ny = side == 0 ? -0.0 : (side == 1 ? 0.0 : (side == 2 ? -1.0 : 1.0));
    p = boundary_value(zc, nx, ny, flag);
    zn[0] = p.r;
    zn[1] = p.u;
    zn[2] = p.v;
    zn[3] = p.p;
}

// PRED: the predictor of the predictor-corrector scheme (k_stage1,
// sm_fluid.cpp:176-253) follows in the same thread from the gradients just
// computed, into a.zhalf.
template <bool PRED>
__global__ void __launch_bounds__(BLOCK, GM) k_grad_pre(SmfArgs a, PrimPtr z, const double4 *sg, const double4 *bm) {
    int ic = blockIdx.x * BLOCK + threadIdx.x;
    if (ic >= a.smesh.n) return;
    const Prim zc = load_prim(z, ic);
    const double zcv[4] = {zc.r, zc.u, zc.v, zc.p};
    double Fx[4] = {0.0, 0.0, 0.0, 0.0}, Fy[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll 1
    for (int s = 0; s < 8; ++s) {
        const int flag = a.smesh.fb[8 * ic + s];
        if (flag == BC_UNDEFINED) continue;
        double zn[4];
        slot_values(a, z, zc, ic, s, flag, zn);
        const double4 G = sg[8 * ic + s];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const double dF = zn[k] - zcv[k];
            Fx[k] += G.z * dF;
            Fy[k] += G.w * dF;
        }
    }
    const double4 B = bm[ic];
    double g0x[4], g0y[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        g0x[k] = B.x * Fx[k] + B.y * Fy[k];
        g0y[k] = B.z * Fx[k] + B.w * Fy[k];
    }
    double Lx[4] = {0.0, 0.0, 0.0, 0.0}, Ly[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll 1
    for (int s = 0; s < 8; ++s) {
        const int flag = a.smesh.fb[8 * ic + s];
        if (flag == BC_UNDEFINED) continue;
        double zn[4];
        slot_values(a, z, zc, ic, s, flag, zn);
        const double4 G = sg[8 * ic + s];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const double dF_p = zn[k] - zcv[k];
            const double du_n = g0x[k] * G.x + g0y[k] * G.y;
            const double dF_m = 2.0 * du_n - dF_p;
            const double dF_lim = limiter_rcp(a.limiter, dF_m, dF_p) * dF_p;
            Lx[k] += G.z * dF_lim;
            Ly[k] += G.w * dF_lim;
        }
    }
    double gx[4], gy[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        gx[k] = B.x * Lx[k] + B.y * Ly[k];
        gy[k] = B.z * Lx[k] + B.w * Ly[k];
        a.gx[k][ic] = gx[k];
        a.gy[k][ic] = gy[k];
    }
    if constexpr (PRED) {
        if (a.wait_in[ic] > 0) {
            store_prim(a.zhalf, ic, zc);
            return;
        }
        SlotFastAcc c(a, ic);
        const double dt = finalize_dt(a), pcx = c.cx(), pcy = c.cy();
        Cons q = q_from_p(zc);
        Cons F{0.0, 0.0, 0.0, 0.0};
#pragma unroll 1
        for (int s = 0; s < 8; ++s) {
            const FaceG g = c.face(s);
            if (g.flag == BC_UNDEFINED) continue;
            const double dx = g.fcx - pcx, dy = g.fcy - pcy;
            Prim zm;  // extrap (face_extra.h:135-163)
            zm.r = zc.r + (gx[0] * dx + gy[0] * dy);
            zm.u = zc.u + (gx[1] * dx + gy[1] * dy);
            zm.v = zc.v + (gx[2] * dx + gy[2] * dy);
            zm.p = zc.p + (gx[3] * dx + gy[3] * dy);
            zm.e = a.eos.energy_rP(zm.r, zm.p);
            if (is_bad(zm, a.eos)) zm = zc;
            double cs, sn;
            frame<SlotFastAcc>(g, cs, sn);
            rot_local(zm.u, zm.v, cs, sn);
            Cons lf = flux_from_p(zm);
            rot_global(lf.mu, lf.mv, cs, sn);
            add_area(F, lf, g.area);
        }
        update(q, 0.5 * dt / c.vol(), F);
        Prim h = p_from_q(q, a.eos);
        if (is_bad(h, a.eos)) h = zc;
        store_prim(a.zhalf, ic, h);
    }
}

void launch_grad_geometry(const SmfArgs &a, double4 *sg, double4 *bm, void *stream) {
    k_grad_geometry<<<blocks(a), BLOCK, 0, (cudaStream_t)stream>>>(a, sg, bm);
}
void launch_grad_pre(const SmfArgs &a, PrimPtr z, const double4 *sg, const double4 *bm, bool predictor,
                     void *stream) {
    cudaStream_t st = (cudaStream_t)stream;
    if (predictor) k_grad_pre<true><<<blocks(a), BLOCK, 0, st>>>(a, z, sg, bm);
    else k_grad_pre<false><<<blocks(a), BLOCK, 0, st>>>(a, z, sg, bm);
}

// --- face-once corrector / Heun stages --------------------------------------
// One thread per face of the list (computes_face in smf_struct.cuh decides
// which cell evaluates a face): the corrector's face flux into the slot.
template <int FX, bool HEUN>
__global__ void __launch_bounds__(BLOCK, S2M) k_faces_once(SmfArgs a, PrimPtr zin, FaceFlux ff) {
    int t = blockIdx.x * BLOCK + threadIdx.x;
    if (t >= ff.nfaces) return;
    const int f = ff.list[t], ic = f >> 3, s = f & 7;
    SlotFastAcc c(a, ic);
    const FaceG g = c.face(s);
    const Prim zc = load_prim(zin, ic);
    const int wc = HEUN ? 0 : a.wait_in[ic];
    Cons lf = corrector_face<FX>(a, zin, HEUN ? nullptr : a.wait_in, c, s, g, zc, c.cx(), c.cy(), wc);
    ff.f[t] = make_double4(lf.r, lf.mu, lf.mv, lf.E);
}

// k_stage2's update (sm_fluid.cpp:342-366) from the summed face fluxes.
// With ff.dt_next, every thread of the block (those past the last cell with
// the neutral value) reaches the one block-wide CFL minimum at the end.
__global__ void __launch_bounds__(BLOCK) k_stage2_sum(SmfArgs a, FaceFlux ff) {
    int ic = blockIdx.x * BLOCK + threadIdx.x;
    unsigned long long best = 0x7FEFFFFFFFFFFFFFull;  // bits of DBL_MAX
    if (ic < a.smesh.n) {
        const double dt = finalize_dt(a);
        const Prim zc = load_prim(a.z, ic);
        const int wc = a.wait_in[ic];
        Cons q = q_from_p(zc);
        const Cons F = sum_faces(ic, ff);
        update(q, dt / a.smesh.vol[ic], F);
        Prim n = p_from_q(q, a.eos);
        int wn = wc;
        if (is_bad(n, a.eos)) {
            n = zc;
            wn = 3;
        } else if (wn > 0) {
            --wn;
        }
        store_prim(a.znext, ic, n);
        a.wait_out[ic] = wn;
        if (ff.dt_next) best = cfl_bits(a, a.smesh.inc[ic], n.r, n.u, n.v, n.p);
    }
    if (ff.dt_next) commit_cfl_min<BLOCK>(a, best, ff.dt_next);
}

// k_heun's update from the summed face fluxes (the final stage with
// ff.dt_next: the CFL minimum as in k_stage2_sum)
template <bool FINAL>
__global__ void __launch_bounds__(BLOCK) k_heun_sum(SmfArgs a, PrimPtr zin, PrimPtr zout, FaceFlux ff) {
    int ic = blockIdx.x * BLOCK + threadIdx.x;
    unsigned long long best = 0x7FEFFFFFFFFFFFFFull;
    if (ic < a.smesh.n) {
        const double dt = finalize_dt(a);
        Cons q = q_from_p(load_prim(zin, ic));
        const Cons F = sum_faces(ic, ff);
        update(q, dt / a.smesh.vol[ic], F);
        if (FINAL) {
            Cons q0 = q_from_p(load_prim(a.z, ic));
            q.r = 0.5 * (q0.r + q.r);
            q.mu = 0.5 * (q0.mu + q.mu);
            q.mv = 0.5 * (q0.mv + q.mv);
            q.E = 0.5 * (q0.E + q.E);
        }
        const Prim n = p_from_q(q, a.eos);
        store_prim(zout, ic, n);
        if (FINAL && ff.dt_next) best = cfl_bits(a, a.smesh.inc[ic], n.r, n.u, n.v, n.p);
    }
    if (FINAL && ff.dt_next) commit_cfl_min<BLOCK>(a, best, ff.dt_next);
}

template <int FX>
static void faces_fx(const SmfArgs &a, PrimPtr zin, FaceFlux ff, bool heun, void *stream) {
    if (ff.nfaces <= 0) return;
    cudaStream_t st = (cudaStream_t)stream;
    const unsigned nb = (unsigned)((ff.nfaces + BLOCK - 1) / BLOCK);
    if (heun) k_faces_once<FX, true><<<nb, BLOCK, 0, st>>>(a, zin, ff);
    else k_faces_once<FX, false><<<nb, BLOCK, 0, st>>>(a, zin, ff);
}
void launch_stage2_faces(const SmfArgs &a, FaceFlux ff, void *stream) {
    ZG_FLUX_FAMILY(faces_fx, a, a.zhalf, ff, false, stream);
}
void launch_stage2_sum(const SmfArgs &a, FaceFlux ff, void *stream) {
    k_stage2_sum<<<blocks(a), BLOCK, 0, (cudaStream_t)stream>>>(a, ff);
}
void launch_heun_faces(const SmfArgs &a, PrimPtr zin, FaceFlux ff, void *stream) {
    ZG_FLUX_FAMILY(faces_fx, a, zin, ff, true, stream);
}
void launch_heun_sum(const SmfArgs &a, PrimPtr zin, PrimPtr zout, bool final, FaceFlux ff, void *stream) {
    cudaStream_t st = (cudaStream_t)stream;
    if (final) k_heun_sum<true><<<blocks(a), BLOCK, 0, st>>>(a, zin, zout, ff);
    else k_heun_sum<false><<<blocks(a), BLOCK, 0, st>>>(a, zin, zout, ff);
}

// Refinement flags by the density-gradient criterion |grad rho| h / rho (h =
// sqrt(volume)): 1 above `refine`, -1 below `coarsen`, 0 between.  The
// gradient is the unlimited least-squares one (gradient.h:226-282 for the
// density alone): a limited slope vanishes next to an isolated jump, which is
// where refinement is wanted.
__global__ void __launch_bounds__(BLOCK) k_grad_flags(SmfArgs a, int *flags, double refine, double coarsen) {
    int ic = blockIdx.x * BLOCK + threadIdx.x;
    if (ic >= a.smesh.n) return;
    SlotFastAcc c(a, ic);
    const double rc = a.z.r[ic];
    double A00 = 0.0, A01 = 0.0, A10 = 0.0, A11 = 0.0, Fx = 0.0, Fy = 0.0;
#pragma unroll 1
    for (int s = 0; s < 8; ++s) {
        FaceG g = c.face(s);
        if (g.flag == BC_UNDEFINED) continue;
        const double rn = is_boundary(g.flag) ? rc : a.z.r[g.nb];
        double ncx, ncy;
        neib_center(c, g, s, c.cx(), c.cy(), ncx, ncy);
        const double rx = ncx - c.cx(), ry = ncy - c.cy();
        const double d = rx * g.nx + ry * g.ny, nxx = d * g.nx, nyy = d * g.ny;
        const double an = sqrt(nxx * nxx + nyy * nyy), w = g.area / (an * an * an);
        A00 += w * nxx * rx;
        A01 += w * nxx * ry;
        A10 += w * nyy * rx;
        A11 += w * nyy * ry;
        Fx += w * (rn - rc) * nxx;
        Fy += w * (rn - rc) * nyy;
    }
    if (fabs(A11) < 1e-8) A11 = 1.0;
    const double inv = 1.0 / (A11 * A00 - A01 * A10);
    const double gx = (A11 * Fx - A01 * Fy) * inv, gy = (-A10 * Fx + A00 * Fy) * inv;
    const double crit = sqrt(gx * gx + gy * gy) * sqrt(c.vol()) / rc;
    flags[ic] = crit > refine ? 1 : (crit < coarsen ? -1 : 0);
}
void launch_grad_flags(const SmfArgs &a, int *flags, double refine, double coarsen, void *stream) {
    k_grad_flags<<<blocks(a), BLOCK, 0, (cudaStream_t)stream>>>(a, flags, refine, coarsen);
}

}  // namespace slotfast
}  // namespace zg
