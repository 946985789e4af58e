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
#define ZG_SLOT_GRAD_MINB 5
#endif
#ifndef ZG_SLOT_S1_MINB
#define ZG_SLOT_S1_MINB 6
#endif
#ifndef ZG_SLOT_S2_MINB
#define ZG_SLOT_S2_MINB 5
#endif
constexpr int GM = ZG_SLOT_GRAD_MINB, S1M = ZG_SLOT_S1_MINB, S2M = ZG_SLOT_S2_MINB;

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
void launch_stage1(const SmfArgs &a, void *stream) {
    k_stage1<SlotFastAcc, BLOCK, S1M><<<blocks(a), BLOCK, 0, (cudaStream_t)stream>>>(a);
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

// the face fluxes of cell ic summed in slot order
__device__ __forceinline__ Cons sum_faces(int ic, const FaceFlux &ff) {
    Cons F{0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int s = 0; s < 8; ++s) {
        const int x = ff.fidx[8 * ic + s];
        if (x == FACE_NONE) continue;
        const double4 v = ff.f[x >= 0 ? x : -x - 1];
        if (x >= 0) {
            F.r += v.x;
            F.mu += v.y;
            F.mv += v.z;
            F.E += v.w;
        } else {
            F.r -= v.x;
            F.mu -= v.y;
            F.mv -= v.z;
            F.E -= v.w;
        }
    }
    return F;
}

// k_stage2's update (sm_fluid.cpp:342-366) from the summed face fluxes
__global__ void __launch_bounds__(BLOCK) k_stage2_sum(SmfArgs a, FaceFlux ff) {
    int ic = blockIdx.x * BLOCK + threadIdx.x;
    if (ic >= a.smesh.n) return;
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
}

// k_heun's update from the summed face fluxes
template <bool FINAL>
__global__ void __launch_bounds__(BLOCK) k_heun_sum(SmfArgs a, PrimPtr zin, PrimPtr zout, FaceFlux ff) {
    int ic = blockIdx.x * BLOCK + threadIdx.x;
    if (ic >= a.smesh.n) return;
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
    store_prim(zout, ic, p_from_q(q, a.eos));
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
