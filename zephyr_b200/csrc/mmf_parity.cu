// mmf_parity.cu -- kernels of zephyr's multi-material first-order step
// MmFluid::update (math/solver/mm_fluid.cpp:112-171, DirSplit::NONE,
// accuracy 1) on a rectangle: CFL time step, PLIC interface reconstruction,
// and the face loop with mixture HLLC / composite Riemann fluxes and the
// PT-equilibrium closure of every updated cell.  One thread per cell; each
// cell evaluates its own faces in the reference's order (gather form).
// Compiled with -fmad=false: results agree bit for bit with the reference.
#include <cuda_runtime.h>

#include <algorithm>

#include "mmf_pure.cuh"

namespace zg {
namespace mmf {

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
    if (ic == 0 && !a.keep_lists) {  // empty work lists for this step's face loop
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
    } else if (a.crp == CRP_MUSCL) {
        a_sig = MM_NAN;  // alpha_sigma has no face fraction for MUSCL (mm_fluid.cpp:245-250)
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
    if (a.crp == CRP_MUSCL && !crp_plain(zm, zp, iA)) {
        atomicOr(a.err, 2);  // calc_crp_flux's assert on a_sig rejects the NaN (mm_fluid.cpp:276)
        return qv_zero<NM>();
    }
    return crp_flux(a.mix, zm, zp, hL, hR, iA, a_sig, dt, bad);
}

// Rotate::to_local of a velocity (rotate.cpp:7-41); axis normals are unit
// vectors, so normalized() leaves them unchanged.
__device__ __forceinline__ void to_local(double cs, double sn, double vx, double vy, double &ox, double &oy) {
    ox = cs * vx + sn * vy + 0.0 * 0.0;
    oy = -sn * vx + cs * vy + 0.0 * 0.0;
}
// One part of a face of the first-order face loop for two threads: the face
// flux of calc_flux as face_term computes it, with a composite flux split by
// crp_part.  Part 0 writes the plain flux (pure states on both sides, or
// crp_flux's plain-HLLC case) or its part of the composite one, with the
// face's a_sig and flags (bit 0: composite, bit 1: part 0 is fA); part 1
// writes the other part of a composite flux.  Rotation to the global frame
// and the face area follow in k_crp_update_parts.
__device__ void face_part(const MmArgs &a, int ic, int s, int f, int part, double dt, bool &bad) {
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
    const double hL = V_c / S, hR = V_n / S;
    // calc_flux (mm_fluid.cpp:347-371): the plain-HLLC cases
    bool plain = a.crp == CRP_NONE || (frac_index(zm.b) >= 0 && frac_index(zp.b) >= 0);
    int iA = 0;
    double a_sig = 0.0;
    if (!plain) {
        iA = master_component(zm, zp);
        double a_L = alpha_rt(zm, iA), a_R = alpha_rt(zp, iA);
        if (a.crp == CRP_V3) {
            a_sig = face_fraction_v3(a_L, a_R);
        } else if (a.crp == CRP_V5) {
            a_sig = face_fraction_v5(a_L, a_R);
        } else if (a.crp == CRP_VS) {
            a_sig = face_fraction_s(a_L, a_R);
        } else if (a.crp == CRP_MUSCL) {
            a_sig = MM_NAN;  // alpha_sigma has no face fraction for MUSCL (mm_fluid.cpp:245-250)
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
            double csn = g.nx * nx + g.ny * ny + 0.0 * 0.0;
            a_sig = between(average_flux(upwind ? a_L : a_R, csn, cfl), a_L, a_R);
        }
        plain = crp_plain(zm, zp, iA);
    }
    double *out = a.fbuf + ((size_t)f * 2 + part) * (4 + NM);
    QVd<NM> lf;
    if (!plain && a.crp == CRP_MUSCL) {
        atomicOr(a.err, 2);  // calc_crp_flux's assert on a_sig rejects the NaN (mm_fluid.cpp:276)
        if (part == 0) a.fflag[f] = 0;
        lf = qv_zero<NM>();
    } else if (plain) {
        if (part != 0) return;
        lf = hllc(a.mix, zm, zp, bad);
        a.fflag[f] = 0;
    } else {
        bool isA = true;
        lf = crp_part(a.mix, zm, zp, hL, hR, iA, a_sig, dt, part, isA, bad);
        if (part == 0) {
            a.fsig[f] = a_sig;
            a.fflag[f] = 1 | (isA ? 2 : 0);
        }
    }
#pragma unroll
    for (int k = 0; k < 4 + NM; ++k) out[k] = lf.a[k];
}

// --- work lists ------------------------------------------------------------
constexpr int LIST_BLOCKS = 148 * 4;

// Cells next to a mixed state, first order: two threads per face, in
// different warps (warp 2w + p takes part p of the faces of warp pair w), so
// the two sub-fluxes of a composite flux run side by side.
__global__ void __launch_bounds__(BLOCK) k_crp_parts(MmArgs a) {
    const double dt = a.dt_scale * *a.dt_out;
    const int faces = 4 * a.counts[0];
    const int tasks = 2 * ((faces + 31) & ~31);
    for (int t = blockIdx.x * BLOCK + threadIdx.x; t < tasks; t += gridDim.x * BLOCK) {
        const int w = t >> 5, part = w & 1, f = ((w >> 1) << 5) + (t & 31);
        if (f >= faces || skip_face(a.dir, f & 3)) continue;
        bool bad = false;
        face_part(a, a.list_crp[f >> 2], f & 3, f, part, dt, bad);
        if (bad) atomicOr(a.err, 1);
    }
}
// Per listed cell: each face's flux from its parts (blend(a_sig, fA, fB) of
// calc_crp_flux, mm_fluid.cpp:266-345), turned back to the global frame and
// multiplied by the area as face_term does, summed in slot order; update
// and closure as in k_crp_update.
__global__ void __launch_bounds__(BLOCK) k_crp_update_parts(MmArgs a) {
    const double dt = a.dt_scale * *a.dt_out;
    const int count = a.counts[0];
    for (int k = blockIdx.x * BLOCK + threadIdx.x; k < count; k += gridDim.x * BLOCK) {
        int ic = a.list_crp[k];
        StructAcc c(a.mesh, ic);
        MSt<NM> zc = load(a.z, ic);
        QVd<NM> flux = qv_zero<NM>();
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            if (skip_face(a.dir, s)) continue;
            const int f = 4 * k + s;
            const double *p0 = a.fbuf + (size_t)f * 2 * (4 + NM), *p1 = p0 + (4 + NM);
            const int fl = a.fflag[f];
            QVd<NM> lf;
            if (fl & 1) {
                QVd<NM> fA, fB;
#pragma unroll
                for (int j = 0; j < 4 + NM; ++j) {
                    fA.a[j] = (fl & 2) ? p0[j] : p1[j];
                    fB.a[j] = (fl & 2) ? p1[j] : p0[j];
                }
                lf = blend(a.fsig[f], fA, fB);
            } else {
#pragma unroll
                for (int j = 0; j < 4 + NM; ++j) lf.a[j] = p0[j];
            }
            const FaceG g = c.face(s);
            const double cs = g.nx, sn = g.ny;
            // Rotate::to_global of the momentum (rotate.cpp:43-77)
            double mx = cs * lf.a[1] + -sn * lf.a[2] + 0.0 * 0.0;
            double my = sn * lf.a[1] + cs * lf.a[2] + 0.0 * 0.0;
            lf.a[1] = mx;
            lf.a[2] = my;
            const double S = g.area;
#pragma unroll
            for (int j = 0; j < 4 + NM; ++j) flux.a[j] += lf.a[j] * S;
        }
        QVd<NM> q = q_of(zc);
        double coef = dt / a.mesh.vol;
#pragma unroll
        for (int j = 0; j < 4 + NM; ++j) q.a[j] -= coef * flux.a[j];
        if (q.a[0] < 0.0) atomicOr(a.err, 1);  // the reference throws (mm_fluid.cpp:431-433)
        store(a.znext, ic, state_of_q(a.mix, q, zc.P, zc.T, zc.r));
    }
}
__global__ void __launch_bounds__(BLOCK) k_crp_update(MmArgs a) {
    const double dt = a.dt_scale * *a.dt_out;
    const int count = a.counts[0];
    for (int k = blockIdx.x * BLOCK + threadIdx.x; k < count; k += gridDim.x * BLOCK) {
        int ic = a.list_crp[k];
        MSt<NM> zc = load(a.z, ic);
        QVd<NM> flux = qv_zero<NM>();
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            if (skip_face(a.dir, s)) continue;
#pragma unroll
            for (int j = 0; j < 4 + NM; ++j) flux.a[j] += a.fbuf[(size_t)(4 * k + s) * (4 + NM) + j];
        }
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

// ---------------------------------------------------------------------------
// Second order (MmFluid::integrate with accuracy 2, mm_fluid.cpp:152-168).
// The state as an array of NG components; the reference's mmf::PState also
// carries vz and the unused fraction / density slots, whose gradients are 0
// and NaN and never reach a result here.
__device__ __forceinline__ void to_arr(const MSt<NM> &z, double *v) {
    v[0] = z.rho;
    v[1] = z.vx;
    v[2] = z.vy;
    v[3] = z.P;
    v[4] = z.e;
    v[5] = z.T;
#pragma unroll
    for (int i = 0; i < NM; ++i) {
        v[6 + i] = z.b.f[i];
        v[6 + NM + i] = z.r[i];
    }
}
__device__ __forceinline__ MSt<NM> from_arr(const double *v) {
    MSt<NM> z;
    z.rho = v[0];
    z.vx = v[1];
    z.vy = v[2];
    z.P = v[3];
    z.e = v[4];
    z.T = v[5];
#pragma unroll
    for (int i = 0; i < NM; ++i) {
        z.b.f[i] = v[6 + i];
        z.r[i] = v[6 + NM + i];
    }
    return z;
}

// boundary_value (mm_fluid.cpp:88-97) of a state for slot geometry g
__device__ __forceinline__ MSt<NM> ghost(const MSt<NM> &zc, const FaceG &g) {
    MSt<NM> zn = zc;
    if (g.flag == BC_WALL) wall_velocity(g, zc.vx, zc.vy, zn.vx, zn.vy);
    return zn;
}

// compute_grad (mm_fluid.cpp:439-467): in CRP modes zero gradients in and
// next to mixed cells; else gradient::LSM and gradient::limiting
// (gradient.h:226-282, 412-474) on every component, in the 2-D reduction of
// the 3x3 system (A(i,2), A(2,j) exact zeros, A(2,2) set to 1).
// component k of the to_arr order, selected without indexing the parameter
// block dynamically
__device__ __forceinline__ double *comp_ptr(const MmField &f, int k) {
    double *p = f.rho;
    if (k == 1) p = f.vx;
    if (k == 2) p = f.vy;
    if (k == 3) p = f.P;
    if (k == 4) p = f.e;
    if (k == 5) p = f.T;
#pragma unroll
    for (int i = 0; i < NM; ++i) {
        if (k == 6 + i) p = f.b[i];
        if (k == 6 + NM + i) p = f.r[i];
    }
    return p;
}
__device__ __forceinline__ double *grad_ptr(double *const *g, int k) {
    double *p = g[0];
#pragma unroll
    for (int j = 1; j < NG; ++j)
        if (k == j) p = g[j];
    return p;
}

// The face geometry (weights, offsets, the 2x2 system) is formed once; the
// components then go one at a time through the same least-squares and
// limiting arithmetic, so only one component's neighbour differences are
// live at a time.
__global__ void __launch_bounds__(BLOCK) k_grad2(MmArgs a) {
    const int ic = blockIdx.x * BLOCK + threadIdx.x;
    if (ic >= a.mesh.n) return;
    StructAcc c(a.mesh, ic);
    bool set_zero = false;
    if (a.crp != CRP_NONE) {
        Frac<NM> b;
#pragma unroll
        for (int i = 0; i < NM; ++i) b.f[i] = a.z.b[i][ic];
        set_zero = frac_index(b) < 0;
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            FaceG g = c.face(s);
#pragma unroll
            for (int i = 0; i < NM; ++i) b.f[i] = a.z.b[i][g.nb];
            if (frac_index(b) < 0) set_zero = true;
        }
    }
    if (set_zero) {
#pragma unroll
        for (int k = 0; k < NG; ++k) {
            a.gx[k][ic] = 0.0;
            a.gy[k][ic] = 0.0;
        }
        return;
    }
    const double pcx = c.cx(), pcy = c.cy();
    double wv[4], drx[4], dry[4], drnx[4], drny[4], gvx[4], gvy[4];
    int nb[4];
    bool bnd[4];
    const double zvx = a.z.vx[ic], zvy = a.z.vy[ic];
    double A00 = 0.0, A01 = 0.0, A10 = 0.0, A11 = 0.0;
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        FaceG g = c.face(s);
        nb[s] = g.nb;
        bnd[s] = is_boundary(g.flag);
        gvx[s] = zvx;  // boundary_value: the cell's own state, walls reflect the velocity
        gvy[s] = zvy;
        if (g.flag == BC_WALL) wall_velocity(g, zvx, zvy, gvx[s], gvy[s]);
        double ncx, ncy;
        neib_center(c, g, s, pcx, pcy, ncx, ncy);
        const double rx = ncx - pcx, ry = ncy - pcy;
        const double d = rx * g.nx + ry * g.ny;
        const double nxx = d * g.nx, nyy = d * g.ny;
        const double w = 1.0 * g.area / cube_rn(sqrt(nxx * nxx + nyy * nyy));
        const double wdx = w * nxx, wdy = w * nyy;
        A00 += wdx * rx;
        A01 += wdx * ry;
        A10 += wdy * rx;
        A11 += wdy * ry;
        wv[s] = w;
        drx[s] = rx;
        dry[s] = ry;
        drnx[s] = nxx;
        drny[s] = nyy;
    }
    if (fabs(A11) < 1e-8) A11 = 1.0;
    const double det = A11 * A00 + (-A01) * A10;
    const double inv = 1.0 / det;
    const double B00 = A11 * inv, B01 = (-A01) * inv, B10 = (-A10) * inv, B11 = A00 * inv;
#pragma unroll 2  // two components in flight: measured 6 % faster than one
    for (int k = 0; k < NG; ++k) {
        const double *f = comp_ptr(a.z, k);
        const double zk = f[ic];
        double dn[4], Fx = 0.0, Fy = 0.0;
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            double zn = bnd[s] ? zk : f[nb[s]];
            if (bnd[s] && k == 1) zn = gvx[s];
            if (bnd[s] && k == 2) zn = gvy[s];
            const double dF = zn - zk;
            dn[s] = dF;
            Fx += wv[s] * dF * drnx[s];
            Fy += wv[s] * dF * drny[s];
        }
        const double g0x = B00 * Fx + B01 * Fy;
        const double g0y = B10 * Fx + B11 * Fy;
        double lx = 0.0, ly = 0.0;
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            const double dF_p = dn[s];
            const double du_n = g0x * drx[s] + g0y * dry[s];
            const double dF_m = 2.0 * du_n - dF_p;
            const double dF_lim = limiter2(a.limiter, dF_m, dF_p) * dF_p;
            lx += wv[s] * dF_lim * drnx[s];
            ly += wv[s] * dF_lim * drny[s];
        }
        grad_ptr(a.gx, k)[ic] = B00 * lx + B01 * ly;
        grad_ptr(a.gy, k)[ic] = B10 * lx + B11 * ly;
    }
}

// MmFluid::fractions_grad (mm_fluid.cpp:469-482), the volume-fraction
// gradients of CrpMode::MUSCL: gradient::LSM and gradient::limiting
// (gradient.h:226-282, 412-474) of PState::volume_fractions (models.cpp:
// 239-249: beta_i rho / rho_i where beta_i > 0, else 0) with
// boundary_value_a, the cell's own fractions (mm_fluid.cpp:108-110); the
// geometry and arithmetic of k_grad2.  Output ga[2 i] = d alpha_i / dx,
// ga[2 i + 1] = d alpha_i / dy.
__device__ __forceinline__ double vol_frac(const MmField &z, int i, int ic) {
    double b = z.b[0][ic], r = z.r[0][ic];
#pragma unroll
    for (int k = 1; k < NM; ++k)
        if (k == i) {
            b = z.b[k][ic];
            r = z.r[k][ic];
        }
    return b > 0.0 ? b * z.rho[ic] / r : 0.0;
}
__global__ void __launch_bounds__(BLOCK) k_grad_a(MmArgs a) {
    const int ic = blockIdx.x * BLOCK + threadIdx.x;
    if (ic >= a.mesh.n) return;
    StructAcc c(a.mesh, ic);
    const double pcx = c.cx(), pcy = c.cy();
    double wv[4], drx[4], dry[4], drnx[4], drny[4];
    int nb[4];
    bool bnd[4];
    double A00 = 0.0, A01 = 0.0, A10 = 0.0, A11 = 0.0;
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        FaceG g = c.face(s);
        nb[s] = g.nb;
        bnd[s] = is_boundary(g.flag);
        double ncx, ncy;
        neib_center(c, g, s, pcx, pcy, ncx, ncy);
        const double rx = ncx - pcx, ry = ncy - pcy;
        const double d = rx * g.nx + ry * g.ny;
        const double nxx = d * g.nx, nyy = d * g.ny;
        const double w = 1.0 * g.area / cube_rn(sqrt(nxx * nxx + nyy * nyy));
        const double wdx = w * nxx, wdy = w * nyy;
        A00 += wdx * rx;
        A01 += wdx * ry;
        A10 += wdy * rx;
        A11 += wdy * ry;
        wv[s] = w;
        drx[s] = rx;
        dry[s] = ry;
        drnx[s] = nxx;
        drny[s] = nyy;
    }
    if (fabs(A11) < 1e-8) A11 = 1.0;
    const double det = A11 * A00 + (-A01) * A10;
    const double inv = 1.0 / det;
    const double B00 = A11 * inv, B01 = (-A01) * inv, B10 = (-A10) * inv, B11 = A00 * inv;
    const size_t n = (size_t)a.mesh.n;
#pragma unroll
    for (int i = 0; i < NM; ++i) {
        const double zk = vol_frac(a.z, i, ic);
        double dn[4], Fx = 0.0, Fy = 0.0;
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            const double zn = bnd[s] ? zk : vol_frac(a.z, i, nb[s]);
            const double dF = zn - zk;
            dn[s] = dF;
            Fx += wv[s] * dF * drnx[s];
            Fy += wv[s] * dF * drny[s];
        }
        const double g0x = B00 * Fx + B01 * Fy;
        const double g0y = B10 * Fx + B11 * Fy;
        double lx = 0.0, ly = 0.0;
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            const double dF_p = dn[s];
            const double du_n = g0x * drx[s] + g0y * dry[s];
            const double dF_m = 2.0 * du_n - dF_p;
            const double dF_lim = limiter2(a.limiter, dF_m, dF_p) * dF_p;
            lx += wv[s] * dF_lim * drnx[s];
            ly += wv[s] * dF_lim * drny[s];
        }
        a.grad_a[(2 * i) * n + ic] = B00 * lx + B01 * ly;
        a.grad_a[(2 * i + 1) * n + ic] = B10 * lx + B11 * ly;
    }
}

// FaceExtra::Direct (face_extra.h:121-171): z shifted along cell o's
// gradients by (dx, dy)
__device__ __forceinline__ MSt<NM> shifted(const MmArgs &a, const MSt<NM> &z, int o, double dx, double dy) {
    double v[NG];
    to_arr(z, v);
#pragma unroll
    for (int k = 0; k < NG; ++k) v[k] = v[k] + (a.gx[k][o] * dx + a.gy[k][o] * dy);
    return from_arr(v);
}

// PState::interpolation_update (models.cpp:381-391): fractions normalised,
// true densities, energy and temperature from (density, pressure) by get_reT
// with the extrapolated temperature and densities as the guesses
__device__ __forceinline__ void interp_update(const MixD<NM> &mx, MSt<NM> &z) {
    normalize(z.b);
    const int idx = frac_index(z.b);
    if (idx >= 0) {
#pragma unroll
        for (int i = 0; i < NM; ++i) z.r[i] = i == idx ? z.rho : MM_NAN;
        z.e = m_energy_rP(mx.mat[idx], z.rho, z.P);
        z.T = m_temperature_rP(mx.mat[idx], z.rho, z.P);
    } else {
        RhoSet<NM> rh;
        double T;
        double r0[NM];
#pragma unroll
        for (int i = 0; i < NM; ++i) r0[i] = z.r[i];
        z.e = find_reT_rP(mx, z.rho, z.P, z.b, z.T, r0, rh, T, false).val;
        z.T = T;
#pragma unroll
        for (int i = 0; i < NM; ++i) z.r[i] = rh.r[i];
    }
}

// fluxes_stage1 (mm_fluid.cpp:521-587): the half step of the cells that are
// not mixed, from the physical fluxes of their own face values
__global__ void __launch_bounds__(BLOCK) k_stage1(MmArgs a) {
    const int ic = blockIdx.x * BLOCK + threadIdx.x;
    if (ic >= a.mesh.n) return;
    const double dt = a.dt_scale * *a.dt_out;
    StructAcc c(a.mesh, ic);
    const MSt<NM> zc = load(a.z, ic);
    if (frac_index(zc.b) < 0) {
        store(a.zhalf, ic, zc);
        return;
    }
    const double pcx = c.cx(), pcy = c.cy();
    QVd<NM> flux = qv_zero<NM>();
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        if (skip_face(a.dir, s)) continue;
        FaceG g = c.face(s);
        MSt<NM> zm = shifted(a, zc, ic, g.fcx - pcx, g.fcy - pcy);
        interp_update(a.mix, zm);
        to_local(g.nx, g.ny, zm.vx, zm.vy, zm.vx, zm.vy);
        QVd<NM> lf = f_of(zm);
        const double mxx = g.nx * lf.a[1] + -g.ny * lf.a[2] + 0.0 * 0.0;
        const double myy = g.ny * lf.a[1] + g.nx * lf.a[2] + 0.0 * 0.0;
        lf.a[1] = mxx;
        lf.a[2] = myy;
#pragma unroll
        for (int k = 0; k < 4 + NM; ++k) flux.a[k] += lf.a[k] * g.area;
    }
    QVd<NM> q = q_of(zc);
    const double coef = 0.5 * dt / c.vol();
#pragma unroll
    for (int k = 0; k < 4 + NM; ++k) q.a[k] -= coef * flux.a[k];
    store(a.zhalf, ic, state_of_q(a.mix, q, zc.P, zc.T, zc.r));
}

// fluxes_stage2 (mm_fluid.cpp:589-680): the step from the half-step face
// values, extrapolated with the old layer's gradients, through calc_flux.
// One face of cell ic: the flux through face s, in the global frame, times
// the face area.
__device__ void face_term2(const MmArgs &a, int ic, int s, double dt, double *out, bool &bad) {
    StructAcc c(a.mesh, ic);
    const double pcx = c.cx(), pcy = c.cy(), V_c = c.vol();
    FaceG g = c.face(s);
    const bool bnd = is_boundary(g.flag);
    double ncx, ncy;
    neib_center(c, g, s, pcx, pcy, ncx, ncy);
    const double V_n = V_c;
    MSt<NM> zm = shifted(a, load(a.zhalf, ic), ic, g.fcx - pcx, g.fcy - pcy);
    interp_update(a.mix, zm);
    MSt<NM> zp;
    if (!bnd) {
        zp = shifted(a, load(a.zhalf, g.nb), g.nb, g.fcx - ncx, g.fcy - ncy);
        interp_update(a.mix, zp);
    } else {
        zp = ghost(zm, g);
    }
    to_local(g.nx, g.ny, zm.vx, zm.vy, zm.vx, zm.vy);
    to_local(g.nx, g.ny, zp.vx, zp.vy, zp.vx, zp.vy);
    const double S = g.area;
    QVd<NM> lf = calc_flux(a, dt, ic, g, zm, zp, V_c / S, V_n / S, bad);
    const double mxx = g.nx * lf.a[1] + -g.ny * lf.a[2] + 0.0 * 0.0;
    const double myy = g.ny * lf.a[1] + g.nx * lf.a[2] + 0.0 * 0.0;
    lf.a[1] = mxx;
    lf.a[2] = myy;
#pragma unroll
    for (int k = 0; k < 4 + NM; ++k) out[k] = lf.a[k] * S;
}

// the update of cell ic from its summed face terms (mm_fluid.cpp:662-679)
__device__ __forceinline__ void update2(const MmArgs &a, int ic, double dt, const QVd<NM> &flux, bool bad) {
    const MSt<NM> zc = load(a.z, ic);
    QVd<NM> q = q_of(zc);
    const double coef = dt / a.mesh.vol;
#pragma unroll
    for (int k = 0; k < 4 + NM; ++k) q.a[k] -= coef * flux.a[k];
    if (q.a[0] < 0.0) bad = true;  // the reference throws (mm_fluid.cpp:670-672)
    if (bad) atomicOr(a.err, 1);
    store(a.znext, ic, state_of_q(a.mix, q, zc.P, zc.T, zc.r));
}

// Every face of every cell (used without composite fluxes, CRP mode NONE).
__global__ void __launch_bounds__(BLOCK) k_stage2(MmArgs a) {
    const int ic = blockIdx.x * BLOCK + threadIdx.x;
    if (ic >= a.mesh.n) return;
    const double dt = a.dt_scale * *a.dt_out;
    QVd<NM> flux = qv_zero<NM>();
    bool bad = false;
#pragma unroll 1
    for (int s = 0; s < 4; ++s) {
        if (skip_face(a.dir, s)) continue;
        double term[4 + NM];
        face_term2(a, ic, s, dt, term, bad);
#pragma unroll
        for (int k = 0; k < 4 + NM; ++k) flux.a[k] += term[k];
    }
    update2(a, ic, dt, flux, bad);
}

// interpolation_update of a face value that came out pure (the common case);
// false, and z untouched past its fractions, when it is mixed
__device__ __forceinline__ bool interp_pure(const MixD<NM> &mx, MSt<NM> &z) {
    normalize(z.b);
    const int idx = frac_index(z.b);
    if (idx < 0) return false;
#pragma unroll
    for (int i = 0; i < NM; ++i) z.r[i] = i == idx ? z.rho : MM_NAN;
    z.e = m_energy_rP(mx.mat[idx], z.rho, z.P);
    z.T = m_temperature_rP(mx.mat[idx], z.rho, z.P);
    return true;
}

// With composite fluxes (CRP modes): cells all of whose face values come out
// pure take calc_flux's plain-HLLC branch here, with the same operations as
// face_term2; a cell with a mixed face value goes to the work list, whose
// faces k_stage2_faces evaluates one per thread and k_crp_update sums in slot
// order.  The lean kernel keeps the Newton closures and the composite Riemann
// solver out of the common path (fewer registers, more resident warps).
// (four resident blocks: 128 registers, measured 9 % faster than three)
// R = double: the reference's arithmetic.  R = float: the mixed form -- the
// reconstruction and its closures in FP64, the HLLC flux of the two pure
// face states in FP32 (hllc_pure), widened to FP64 for the sums.
__device__ __forceinline__ PureSt<float> pure_f(const MSt<NM> &z) {
    PureSt<float> o;
    o.rho = (float)z.rho;
    o.vx = (float)z.vx;
    o.vy = (float)z.vy;
    o.P = (float)z.P;
    o.e = (float)z.e;
#pragma unroll
    for (int i = 0; i < NM; ++i) o.b[i] = (float)z.b.f[i];
    o.idx = frac_index(z.b);
    return o;
}
template <typename R>
__global__ void __launch_bounds__(BLOCK, 4) k_stage2_pure(MmArgs a) {
    const int ic = blockIdx.x * BLOCK + threadIdx.x;
    if (ic >= a.mesh.n) return;
    const double dt = a.dt_scale * *a.dt_out;
    StructAcc c(a.mesh, ic);
    const double pcx = c.cx(), pcy = c.cy();
    const MSt<NM> zch = load(a.zhalf, ic);
    QVd<NM> flux = qv_zero<NM>();
    bool bad = false;
#pragma unroll 1
    for (int s = 0; s < 4; ++s) {
        if (skip_face(a.dir, s)) continue;
        FaceG g = c.face(s);
        const bool bnd = is_boundary(g.flag);
        double ncx, ncy;
        neib_center(c, g, s, pcx, pcy, ncx, ncy);
        MSt<NM> zm = shifted(a, zch, ic, g.fcx - pcx, g.fcy - pcy);
        bool pure = interp_pure(a.mix, zm);
        MSt<NM> zp;
        if (pure && !bnd) {
            zp = shifted(a, load(a.zhalf, g.nb), g.nb, g.fcx - ncx, g.fcy - ncy);
            pure = interp_pure(a.mix, zp);
        } else {
            zp = ghost(zm, g);
        }
        if (!pure) {
            a.list_crp[atomicAdd(&a.counts[0], 1)] = ic;
            return;
        }
        to_local(g.nx, g.ny, zm.vx, zm.vy, zm.vx, zm.vy);
        to_local(g.nx, g.ny, zp.vx, zp.vy, zp.vx, zp.vy);
        const double S = g.area;
        QVd<NM> lf;
        if constexpr (sizeof(R) == 8) {
            lf = hllc(a.mix, zm, zp, bad);
        } else {
            float F[4 + NM];
            hllc_pure<float>(a.mix, pure_f(zm), pure_f(zp), F, bad);
#pragma unroll
            for (int k = 0; k < 4 + NM; ++k) lf.a[k] = (double)F[k];
        }
        const double mxx = g.nx * lf.a[1] + -g.ny * lf.a[2] + 0.0 * 0.0;
        const double myy = g.ny * lf.a[1] + g.nx * lf.a[2] + 0.0 * 0.0;
        lf.a[1] = mxx;
        lf.a[2] = myy;
#pragma unroll
        for (int k = 0; k < 4 + NM; ++k) flux.a[k] += lf.a[k] * S;
    }
    update2(a, ic, dt, flux, bad);
}
__global__ void __launch_bounds__(BLOCK) k_stage2_faces(MmArgs a) {
    const double dt = a.dt_scale * *a.dt_out;
    const int count = 4 * a.counts[0];
    for (int t = blockIdx.x * BLOCK + threadIdx.x; t < count; t += gridDim.x * BLOCK) {
        if (skip_face(a.dir, t & 3)) continue;
        bool bad = false;
        double term[4 + NM];
        face_term2(a, a.list_crp[t >> 2], t & 3, dt, term, bad);
#pragma unroll
        for (int k = 0; k < 4 + NM; ++k) a.fbuf[(size_t)t * (4 + NM) + k] = term[k];
        if (bad) atomicOr(a.err, 1);
    }
}

static inline unsigned blocks(const MmArgs &a) { return (unsigned)((a.mesh.n + BLOCK - 1) / BLOCK); }

void launch_dt(const MmArgs &a, void *stream) { k_dt<<<blocks(a), BLOCK, 0, (cudaStream_t)stream>>>(a); }
void launch_recover(const MmArgs &a, void *stream) { k_recover<<<blocks(a), BLOCK, 0, (cudaStream_t)stream>>>(a); }
void launch_flux_pure(const MmArgs &a, void *stream) {
    if (a.fp32_flux) launch_flux_pure_fp32(a, stream);
    else k_flux_pure<double><<<blocks(a), BLOCK, 0, (cudaStream_t)stream>>>(a);
}
// The cells whose stencil (the cell and its four neighbours, boundary slots
// counting as the cell itself) holds a mixed state: the list that
// k_flux_pure builds, built ahead of it.
__global__ void __launch_bounds__(BLOCK) k_classify(MmArgs a) {
    int ic = blockIdx.x * BLOCK + threadIdx.x;
    if (ic >= a.mesh.n) return;
    StructAcc c(a.mesh, ic);
    const int idx_c = pure_index(a.z, ic);
    bool pure = idx_c >= 0;
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        FaceG g = c.face(s);
        pure = pure && (is_boundary(g.flag) ? idx_c : pure_index(a.z, g.nb)) >= 0;
    }
    if (!pure) a.list_crp[atomicAdd(&a.counts[0], 1)] = ic;
}
void launch_classify(const MmArgs &a, void *stream) {
    k_classify<<<blocks(a), BLOCK, 0, (cudaStream_t)stream>>>(a);
}
void launch_crp_faces(const MmArgs &a, void *stream) {
    k_crp_parts<<<std::min<unsigned>(8 * blocks(a), 2 * LIST_BLOCKS), BLOCK, 0, (cudaStream_t)stream>>>(a);
}
void launch_crp_update(const MmArgs &a, void *stream) {
    k_crp_update_parts<<<std::min<unsigned>(blocks(a), LIST_BLOCKS), BLOCK, 0, (cudaStream_t)stream>>>(a);
}
void launch_closure(const MmArgs &a, void *stream) {
    k_closure<<<std::min<unsigned>(blocks(a), LIST_BLOCKS), BLOCK, 0, (cudaStream_t)stream>>>(a);
}
void launch_grad2(const MmArgs &a, void *stream) { k_grad2<<<blocks(a), BLOCK, 0, (cudaStream_t)stream>>>(a); }
void launch_grad_a(const MmArgs &a, void *stream) { k_grad_a<<<blocks(a), BLOCK, 0, (cudaStream_t)stream>>>(a); }
void launch_stage1(const MmArgs &a, void *stream) { k_stage1<<<blocks(a), BLOCK, 0, (cudaStream_t)stream>>>(a); }
void launch_stage2(const MmArgs &a, void *stream) {
    cudaStream_t st = (cudaStream_t)stream;
    if (a.crp == CRP_NONE) {
        k_stage2<<<blocks(a), BLOCK, 0, st>>>(a);
        return;
    }
    if (a.fp32_flux) k_stage2_pure<float><<<blocks(a), BLOCK, 0, st>>>(a);
    else k_stage2_pure<double><<<blocks(a), BLOCK, 0, st>>>(a);
    k_stage2_faces<<<std::min<unsigned>(4 * blocks(a), LIST_BLOCKS), BLOCK, 0, st>>>(a);
    k_crp_update<<<std::min<unsigned>(blocks(a), LIST_BLOCKS), BLOCK, 0, st>>>(a);
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
