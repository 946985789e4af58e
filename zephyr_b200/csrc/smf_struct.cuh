// smf_struct.cuh -- FP64 kernels of SmFluid::update in the reference's
// per-cell gather form: every cell walks its face slots in slot order (L, R,
// B, T, then the second halves of split sides) and evaluates each face flux in
// its own frame, exactly as math/solver/sm_fluid.cpp does.  Compiled with
// -fmad=false these kernels are the parity path.
//
// The kernels are templated on a mesh accessor:
//  * StructAcc: a uniform rectangle (zephyr's AmrCells(Rectangle) before any
//    refinement), cell numbering ic = i * ny + j (amr_cells_gen.cpp:145-151),
//    geometry from per-axis tables filled with the reference's formulas
//    (amr_cells_gen.cpp:158-253, quad.cpp:429-436);
//  * SlotAcc: any mesh given cell by cell with 8 face slots (AMR meshes with
//    hanging faces).
#pragma once

#include "smf_math.cuh"
#include "smf_types.h"

namespace zg {

// ---------------------------------------------------------------------------
// Face geometry of slot s (0 L, 1 R, 2 B, 3 T) of cell (i, j).
struct FaceG {
    int flag;     // boundary flag of the slot
    int nb;       // neighbour cell (the cell itself on boundary slots)
    double nx, ny;  // outward unit normal
    double fcx, fcy;  // face centre
    double area;
};

// Uniform rectangle.
struct StructAcc {
    static constexpr int NSLOT = 4;
    static constexpr bool UNIT_NORMALS = true;  // axis normals: no normalisation
    static constexpr bool LSM_TWO_PASS = false;
    const StructMesh &m;
    int ic, i, j;
    __device__ StructAcc(const SmfArgs &a, int ic_) : m(a.mesh), ic(ic_) {
        i = ic / m.ny;
        j = ic - i * m.ny;
    }
    __device__ StructAcc(const StructMesh &mesh, int ic_) : m(mesh), ic(ic_) {
        i = ic / m.ny;
        j = ic - i * m.ny;
    }
    __device__ static int n(const SmfArgs &a) { return a.mesh.n; }
    __device__ double cx() const { return m.cx[i]; }
    __device__ double cy() const { return m.cy[j]; }
    __device__ double vol() const { return m.vol; }
    // the flux geometry (SmFluid's face.area(m_axial), cell.volume(m_axial)):
    // plain on a rectangle
    static constexpr bool axial() { return false; }
    __device__ double flux_area(const FaceG &g, int) const { return g.area; }
    __device__ double flux_vol() const { return m.vol; }
    // incircle diameter (amr_cells.cpp:107-116)
    __device__ double dinc() const { return sqrt(smin(m.inc2x[i], m.inc2y[j])); }

    // Face geometry of slot s (0 L, 1 R, 2 B, 3 T).
    __device__ FaceG face(int s) const {
        FaceG g;
        if (s == 0) {
            g.flag = i > 0 ? BC_INNER : m.bc[0];
            g.nb = i > 0 ? ic - m.ny : (m.xper ? ic + (m.nx - 1) * m.ny : ic);
            g.nx = -1.0; g.ny = -0.0;
            g.fcx = m.X[i]; g.fcy = m.fym[j];
            g.area = m.hy;
        } else if (s == 1) {
            g.flag = i < m.nx - 1 ? BC_INNER : m.bc[1];
            g.nb = i < m.nx - 1 ? ic + m.ny : (m.xper ? ic - (m.nx - 1) * m.ny : ic);
            g.nx = 1.0; g.ny = 0.0;
            g.fcx = m.X[i + 1]; g.fcy = m.fym[j];
            g.area = m.hy;
        } else if (s == 2) {
            g.flag = j > 0 ? BC_INNER : m.bc[2];
            g.nb = j > 0 ? ic - 1 : (m.yper ? ic + (m.ny - 1) : ic);
            g.nx = -0.0; g.ny = -1.0;
            g.fcx = m.fxm[i]; g.fcy = m.Y[j];
            g.area = m.hx;
        } else {
            g.flag = j < m.ny - 1 ? BC_INNER : m.bc[3];
            g.nb = j < m.ny - 1 ? ic + 1 : (m.yper ? ic - (m.ny - 1) : ic);
            g.nx = 0.0; g.ny = 1.0;
            g.fcx = m.fxm[i]; g.fcy = m.Y[j + 1];
            g.area = m.hx;
        }
        return g;
    }
    // Centre of the neighbour across slot s (INNER faces only).
    __device__ void nb_center(const FaceG &g, int s, double &ncx, double &ncy) const {
        int in = i, jn = j;
        if (s == 0) in = i - 1;
        else if (s == 1) in = i + 1;
        else if (s == 2) jn = j - 1;
        else jn = j + 1;
        ncx = m.cx[in];
        ncy = m.cy[jn];
    }
};

// Mesh given slot by slot (AMR).
struct SlotAcc {
    static constexpr int NSLOT = 8;
    static constexpr bool UNIT_NORMALS = false;
    static constexpr bool LSM_TWO_PASS = false;
    const SlotMesh &m;
    int ic;
    __device__ SlotAcc(const SmfArgs &a, int ic_) : m(a.smesh), ic(ic_) {}
    __device__ static int n(const SmfArgs &a) { return a.smesh.n; }
    __device__ double cx() const { return m.cx[ic]; }
    __device__ double cy() const { return m.cy[ic]; }
    __device__ double vol() const { return m.vol[ic]; }
    __device__ double dinc() const { return m.inc[ic]; }
    // the flux geometry: area_alt and volume_alt on an axisymmetric mesh
    // (sm_fluid.cpp:160-164, 236-240, 341-345)
    __device__ bool axial() const { return m.vol_alt != nullptr; }
    __device__ double flux_area(const FaceG &g, int s) const { return m.fa_alt ? m.fa_alt[8 * ic + s] : g.area; }
    __device__ double flux_vol() const { return m.vol_alt ? m.vol_alt[ic] : m.vol[ic]; }
    __device__ FaceG face(int s) const {
        const int f = 8 * ic + s;
        FaceG g;
        g.flag = m.fb[f];
        g.nb = m.fn[f];
        g.nx = m.fnx[f];
        g.ny = m.fny[f];
        g.fcx = m.fcx[f];
        g.fcy = m.fcy[f];
        g.area = m.fa[f];
        return g;
    }
    __device__ void nb_center(const FaceG &g, int, double &ncx, double &ncy) const {
        ncx = m.cx[g.nb];
        ncy = m.cy[g.nb];
    }
};

// Slot accessor of an adaptive rectangle (a quadtree of axis-aligned cells):
// the face geometry follows from the cell's centre, its level and the slot,
// so per slot only the boundary flag and the neighbour are read.  Slot side
// (0 L, 1 R, 2 B, 3 T) holds the whole side, or, when slot side + 4 is
// defined, its first half (lower / left along the side) and side + 4 the
// second half (subface_nodes2d).  Used by the FAST slot kernels; on dyadic
// meshes it reproduces the stored geometry exactly.
struct SlotFastAcc {
    static constexpr int NSLOT = 8;
    static constexpr bool UNIT_NORMALS = true;
    static constexpr bool LSM_TWO_PASS = true;
    const SlotMesh &m;
    int ic;
    double hx, hy, pcx, pcy;
    __device__ SlotFastAcc(const SmfArgs &a, int ic_) : m(a.smesh), ic(ic_) {
        const int L = m.level[ic];
        hx = ldexp(m.hx0, -L);
        hy = ldexp(m.hy0, -L);
        pcx = m.cx[ic];
        pcy = m.cy[ic];
    }
    __device__ static int n(const SmfArgs &a) { return a.smesh.n; }
    __device__ double cx() const { return pcx; }
    __device__ double cy() const { return pcy; }
    __device__ double vol() const { return m.vol[ic]; }
    __device__ double dinc() const { return m.inc[ic]; }
    static constexpr bool axial() { return false; }
    __device__ double flux_area(const FaceG &g, int) const { return g.area; }
    __device__ double flux_vol() const { return m.vol[ic]; }
    __device__ FaceG face(int s) const {
        const int f = 8 * ic + s;
        FaceG g;
        g.flag = m.fb[f];
        if (g.flag == BC_UNDEFINED) return g;
        g.nb = m.fn[f];
        const int side = s & 3;
        const bool split = s >= 4 || m.fb[f + 4] != BC_UNDEFINED;
        const double q = s >= 4 ? 0.25 : -0.25;  // offset of a half face along the side
        if (side < 2) {
            const bool hi = side == 1;
            g.nx = hi ? 1.0 : -1.0;
            g.ny = hi ? 0.0 : -0.0;
            g.fcx = pcx + (hi ? 0.5 : -0.5) * hx;
            g.fcy = split ? pcy + q * hy : pcy;
            g.area = split ? 0.5 * hy : hy;
        } else {
            const bool hi = side == 3;
            g.nx = hi ? 0.0 : -0.0;
            g.ny = hi ? 1.0 : -1.0;
            g.fcx = split ? pcx + q * hx : pcx;
            g.fcy = pcy + (hi ? 0.5 : -0.5) * hy;
            g.area = split ? 0.5 * hx : hx;
        }
        return g;
    }
    __device__ void nb_center(const FaceG &g, int, double &ncx, double &ncy) const {
        ncx = m.cx[g.nb];
        ncy = m.cy[g.nb];
    }
};

// The face-once form's choice of the cell that evaluates a face (slot s of
// cell ic, flag, neighbour nb): a boundary face its cell; a face between a
// coarse and a fine cell the fine one (its full face is the coarse cell's
// half face, with the same centre and area); a face between cells of one
// level the cell on its low side (the face is that cell's x-high or y-high
// slot).  The other cell reads the flux from the neighbour's slot of the
// opposite side, which is a full slot (< 4) in both cases.
__device__ __forceinline__ bool computes_face(const SlotMesh &m, int ic, int s, int flag, int nb) {
    if (is_boundary(flag)) return true;
    const int ln = m.level[nb], lc = m.level[ic];
    if (ln != lc) return ln < lc;
    return (s & 1) == 1;
}

// The face-once fluxes of cell ic (slotfast::FaceFlux records, signed by
// the slot index) summed in slot order.
__device__ __forceinline__ Cons sum_faces(int ic, const slotfast::FaceFlux &ff) {
    Cons F{0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int s = 0; s < 8; ++s) {
        const int x = ff.fidx[8 * ic + s];
        if (x == slotfast::FACE_NONE) continue;
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

// Centre of the neighbour across slot s, or the mirror of the cell centre in
// the face (sm_fluid.cpp:211-212; amr_faces.h:197-199 symm_point).
template <class Acc>
__device__ inline void neib_center(const Acc &c, const FaceG &g, int s, double pcx, double pcy, double &ncx,
                                   double &ncy) {
    if (g.flag == BC_INNER) {
        c.nb_center(g, s, ncx, ncy);
    } else {
        double d = (g.fcx - pcx) * g.nx + (g.fcy - pcy) * g.ny;
        double t = 2.0 * d;
        ncx = pcx + t * g.nx;
        ncy = pcy + t * g.ny;
    }
}

__device__ inline Prim load_prim(const PrimPtr &z, int ic) {
    Prim s;
    s.r = z.r[ic];
    s.u = z.u[ic];
    s.v = z.v[ic];
    s.p = z.p[ic];
    s.e = z.e[ic];
    return s;
}
__device__ inline void store_prim(const PrimPtr &z, int ic, const Prim &s) {
    z.r[ic] = s.r;
    z.u[ic] = s.u;
    z.v[ic] = s.v;
    z.p[ic] = s.p;
    z.e[ic] = s.e;
}

// sm_fluid.cpp:69-79
__device__ inline Prim boundary_value(const Prim &zc, double nx, double ny, int flag) {
    if (flag != BC_WALL) return zc;
    Prim zn = zc;
    double d = zc.u * nx + zc.v * ny;
    double vx = nx * d, vy = ny * d;
    zn.u = zc.u - 2.0 * vx;
    zn.v = zc.v - 2.0 * vy;
    return zn;
}

// dt of the current step, written by the last block of k_dt.
__device__ inline double finalize_dt(const SmfArgs &a) { return *a.dt_out; }

// Rotation of a velocity into / out of the face frame (rotate.cpp:7-77): the
// normal is normalised first.  Axis normals of a rectangle are unit vectors
// already, so the structured accessor skips the normalisation.
template <class Acc>
__device__ inline void frame(const FaceG &g, double &c, double &s) {
    c = g.nx;
    s = g.ny;
    if (!Acc::UNIT_NORMALS) {
        double sn = g.nx * g.nx + g.ny * g.ny;
        if (sn > 0.0) {
            double r = sqrt(sn);
            c = g.nx / r;
            s = g.ny / r;
        }
    }
}

// ---------------------------------------------------------------------------
// K1: CFL minimum over cells (sm_fluid.cpp:104-114, amr_cells.cpp:107-116).
// The CFL bound of one cell, incircle / (|v| + c), as the bits of a
// non-negative double (compute_dt, sm_fluid.cpp:104-116).  std::min skips a
// NaN in its second slot; NaN bits sort above all finite positives, so the
// unsigned minimum skips it too.
__device__ inline unsigned long long cfl_bits(const SmfArgs &a, double dinc, double rho, double u, double v,
                                              double p) {
    double cs = a.eos.sound_speed_rP(rho, p);
    double lam = dinc / (sqrt(u * u + v * v) + cs);
    unsigned long long b = dbits(lam);
    if (!(lam >= 0.0)) b = 0x7FEFFFFFFFFFFFFFull;
    return b;
}

// Block minimum of `best`, then the grid minimum through a.dmin_bits: the
// last block to finish turns it into dt = min(CFL * min, max_dt)
// (sm_fluid.cpp:112) at *dst and resets the accumulator for the next use.
// No block waits for another.  Every thread of the block calls it, from one
// call site (it holds a block barrier).
template <int BLOCK>
__device__ inline void commit_cfl_min(const SmfArgs &a, unsigned long long best, double *dst) {
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
                *dst = smin(a.CFL * dmin, a.max_dt);
                *a.dmin_bits = 0x7FEFFFFFFFFFFFFFull;
                *a.dt_ticket = 0u;
                __threadfence();
            }
        }
    }
}

template <class Acc, int BLOCK, int MINB = 1>
__global__ void __launch_bounds__(BLOCK, MINB) k_dt(SmfArgs a) {
    int ic = blockIdx.x * BLOCK + threadIdx.x;
    unsigned long long best = 0x7FEFFFFFFFFFFFFFull;  // bits of DBL_MAX
    if (ic < Acc::n(a)) {
        Acc c(a, ic);
        best = cfl_bits(a, c.dinc(), a.z.r[ic], a.z.u[ic], a.z.v[ic], a.z.p[ic]);
    }
    commit_cfl_min<BLOCK>(a, best, a.dt_out);
}

__device__ inline void add_area(Cons &F, const Cons &lf, double area) {
    F.r += lf.r * area;
    F.mu += lf.mu * area;
    F.mv += lf.mv * area;
    F.E += lf.E * area;
}

__device__ inline void update(Cons &q, double coef, const Cons &F) {
    q.r -= coef * F.r;
    q.mu -= coef * F.mu;
    q.mv -= coef * F.mv;
    q.E -= coef * F.E;
}

// ---------------------------------------------------------------------------
// K2: first-order step (sm_fluid.cpp:127-174).
template <class Acc, int BLOCK, int MINB = 1, int FX = -1>
__global__ void __launch_bounds__(BLOCK, MINB) k_flux1(SmfArgs a) {
    int ic = blockIdx.x * BLOCK + threadIdx.x;
    if (ic >= Acc::n(a)) return;
    Acc c(a, ic);
    double dt = finalize_dt(a);
    Prim zc = load_prim(a.z, ic);
    Cons q = q_from_p(zc);
    Cons F{0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int s = 0; s < Acc::NSLOT; ++s) {
        FaceG g = c.face(s);
        if (g.flag == BC_UNDEFINED) continue;
        Prim zn = !is_boundary(g.flag) ? load_prim(a.z, g.nb) : boundary_value(zc, g.nx, g.ny, g.flag);
        double cs, sn;
        frame<Acc>(g, cs, sn);
        Prim zm = zc, zp = zn;
        rot_local(zm.u, zm.v, cs, sn);
        rot_local(zp.u, zp.v, cs, sn);
        Cons lf = flux_fx<FX>(a.flux, zm, zp, a.eos);
        rot_global(lf.mu, lf.mv, cs, sn);
        add_area(F, lf, c.flux_area(g, s));
    }
    update(q, dt / c.flux_vol(), F);
    if (c.axial()) {  // pressure source of the radial momentum (sm_fluid.cpp:166-169)
        double coeff = c.vol() / c.flux_vol();
        q.mv += coeff * zc.p * dt;
    }
    store_prim(a.znext, ic, p_from_q(q, a.eos));
}

// ---------------------------------------------------------------------------
// K3: least-squares gradient and its limited re-fit
// (gradient.h:226-282 LSM, gradient.h:412-474 limiting), for the four
// fields that the later stages read: density, vx, vy, pressure.  (The energy
// gradient is computed by the reference but every use overwrites it with
// energy_rP, sm_fluid.cpp:223 and 312/322.)
//
// 2-D reduction of the 3x3 system: A(i,2) and A(2,j) are exact zeros, A(2,2)
// is set to 1 (gradient.h:268-273), and Eigen's cofactor inverse then gives
//   det = A11*A00 + (-A01)*A10,  B = [A11 -A01; -A10 A00] * (1/det).
template <class Acc>
__device__ inline void lsm_limited(const Acc &c, const PrimPtr &z, int lim, const Prim &zc, double gx[4],
                                   double gy[4]) {
    constexpr int NS = Acc::NSLOT;
    const double pcx = c.cx(), pcy = c.cy();
    double wv[NS], drx[NS], dry[NS], drnx[NS], drny[NS], dn[NS][4];
    bool on[NS];
    double A00 = 0.0, A01 = 0.0, A10 = 0.0, A11 = 0.0;
    double Fx[4] = {0.0, 0.0, 0.0, 0.0}, Fy[4] = {0.0, 0.0, 0.0, 0.0};
    const double zcv[4] = {zc.r, zc.u, zc.v, zc.p};
#pragma unroll
    for (int s = 0; s < NS; ++s) {
        FaceG g = c.face(s);
        on[s] = g.flag != BC_UNDEFINED;
        if (!on[s]) continue;
        Prim zn = !is_boundary(g.flag) ? load_prim(z, g.nb) : boundary_value(zc, g.nx, g.ny, g.flag);
        double ncx, ncy;
        neib_center(c, g, s, pcx, pcy, ncx, ncy);
        double rx = ncx - pcx, ry = ncy - pcy;
        double d = rx * g.nx + ry * g.ny;
        double nxx = d * g.nx, nyy = d * g.ny;
        double w = g.area / cube_rn(sqrt(nxx * nxx + nyy * nyy));
        double wdx = w * nxx, wdy = w * nyy;
        A00 += wdx * rx;
        A01 += wdx * ry;
        A10 += wdy * rx;
        A11 += wdy * ry;
        wv[s] = w; drx[s] = rx; dry[s] = ry; drnx[s] = nxx; drny[s] = nyy;
        const double znv[4] = {zn.r, zn.u, zn.v, zn.p};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            double dF = znv[k] - zcv[k];
            dn[s][k] = dF;
            Fx[k] += w * dF * nxx;
            Fy[k] += w * dF * nyy;
        }
    }
    if (fabs(A11) < 1e-8) A11 = 1.0;  // 1-D case (gradient.h:270-272)
    double det = A11 * A00 + (-A01) * A10;
    double inv = 1.0 / det;
    double B00 = A11 * inv, B01 = (-A01) * inv, B10 = (-A10) * inv, B11 = A00 * inv;
    double g0x[4], g0y[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        g0x[k] = B00 * Fx[k] + B01 * Fy[k];
        g0y[k] = B10 * Fx[k] + B11 * Fy[k];
    }
    double Lx[4] = {0.0, 0.0, 0.0, 0.0}, Ly[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int s = 0; s < NS; ++s) {
        if (!on[s]) continue;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            double dF_p = dn[s][k];
            double du_n = g0x[k] * drx[s] + g0y[k] * dry[s];
            double dF_m = 2.0 * du_n - dF_p;
            double dF_lim = limiter2(lim, dF_m, dF_p) * dF_p;
            Lx[k] += wv[s] * dF_lim * drnx[s];
            Ly[k] += wv[s] * dF_lim * drny[s];
        }
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        gx[k] = B00 * Lx[k] + B01 * Ly[k];
        gy[k] = B10 * Lx[k] + B11 * Ly[k];
    }
}

// The same computation in two passes over the slots that both evaluate the
// slot's geometry and neighbour difference (the second pass re-reads them),
// instead of holding eight slots' worth of them in registers: same
// operations, same results, a fraction of the registers.
template <class Acc>
__device__ inline void lsm_limited_2pass(const Acc &c, const PrimPtr &z, int lim, const Prim &zc, double gx[4],
                                         double gy[4]) {
    constexpr int NS = Acc::NSLOT;
    const double pcx = c.cx(), pcy = c.cy();
    double A00 = 0.0, A01 = 0.0, A10 = 0.0, A11 = 0.0;
    double Fx[4] = {0.0, 0.0, 0.0, 0.0}, Fy[4] = {0.0, 0.0, 0.0, 0.0};
    const double zcv[4] = {zc.r, zc.u, zc.v, zc.p};
    struct SlotTerms {
        double w, rx, ry, nxx, nyy, dF[4];
    };
    auto terms = [&](const FaceG &g, int s, SlotTerms &t) {
        Prim zn = !is_boundary(g.flag) ? load_prim(z, g.nb) : boundary_value(zc, g.nx, g.ny, g.flag);
        double ncx, ncy;
        neib_center(c, g, s, pcx, pcy, ncx, ncy);
        t.rx = ncx - pcx;
        t.ry = ncy - pcy;
        double d = t.rx * g.nx + t.ry * g.ny;
        t.nxx = d * g.nx;
        t.nyy = d * g.ny;
        t.w = g.area / cube_rn(sqrt(t.nxx * t.nxx + t.nyy * t.nyy));
        const double znv[4] = {zn.r, zn.u, zn.v, zn.p};
#pragma unroll
        for (int k = 0; k < 4; ++k) t.dF[k] = znv[k] - zcv[k];
    };
#pragma unroll 1
    for (int s = 0; s < NS; ++s) {
        FaceG g = c.face(s);
        if (g.flag == BC_UNDEFINED) continue;
        SlotTerms t;
        terms(g, s, t);
        double wdx = t.w * t.nxx, wdy = t.w * t.nyy;
        A00 += wdx * t.rx;
        A01 += wdx * t.ry;
        A10 += wdy * t.rx;
        A11 += wdy * t.ry;
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            Fx[k] += t.w * t.dF[k] * t.nxx;
            Fy[k] += t.w * t.dF[k] * t.nyy;
        }
    }
    if (fabs(A11) < 1e-8) A11 = 1.0;  // 1-D case (gradient.h:270-272)
    double det = A11 * A00 + (-A01) * A10;
    double inv = 1.0 / det;
    double B00 = A11 * inv, B01 = (-A01) * inv, B10 = (-A10) * inv, B11 = A00 * inv;
    double g0x[4], g0y[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        g0x[k] = B00 * Fx[k] + B01 * Fy[k];
        g0y[k] = B10 * Fx[k] + B11 * Fy[k];
    }
    double Lx[4] = {0.0, 0.0, 0.0, 0.0}, Ly[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll 1
    for (int s = 0; s < NS; ++s) {
        FaceG g = c.face(s);
        if (g.flag == BC_UNDEFINED) continue;
        SlotTerms t;
        terms(g, s, t);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            double dF_p = t.dF[k];
            double du_n = g0x[k] * t.rx + g0y[k] * t.ry;
            double dF_m = 2.0 * du_n - dF_p;
            double dF_lim = limiter2(lim, dF_m, dF_p) * dF_p;
            Lx[k] += t.w * dF_lim * t.nxx;
            Ly[k] += t.w * dF_lim * t.nyy;
        }
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        gx[k] = B00 * Lx[k] + B01 * Ly[k];
        gy[k] = B10 * Lx[k] + B11 * Ly[k];
    }
}

template <class Acc, int BLOCK, int MINB = 1>
__global__ void __launch_bounds__(BLOCK, MINB) k_grad(SmfArgs a, PrimPtr z) {
    int ic = blockIdx.x * BLOCK + threadIdx.x;
    if (ic >= Acc::n(a)) return;
    Acc c(a, ic);
    Prim zc = load_prim(z, ic);
    double gx[4], gy[4];
    if constexpr (Acc::LSM_TWO_PASS) lsm_limited_2pass(c, z, a.limiter, zc, gx, gy);
    else lsm_limited(c, z, a.limiter, zc, gx, gy);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        a.gx[k][ic] = gx[k];
        a.gy[k][ic] = gy[k];
    }
}

// face_extra.h:135-163: value + grad . (x_face - x_cell); the energy entry
// is recomputed from the EoS by every caller.
__device__ inline Prim extrap(const Prim &u, const SmfArgs &a, int ic, double dx, double dy) {
    Prim o;
    o.r = u.r + (a.gx[0][ic] * dx + a.gy[0][ic] * dy);
    o.u = u.u + (a.gx[1][ic] * dx + a.gy[1][ic] * dy);
    o.v = u.v + (a.gx[2][ic] * dx + a.gy[2][ic] * dy);
    o.p = u.p + (a.gx[3][ic] * dx + a.gy[3][ic] * dy);
    o.e = 0.0;
    return o;
}

// ---------------------------------------------------------------------------
// K4: predictor, half step with the physical flux (sm_fluid.cpp:176-253).
template <class Acc, int BLOCK, int MINB = 1>
__global__ void __launch_bounds__(BLOCK, MINB) k_stage1(SmfArgs a) {
    int ic = blockIdx.x * BLOCK + threadIdx.x;
    if (ic >= Acc::n(a)) return;
    Acc c(a, ic);
    double dt = finalize_dt(a);
    Prim zc = load_prim(a.z, ic);
    if (a.wait_in[ic] > 0) {
        store_prim(a.zhalf, ic, zc);
        return;
    }
    double pcx = c.cx(), pcy = c.cy();
    Cons q = q_from_p(zc);
    Cons F{0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int s = 0; s < Acc::NSLOT; ++s) {
        FaceG g = c.face(s);
        if (g.flag == BC_UNDEFINED) continue;
        Prim zm = extrap(zc, a, ic, g.fcx - pcx, g.fcy - pcy);
        zm.e = a.eos.energy_rP(zm.r, zm.p);
        if (is_bad(zm, a.eos)) zm = zc;
        double cs, sn;
        frame<Acc>(g, cs, sn);
        rot_local(zm.u, zm.v, cs, sn);
        Cons lf = flux_from_p(zm);
        rot_global(lf.mu, lf.mv, cs, sn);
        add_area(F, lf, c.flux_area(g, s));
    }
    update(q, 0.5 * dt / c.flux_vol(), F);
    if (c.axial()) {  // sm_fluid.cpp:242-245
        double coeff = c.vol() / c.flux_vol();
        q.mv += 0.5 * coeff * zc.p * dt;
    }
    Prim h = p_from_q(q, a.eos);
    if (is_bad(h, a.eos)) h = zc;
    store_prim(a.zhalf, ic, h);
}

// Face flux of the corrector (sm_fluid.cpp:271-341): reconstruct with the
// gradients of z at the states zh and solve the Riemann problem; returned
// multiplied by the face area.
template <int FX, class Acc>
__device__ inline Cons corrector_face(const SmfArgs &a, const PrimPtr &zh, const int *wt, const Acc &c, int s,
                                      const FaceG &g, const Prim &zch, double pcx, double pcy, int wc) {
    const int ic = c.ic;
    bool bnd = is_boundary(g.flag);
    Prim z_nh = !bnd ? load_prim(zh, g.nb) : boundary_value(zch, g.nx, g.ny, g.flag);
    Prim zm, zp;
    bool robust = wc > 0 || (wt != nullptr && wt[g.nb] > 0);
    if (robust) {
        zm = zch;
        zp = z_nh;
    } else {
        double ncx, ncy;
        neib_center(c, g, s, pcx, pcy, ncx, ncy);
        zm = extrap(zch, a, ic, g.fcx - pcx, g.fcy - pcy);
        zm.e = a.eos.energy_rP(zm.r, zm.p);
        if (is_bad(zm, a.eos)) zm = zch;
        if (!bnd) {
            zp = extrap(z_nh, a, g.nb, g.fcx - ncx, g.fcy - ncy);
            zp.e = a.eos.energy_rP(zp.r, zp.p);
            if (is_bad(zp, a.eos)) zp = z_nh;
        } else {
            zp = boundary_value(zm, g.nx, g.ny, g.flag);
        }
    }
    double cs, sn;
    frame<Acc>(g, cs, sn);
    rot_local(zm.u, zm.v, cs, sn);
    rot_local(zp.u, zp.v, cs, sn);
    Cons lf = robust ? hll(zm, zp, a.eos) : flux_fx<FX>(a.flux, zm, zp, a.eos);
    rot_global(lf.mu, lf.mv, cs, sn);
    const double area = c.flux_area(g, s);
    lf.r *= area;
    lf.mu *= area;
    lf.mv *= area;
    lf.E *= area;
    return lf;
}

// K5: corrector with the isolation bit (sm_fluid.cpp:255-366).  `wait` is
// read from the previous step's array and written to the other one.
template <class Acc, int BLOCK, int MINB = 1, int FX = -1>
__global__ void __launch_bounds__(BLOCK, MINB) k_stage2(SmfArgs a) {
    int ic = blockIdx.x * BLOCK + threadIdx.x;
    if (ic >= Acc::n(a)) return;
    Acc c(a, ic);
    double dt = finalize_dt(a);
    double pcx = c.cx(), pcy = c.cy();
    Prim zc = load_prim(a.z, ic);
    Prim zch = load_prim(a.zhalf, ic);
    int wc = a.wait_in[ic];
    Cons q = q_from_p(zc);
    Cons F{0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int s = 0; s < Acc::NSLOT; ++s) {
        FaceG g = c.face(s);
        if (g.flag == BC_UNDEFINED) continue;
        Cons lf = corrector_face<FX>(a, a.zhalf, a.wait_in, c, s, g, zch, pcx, pcy, wc);
        F.r += lf.r;
        F.mu += lf.mu;
        F.mv += lf.mv;
        F.E += lf.E;
    }
    update(q, dt / c.flux_vol(), F);
    if (c.axial()) {  // sm_fluid.cpp:347-350, with the half-step pressure
        double coeff = c.vol() / c.flux_vol();
        q.mv += coeff * zch.p * dt;
    }
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

// ---------------------------------------------------------------------------
// Heun extension (no counterpart in the reference; same operator L as the
// corrector with z_half = z, no isolation):
//   stage A: z* = P(Q(z^n) - dt/V * sum F(z^n))
//   stage B: z^{n+1} = P(0.5 * (Q(z^n) + Q(z*) - dt/V * sum F(z*)))
template <class Acc, int BLOCK, bool FINAL, int MINB = 1, int FX = -1>
__global__ void __launch_bounds__(BLOCK, MINB) k_heun(SmfArgs a, PrimPtr zin, PrimPtr zout) {
    int ic = blockIdx.x * BLOCK + threadIdx.x;
    if (ic >= Acc::n(a)) return;
    Acc c(a, ic);
    double dt = finalize_dt(a);
    double pcx = c.cx(), pcy = c.cy();
    Prim zc = load_prim(zin, ic);
    Cons q = q_from_p(zc);
    Cons F{0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int s = 0; s < Acc::NSLOT; ++s) {
        FaceG g = c.face(s);
        if (g.flag == BC_UNDEFINED) continue;
        Cons lf = corrector_face<FX>(a, zin, nullptr, c, s, g, zc, pcx, pcy, 0);
        F.r += lf.r;
        F.mu += lf.mu;
        F.mv += lf.mv;
        F.E += lf.E;
    }
    update(q, dt / c.vol(), F);
    if (FINAL) {
        Cons q0 = q_from_p(load_prim(a.z, ic));
        q.r = 0.5 * (q0.r + q.r);
        q.mu = 0.5 * (q0.mu + q.mu);
        q.mv = 0.5 * (q0.mv + q.mv);
        q.E = 0.5 * (q0.E + q.E);
    }
    store_prim(zout, ic, p_from_q(q, a.eos));
}

// ---------------------------------------------------------------------------
// AMR flags by neighbour jumps (sm_fluid.cpp:517-559).
template <class Acc, int BLOCK, int MINB = 1>
__global__ void __launch_bounds__(BLOCK, MINB) k_flags(SmfArgs a, int *flags) {
    int ic = blockIdx.x * BLOCK + threadIdx.x;
    if (ic >= Acc::n(a)) return;
    Acc c(a, ic);
    const double xi_dens = 0.05, xi_pres = 0.05;
    double dens = a.z.r[ic], pres = a.z.p[ic];
    double dens_split = xi_dens * fabs(dens);
    double pres_split = xi_pres * fabs(pres);
    int fl = -1;
    for (int s = 0; s < Acc::NSLOT; ++s) {
        FaceG g = c.face(s);
        if (g.flag == BC_UNDEFINED || is_boundary(g.flag)) continue;
        double dn = a.z.r[g.nb], pn = a.z.p[g.nb];
        if (fabs(dn - dens) > dens_split || fabs(pn - pres) > pres_split) {
            fl = 1;
            break;
        }
        if (fabs(dn - dens) > 0.4 * dens_split || fabs(pn - pres) > 0.4 * pres_split) fl = 0;
    }
    flags[ic] = fl;
}

}  // namespace zg
