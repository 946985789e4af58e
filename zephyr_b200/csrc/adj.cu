// adj.cu -- discrete adjoint of the Heun step (the adjoint mode, no
// counterpart in the reference), the C ABI zg_adj_*.
//
// Forward: Heun's method at a fixed dt on a uniform periodic rectangle
// (adj_math.cuh has the step's definition), state U = (rho, rho u, rho v,
// rho E) as four arrays of n doubles, cell ic = i * ny + j.
// Objective: J = mean pressure over the cells whose centre lies in the probe
// box.  Gradient: dJ / d rho_0 (the initial density field, the initial
// velocity and pressure held fixed) and dJ / d gamma.
//
// Reverse sweep.  With lambda^n = dJ/dU^n and mu = a cotangent of L(X):
//   U* = U + dt L(U),  U^{n+1} = 1/2 U + 1/2 U* + 1/2 dt L(U*)
//   lambda*   = 1/2 lambda^{n+1} + L'(U*)^T (1/2 dt lambda^{n+1})
//   lambda^n  = 1/2 lambda^{n+1} + lambda* + L'(U)^T (dt lambda*)
// and the gamma derivative collects <mu, dL/dgamma> of both stages.  The
// vector-Jacobian product L'(X)^T mu is two passes: per cell, the four face
// fluxes' partials with respect to their two face states and gamma (the
// hand-written reverse of the HLLC formulas) give the cotangents of the cell's face
// states, hence of its primitive state and its two slopes; per cell again,
// the slopes' partials carry those back to the three cells each slope reads,
// and the primitive map's partials to U and gamma.  HLLC branches and the
// limiter are differentiated on the side the forward took.
//
// Precision.  The FP64 form is FP64 throughout.  The mixed form keeps the
// primal step (face states, HLLC fluxes, states) in FP64 and stores the
// slopes in FP32 (computed in FP32 from FP64 neighbour differences); its
// reverse sweep evaluates the slopes' partials, the face states, the HLLC
// reverse and the face cotangents in FP32, with the adjoint states, their
// sums, the primitive map and gamma in FP64.  The primal stays FP64 because
// its rounding noise reaches the gradient through the limiter's partials
// (FP32 fluxes: gradient 1.6e-5 from the FP64 one in L2 on the 1024^2,
// 100-step problem; FP64 reverse arithmetic alone left that unchanged);
// the reverse's own FP32 arithmetic costs 1e-6.
//
// Checkpoints: U is kept every `checkpoint_every` steps during the forward;
// the reverse sweep recomputes each segment's U^n and U* from its checkpoint
// and walks it backwards, so memory grows with steps / checkpoint_every plus
// two segments, not with the number of steps.  The forward keeps the last two
// segments whole; each earlier one is recomputed on a second stream while
// the segment after it is swept.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/zephyr_gpu.h"
#include "adj_math.cuh"

namespace zg {
namespace adj {

constexpr int BLOCK = 128;
// Minimum resident blocks per SM of the heavy kernels.  They are latency-
// bound; these caps on their registers (a few spilled bytes in some) were
// chosen by timing the 1024^2, 100-step forward and gradient runs over a
// sweep of the values on a B200 (-D overrides).
#ifndef ZG_ADJ_PG_MINB
#define ZG_ADJ_PG_MINB 8
#endif
#ifndef ZG_ADJ_FU_MINB
#define ZG_ADJ_FU_MINB 6
#endif
#ifndef ZG_ADJ_VF_MINB
#define ZG_ADJ_VF_MINB 6
#endif

struct Grid {
    int nx, ny, n;
    double hx, hy, vol;
    double x0, y0;
};
// four field arrays of element type S (FP64 state, adjoint and primitive
// fields are double; the slopes and face cotangents are S = double in the
// FP64 form and S = float in the mixed form)
template <class S>
struct F4T {
    S *f[4];
};
template <class S>
struct CF4T {
    const S *f[4];
};
using F4 = F4T<double>;
using CF4 = CF4T<double>;

// A cell with its (i, j): the periodic neighbours follow without integer
// division (one division per thread, in cell_of).
struct Cell {
    int ic, i, j;
};
__device__ __forceinline__ Cell cell_of(const Grid &g, int ic) {
    int i = ic / g.ny;
    return Cell{ic, i, ic - i * g.ny};
}
__device__ __forceinline__ Cell xm(const Grid &g, Cell c) {
    return c.i > 0 ? Cell{c.ic - g.ny, c.i - 1, c.j} : Cell{c.ic + (g.nx - 1) * g.ny, g.nx - 1, c.j};
}
__device__ __forceinline__ Cell xp(const Grid &g, Cell c) {
    return c.i < g.nx - 1 ? Cell{c.ic + g.ny, c.i + 1, c.j} : Cell{c.ic - (g.nx - 1) * g.ny, 0, c.j};
}
__device__ __forceinline__ Cell ym(const Grid &g, Cell c) {
    return c.j > 0 ? Cell{c.ic - 1, c.i, c.j - 1} : Cell{c.ic + (g.ny - 1), c.i, g.ny - 1};
}
__device__ __forceinline__ Cell yp(const Grid &g, Cell c) {
    return c.j < g.ny - 1 ? Cell{c.ic + 1, c.i, c.j + 1} : Cell{c.ic - (g.ny - 1), c.i, 0};
}

__device__ __forceinline__ void load4(const CF4 &a, int ic, double o[4]) {
#pragma unroll
    for (int k = 0; k < 4; ++k) o[k] = a.f[k][ic];
}
__device__ __forceinline__ void prim_at(const CF4 &U, int ic, double gamma, double W[4]) {
    double u[4];
    load4(U, ic, u);
    prim<double>(u, gamma, W);
}

// U from (rho, u, v, p)
__global__ void k_init(Grid g, CF4 W0, double gamma, F4 U) {
    int ic = blockIdx.x * BLOCK + threadIdx.x;
    if (ic >= g.n) return;
    double r = W0.f[0][ic], u = W0.f[1][ic], v = W0.f[2][ic], p = W0.f[3][ic];
    U.f[0][ic] = r;
    U.f[1][ic] = r * u;
    U.f[2][ic] = r * v;
    U.f[3][ic] = p / (gamma - 1.0) + 0.5 * (r * (u * u + v * v));
}

// primitive state and limited slopes of every cell: the primitive map and
// the neighbour differences in FP64, the slopes from the differences in S
template <class S>
__global__ void __launch_bounds__(BLOCK, ZG_ADJ_PG_MINB) k_prim_grad(Grid g, CF4 U, double gamma, double eps,
                                                                     F4 W, F4T<S> gx, F4T<S> gy) {
    int ic = blockIdx.x * BLOCK + threadIdx.x;
    if (ic >= g.n) return;
    double wc[4], wl[4], wr[4], wb[4], wt[4];
    prim_at(U, ic, gamma, wc);
    const Cell c = cell_of(g, ic);
    prim_at(U, xm(g, c).ic, gamma, wl);
    prim_at(U, xp(g, c).ic, gamma, wr);
    prim_at(U, ym(g, c).ic, gamma, wb);
    prim_at(U, yp(g, c).ic, gamma, wt);
    const S i2x = S(0.5 / g.hx), i2y = S(0.5 / g.hy), e = S(eps);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        W.f[k][ic] = wc[k];
        gx.f[k][ic] = slope<S>(S(wl[k] - wc[k]), S(wr[k] - wc[k]), i2x, e);
        gy.f[k][ic] = slope<S>(S(wb[k] - wc[k]), S(wt[k] - wc[k]), i2y, e);
    }
}

// Face states of the face between `lo` and `hi` along an axis, in the face
// frame (x faces: (rho, u, v, p); y faces: (rho, v, -u, p)): the FP64
// primitive state rounded to S, plus or minus the slope times h / 2 in S.
template <class S>
__device__ __forceinline__ void face_states(const CF4 &W, const CF4T<S> &G, int lo, int hi, S half_h, bool yface,
                                            S L[4], S R[4]) {
    S a[4], b[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        a[k] = S(W.f[k][lo]) + G.f[k][lo] * half_h;
        b[k] = S(W.f[k][hi]) - G.f[k][hi] * half_h;
    }
    if (!yface) {
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            L[k] = a[k];
            R[k] = b[k];
        }
    } else {
        L[0] = a[0]; L[1] = a[2]; L[2] = -a[1]; L[3] = a[3];
        R[0] = b[0]; R[1] = b[2]; R[2] = -b[1]; R[3] = b[3];
    }
}
// face-frame flux back to the global frame
template <class S>
__device__ __forceinline__ void flux_global(const S Fl[4], bool yface, S F[4]) {
    if (!yface) {
#pragma unroll
        for (int k = 0; k < 4; ++k) F[k] = Fl[k];
    } else {
        F[0] = Fl[0];
        F[1] = -Fl[2];
        F[2] = Fl[1];
        F[3] = Fl[3];
    }
}

// out = alpha * base + beta * (X + dt L(X)), L from the face fluxes of W, G
template <class S>
__global__ void __launch_bounds__(BLOCK, ZG_ADJ_FU_MINB) k_flux_update(Grid g, CF4 W, CF4T<S> gx, CF4T<S> gy,
                                                                       double gamma, CF4 X, CF4 base, double alpha,
                                                                       double beta, double dt, F4 out) {
    int ic = blockIdx.x * BLOCK + threadIdx.x;
    if (ic >= g.n) return;
    const Cell cc = cell_of(g, ic);
    const int nb[4] = {xm(g, cc).ic, xp(g, cc).ic, ym(g, cc).ic, yp(g, cc).ic};
    double sum[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        const bool yface = s >= 2, high = (s & 1) == 1;
        const int lo = high ? ic : nb[s], hi = high ? nb[s] : ic;
        const double half_h = 0.5 * (yface ? g.hy : g.hx), A = yface ? g.hx : g.hy;
        // face states and HLLC in FP64 in both forms (the slopes are FP32 in
        // the mixed form): FP32 fluxes carry rounding errors of ~1e-7 of the
        // flux, ~1e-4 of the flux difference across a cell of a smooth
        // field, and the limiter's partials, which depend on neighbour
        // differences, carry that noise of the trajectory into the gradient
        double L[4], R[4], Fl[4], F[4];
        {
            const CF4T<S> &G = yface ? gy : gx;
            double a_[4], b_[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                a_[k] = W.f[k][lo] + (double)G.f[k][lo] * half_h;
                b_[k] = W.f[k][hi] - (double)G.f[k][hi] * half_h;
            }
            if (!yface) {
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    L[k] = a_[k];
                    R[k] = b_[k];
                }
            } else {
                L[0] = a_[0]; L[1] = a_[2]; L[2] = -a_[1]; L[3] = a_[3];
                R[0] = b_[0]; R[1] = b_[2]; R[2] = -b_[1]; R[3] = b_[3];
            }
        }
        hllc<double>(L, R, gamma, Fl);
        flux_global<double>(Fl, yface, F);
        const double sgn = high ? A : -A;  // outward flux of this cell
#pragma unroll
        for (int k = 0; k < 4; ++k) sum[k] += sgn * (double)F[k];
    }
    const double c = dt / g.vol;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        double v = beta * (X.f[k][ic] - c * sum[k]);
        if (alpha != 0.0) v += alpha * base.f[k][ic];
        out.f[k][ic] = v;
    }
}

__device__ __forceinline__ bool in_probe(const Grid &g, int ic, const double probe[4]) {
    int i = ic / g.ny, j = ic - (ic / g.ny) * g.ny;
    double cx = g.x0 + (i + 0.5) * g.hx, cy = g.y0 + (j + 0.5) * g.hy;
    return cx >= probe[0] && cx <= probe[1] && cy >= probe[2] && cy <= probe[3];
}

// Deterministic block sums: thread 0 of block b adds the block's sum to acc[b]
// (each kernel of the sweep launches the same number of blocks).
__device__ __forceinline__ void block_add(double x, double *acc) {
    __shared__ double sm[BLOCK / 32];
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = x;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int w = 0; w < BLOCK / 32; ++w) s += sm[w];
        acc[blockIdx.x] += s;
    }
    __syncthreads();  // sm is reused by the next call
}

// J partial sums (sum of p over the probe) and, with lam != null, dJ/dU at the
// final state (scale = 1 / probe cells) with the gamma part into gacc.
__global__ void __launch_bounds__(BLOCK) k_probe(Grid g, CF4 U, double gamma, double p0, double p1, double p2,
                                                 double p3, double scale, double *jacc, F4 lam, double *gacc) {
    int ic = blockIdx.x * BLOCK + threadIdx.x;
    const double probe[4] = {p0, p1, p2, p3};
    double pj = 0.0, gj = 0.0;
    if (ic < g.n) {
        double u[4];
        load4(U, ic, u);
        bool in = in_probe(g, ic, probe);
        double ke = 0.5 * ((u[1] * u[1] + u[2] * u[2]) / u[0]);
        if (in) {
            pj = (gamma - 1.0) * (u[3] - ke);
            gj = scale * (u[3] - ke);
        }
        if (lam.f[0]) {
            double vx = u[1] / u[0], vy = u[2] / u[0];
            double s = in ? scale * (gamma - 1.0) : 0.0;
            lam.f[0][ic] = s * 0.5 * (vx * vx + vy * vy);
            lam.f[1][ic] = -s * vx;
            lam.f[2][ic] = -s * vy;
            lam.f[3][ic] = s;
        }
    }
    block_add(pj, jacc);
    if (lam.f[0]) block_add(gj, gacc);
}

// --- vector-Jacobian product of L, pass 1: per face --------------------------
// mu_eff = coef * mu.  Each cell takes its two high faces (x and y): the
// cotangents of the face's low-side and high-side states, in the global
// primitive frame, go to fb[face][0..3] and fb[face][4..7]; the faces' gamma
// parts to gacc.
template <class S>
__global__ void __launch_bounds__(BLOCK, ZG_ADJ_VF_MINB) k_vjp_faces(Grid g, CF4 W, CF4T<S> gx, CF4T<S> gy,
                                                                     double gamma, CF4 mu, double coef, S *fbx,
                                                                     S *fby, double *gacc) {
    int ic = blockIdx.x * BLOCK + threadIdx.x;
    double gpart = 0.0;
    if (ic < g.n) {
        const double cv = coef / g.vol;
#pragma unroll 1
        for (int axis = 0; axis < 2; ++axis) {
            const bool yface = axis == 1;
            const Cell c = cell_of(g, ic);
            const int lo = ic, hi = yface ? yp(g, c).ic : xp(g, c).ic;
            const double half_h = 0.5 * (yface ? g.hy : g.hx), A = yface ? g.hx : g.hy;
            // cotangent of the global face flux: L_lo gets -A/V F, L_hi +A/V F
            double mF[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) mF[k] = cv * A * (mu.f[k][hi] - mu.f[k][lo]);
            S ml[4];  // in the face frame (transpose of flux_global)
            if (!yface) {
#pragma unroll
                for (int k = 0; k < 4; ++k) ml[k] = S(mF[k]);
            } else {
                ml[0] = S(mF[0]);
                ml[1] = S(mF[2]);
                ml[2] = S(-mF[1]);
                ml[3] = S(mF[3]);
            }
            S L[4], R[4], Lb[4], Rb[4];
            face_states<S>(W, yface ? gy : gx, lo, hi, S(half_h), yface, L, R);
            if constexpr (sizeof(S) == sizeof(double)) {
                hllc_vjp<double>(L, R, gamma, ml, Lb, Rb, gpart);
            } else {
                S gb = S(0);
                hllc_vjp<S>(L, R, S(gamma), ml, Lb, Rb, gb);
                gpart += (double)gb;
            }
            S *fb = yface ? fby : fbx;
            const size_t n = (size_t)g.n;
            // face frame -> global primitive (transpose of face_states' permutation)
            if (!yface) {
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    fb[k * n + ic] = Lb[k];
                    fb[(4 + k) * n + ic] = Rb[k];
                }
            } else {
                fb[0 * n + ic] = Lb[0];
                fb[1 * n + ic] = -Lb[2];
                fb[2 * n + ic] = Lb[1];
                fb[3 * n + ic] = Lb[3];
                fb[4 * n + ic] = Rb[0];
                fb[5 * n + ic] = -Rb[2];
                fb[6 * n + ic] = Rb[1];
                fb[7 * n + ic] = Rb[3];
            }
        }
    }
    block_add(gpart, gacc);
}

// --- vector-Jacobian product of L, pass 2: per cell ----------------------------
// A cell's state enters the face states of its four faces (as W_c +- slope
// h/2) and the slopes of itself and of its two neighbours on each axis; the
// cotangents come back here, then through the primitive map to U and gamma.
// out = base_coef * base + add + Ubar.
// Tiles of VJ x VI cells (j x i): every cell's slope partials are computed
// once and shared through shared memory with its two neighbours on each axis.
// Tile positions map to periodically wrapped cells, so a position outside the
// mesh (last tiles) holds a copy of the wrapped cell and every neighbour read
// from shared memory is the true periodic neighbour.
constexpr int VJ = 32, VI = 8;
#ifndef ZG_ADJ_VT_MINB
#define ZG_ADJ_VT_MINB 4
#endif

__device__ __forceinline__ int wrapc(int x, int n) {
    if (x < 0) x += n;
    if (x >= n) {
        x -= n;
        if (x >= n) x %= n;
    }
    return x;
}

// d0 * gb and d2 * gb of a cell's slope along one axis (its contributions to
// its low and high neighbour), and d1 * gb (its own), for field k: the
// differences in FP64, the partials in S
template <class S>
__device__ __forceinline__ void slope_terms(double wm, double w0, double wp, S i2h, S eps, S gb, double &to_lo,
                                            double &own, double &to_hi) {
    S d[3];
    slope_partials<S>(S(wm - w0), S(wp - w0), i2h, eps, d);
    to_lo = (double)(d[0] * gb);
    own = (double)(d[1] * gb);
    to_hi = (double)(d[2] * gb);
}

template <class S>
__global__ void __launch_bounds__(VJ *VI, ZG_ADJ_VT_MINB) k_vjp_cells_tiled(
    Grid g, CF4 W, double gamma, double eps, const S *fbx, const S *fby, CF4 base, double base_coef, CF4 add,
    F4 out, double *gacc) {
    // contributions of tile positions to their neighbours, for two fields at
    // a time: x (i) rows -1..VI, y (j) columns -1..VJ
    __shared__ double sx_lo[2][VI + 2][VJ], sx_hi[2][VI + 2][VJ];
    __shared__ double sy_lo[2][VI][VJ + 2], sy_hi[2][VI][VJ + 2];
    __shared__ double red[VJ * VI / 32];
    const int tj = threadIdx.x, ti = threadIdx.y, tid = ti * VJ + tj;
    const int i0 = blockIdx.y * VI, j0 = blockIdx.x * VJ;
    const size_t n = (size_t)g.n;
    const S i2x = S(0.5 / g.hx), i2y = S(0.5 / g.hy), hx2 = S(0.5 * g.hx), hy2 = S(0.5 * g.hy), se = S(eps);
    const Cell c{wrapc(i0 + ti, g.nx) * g.ny + wrapc(j0 + tj, g.ny), wrapc(i0 + ti, g.nx), wrapc(j0 + tj, g.ny)};
    const Cell cl = xm(g, c), cr = xp(g, c), cb = ym(g, c), ct = yp(g, c);
    const bool live = i0 + ti < g.nx && j0 + tj < g.ny;
    // halo work: positions of row -1 / VI (x terms only) and columns -1 / VJ
    // (y terms only), one per thread for the first 2 (VJ + VI) threads
    int h_axis = -1, h_side = 0, h_pos = 0;
    if (tid < 2 * VJ) {
        h_axis = 0;
        h_side = tid < VJ ? 0 : 1;
        h_pos = tid % VJ;
    } else if (tid < 2 * VJ + 2 * VI) {
        h_axis = 1;
        h_side = tid - 2 * VJ < VI ? 0 : 1;
        h_pos = (tid - 2 * VJ) % VI;
    }
    Cell hc{}, hm{}, hp{};
    if (h_axis == 0) {
        int hi_ = wrapc(h_side == 0 ? i0 - 1 : i0 + VI, g.nx), hj = wrapc(j0 + h_pos, g.ny);
        hc = Cell{hi_ * g.ny + hj, hi_, hj};
        hm = xm(g, hc);
        hp = xp(g, hc);
    } else if (h_axis == 1) {
        int hi_ = wrapc(i0 + h_pos, g.nx), hj = wrapc(h_side == 0 ? j0 - 1 : j0 + VJ, g.ny);
        hc = Cell{hi_ * g.ny + hj, hi_, hj};
        hm = ym(g, hc);
        hp = yp(g, hc);
    }
    // two fields per pair of barriers: their loads are in flight together
    double wt[4], wc[4];
#pragma unroll
    for (int k0 = 0; k0 < 4; k0 += 2) {
        double part[2];
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            const int k = k0 + q;
            const S *fl = fbx + k * n, *fh = fbx + (4 + k) * n, *gl = fby + k * n, *gh = fby + (4 + k) * n;
            const double *w = W.f[k];
            // own position: slope cotangents and partials on both axes
            const S xl_c = fl[c.ic], xh_l = fh[cl.ic], yl_c = gl[c.ic], yh_b = gh[cb.ic];
            const double w_c = w[c.ic];
            wc[k] = w_c;
            double ox, oy, lo, hi;
            slope_terms<S>(w[cl.ic], w_c, w[cr.ic], i2x, se, hx2 * (xl_c - xh_l), lo, ox, hi);
            sx_lo[q][ti + 1][tj] = lo;
            sx_hi[q][ti + 1][tj] = hi;
            slope_terms<S>(w[cb.ic], w_c, w[ct.ic], i2y, se, hy2 * (yl_c - yh_b), lo, oy, hi);
            sy_lo[q][ti][tj + 1] = lo;
            sy_hi[q][ti][tj + 1] = hi;
            part[q] = (double)xl_c + (double)xh_l + (double)yl_c + (double)yh_b + ox + oy;
            if (h_axis == 0) {
                const S gb = hx2 * (fl[hc.ic] - fh[hm.ic]);
                double o;
                slope_terms<S>(w[hm.ic], w[hc.ic], w[hp.ic], i2x, se, gb, lo, o, hi);
                if (h_side == 0) sx_hi[q][0][h_pos] = hi;
                else sx_lo[q][VI + 1][h_pos] = lo;
            } else if (h_axis == 1) {
                const S gb = hy2 * (gl[hc.ic] - gh[hm.ic]);
                double o;
                slope_terms<S>(w[hm.ic], w[hc.ic], w[hp.ic], i2y, se, gb, lo, o, hi);
                if (h_side == 0) sy_hi[q][h_pos][0] = hi;
                else sy_lo[q][h_pos][VJ + 1] = lo;
            }
        }
        __syncthreads();
#pragma unroll
        for (int q = 0; q < 2; ++q)  // the low neighbours' slopes (this cell is their high neighbour), the high ones'
            wt[k0 + q] = part[q] + sx_hi[q][ti][tj] + sx_lo[q][ti + 2][tj] + sy_hi[q][ti][tj] + sy_lo[q][ti][tj + 2];
        __syncthreads();
    }
    double gpart = 0.0;
    if (live) {
        const int ic = c.ic;
        // the primitive map's partials at the stage's primitive state
        // (rho, u, v, p): E - rho |v|^2 / 2 = p / (gamma - 1)
        const double ir = 1.0 / wc[0], u = wc[1], v = wc[2], gm1 = gamma - 1.0;
        double ub[4];
        ub[0] = wt[0] - wt[1] * u * ir - wt[2] * v * ir + wt[3] * gm1 * 0.5 * (u * u + v * v);
        ub[1] = wt[1] * ir - wt[3] * gm1 * u;
        ub[2] = wt[2] * ir - wt[3] * gm1 * v;
        ub[3] = wt[3] * gm1;
        gpart = wt[3] * (wc[3] / gm1);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            double vv = ub[k];
            if (base.f[0]) vv += base_coef * base.f[k][ic];
            if (add.f[0]) vv += add.f[k][ic];
            out.f[k][ic] = vv;
        }
    }
    for (int o = 16; o > 0; o >>= 1) gpart += __shfl_xor_sync(0xffffffffu, gpart, o);
    if ((tid & 31) == 0) red[tid >> 5] = gpart;
    __syncthreads();
    if (tid == 0) {
        double s2 = 0.0;
        for (int w2 = 0; w2 < VJ * VI / 32; ++w2) s2 += red[w2];
        gacc[blockIdx.y * gridDim.x + blockIdx.x] += s2;
    }
}

// dJ/d rho_0 from lambda^0 (U_0 = (rho, rho u, rho v, p/(gamma-1) + rho |v|^2 / 2)),
// and the gamma part of U_0's energy.
__global__ void __launch_bounds__(BLOCK) k_seed(Grid g, CF4 W0, double gamma, CF4 lam, double *grad,
                                                double *gacc) {
    int ic = blockIdx.x * BLOCK + threadIdx.x;
    double gpart = 0.0;
    if (ic < g.n) {
        double u = W0.f[1][ic], v = W0.f[2][ic], p = W0.f[3][ic];
        double l0 = lam.f[0][ic], l1 = lam.f[1][ic], l2 = lam.f[2][ic], l3 = lam.f[3][ic];
        if (grad) grad[ic] = l0 + l1 * u + l2 * v + l3 * (0.5 * (u * u + v * v));
        double gm1 = gamma - 1.0;
        gpart = l3 * (-p / (gm1 * gm1));
    }
    block_add(gpart, gacc);
}

}  // namespace adj
}  // namespace zg

using namespace zg::adj;

struct zg_adj {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    Grid g{};
    // storage
    double *d_all = nullptr;
    size_t cap_ckpt = 0, cap_seg = 0;  // checkpoints and segment states held
    double *d_acc = nullptr;           // per-block accumulators: J, gamma
    F4 U0{}, Ua{}, Ub{}, Ustar{}, W{}, gx{}, gy{}, lamA{}, lamB{}, lamS{};
    double *fbx = nullptr, *fby = nullptr;  // face-state cotangents, 8 n each
    std::vector<F4> ckpt;
    // two sets of segment storage: the states, stage values, primitive states
    // and slopes of both stages of every step of a segment, kept from the
    // segment's recomputation for the reverse sweep.  Segment sg lives in set
    // sg & 1, so the recomputation of segment sg - 1 (on `rstream`) runs while
    // segment sg is swept backwards (on `stream`).
    std::vector<F4> seg[2], segstar[2], segW[2], segGx[2], segGy[2];
    cudaStream_t rstream = nullptr;                                    // segment recomputation
    cudaEvent_t ev_fwd = nullptr, ev_rec = nullptr, ev_rev = nullptr;  // ordering between the two streams
    long long launches = 0;
};

namespace {

struct DevGuard {
    int prev = -1;
    explicit DevGuard(int d) {
        cudaGetDevice(&prev);
        if (prev != d) cudaSetDevice(d);
    }
    ~DevGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

int afail(zg_adj *a, int code, const std::string &m) {
    if (a) a->err = m;
    return code;
}

CF4 cf(const F4 &x) { return CF4{{x.f[0], x.f[1], x.f[2], x.f[3]}}; }
const CF4 kNull{{nullptr, nullptr, nullptr, nullptr}};
const F4 kNullW{{nullptr, nullptr, nullptr, nullptr}};

unsigned nblocks(const zg_adj *a) { return (unsigned)((a->g.n + BLOCK - 1) / BLOCK); }
dim3 vtiles(const zg_adj *a) { return dim3((unsigned)((a->g.ny + VJ - 1) / VJ), (unsigned)((a->g.nx + VI - 1) / VI)); }
// per-block accumulator slots: enough for the 1-D kernels and the tiles
unsigned nacc(const zg_adj *a) {
    dim3 t = vtiles(a);
    return std::max(nblocks(a), t.x * t.y);
}

// (re)allocate for `ckpts` checkpoints and segments of `seglen` steps
int reserve(zg_adj *a, size_t ckpts, size_t seglen) {
    if (a->d_all && ckpts <= a->cap_ckpt && seglen <= a->cap_seg) return ZG_OK;
    cudaFree(a->d_all);
    a->d_all = nullptr;
    size_t n = (size_t)a->g.n;
    size_t fields = 10 * 4 + 16 + 4 * ckpts + 2 * (4 * (seglen + 1) + 4 * seglen + 3 * 4 * (2 * seglen));
    cudaError_t e = cudaMalloc(&a->d_all, fields * n * sizeof(double));
    if (e != cudaSuccess) return afail(a, ZG_ERR_ALLOC, std::string("adjoint storage: ") + cudaGetErrorString(e));
    double *p = a->d_all;
    auto take = [&p, n]() {
        F4 x;
        for (int k = 0; k < 4; ++k) {
            x.f[k] = p;
            p += n;
        }
        return x;
    };
    for (F4 *x : {&a->U0, &a->Ua, &a->Ub, &a->Ustar, &a->W, &a->gx, &a->gy, &a->lamA, &a->lamB, &a->lamS})
        *x = take();
    a->fbx = take().f[0];  // two consecutive groups of 4 n: 8 n
    take();
    a->fby = take().f[0];
    take();
    a->ckpt.assign(ckpts, F4{});
    for (auto &c : a->ckpt) c = take();
    for (int b = 0; b < 2; ++b) {
        a->seg[b].assign(seglen + 1, F4{});
        for (auto &c : a->seg[b]) c = take();
        a->segstar[b].assign(seglen, F4{});
        for (auto &c : a->segstar[b]) c = take();
        for (auto *v : {&a->segW[b], &a->segGx[b], &a->segGy[b]}) {
            v->assign(2 * seglen, F4{});
            for (auto &c : *v) c = take();
        }
    }
    a->cap_ckpt = ckpts;
    a->cap_seg = seglen;
    return ZG_OK;
}

void copy4(zg_adj *a, cudaStream_t st, const F4 &dst, const F4 &src) {
    for (int k = 0; k < 4; ++k)
        cudaMemcpyAsync(dst.f[k], src.f[k], (size_t)a->g.n * sizeof(double), cudaMemcpyDeviceToDevice, st);
}

struct WG {  // primitive states and slopes of one stage
    F4 W, gx, gy;
};

// one Heun step: X -> out (stage value into `star`); the stages' primitive
// states and slopes go to sa and sb
// (need_out = false: the step's result is not wanted, only its stages)
// the same arrays viewed as element type S (the mixed form keeps its FP32
// slopes and face cotangents in the first half of the FP64-sized buffers;
// the primitive states are FP64 in both forms)
template <class S>
F4T<S> as(const F4 &x) {
    return F4T<S>{{reinterpret_cast<S *>(x.f[0]), reinterpret_cast<S *>(x.f[1]), reinterpret_cast<S *>(x.f[2]),
                   reinterpret_cast<S *>(x.f[3])}};
}
template <class S>
CF4T<S> cas(const F4 &x) {
    F4T<S> y = as<S>(x);
    return CF4T<S>{{y.f[0], y.f[1], y.f[2], y.f[3]}};
}

template <class S>
void heun_step_t(zg_adj *a, cudaStream_t st, const zg_adj_params &p, const F4 &X, const F4 &star, const F4 &out,
                 const WG &sa, const WG &sb, bool need_out) {
    unsigned nb = nblocks(a);
    k_prim_grad<S><<<nb, BLOCK, 0, st>>>(a->g, cf(X), p.gamma, p.limiter_eps, sa.W, as<S>(sa.gx), as<S>(sa.gy));
    k_flux_update<S><<<nb, BLOCK, 0, st>>>(a->g, cf(sa.W), cas<S>(sa.gx), cas<S>(sa.gy), p.gamma, cf(X), kNull,
                                           0.0, 1.0, p.dt, star);
    k_prim_grad<S><<<nb, BLOCK, 0, st>>>(a->g, cf(star), p.gamma, p.limiter_eps, sb.W, as<S>(sb.gx), as<S>(sb.gy));
    a->launches += 3;
    if (!need_out) return;
    k_flux_update<S><<<nb, BLOCK, 0, st>>>(a->g, cf(sb.W), cas<S>(sb.gx), cas<S>(sb.gy), p.gamma, cf(star),
                                           cf(X), 0.5, 0.5, p.dt, out);
    ++a->launches;
}
void heun_step(zg_adj *a, cudaStream_t st, const zg_adj_params &p, const F4 &X, const F4 &star, const F4 &out,
               const WG &sa, const WG &sb, bool need_out = true) {
    if (p.precision == ZG_MIXED) heun_step_t<float>(a, st, p, X, star, out, sa, sb, need_out);
    else heun_step_t<double>(a, st, p, X, star, out, sa, sb, need_out);
}
WG scratch(const zg_adj *a) { return WG{a->W, a->gx, a->gy}; }
WG seg_stage(const zg_adj *a, int b, int t, int stage) {
    return WG{a->segW[b][2 * t + stage], a->segGx[b][2 * t + stage], a->segGy[b][2 * t + stage]};
}
// recompute segment sg (len steps from checkpoint sg) into set sg & 1
void recompute(zg_adj *a, cudaStream_t st, const zg_adj_params &p, int sg, int len) {
    const int b = sg & 1;
    copy4(a, st, a->seg[b][0], a->ckpt[sg]);
    for (int t = 0; t < len; ++t)
        heun_step(a, st, p, a->seg[b][t], a->segstar[b][t], a->seg[b][t + 1], seg_stage(a, b, t, 0),
                  seg_stage(a, b, t, 1), t + 1 < len);
}

// out = base_coef * base + add + L'(X)^T (coef * mu), with X's primitive
// states and slopes in wg (X itself is not read: the primitive map's partials
// are taken at its primitive state)
template <class S>
void vjp_t(zg_adj *a, const zg_adj_params &p, const WG &wg, const F4 &mu, double coef, const F4 &base,
           double base_coef, const CF4 &add, const F4 &out, double *gacc) {
    unsigned nb = nblocks(a);
    S *fbx = reinterpret_cast<S *>(a->fbx), *fby = reinterpret_cast<S *>(a->fby);
    k_vjp_faces<S><<<nb, BLOCK, 0, a->stream>>>(a->g, cf(wg.W), cas<S>(wg.gx), cas<S>(wg.gy), p.gamma, cf(mu),
                                                coef, fbx, fby, gacc);
    k_vjp_cells_tiled<S><<<vtiles(a), dim3(VJ, VI), 0, a->stream>>>(a->g, cf(wg.W), p.gamma, p.limiter_eps, fbx,
                                                                     fby, cf(base), base_coef, add, out, gacc);
    a->launches += 2;
}
void vjp(zg_adj *a, const zg_adj_params &p, const WG &wg, const F4 &mu, double coef, const F4 &base,
         double base_coef, const CF4 &add, const F4 &out, double *gacc) {
    if (p.precision == ZG_MIXED) vjp_t<float>(a, p, wg, mu, coef, base, base_coef, add, out, gacc);
    else vjp_t<double>(a, p, wg, mu, coef, base, base_coef, add, out, gacc);
}

int check_params(zg_adj *a, const zg_adj_params *p) {
    if (!p) return afail(a, ZG_ERR_ARG, "null parameters");
    if (!(p->gamma > 1.0)) return afail(a, ZG_ERR_ARG, "gamma must exceed 1");
    if (!(p->dt > 0.0)) return afail(a, ZG_ERR_ARG, "dt must be positive (see zg_adj_cfl_dt)");
    if (p->steps < 1 || p->checkpoint_every < 1) return afail(a, ZG_ERR_ARG, "steps and checkpoint_every >= 1");
    if (!(p->limiter_eps > 0.0)) return afail(a, ZG_ERR_ARG, "limiter_eps must be positive");
    if (p->precision != ZG_FP64 && p->precision != ZG_MIXED) return afail(a, ZG_ERR_ARG, "unknown precision");
    return ZG_OK;
}

int finish_sum(zg_adj *a, double *out2) {
    unsigned nb = nacc(a);
    std::vector<double> h(2 * (size_t)nb);
    cudaError_t e = cudaMemcpyAsync(h.data(), a->d_acc, h.size() * sizeof(double), cudaMemcpyDeviceToHost, a->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(a->stream);
    if (e != cudaSuccess) return afail(a, ZG_ERR_CUDA, cudaGetErrorString(e));
    out2[0] = out2[1] = 0.0;
    for (unsigned b = 0; b < nb; ++b) out2[0] += h[b];
    for (unsigned b = 0; b < nb; ++b) out2[1] += h[nb + b];
    return ZG_OK;
}

int probe_count(const zg_adj *a, const zg_adj_params &p) {
    int c = 0;
    for (int i = 0; i < a->g.nx; ++i)
        for (int j = 0; j < a->g.ny; ++j) {
            double cx = a->g.x0 + (i + 0.5) * a->g.hx, cy = a->g.y0 + (j + 0.5) * a->g.hy;
            if (cx >= p.probe[0] && cx <= p.probe[1] && cy >= p.probe[2] && cy <= p.probe[3]) ++c;
        }
    return c;
}

}  // namespace

extern "C" {

void zg_adj_default_params(zg_adj_params *p) {
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->gamma = 1.4;
    p->dt = 0.0;
    p->steps = 100;
    p->checkpoint_every = 10;
    p->limiter_eps = 1.0e-8;
    p->probe[0] = 0.6;
    p->probe[1] = 0.7;
    p->probe[2] = 0.6;
    p->probe[3] = 0.7;
}

int zg_adj_create(zg_adj **out, int device, int nx, int ny, double x_min, double x_max, double y_min, double y_max) {
    if (!out) return ZG_ERR_ARG;
    *out = nullptr;
    if (nx < 3 || ny < 3 || !(x_max > x_min) || !(y_max > y_min)) return ZG_ERR_ARG;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || device < 0 || device >= count) return ZG_ERR_CUDA;
    auto *a = new zg_adj();
    a->device = device;
    a->g.nx = nx;
    a->g.ny = ny;
    a->g.n = nx * ny;
    a->g.hx = (x_max - x_min) / nx;
    a->g.hy = (y_max - y_min) / ny;
    a->g.vol = a->g.hx * a->g.hy;
    a->g.x0 = x_min;
    a->g.y0 = y_min;
    DevGuard gd(device);
    if (cudaMalloc(&a->d_acc, 2 * nacc(a) * sizeof(double)) != cudaSuccess) {
        delete a;
        return ZG_ERR_ALLOC;
    }
    int lo = 0, hi = 0;
    cudaDeviceGetStreamPriorityRange(&lo, &hi);  // lo: the numerically largest, lowest priority
    if (cudaStreamCreateWithPriority(&a->rstream, cudaStreamNonBlocking, lo) != cudaSuccess ||
        cudaEventCreateWithFlags(&a->ev_fwd, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&a->ev_rec, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&a->ev_rev, cudaEventDisableTiming) != cudaSuccess) {
        zg_adj_destroy(a);
        return ZG_ERR_CUDA;
    }
    *out = a;
    return ZG_OK;
}

int zg_adj_destroy(zg_adj *a) {
    if (!a) return ZG_ERR_ARG;
    {
        DevGuard gd(a->device);
        if (a->stream) cudaStreamSynchronize(a->stream);
        else cudaDeviceSynchronize();
        if (a->rstream) {
            cudaStreamSynchronize(a->rstream);
            cudaStreamDestroy(a->rstream);
        }
        for (cudaEvent_t e : {a->ev_fwd, a->ev_rec, a->ev_rev})
            if (e) cudaEventDestroy(e);
        cudaFree(a->d_all);
        cudaFree(a->d_acc);
    }
    delete a;
    return ZG_OK;
}

const char *zg_adj_last_error(const zg_adj *a) { return a ? a->err.c_str() : "null handle"; }

int zg_adj_set_stream(zg_adj *a, void *stream) {
    if (!a) return ZG_ERR_ARG;
    a->stream = (cudaStream_t)stream;
    return ZG_OK;
}

int zg_adj_launch_count(const zg_adj *a, long long *count) {
    if (!a || !count) return ZG_ERR_ARG;
    *count = a->launches;
    return ZG_OK;
}

int zg_adj_forward(zg_adj *a, const zg_adj_params *p, const double *rho, const double *u, const double *v,
                   const double *pr, double *J) {
    if (!a) return ZG_ERR_ARG;
    int rc = check_params(a, p);
    if (rc != ZG_OK) return rc;
    if (!rho || !u || !v || !pr || !J) return afail(a, ZG_ERR_ARG, "null array");
    DevGuard gd(a->device);
    rc = reserve(a, std::max<size_t>(a->cap_ckpt, 1), std::max<size_t>(a->cap_seg, 1));
    if (rc != ZG_OK) return rc;
    unsigned nb = nblocks(a);
    CF4 w0{{rho, u, v, pr}};
    k_init<<<nb, BLOCK, 0, a->stream>>>(a->g, w0, p->gamma, a->Ua);
    ++a->launches;
    F4 cur = a->Ua, nxt = a->Ub;
    for (int s = 0; s < p->steps; ++s) {
        heun_step(a, a->stream, *p, cur, a->Ustar, nxt, scratch(a), scratch(a));
        std::swap(cur, nxt);
    }
    cudaMemsetAsync(a->d_acc, 0, 2 * nacc(a) * sizeof(double), a->stream);
    int np = probe_count(a, *p);
    if (np == 0) return afail(a, ZG_ERR_ARG, "no cell centre inside the probe box");
    k_probe<<<nb, BLOCK, 0, a->stream>>>(a->g, cf(cur), p->gamma, p->probe[0], p->probe[1], p->probe[2], p->probe[3],
                                         1.0 / np, a->d_acc, kNullW, a->d_acc + nacc(a));
    ++a->launches;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return afail(a, ZG_ERR_CUDA, cudaGetErrorString(e));
    double s2[2];
    rc = finish_sum(a, s2);
    if (rc != ZG_OK) return rc;
    *J = s2[0] / np;
    return ZG_OK;
}

int zg_adj_gradient(zg_adj *a, const zg_adj_params *p, const double *rho, const double *u, const double *v,
                    const double *pr, double *J, double *dJ_drho, double *dJ_dgamma) {
    if (!a) return ZG_ERR_ARG;
    int rc = check_params(a, p);
    if (rc != ZG_OK) return rc;
    if (!rho || !u || !v || !pr || !J) return afail(a, ZG_ERR_ARG, "null array");
    DevGuard gd(a->device);
    const int N = p->steps, K = p->checkpoint_every;
    const int nseg = (N + K - 1) / K;
    rc = reserve(a, (size_t)nseg, (size_t)std::min(K, N));
    if (rc != ZG_OK) return rc;
    const unsigned nb = nblocks(a);
    const int np = probe_count(a, *p);
    if (np == 0) return afail(a, ZG_ERR_ARG, "no cell centre inside the probe box");
    CF4 w0{{rho, u, v, pr}};

    // forward with checkpoints at steps 0, K, 2K, ...; the last two segments
    // keep their states and stages (one in each set) for the reverse sweep
    const int stored0 = std::max(0, nseg - 2);  // first segment the forward keeps
    const int keep0 = stored0 * K;
    k_init<<<nb, BLOCK, 0, a->stream>>>(a->g, w0, p->gamma, a->ckpt[0]);
    ++a->launches;
    F4 cur = a->ckpt[0];
    for (int s = 0; s < N; ++s) {
        if (s >= keep0) {
            const int sg = s / K, t = s - sg * K, b = sg & 1;
            if (t == 0) copy4(a, a->stream, a->seg[b][0], cur);
            heun_step(a, a->stream, *p, a->seg[b][t], a->segstar[b][t], a->seg[b][t + 1], seg_stage(a, b, t, 0),
                      seg_stage(a, b, t, 1));
            cur = a->seg[b][t + 1];
            continue;
        }
        bool keep = (s + 1) % K == 0 && (s + 1) / K < nseg;
        F4 nxt = keep ? a->ckpt[(s + 1) / K] : (cur.f[0] == a->Ua.f[0] ? a->Ub : a->Ua);
        heun_step(a, a->stream, *p, cur, a->Ustar, nxt, scratch(a), scratch(a));
        cur = nxt;
    }
    // J and lambda^N
    cudaMemsetAsync(a->d_acc, 0, 2 * nacc(a) * sizeof(double), a->stream);
    F4 lam = a->lamA, lam_prev = a->lamB;
    k_probe<<<nb, BLOCK, 0, a->stream>>>(a->g, cf(cur), p->gamma, p->probe[0], p->probe[1], p->probe[2], p->probe[3],
                                         1.0 / np, a->d_acc, lam, a->d_acc + nacc(a));
    ++a->launches;
    double *gacc = a->d_acc + nacc(a);

    // reverse sweep, segment by segment.  Below the two kept segments, the
    // recomputation of segment sg - 1 (rstream, set (sg - 1) & 1) overlaps the
    // sweep of segment sg (stream, set sg & 1); it starts once the checkpoints
    // exist and the sweep of segment sg + 1, which used the same set, is
    // done.  Every recomputation is waited for on `stream` before its segment
    // is swept, so the work of both streams has ended when `stream` has.
    cudaEventRecord(a->ev_fwd, a->stream);
    cudaStreamWaitEvent(a->rstream, a->ev_fwd, 0);
    for (int sg = nseg - 1; sg >= 0; --sg) {
        const int s0 = sg * K, len = std::min(K, N - s0), b = sg & 1;
        if (sg < stored0) cudaStreamWaitEvent(a->stream, a->ev_rec, 0);  // segment sg recomputed
        if (sg > 0 && sg - 1 < stored0) {
            if (sg + 1 < nseg) cudaStreamWaitEvent(a->rstream, a->ev_rev, 0);  // set of sg - 1 free
            recompute(a, a->rstream, *p, sg - 1, K);
            cudaEventRecord(a->ev_rec, a->rstream);
        }
        for (int t = len - 1; t >= 0; --t) {
            // stage B: lambda* = 1/2 lambda^{n+1} + L'(U*)^T (dt/2 lambda^{n+1})
            vjp(a, *p, seg_stage(a, b, t, 1), lam, 0.5 * p->dt, lam, 0.5, kNull, a->lamS, gacc);
            // stage A: lambda^n = 1/2 lambda^{n+1} + lambda* + L'(U^n)^T (dt lambda*)
            vjp(a, *p, seg_stage(a, b, t, 0), a->lamS, p->dt, lam, 0.5, cf(a->lamS), lam_prev, gacc);
            std::swap(lam, lam_prev);
        }
        cudaEventRecord(a->ev_rev, a->stream);
    }
    k_seed<<<nb, BLOCK, 0, a->stream>>>(a->g, w0, p->gamma, cf(lam), dJ_drho, gacc);
    ++a->launches;
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return afail(a, ZG_ERR_CUDA, cudaGetErrorString(e));
    double s2[2];
    rc = finish_sum(a, s2);
    if (rc != ZG_OK) return rc;
    *J = s2[0] / np;
    if (dJ_dgamma) *dJ_dgamma = s2[1];
    return ZG_OK;
}

int zg_adj_cfl_dt(zg_adj *a, double gamma, double CFL, const double *rho, const double *u, const double *v,
                  const double *pr, double *dt) {
    if (!a || !rho || !u || !v || !pr || !dt) return ZG_ERR_ARG;
    DevGuard gd(a->device);
    size_t n = (size_t)a->g.n;
    std::vector<double> r(n), uu(n), vv(n), pp(n);
    const double *src[4] = {rho, u, v, pr};
    double *dst[4] = {r.data(), uu.data(), vv.data(), pp.data()};
    for (int k = 0; k < 4; ++k)
        if (cudaMemcpyAsync(dst[k], src[k], n * sizeof(double), cudaMemcpyDeviceToHost, a->stream) != cudaSuccess)
            return afail(a, ZG_ERR_CUDA, "zg_adj_cfl_dt copy");
    if (cudaStreamSynchronize(a->stream) != cudaSuccess) return afail(a, ZG_ERR_CUDA, "zg_adj_cfl_dt sync");
    // SmFluid::compute_dt (sm_fluid.cpp:104-114) with the incircle of a
    // rectangle cell: min(hx, hy) / (|v| + c)
    double h = std::min(a->g.hx, a->g.hy), best = 1.0e300;
    for (size_t i = 0; i < n; ++i) {
        double c = std::sqrt(gamma * pp[i] / r[i]);
        best = std::min(best, h / (std::sqrt(uu[i] * uu[i] + vv[i] * vv[i]) + c));
    }
    *dt = CFL * best;
    return ZG_OK;
}

}  // extern "C"
