// tr_vof.cu -- zephyr's scalar VOF transport solver Transfer
// (math/solver/transfer.cpp) on a uniform non-periodic rectangle: the VOF
// and VOF_CRP fluxes from swept polygons (flux_VOF, transfer.cpp:250-292),
// the CRP family (CRP_V3, CRP_V5, CRP_SE, CRP_N1, CRP_N2; transfer.cpp:
// 109-248), the MUSCL family (transfer.cpp:345-469), the interface
// reconstruction InterfaceRecovery
// (geom/interface_recovery.cpp) with the polygon clipping and Newton section
// search of geom/primitives/polygon.cpp, and the CFL time step.
//
// Layout: one thread per face for the fluxes, one per cell for the rest.
// Cell ic = i * ny + j (the reference's order); x faces i * ny + j
// (i = 0..nx), y faces i * (ny + 1) + j (j = 0..ny).  Each interior face is
// evaluated once: the reference evaluates it from both cells, and the two
// results are exact negatives except where the normal velocity is exactly 0
// (both cells then take the other one as upwind) and for CRP_N2 (whose
// neighbour plane differs); those cases are evaluated from each side, and so
// is every face of the MUSCL family.  Each cell sums its faces in slot order
// L, R, B, T as the reference does.
//
// Arithmetic follows the reference term by term (compiled with -fmad=false).
// The reference's vectors carry a z component that is +-0 throughout the
// 2-D problem; it only ever adds a signed zero to a sum, which at most changes
// the sign of an exact zero, and no comparison or later product here tells
// the two zeros apart, so the kernels drop it.  Two deliberate departures,
// neither seen on any tested input:
//  * an upwind cell with u1 == 0 contributes 0 * area(swept polygon); the
//    kernel returns 0 without clipping (the polygon's area is finite unless
//    a clip meets an edge lying exactly on its line with opposite-signed
//    rounding, where the reference's product would be NaN);
//  * the normal-adjustment pass reads the neighbours' normals from before the
//    pass (the reference loop updates in place, in cell order).  Only whether
//    a neighbour's normal is zero is read, and an adjusted normal is zero only
//    if its two section points coincide exactly.
#include <math_constants.h>

#include <cfloat>
#include <cstdint>

#include "mmf_math.cuh"
#include "tr_types.h"

namespace zg {
namespace tr {
namespace {

using mmf::average_flux;
using mmf::between;
using mmf::face_fraction;
using mmf::face_fraction_s;
using mmf::face_fraction_v3;
using mmf::face_fraction_v5;
using mmf::sgn;
using mmf::sorted2;

constexpr int BLOCK = 128;
constexpr int MAXV = 12;  // polygon capacity (a convex quadrilateral clipped three times has at most 7)

__device__ __forceinline__ double dmin(double a, double b) { return (b < a) ? b : a; }  // std::min
__device__ __forceinline__ double dmax(double a, double b) { return (a < b) ? b : a; }  // std::max

struct P2 {
    double x, y;
};
__device__ __forceinline__ P2 mk(double x, double y) {
    P2 r;
    r.x = x;
    r.y = y;
    return r;
}
__device__ __forceinline__ double cross2(P2 a, P2 b) { return a.x * b.y - a.y * b.x; }
// [v1 - c, v2 - c].z (polygon.cpp:153-157)
__device__ __forceinline__ double cross_c(double cx, double cy, double x1, double y1, double x2, double y2) {
    return (x1 - cx) * (y2 - cy) - (y1 - cy) * (x2 - cx);
}
// Eigen normalized(): divide by sqrt(squaredNorm) when that is positive
__device__ __forceinline__ P2 normalized(P2 a) {
    double sn = a.x * a.x + a.y * a.y;
    if (sn > 0.0) {
        double s = sqrt(sn);
        return mk(a.x / s, a.y / s);
    }
    return a;
}
// Eigen isZero(1e-12): no component above 1e-12 in magnitude (NaN passes)
__device__ __forceinline__ bool is_zero(double x, double y) { return !(fabs(x) > 1.0e-12) && !(fabs(y) > 1.0e-12); }

// Polygon with its m_center, the mean of the vertices (polygon.cpp:35-45).
struct Poly {
    int n;
    double cx, cy;
    double x[MAXV], y[MAXV];
};

__device__ __forceinline__ void set_center(Poly &P) {
    double sx = 0.0, sy = 0.0;
    for (int k = 0; k < P.n; ++k) {
        sx = sx + P.x[k];
        sy = sy + P.y[k];
    }
    if (P.n > 0) {
        sx = sx / double(P.n);
        sy = sy / double(P.n);
    }
    P.cx = sx;
    P.cy = sy;
}

// Polygon::area (polygon.cpp:191-209)
__device__ double area(const Poly &P) {
    double S = 0.0;
    for (int i = 0; i < P.n; ++i) {
        int k = i + 1 == P.n ? 0 : i + 1;
        S += cross_c(P.cx, P.cy, P.x[i], P.y[i], P.x[k], P.y[k]);
    }
    return 0.5 * S;
}

// Polygon::clip (polygon.cpp:266-293): the part with (v - p).n <= 1e-14.
__device__ void clip(const Poly &P, P2 p, P2 n, Poly &Q, int *err) {
    Q.n = 0;
    if (P.n > 0) {
        const double d0 = (P.x[0] - p.x) * n.x + (P.y[0] - p.y) * n.y;
        double dot1 = d0;
        for (int i = 0; i < P.n; ++i) {
            const bool last = i + 1 == P.n;
            const int k = last ? 0 : i + 1;
            const double x1 = P.x[i], y1 = P.y[i], x2 = P.x[k], y2 = P.y[k];
            const double dot2 = last ? d0 : (x2 - p.x) * n.x + (y2 - p.y) * n.y;
            const double Det = (x2 - x1) * n.x + (y2 - y1) * n.y;
            if (dot1 <= 1.0e-14) {
                if (Q.n < MAXV) {
                    Q.x[Q.n] = x1;
                    Q.y[Q.n] = y1;
                    ++Q.n;
                } else {
                    atomicAdd(err, 1);
                }
            }
            if (dot1 * dot2 < 0.0) {
                if (Q.n < MAXV) {
                    Q.x[Q.n] = (dot2 * x1 - dot1 * x2) / Det;
                    Q.y[Q.n] = (dot2 * y1 - dot1 * y2) / Det;
                    ++Q.n;
                } else {
                    atomicAdd(err, 1);
                }
            }
            dot1 = dot2;
        }
    }
    set_center(Q);
}

// intersection2D::exist(ray, segment) (intersection.cpp:10-29)
__device__ bool exist_ray(P2 rp, P2 tau, double x1, double y1, double x2, double y2) {
    double dot1 = cross2(mk(x1 - rp.x, y1 - rp.y), tau);
    double dot2 = cross2(mk(x2 - rp.x, y2 - rp.y), tau);
    if (dot1 * dot2 <= 0.0 && dot2 != 0.0) {
        double det = dot2 - dot1;
        double vx = (dot2 * x1 - dot1 * x2) / det, vy = (dot2 * y1 - dot1 * y2) / det;
        if ((vx - rp.x) * tau.x + (vy - rp.y) * tau.y > 0.0) return true;
    }
    return false;
}

// Polygon::inside (polygon.cpp:159-172)
__device__ bool inside(const Poly &P, P2 p) {
    const P2 tau = mk(0.123, 0.346433);
    int counter = 0;
    for (int i = 0; i < P.n; ++i) {
        int k = i + 1 == P.n ? 0 : i + 1;
        if (exist_ray(p, tau, P.x[i], P.y[i], P.x[k], P.y[k])) ++counter;
    }
    return counter % 2 > 0;
}

__device__ __forceinline__ bool bad_normal(P2 n) {  // polygon.cpp:14-16
    return isnan(n.x) || isnan(n.y) || n.x * n.x + n.y * n.y == 0.0;
}

struct AnS {
    double area;
    P2 p1, p2;
    bool tri_in, tri_out;
};

// clip_area_and_slice (polygon.cpp:310-400)
__device__ AnS clip_area_and_slice(const Poly &P, P2 p, P2 n, bool slice) {
    AnS r;
    r.area = 0.0;
    r.tri_in = r.tri_out = false;
    r.p1 = r.p2 = mk(0.0, 0.0);
    if (P.n == 0) {
        r.p1 = r.p2 = mk(CUDART_NAN, CUDART_NAN);
        return r;
    }
    if (bad_normal(n)) {
        r.p1 = r.p2 = mk(CUDART_NAN, CUDART_NAN);
        r.area = inside(P, p) ? area(P) : 0.0;
        return r;
    }
    const int size = P.n;
    int idx_out_in = -1, idx_in_out = -1;
    P2 sec_out_in = mk(0.0, 0.0), sec_in_out = mk(0.0, 0.0);
    double dot1 = (P.x[size - 1] - p.x) * n.x + (P.y[size - 1] - p.y) * n.y;
    for (int i2 = 0; i2 < size; ++i2) {
        const double dot2 = (P.x[i2] - p.x) * n.x + (P.y[i2] - p.y) * n.y;
        if (dot1 * dot2 < 0.0) {
            const int i1 = i2 == 0 ? size - 1 : i2 - 1;
            const double x1 = P.x[i1], y1 = P.y[i1], x2 = P.x[i2], y2 = P.y[i2];
            const double Det = (x2 - x1) * n.x + (y2 - y1) * n.y;
            const P2 sec = mk((dot2 * x1 - dot1 * x2) / Det, (dot2 * y1 - dot1 * y2) / Det);
            if (dot1 <= 0.0) {
                idx_in_out = i1;
                sec_in_out = sec;
            } else {
                idx_out_in = i1;
                sec_out_in = sec;
            }
        }
        dot1 = dot2;
    }
    if (idx_in_out < 0 || idx_out_in < 0) {
        r.area = dot1 < 0.0 ? area(P) : 0.0;
        return r;
    }
    if (slice) {
        r.p1 = sec_in_out;
        r.p2 = sec_out_in;
        r.tri_in = (idx_in_out - idx_out_in + size) % size == 1;
        r.tri_out = (idx_out_in - idx_in_out + size) % size == 1;
    }
    const int k1 = idx_out_in + 1 == size ? 0 : idx_out_in + 1;
    double a = 0.0;
    a += cross_c(P.cx, P.cy, sec_out_in.x, sec_out_in.y, P.x[k1], P.y[k1]);
    a += cross_c(P.cx, P.cy, P.x[idx_in_out], P.y[idx_in_out], sec_in_out.x, sec_in_out.y);
    a += cross_c(P.cx, P.cy, sec_in_out.x, sec_in_out.y, sec_out_in.x, sec_out_in.y);
    int end = idx_in_out < idx_out_in ? idx_in_out + size : idx_in_out;
    for (int i = idx_out_in + 1; i < end; ++i) {
        const int ia = i % size, ib = (i + 1) % size;
        a += cross_c(P.cx, P.cy, P.x[ia], P.y[ia], P.x[ib], P.y[ib]);
    }
    r.area = a * 0.5;
    return r;
}

// ---------------------------------------------------------------------------
// Polygon operations on the cell's own rectangle (x0, x1) x (y0, y1),
// vertices v0 = (x0, y0), v1 = (x1, y0), v2 = (x1, y1), v3 = (x0, y1) in
// AmrCells::polygon order (vs<-1,-1>, vs<+1,-1>, vs<+1,+1>, vs<-1,+1>,
// amr_cells.cpp:157-180): every vertex index is static or selected, so the
// polygon stays in registers.  The operations and their order are those of
// clip_area_and_slice above and of Polygon::find_section (polygon.cpp:555-574)
// with find_section_newton (polygon.cpp:487-553).
struct Rect {
    double x0, x1, y0, y1, cx, cy;
    __device__ __forceinline__ double vx(int k) const { return (k == 1 || k == 2) ? x1 : x0; }
    __device__ __forceinline__ double vy(int k) const { return k >= 2 ? y1 : y0; }
};

__device__ __forceinline__ Rect make_rect(const TrMesh &m, int i, int j) {
    Rect r;
    r.x0 = m.X[i];
    r.x1 = m.X[i + 1];
    r.y0 = m.Y[j];
    r.y1 = m.Y[j + 1];
    // m_center: ((0 + v0) + v1 + v2 + v3) / 4
    r.cx = (((0.0 + r.x0) + r.x1) + r.x1 + r.x0) / 4.0;
    r.cy = (((0.0 + r.y0) + r.y0) + r.y1 + r.y1) / 4.0;
    return r;
}

__device__ __forceinline__ double rect_area(const Rect &r) {
    double S = 0.0;
#pragma unroll
    for (int k = 0; k < 4; ++k) S += cross_c(r.cx, r.cy, r.vx(k), r.vy(k), r.vx((k + 1) & 3), r.vy((k + 1) & 3));
    return 0.5 * S;
}

__device__ AnS rect_clip_area_and_slice(const Rect &r, P2 p, P2 n) {
    AnS res;
    res.area = 0.0;
    res.tri_in = res.tri_out = false;
    res.p1 = res.p2 = mk(0.0, 0.0);
    if (bad_normal(n)) {
        // Polygon::inside on the rectangle (unreached from find_section, whose
        // normal is unit)
        const P2 tau = mk(0.123, 0.346433);
        int counter = 0;
#pragma unroll
        for (int k = 0; k < 4; ++k)
            if (exist_ray(p, tau, r.vx(k), r.vy(k), r.vx((k + 1) & 3), r.vy((k + 1) & 3))) ++counter;
        res.p1 = res.p2 = mk(CUDART_NAN, CUDART_NAN);
        res.area = counter % 2 > 0 ? rect_area(r) : 0.0;
        return res;
    }
    double d[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) d[k] = (r.vx(k) - p.x) * n.x + (r.vy(k) - p.y) * n.y;
    int idx_out_in = -1, idx_in_out = -1;
    P2 sec_out_in = mk(0.0, 0.0), sec_in_out = mk(0.0, 0.0);
#pragma unroll
    for (int i2 = 0; i2 < 4; ++i2) {
        const int i1 = (i2 + 3) & 3;
        const double dot1 = d[i1], dot2 = d[i2];
        if (dot1 * dot2 < 0.0) {
            const double x1 = r.vx(i1), y1 = r.vy(i1), x2 = r.vx(i2), y2 = r.vy(i2);
            const double Det = (x2 - x1) * n.x + (y2 - y1) * n.y;
            const P2 sec = mk((dot2 * x1 - dot1 * x2) / Det, (dot2 * y1 - dot1 * y2) / Det);
            if (dot1 <= 0.0) {
                idx_in_out = i1;
                sec_in_out = sec;
            } else {
                idx_out_in = i1;
                sec_out_in = sec;
            }
        }
    }
    if (idx_in_out < 0 || idx_out_in < 0) {
        res.area = d[3] < 0.0 ? rect_area(r) : 0.0;
        return res;
    }
    res.p1 = sec_in_out;
    res.p2 = sec_out_in;
    res.tri_in = ((idx_in_out - idx_out_in + 4) & 3) == 1;
    res.tri_out = ((idx_out_in - idx_in_out + 4) & 3) == 1;
    const int k1 = (idx_out_in + 1) & 3;
    double a = 0.0;
    a += cross_c(r.cx, r.cy, sec_out_in.x, sec_out_in.y, r.vx(k1), r.vy(k1));
    a += cross_c(r.cx, r.cy, r.vx(idx_in_out), r.vy(idx_in_out), sec_in_out.x, sec_in_out.y);
    a += cross_c(r.cx, r.cy, sec_in_out.x, sec_in_out.y, sec_out_in.x, sec_out_in.y);
    const int end = idx_in_out < idx_out_in ? idx_in_out + 4 : idx_in_out;
#pragma unroll
    for (int q = 1; q < 4; ++q) {
        const int i = idx_out_in + q;
        if (i < end) a += cross_c(r.cx, r.cy, r.vx(i & 3), r.vy(i & 3), r.vx((i + 1) & 3), r.vy((i + 1) & 3));
    }
    res.area = a * 0.5;
    return res;
}

__device__ P2 rect_find_section(const Rect &r, P2 n_in, double alpha) {
    const P2 n = normalized(n_in);
    if (bad_normal(n)) return alpha < 0.5 ? mk(CUDART_NAN, CUDART_NAN) : mk(r.cx, r.cy);
    int imin = 0, imax = 0;
    double min_dot = r.vx(0) * n.x + r.vy(0) * n.y, max_dot = min_dot;
#pragma unroll
    for (int k = 1; k < 4; ++k) {
        const double dk = r.vx(k) * n.x + r.vy(k) * n.y;
        if (dk < min_dot) {
            imin = k;
            min_dot = dk;
        } else if (dk > max_dot) {
            imax = k;
            max_dot = dk;
        }
    }
    const P2 vmin = mk(r.vx(imin), r.vy(imin)), vmax = mk(r.vx(imax), r.vy(imax));
    if (alpha < 1.0e-14) return mk(vmin.x - 0.1 * n.x, vmin.y - 0.1 * n.y);
    if (alpha > 1.0 - 1.0e-14) return mk(vmax.x + 0.1 * n.x, vmax.y + 0.1 * n.y);
    const double DV = (vmax.x - vmin.x) * n.x + (vmax.y - vmin.y) * n.y;
    const P2 dv = mk(DV * n.x, DV * n.y);
    const double S = rect_area(r);
    double x = alpha;
    AnS f = rect_clip_area_and_slice(r, mk(vmin.x + x * dv.x, vmin.y + x * dv.y), n);
    double err = fabs(f.area / S - alpha);
    int it = 0;
    while (err > 1.0e-12 && it < 30) {
        const double dx = f.p2.x - f.p1.x, dy = f.p2.y - f.p1.y;
        const double slice = sqrt(dx * dx + dy * dy);
        if (f.tri_in) x = sqrt(2.0 * alpha * x * S / (DV * slice));
        else if (f.tri_out) x = 1.0 - sqrt(2.0 * (1.0 - alpha) * (1.0 - x) * S / (DV * slice));
        else x -= (f.area - alpha * S) / (DV * slice);
        x = dmax(0.0, dmin(x, 1.0));
        f = rect_clip_area_and_slice(r, mk(vmin.x + x * dv.x, vmin.y + x * dv.y), n);
        err = fabs(f.area / S - alpha);
        ++it;
    }
    return mk(0.5 * (f.p1.x + f.p2.x), 0.5 * (f.p1.y + f.p2.y));
}

// The transfer problem's velocity field (problems/transfer.cpp:367-380);
// the rotation is omega x (q - center) with omega = (0, 0, w).
__device__ __forceinline__ P2 velocity(const TrVel &v, double qx, double qy) {
    if (v.kind == 0) return mk(v.vx, v.vy);
    const double rx = qx - v.cx, ry = qy - v.cy;
    return mk(0.0 - v.w * ry, v.w * rx - 0.0);
}

// perpendicular (line.cpp:18-20): the unit normal of tau in the plane of
// tau and a, on a's side: (tau x a) x tau, normalised.
__device__ __forceinline__ P2 perpendicular(P2 tau, P2 a) {
    const double cz = tau.x * a.y - tau.y * a.x;
    return normalized(mk(0.0 - cz * tau.y, cz * tau.x - 0.0));
}

// flux_VOF (transfer.cpp:250-292): the part of the upwind cell (i, j) swept
// through the face (v1, v2, centre fc) in dt by the face's vertex
// velocities W1, W2, times its fraction; fn is the face normal pointing out
// of the upwind cell.
// The flux of an upwind cell with u1 < 1e-8 is 0 when the tangential part
// of the mean face velocity dominates, and 0 * area = 0 when u1 == 0; no
// polygon is clipped then.
__device__ __forceinline__ bool vof_trivial(double u, P2 W1, P2 W2, P2 fn, P2 &Vn) {
    const P2 Vc = mk(0.5 * (W1.x + W2.x), 0.5 * (W1.y + W2.y));
    const double vcn = Vc.x * fn.x + Vc.y * fn.y;
    Vn = mk(vcn * fn.x, vcn * fn.y);
    const P2 Vt = mk(Vc.x - Vn.x, Vc.y - Vn.y);
    return u < 1.0e-8 && (!(Vn.x * Vn.x + Vn.y * Vn.y > Vt.x * Vt.x + Vt.y * Vt.y) || u == 0.0);
}

// POLY false: only for faces whose fluxes clip no polygon (all trivial).
template <bool POLY>
__device__ double flux_vof(const TrArgs &a, int i, int j, P2 v1, P2 v2, P2 fc, P2 W1, P2 W2, P2 fn, double dt) {
    if (!POLY) return 0.0;
    const int ic = i * a.m.ny + j;
    const double u = a.u[ic];
    P2 Vn;
    if (vof_trivial(u, W1, W2, fn, Vn)) return 0.0;
    const double xi = dt * sqrt(Vn.x * Vn.x + Vn.y * Vn.y);
    // the two lines through the face's vertices along the velocities
    const P2 l1b = mk(v1.x - W1.x, v1.y - W1.y), l2b = mk(v2.x - W2.x, v2.y - W2.y);
    const P2 c1 = mk(0.5 * (v1.x + l1b.x), 0.5 * (v1.y + l1b.y));
    const P2 c2 = mk(0.5 * (v2.x + l2b.x), 0.5 * (v2.y + l2b.y));
    const P2 n1 = perpendicular(mk(l1b.x - v1.x, l1b.y - v1.y), mk(v1.x - fc.x, v1.y - fc.y));
    const P2 n2 = perpendicular(mk(l2b.x - v2.x, l2b.y - v2.y), mk(v2.x - fc.x, v2.y - fc.y));

    Poly A, B;
    {
        // AmrCells::polygon of the linear cell (amr_cells.cpp:157-180)
        const double x0 = a.m.X[i], x1 = a.m.X[i + 1], y0 = a.m.Y[j], y1 = a.m.Y[j + 1];
        A.n = 4;
        A.x[0] = x0;
        A.y[0] = y0;
        A.x[1] = x1;
        A.y[1] = y0;
        A.x[2] = x1;
        A.y[2] = y1;
        A.x[3] = x0;
        A.y[3] = y1;
    }
    clip(A, mk(fc.x - xi * fn.x, fc.y - xi * fn.y), mk(-fn.x, -fn.y), B, a.err);
    clip(B, c1, n1, A, a.err);
    clip(A, c2, n2, B, a.err);
    if (u < 1.0e-8) return u * area(B);
    if (u > 1.0 - 1.0e-8) return area(B);
    const int c = a.cur;
    return clip_area_and_slice(B, mk(a.px[c][ic], a.py[c][ic]), mk(a.nx[c][ic], a.ny[c][ic]), false).area;
}

// flux_2D (transfer.cpp:109-122)
__device__ __forceinline__ double flux_2D(double a1, double a2, double S, double V1, double V2, double as, double vn,
                                          double dt) {
    const double aa = vn > 0.0 ? a1 : a2;
    const double V = vn > 0.0 ? V1 : V2;
    const double gamma = dt * fabs(vn) * S;
    const double F_min = dmax(0.0, gamma - (1.0 - aa) * V);
    const double F_max = aa * V;
    return sgn(vn) * between(gamma * as, F_min, F_max);
}

// limiters::vanAlbada2(a, b) (limiter.cxx:92-96)
__device__ __forceinline__ double van_albada2(double a, double b) {
    if (a * b <= 0.0) return 0.0;
    const double eps = 10e-6;
    return (2.0 * a * b + eps) / (a * a + b * b + eps);
}

// best_face_fraction + flux_CRP (transfer.cpp:179-206)
__device__ __forceinline__ double flux_crp(double a1, double a2, double S, double V1, double V2, double vn, double dt,
                                           double Flux) {
    double a_sig;
    if (vn == 0.0) {
        a_sig = 0.5 * (a1 + a2);
    } else {
        double lo, hi;
        sorted2(a1, a2, lo, hi);
        a_sig = between(Flux / (dt * vn * S), lo, hi);
    }
    return flux_2D(a1, a2, S, V1, V2, a_sig, vn, dt);
}

// The face between cells A (left / lower) and B (right / upper): its
// vertices, centre and the normal out of A (the normal out of B is its
// negative, (-1, -0) or (-0, -1) as the reference stores it).
struct Face {
    int iA, jA, iB, jB;
    P2 v1, v2, fc, fn;
    double S;
};

__device__ __forceinline__ Face x_face(const TrMesh &m, int i, int j) {
    Face f;
    f.iA = i - 1;
    f.jA = j;
    f.iB = i;
    f.jB = j;
    f.v1 = mk(m.X[i], m.Y[j]);
    f.v2 = mk(m.X[i], m.Y[j + 1]);
    f.fc = mk(m.X[i], m.fym[j]);
    f.fn = mk(1.0, 0.0);
    f.S = m.hy;
    return f;
}

__device__ __forceinline__ Face y_face(const TrMesh &m, int i, int j) {
    Face f;
    f.iA = i;
    f.jA = j - 1;
    f.iB = i;
    f.jB = j;
    f.v1 = mk(m.X[i], m.Y[j]);
    f.v2 = mk(m.X[i + 1], m.Y[j]);
    f.fc = mk(m.fxm[i], m.Y[j]);
    f.fn = mk(0.0, 1.0);
    f.S = m.hx;
    return f;
}

// The vertex velocities of the face (projected on its normal under direction
// splitting) and the normal velocity seen from A (transfer.cpp:300-313).
__device__ __forceinline__ double face_velocities(const TrArgs &a, const Face &f, int dir, P2 &U1, P2 &U2, double &sx,
                                                  double &sy) {
    const P2 W1 = velocity(a.vel, f.v1.x, f.v1.y), W2 = velocity(a.vel, f.v2.x, f.v2.y);
    sx = W1.x + W2.x;
    sy = W1.y + W2.y;
    U1 = W1;
    U2 = W2;
    if (dir != 0) {
        const double d1 = W1.x * f.fn.x + W1.y * f.fn.y, d2 = W2.x * f.fn.x + W2.y * f.fn.y;
        U1 = mk(d1 * f.fn.x, d1 * f.fn.y);
        U2 = mk(d2 * f.fn.x, d2 * f.fn.y);
    }
    return 0.5 * (sx * f.fn.x + sy * f.fn.y);
}

// Whether the face's VOF flux clips a polygon (else face_vof takes only the
// trivial branches of flux_vof).
__device__ bool face_needs_polygon(const TrArgs &a, const Face &f, int dir) {
    P2 U1, U2, Vn;
    double sx, sy;
    const double vn = face_velocities(a, f, dir, U1, U2, sx, sy);
    const P2 fnB = mk(-f.fn.x, -f.fn.y);
    const double uA = a.u[f.iA * a.m.ny + f.jA], uB = a.u[f.iB * a.m.ny + f.jB];
    if (vn > 0.0) return !vof_trivial(uA, U1, U2, f.fn, Vn);
    if (vn < 0.0) return !vof_trivial(uB, U1, U2, fnB, Vn);
    return !vof_trivial(uB, U1, U2, fnB, Vn) || !vof_trivial(uA, U1, U2, f.fn, Vn);
}

// Transfer::fluxes_VOF for one face (transfer.cpp:294-340): the flux summed
// by A (fa) and by B (fb).
template <bool POLY>
__device__ void face_vof(const TrArgs &a, const Face &f, int dir, double dt, double &fa, double &fb) {
    const P2 fnB = mk(-f.fn.x, -f.fn.y);
    P2 U1, U2;
    double sx, sy;
    const double vn = face_velocities(a, f, dir, U1, U2, sx, sy);
    const int icA = f.iA * a.m.ny + f.jA, icB = f.iB * a.m.ny + f.jB;
    if (vn > 0.0) {
        fa = flux_vof<POLY>(a, f.iA, f.jA, f.v1, f.v2, f.fc, U1, U2, f.fn, dt);
        fb = -fa;
    } else if (vn < 0.0) {
        fb = flux_vof<POLY>(a, f.iB, f.jB, f.v1, f.v2, f.fc, U1, U2, fnB, dt);
        fa = -fb;
    } else {
        // each cell takes the other as upwind
        fa = -flux_vof<POLY>(a, f.iB, f.jB, f.v1, f.v2, f.fc, U1, U2, fnB, dt);
        fb = -flux_vof<POLY>(a, f.iA, f.jA, f.v1, f.v2, f.fc, U1, U2, f.fn, dt);
    }
    if (a.method == VOF_CRP) {
        const double uA = a.u[icA], uB = a.u[icB];
        fa = flux_crp(uA, uB, f.S, a.m.vol, a.m.vol, vn, dt, fa);
        if (vn != 0.0) {
            fb = -fa;
        } else {
            const double vnB = 0.5 * (sx * fnB.x + sy * fnB.y);
            fb = flux_crp(uB, uA, f.S, a.m.vol, a.m.vol, vnB, dt, fb);
        }
    }
}

// face_fraction_n2 (transfer.cpp:139-176) seen from cell c (neighbour d),
// with the neighbour plane's offset p.p as the reference writes it.
__device__ double fraction_n2(const TrArgs &a, int ic, int id, P2 v1, P2 v2, double vn) {
    const int c = a.cur;
    const P2 pc = mk(a.px[c][ic], a.py[c][ic]), nc = mk(a.nx[c][ic], a.ny[c][ic]);
    const P2 pd = mk(a.px[c][id], a.py[c][id]), nd = mk(a.nx[c][id], a.ny[c][id]);
    const double pp = vn > 0.0 ? pc.x * nc.x + pc.y * nc.y : pd.x * pd.x + pd.y * pd.y;
    const P2 pn = vn > 0.0 ? nc : nd;
    const bool in1 = v1.x * pn.x + v1.y * pn.y < pp, in2 = v2.x * pn.x + v2.y * pn.y < pp;
    double a_sig;
    if (in1 && in2) {
        a_sig = 1.0;
    } else if (!in1 && !in2) {
        a_sig = 0.0;
    } else {
        const P2 tau = mk(v2.x - v1.x, v2.y - v1.y);
        const double t = (pp - (pn.x * v2.x + pn.y * v2.y)) / (pn.x * tau.x + pn.y * tau.y);
        const P2 in = mk(v2.x + tau.x * t, v2.y + tau.y * t);
        const double len = sqrt(tau.x * tau.x + tau.y * tau.y);
        const P2 d = in1 ? mk(in.x - v1.x, in.y - v1.y) : mk(in.x - v2.x, in.y - v2.y);
        a_sig = sqrt(d.x * d.x + d.y * d.y) / len;
    }
    double lo, hi;
    sorted2(a.u[ic], a.u[id], lo, hi);
    return between(a_sig, lo, hi);
}

// Transfer::fluxes_CRP for one face seen from cell c (transfer.cpp:208-248);
// fn is the normal out of c.
__device__ double face_crp_side(const TrArgs &a, int ic, int id, P2 v1, P2 v2, P2 fc, P2 fn, double S, double dt) {
    const double a1 = a.u[ic], a2 = a.u[id];
    const P2 V = velocity(a.vel, fc.x, fc.y);
    const double vn = V.x * fn.x + V.y * fn.y;
    double a_sig;
    switch (a.method) {
        case CRP_V3: a_sig = face_fraction_v3(a1, a2); break;
        case CRP_V5: a_sig = face_fraction_v5(a1, a2); break;
        case CRP_N1: {  // face_fraction_n1 (transfer.cpp:127-137)
            const int c = a.cur;
            const double aa = vn > 0.0 ? a1 : a2;
            const double cs = vn > 0.0 ? a.nx[c][ic] * fn.x + a.ny[c][ic] * fn.y
                                       : -(a.nx[c][id] * fn.x + a.ny[c][id] * fn.y);
            const double C = dt * fabs(vn) * S / a.m.vol;
            a_sig = between(average_flux(aa, cs, C), a1, a2);
            break;
        }
        case CRP_N2: a_sig = fraction_n2(a, ic, id, v1, v2, vn); break;
        default: a_sig = face_fraction_s(a1, a2); break;
    }
    return flux_2D(a1, a2, S, a.m.vol, a.m.vol, a_sig, vn, dt);
}

// Transfer::fluxes_MUSCL for one face seen from cell c (i, j) with neighbour
// d (di, dj) (transfer.cpp:345-402); fn is the normal out of c.  The face
// value is FaceExtra::Direct for MUSCL_MC (face_extra.h:121-171, limited to
// the two cells' values) and FaceExtra::ATvL otherwise (face_extra.h:
// 264-350, van Albada 2); the CRP forms then pass the flux through
// flux_CRP.  The two cells' views of a face are not exact negatives (the
// ATvL value is formed from each side's geometry), so each is evaluated.
__device__ double face_muscl_side(const TrArgs &a, int ci, int cj, int di, int dj, P2 fc, P2 fn, double S,
                                  double dt) {
    const int ic = ci * a.m.ny + cj, id = di * a.m.ny + dj;
    const P2 V = velocity(a.vel, fc.x, fc.y);
    const double vn = V.x * fn.x + V.y * fn.y;
    const double uc = a.u[ic], un = a.u[id];
    const double ccx = a.m.cx[ci], ccy = a.m.cy[cj], ncx = a.m.cx[di], ncy = a.m.cy[dj];
    double a_sig;
    if (a.method == MUSCL_MC || a.method == MUSCL_MC_CRP) {
        const double duc = a.gx[ic] * (fc.x - ccx) + a.gy[ic] * (fc.y - ccy) + 0.0 * 0.0;
        const double dun = a.gx[id] * (fc.x - ncx) + a.gy[id] * (fc.y - ncy) + 0.0 * 0.0;
        a_sig = vn > 0.0 ? uc + duc : un + dun;
        a_sig = between(a_sig, uc, un);
    } else {
        const double rcx = fc.x - ccx, rcy = fc.y - ccy, rnx = ncx - fc.x, rny = ncy - fc.y;
        const double dx_c = sqrt(rcx * rcx + rcy * rcy), dx_n = sqrt(rnx * rnx + rny * rny);
        const double dx = dx_c + dx_n;
        if (vn > 0.0) {  // m(u_c)
            const double du_c = (a.gx[ic] * rcx + a.gy[ic] * rcy + 0.0 * 0.0) / dx_c;
            const double delta = dx_c / dx;
            const double eta = (12.0 * delta * delta - 1.0) / 24.0;
            const double dzp = un - uc;
            const double dzm = 2.0 * du_c * dx - dzp;
            const double s = van_albada2(dzm, dzp);
            a_sig = uc + s * ((0.5 * delta - s * eta) * dzm + (0.5 * delta + s * eta) * dzp);
        } else {  // p(u_n)
            const double du_n = (a.gx[id] * rnx + a.gy[id] * rny + 0.0 * 0.0) / dx_n;
            const double delta = dx_n / dx;
            const double eta = (12.0 * delta * delta - 1.0) / 24.0;
            const double dzm = un - uc;
            const double dzp = 2.0 * du_n * dx - dzm;
            const double s = van_albada2(dzm, dzp);
            a_sig = un - s * ((0.5 * delta + s * eta) * dzm + (0.5 * delta - s * eta) * dzp);
        }
    }
    double Flux = a_sig * vn * dt * S;
    if (a.method == MUSCLd_CRP || a.method == MUSCLn_CRP || a.method == MUSCL_MC_CRP)
        Flux = flux_crp(uc, un, S, a.m.vol, a.m.vol, vn, dt, Flux);
    return Flux;
}

template <bool POLY>
__device__ __forceinline__ void face_fluxes(const TrArgs &a, const Face &f, int dir, double &fa, double &fb) {
    const double dt = *a.dt;
    if (vof_type(a.method)) {
        face_vof<POLY>(a, f, dir, dt, fa, fb);
    } else if (muscl_type(a.method)) {
        fa = face_muscl_side(a, f.iA, f.jA, f.iB, f.jB, f.fc, f.fn, f.S, dt);
        fb = face_muscl_side(a, f.iB, f.jB, f.iA, f.jA, f.fc, mk(-f.fn.x, -f.fn.y), f.S, dt);
    } else {
        const int icA = f.iA * a.m.ny + f.jA, icB = f.iB * a.m.ny + f.jB;
        fa = face_crp_side(a, icA, icB, f.v1, f.v2, f.fc, f.fn, f.S, dt);
        fb = face_crp_side(a, icB, icA, f.v1, f.v2, f.fc, mk(-f.fn.x, -f.fn.y), f.S, dt);
    }
}

// Faces of one update: the interior x faces (i = 1..nx-1) unless dir is Y,
// then the interior y faces (j = 1..ny-1) unless dir is X.
__device__ __forceinline__ long long n_x_faces(const TrMesh &m, int dir) {
    return dir != 2 ? (long long)(m.nx - 1) * m.ny : 0;
}
__device__ __forceinline__ long long n_faces(const TrMesh &m, int dir) {
    return n_x_faces(m, dir) + (dir != 1 ? (long long)m.nx * (m.ny - 1) : 0);
}
__device__ __forceinline__ Face face_at(const TrMesh &m, int dir, long long t, bool &is_x, size_t &slot) {
    const long long tx = n_x_faces(m, dir);
    if (t < tx) {
        const int i = 1 + (int)(t / m.ny), j = (int)(t - (long long)(i - 1) * m.ny);
        is_x = true;
        slot = (size_t)i * m.ny + j;
        return x_face(m, i, j);
    }
    t -= tx;
    const int nyi = m.ny - 1;
    const int i = (int)(t / nyi), j = 1 + (int)(t - (long long)i * nyi);
    is_x = false;
    slot = (size_t)i * (m.ny + 1) + j;
    return y_face(m, i, j);
}
__device__ __forceinline__ void store_face(const TrArgs &a, bool is_x, size_t slot, double fa, double fb) {
    if (is_x) {
        a.fxa[slot] = fa;
        a.fxb[slot] = fb;
    } else {
        a.fya[slot] = fa;
        a.fyb[slot] = fb;
    }
}

// Append `value` to a work list for the lanes that want it (all 32 lanes of
// the warp take part).
__device__ __forceinline__ void append(int *count, int *list, bool want, int value) {
    const unsigned mask = __ballot_sync(0xffffffffu, want);
    if (!mask) return;
    const int lane = threadIdx.x & 31, leader = __ffs(mask) - 1;
    int base = 0;
    if (lane == leader) base = atomicAdd(count, __popc(mask));
    base = __shfl_sync(0xffffffffu, base, leader);
    if (want) list[base + __popc(mask & ((1u << lane) - 1u))] = value;
}

// Every face of the update: CRP fluxes directly; VOF fluxes directly where
// they clip no polygon, the rest onto the face work list.
__global__ void __launch_bounds__(BLOCK) k_flux_classify(TrArgs a, int dir) {
    const long long t = (long long)blockIdx.x * BLOCK + threadIdx.x;
    const bool live = t < n_faces(a.m, dir);
    bool is_x = false, defer = false;
    size_t slot = 0;
    Face f;
    if (live) {
        f = face_at(a.m, dir, t, is_x, slot);
        defer = vof_type(a.method) && face_needs_polygon(a, f, dir);
        // plain VOF: a face that clips no polygon carries +-0, which the
        // update skips (k_update); nothing to store
        if (!defer && a.method != VOF) {
            double fa, fb;
            face_fluxes<false>(a, f, dir, fa, fb);
            store_face(a, is_x, slot, fa, fb);
        }
    }
    append(a.count + 0, a.flist, defer, (int)t);
}

// The deferred VOF faces.
__global__ void __launch_bounds__(BLOCK, 4) k_flux_list(TrArgs a, int dir) {
    const int cnt = a.count[0];
    for (int k = blockIdx.x * BLOCK + threadIdx.x; k < cnt; k += gridDim.x * BLOCK) {
        bool is_x;
        size_t slot;
        const Face f = face_at(a.m, dir, a.flist[k], is_x, slot);
        double fa, fb;
        face_fluxes<true>(a, f, dir, fa, fb);
        store_face(a, is_x, slot, fa, fb);
    }
}

// u1 <- between(u1 - sum of fluxes / volume, 0, 1), faces in slot order
// L, R, B, T (update_VOF / update_CRP, transfer.cpp:487-511)
// For plain VOF a face that clips no polygon carries +-0: adding it changes
// no sum except the sign of an exact zero, which u1 - 0 / V does not show,
// so such faces are skipped (and k_flux_classify stores nothing for them).
// The new u1 goes to the other buffer: the predicate reads the neighbours'
// old u1.
__device__ __forceinline__ bool carries_flux(const TrArgs &a, const Face &f, int dir) {
    return a.method != VOF || face_needs_polygon(a, f, dir);
}

__global__ void __launch_bounds__(BLOCK) k_update(TrArgs a, int dir) {
    const int nx = a.m.nx, ny = a.m.ny;
    const int ic = blockIdx.x * BLOCK + threadIdx.x;
    if (ic >= nx * ny) return;
    const int i = ic / ny, j = ic - i * ny;
    double fl = 0.0;
    if (dir != 2) {
        if (i > 0 && carries_flux(a, x_face(a.m, i, j), dir)) fl += a.fxb[(size_t)i * ny + j];
        if (i < nx - 1 && carries_flux(a, x_face(a.m, i + 1, j), dir)) fl += a.fxa[(size_t)(i + 1) * ny + j];
    }
    if (dir != 1) {
        if (j > 0 && carries_flux(a, y_face(a.m, i, j), dir)) fl += a.fyb[(size_t)i * (ny + 1) + j];
        if (j < ny - 1 && carries_flux(a, y_face(a.m, i, j + 1), dir)) fl += a.fya[(size_t)i * (ny + 1) + j + 1];
    }
    const double u2 = a.u[ic] - fl / a.m.vol;
    a.u_next[ic] = dmax(0.0, dmin(u2, 1.0));
}

// compute_normal (interface_recovery.cpp:18-38) for every cell.  Cells
// with a zero normal get their section (the centre, :46-53) in both
// buffers and keep it through the smoothing passes; the others go onto the
// cell work list.
__global__ void __launch_bounds__(BLOCK) k_normals(TrArgs a) {
    const int nx = a.m.nx, ny = a.m.ny;
    const int ic = blockIdx.x * BLOCK + threadIdx.x;
    bool listed = false;
    if (ic < nx * ny) {
        const int i = ic / ny, j = ic - i * ny;
        const double uc = a.u[ic];
        P2 n = mk(0.0, 0.0);
        if (!(uc < 1.0e-12 || uc > 1.0 - 1.0e-12)) {
            // -sum face_fraction * normal * area over the inner faces, slots L, R, B, T
            double ax = 0.0, ay = 0.0;
            if (i > 0) {
                const double ff = face_fraction(uc, a.u[ic - ny]);
                ax = ax - ff * (-1.0 * a.m.hy);
                ay = ay - ff * (-0.0 * a.m.hy);
            }
            if (i < nx - 1) {
                const double ff = face_fraction(uc, a.u[ic + ny]);
                ax = ax - ff * (1.0 * a.m.hy);
                ay = ay - ff * (0.0 * a.m.hy);
            }
            if (j > 0) {
                const double ff = face_fraction(uc, a.u[ic - 1]);
                ax = ax - ff * (-0.0 * a.m.hx);
                ay = ay - ff * (-1.0 * a.m.hx);
            }
            if (j < ny - 1) {
                const double ff = face_fraction(uc, a.u[ic + 1]);
                ax = ax - ff * (0.0 * a.m.hx);
                ay = ay - ff * (1.0 * a.m.hx);
            }
            n = normalized(mk(ax, ay));
        }
        const int c = a.cur;
        if (is_zero(n.x, n.y)) {
            // zero_np[ic] = 1: both buffers already hold this normal and the centre
            if (!(a.zero_np[ic] && n.x == 0.0 && n.y == 0.0 && !signbit(n.x) && !signbit(n.y))) {
                const double px = a.m.cx[i], py = a.m.cy[j];
                for (int b = 0; b < 2; ++b) {
                    a.nx[b][ic] = n.x;
                    a.ny[b][ic] = n.y;
                    a.px[b][ic] = px;
                    a.py[b][ic] = py;
                }
                a.zero_np[ic] = (n.x == 0.0 && n.y == 0.0 && !signbit(n.x) && !signbit(n.y)) ? 1 : 0;
            }
        } else {
            a.nx[c][ic] = n.x;
            a.ny[c][ic] = n.y;
            if (a.zero_np[ic]) a.zero_np[ic] = 0;
            listed = true;
        }
    }
    append(a.count + 1, a.clist, listed, ic);
}

// find_section (interface_recovery.cpp:46-53) for the listed cells.
__global__ void __launch_bounds__(BLOCK) k_sections(TrArgs a) {
    const int cnt = a.count[1], ny = a.m.ny, c = a.cur;
    for (int k = blockIdx.x * BLOCK + threadIdx.x; k < cnt; k += gridDim.x * BLOCK) {
        const int ic = a.clist[k];
        const int i = ic / ny, j = ic - i * ny;
        const P2 p = rect_find_section(make_rect(a.m, i, j), mk(a.nx[c][ic], a.ny[c][ic]), a.u[ic]);
        a.px[c][ic] = p.x;
        a.py[c][ic] = p.y;
    }
}

// adjust_normal (interface_recovery.cpp:61-98) and find_section, from the
// buffers `cur` into the other ones, for the listed cells (the others keep a
// zero normal: adjust_normal leaves it and the section stays the centre).
__device__ void adjust_cell(const TrArgs &a, int ic) {
    const int nx = a.m.nx, ny = a.m.ny;
    const int i = ic / ny, j = ic - i * ny;
    const int c = a.cur, o = 1 - c;
    const double uc = a.u[ic];
    const P2 pn = mk(a.nx[c][ic], a.ny[c][ic]);
    P2 n = pn;
    if (!is_zero(pn.x, pn.y)) {
        const P2 pc = mk(a.px[c][ic], a.py[c][ic]);
        const double pp = pc.x * pn.x + pc.y * pn.y;
        const P2 r0 = mk(pp * pn.x, pp * pn.y);
        P2 q0 = mk(0.0, 0.0), q1 = mk(0.0, 0.0);  // the first two section points
        int cnt = 0;
        for (int s = 0; s < 4; ++s) {
            // face vertices (face_nodes2d, indexing.h:279-284) and the neighbour
            // (the cell itself across a boundary face)
            P2 v1, v2;
            int nb;
            if (s == 0) {
                v1 = mk(a.m.X[i], a.m.Y[j]);
                v2 = mk(a.m.X[i], a.m.Y[j + 1]);
                nb = i > 0 ? ic - ny : ic;
            } else if (s == 1) {
                v1 = mk(a.m.X[i + 1], a.m.Y[j]);
                v2 = mk(a.m.X[i + 1], a.m.Y[j + 1]);
                nb = i < nx - 1 ? ic + ny : ic;
            } else if (s == 2) {
                v1 = mk(a.m.X[i], a.m.Y[j]);
                v2 = mk(a.m.X[i + 1], a.m.Y[j]);
                nb = j > 0 ? ic - 1 : ic;
            } else {
                v1 = mk(a.m.X[i], a.m.Y[j + 1]);
                v2 = mk(a.m.X[i + 1], a.m.Y[j + 1]);
                nb = j < ny - 1 ? ic + 1 : ic;
            }
            // intersection2D::exist(plane, segment)
            const double d1 = pn.x * (v1.x - r0.x) + pn.y * (v1.y - r0.y);
            const double d2 = pn.x * (v2.x - r0.x) + pn.y * (v2.y - r0.y);
            if (!(d1 * d2 <= 0.0)) continue;
            const P2 tau = mk(v2.x - v1.x, v2.y - v1.y);
            P2 q;
            if (is_zero(a.nx[c][nb], a.ny[c][nb])) {
                const double t = (pn.x * tau.x + pn.y * tau.y) * (a.u[nb] - 0.5) > 0.0 ? 1.001 : -0.001;
                q = mk(v1.x + tau.x * t, v1.y + tau.y * t);
            } else {
                // find_fast(seg, {r0, p_nb}) (intersection.cpp:45-57)
                const P2 pb = mk(a.px[c][nb], a.py[c][nb]);
                const P2 l2t = mk(pb.x - r0.x, pb.y - r0.y);
                const double det = cross2(tau, l2t);
                const double t = cross2(mk(pb.x - v1.x, pb.y - v1.y), l2t) / det;
                q = mk(v1.x + tau.x * t, v1.y + tau.y * t);
            }
            if (cnt == 0) q0 = q;
            else if (cnt == 1) q1 = q;
            ++cnt;
        }
        if (cnt > 1) {
            P2 nn = mk(q0.y - q1.y, q1.x - q0.x);
            if (nn.x * pn.x + nn.y * pn.y < 0.0) nn = mk(nn.x * -1.0, nn.y * -1.0);
            n = normalized(nn);
        }
    }
    P2 p;
    if (is_zero(n.x, n.y)) p = mk(a.m.cx[i], a.m.cy[j]);
    else p = rect_find_section(make_rect(a.m, i, j), n, uc);
    a.nx[o][ic] = n.x;
    a.ny[o][ic] = n.y;
    a.px[o][ic] = p.x;
    a.py[o][ic] = p.y;
}

__global__ void __launch_bounds__(BLOCK) k_adjust(TrArgs a) {
    const int cnt = a.count[1];
    for (int k = blockIdx.x * BLOCK + threadIdx.x; k < cnt; k += gridDim.x * BLOCK) adjust_cell(a, a.clist[k]);
}

// Transfer::compute_dt (transfer.cpp:88-105): CFL * min over cells of
// volume / max face area / |v(centre)|; the last block finishes the step.
__global__ void __launch_bounds__(BLOCK) k_dt(TrArgs a, int advance, double t_end) {
    const int nx = a.m.nx, ny = a.m.ny, n = nx * ny;
    __shared__ double red[BLOCK];
    __shared__ bool last;
    double tau = DBL_MAX;
    const double max_area = dmax(dmax(dmax(dmax(0.0, a.m.hy), a.m.hy), a.m.hx), a.m.hx);
    const double dx = a.m.vol / max_area;
    for (int ic = blockIdx.x * BLOCK + threadIdx.x; ic < n; ic += gridDim.x * BLOCK) {
        const int i = ic / ny, j = ic - i * ny;
        const P2 V = velocity(a.vel, a.m.cx[i], a.m.cy[j]);
        tau = dmin(tau, dx / sqrt(V.x * V.x + V.y * V.y));
    }
    red[threadIdx.x] = tau;
    __syncthreads();
    for (int s = BLOCK / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] = dmin(red[threadIdx.x], red[threadIdx.x + s]);
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        // min over non-negative doubles (NaN never wins, as std::min keeps tau)
        const double b = red[0];
        if (b == b) atomicMin(a.dmin, (unsigned long long)__double_as_longlong(b));
        __threadfence();
        last = atomicAdd(a.ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (last && threadIdx.x == 0) {
        __threadfence();
        const double m = __longlong_as_double((long long)atomicAdd(a.dmin, 0ull));
        double dt = a.CFL * m;
        if (advance) {
            const double t = *a.time;
            if (t + dt > t_end) dt = t_end - t;
            *a.time = t + dt;
        }
        *a.dt = dt;
        *a.dmin = (unsigned long long)__double_as_longlong(DBL_MAX);
        *a.ticket = 0u;
    }
}

// Transfer::set_flags (transfer.cpp:660-680)
__global__ void __launch_bounds__(BLOCK) k_flags(TrArgs a, int *flags) {
    const int nx = a.m.nx, ny = a.m.ny;
    const int ic = blockIdx.x * BLOCK + threadIdx.x;
    if (ic >= nx * ny) return;
    const int i = ic / ny, j = ic - i * ny;
    double lo = a.u[ic], hi = lo;
    if (i > 0) lo = dmin(lo, a.u[ic - ny]), hi = dmax(hi, a.u[ic - ny]);
    if (i < nx - 1) lo = dmin(lo, a.u[ic + ny]), hi = dmax(hi, a.u[ic + ny]);
    if (j > 0) lo = dmin(lo, a.u[ic - 1]), hi = dmax(hi, a.u[ic - 1]);
    if (j < ny - 1) lo = dmin(lo, a.u[ic + 1]), hi = dmax(hi, a.u[ic + 1]);
    flags[ic] = hi - lo > 0.0 ? 1 : -1;
}

inline unsigned blocks(long long n) { return (unsigned)((n + BLOCK - 1) / BLOCK); }

// Transfer::compute_slopes (transfer.cpp:404-469), one thread per cell,
// faces in slot order L, R, B, T with the reference's normals (signed zeros
// included).  MUSCLn, MUSCLn_CRP: the part of each face under the cell's
// interface plane, sum a_sig S n / V.  The others: gradient::LSM of u1
// (gradient.h:226-282; boundary faces take the cell's own value at the
// mirrored centre), limited (gradient.h:412-474) for MUSCL_MC, with the
// 2-D reduction of the 3x3 system that the single-material kernels use.
__global__ void __launch_bounds__(BLOCK) k_slopes(TrArgs a) {
    const int nx = a.m.nx, ny = a.m.ny;
    const int ic = blockIdx.x * BLOCK + threadIdx.x;
    if (ic >= nx * ny) return;
    const int i = ic / ny, j = ic - i * ny;
    const double fnx[4] = {-1.0, 1.0, -0.0, 0.0}, fny[4] = {-0.0, 0.0, -1.0, 1.0};
    const double S[4] = {a.m.hy, a.m.hy, a.m.hx, a.m.hx};
    if (a.method == MUSCLn || a.method == MUSCLn_CRP) {
        const int c = a.cur;
        const double pnx = a.nx[c][ic], pny = a.ny[c][ic];
        const double pp = a.px[c][ic] * pnx + a.py[c][ic] * pny;
        // face vertices (face_nodes2d): L, R from bottom to top; B, T from left to right
        const double xl = a.m.X[i], xr = a.m.X[i + 1], yb = a.m.Y[j], yt = a.m.Y[j + 1];
        const P2 vs1[4] = {mk(xl, yb), mk(xr, yb), mk(xl, yb), mk(xl, yt)};
        const P2 vs2[4] = {mk(xl, yt), mk(xr, yt), mk(xr, yb), mk(xr, yt)};
        double gx = 0.0, gy = 0.0;
#pragma unroll
        for (int s = 0; s < 4; ++s) {
            const P2 v1 = vs1[s], v2 = vs2[s];
            const bool in1 = v1.x * pnx + v1.y * pny < pp, in2 = v2.x * pnx + v2.y * pny < pp;
            double a_sig;
            if (in1 && in2) {
                a_sig = 1.0;
            } else if (!in1 && !in2) {
                a_sig = 0.0;
            } else {
                // find_fast(plane, seg): line {v2, v2 - v1} (intersection.cpp:63-70)
                const double tx = v2.x - v1.x, ty = v2.y - v1.y;
                const double t = (pp - (pnx * v2.x + pny * v2.y)) / (pnx * tx + pny * ty);
                const double qx = v2.x + t * tx, qy = v2.y + t * ty;
                const double len = sqrt(tx * tx + ty * ty);
                a_sig = in1 ? sqrt((qx - v1.x) * (qx - v1.x) + (qy - v1.y) * (qy - v1.y)) / len
                            : sqrt((qx - v2.x) * (qx - v2.x) + (qy - v2.y) * (qy - v2.y)) / len;
            }
            gx += a_sig * S[s] * fnx[s];
            gy += a_sig * S[s] * fny[s];
        }
        a.gx[ic] = gx / a.m.vol;
        a.gy[ic] = gy / a.m.vol;
        return;
    }
    const double uc = a.u[ic], pcx = a.m.cx[i], pcy = a.m.cy[j];
    double wv[4], drx[4], dry[4], drnx[4], drny[4], dn[4];
    double A00 = 0.0, A01 = 0.0, A10 = 0.0, A11 = 0.0, Fx = 0.0, Fy = 0.0;
#pragma unroll
    for (int s = 0; s < 4; ++s) {
        const bool bnd = (s == 0 && i == 0) || (s == 1 && i == nx - 1) || (s == 2 && j == 0) || (s == 3 && j == ny - 1);
        const int nb = s == 0 ? ic - ny : s == 1 ? ic + ny : s == 2 ? ic - 1 : ic + 1;
        double ncx, ncy;
        if (!bnd) {
            ncx = s < 2 ? a.m.cx[s == 0 ? i - 1 : i + 1] : pcx;
            ncy = s < 2 ? pcy : a.m.cy[s == 2 ? j - 1 : j + 1];
        } else {  // symm_point (amr_faces.h:197-199)
            const double fcx = s < 2 ? a.m.X[s == 0 ? i : i + 1] : a.m.fxm[i];
            const double fcy = s < 2 ? a.m.fym[j] : a.m.Y[s == 2 ? j : j + 1];
            const double d2 = 2.0 * ((fcx - pcx) * fnx[s] + (fcy - pcy) * fny[s]);
            ncx = pcx + d2 * fnx[s];
            ncy = pcy + d2 * fny[s];
        }
        const double un = bnd ? uc : a.u[nb];
        const double rx = ncx - pcx, ry = ncy - pcy;
        const double d = rx * fnx[s] + ry * fny[s];
        const double nxx = d * fnx[s], nyy = d * fny[s];
        const double w = 1.0 * S[s] / cube_rn(sqrt(nxx * nxx + nyy * nyy));
        const double wdx = w * nxx, wdy = w * nyy;
        A00 += wdx * rx;
        A01 += wdx * ry;
        A10 += wdy * rx;
        A11 += wdy * ry;
        const double dF = un - uc;
        Fx += w * dF * nxx;
        Fy += w * dF * nyy;
        wv[s] = w;
        drx[s] = rx;
        dry[s] = ry;
        drnx[s] = nxx;
        drny[s] = nyy;
        dn[s] = dF;
    }
    if (fabs(A11) < 1e-8) A11 = 1.0;
    const double det = A11 * A00 + (-A01) * A10;
    const double inv = 1.0 / det;
    const double B00 = A11 * inv, B01 = (-A01) * inv, B10 = (-A10) * inv, B11 = A00 * inv;
    const double g0x = B00 * Fx + B01 * Fy, g0y = B10 * Fx + B11 * Fy;
    if (a.method != MUSCL_MC && a.method != MUSCL_MC_CRP) {
        a.gx[ic] = g0x;
        a.gy[ic] = g0y;
        return;
    }
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
    a.gx[ic] = B00 * lx + B01 * ly;
    a.gy[ic] = B10 * lx + B11 * ly;
}

// WENO5 (math/calc/weno.h:113-169) on the five values q[0..4] centred on
// q[2]: the value at the centre cell's right face (p) or left face (m)
__device__ __forceinline__ double weno_beta(int kind, const double *q) {  // weno.h:88-107
    const double d2 = q[0] - 2.0 * q[1] + q[2];
    const double d1 = kind == 2 ? q[0] - 4.0 * q[1] + 3.0 * q[2] : (kind == 1 ? q[0] - q[2] : 3.0 * q[0] - 4.0 * q[1] + q[2]);
    return 13.0 / 12.0 * d2 * d2 + 1.0 / 4.0 * d1 * d1;
}
__device__ double weno5(const double u[5], bool right) {
    const double *s2 = u, *s1 = u + 1, *s0 = u + 2;
    const double b0 = weno_beta(0, s0), b1 = weno_beta(1, s1), b2 = weno_beta(2, s2);
    double d0_c, d1_c, d2_c, e0, e1, e2;
    if (right) {
        d0_c = 3.0 / 10.0, d1_c = 6.0 / 10.0, d2_c = 1.0 / 10.0;
        e0 = +1.0 / 3.0 * s0[0] + +5.0 / 6.0 * s0[1] + -1.0 / 6.0 * s0[2];
        e1 = -1.0 / 6.0 * s1[0] + +5.0 / 6.0 * s1[1] + +1.0 / 3.0 * s1[2];
        e2 = +1.0 / 3.0 * s2[0] + -7.0 / 6.0 * s2[1] + 11.0 / 6.0 * s2[2];
    } else {
        d0_c = 1.0 / 10.0, d1_c = 6.0 / 10.0, d2_c = 3.0 / 10.0;
        e0 = 11.0 / 6.0 * s0[0] + -7.0 / 6.0 * s0[1] + +1.0 / 3.0 * s0[2];
        e1 = +1.0 / 3.0 * s1[0] + +5.0 / 6.0 * s1[1] + -1.0 / 6.0 * s1[2];
        e2 = -1.0 / 6.0 * s2[0] + +5.0 / 6.0 * s2[1] + +1.0 / 3.0 * s2[2];
    }
    const double d0 = d0_c / ((1.0e-8 + b0) * (1.0e-8 + b0));
    const double d1 = d1_c / ((1.0e-8 + b1) * (1.0e-8 + b1));
    const double d2 = d2_c / ((1.0e-8 + b2) * (1.0e-8 + b2));
    const double w0 = d0 / (d0 + d1 + d2);
    const double w1 = d1 / (d0 + d1 + d2);
    const double w2 = d2 / (d0 + d1 + d2);
    return w0 * e0 + w1 * e1 + w2 * e2;
}

// Transfer::update_WENO's face loop and update (transfer.cpp:541-666), one
// thread per cell: every face of the direction, boundary faces included
// (their neighbour is the cell itself), each with the five-cell stencil of
// its upwind cell taken through EuMesh::operator()(i, j)'s periodic index
// wrap (eu_mesh.cpp:826-830); faces in slot order L, R, B, T, then
// u_next = between(u1 - sum / V, 0, 1).
__global__ void __launch_bounds__(BLOCK) k_weno(TrArgs a, int dir) {
    const int nx = a.m.nx, ny = a.m.ny;
    const int ic = blockIdx.x * BLOCK + threadIdx.x;
    if (ic >= nx * ny) return;
    const int i = ic / ny, j = ic - i * ny;
    const double dt = *a.dt;
    const double fnx[4] = {-1.0, 1.0, -0.0, 0.0}, fny[4] = {-0.0, 0.0, -1.0, 1.0};
    double fluxes = 0.0;
#pragma unroll 1
    for (int s = 0; s < 4; ++s) {
        if ((s < 2 && dir == 2) || (s >= 2 && dir == 1)) continue;
        const P2 fc = s < 2 ? mk(a.m.X[s == 0 ? i : i + 1], a.m.fym[j]) : mk(a.m.fxm[i], a.m.Y[s == 2 ? j : j + 1]);
        const double S = s < 2 ? a.m.hy : a.m.hx;
        const bool bnd = (s == 0 && i == 0) || (s == 1 && i == nx - 1) || (s == 2 && j == 0) || (s == 3 && j == ny - 1);
        const int nb = bnd ? ic : (s == 0 ? ic - ny : s == 1 ? ic + ny : s == 2 ? ic - 1 : ic + 1);
        const P2 V = velocity(a.vel, fc.x, fc.y);
        const double vn = V.x * fnx[s] + V.y * fny[s];
        const bool low = s == 0 || s == 2;
        const int K = (s < 2 ? i : j) + (vn > 0.0 ? 0 : (low ? -1 : 1));
        double st[5];
#pragma unroll
        for (int k = 0; k < 5; ++k) {
            const int q = K - 2 + k;
            st[k] = s < 2 ? a.u[(size_t)ny * ((q + nx) % nx) + j] : a.u[(size_t)ny * i + (q + ny) % ny];
        }
        const double a_sig = between(weno5(st, vn > 0.0 ? !low : low), 0.0, 1.0);
        double Flux = a_sig * vn * dt * S;
        if (a.method == WENO_CRP) Flux = flux_crp(a.u[ic], a.u[nb], S, a.m.vol, a.m.vol, vn, dt, Flux);
        fluxes += Flux;
    }
    const double u2 = a.u[ic] - fluxes / a.m.vol;
    a.u_next[ic] = dmax(0.0, dmin(u2, 1.0));
}

}  // namespace

void launch_weno(const TrArgs &a, int dir, cudaStream_t st) {
    const int n = a.m.nx * a.m.ny;
    k_weno<<<(n + BLOCK - 1) / BLOCK, BLOCK, 0, st>>>(a, dir);
}

void launch_compute_dt(const TrArgs &a, bool advance, double t_end, cudaStream_t st) {
    const long long n = (long long)a.m.nx * a.m.ny;
    unsigned g = blocks(n);
    if (g > 148u * 16u) g = 148u * 16u;
    k_dt<<<g, BLOCK, 0, st>>>(a, advance ? 1 : 0, t_end);
}

// Grid of a work-list kernel: the blocks that are resident at once (SMs x
// blocks per SM at the kernel's register use), striding over the list.
template <class K>
unsigned list_blocks(K kernel, long long n) {
    static thread_local const void *keys[4] = {};
    static thread_local unsigned vals[4] = {};
    unsigned resident = 0;
    int slot = 0;
    for (; slot < 4 && keys[slot]; ++slot)
        if (keys[slot] == (const void *)kernel) resident = vals[slot];
    if (!resident) {
        int dev = 0, sms = 148, per_sm = 1;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, BLOCK, 0);
        resident = (unsigned)(sms * (per_sm > 0 ? per_sm : 1));
        if (slot < 4) {
            keys[slot] = (const void *)kernel;
            vals[slot] = resident;
        }
    }
    const unsigned g = blocks(n);
    return g < resident ? (g ? g : 1u) : resident;
}

void launch_slopes(const TrArgs &a, cudaStream_t st) {
    const int n = a.m.nx * a.m.ny;
    k_slopes<<<(n + BLOCK - 1) / BLOCK, BLOCK, 0, st>>>(a);
}

void launch_flux(const TrArgs &a, int dir, cudaStream_t st) {
    const long long nx = a.m.nx, ny = a.m.ny;
    const long long nf = (dir != 2 ? (nx - 1) * ny : 0) + (dir != 1 ? nx * (ny - 1) : 0);
    if (nf == 0) return;
    cudaMemsetAsync(a.count + 0, 0, sizeof(int), st);
    k_flux_classify<<<blocks(nf), BLOCK, 0, st>>>(a, dir);
    if (vof_type(a.method)) k_flux_list<<<list_blocks(k_flux_list, nf), BLOCK, 0, st>>>(a, dir);
}

void launch_apply(const TrArgs &a, int dir, cudaStream_t st) {
    k_update<<<blocks((long long)a.m.nx * a.m.ny), BLOCK, 0, st>>>(a, dir);
}

void launch_normals(const TrArgs &a, cudaStream_t st) {
    const long long n = (long long)a.m.nx * a.m.ny;
    cudaMemsetAsync(a.count + 1, 0, sizeof(int), st);
    k_normals<<<blocks(n), BLOCK, 0, st>>>(a);
    k_sections<<<list_blocks(k_sections, n), BLOCK, 0, st>>>(a);
}

void launch_adjust(const TrArgs &a, cudaStream_t st) {
    k_adjust<<<list_blocks(k_adjust, (long long)a.m.nx * a.m.ny), BLOCK, 0, st>>>(a);
}

void launch_flags(const TrArgs &a, int *flags, cudaStream_t st) {
    k_flags<<<blocks((long long)a.m.nx * a.m.ny), BLOCK, 0, st>>>(a, flags);
}

}  // namespace tr
}  // namespace zg
