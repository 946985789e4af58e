// amr_core.cuh -- quadtree adaptation of a 2-D mesh in zephyr's AmrCells
// layout (mesh/euler/amr_cells.h, amr_faces.h): one rank, plane (non-axial)
// cells.  Per-cell routines shared by the GPU kernels of amr_refine.cu; every
// one follows the reference's algorithm (mesh/amr/*.h) and its floating-point
// operation order, so that the adapted mesh -- cell order, geometry, face
// connectivity and the distributed states -- matches the reference's
// EuMesh::refine bit for bit (compile with -fmad=false).
//
// Layout (capacity `cap` cells, face slot s of cell i at 8 i + s, slot side
// and side + 4 for the two halves of a split side, map point k of cell i at
// 9 i + k with k = 3 (j + 1) + (i + 1) for the point (i, j) of the square map
// SqQuad):
//   cells: vx, vy (9 map points), cx, cy (centroid), vol, level, flag,
//          b_idx, z_idx, next, index (< 0: undefined slot)
//   faces: fb (Boundary code, -1 UNDEFINED), fadj (neighbour), fv (2 map
//          points per face), fnx, fny (outward normal), fcx, fcy, fa
#pragma once

#include <cuda_runtime.h>

#include <cmath>

#include "smf_math.cuh"

#ifdef __CUDACC__
#define ZA_HD __host__ __device__ __forceinline__
#else
#define ZA_HD inline
#endif

namespace zg {
namespace amr {

constexpr int L = 0, R = 1, B = 2, T = 3;  // Side2D

struct View {
    int n;  // cells before adaptation
    double *vx, *vy, *cx, *cy, *vol;
    int *level, *flag, *b_idx, *z_idx, *next, *index;
    int *fb, *fadj;
    signed char *fv;
    double *fnx, *fny, *fcx, *fcy, *fa;
    // SmFluid state (field `init`), isolation counters (`wait`) and the
    // limited gradients of rho, u, v, p (fields d_dx, d_dy) for the slope
    // split.  All of a cell's fields travel with it when it is moved; a new
    // cell starts with zero gradients (the storage rows the reference appends
    // for new cells are zero-filled), which a later split without a fresh
    // gradient computation reads as the reference does.
    double *zr, *zu, *zv, *zp, *ze;
    int *wait;
    double *gx[4], *gy[4];
    int slope;  // distributor: 1 "slope", 0 "const" (SmFluid::distributor, sm_fluid.cpp:372-470)
    EosD eos;
};

// ---- index tables (geom/indexing.h) -----------------------------------------
ZA_HD int vs(int i, int j) { return 3 * (j + 1) + (i + 1); }
// map points of the simple face of each side, and of the halves of a split side
ZA_HD void sf(int side, int &a, int &b) {  // face_nodes2d
    const int t[4][2] = {{0, 6}, {2, 8}, {0, 2}, {6, 8}};
    a = t[side][0];
    b = t[side][1];
}
ZA_HD void cf(int sub, int &a, int &b) {  // subface_nodes2d
    const int t[8][2] = {{0, 3}, {2, 5}, {0, 1}, {6, 7}, {3, 6}, {5, 8}, {1, 2}, {7, 8}};
    a = t[sub][0];
    b = t[sub][1];
}
ZA_HD int child_by_subface(int sub) {  // child_by_subface_2D
    const int t[8] = {0, 1, 0, 2, 2, 3, 1, 3};
    return t[sub];
}
ZA_HD void children_by_side(int side, int &c0, int &c1) {  // children_by_face_2D
    const int t[4][2] = {{0, 2}, {1, 3}, {0, 1}, {2, 3}};
    c0 = t[side][0];
    c1 = t[side][1];
}
ZA_HD int subface_by_child(int side, int child) {  // subface_by_side_child_2D
    const int t[4][4] = {{0, -1, 4, -1}, {-1, 1, -1, 5}, {2, 6, -1, -1}, {-1, -1, 3, 7}};
    return t[side][child];
}
ZA_HD int neib_child(int sub) {  // neib_child_by_symm_subface_2D[0] (no rotation on one rank)
    const int t[8] = {1, 0, 2, 0, 3, 2, 3, 1};
    return t[sub];
}
ZA_HD int adjacent_child(int side, int child) { return neib_child(subface_by_child(side, child)); }
// child index of (i, j) in {-1, +1}^2 (Quad::iss)
ZA_HD int iss(int i, int j) { return (j > 0 ? 2 : 0) + (i > 0 ? 1 : 0); }

ZA_HD bool is_bnd(int flag) { return flag != BC_INNER && flag != BC_PERIODIC && flag != BC_UNDEFINED; }

// ---- geometry (geom/primitives/quad.cpp, line.cpp) ------------------------------
struct P2 {
    double x, y;
};
ZA_HD P2 map_pt(const View &m, int ic, int k) { return {m.vx[9 * ic + k], m.vy[9 * ic + k]}; }

// Quad::get (quad.cpp:282-287): bilinear point of the quad (v00, v10, v01, v11)
ZA_HD P2 quad_get(P2 v00, P2 v10, P2 v01, P2 v11, double x, double y) {
    double a = (1.0 - x) * (1.0 - y), b = (1.0 + x) * (1.0 - y), c = (1.0 - x) * (1.0 + y), d = (1.0 + x) * (1.0 + y);
    return {0.25 * (a * v00.x + b * v10.x + c * v01.x + d * v11.x),
            0.25 * (a * v00.y + b * v10.y + c * v01.y + d * v11.y)};
}
// Line::normal (line.cpp:18-20, 65-67): perpendicular(v1 - v0, v0 - view)
ZA_HD P2 line_normal(P2 v0, P2 v1, P2 view) {
    double tx = v1.x - v0.x, ty = v1.y - v0.y;
    double ax = v0.x - view.x, ay = v0.y - view.y;
    // (tau x a) x tau with zero z components, then normalized()
    double w = tx * ay - ty * ax;
    double c0 = ty * 0.0 - 0.0 * ay, c1 = 0.0 * ax - tx * 0.0;
    double x = c1 * 0.0 - w * ty, y = w * tx - c0 * 0.0, z = c0 * ty - c1 * tx;
    double s = x * x + y * y + z * z;
    if (s > 0.0) {
        double r = sqrt(s);
        return {x / r, y / r};
    }
    return {x, y};
}
ZA_HD double line_length(P2 v0, P2 v1) {
    double dx = v1.x - v0.x, dy = v1.y - v0.y, dz = 0.0 - 0.0;
    return sqrt(dx * dx + dy * dy + dz * dz);
}

// AmrCells::set_cell(ic, Quad, axial = false) (amr_cells.cpp:725-784) for the
// quad of corners (v00, v10, v01, v11): map points, area, centroid, the four
// simple faces (INNER, no neighbour yet), the four half-face slots UNDEFINED.
ZA_HD void set_cell(const View &m, int ic, P2 v00, P2 v10, P2 v01, P2 v11) {
    // Quad::area (quad.cpp:322-324): 0.5 |(v11 - v00) x (v01 - v10)|
    double ax = v11.x - v00.x, ay = v11.y - v00.y, bx = v01.x - v10.x, by = v01.y - v10.y;
    double cz0 = ay * 0.0 - 0.0 * by, cz1 = 0.0 * bx - ax * 0.0, cz = ax * by - ay * bx;
    double area = 0.5 * sqrt(cz0 * cz0 + cz1 * cz1 + cz * cz);
    // Quad::centroid_oxy (quad.cpp:358-377), corners in the order 0, 1, 3, 2
    const P2 q[4] = {v00, v10, v11, v01};
    double Cx = 0.0, Cy = 0.0;
    for (int i = 0; i < 4; ++i) {
        P2 p1 = q[i], p2 = q[(i + 1) % 4];
        Cx += (p2.y - p1.y) * (p2.x * p2.x + p2.x * p1.x + p1.x * p1.x);
        Cy -= (p2.x - p1.x) * (p2.y * p2.y + p2.y * p1.y + p1.y * p1.y);
    }
    double d6 = 6.0 * area;
    Cx /= d6;
    Cy /= d6;
    m.vol[ic] = area;
    m.cx[ic] = Cx;
    m.cy[ic] = Cy;
    m.flag[ic] = 0;
    m.b_idx[ic] = -1;
    m.z_idx[ic] = -1;
    m.level[ic] = -1;
    m.index[ic] = -1;
    // SqQuad(const Quad&) (quad.cpp:452-457)
    const P2 pts[9] = {v00, quad_get(v00, v10, v01, v11, 0.0, -1.0), v10,
                       quad_get(v00, v10, v01, v11, -1.0, 0.0), quad_get(v00, v10, v01, v11, 0.0, 0.0),
                       quad_get(v00, v10, v01, v11, +1.0, 0.0), v01, quad_get(v00, v10, v01, v11, 0.0, +1.0),
                       v11};
    for (int k = 0; k < 9; ++k) {
        m.vx[9 * ic + k] = pts[k].x;
        m.vy[9 * ic + k] = pts[k].y;
    }
    // AmrFaces::insert(AMR2D) then the four simple faces
    const P2 C{Cx, Cy};
    for (int s = 0; s < 8; ++s) {
        int f = 8 * ic + s;
        m.fb[f] = BC_UNDEFINED;
        m.fadj[f] = -1;
    }
    for (int s = 0; s < 4; ++s) {
        int f = 8 * ic + s, a, b;
        sf(s, a, b);
        m.fv[2 * f] = (signed char)a;
        m.fv[2 * f + 1] = (signed char)b;
        P2 p0 = pts[a], p1 = pts[b];
        m.fa[f] = line_length(p0, p1);
        m.fcx[f] = 0.5 * (p0.x + p1.x);
        m.fcy[f] = 0.5 * (p0.y + p1.y);
        P2 nn = line_normal(p0, p1, C);
        m.fnx[f] = nn.x;
        m.fny[f] = nn.y;
        m.fb[f] = BC_INNER;
    }
}

// setup_face_geom (faces.h) of slot f of cell ic with the cell's map
ZA_HD void face_geom(const View &m, int ic, int f) {
    P2 C = map_pt(m, ic, 4);  // SqQuad::center (quad.cpp:534-536)
    P2 p0 = map_pt(m, ic, m.fv[2 * f]), p1 = map_pt(m, ic, m.fv[2 * f + 1]);
    m.fa[f] = line_length(p0, p1);
    m.fcx[f] = 0.5 * (p0.x + p1.x);
    m.fcy[f] = 0.5 * (p0.y + p1.y);
    P2 nn = line_normal(p0, p1, C);
    m.fnx[f] = nn.x;
    m.fny[f] = nn.y;
}
// split_face (faces.h): side -> halves side (cf(side)) and side + 4
ZA_HD void split_face(const View &m, int ic, int side) {
    int f0 = 8 * ic + side, f1 = 8 * ic + side + 4, a, b;
    cf(side, a, b);
    m.fv[2 * f0] = (signed char)a;
    m.fv[2 * f0 + 1] = (signed char)b;
    cf(side + 4, a, b);
    m.fv[2 * f1] = (signed char)a;
    m.fv[2 * f1 + 1] = (signed char)b;
    m.fb[f1] = m.fb[f0];
    m.fadj[f1] = m.fadj[f0];
    face_geom(m, ic, f0);
    face_geom(m, ic, f1);
}
// merge_faces (faces.h): the two halves -> the simple face of `side`
ZA_HD void merge_faces(const View &m, int ic, int side) {
    int f0 = 8 * ic + side, f1 = 8 * ic + side + 4, a, b;
    sf(side, a, b);
    m.fv[2 * f0] = (signed char)a;
    m.fv[2 * f0 + 1] = (signed char)b;
    m.fb[f1] = BC_UNDEFINED;
    m.fadj[f1] = -1;
    face_geom(m, ic, f0);
}
ZA_HD bool simple_face(const View &m, int ic, int side) { return m.fb[8 * ic + side + 4] == BC_UNDEFINED; }

// ---- siblings (mesh/amr/siblings.h) --------------------------------------------
ZA_HD int next_sibling_side(int z) {  // side_to_next_sibling<2>: RIGHT, TOP, BOTTOM, LEFT
    const int t[4] = {R, T, B, L};
    return t[z];
}
ZA_HD bool can_coarse(const View &m, int ic) {
    if (m.flag[ic] >= 0) return false;
    for (int i = 0; i < 3; ++i) {
        int z = m.z_idx[ic] % 4;
        int jface = 8 * ic + next_sibling_side(z);
        int jc = m.fadj[jface];
        if (m.fb[jface] == BC_UNDEFINED) return false;  // adjacent.rank != rank
        if (m.level[ic] != m.level[jc]) return false;
        if (m.flag[jc] >= 0) return false;
        ic = jc;
    }
    return true;
}
ZA_HD void get_siblings(const View &m, int ic, int sibs[3]) {
    int jc = ic;
    for (int i = 0; i < 3; ++i) {
        int z = m.z_idx[jc] % 4;
        jc = m.fadj[8 * jc + next_sibling_side(z)];
        sibs[i] = jc;
    }
}

// ---- flag balancing (mesh/amr/balancing_restrictions.h, balancing_fast.h) -----
// base_restriction: flags to {-1, 0, 1}, levels kept in [0, max_level],
// coarsening only when all four siblings want it
ZA_HD void base_restriction(const View &m, int ic, int max_level) {
    int flag = m.flag[ic];
    if (flag != 0) flag = flag > 0 ? 1 : -1;
    int lvl = m.level[ic];
    if (lvl + flag < 0) {
        flag = 0;
    } else if (lvl + flag > max_level) {
        flag = lvl > max_level ? -1 : 0;
    }
    // can_coarse reads this cell's flag as it was before this restriction
    // (negative whenever the restricted flag is, for levels <= max_level)
    if (flag < 0 && !can_coarse(m, ic)) flag = 0;
    m.flag[ic] = flag;
}
// retain_update_flag: a kept cell refines when a neighbour wants two levels finer
ZA_HD void retain_update(const View &m, int ic) {
    for (int s = 0; s < 8; ++s) {
        int f = 8 * ic + s;
        if (m.fb[f] == BC_UNDEFINED || is_bnd(m.fb[f])) continue;
        int jc = m.fadj[f];
        if (m.level[jc] + m.flag[jc] > m.level[ic] + 1) {
            m.flag[ic] = 1;
            return;
        }
    }
}
// coarse_update_flag: a coarsening cell keeps or refines by its neighbours' wishes
ZA_HD void coarse_update(const View &m, int ic) {
    if (m.flag[ic] >= 0) return;
    for (int s = 0; s < 8; ++s) {
        int f = 8 * ic + s;
        if (m.fb[f] == BC_UNDEFINED || is_bnd(m.fb[f])) continue;
        int jc = m.fadj[f];
        int wanted = m.level[jc] + m.flag[jc];
        if (wanted > m.level[ic]) {
            if (wanted > m.level[ic] + 1) {
                m.flag[ic] = 1;
                return;
            }
            m.flag[ic] = 0;
        }
    }
}
// coarse_update_flag_by_sibs: no coarsening unless every sibling coarsens
ZA_HD void coarse_update_by_sibs(const View &m, int ic) {
    if (m.flag[ic] >= 0) return;
    int sibs[3];
    get_siblings(m, ic, sibs);
    for (int k = 0; k < 3; ++k) {
        if (m.flag[sibs[k]] >= 0) {
            m.flag[ic] = 0;
            break;
        }
    }
}

// ---- distributor (SmFluid::distributor, sm_fluid.cpp:372-470) ----------------
ZA_HD void state_get(const View &m, int ic, Prim &z) {
    z.r = m.zr[ic];
    z.u = m.zu[ic];
    z.v = m.zv[ic];
    z.p = m.zp[ic];
    z.e = m.ze[ic];
}
ZA_HD void zero_grad(const View &m, int ic) {
    for (int k = 0; k < 4; ++k) {
        m.gx[k][ic] = 0.0;
        m.gy[k][ic] = 0.0;
    }
}
ZA_HD void state_put(const View &m, int ic, const Prim &z) {
    m.zr[ic] = z.r;
    m.zu[ic] = z.u;
    m.zv[ic] = z.v;
    m.zp[ic] = z.p;
    m.ze[ic] = z.e;
    m.wait[ic] = 0;
}
// split: "slope" extrapolates with the parent's limited gradients (density,
// velocity, pressure; energy through the EoS derivatives), "const" copies
ZA_HD void split_states(const View &m, int ip, int main_child) {
    Prim zp;
    state_get(m, ip, zp);
    if (m.slope) {
        const double gxr = m.gx[0][ip], gxu = m.gx[1][ip], gxv = m.gx[2][ip], gxp = m.gx[3][ip];
        const double gyr = m.gy[0][ip], gyu = m.gy[1][ip], gyv = m.gy[2][ip], gyp = m.gy[3][ip];
        // pressure_re derivatives (ideal_gas.cpp:26-33, stiffened_gas.cpp:104-111)
        const double PdR = m.eos.kind == EOS_IDEAL ? m.eos.gm1 * zp.e : m.eos.gm1 * (zp.e - m.eos.e0);
        const double PdE = m.eos.gm1 * zp.r;
        const double gex = (gxp - PdR * gxr) / PdE, gey = (gyp - PdR * gyr) / PdE;
        const double gez = (0.0 - PdR * 0.0) / PdE;
        bool bad_grad = false;
        Prim zc[4];
        for (int k = 0; k < 4; ++k) {
            int ic = main_child + k;
            double drx = m.cx[ic] - m.cx[ip], dry = m.cy[ic] - m.cy[ip], drz = 0.0 - 0.0;
            Prim c = zp;
            c.r = zp.r + gxr * drx + gyr * dry + 0.0 * drz;
            double ratio = zp.r / c.r;
            c.u = zp.u + ratio * (gxu * drx + gyu * dry + 0.0 * drz);
            c.v = zp.v + ratio * (gxv * drx + gyv * dry + 0.0 * drz);
            double du = zp.u - c.u, dv = zp.v - c.v, dw = 0.0 - 0.0;
            c.e = zp.e - 0.5 * (du * du + dv * dv + dw * dw) + ratio * (gex * drx + gey * dry + gez * drz);
            c.p = m.eos.pressure_re(c.r, c.e);
            if (is_bad(c, m.eos)) {
                bad_grad = true;
                break;
            }
            zc[k] = c;
        }
        if (!bad_grad) {
            for (int k = 0; k < 4; ++k) state_put(m, main_child + k, zc[k]);
            return;
        }
    }
    for (int k = 0; k < 4; ++k) state_put(m, main_child + k, zp);
}
// merge: volume-weighted sum of the children's conservative states
ZA_HD void merge_states(const View &m, const int ch[4], int ip) {
    Cons q{0.0, 0.0, 0.0, 0.0};
    for (int k = 0; k < 4; ++k) {
        Prim z;
        state_get(m, ch[k], z);
        Cons qc = q_from_p(z);
        double w = m.vol[ch[k]];
        q.r += qc.r * w;
        q.mu += qc.mu * w;
        q.mv += qc.mv * w;
        q.E += qc.E * w;
    }
    double V = m.vol[ip];
    q.r /= V;
    q.mu /= V;
    q.mv /= V;
    q.E /= V;
    state_put(m, ip, p_from_q(q, m.eos));
}

// ---- retain / refine / coarse (mesh/amr/retain.h, refine.h, coarse.h) ------------
// A kept cell: its faces now point at the neighbours' new cells.
ZA_HD void retain_cell(const View &m, int ic) {
    const int lvl_c = m.level[ic];
    for (int side = 0; side < 4; ++side) {
        const int f = 8 * ic + side;
        if (m.fb[f] == BC_UNDEFINED) continue;
        if (is_bnd(m.fb[f])) {
            m.fadj[f] = m.next[ic];
            continue;
        }
        const int jc = m.fadj[f];
        const int lvl_n = m.level[jc];
        if (lvl_c == lvl_n) {
            const int neib_next = m.next[jc];
            if (m.flag[jc] > 0) {
                split_face(m, ic, side);
                m.fadj[f] = m.next[neib_next + neib_child(side)];
                m.fadj[f + 4] = m.next[neib_next + neib_child(side + 4)];
            } else if (m.flag[jc] == 0) {
                m.fadj[f] = neib_next;
            } else {
                m.fadj[f] = m.next[neib_next];
            }
        } else if (lvl_c < lvl_n) {
            if (m.flag[jc] < 0) {
                merge_faces(m, ic, side);
                m.fadj[f] = m.next[m.next[jc]];
            } else {
                for (int sub = side; sub < 8; sub += 4) {
                    int kc = m.fadj[8 * ic + sub];
                    m.fadj[8 * ic + sub] = m.next[kc];
                }
            }
        } else {
            if (m.flag[jc] == 0) {
                m.fadj[f] = m.next[jc];
            } else {
                int zch = adjacent_child(side, m.z_idx[ic] % 4);
                m.fadj[f] = m.next[m.next[jc] + zch];
            }
        }
    }
}

// A refined cell: four children at next[ip].., linked to each other and to the
// neighbours' new cells, states split by the distributor.
ZA_HD void refine_cell(const View &m, int ip) {
    const int mc = m.next[ip];
    // SqQuad::children + reduce (quad.cpp:641-661, 459-461): corners from the
    // parent's map points
    const int corner[4][4] = {{vs(-1, -1), vs(0, -1), vs(-1, 0), vs(0, 0)},
                              {vs(0, -1), vs(1, -1), vs(0, 0), vs(1, 0)},
                              {vs(-1, 0), vs(0, 0), vs(-1, 1), vs(0, 1)},
                              {vs(0, 0), vs(1, 0), vs(0, 1), vs(1, 1)}};
    for (int k = 0; k < 4; ++k)
        set_cell(m, mc + k, map_pt(m, ip, corner[k][0]), map_pt(m, ip, corner[k][1]), map_pt(m, ip, corner[k][2]),
                 map_pt(m, ip, corner[k][3]));
    for (int k = 0; k < 4; ++k) {
        int ich = mc + k;
        zero_grad(m, ich);
        m.index[ich] = ich;
        m.flag[ich] = 0;
        m.b_idx[ich] = m.b_idx[ip];
        m.level[ich] = m.level[ip] + 1;
        m.z_idx[ich] = 4 * m.z_idx[ip] + k;
    }
    // link_siblings (refine.h:30-45): child, side, sibling
    const int link[8][3] = {{0, R, 1}, {0, T, 2}, {1, L, 0}, {1, T, 3}, {2, R, 3}, {2, B, 0}, {3, L, 2}, {3, B, 1}};
    for (int k = 0; k < 8; ++k) {
        int f = 8 * (mc + link[k][0]) + link[k][1];
        m.fb[f] = BC_INNER;
        m.fadj[f] = m.next[mc + link[k][2]];
    }
    const int face_beg = 8 * ip;
    for (int side = 0; side < 4; ++side) {
        int c0, c1;
        children_by_side(side, c0, c1);
        const int cs[2] = {c0, c1};
        const int flag = m.fb[face_beg + side];
        if (flag == BC_UNDEFINED) continue;
        for (int i : cs) m.fb[8 * (mc + i) + side] = flag;
        if (is_bnd(flag)) {
            for (int i : cs) m.fadj[8 * (mc + i) + side] = m.next[mc + i];
            continue;
        }
        if (simple_face(m, ip, side)) {
            const int jc = m.fadj[face_beg + side];
            for (int i : cs) {
                int chf = 8 * (mc + i) + side;
                if (m.level[ip] > m.level[jc]) {
                    int zch = adjacent_child(side, m.z_idx[ip] % 4);
                    m.fadj[chf] = m.next[m.next[jc] + zch];
                } else if (m.flag[jc] == 0) {
                    m.fadj[chf] = m.next[jc];
                } else {
                    int zch = adjacent_child(side, i);
                    m.fadj[chf] = m.next[m.next[jc] + zch];
                }
            }
        } else {
            for (int i : cs) {
                int chf = 8 * (mc + i) + side;
                int jc = m.fadj[face_beg + subface_by_child(side, i)];
                if (m.flag[jc] == 0) m.fadj[chf] = m.next[jc];
                else if (m.flag[jc] < 0) m.fadj[chf] = m.next[m.next[jc]];
                else m.fadj[chf] = jc;  // fixed below
            }
        }
    }
    // a child's side next to a neighbour that is finer and refines again
    for (int side = 0; side < 4; ++side) {
        const int pf = face_beg + side;
        if (simple_face(m, ip, side) || m.fb[pf] == BC_UNDEFINED || is_bnd(m.fb[pf])) continue;
        int c0, c1;
        children_by_side(side, c0, c1);
        const int cs[2] = {c0, c1};
        for (int i : cs) {
            const int ich = mc + i;
            const int jc = m.fadj[face_beg + subface_by_child(side, i)];
            if (m.level[jc] + m.flag[jc] > m.level[ich]) {
                split_face(m, ich, side);
                const int neib_next = m.next[jc];
                for (int sub = side; sub < 8; sub += 4) m.fadj[8 * ich + sub] = m.next[neib_next + neib_child(sub)];
            }
        }
    }
    split_states(m, ip, mc);
    m.index[ip] = -1;
}

// A coarsened family: the sibling with z_idx % 4 == 0 builds the parent at its
// next[] from the children's map points; the others only leave.
ZA_HD void coarse_cell(const View &m, int ich) {
    if (m.z_idx[ich] % 4 != 0) {
        m.index[ich] = -1;
        return;
    }
    int sibs[3], ch[4];
    get_siblings(m, ich, sibs);
    ch[0] = ich;
    for (int k = 0; k < 3; ++k) ch[m.z_idx[sibs[k]] % 4] = sibs[k];
    const int ip = m.next[ich];
    // parent_vs (coarse.h:55-70) then set_cell(SqQuad) -> reduce: the corners
    set_cell(m, ip, map_pt(m, ch[0], vs(-1, -1)), map_pt(m, ch[1], vs(+1, -1)), map_pt(m, ch[2], vs(-1, +1)),
             map_pt(m, ch[3], vs(+1, +1)));
    const int ip_next = m.next[ip];
    zero_grad(m, ip);
    m.index[ip] = ip;
    m.flag[ip] = 0;
    m.b_idx[ip] = m.b_idx[ch[0]];
    m.level[ip] = m.level[ch[0]] - 1;
    m.z_idx[ip] = m.z_idx[ch[0]] / 4;
    const int face_beg = 8 * ip;
    for (int side = 0; side < 4; ++side) {
        const int some_ch = ch[child_by_subface(side)];
        const int scf = 8 * some_ch + side;
        m.fb[face_beg + side] = m.fb[scf];
        if (is_bnd(m.fb[scf])) {
            m.fadj[face_beg + side] = ip_next;
            continue;
        }
        const int some_neib = m.fadj[scf];
        const int wanted = m.level[some_neib] + m.flag[some_neib];
        if (wanted <= m.level[ip]) {
            m.fadj[face_beg + side] = m.flag[some_neib] == 0 ? m.next[some_neib] : m.next[m.next[some_neib]];
            m.fb[face_beg + side + 4] = BC_UNDEFINED;
            m.fadj[face_beg + side + 4] = -1;
            continue;
        }
        split_face(m, ip, side);
        for (int sub = side; sub < 8; sub += 4) {
            const int ic2 = ch[child_by_subface(sub)];
            const int jc = m.fadj[8 * ic2 + side];
            int v;
            if (m.level[ic2] > m.level[jc]) v = m.next[m.next[jc] + neib_child(sub)];
            else if (m.flag[jc] == 0) v = m.next[jc];
            else v = m.next[m.next[jc]];
            m.fadj[face_beg + sub] = v;
        }
    }
    merge_states(m, ch, ip);
    m.index[ich] = -1;
}

// move_item (amr_cells.cpp:428-468) with the cell's data: from -> to
ZA_HD void move_cell(const View &m, int from, int to) {
    m.next[to] = to;
    m.index[to] = to;
    m.flag[to] = m.flag[from];
    m.level[to] = m.level[from];
    m.b_idx[to] = m.b_idx[from];
    m.z_idx[to] = m.z_idx[from];
    m.cx[to] = m.cx[from];
    m.cy[to] = m.cy[from];
    m.vol[to] = m.vol[from];
    for (int s = 0; s < 8; ++s) {
        int a = 8 * from + s, b = 8 * to + s;
        m.fb[b] = m.fb[a];
        m.fnx[b] = m.fnx[a];
        m.fny[b] = m.fny[a];
        m.fcx[b] = m.fcx[a];
        m.fcy[b] = m.fcy[a];
        m.fa[b] = m.fa[a];
        m.fv[2 * b] = m.fv[2 * a];
        m.fv[2 * b + 1] = m.fv[2 * a + 1];
        m.fadj[b] = m.fadj[a];
    }
    for (int k = 0; k < 9; ++k) {
        m.vx[9 * to + k] = m.vx[9 * from + k];
        m.vy[9 * to + k] = m.vy[9 * from + k];
    }
    m.zr[to] = m.zr[from];
    m.zu[to] = m.zu[from];
    m.zv[to] = m.zv[from];
    m.zp[to] = m.zp[from];
    m.ze[to] = m.ze[from];
    m.wait[to] = m.wait[from];
    for (int k = 0; k < 4; ++k) {
        m.gx[k][to] = m.gx[k][from];
        m.gy[k][to] = m.gy[k][from];
    }
    m.index[from] = -1;
}

}  // namespace amr
}  // namespace zg
