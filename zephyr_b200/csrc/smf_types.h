// smf_types.h -- plain structs shared by the host orchestration and the
// kernels of the single-material step.
#pragma once

#include <cstdint>

#include "smf_math.cuh"

namespace zg {

// Structured rectangle, geometry in per-axis tables filled on the host with
// the reference's formulas (amr_cells_gen.cpp:128-253).
struct StructMesh {
    int nx, ny, n;
    int bc[4];       // L, R, B, T boundary flags (PERIODIC on both sides of a periodic axis)
    bool xper, yper;
    const double *X, *Y;      // vertex coordinates, nx+1 / ny+1
    const double *cx, *cy;    // cell centres (SqQuad vs<0,0>)
    const double *fxm, *fym;  // mid-edge coordinates 0.5*(X[i]+X[i+1]), 0.5*(Y[j]+Y[j+1])
    const double *inc2x, *inc2y;  // squared incircle extents per column / row
    double hx, hy, vol;
};

// Mesh given cell by cell in the layout of zephyr's AmrCells / AmrFaces
// (amr_cells.h:49-104, amr_faces.h:83-154): 8 face slots per cell
// (face_begin = 8 * ic), UNDEFINED slots skipped in slot order; hanging faces
// of a refined neighbour occupy slots side and side + 4.  Used for AMR meshes.
struct SlotMesh {
    int n;
    const double *cx, *cy, *vol, *inc;  // centre, volume, incircle diameter
    const int *fb, *fn;                 // per slot: boundary flag, neighbour cell
    const double *fnx, *fny, *fcx, *fcy, *fa;  // per slot: normal, centre, area
    // adaptive rectangle only: cell levels and the base cell size (a cell of
    // level L is hx0 / 2^L by hy0 / 2^L, axis-aligned); null level otherwise
    const int *level;
    double hx0, hy0;
    // axisymmetric meshes only (y the radius): per cell volume_alt, per slot
    // area_alt (AmrCells / AmrFaces), null otherwise
    const double *vol_alt, *fa_alt;
};

struct PrimPtr {
    double *r, *u, *v, *p, *e;
};

struct SmfArgs {
    StructMesh mesh;
    SlotMesh smesh;  // used instead of `mesh` by the slot-mesh kernels
    EosD eos;
    int flux, limiter;
    double CFL, max_dt;
    PrimPtr z, zhalf, znext;
    double *gx[4], *gy[4];  // limited gradients of density, vx, vy, pressure
    const int *wait_in;
    int *wait_out;
    unsigned long long *dmin_bits;  // running minimum of the CFL time step (bit image)
    unsigned int *dt_ticket;        // blocks of the dt kernel that have finished
    double *dt_out;                 // dt of the current step, written by the dt kernel
};

// Launchers (one set per numerics flavour).
// Parity kernels; `slots` selects the slot-mesh (AMR) geometry.
namespace parity {
void launch_dt(const SmfArgs &a, PrimPtr z, bool slots, void *stream);
void launch_flux1(const SmfArgs &a, bool slots, void *stream);
void launch_grad(const SmfArgs &a, PrimPtr z, bool slots, void *stream);
void launch_stage1(const SmfArgs &a, bool slots, void *stream);
void launch_stage2(const SmfArgs &a, bool slots, void *stream);
void launch_heun(const SmfArgs &a, PrimPtr zin, PrimPtr zout, bool final, bool slots, void *stream);
void launch_flags(const SmfArgs &a, int *flags, bool slots, void *stream);
}  // namespace parity

// FAST kernels on an adaptive rectangle (SlotFastAcc; smf_slot_fast.cu).
namespace slotfast {
void launch_dt(const SmfArgs &a, PrimPtr z, void *stream);
void launch_flux1(const SmfArgs &a, void *stream);
void launch_grad(const SmfArgs &a, PrimPtr z, void *stream);
void launch_grad_flags(const SmfArgs &a, int *flags, double refine, double coarsen, void *stream);

// Face-once form of the corrector and of the Heun stages: each face's flux
// (times its area, outward from the cell that computes it) is evaluated once,
// by one of its two cells, into the slot of that cell (8 slots per cell, one
// array per conserved component), and every cell then sums its slots in slot
// order, taking a face it does not compute from the neighbour's slot with
// the opposite sign.
struct FaceFlux {
    double4 *f;        // per face of `list`: (rho, rho u, rho v, rho E) flux times area
    const int *list;   // the slots 8 ic + s whose face cell ic computes, in cell order
    const int *fidx;   // per slot 8 ic + s: t >= 0, the face list entry it computes; -(t + 1), the
                       // neighbour's entry it takes with the opposite sign; FACE_NONE, no face
    int nfaces;        // entries of `list`
    double *dt_next;   // non-null: the cell sums also give the next step's dt (of the state they write) here
};
constexpr int FACE_NONE = -2147483647 - 1;
// The limited least-squares gradients over per-slot geometry built once per
// mesh change: sg[8 ic + s] = (rx, ry, w nx^, w ny^) (the centre offset and
// the weighted normal projections of gradient.h:251-275), bm[ic] = the
// inverse of the cell's 2x2 least-squares matrix (B00, B01, B10, B11).
void launch_grad_geometry(const SmfArgs &a, double4 *sg, double4 *bm, void *stream);
// predictor: the predictor stage (k_stage1) fused after the gradients
void launch_grad_pre(const SmfArgs &a, PrimPtr z, const double4 *sg, const double4 *bm, bool predictor,
                     void *stream);
void launch_stage2_faces(const SmfArgs &a, FaceFlux ff, void *stream);
void launch_stage2_sum(const SmfArgs &a, FaceFlux ff, void *stream);
void launch_heun_faces(const SmfArgs &a, PrimPtr zin, FaceFlux ff, void *stream);
void launch_heun_sum(const SmfArgs &a, PrimPtr zin, PrimPtr zout, bool final, FaceFlux ff, void *stream);

// Morton order of the cells for the FAST step (smf_slot_order.cu): device
// buffers of `cap` cells (keys 2 cap), cub scratch of tmp_bytes
struct OrderBuffers {
    int cap;
    unsigned long long *keys;
    int *idx, *perm, *inv;
    void *tmp;
    size_t tmp_bytes;
    double *cx, *cy, *vol, *inc;
    int *level, *fb, *fn;
    int *fcnt, *foff;  // faces each cell computes, their exclusive prefix sum (cap + 1 each)
    int *flist;        // FaceFlux::list (8 cap)
    int *fidx;         // FaceFlux::fidx (8 cap)
    int nfaces;
    double4 *sg, *bm;  // gradient geometry (8 cap, cap)
};
size_t order_scratch_bytes(int cap);
// fills b.perm (position -> cell), b.inv and the reordered mesh arrays, and
// `out`, the mesh view over them; key_bits: bits of a finest-cell index per
// axis (at most 21); 0 on success
int build_order(const SlotMesh &m, int n, double x0, double y0, double hx, double hy, int key_bits,
                OrderBuffers &b, SlotMesh &out, void *stream);
void gather_state(const int *perm, int n, PrimPtr src, PrimPtr dst, const int *wsrc, int *wdst, void *stream);
// the MIXED representation (FP64 conserved, FP32 primitive mirror) and the
// counters, into and out of the order
struct MixedState {
    double *q[4];
    float *w[5];
};
void gather_mixed(const int *perm, int n, MixedState src, MixedState dst, const int *wsrc, int *wdst, void *stream);
// eight fields of n doubles (the gradients) from the order back to the mesh's
struct Fields8 {
    double *f[8];
};
void scatter_fields8(const int *perm, int n, Fields8 src, Fields8 dst, void *stream);
void scatter_mixed(const int *perm, int n, MixedState src, MixedState dst, const int *wsrc, int *wdst,
                   void *stream);
void scatter_state(const int *perm, int n, PrimPtr src, PrimPtr dst, const int *wsrc, int *wdst, void *stream);
}  // namespace slotfast

}  // namespace zg
