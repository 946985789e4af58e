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

struct PrimPtr {
    double *r, *u, *v, *p, *e;
};

struct SmfArgs {
    StructMesh mesh;
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
namespace parity {
void launch_dt(const SmfArgs &a, PrimPtr z, void *stream);
void launch_flux1(const SmfArgs &a, void *stream);
void launch_grad(const SmfArgs &a, PrimPtr z, void *stream);
void launch_stage1(const SmfArgs &a, void *stream);
void launch_stage2(const SmfArgs &a, void *stream);
void launch_heun(const SmfArgs &a, PrimPtr zin, PrimPtr zout, bool final, void *stream);
void launch_flags(const SmfArgs &a, int *flags, void *stream);
}  // namespace parity

}  // namespace zg
