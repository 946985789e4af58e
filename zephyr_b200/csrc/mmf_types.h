// mmf_types.h -- arguments and launchers of the multi-material step
// (MmFluid, first order) on a rectangle mesh.
#pragma once

#include "mmf_math.cuh"
#include "smf_types.h"

namespace zg {
namespace mmf {

constexpr int NMAT = 2;  // materials per mixture in the compiled kernels
// second order: components of the state's gradients (density, vx, vy,
// pressure, energy, temperature, mass fractions, true densities)
constexpr int NG = 6 + 2 * NMAT;

// Primitive mixture state of every cell, one array per field (structure of
// arrays): density, velocity, pressure, specific internal energy,
// temperature, mass fractions and true densities (the fields of
// mmf::PState, math/cfd/models.h:167-180).
struct MmField {
    double *rho, *vx, *vy, *P, *e, *T;
    double *b[NMAT];
    double *r[NMAT];
};

struct MmArgs {
    StructMesh mesh;
    MixD<NMAT> mix;
    int crp;
    int fp32_flux;  // mixed form: FP32 face arithmetic in the pure-stencil kernel
    // direction splitting: the faces of this sub-step (0 all, 1 x faces, 2 y
    // faces; AmrFaces::to_skip, amr_faces.cpp:186-197) and its share of dt
    int dir;
    double dt_scale;
    double CFL, max_dt;
    MmField z, znext;
    double *nrm_x[NMAT], *nrm_y[NMAT], *off[NMAT];  // interface reconstruction per material
    unsigned long long *dmin_bits;
    unsigned int *dt_ticket;
    double *dt_out;
    int *err;  // set to 1 where the reference would throw
    // Work lists of the face loop: cells whose stencil holds a mixed state
    // (composite Riemann fluxes) and cells whose update came out mixed
    // (Newton closure), with their conservative states.
    int *counts;     // [0] cells in list_crp, [1] cells in list_closure
    int *list_crp, *list_closure;
    // list_crp filled beforehand (launch_classify): the pure-stencil kernel
    // only skips the listed cells, so it may run beside the composite faces
    int presorted;
    // dt kernel: leave the work lists alone (they are emptied on another
    // stream while it runs)
    int keep_lists;
    double *qbuf;    // (4 + NMAT) doubles per closure-list entry
    // face fluxes of the list_crp cells (4 faces per cell): first order, two
    // parts of (4 + NMAT) doubles per face with the face's a_sig and flags
    // (k_crp_parts); second order, one face term of (4 + NMAT) doubles
    double *fbuf;
    double *fsig;
    int *fflag;
    // second order (MmFluid::set_accuracy(2)): limiter, the half-step state
    // and the limited gradients (x, y) of the state at the old layer
    int acc, limiter;
    MmField zhalf;
    double *gx[NG], *gy[NG];
    // CrpMode::MUSCL: volume-fraction gradients, x and y per material
    // (2 NMAT arrays of n doubles)
    double *grad_a;
};

void launch_dt(const MmArgs &a, void *stream);
void launch_recover(const MmArgs &a, void *stream);
// the face loop: pure stencils, then the two work lists
void launch_flux_pure(const MmArgs &a, void *stream);
void launch_flux_pure_fp32(const MmArgs &a, void *stream);  // mmf_mixed.cu
// the same two halves separately, and the list of cells whose stencil holds a
// mixed state (built before the pure-stencil kernel when the two overlap)
void launch_classify(const MmArgs &a, void *stream);
void launch_crp_faces(const MmArgs &a, void *stream);
void launch_crp_update(const MmArgs &a, void *stream);
void launch_closure(const MmArgs &a, void *stream);
void launch_grad_a(const MmArgs &a, void *stream);  // CrpMode::MUSCL
void launch_flags(const MmArgs &a, int *flags, void *stream);
// second order: compute_grad, fluxes_stage1, fluxes_stage2 (mm_fluid.cpp:439-680)
void launch_grad2(const MmArgs &a, void *stream);
void launch_stage1(const MmArgs &a, void *stream);
void launch_stage2(const MmArgs &a, void *stream);
void launch_make_states(const MmArgs &a, const double *rho, const double *vx, const double *vy, const double *P,
                        const double *beta, void *stream);

}  // namespace mmf
}  // namespace zg
