// tr_types.h -- the scalar VOF transport solver (zephyr's Transfer,
// math/solver/transfer.cpp) on a uniform rectangle: device state and the
// launchers of tr_vof.cu.
#pragma once

#include <cuda_runtime.h>

namespace zg {
namespace tr {

// Transfer::Method values (transfer.h:25-51) with GPU kernels.
enum Method {
    CRP_V3 = 0, CRP_V5 = 1, CRP_SE = 2, CRP_N1 = 3, CRP_N2 = 4, VOF = 5, VOF_CRP = 6,
    MUSCLd = 7, MUSCLn = 8, MUSCLd_CRP = 9, MUSCLn_CRP = 10, MUSCL_MC = 11, MUSCL_MC_CRP = 12, WENO = 13,
    WENO_CRP = 14
};

__host__ __device__ inline bool vof_type(int m) { return m == VOF || m == VOF_CRP; }
__host__ __device__ inline bool muscl_type(int m) { return m >= MUSCLd && m <= MUSCL_MC_CRP; }  // transfer.cpp:29-36
__host__ __device__ inline bool weno_type(int m) { return m == WENO || m == WENO_CRP; }         // transfer.cpp:38-41

// Uniform non-periodic rectangle, cell ic = i * ny + j; geometry tables with
// the reference's formulas (filled by zg_mesh_rectangle).
struct TrMesh {
    int nx, ny;
    const double *X, *Y;      // vertex coordinates, nx + 1 / ny + 1
    const double *cx, *cy;    // cell centres
    const double *fxm, *fym;  // mid-edge coordinates (face centres)
    double hx, hy, vol;       // face lengths and cell volume
};

// The velocity field: 0 a translation (vx, vy); 1 a rotation omega about
// (cx, cy) (problems/transfer.cpp:367-380).
struct TrVel {
    int kind;
    double vx, vy, cx, cy, w;
};

struct TrArgs {
    TrMesh m;
    TrVel vel;
    int method;
    double CFL;
    double *u;                               // volume fraction u1 per cell
    double *u_next;                          // u1 after the update (the host swaps u and u_next)
    double *nx[2], *ny[2], *px[2], *py[2];   // interface normal and base point, two buffers
    int cur;                                 // buffer holding the current n and p
    double *fxa, *fxb;  // x faces ((nx + 1) * ny, face i * ny + j): flux summed by the left / right cell
    double *fya, *fyb;  // y faces (nx * (ny + 1), face i * (ny + 1) + j): by the lower / upper cell
    double *dt;         // time step used by the update kernels
    double *time;       // current time, advanced by the dt kernel in advance mode
    unsigned long long *dmin;  // running CFL minimum (bit image of a non-negative double)
    unsigned int *ticket;      // blocks of the dt kernel that have finished
    int *err;                  // [0] polygon capacity overflows
    int *count;                // work-list lengths: [0] faces, [1] cells
    int *flist;                // faces whose VOF flux clips polygons (index over the update's faces)
    int *clist;                // cells with a non-zero interface normal
    unsigned char *zero_np;    // 1: both n / p buffers of the cell hold n = (+0, +0) and p = its centre
    double *gx, *gy;           // the MUSCL slopes du_dx, du_dy per cell
    int limiter;               // m_limiter of MUSCL_MC (transfer.cpp:47: MC)
};

// Transfer::compute_dt (transfer.cpp:88-105) into *a.dt.  With `advance`
// the step is clipped to end at t_end and *a.time advances by it, as the
// transfer problem's time loop does (problems/transfer.cpp:213-232).
void launch_compute_dt(const TrArgs &a, bool advance, double t_end, cudaStream_t st);

// Transfer::compute_slopes (transfer.cpp:404-469) of the MUSCL methods.
void launch_slopes(const TrArgs &a, cudaStream_t st);

// Fluxes through the interior faces of direction dir (0 ANY, 1 X, 2 Y):
// swept polygons (VOF, VOF_CRP), the CRP formulas, or the MUSCL face values.
void launch_flux(const TrArgs &a, int dir, cudaStream_t st);

// Transfer::update_WENO's fluxes and update (transfer.cpp:541-666) into
// u_next; the caller swaps u and u_next.
void launch_weno(const TrArgs &a, int dir, cudaStream_t st);

// u_next <- between(u1 - sum of face fluxes / volume, 0, 1); the caller
// swaps u and u_next.
void launch_apply(const TrArgs &a, int dir, cudaStream_t st);

// compute_normals + find_sections into the buffers a.cur.
void launch_normals(const TrArgs &a, cudaStream_t st);

// adjust_normals + find_sections from the buffers a.cur into the others
// (the caller flips a.cur).
void launch_adjust(const TrArgs &a, cudaStream_t st);

// Transfer::set_flags (transfer.cpp:660-680).
void launch_flags(const TrArgs &a, int *flags, cudaStream_t st);

}  // namespace tr
}  // namespace zg
