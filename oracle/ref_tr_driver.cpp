// ref_tr_driver.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Runs the reference's own Transfer solver (math/solver/transfer.cpp) with its
// InterfaceRecovery (geom/interface_recovery.cpp) and Polygon clipping
// (geom/primitives/polygon.cpp) on the reference's own EuMesh, all compiled
// from the reference sources, and exposes a C interface so that tests can pin
// the oracle's VOF transport restatement (and through it the GPU kernels) to
// the reference.  Built by oracle/ref_build.py into oracle/_ref/libzref_mesh.so.
//
// The velocity field is the one of the reference's transfer problem
// (problems/transfer.cpp:367-380): a translation V0, or a rotation omega x
// (p - center) about the z axis.
#include <cmath>
#include <memory>

#include <zephyr/geom/generator/rectangle.h>
#include <zephyr/geom/primitives/polygon.h>
#include <zephyr/math/solver/transfer.h>
#include <zephyr/mesh/euler/eu_mesh.h>

using namespace zephyr;
using geom::Boundary;
using geom::Vector3d;
using mesh::EuCell;
using mesh::EuMesh;

namespace {

class VelTransfer : public math::Transfer {
public:
    int kind = 0;                     // 0 translation, 1 rotation
    Vector3d V0{0.7, -0.35, 0.0};     // translation velocity
    Vector3d center{0.5, 0.5, 0.0};   // rotation centre
    Vector3d omega{0.0, 0.0, M_PI};   // angular velocity

    Vector3d velocity(const Vector3d &p) const override {
        if (kind == 0) return V0;
        return omega.cross(p - center);
    }
};

struct RefTr {
    std::unique_ptr<EuMesh> mesh;
    VelTransfer solver;
};

}  // namespace

extern "C" {

// Transfer on Rectangle(x_min, x_max, y_min, y_max), nx by ny cells, boundary
// flags {left, right, bottom, top}.  method: the value of Transfer::Method;
// vel_kind 0: vel = {vx, vy}; 1: vel = {cx, cy, omega}.
void *ztr_create(int nx, int ny, double x_min, double x_max, double y_min, double y_max, const int *bounds,
                 int method, double CFL, int vel_kind, const double *vel) {
    auto *r = new RefTr();
    geom::generator::Rectangle gen(x_min, x_max, y_min, y_max);
    gen.set_boundaries({.left = Boundary(bounds[0]), .right = Boundary(bounds[1]),
                        .bottom = Boundary(bounds[2]), .top = Boundary(bounds[3])});
    gen.set_sizes(nx, ny);
    r->mesh = std::make_unique<EuMesh>(gen);
    r->solver.kind = vel_kind;
    if (vel_kind == 0) {
        r->solver.V0 = Vector3d(vel[0], vel[1], 0.0);
    } else {
        r->solver.center = Vector3d(vel[0], vel[1], 0.0);
        r->solver.omega = Vector3d(0.0, 0.0, vel[2]);
    }
    r->solver.set_CFL(CFL);
    r->solver.set_method(math::Transfer::Method(method));
    r->solver.add_types(*r->mesh);
    return r;
}

void ztr_free(void *p) { delete static_cast<RefTr *>(p); }

int ztr_n_cells(void *p) { return (int)static_cast<RefTr *>(p)->mesh->n_cells(); }

// BodyDisk::initial (problems/transfer.cpp:348-354): u1 = |cell ∩ disk| / volume.
void ztr_disk(void *p, double cx, double cy, double R, double *u1) {
    auto *r = static_cast<RefTr *>(p);
    int n = (int)r->mesh->n_cells();
    for (int i = 0; i < n; ++i) {
        EuCell cell = (*r->mesh)[i];
        u1[i] = cell.polygon().disk_clip_area(Vector3d(cx, cy, 0.0), R) / cell.volume();
    }
}

void ztr_set_u(void *p, const double *u1) {
    auto *r = static_cast<RefTr *>(p);
    int n = (int)r->mesh->n_cells();
    for (int i = 0; i < n; ++i) {
        EuCell cell = (*r->mesh)[i];
        cell[r->solver.data.u1] = u1[i];
        cell[r->solver.data.u2] = 0.0;
    }
}

void ztr_update_interface(void *p, int smoothing) {
    auto *r = static_cast<RefTr *>(p);
    r->solver.update_interface(*r->mesh, smoothing);
}

double ztr_compute_dt(void *p) {
    auto *r = static_cast<RefTr *>(p);
    return r->solver.compute_dt(*r->mesh);
}

void ztr_set_dt(void *p, double dt) { static_cast<RefTr *>(p)->solver.set_dt(dt); }

// Transfer::update(mesh, dir): dir 0 ANY, 1 X, 2 Y.
void ztr_update(void *p, int dir) {
    auto *r = static_cast<RefTr *>(p);
    r->solver.update(*r->mesh, mesh::Direction(dir));
}

// u1 per cell; interface normal and base point (x, y) per cell.
void ztr_get(void *p, double *u1, double *nrm, double *pt) {
    auto *r = static_cast<RefTr *>(p);
    int n = (int)r->mesh->n_cells();
    for (int i = 0; i < n; ++i) {
        EuCell cell = (*r->mesh)[i];
        u1[i] = cell[r->solver.data.u1];
        Vector3d nv = cell[r->solver.data.n], pv = cell[r->solver.data.p];
        nrm[2 * i] = nv.x();
        nrm[2 * i + 1] = nv.y();
        pt[2 * i] = pv.x();
        pt[2 * i + 1] = pv.y();
    }
}

// Transfer::set_flags: refinement flags per cell.
void ztr_flags(void *p, int *flags) {
    auto *r = static_cast<RefTr *>(p);
    r->solver.set_flags(*r->mesh);
    int n = (int)r->mesh->n_cells();
    for (int i = 0; i < n; ++i) flags[i] = (*r->mesh)[i].flag();
}

}  // extern "C"
